"""Write tests/golden/autotune_timings.jsonl.gz from the autotuner's timing log.

The records are measurements made on a B200 by ``python bench.py --workload
costmodel`` (random expression DAGs; training DAGs timed on a random subset of
the schedule candidates, held-out DAGs on every candidate), which appends them to
the autotuner's JSON-lines log. This keeps the fields the cost model reads.

    python tests/golden/make_autotune_fixture.py <timings.jsonl> [max_train_records]
"""
import gzip
import json
import os
import random
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main() -> None:
    src = sys.argv[1]
    cap = int(sys.argv[2]) if len(sys.argv) > 2 else 6000
    recs = []
    with open(src) as fh:
        for line in fh:
            r = json.loads(line)
            if str(r.get("tag", "")).startswith("cm-"):
                recs.append({"key": r["key"], "tag": r["tag"], "features": r["features"], "schedule": r["schedule"],
                             "cfg": r["cfg"], "ms": round(float(r["ms"]), 6)})
    train = [r for r in recs if r["tag"].startswith("cm-train")]
    hold = [r for r in recs if r["tag"].startswith("cm-hold")]
    if len(train) > cap:   # whole passes only, so per-pass centring stays meaningful
        passes = sorted({r["tag"] + ":" + r["key"] for r in train})
        random.Random(0).shuffle(passes)
        keep, n = set(), 0
        per = {}
        for r in train:
            per.setdefault(r["tag"] + ":" + r["key"], []).append(r)
        for p in passes:
            if n + len(per[p]) > cap:
                break
            keep.add(p)
            n += len(per[p])
        train = [r for r in train if r["tag"] + ":" + r["key"] in keep]
    out = os.path.join(HERE, "autotune_timings.jsonl.gz")
    with gzip.open(out, "wt") as fh:
        for r in train + hold:
            fh.write(json.dumps(r, separators=(",", ":")) + "\n")
    print(f"{len(train)} training + {len(hold)} held-out records -> {out}")


if __name__ == "__main__":
    main()
