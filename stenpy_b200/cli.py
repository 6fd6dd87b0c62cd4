"""``stenpy`` command line: ``python -m stenpy_b200 --field f=data.npy --expr "curl(f)" --device cuda``.

The reference advertises ``stenpy --field f=data.h5 --expr "curl(f)" --device cuda``
(README.md:21) but ships no entry point; this one maps the flags onto ``Pipeline``
semantics (periodic boundary by default, unit spacing). Fields are ``.npy`` /
``.npz`` / ``.pt`` files (HDF5 needs h5py, absent here). ``--output`` writes the
result; without it a one-line summary (shape, min, max, mean) is printed.
``--lazy`` streams the fields from pinned host memory in chunks under
``--budget-gb`` of device memory.
"""
from __future__ import annotations

import argparse
import json
import sys
from typing import List, Optional

import torch

_DT = {"fp32": torch.float32, "bf16": torch.bfloat16, "fp16": torch.float16, "fp64": torch.float64}


def main(argv: Optional[List[str]] = None) -> int:
    ap = argparse.ArgumentParser(prog="stenpy", description="Evaluate a stencil expression on volumetric fields")
    ap.add_argument("--field", action="append", default=[], metavar="NAME=PATH",
                    help="field binding, repeatable (e.g. f=data.npy)")
    ap.add_argument("--const", action="append", default=[], metavar="NAME=VALUE", help="scalar constant")
    ap.add_argument("--expr", required=True, help='expression, e.g. "laplacian(f) + tanh(f)"')
    ap.add_argument("--device", default="cuda")
    ap.add_argument("--boundary", default="periodic")
    ap.add_argument("--dx", type=float, default=1.0)
    ap.add_argument("--dtype", choices=sorted(_DT), default=None, help="storage dtype of fields and result")
    ap.add_argument("--output", default=None, help="write the result (.npy/.npz/.pt)")
    ap.add_argument("--lazy", action="store_true", help="stream fields from host memory in chunks")
    ap.add_argument("--budget-gb", type=float, default=8.0)
    ap.add_argument("--perf-report", action="store_true")
    a = ap.parse_args(argv)
    if torch.device(a.device).type != "cuda":
        print("stenpy: this executor runs on CUDA devices only (use --device cuda)", file=sys.stderr)
        return 2
    from .pipeline import Pipeline
    p = Pipeline("cli", a.expr)
    p.set(device=a.device, boundary=a.boundary, dx=a.dx, perf_report=a.perf_report)
    if a.dtype:
        p.dtype = _DT[a.dtype]
    if a.lazy:
        p.set(stream_i=True, chunk_mb=a.budget_gb * 1024 / 6)
    for item in a.field:
        name, _, path = item.partition("=")
        if not path:
            ap.error(f"--field expects NAME=PATH, got {item!r}")
        setattr(p, name, path)
    for item in a.const:
        name, _, val = item.partition("=")
        setattr(p, name, float(val))
    if a.output:
        p.output = a.output
        out = p.value
    else:
        out = p.run()
    t = out.double() if isinstance(out, torch.Tensor) else torch.tensor(float(out))
    print(json.dumps({"shape": list(t.shape), "min": float(t.min()), "max": float(t.max()),
                      "mean": float(t.mean()), "output": a.output}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
