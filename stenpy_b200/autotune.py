"""Schedule autotuner for fused passes.

A pass's *schedule* is its ``PassConfig``: tile rows TJ × columns TK of the
(dim1, dim2) plane, threads per CTA (each thread owns one column and TJ·TK/threads
consecutive rows), z-march segment length and TMA prefetch depth. Results never
depend on it (every schedule evaluates the same arithmetic per voxel), only time
does. The reference's only schedule model is an analytic arithmetic-intensity /
register estimate (fused_compiler.py:20-43); here schedules are measured.

``candidates(spec)`` lists up to 24 valid schedules; ``tune_pass`` times each with
CUDA events (median of repeated launches on the pass's real inputs) and keeps the
fastest; every measurement is appended to a JSON-lines log together with the
pass's features (``features``), which is the training set of the learned ranking
model (``costmodel.py``). Exhaustive tuning is the fallback and the yardstick of
the model's regret.
"""
from __future__ import annotations

import dataclasses
import hashlib
import json
import os
import threading
import time
from typing import Any, Dict, List, Optional, Sequence, Tuple

import torch

from . import _native as N
from . import fused_compiler as FC
from .codegen import (ESIZE, SHELL_THREADS, PassConfig, PassSpec, emit_pass, is_flat, pass_grid, plane_bytes,
                      shell_count, shell_ctas, shell_regions, smem_layout, valid_shape, with_config)

LOG_PATH = os.environ.get("STENPY_TUNE_LOG", os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                          "_tune", "timings.jsonl"))
_BEST_PATH = os.path.join(os.path.dirname(LOG_PATH), "best.json")
_lock = threading.Lock()
SMEM_LIMIT = 227 * 1024

# (TK, threads, rows per thread) x segment lengths x boundary strategy = 6 x 2 x 2 = 24
_SHAPES = [(32, 128, 4), (32, 128, 8), (64, 128, 2), (64, 128, 4), (64, 256, 4), (64, 256, 8)]
_SEGS = (32, 128)
_SHAPES_KV4 = [(64, 128, 4), (64, 128, 2), (64, 256, 2)]   # (TK, threads, rows per thread) with KV = 4
# KV = 8 (16-byte chunks) is a valid schedule but not a candidate: on B200 at 512^3 the
# 16-bit passes of the config-1 step ran 3-14 % slower with it than with KV = 4
_GHOST = (True, False)


def _valid(spec: PassSpec, cfg: PassConfig) -> bool:
    if not valid_shape(cfg):
        return False
    trial = with_config(spec, cfg)
    for f in spec.fields:
        w, h = trial.box(f)
        if f.tma and (w > 256 or h > 256 or (w * ESIZE[f.dtype]) % 16):
            return False
    total, _, _ = smem_layout(trial)
    return total <= SMEM_LIMIT and 2 * spec.radius + 1 + cfg.prefetch <= FC.MAX_RING_SLOTS


def default_kv(spec: PassSpec) -> int:
    """Two k-adjacent voxels per thread for interleaved 3-component 16-bit fields: a
    thread's 12-byte chunk makes consecutive threads' shared-memory reads
    conflict-free (6-byte voxels put every other thread on a shared bank)."""
    return 2 if any(f.nc == 3 and ESIZE[f.dtype] == 2 for f in spec.fields) else 1


def candidates(spec: PassSpec) -> List[PassConfig]:
    out = []
    uses_ghost = with_config(spec, dataclasses.replace(spec.cfg, ghost=True)).ghosts is not None
    kv = default_kv(spec)
    for tk, nt, vpt in _SHAPES:
        for seg in _SEGS:
            for gh in (_GHOST if uses_ghost else (True,)):
                cfg = PassConfig(tj=(nt // tk) * vpt, tk=tk, threads=nt, prefetch=2, seg_len=seg, ghost=gh, kv=kv)
                if not valid_shape(cfg):
                    cfg.kv = 1
                if spec.has_scan:
                    cfg.seg_len = spec.cfg.seg_len
                if _valid(spec, cfg):
                    out.append(cfg)
    # 16-bit passes also try four k-adjacent voxels per thread (8-byte chunks, paired
    # 16-bit stores), keeping the rows per thread: measured faster for 16-bit stencils
    if not is_flat(spec) and not spec.has_scan and spec.fields and all(ESIZE[f.dtype] == 2 for f in spec.fields):
        for kv, shapes in ((4, _SHAPES_KV4),):
            for tk, nt, vpt in shapes:
                for seg in _SEGS:
                    for gh in (_GHOST if uses_ghost else (True,)):
                        cfg = PassConfig(tj=(nt * kv // tk) * vpt, tk=tk, threads=nt, prefetch=2, seg_len=seg,
                                         ghost=gh, kv=kv)
                        if valid_shape(cfg) and _valid(spec, cfg):
                            out.append(cfg)
                        if kv == 4 and vpt == 4 and nt == 128:
                            # the same tile capped at 80 registers (6 CTAs per SM): measured
                            # 3 % faster for the 16-bit Laplacian-with-statistics pass
                            capped = dataclasses.replace(cfg, min_blocks=6)
                            if valid_shape(capped) and _valid(spec, capped):
                                out.append(capped)
    # row-staged fields land in their ring slot one iteration after the request: one
    # plane of prefetch suffices, and the slot it saves can buy a resident CTA
    if any(f.staged and not f.tma for f in spec.fields):
        out += [c for c in (dataclasses.replace(c, prefetch=1) for c in out) if _valid(spec, c)]
    # keep distinct schedules only (scan passes collapse the segment axis)
    seen, uniq = set(), []
    for c in out:
        # a flat pass only uses the block size
        k = (c.threads,) if is_flat(spec) else (c.tj, c.tk, c.threads, c.seg_len, c.prefetch, c.ghost, c.kv,
                                                 c.min_blocks)
        if k not in seen:
            seen.add(k)
            uniq.append(c)
    return uniq


def features(spec: PassSpec, shape: Sequence[int]) -> Dict[str, float]:
    """Schedule-independent description of a pass (graph op mix, reach, dtypes, grid).
    A weighted-tap stencil counts as (taps / 7) Laplacians, by the neighbours it reads."""
    ops: Dict[str, float] = {}
    for n in spec.graph.nodes:
        ops[n.op] = ops.get(n.op, 0) + 1
        if n.op == "taps":
            ops["lap"] = ops.get("lap", 0) + len(n.a("taps")) / 7.0
    trans = sum(ops.get(k, 0) for k in ("exp", "log", "sqrt", "sin", "cos", "tanh", "normalize", "norm", "eig",
                                        "surfnorm"))
    arith = sum(ops.get(k, 0) for k in ("add", "sub", "mul", "div", "neg", "abs", "clamp", "mulk", "trace",
                                        "select", "stack"))
    in_bytes = sum(ESIZE[f.dtype] * f.nc for f in spec.fields)
    out_bytes = sum(ESIZE[r.out_dtype] * spec.graph.nodes[r.node].nc for r in spec.roots if r.kind in ("out", "scan"))
    n0, n1, n2 = shape
    return {
        "radius": spec.radius, "n_fields": len(spec.fields), "in_bytes": in_bytes, "out_bytes": out_bytes,
        "n_d1": ops.get("d1", 0), "n_lap": ops.get("lap", 0), "n_trans": trans, "n_arith": arith,
        "n_eig": ops.get("eig", 0), "n_out": sum(1 for r in spec.roots if r.kind == "out"),
        "n_red": sum(1 for r in spec.roots if r.kind == "red"), "n_slots": spec.nslots,
        "narrow": float(any(f.dtype in ("bf16", "f16") for f in spec.fields)),
        "max_nc": max([f.nc for f in spec.fields] + [1]), "n0": n0, "n1": n1, "n2": n2,
        "voxels": float(n0) * n1 * n2,
    }


def schedule_features(spec: PassSpec, cfg: PassConfig) -> Dict[str, float]:
    trial = with_config(spec, cfg)
    smem, _, _ = smem_layout(trial)
    return {"tj": cfg.tj, "tk": cfg.tk, "threads": cfg.threads, "vpt": cfg.tj * cfg.tk // (cfg.threads * cfg.kv),
            "seg_len": cfg.seg_len, "prefetch": cfg.prefetch, "smem": smem, "ghost": float(cfg.ghost),
            "shell": float(shell_regions(trial) != ""), "kv": cfg.kv}


def pass_key(spec: PassSpec, shape: Sequence[int]) -> str:
    src = emit_pass(with_config(spec, PassConfig()))
    return hashlib.sha256((src + repr(tuple(shape))).encode()).hexdigest()[:24]


def _launches(pp: FC.PassPlan, spec: PassSpec, values: Dict[str, Any], shape, device, part, table, err):
    """Main + shell launches of a pass for a given schedule (mirrors build_program)."""
    n0, n1, n2 = shape
    cfg = spec.cfg
    tiles_k = -(-n2 // cfg.tk)
    gx, gy = pass_grid(spec, n1, n2, n0)
    grid = (gx, gy, 1)
    ncta = grid[0] * grid[1]
    fptrs = [values[nid].data_ptr() for nid in pp.field_nodes]
    tmaps = FC.encode_tmaps(spec, fptrs, n0, n1, n2)
    outs = []
    for (nid, kind, nc), r in zip(pp.out_nodes, [r for r in spec.roots if r.kind in ("out", "scan")]):
        outs.append(torch.empty((n0, n1, n2) + FC.comp_shape(nc), dtype=FC.DT_TORCH[r.out_dtype], device=device))
    nbins = max([r.slot + r.bins for r in spec.roots if r.kind == "red" and r.red == "hist"] + [0])
    hist = torch.zeros(max(nbins, 1), dtype=torch.int64, device=device)
    outs.append(hist)   # keeps the histogram buffer alive with the launches
    vals = dict(fld=fptrs, out=[o.data_ptr() for o in outs[:-1]], scal=table.data_ptr(), part=part.data_ptr(),
                hist=hist.data_ptr(),
                err=err.data_ptr(), n0g=n0, n1=n1, n2=n2, nl=n0, i_base=0, out_lo=0, n_out=n0,
                seg_len=cfg.seg_len, tiles_k=tiles_k, cta_off=0)
    ls = [(grid, (cfg.threads, 1, 1), FC.pack_params(spec, vals, tmaps))]
    if FC.has_shell(spec):
        sh = shell_ctas(shell_count(shape, spec.radius, regions=shell_regions(spec)))
        ls.append(((sh, 1, 1), (SHELL_THREADS, 1, 1), FC.pack_params(spec, dict(vals, cta_off=ncta), tmaps)))
    return ls, outs, ncta


def time_schedule(pp: FC.PassPlan, cfg: PassConfig, values: Dict[str, Any], shape, device,
                  reps: int = 5, unload: bool = False) -> float:
    """Median milliseconds of one pass (main + shell kernel) under ``cfg``."""
    dev_idx = device.index if device.index is not None else torch.cuda.current_device()
    spec = with_config(pp.spec, cfg)
    src = emit_pass(spec)
    smem, _, _ = smem_layout(spec)
    key, cubin = N.compile_cached(src, FC.NVRTC_OPTS)
    mod = N.load_module(key, cubin, "sten_kernel", smem, dev_idx)
    shell_mod = N.load_module(key + ":shell", cubin, "sten_shell", 0, dev_idx) if FC.has_shell(spec) else None
    n_shell = shell_ctas(shell_count(shape, spec.radius, regions=shell_regions(spec)))
    gx, gy = pass_grid(spec, shape[1], shape[2], shape[0])
    tiles = gx * gy
    part = torch.empty(max((tiles + n_shell) * spec.nslots, 1), dtype=torch.float64, device=device)
    table = torch.zeros(max(spec.n_scalars, 1) + 8, dtype=torch.float64, device=device)
    err = FC.ErrorFlag.get(device)
    ls, outs, _ = _launches(pp, spec, values, shape, device, part, table, err)
    mods = [mod, shell_mod]
    stream = torch.cuda.current_stream(device)
    s = stream.cuda_stream

    def run():
        for (grid, block, params), m in zip(ls, mods):
            N.launch(m, grid, block, smem if m == mod else 0, s, params)

    for _ in range(2):
        run()
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        run()
        b.record(stream)
        b.synchronize()
        ts.append(a.elapsed_time(b))
    FC.ErrorFlag.check(device)
    if unload:   # a one-off timing (cost-model data): do not keep thousands of modules loaded
        N.unload_module(key, dev_idx)
        if shell_mod is not None:
            N.unload_module(key + ":shell", dev_idx)
    ts.sort()
    return ts[len(ts) // 2]


def log_record(rec: Dict[str, Any]) -> None:
    with _lock:
        os.makedirs(os.path.dirname(LOG_PATH), exist_ok=True)
        with open(LOG_PATH, "a") as fh:
            fh.write(json.dumps(rec) + "\n")


def _load_best() -> Dict[str, Any]:
    try:
        with open(_BEST_PATH) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _save_best(best: Dict[str, Any]) -> None:
    with _lock:
        os.makedirs(os.path.dirname(_BEST_PATH), exist_ok=True)
        tmp = _BEST_PATH + f".{os.getpid()}.tmp"
        with open(tmp, "w") as fh:
            json.dump(best, fh)
        os.replace(tmp, _BEST_PATH)


def tune_pass(pp: FC.PassPlan, values: Dict[str, Any], shape, device, cands: Optional[List[PassConfig]] = None,
              tag: str = "", reuse: bool = True, unload: bool = False
              ) -> Tuple[PassConfig, List[Tuple[PassConfig, float]]]:
    """Exhaustively time ``cands`` (default: all candidates) and return the fastest."""
    key = pass_key(pp.spec, shape)
    best_db = _load_best() if reuse else {}
    if reuse and key in best_db and cands is None:
        return PassConfig(**best_db[key]["cfg"]), []
    exhaustive = cands is None
    cands = candidates(pp.spec) if exhaustive else cands
    feats = features(pp.spec, shape)
    results = []
    for cfg in cands:
        ms = time_schedule(pp, cfg, values, shape, device, unload=unload)
        results.append((cfg, ms))
        log_record({"key": key, "tag": tag, "features": feats, "schedule": schedule_features(pp.spec, cfg),
                    "cfg": vars(cfg), "ms": ms, "time": time.time()})
    best = min(results, key=lambda x: x[1])
    if exhaustive:
        db = _load_best()
        db[key] = {"cfg": vars(best[0]), "ms": best[1]}
        _save_best(db)
    return best[0], results


def tune_plan(plan: FC.FusedPlan, values: Dict[str, Any], device, tag: str = "", reuse: bool = True,
              chooser=None) -> List[Tuple[PassConfig, float]]:
    """Tune every pass of ``plan`` in place (the plan's passes are recompiled with
    their best schedule). ``chooser(pp, cands) -> cands`` may prune candidates (the
    learned ranking model); exhaustive search otherwise."""
    out = []
    for pp in plan.passes:
        cands = None
        if chooser is not None:
            cands = chooser(pp, candidates(pp.spec), plan.shape)
        cfg, res = tune_pass(pp, values, plan.shape, device, cands, tag=tag, reuse=reuse)
        if vars(cfg) != vars(pp.spec.cfg):
            pp.spec = with_config(pp.spec, cfg)
            pp.module = None
            pp.shell_module = None
        out.append((cfg, min([m for _, m in res]) if res else float("nan")))
    return out
