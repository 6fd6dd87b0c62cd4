"""Ahead-of-time filling of the NVRTC kernel cache (a build step).

Kernels are generated per graph and compiled at run time; the cubins are cached on
disk (``_native.CACHE_DIR``), keyed by the full source. This module enumerates the
sources a workload will need — every pass of its plans under every autotuner
candidate schedule — and compiles them in a process pool, so that the first run
on a fresh machine does not spend minutes in the compiler. Planning needs only
shapes and dtypes: fields are stride-0 placeholders, no memory is allocated.
"""
from __future__ import annotations

import multiprocessing as mp
import os
from typing import Iterable, List, Optional, Sequence

import torch

EXPR_FIELDS = "divergence(gradient(f)) + l2norm(curl(u))"
# storage form -> (field dtype, result dtype)
FORMS = {"fp32": (torch.float32, torch.float32), "fp16": (torch.float16, torch.float16),
         "bf16": (torch.bfloat16, torch.bfloat16), "bf16in": (torch.bfloat16, torch.float32)}


def _placeholder(shape: Sequence[int], dtype: torch.dtype) -> torch.Tensor:
    return torch.zeros(1, dtype=dtype).expand(*shape)


def plan_sources(graph, wanted, out_dtype=torch.float32, cfg=None, candidates: bool = False) -> List[str]:
    """Sources of every pass of the graph's plan (and of each autotuner candidate)."""
    from . import autotune as AT
    from . import fused_compiler as FC
    plan = FC.Planner(graph, wanted, out_dtype, cfg).plan()
    out = []
    for pp in plan.passes:
        out.append(FC.emit_pass(pp.spec))
        if candidates:
            out += [FC.emit_pass(AT.with_config(pp.spec, c)) for c in AT.candidates(pp.spec)]
    if plan.scalar_source:
        out.append(plan.scalar_source)
    return out


def sources_fields(size: int = 512, forms: Iterable[str] = tuple(FORMS)) -> List[str]:
    """The 512^3 fused step (default schedule and every tuning candidate), per form."""
    from . import compile_expression
    out = []
    for form in forms:
        dt, odt = FORMS[form]
        g, sink, *_ = compile_expression(EXPR_FIELDS, dx=1.0, boundary="periodic",
                                         field_map={"f": _placeholder((size,) * 3, dt),
                                                    "u": _placeholder((size,) * 3 + (3,), dt)})
        wanted = [sink] + [g.add(r, (sink,), {}) for r in ("sum", "mean", "variance")]
        out += plan_sources(g, wanted, odt, candidates=True)
    return out


def sources_batch(n: int = 256, seed: int = 0, lo: int = 32, hi: int = 320) -> List[str]:
    """The batched workload's module under every batch candidate schedule."""
    from . import batch as B
    from . import compile_expression
    from .codegen import emit_batch_module
    from .synth import batch_specs
    jobs = []
    for expr, dt, shape, _ in batch_specs(n, seed=seed, lo=lo, hi=hi):
        full = tuple(shape) + ((3,) if expr.startswith("curl") else ())
        g, sink, *_ = compile_expression(expr, boundary="periodic", field_map={"f": _placeholder(full, dt)})
        jobs.append(B.BatchJob(g, [sink]))
    out = []
    for cfg in B.batch_candidates():
        specs, seen = [], set()
        for j in jobs:
            for pp in B.plan_job(j, cfg).passes:
                k = B.program_key(pp.spec)
                if k not in seen:
                    seen.add(k)
                    specs.append(pp.spec)
        out.append(emit_batch_module(specs, cfg.threads, B.batch_min_blocks(cfg.threads)))
    return out


def _compile(src: str) -> int:
    from . import _native as N
    from . import fused_compiler as FC
    N.compile_cached(src, FC.NVRTC_OPTS)
    return 1


def compile_all(sources: Iterable[str], workers: Optional[int] = None) -> int:
    """Compile into the cache with a spawn-started pool (safe next to CUDA state)."""
    todo = list(dict.fromkeys(sources))
    if not todo:
        return 0
    workers = workers or max(1, min(32, (os.cpu_count() or 2) - 1))
    with mp.get_context("spawn").Pool(workers) as pool:
        return sum(pool.map(_compile, todo, chunksize=2))
