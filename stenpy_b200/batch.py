"""Batched persistent executor: many independent graphs in ONE kernel launch.

Each job is a graph over its own fields — grids of uneven shapes, FP32 or BF16
storage — with its own wanted nodes. Every job is planned exactly as
``Runtime.run`` plans it (``fused_compiler.Planner``: passes split at reduction
barriers), and every distinct pass program (the generated z-march code, which
depends on the graph, dtypes and schedule but not on the grid size) is emitted
once into a single module next to ``sten_batch``, a persistent kernel whose CTAs
take work items from a queue: one z-march tile (TJ x TK columns x seg_len planes)
or one block of boundary-shell voxels of one pass of one job. A pass whose
kernels read scalars produced by an earlier pass of the same job (min/max before
a histogram, a mean before a centred value) waits for that pass's ready flag,
which the CTA finishing its last item sets after combining its partials. The
launch leaves the queue reset, so it can be replayed from a CUDA graph.

The reference has no batched path: it runs one graph at a time through
``Runtime.run`` (stenpy_engine.py:509-1146) and its Triton kernels are launched
per operator with fixed grids (stenpy_engine.py:1961-1981). Per-voxel results are
bit-identical to ``Runtime(out_dtype=...).run`` of the same graph (same generated
arithmetic at every voxel); reductions agree to FP64 rounding (same partial
rows, combined by a tree of the batch kernel's block size).

Schedules: ``tune_batch`` times each group of structurally equal jobs under every
candidate tile shape and z-segment length inside the persistent kernel itself and
keeps the fastest per group (all groups share the block size).
"""
from __future__ import annotations

import dataclasses
import hashlib
import statistics
import struct
from dataclasses import dataclass, field as dc_field
from typing import Any, Dict, List, Optional, Sequence, Tuple

import torch

from . import _native as N
from . import fused_compiler as FC
from .codegen import (PassConfig, PassSpec, emit_batch_module, emit_pass, pass_grid, shell_count, shell_regions,
                      smem_layout)
from .graph import Graph
from .runtime import default_wanted

PHASE_FMT = "<4Q12i"    # struct BPhase
RED_FMT = "<4i2d"       # struct BRed
HIST_FMT = "<4id"       # struct BHist
ARGS_FMT = "<6Q2i"      # struct BatchArgs
assert struct.calcsize(PHASE_FMT) == 80 and struct.calcsize(RED_FMT) == 32 and struct.calcsize(HIST_FMT) == 24

BATCH_SHAPES = {128: [(32, 4), (32, 8), (64, 2), (64, 4)], 256: [(64, 4), (64, 8)]}  # (TK, rows per thread)
BATCH_SEGS = (32, 128)


def batch_candidates(threads: Optional[int] = None) -> List[PassConfig]:
    """Tile shape x z-segment candidates (ghost-cell boundaries), grouped by block size."""
    out = []
    for nt, shapes in BATCH_SHAPES.items():
        if threads is not None and nt != threads:
            continue
        for tk, vpt in shapes:
            for seg in BATCH_SEGS:
                out.append(PassConfig(tj=(nt // tk) * vpt, tk=tk, threads=nt, prefetch=2, seg_len=seg, ghost=True))
    return out


def batch_min_blocks(threads: int) -> int:
    return max(1, 512 // threads)


def program_key(spec: PassSpec) -> str:
    return hashlib.sha1(emit_pass(spec).encode()).hexdigest()[:20]


def _storage_dtype(graph: Graph, wanted: Sequence[str]) -> torch.dtype:
    for nid in graph.live_nodes(list(wanted)):
        node = graph._nodes[nid]
        v = node.params.get("value") if node.op_name == "_constant" else None
        if FC.is_field_value(v):
            return v.dtype
    return torch.float32


@dataclass
class BatchJob:
    """One graph of a batch and the node ids wanted from it. Per-voxel outputs are
    stored as ``out_dtype`` (default: the storage dtype of the job's fields)."""
    graph: Graph
    wanted: List[str] = dc_field(default_factory=list)
    out_dtype: Optional[torch.dtype] = None
    outputs: Dict[str, torch.Tensor] = dc_field(default_factory=dict)  # reused across builds

    def __post_init__(self):
        if not self.wanted:
            self.wanted = default_wanted(self.graph)
        if self.out_dtype is None:
            self.out_dtype = _storage_dtype(self.graph, self.wanted)


def plan_job(job: BatchJob, cfg: PassConfig) -> FC.FusedPlan:
    from .autotune import default_kv
    from .codegen import valid_shape
    plan = FC.Planner(job.graph, job.wanted, job.out_dtype, cfg).plan()
    kv = max([default_kv(pp.spec) for pp in plan.passes] + [1])
    if kv != cfg.kv:
        cfg2 = dataclasses.replace(cfg, kv=kv)
        if valid_shape(cfg2):
            plan = FC.Planner(job.graph, job.wanted, job.out_dtype, cfg2).plan()
    if plan.scalar_source:
        raise FC.FusionError("batch: sinks that are expressions of reduction results are not batched")
    if any(pp.spec.has_scan for pp in plan.passes):
        raise FC.FusionError("batch: cumulative_integral is not batched")
    if not plan.passes:
        raise FC.FusionError("batch: a job has no per-voxel work")
    return plan


def group_key(job: BatchJob, threads: int = 128) -> str:
    """Jobs with equal keys run the same programs (same graph structure, dtypes and
    TMA-eligibility of their rows) and share a schedule."""
    cfg = batch_candidates(threads)[0]
    return "|".join(program_key(pp.spec) for pp in plan_job(job, cfg).passes)


class BatchModule:
    """The compiled batch kernel for a set of pass programs (one block size)."""

    def __init__(self, specs: Sequence[PassSpec], threads: int, device: torch.device,
                 min_blocks: Optional[int] = None):
        # at most 128 registers a thread: the kernel's register count is the maximum
        # over all of its programs, so the heaviest would otherwise set the occupancy
        min_blocks = min_blocks or batch_min_blocks(threads)
        self.threads = threads
        self.keys: List[str] = []
        self.index: Dict[str, int] = {}
        uniq: List[PassSpec] = []
        for sp in specs:
            k = program_key(sp)
            if k not in self.index:
                self.index[k] = len(uniq)
                self.keys.append(k)
                uniq.append(sp)
        self.specs = uniq
        self.source = emit_batch_module(uniq, threads, min_blocks)
        self.smem = max([smem_layout(sp)[0] for sp in uniq] + [1024])
        dev_idx = device.index if device.index is not None else torch.cuda.current_device()
        key, cubin = N.compile_cached(self.source, FC.NVRTC_OPTS)
        self.key = key
        self.module = N.load_module(key, cubin, "sten_batch", self.smem, dev_idx)
        self.blocks_per_sm, self.regs, self.local_bytes = N.module_info(self.module, threads, self.smem)
        if self.blocks_per_sm < 1:
            raise FC.FusionError(f"batch kernel cannot be resident ({self.smem} B shared, {self.regs} registers)")
        self.sm_count = N.device_props(dev_idx)[0]


@dataclass
class _Phase:
    job: int
    pass_index: int
    prog: int
    gdx: int
    nseg: int
    shell_items: int
    ncta: int
    nslots: int
    dep: int
    work: float


def build_queue(phases: Sequence[_Phase]) -> List[int]:
    """Work items (phase, kind, bx, by), flattened, in queue order: passes that other
    passes wait for first, then the other independent passes, then dependent passes
    by depth; larger jobs first within each class (short tail). Within a pass: tiles
    segment-major (CTAs taking consecutive items share halos in L2), then shell
    blocks. Every pass's prerequisites precede it, so a CTA that waits only waits on
    items already taken by running CTAs."""
    depth: List[int] = []
    for i, ph in enumerate(phases):
        if ph.dep >= i:
            raise ValueError("a pass may only depend on an earlier pass")
        depth.append(0 if ph.dep < 0 else depth[ph.dep] + 1)
    has_dependent = {ph.dep for ph in phases if ph.dep >= 0}
    order = sorted(range(len(phases)),
                   key=lambda i: (depth[i], 0 if i in has_dependent else 1, -phases[i].work, i))
    items: List[int] = []
    for i in order:
        ph = phases[i]
        for by in range(ph.nseg):
            for bx in range(ph.gdx):
                items += (i, 0, bx, by)
        for bx in range(ph.shell_items):
            items += (i, 1, bx, 0)
    return items


def check_queue(items: torch.Tensor, phases: Sequence[_Phase]) -> None:
    """Every item names an existing pass and a tile / shell block inside it, each
    exactly once (the kernel trusts these indices)."""
    if items.ndim != 2 or items.shape[1] != 4:
        raise ValueError("work items must be (n, 4)")
    ph = items[:, 0].long()
    if len(phases) == 0 or int(ph.min()) < 0 or int(ph.max()) >= len(phases):
        raise ValueError("work item names a missing pass")
    gdx = torch.tensor([p.gdx for p in phases])[ph]
    nseg = torch.tensor([p.nseg for p in phases])[ph]
    nsh = torch.tensor([p.shell_items for p in phases])[ph]
    kind, bx, by = items[:, 1].long(), items[:, 2].long(), items[:, 3].long()
    tile_ok = (kind == 0) & (bx >= 0) & (bx < gdx) & (by >= 0) & (by < nseg)
    shell_ok = (kind == 1) & (bx >= 0) & (bx < nsh) & (by == 0)
    if not bool((tile_ok | shell_ok).all()):
        raise ValueError("work item outside its pass")
    if items.shape[0] != sum(p.ncta for p in phases) or \
            torch.unique(items, dim=0).shape[0] != items.shape[0]:
        raise ValueError("work items must cover every tile and shell block exactly once")


class BatchProgram:
    """A batch resolved against its tensors: per-job plans, the work queue, scalar
    tables, partial rows, histograms and outputs, and the packed kernel arguments.
    ``enqueue`` issues the single launch; ``collect`` returns per-job results."""

    def __init__(self, jobs: Sequence[BatchJob], plans: Sequence[FC.FusedPlan], module: BatchModule,
                 device: torch.device):
        self.jobs, self.plans, self.mod, self.device = list(jobs), list(plans), module, device
        nt = module.threads
        err = FC.ErrorFlag.get(device)
        phases: List[_Phase] = []
        table_off, hist_off = [], []
        t_total = h_total = 0
        for ji, plan in enumerate(self.plans):
            table_off.append(t_total)
            hist_off.append(h_total)
            t_total += plan.table_size
            h_total += plan.hist_size
            n0, n1, n2 = plan.shape
            for pi, pp in enumerate(plan.passes):
                spec = pp.spec
                if spec.cfg.threads != nt:
                    raise FC.FusionError("batch: every pass must use the module's block size")
                prog = module.index.get(program_key(spec))
                if prog is None:
                    raise FC.FusionError("batch: pass program missing from the module")
                gdx, nseg = pass_grid(spec, n1, n2, n0)
                n_shell = shell_count(plan.shape, spec.radius, regions=shell_regions(spec))
                shell_items = -(-n_shell // nt)
                phases.append(_Phase(ji, pi, prog, gdx, nseg, shell_items, gdx * nseg + shell_items,
                                     spec.nslots, len(phases) - 1 if pi > 0 else -1, float(n0 * n1 * n2)))
        self.phases = phases
        dev = device
        self.table = torch.zeros(max(t_total, 1), dtype=torch.float64, device=dev)
        self.hist = torch.zeros(max(h_total, 1), dtype=torch.int64, device=dev)
        part_off, p_total = [], 0
        for ph in phases:
            part_off.append(p_total)
            p_total += ph.ncta * ph.nslots
        self.part = torch.zeros(max(p_total, 1), dtype=torch.float64, device=dev)
        # constants of every job's scalar table, written once
        consts = torch.zeros(max(t_total, 1), dtype=torch.float64)
        self.results: List[Dict[str, Any]] = []
        params_blobs: List[bytes] = []
        phase_recs, red_recs, hist_recs = [], [], []
        pidx = 0
        for ji, (job, plan) in enumerate(zip(self.jobs, self.plans)):
            values = {nid: job.graph._nodes[nid].params["value"] for nid in plan.live
                      if job.graph._nodes[nid].op_name == "_constant"}
            for nid, idx in plan.const_index.items():
                v = values[nid]
                consts[table_off[ji] + idx] = float(v.item() if isinstance(v, torch.Tensor) else v)
            n0, n1, n2 = plan.shape
            res: Dict[str, Any] = {}
            for pi, pp in enumerate(plan.passes):
                ph = phases[pidx]
                spec = pp.spec
                fptrs = []
                for f, nid in zip(spec.fields, pp.field_nodes):
                    t = values[nid]
                    if not isinstance(t, torch.Tensor) or t.device != dev or not t.is_contiguous():
                        raise FC.FusionError(f"batch job {ji}: field {nid} must be a contiguous tensor on {dev}")
                    if FC.DT_TORCH[f.dtype] != t.dtype:
                        raise FC.FusionError(f"batch job {ji}: field {nid} planned {f.dtype}, got {t.dtype}")
                    fptrs.append(t.data_ptr())
                outs = []
                for (nid, okind, nc), r in zip(pp.out_nodes, [r for r in spec.roots if r.kind == "out"]):
                    shape = plan.out_shape(nc, nid)
                    o = job.outputs.get(nid)
                    if o is None or tuple(o.shape) != shape or o.dtype != FC.DT_TORCH[r.out_dtype]:
                        o = torch.empty(shape, dtype=FC.DT_TORCH[r.out_dtype], device=dev)
                        job.outputs[nid] = o
                    outs.append(o)
                    if nid in plan.wanted:
                        res[nid] = o
                tmaps = FC.encode_tmaps(spec, fptrs, n0, n1, n2)
                tbl = self.table.data_ptr() + 8 * table_off[ji]
                hst = self.hist.data_ptr() + 8 * hist_off[ji]
                prt = self.part.data_ptr() + 8 * part_off[pidx]
                blob = FC.pack_params(spec, dict(fld=fptrs, out=[o.data_ptr() for o in outs], scal=tbl, part=prt,
                                                 hist=hst, err=err.data_ptr(), n0g=n0, n1=n1, n2=n2, nl=n0,
                                                 i_base=0, out_lo=0, n_out=n0, seg_len=spec.cfg.seg_len,
                                                 tiles_k=-(-n2 // spec.cfg.tk), cta_off=0), tmaps)
                params_blobs.append(blob)
                reds = [struct.pack(RED_FMT, r.kind, r.slot, r.table_index, r.unbiased, r.count, r.eps)
                        for r in pp.reductions]
                hists = [struct.pack(HIST_FMT, r.slot, r.bins, r.lohi_index, r.table_index,
                                     float(n0 * n1 * n2 * spec.graph.nodes[r.node].nc)) for r in pp.hists]
                phase_recs.append((ph, tbl, hst, prt, len(red_recs), len(reds), len(hist_recs), len(hists)))
                red_recs += reds
                hist_recs += hists
                pidx += 1
            for nid, idx in plan.red_index.items():
                if nid in plan.wanted:
                    res[nid] = (table_off[ji] + idx, 2 if plan.infos[nid].nc == 2 else 1)
            for nid in plan.wanted:
                if nid not in res:
                    res[nid] = values[nid]
            self.results.append(res)
        self.table.copy_(consts.to(dev))
        # Params blobs at 64-byte aligned offsets (TMA descriptors must be 64-byte aligned)
        offs, blob_total = [], 0
        for b in params_blobs:
            offs.append(blob_total)
            blob_total += (len(b) + 63) // 64 * 64
        pbuf = bytearray(max(blob_total, 64))
        for o, b in zip(offs, params_blobs):
            pbuf[o:o + len(b)] = b
        self.params = torch.frombuffer(pbuf, dtype=torch.uint8).to(dev)
        assert self.params.data_ptr() % 64 == 0
        prec = bytearray()
        for (ph, tbl, hst, prt, r0, nr, h0, nh), o in zip(phase_recs, offs):
            prec += struct.pack(PHASE_FMT, self.params.data_ptr() + o, prt, tbl, hst, ph.prog,
                                ph.gdx * ph.nseg + ph.shell_items, ph.dep, ph.gdx, ph.gdx * ph.nseg, ph.ncta,
                                ph.nslots, r0, nr, h0, nh, 0)
        self.phase_buf = torch.frombuffer(bytearray(prec), dtype=torch.uint8).to(dev)
        self.red_buf = torch.frombuffer(bytearray(b"".join(red_recs) or bytes(32)), dtype=torch.uint8).to(dev)
        self.hist_buf = torch.frombuffer(bytearray(b"".join(hist_recs) or bytes(24)), dtype=torch.uint8).to(dev)
        items = torch.tensor(build_queue(self.phases), dtype=torch.int32).reshape(-1, 4)
        check_queue(items, self.phases)
        self.n_items = int(items.shape[0])
        self.items = items.to(dev)
        self.ctl = torch.zeros(2 + 2 * len(phases), dtype=torch.int32, device=dev)
        self.n_ctas = max(1, min(self.n_items, module.sm_count * module.blocks_per_sm))
        self.args = struct.pack(ARGS_FMT, self.items.data_ptr(), self.phase_buf.data_ptr(), self.red_buf.data_ptr(),
                                self.hist_buf.data_ptr(), self.ctl.data_ptr(), err.data_ptr(),
                                self.n_items, len(phases))
        self.err = err

    # -- execution
    @property
    def launches(self) -> int:
        return 1

    def enqueue(self, stream: torch.cuda.Stream) -> int:
        N.launch(self.mod.module, (self.n_ctas, 1, 1), (self.mod.threads, 1, 1), self.mod.smem,
                 stream.cuda_stream, self.args)
        return 1

    def check(self) -> None:
        """Raise if a kernel reported an expired bounded wait (queue state is reset)."""
        v = int(self.err.item())
        if v:
            self.err.zero_()
            self.ctl.zero_()
            raise RuntimeError(f"stenpy_b200 batch: device status {v} (bounded wait expired)")

    def collect(self) -> List[Dict[str, Any]]:
        out = []
        for res in self.results:
            d: Dict[str, Any] = {}
            for nid, v in res.items():
                if isinstance(v, tuple):
                    idx, n = v
                    d[nid] = self.table[idx:idx + n].clone() if n == 2 else self.table[idx].clone()
                else:
                    d[nid] = v
            out.append(d)
        return out

    def algorithmic_bytes(self) -> int:
        """Unique bytes a step must move: every input field read once and every
        per-voxel output written once, at storage dtype."""
        total = 0
        for job, plan in zip(self.jobs, self.plans):
            seen = set()
            for pp in plan.passes:
                for nid in pp.field_nodes:
                    if nid not in seen:
                        seen.add(nid)
                        v = job.graph._nodes[nid].params["value"]
                        total += v.numel() * v.element_size()
                for nid, okind, nc in pp.out_nodes:
                    o = job.outputs[nid]
                    total += o.numel() * o.element_size()
        return total

    def voxels(self) -> int:
        return sum(p.shape[0] * p.shape[1] * p.shape[2] for p in self.plans)


def _as_jobs(jobs: Sequence[Any]) -> List[BatchJob]:
    out = []
    for j in jobs:
        if isinstance(j, BatchJob):
            out.append(j)
        elif isinstance(j, Graph):
            out.append(BatchJob(j))
        else:
            g, wanted = j
            out.append(BatchJob(g, list(wanted)))
    return out


def build(jobs: Sequence[Any], device: Any = "cuda", configs: Optional[Dict[str, PassConfig]] = None,
          threads: int = 128, min_blocks: Optional[int] = None) -> BatchProgram:
    """Plan, compile and resolve a batch. ``configs`` maps group keys (``group_key``)
    to schedules; groups without an entry use the first candidate of ``threads``."""
    device = torch.device(device)
    if device.type != "cuda":
        raise NotImplementedError("stenpy_b200 batches run on CUDA devices only")
    if device.index is None:
        device = torch.device("cuda", torch.cuda.current_device())
    jobs = _as_jobs(jobs)
    default = batch_candidates(threads)[0]
    plans = []
    for job in jobs:
        cfg = default
        if configs:
            cfg = configs.get(group_key(job, threads), default)
        if cfg.threads != threads:
            raise FC.FusionError("batch: all schedules must share the block size")
        plans.append(plan_job(job, cfg))
    module = BatchModule([pp.spec for p in plans for pp in p.passes], threads, device, min_blocks)
    return BatchProgram(jobs, plans, module, device)


def run_batch(jobs: Sequence[Any], device: Any = "cuda", configs: Optional[Dict[str, PassConfig]] = None,
              threads: int = 128) -> List[Dict[str, Any]]:
    """Evaluate every job in one persistent launch; per-job ``{node_id: value}``."""
    prog = build(jobs, device, configs, threads)
    stream = torch.cuda.current_stream(prog.device)
    with torch.no_grad():
        prog.enqueue(stream)
    stream.synchronize()
    prog.check()
    return prog.collect()


def time_program(prog: BatchProgram, reps: int = 5, warmup: int = 2) -> float:
    """Median device time (ms) of one launch, CUDA events on the launching stream."""
    stream = torch.cuda.current_stream(prog.device)
    for _ in range(warmup):
        prog.enqueue(stream)
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        prog.enqueue(stream)
        b.record(stream)
        b.synchronize()
        ts.append(a.elapsed_time(b))
    prog.check()
    return statistics.median(ts)


def tune_batch(jobs: Sequence[Any], device: Any = "cuda", cands: Optional[List[PassConfig]] = None,
               reps: int = 5, log: Optional[List[Dict[str, Any]]] = None) -> Tuple[int, Dict[str, PassConfig]]:
    """Exhaustive schedule search inside the persistent kernel: for every candidate
    (tile shape x z-segment), compile the batch module once and time each group of
    structurally equal jobs on its own; keep the fastest candidate per group, then
    the block size whose per-group optima sum lowest. Returns (threads, configs)."""
    device = torch.device(device)
    if device.index is None:
        device = torch.device("cuda", torch.cuda.current_device())
    jobs = _as_jobs(jobs)
    cands = cands or batch_candidates()
    groups: Dict[str, List[int]] = {}
    for i, job in enumerate(jobs):
        groups.setdefault(group_key(job), []).append(i)
    best: Dict[int, Dict[str, Tuple[float, PassConfig]]] = {}
    for cfg in cands:
        plans = [plan_job(job, cfg) for job in jobs]
        module = BatchModule([pp.spec for p in plans for pp in p.passes], cfg.threads, device)
        for gk, idx in groups.items():
            prog = BatchProgram([jobs[i] for i in idx], [plans[i] for i in idx], module, device)
            t = time_program(prog, reps)
            if log is not None:
                j0, p0 = jobs[idx[0]], plans[idx[0]]
                label = "+".join(j0.graph._nodes[w].op_name for w in j0.wanted)
                label += f" {FC.TORCH_DT[j0.out_dtype]} tma={any(f.tma for pp in p0.passes for f in pp.spec.fields)}"
                vox = sum(plans[i].shape[0] * plans[i].shape[1] * plans[i].shape[2] for i in idx)
                log.append({"group": gk[:12], "label": label, "jobs": len(idx), "voxels": vox,
                            "cfg": vars(cfg).copy(), "ms": t, "blocks_per_sm": module.blocks_per_sm,
                            "regs": module.regs})
            cur = best.setdefault(cfg.threads, {}).get(gk)
            if cur is None or t < cur[0]:
                best[cfg.threads][gk] = (t, cfg)
            del prog
    threads = min(best, key=lambda nt: sum(t for t, _ in best[nt].values()))
    return threads, {gk: c for gk, (t, c) in best[threads].items()}
