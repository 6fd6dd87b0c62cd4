"""Out-of-core (lazy) execution: fields in pinned host memory, streamed in dim-0 chunks.

Replaces the reference's ``Runtime.run_chunked`` / ``_read_halo_chunk`` /
``_lazy_to_gpu`` path (stenpy_engine.py:647-888, 144-199), where a reader thread
fills a prefetch queue, the main thread copies each halo'd chunk to the GPU, runs
the whole graph, crops, copies back synchronously and a writer thread stores it.
Here the same fused kernels run on chunk slabs:

* chunk [s, e) of dim 0 is computed from the slab [s - H, e + H) — wrapped for
  periodic boundaries, clipped otherwise — where H is the pass's stencil reach
  (+1 when one-sided torch.gradient edges are involved, whose formulas reach one
  plane further). The kernels keep global coordinates (``i_base``/``out_lo``), so
  every voxel takes exactly the same arithmetic as in a whole-field run and the
  per-voxel results are bit-identical to it (seam test);
* slabs and outputs are double-buffered on the device; H2D copies, kernels and
  D2H copies run on three streams ordered by events, so chunk c+1 uploads while
  chunk c computes and chunk c-1 downloads;
* reduction partials of every chunk go to one FP64 partials array (a CTA-row
  offset per chunk) and are finalized once on the device;
* the whole schedule can be captured as one CUDA graph and replayed.

Buffers are sized from a device budget (``budget_bytes``), like the reference's
free-VRAM-based chunk sizing (stenpy_engine.py:606-631) but deterministic.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Any, Dict, List, Optional, Sequence, Tuple

import torch

from . import _native as N
from . import fused_compiler as FC
from .codegen import SHELL_THREADS, PassConfig, pass_grid, shell_count, shell_ctas, shell_regions
from .graph import Graph


@dataclass
class Chunk:
    s: int          # first output plane (global)
    e: int          # one past the last output plane
    lo: int         # first slab plane (global, may be < 0 when wrapped)
    hi: int         # one past the last slab plane (may exceed n0 when wrapped)


def chunk_bounds(s: int, e: int, n0: int, halo: int, periodic: bool) -> Chunk:
    """Slab [lo, hi) that output planes [s, e) read: ``halo`` planes either side,
    wrapped for periodic runs, clipped to the field otherwise."""
    if periodic:
        lo, hi = s - halo, e + halo
        if hi - lo > n0:           # slab would cover the whole ring twice: take it all
            lo, hi = s - halo, s - halo + n0
    else:
        lo, hi = max(0, s - halo), min(n0, e + halo)
    return Chunk(s, e, lo, hi)


def plan_chunks(n0: int, chunk: int, halo: int, periodic: bool) -> List[Chunk]:
    return [chunk_bounds(s, min(n0, s + chunk), n0, halo, periodic) for s in range(0, n0, chunk)]


def chunk_launches(pp: FC.PassPlan, c: Chunk, shape: Tuple[int, int, int], fptrs: Sequence[int],
                   optrs: Sequence[int], table_ptr: int, err_ptr: int, part_ptr: int, cta_off: int
                   ) -> Tuple[FC.Launch, Optional[FC.Launch], int]:
    """The main (z-march) launch and the shell launch (or None) that compute output
    planes [c.s, c.e) of pass ``pp`` from a device slab holding planes [c.lo, c.hi)
    (field pointers ``fptrs``) into outputs holding planes [c.s, c.e) (``optrs``).
    The kernels keep global coordinates (``i_base`` = c.lo, ``n0g`` = the field's
    planes), so every voxel is computed exactly as in a whole-field run. Partial rows
    start at ``cta_off``; returns the launches and the number of rows they write."""
    n0, n1, n2 = shape
    spec = pp.spec
    cfg = spec.cfg
    n_out = c.e - c.s
    gx, gy = pass_grid(spec, n1, n2, n_out)
    grid = (gx, gy, 1)
    nl = c.hi - c.lo
    tmaps = FC.encode_tmaps(spec, list(fptrs), nl, n1, n2)
    vals = dict(fld=list(fptrs), out=list(optrs), scal=table_ptr, part=part_ptr, hist=0, err=err_ptr, n0g=n0,
                n1=n1, n2=n2, nl=nl, i_base=c.lo, out_lo=c.s - c.lo, n_out=n_out, seg_len=cfg.seg_len,
                tiles_k=-(-n2 // cfg.tk), cta_off=cta_off)
    ncta = grid[0] * grid[1]
    n_shell = shell_count(shape, spec.radius, c.s, c.e, shell_regions(spec)) if FC.has_shell(spec) else 0
    sh = shell_ctas(n_shell)
    main = FC.Launch(pp.module, grid, (cfg.threads, 1, 1), pp.smem, FC.pack_params(spec, vals, tmaps))
    shell = None
    if sh:
        shell = FC.Launch(pp.shell_module, (sh, 1, 1), (SHELL_THREADS, 1, 1), 0,
                          FC.pack_params(spec, dict(vals, cta_off=cta_off + ncta), tmaps))
    return main, shell, ncta + sh


def chunk_rows(pp: FC.PassPlan, c: Chunk, shape: Tuple[int, int, int]) -> int:
    """Partial rows ``chunk_launches`` writes for chunk ``c`` (no device work)."""
    n0, n1, n2 = shape
    spec = pp.spec
    gx, gy = pass_grid(spec, n1, n2, c.e - c.s)
    n_shell = shell_count(shape, spec.radius, c.s, c.e, shell_regions(spec)) if FC.has_shell(spec) else 0
    return gx * gy + shell_ctas(n_shell)


def slab_pieces(c: Chunk, n0: int) -> List[Tuple[int, int, int]]:
    """(global start, global end, slab offset) host ranges that make up the slab."""
    pieces = []
    g = c.lo
    off = 0
    while g < c.hi:
        gm = g % n0
        take = min(c.hi - g, n0 - gm)
        pieces.append((gm, gm + take, off))
        g += take
        off += take
    return pieces


def wraps_dim0(spec) -> bool:
    """Whether a pass reads across the dim-0 faces with periodic wrap (then every
    chunk's slab must hold the wrapped planes): a periodic first derivative along
    dim 0, a periodic Laplacian, or periodic taps with a dim-0 offset."""
    for n in spec.graph.nodes:
        if n.op == "d1" and n.a("axis") == 0 and n.a("mode") == "periodic":
            return True
        if n.op == "lap" and n.a("pad") == "periodic":
            return True
        if n.op == "taps" and n.a("pad") == "periodic" and any(t[0] for t in n.a("taps")):
            return True
    return False


def pass_halo(pp: FC.PassPlan) -> int:
    R = pp.spec.radius
    onesided = any(n.op == "d1" and n.a("mode") in ("edge2", "edge1") for n in pp.spec.graph.nodes)
    return R + (1 if (onesided and R > 0) else 0)


class LazyPipeline:
    """Run a graph whose fields are host tensors larger than the device budget."""

    def __init__(self, graph: Graph, wanted: Sequence[str], device: Any = "cuda",
                 budget_bytes: int = 8 << 30, out_dtype: torch.dtype = torch.float32,
                 chunk: Optional[int] = None, config: Optional[PassConfig] = None, periodic: Optional[bool] = None):
        self.graph = graph
        self.wanted = list(wanted)
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.plan = FC.Planner(graph, self.wanted, out_dtype, config).plan()
        if self.plan.dims2:
            raise FC.FusionError("lazy mode chunks 3-D fields along dim 0; 2-D fields run whole")
        if any(pp.spec.has_scan for pp in self.plan.passes):
            raise FC.FusionError("cumulative_integral is not supported in lazy mode")
        if self.plan.hist_size:
            raise FC.FusionError("entropy_hist is not supported in lazy mode")
        self.values = {nid: graph._nodes[nid].params["value"] for nid in self.plan.live
                       if graph._nodes[nid].op_name == "_constant"}
        self.n0, self.n1, self.n2 = self.plan.shape
        if periodic is None:
            periodic = any(p.get("boundary") == "periodic" for p in
                           (graph._nodes[n].params for n in self.plan.live))
        self.periodic = periodic
        self.budget = int(budget_bytes)
        self.chunk = chunk
        self.streams = [torch.cuda.Stream(self.device) for _ in range(3)]
        self._prepared = False

    # ------------------------------------------------------------------ sizing
    def _plane_bytes(self, t: torch.Tensor) -> int:
        return (t.numel() // self.n0) * t.element_size()

    def _choose_chunk(self, pp: FC.PassPlan, H: int) -> int:
        if self.chunk:
            return max(self.chunk, 2 * H + 1)
        fin = sum(self._plane_bytes(self.values[n]) for n in pp.field_nodes)
        fout = 0
        for nid, kind, nc in pp.out_nodes:
            fout += self.n1 * self.n2 * nc * torch.empty((), dtype=self.plan.out_dtype).element_size()
        reserve = 256 << 20
        c = (self.budget - reserve - 2 * 2 * H * fin) // (2 * (fin + fout))
        c = int(max(2 * H + 1, min(c, self.n0)))
        return c

    # ------------------------------------------------------------------ run
    def prepare(self, outputs: Optional[Dict[str, torch.Tensor]] = None) -> None:
        dev = self.device
        dev_idx = dev.index
        plan = self.plan
        self.table = torch.zeros(plan.table_size, dtype=torch.float64, device=dev)
        self.err = FC.ErrorFlag.get(dev)
        if plan.const_index:
            ch = torch.zeros(plan.table_size, dtype=torch.float64)
            for nid, idx in plan.const_index.items():
                v = self.values[nid]
                ch[idx] = float(v.item() if isinstance(v, torch.Tensor) else v)
            self.const_host = ch.pin_memory()
        else:
            self.const_host = None
        self.host_out: Dict[str, torch.Tensor] = {}
        self.passes = []
        for pp in plan.passes:
            FC.compile_pass(pp, dev_idx)
            H = pass_halo(pp)
            C = self._choose_chunk(pp, H)
            # a pass that wraps along dim 0 always gets wrapped slabs, whatever the
            # caller's ``periodic`` says (its slow path reads planes across the faces)
            chunks = plan_chunks(self.n0, C, H, self.periodic or wraps_dim0(pp.spec))
            maxslab = max(c.hi - c.lo for c in chunks)
            spec = pp.spec
            cfg = spec.cfg
            # device slabs / outputs, double buffered
            slabs = []
            for nid in pp.field_nodes:
                src = self.values[nid] if nid in self.values else self.host_out[nid]
                shp = (maxslab,) + tuple(src.shape[1:])
                slabs.append([torch.empty(shp, dtype=src.dtype, device=dev) for _ in range(2)])
            outs = []
            for nid, kind, nc in pp.out_nodes:
                dt = FC.DT_TORCH[[r for r in spec.roots if r.kind in ("out", "scan")][len(outs)].out_dtype]
                comp = FC.comp_shape(nc) + ((1,) if nid in plan.keepdim else ())
                host = outputs.get(nid) if outputs else None
                if host is None:
                    host = torch.empty((self.n0, self.n1, self.n2) + comp, dtype=dt, pin_memory=True)
                self.host_out[nid] = host
                outs.append([torch.empty((C, self.n1, self.n2) + comp, dtype=dt, device=dev) for _ in range(2)])
            total_rows = sum(chunk_rows(pp, c, plan.shape) for c in chunks)
            part = torch.zeros(max(total_rows * spec.nslots, 1), dtype=torch.float64, device=dev)
            packed = []
            cta_off = 0
            for ci, c in enumerate(chunks):
                b = ci % 2
                main, shell, rows = chunk_launches(pp, c, plan.shape, [bufs[b].data_ptr() for bufs in slabs],
                                                   [o[b].data_ptr() for o in outs], self.table.data_ptr(),
                                                   self.err.data_ptr(), part.data_ptr(), cta_off)
                packed.append((c, b, main, shell))
                cta_off += rows
            descs = [N.ReduceDesc(r.kind, r.slot, r.table_index, r.unbiased, r.count, r.eps) for r in pp.reductions]
            self.passes.append(dict(pp=pp, chunks=chunks, C=C, H=H, slabs=slabs, outs=outs, launches=packed,
                                    part=part, ncta_total=cta_off, descs=descs))
        self._prepared = True

    def enqueue(self, timing: bool = False) -> Dict[str, Any]:
        """Enqueue the whole schedule; the compute stream joins the others at the end.
        With ``timing`` it records per-stage CUDA events for the overlap report."""
        if not self._prepared:
            self.prepare()
        h2d, comp, d2h = self.streams
        cur = torch.cuda.current_stream(self.device)
        h2d.wait_stream(cur)
        comp.wait_stream(cur)
        d2h.wait_stream(cur)
        stamps: Dict[str, List] = {"h2d": [], "compute": [], "d2h": []}
        if self.const_host is not None:
            with torch.cuda.stream(comp):
                self.table.copy_(self.const_host, non_blocking=True)
        n_kernels = 0

        def ev():
            return torch.cuda.Event(enable_timing=timing)

        for P in self.passes:
            pp = P["pp"]
            uploaded: List[Optional[torch.cuda.Event]] = [None, None]
            computed: List[Optional[torch.cuda.Event]] = [None, None]
            downloaded: List[Optional[torch.cuda.Event]] = [None, None]
            for c, b, main, shell in P["launches"]:
                # upload slab b once compute of the chunk that last used it is done
                with torch.cuda.stream(h2d):
                    if computed[b] is not None:
                        h2d.wait_event(computed[b])
                    t0 = ev(); t0.record(h2d)
                    for nid, bufs in zip(pp.field_nodes, P["slabs"]):
                        src = self.values[nid] if nid in self.values else self.host_out[nid]
                        for g0, g1, off in slab_pieces(c, self.n0):
                            bufs[b][off:off + (g1 - g0)].copy_(src[g0:g1], non_blocking=True)
                    u = ev(); u.record(h2d)
                    uploaded[b] = u
                    stamps["h2d"].append((t0, u))
                with torch.cuda.stream(comp):
                    comp.wait_event(uploaded[b])
                    if downloaded[b] is not None:
                        comp.wait_event(downloaded[b])
                    t1 = ev(); t1.record(comp)
                    N.launch(main.module, main.grid, main.block, main.smem, comp.cuda_stream, main.params)
                    n_kernels += 1
                    if shell is not None:
                        N.launch(shell.module, shell.grid, shell.block, shell.smem, comp.cuda_stream, shell.params)
                        n_kernels += 1
                    k = ev(); k.record(comp)
                    computed[b] = k
                    stamps["compute"].append((t1, k))
                with torch.cuda.stream(d2h):
                    d2h.wait_event(computed[b])
                    t2 = ev(); t2.record(d2h)
                    n_out = c.e - c.s
                    for (nid, kind, nc), bufs in zip(pp.out_nodes, P["outs"]):
                        self.host_out[nid][c.s:c.e].copy_(bufs[b][:n_out], non_blocking=True)
                    dn = ev(); dn.record(d2h)
                    downloaded[b] = dn
                    stamps["d2h"].append((t2, dn))
            # the pass is done when its last download and compute are
            comp.wait_stream(d2h)
            comp.wait_stream(h2d)
            if P["descs"]:
                N.finalize(P["part"].data_ptr(), P["ncta_total"], pp.spec.nslots, P["descs"],
                           self.table.data_ptr(), comp.cuda_stream)
                n_kernels += 1
        cur.wait_stream(comp)
        self.n_kernels = n_kernels
        return stamps

    def results(self) -> Dict[str, Any]:
        torch.cuda.current_stream(self.device).synchronize()
        out: Dict[str, Any] = {}
        for nid in self.wanted:
            if nid in self.host_out:
                out[nid] = self.host_out[nid]
            elif nid in self.plan.red_index:
                idx = self.plan.red_index[nid]
                n = 2 if self.plan.infos[nid].nc == 2 else 1
                out[nid] = self.table[idx:idx + n].cpu() if n == 2 else self.table[idx].cpu()
            elif nid in self.plan.scalar_sinks:
                raise FC.FusionError("scalar-expression sinks are not supported in lazy mode")
            else:
                out[nid] = self.values[nid]
        return out

    def run(self) -> Dict[str, Any]:
        self.enqueue()
        return self.results()

    def capture(self) -> torch.cuda.CUDAGraph:
        """Capture the whole chunk schedule (copies, kernels, finalizes) as one graph."""
        if not self._prepared:
            self.prepare()
        torch.cuda.synchronize(self.device)
        side = torch.cuda.Stream(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            self.enqueue(timing=False)
        return g

    @staticmethod
    def overlap_report(stamps: Dict[str, List]) -> Dict[str, float]:
        """Busy time of each stage and the wall time spanned, from recorded events."""
        starts = [a for v in stamps.values() for a, _ in v]
        ends = [b for v in stamps.values() for _, b in v]
        first = starts[0]
        wall = max(first.elapsed_time(e) for e in ends)
        rep = {"wall_ms": wall}
        for k, v in stamps.items():
            busy = sum(a.elapsed_time(b) for a, b in v)
            rep[f"{k}_busy_ms"] = busy
            rep[f"{k}_busy_frac"] = busy / wall if wall > 0 else 0.0
        rep["overlap_factor"] = sum(rep[f"{k}_busy_ms"] for k in stamps) / wall if wall > 0 else 0.0
        return rep


def run_chunked(graph: Graph, sink_id: str, device: Any = "cuda", chunk_size: Optional[int] = None,
                budget_bytes: int = 8 << 30, out_dtype: torch.dtype = torch.float32) -> Dict[str, Any]:
    """Reference-shaped entry (stenpy_engine.py:697-888): stream ``sink_id`` through the
    device and return ``{sink_id: {shape_out, min, max, mean, out, n_chunks}}``
    (``out`` is the pinned host result; the reference writes an HDF5 file)."""
    lp = LazyPipeline(graph, [sink_id], device, budget_bytes, out_dtype, chunk_size)
    res = lp.run()[sink_id]
    r64 = res.double() if isinstance(res, torch.Tensor) else res
    return {sink_id: {"shape_out": tuple(res.shape), "min": float(r64.min()), "max": float(r64.max()),
                      "mean": float(r64.mean()), "out": res,
                      "n_chunks": len(lp.passes[0]["chunks"]) if lp.passes else 0}}
