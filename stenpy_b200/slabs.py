"""Dim-0 slab decomposition of one field across ranks (one process per GPU).

The reference shards a field into dim-0 slabs, swaps radius-thick faces with its
neighbours (``_halo_exchange_1d`` over MPI or torch.distributed,
memory_manager.py:103-147, stenpy_engine.py:3257-3353) and all-reduces global
reductions (memory_manager.py:499-513). Here the same decomposition feeds the
fused executor:

* rank r owns planes [r·n0/W, (r+1)·n0/W) of every field; for each pass its slab
  is [lo, hi) by the chunk rule of the lazy pipeline (``lazy.chunk_bounds``:
  ``pass_halo`` planes either side, wrapped when the pass reads across the dim-0
  faces periodically, clipped at the field's faces otherwise);
* the halo planes come from the neighbouring ranks by point-to-point sends and
  receives into this rank's own slab buffer (NCCL on GPUs, gloo on CPUs; no peer
  memory is read by any kernel and no TMA touches another GPU);
* the pass kernels run on the slab with global coordinates (the lazy pipeline's
  chunk launches), so every voxel is computed exactly as in a whole-field run;
* global reductions: every rank's FP64 partial rows (padded with identity rows to
  a common count) are all-gathered and folded by the finalize kernel in rank
  order on every rank, so all ranks hold the same scalars, bit for bit.

Scans along dim 0 (``cumulative_integral``) and histogram entropy are not
decomposed (``FusionError``).

The steps are split so that one driver can run them with real collectives
(``DistExchange`` over a process group) and another can emulate several ranks in
one process (``LocalRanks``), which is how a single GPU exercises the path.
"""
from __future__ import annotations

from collections import defaultdict, deque
from typing import Any, Dict, List, Optional, Sequence, Tuple

import torch

from . import _native as N
from . import fused_compiler as FC
from .graph import Graph
from .lazy import Chunk, chunk_bounds, chunk_launches, chunk_rows, pass_halo, wraps_dim0


def owned_range(n0: int, rank: int, world: int) -> Tuple[int, int]:
    """Planes [s, e) that ``rank`` owns: balanced, sizes differ by at most one."""
    return rank * n0 // world, (rank + 1) * n0 // world


def plan_slabs(n0: int, world: int, halo: int, periodic: bool) -> List[Chunk]:
    """One chunk per rank (its owned planes and the slab they read)."""
    if world < 1 or n0 < world:
        raise FC.FusionError(f"cannot split {n0} planes over {world} ranks")
    if world == 1:      # the whole field: the kernels wrap dim 0 themselves, as in a whole-field run
        return [Chunk(0, n0, 0, n0)]
    out = [chunk_bounds(*owned_range(n0, r, world), n0, halo, periodic) for r in range(world)]
    if world > 1:
        for c in out:
            if c.e - c.s < halo:
                raise FC.FusionError(f"slab of {c.e - c.s} planes is thinner than the halo ({halo}): "
                                     "use fewer ranks")
            if c.hi - c.lo >= n0 and periodic:
                raise FC.FusionError("periodic halos would cover the whole field: use fewer ranks")
    return out


def _neighbours(rank: int, world: int, periodic: bool) -> Tuple[Optional[int], Optional[int]]:
    left = (rank - 1) % world if (periodic or rank > 0) else None
    right = (rank + 1) % world if (periodic or rank < world - 1) else None
    return left, right


def halo_ops(slab: torch.Tensor, chunks: Sequence[Chunk], rank: int, periodic: bool
             ) -> List[Tuple[str, int, torch.Tensor]]:
    """Point-to-point operations that fill ``slab``'s halo planes, in the order every
    rank issues them: send to the left neighbour, send to the right one, receive the
    right halo, receive the left halo. ``slab`` holds planes [lo, hi) of this rank's
    chunk with its owned planes in place. A rank alone on a periodic ring is its own
    neighbour (the operations pair up locally)."""
    world = len(chunks)
    c = chunks[rank]
    left, right = _neighbours(rank, world, periodic)
    hl, hr = c.s - c.lo, c.hi - c.e
    own0, own1 = c.s - c.lo, c.e - c.lo
    ops: List[Tuple[str, int, torch.Tensor]] = []
    if left is not None:
        cl = chunks[left]
        need = cl.hi - cl.e                    # the left neighbour's right halo: my first planes
        if need:
            ops.append(("send", left, slab[own0:own0 + need]))
    if right is not None:
        cr = chunks[right]
        need = cr.s - cr.lo                    # the right neighbour's left halo: my last planes
        if need:
            ops.append(("send", right, slab[own1 - need:own1]))
    if right is not None and hr:
        ops.append(("recv", right, slab[own1:own1 + hr]))
    if left is not None and hl:
        ops.append(("recv", left, slab[0:hl]))
    return ops


class DistExchange:
    """Collectives of the slab path over a torch.distributed process group (NCCL for
    CUDA tensors, gloo for CPU tensors). Every rank calls each method in the same
    order."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def p2p(self, ops: Sequence[Tuple[str, int, torch.Tensor]]) -> None:
        dist = self.dist
        local = defaultdict(deque)
        p2p = []
        for kind, peer, t in ops:
            if peer == self.rank:              # a rank alone on a periodic ring
                (local[kind]).append(t)
                continue
            buf = t if t.is_contiguous() else t.contiguous()
            op = dist.P2POp(dist.isend if kind == "send" else dist.irecv, buf, peer, self.group)
            p2p.append((op, t, buf))
        while local["send"]:
            local["recv"].popleft().copy_(local["send"].popleft())
        if p2p:
            for req in dist.batch_isend_irecv([op for op, _, _ in p2p]):
                req.wait()
            for op, t, buf in p2p:
                if buf is not t:
                    t.copy_(buf)

    def all_gather_rows(self, rows: torch.Tensor) -> torch.Tensor:
        """Rows of every rank, stacked in rank order."""
        out = torch.empty((self.world,) + tuple(rows.shape), dtype=rows.dtype, device=rows.device)
        if rows.is_cuda:
            self.dist.all_gather_into_tensor(out, rows.contiguous(), group=self.group)
        else:
            parts = list(out.unbind(0))
            self.dist.all_gather(parts, rows.contiguous(), group=self.group)
            out = torch.stack(parts)
        return out.reshape((-1,) + tuple(rows.shape[1:]))


def match_p2p(per_rank_ops: Sequence[Sequence[Tuple[str, int, torch.Tensor]]]) -> None:
    """Carry out the point-to-point operations of several ranks held in one process:
    sends and receives between a pair of ranks match in issue order."""
    queues = defaultdict(deque)
    for r, ops in enumerate(per_rank_ops):
        for kind, peer, t in ops:
            if kind == "send":
                queues[(r, peer)].append(t)
    for r, ops in enumerate(per_rank_ops):
        for kind, peer, t in ops:
            if kind == "recv":
                q = queues[(peer, r)]
                if not q:
                    raise RuntimeError(f"rank {r}: no message from rank {peer}")
                t.copy_(q.popleft())
    left = {k: len(q) for k, q in queues.items() if q}
    if left:
        raise RuntimeError(f"unmatched sends: {left}")


def identity_rows(pp: FC.PassPlan, rows: int, device) -> torch.Tensor:
    """``rows`` partial rows that leave every reduction of the pass unchanged when
    folded: zeros (sums, (n = 0) variance and co-moment rows), (+inf, -inf) for
    min/max."""
    t = torch.zeros((rows, max(pp.spec.nslots, 1)), dtype=torch.float64, device=device)
    for r in pp.reductions:
        if r.kind == N.RED_MIN_MAX:
            t[:, r.slot] = float("inf")
            t[:, r.slot + 1] = float("-inf")
    return t


class SlabRank:
    """One rank's share of a graph: its owned planes of every field in, its owned
    planes of every per-voxel result and every scalar result out.

    ``fields`` maps the graph's field-constant node ids to this rank's owned planes
    (tensors of shape (e - s, n1, n2, ...)); the graph's own constants only give
    shapes and dtypes beyond dim 0, and ``n0`` is the global number of planes."""

    def __init__(self, graph: Graph, wanted: Sequence[str], n0: int, rank: int, world: int, device: Any,
                 out_dtype: torch.dtype = torch.float32, config=None, periodic: Optional[bool] = None):
        self.rank, self.world, self.n0 = rank, world, n0
        self.device = torch.device(device)
        self.wanted = list(wanted)
        g = graph
        self.leaf: Dict[str, torch.Tensor] = {}
        for nid in g.live_nodes(self.wanted):
            node = g._nodes[nid]
            v = node.params.get("value") if node.op_name == "_constant" else None
            if isinstance(v, torch.Tensor) and v.ndim >= 3:
                shape = (n0,) + tuple(v.shape[1:])
                g = g.clone_with_replacement(nid, torch.zeros(1, dtype=v.dtype).expand(*shape))
                self.leaf[nid] = v
        self.plan = FC.Planner(g, self.wanted, out_dtype, config).plan()
        if self.plan.dims2:
            raise FC.FusionError("slab decomposition splits 3-D fields along dim 0")
        if any(pp.spec.has_scan for pp in self.plan.passes) or self.plan.hist_size:
            raise FC.FusionError("cumulative_integral and entropy_hist are not decomposed across ranks")
        if self.plan.scalar_sinks:
            raise FC.FusionError("scalar-expression results are not decomposed across ranks")
        if periodic is None:
            periodic = any(p.get("boundary") == "periodic" for p in
                           (g._nodes[n].params for n in self.plan.live))
        self.periodic = periodic
        _, self.n1, self.n2 = self.plan.shape
        self.s, self.e = owned_range(n0, rank, world)
        for nid, v in self.leaf.items():
            if v.shape[0] != self.e - self.s:
                raise FC.FusionError(f"rank {rank} holds {v.shape[0]} planes of {nid}, owns {self.e - self.s}")
        self.table = torch.zeros(self.plan.table_size, dtype=torch.float64, device=self.device)
        for nid, idx in self.plan.const_index.items():
            c = g._nodes[nid].params["value"]
            self.table[idx] = float(c.item() if isinstance(c, torch.Tensor) else c)
        self.err = FC.ErrorFlag.get(self.device)
        self.outputs: Dict[str, torch.Tensor] = {}
        for pp in self.plan.passes:
            FC.compile_pass(pp, self.device.index if self.device.index is not None else 0)

    # -- one pass, in steps a driver interleaves with the other ranks
    def pass_chunks(self, pi: int) -> List[Chunk]:
        pp = self.plan.passes[pi]
        return plan_slabs(self.n0, self.world, pass_halo(pp), self.periodic or wraps_dim0(pp.spec))

    def pass_begin(self, pi: int) -> List[Tuple[str, int, torch.Tensor]]:
        """Allocate the slabs of pass ``pi``, copy the owned planes in and return the
        halo operations to carry out."""
        pp = self.plan.passes[pi]
        chunks = self.pass_chunks(pi)
        c = chunks[self.rank]
        self._chunks = chunks
        self._slabs = []
        ops = []
        for nid in pp.field_nodes:
            v = self.leaf[nid]
            slab = torch.empty((c.hi - c.lo,) + tuple(v.shape[1:]), dtype=v.dtype, device=self.device)
            slab[c.s - c.lo:c.e - c.lo].copy_(v)
            self._slabs.append(slab)
            ops += halo_ops(slab, chunks, self.rank, self.periodic or wraps_dim0(pp.spec))
        return ops

    def pass_compute(self, pi: int) -> torch.Tensor:
        """Launch the pass on this rank's slab; returns its partial rows padded to the
        largest row count of any rank (identity rows)."""
        pp = self.plan.passes[pi]
        chunks = self._chunks
        c = chunks[self.rank]
        shape = self.plan.shape
        rows_max = max(chunk_rows(pp, ci, shape) for ci in chunks)
        rows = identity_rows(pp, max(rows_max, 1), self.device)
        outs = []
        for (nid, kind, nc), r in zip(pp.out_nodes, [r for r in pp.spec.roots if r.kind in ("out", "scan")]):
            comp = FC.comp_shape(nc) + ((1,) if nid in self.plan.keepdim else ())
            o = torch.empty((c.e - c.s, self.n1, self.n2) + comp, dtype=FC.DT_TORCH[r.out_dtype],
                            device=self.device)
            outs.append(o)
            self.outputs[nid] = o
        main, shell, n = chunk_launches(pp, c, shape, [t.data_ptr() for t in self._slabs],
                                        [o.data_ptr() for o in outs], self.table.data_ptr(), self.err.data_ptr(),
                                        rows.data_ptr(), 0)
        s = torch.cuda.current_stream(self.device).cuda_stream
        N.launch(main.module, main.grid, main.block, main.smem, s, main.params)
        if shell is not None:
            N.launch(shell.module, shell.grid, shell.block, shell.smem, s, shell.params)
        self._rows_keep = (self._slabs, rows)
        return rows

    def pass_finalize(self, pi: int, all_rows: torch.Tensor) -> None:
        """Fold every rank's rows (stacked in rank order) into the scalar table."""
        pp = self.plan.passes[pi]
        if pp.reductions:
            descs = [N.ReduceDesc(r.kind, r.slot, r.table_index, r.unbiased, r.count, r.eps)
                     for r in pp.reductions]
            s = torch.cuda.current_stream(self.device).cuda_stream
            N.finalize(all_rows.data_ptr(), all_rows.shape[0], pp.spec.nslots, descs, self.table.data_ptr(), s)
        self._slabs = []

    def results(self) -> Dict[str, Any]:
        out: Dict[str, Any] = {}
        for nid in self.wanted:
            if nid in self.outputs:
                out[nid] = self.outputs[nid]
            elif nid in self.plan.red_index:
                idx = self.plan.red_index[nid]
                n = 2 if self.plan.infos[nid].nc == 2 else 1
                out[nid] = self.table[idx:idx + n].clone() if n == 2 else self.table[idx].clone()
        return out


def run_distributed(graph: Graph, wanted: Sequence[str], n0: int, device: Any, exchange: DistExchange,
                    **kw) -> Dict[str, Any]:
    """This rank's results of ``graph`` decomposed over ``exchange``'s process group."""
    sr = SlabRank(graph, wanted, n0, exchange.rank, exchange.world, device, **kw)
    for pi in range(len(sr.plan.passes)):
        exchange.p2p(sr.pass_begin(pi))
        rows = sr.pass_compute(pi)
        all_rows = exchange.all_gather_rows(rows) if sr.plan.passes[pi].reductions else rows
        sr.pass_finalize(pi, all_rows)
    FC.ErrorFlag.check(sr.device)
    return sr.results()


class LocalRanks:
    """Several ranks emulated in one process (one device): the halo operations pair
    up by ``match_p2p`` and the partial rows are stacked in rank order, exactly what
    the collectives of ``DistExchange`` deliver. No kernel waits on another rank."""

    def __init__(self, graphs: Sequence[Graph], wanted_per_rank: Sequence[Sequence[str]], n0: int, device: Any,
                 **kw):
        world = len(graphs)
        self.ranks = [SlabRank(g, w, n0, r, world, device, **kw) for r, (g, w) in
                      enumerate(zip(graphs, wanted_per_rank))]

    def run(self) -> List[Dict[str, Any]]:
        npass = len(self.ranks[0].plan.passes)
        for pi in range(npass):
            match_p2p([r.pass_begin(pi) for r in self.ranks])
            rows = [r.pass_compute(pi) for r in self.ranks]
            stacked = torch.cat(rows, 0)
            for r in self.ranks:
                r.pass_finalize(pi, stacked)
        torch.cuda.synchronize(self.ranks[0].device)
        FC.ErrorFlag.check(self.ranks[0].device)
        return [r.results() for r in self.ranks]


def gather_planes(local: torch.Tensor, exchange: DistExchange, n0: int, root: int = 0) -> Optional[torch.Tensor]:
    """Reassemble a per-voxel result from every rank's owned planes (on ``root``)."""
    world = exchange.world
    base = max(owned_range(n0, r, world)[1] - owned_range(n0, r, world)[0] for r in range(world))
    pad = torch.zeros((base,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[:local.shape[0]].copy_(local)
    stacked = exchange.all_gather_rows(pad.reshape(base, -1)).reshape((world, base) + tuple(local.shape[1:]))
    if exchange.rank != root:
        return None
    parts = []
    for r in range(world):
        s, e = owned_range(n0, r, world)
        parts.append(stacked[r, :e - s])
    return torch.cat(parts, 0)
