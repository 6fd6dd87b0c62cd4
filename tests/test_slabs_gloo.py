"""Dim-0 slab decomposition across ranks, on the CPU: slab bounds follow the lazy
pipeline's chunk rule, the halo exchange fills every rank's halo planes with the
neighbours' planes (wrapped for periodic runs, none past a non-periodic face),
owned planes reassemble into the field, and partial rows are stacked in rank
order behind identity padding. Two and three gloo ranks in separate processes,
and the in-process emulation used on one GPU."""
import os
import socket
from types import SimpleNamespace

import pytest
import torch
import torch.multiprocessing as mp

from stenpy_b200 import _native as N
from stenpy_b200.lazy import plan_chunks
from stenpy_b200.slabs import (halo_ops, identity_rows, match_p2p, owned_range, plan_slabs)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _field(n0, seed=0):
    g = torch.Generator().manual_seed(seed)
    return torch.randn((n0, 5, 7, 3), generator=g, dtype=torch.float32)


def _expected_slab(G, c, periodic):
    n0 = G.shape[0]
    idx = torch.arange(c.lo, c.hi)
    return G[idx % n0] if periodic else G[idx.clamp(0, n0 - 1)]


@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("n0,world,halo", [(24, 2, 1), (24, 3, 2), (32, 4, 3), (16, 1, 2)])
def test_slab_bounds_follow_the_chunk_rule(n0, world, halo, periodic):
    if world > 1:
        assert plan_slabs(n0, world, halo, periodic) == plan_chunks(n0, n0 // world, halo, periodic)
    else:                                   # one rank: the whole field, dim 0 wrapped by the kernels
        assert [(c.s, c.e, c.lo, c.hi) for c in plan_slabs(n0, 1, halo, periodic)] == [(0, n0, 0, n0)]
    # uneven splits: owned ranges tile the field, sizes within one plane
    for n in (n0 + 1, n0 + world - 1):
        owned = [owned_range(n, r, world) for r in range(world)]
        assert owned[0][0] == 0 and owned[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(owned, owned[1:]))
        assert max(e - s for s, e in owned) - min(e - s for s, e in owned) <= 1


@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("n0,world,halo", [(20, 1, 2), (20, 2, 2), (21, 3, 1), (23, 4, 2), (12, 3, 3)])
def test_in_process_exchange_fills_halos(n0, world, halo, periodic):
    G = _field(n0)
    chunks = plan_slabs(n0, world, halo, periodic)
    slabs, ops = [], []
    for r, c in enumerate(chunks):
        slab = torch.full((c.hi - c.lo,) + tuple(G.shape[1:]), float("nan"))
        slab[c.s - c.lo:c.e - c.lo] = G[c.s:c.e]
        slabs.append(slab)
        ops.append(halo_ops(slab, chunks, r, periodic))
    match_p2p(ops)
    for c, slab in zip(chunks, slabs):
        assert torch.equal(slab, _expected_slab(G, c, periodic)), c


def test_too_many_ranks_are_refused():
    from stenpy_b200.fused_compiler import FusionError
    with pytest.raises(FusionError):
        plan_slabs(3, 4, 1, True)
    with pytest.raises(FusionError):
        plan_slabs(8, 4, 3, True)       # slabs of 2 planes, halo 3


def test_identity_rows_leave_reductions_unchanged():
    reds = [SimpleNamespace(kind=N.RED_VARIANCE, slot=0), SimpleNamespace(kind=N.RED_MIN_MAX, slot=3),
            SimpleNamespace(kind=N.RED_SUM, slot=5)]
    pp = SimpleNamespace(spec=SimpleNamespace(nslots=6), reductions=reds)
    t = identity_rows(pp, 4, "cpu")
    assert t.shape == (4, 6)
    assert torch.all(t[:, [0, 1, 2, 5]] == 0)
    assert torch.all(t[:, 3] == float("inf")) and torch.all(t[:, 4] == float("-inf"))


def _worker(rank, world, port, periodic, out):
    import torch.distributed as dist
    from stenpy_b200.slabs import DistExchange, gather_planes
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ex = DistExchange()
        n0, halo = 22, 2
        G = _field(n0, seed=3)                        # every rank builds the same field
        chunks = plan_slabs(n0, world, halo, periodic)
        c = chunks[rank]
        slab = torch.full((c.hi - c.lo,) + tuple(G.shape[1:]), float("nan"))
        slab[c.s - c.lo:c.e - c.lo] = G[c.s:c.e]       # only the owned planes are known
        ex.p2p(halo_ops(slab, chunks, rank, periodic))
        ok_halo = torch.equal(slab, _expected_slab(G, c, periodic))
        whole = gather_planes(slab[c.s - c.lo:c.e - c.lo], ex, n0)
        ok_gather = whole is None if rank else torch.equal(whole, G)
        rows = torch.full((3, 2), float(rank), dtype=torch.float64)
        stacked = ex.all_gather_rows(rows)
        ok_rows = torch.equal(stacked, torch.cat([torch.full((3, 2), float(r), dtype=torch.float64)
                                                  for r in range(world)]))
        out.put((rank, ok_halo, ok_gather, ok_rows))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("periodic", [True, False])
def test_gloo_ranks_exchange_halos_and_reassemble(world, periodic):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, periodic, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ok_halo, ok_gather, ok_rows in res:
        assert ok_halo and ok_gather and ok_rows, (rank, ok_halo, ok_gather, ok_rows)
