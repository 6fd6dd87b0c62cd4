"""Multi-process plumbing of replica runs on the CPU: two gloo ranks agree on the
max step time and take disjoint, complete shares of independent jobs."""
import os
import socket

import torch
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    import torch.distributed as dist
    from stenpy_b200.replicas import max_over_ranks, shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = max_over_ranks(1.5 + rank, world)
        mine = shard(list(range(11)), rank, world)
        got = [None] * world
        dist.all_gather_object(got, mine)
        out.put((rank, t, got))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_max_and_shards():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, got in res:
        assert t == 2.5
        assert sorted(x for part in got for x in part) == list(range(11))
        assert not set(got[0]) & set(got[1])
