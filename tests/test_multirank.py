"""Host logic of the N-GPU benchmark on CPU ranks (gloo, world size 2).

Multi-GPU runs are independent replicas: every rank mines its own database
of the same shape (the workload's seed plus the rank), and the only
collective is the max-reduce of the per-rank timings.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        seed = (bench.rank_seed("planted-100k", rank), bench.rank_seed("temporal-100k", rank))
        # rank 1 is slower on the first value, rank 0 on the second
        got = bench.max_over_ranks([1.0 + rank, 5.0 - rank], "cpu")
        out.put((rank, seed, got))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replicas_take_distinct_seeds_and_max_timings():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    seeds = [s for _, s, _ in results]
    assert seeds == [(7, 23), (8, 24)]
    for _, _, got in results:
        assert got == [2.0, 5.0]
