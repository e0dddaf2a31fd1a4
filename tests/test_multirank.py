"""The N > 1 path of bench.py on CPU: two ranks over gloo.

The step does not shard, so N GPUs run N independent replicas; the only
cross-rank work is the timing: every rank's elapsed time is all-reduced with
MAX and the whole-job rate is N replicas' points x steps over that time.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import bench
        mine = 10.0 + 5.0 * rank  # rank 1 is the slower one
        slowest = bench.max_over_ranks(mine, world, device="cpu")
        rate = bench.replicas_rate(world, 128 ** 3, 20, slowest / 1e3)
        dist.barrier()
        q.put((rank, slowest, rate))
    finally:
        dist.destroy_process_group()


def test_two_replicas_time_by_the_slowest_rank():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=5) for _ in range(world))
    for rank, slowest, rate in got:
        assert slowest == 15.0  # both ranks see the max
        assert rate == pytest.approx(2 * 128 ** 3 * 20 / 0.015 / 1e6)


def test_single_rank_passes_through():
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.replicas_rate(1, 100, 10, 2.0) == pytest.approx(100 * 10 / 2.0 / 1e6)
