"""Host logic of a multi-GPU bench run, on CPU: two gloo ranks stand in for
two GPUs.  Each rank is an independent replica (its own seed, no data-path
collective); the whole-job rate is the sum of the ranks' particle-steps over
the slowest rank's time."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    from datetime import timedelta

    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=timedelta(seconds=60))
    try:
        r = bench.Ranks(dist, world, rank, "cpu")
        r.barrier()
        units = [3.0e9, 5.0e9][rank]            # particle-steps done by this rank
        ms = [800.0, 1000.0][rank]              # its device time
        out.put((rank, r.max(ms), r.sum(units), r.rate(units, ms), bench.replica_seed(rank)))
        r.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_sum_work_and_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, tmax, tot, rate, seed in res:
        assert tmax == 1000.0
        assert tot == 8.0e9
        assert rate == pytest.approx(8.0e9 / 1.0)
    assert res[0][4] != res[1][4]                 # replicas do not repeat each other


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    r = bench.Ranks()
    assert r.max(2.5) == 2.5 and r.sum(4.0) == 4.0
    assert r.rate(1e9, 500.0) == pytest.approx(2e9)
