"""The replica path of bench.py under torchrun (N > 1) without a GPU: two gloo ranks on
the CPU.  Each rank times its own replica; every reported timing is the maximum over the
ranks, and a rate is all ranks' units over the slowest rank's time.  CPU only."""

import datetime
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=30))
    try:
        # rank r saw ms = 10 + r for its steps and 50 - r for its Hessian actions
        ms, hms = bench.max_over_ranks([10.0 + rank, 50.0 - rank], world)
        rate = bench.whole_job_rate(1000, ms, world)
        out.put((rank, ms, hms, rate))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_timings_are_the_maximum_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(out.get(timeout=10) for _ in range(2))
    for rank, ms, hms, rate in got:
        assert ms == 11.0 and hms == 50.0            # the slowest rank's figures, on every rank
        assert rate == pytest.approx(2 * 1000 / 0.011)


def test_one_rank_keeps_its_own_figures():
    import bench

    assert bench.max_over_ranks([3, 4.5], 1) == [3.0, 4.5]
    assert bench.whole_job_rate(262144 * 20, 45.0, 1) == pytest.approx(262144 * 20 / 0.045)
