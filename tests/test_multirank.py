"""The N > 1 host path of bench.py (one process per GPU, replicas of the same
workload): timings are the slowest rank's, throughputs add up, and the
whole-job value counts every replica.  Two ranks over gloo on the CPU."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import bench
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        # rank r: a step of 10 + r ms, an end-to-end step of 5 (r + 1) ms,
        # and (serving) 1.5 (r + 1) M cliques/s
        step_ms, e2e_ms = bench.max_over_ranks([10.0 + rank, 5.0 * (rank + 1)], "cpu")
        (rate,) = bench.sum_over_ranks([1.5e6 * (rank + 1)], "cpu")
        torch.distributed.barrier()
        out.put((rank, step_ms, e2e_ms, rate))
    finally:
        torch.distributed.destroy_process_group()


def test_two_ranks_max_sum_and_job_value():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = sorted(out.get(timeout=120) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [g[0] for g in got] == [0, 1]
    for _, step_ms, e2e_ms, rate in got:  # every rank sees the same reduced values
        assert (step_ms, e2e_ms) == (11.0, 10.0)
        assert rate == pytest.approx(4.5e6)
    sys.path.insert(0, ROOT)
    import bench
    # 2 replicas of 100 units in (max) 50 ms: 4,000 units/s for the job
    assert bench.job_value(100, 50.0, 2) == pytest.approx(4000.0)
    assert bench.job_value(100, 50.0, 1) == pytest.approx(2000.0)


def test_single_process_reductions_are_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([3.0, 7.5], "cpu") == [3.0, 7.5]
    assert bench.sum_over_ranks([2.5], "cpu") == [2.5]
