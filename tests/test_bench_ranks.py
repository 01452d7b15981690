"""The multi-rank plumbing of bench.py on CPU: two gloo ranks, as torchrun would start them.

On a GPU node each rank times its own replica of the workload on its own GPU; the job's
duration is the maximum over ranks and its throughput counts every rank's units over that
duration.  Here each rank contributes a different duration and both must see the maximum.
"""
from __future__ import annotations

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = 1.5 + rank  # seconds on this rank
        slowest = bench.max_over_ranks(mine, dist)
        dist.barrier()
        out.put((rank, slowest, bench.replica_value(world, 1000.0, slowest)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slowest, value in res:
        assert slowest == 2.5
        assert value == pytest.approx(2 * 1000.0 / 2.5)


def test_single_process_has_no_reduction():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.25, None) == 3.25
    assert bench.replica_value(1, 10.0, 2.0) == 5.0


def test_error_summary_names_unexplained_instances():
    """bench.summarize_errors: instances over the bar split into those the FP64 form's own
    error explains (FP32-bulk within 10x of it) and those it does not, the latter listed"""
    sys.path.insert(0, ROOT)
    import bench

    err = {"fp32_bulk": [1e-7, 2e-5, 3e-4, 5e-5], "fp64": [1e-9, 1e-5, 1e-7, 6e-6]}
    s = bench.summarize_errors(err, bar=1e-5)
    assert s["fp32_vs_oracle"]["within_bar"] == 1 and s["fp32_vs_oracle"]["n"] == 4
    assert s["over_bar_explained_by_fp64_spread"] == 2  # 2e-5 <= 10 * 1e-5, 5e-5 <= 10 * 6e-6
    assert s["over_bar_unexplained"] == 1
    assert s["unexplained_instances"] == [dict(k=2, fp32=3e-4, fp64=1e-7)]
