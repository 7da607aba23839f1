"""Replica runs (one process per GPU, no data-path collective): the bench's
whole-job aggregation over ranks, exercised with two gloo ranks on the CPU.
Each rank reports its own device time and pushes; the job's step time is the
maximum over ranks and its pushes the sum."""
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
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r: (10 + r) ms for (r + 1) million pushes
        ms_max, total, value = bench.aggregate_ranks(10.0 + rank, 1e6 * (rank + 1), dist, device="cpu")
        out[rank] = (ms_max, total, value, bench.dist_setup())
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_max_time_and_total_pushes():
    world, port = 2, _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
        res = dict(out)
    assert sorted(res) == [0, 1]
    for rank, (ms_max, total, value, setup) in res.items():
        assert ms_max == 11.0
        assert total == 3e6
        assert value == pytest.approx(3e6 / 0.011, rel=1e-12)
        assert setup[:2] == (world, rank)


def test_single_process_needs_no_process_group():
    import bench
    ms_max, total, value = bench.aggregate_ranks(4.0, 2e6)
    assert (ms_max, total) == (4.0, 2e6)
    assert value == pytest.approx(5e8)
