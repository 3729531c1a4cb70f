"""The multi-process parts of bench.py on CPU: two gloo ranks combine their
timings as the maximum over ranks, the job throughput counts every replica,
and the reference arm does no work on ranks other than 0."""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r reports (10 + r, 20 - r) ms: the maxima are (10 + world - 1, 20)
        total, e2e = bench.max_over_ranks([10.0 + rank, 20.0 - rank], torch.device("cpu"))
        out[rank] = (total, e2e)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_timings_are_maxima_over_two_gloo_ranks():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1] == (11.0, 20.0)


def test_job_throughput_counts_every_replica():
    sys.path.insert(0, ROOT)
    import bench

    one = bench.job_throughput(1, 1000, 5, 10.0)
    assert one == pytest.approx(1000 * 5 / 0.010)
    assert bench.job_throughput(4, 1000, 5, 10.0) == pytest.approx(4 * one)


def test_reference_arm_idles_on_other_ranks(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("RANK", "1")
    called = []
    monkeypatch.setattr(bench, "scene", lambda: called.append(1))
    assert bench.run_reference(None) is None
    assert not called
