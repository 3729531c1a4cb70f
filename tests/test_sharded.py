"""Sharding one scene's contact work over ranks (ipc_warp_b200.sharded), on
CPU: the query partition, and the exchange step between two gloo ranks
(force and energy summed, time of impact minimised, status bits ORed)."""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_shard_ranges_partition_the_queries():
    from ipc_warp_b200.sharded import shard_range

    for n in (0, 1, 7, 100, 1_490_112):
        for world in (1, 2, 3, 8):
            covered = []
            sizes = []
            for r in range(world):
                first, count = shard_range(n, r, world)
                covered.extend(range(first, first + count))
                sizes.append(count)
            assert covered == list(range(n))
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    from ipc_warp_b200.sharded import combine

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = torch.Generator().manual_seed(rank)
        force = torch.randn((5, 3), generator=g, dtype=torch.float32)
        mine = force.clone()
        scalars = torch.tensor([0.5 + rank, 10.0 * (rank + 1), 3.0 * rank], dtype=torch.float64)
        toi = torch.tensor([0.7 - 0.2 * rank], dtype=torch.float64)
        status = torch.tensor([1 << rank], dtype=torch.int32)
        combine(force, scalars, toi, status)
        out[rank] = (mine.tolist(), force.tolist(), scalars.tolist(), toi.tolist(), status.tolist())
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_exchange_over_two_gloo_ranks():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    total = torch.tensor(res[0][0]) + torch.tensor(res[1][0])
    for r in range(world):
        _, force, scalars, toi, status = res[r]
        assert torch.allclose(torch.tensor(force), total)
        assert scalars == pytest.approx([2.0, 30.0, 3.0])
        assert toi == pytest.approx([0.5])
        assert status == [3]
