"""The multi-GPU harness logic on two CPU ranks (gloo): plane sharding, the
slowest-rank timing reduction and the optional all-gather of planes, the
same calls bench.py makes under torchrun with NCCL."""
from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, total, out):
    import datetime

    import torch.distributed as dist

    from b200sht import replicas

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        first, count = replicas.shard_planes(total, rank, world)
        local = torch.arange(first, first + count, dtype=torch.float64)[:, None, None].repeat(1, 2, 3)
        counts = [replicas.shard_planes(total, r, world)[1] for r in range(world)]
        gathered = replicas.gather_planes(local, counts)
        slowest = replicas.max_over_ranks(1.0 + rank)
        replicas.barrier()
        out.put((rank, first, count, gathered[:, 0, 0].tolist(), slowest))
    finally:
        dist.destroy_process_group()


def test_shard_planes_partitions_exactly():
    from b200sht.replicas import shard_planes

    for total in (0, 1, 5, 200, 201):
        for world in (1, 2, 3, 8):
            spans = [shard_planes(total, r, world) for r in range(world)]
            assert sum(c for _, c in spans) == total
            assert [f for f, _ in spans] == [sum(c for _, c in spans[:r]) for r in range(world)]
            assert max(c for _, c in spans) - min(c for _, c in spans) <= 1
    with pytest.raises(ValueError):
        shard_planes(10, 2, 2)


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    world, total = 2, 7
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, total, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [(r, f, c) for r, f, c, _, _ in results] == [(0, 0, 4), (1, 4, 3)]
    for _, _, _, gathered, slowest in results:
        assert gathered == [float(i) for i in range(total)]
        assert slowest == 2.0
