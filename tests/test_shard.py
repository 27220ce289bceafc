"""Scenario sharding over ranks and the whole-job combination, with two gloo ranks
on the CPU (the multi-GPU ensemble path has no data-path collective)."""
import os
import socket

import numpy as np
import pytest

from storm_b200 import shard


def test_lpt_shards_cover_every_scenario_once_and_balance():
    rng = np.random.default_rng(0)
    sizes = np.exp(rng.uniform(np.log(20_000), np.log(400_000), size=256)).astype(int)
    for world in (1, 2, 4, 8):
        shares = shard.lpt_shards(sizes, world)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(256))
        assert all(s == sorted(s) for s in shares)
        assert shard.imbalance(sizes, shares) < 1.02
    assert shard.lpt_shards([5, 5, 5], 2) == [[0, 2], [1]]
    with pytest.raises(ValueError):
        shard.lpt_shards([1], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, sizes, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard.lpt_shards(sizes, world)[rank]
        local = {"cell_stages": float(3 * sum(sizes[i] for i in mine)), "device_ms": 10.0 + rank,
                 "scenarios": len(mine), "converged": len(mine) - (1 if rank == 1 else 0)}
        tot = shard.combine(local, dist)
        out.put((rank, mine, tot))
    finally:
        dist.destroy_process_group()


def test_two_rank_combination_over_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    sizes = [30_000, 120_000, 45_000, 400_000, 22_000, 90_000, 61_000]
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    shares = [r[1] for r in res]
    assert sorted(shares[0] + shares[1]) == list(range(len(sizes)))
    for _, _, tot in res:
        assert tot["cell_stages"] == 3.0 * sum(sizes)
        assert tot["device_ms"] == 11.0  # the slowest rank
        assert tot["scenarios"] == len(sizes) and tot["converged"] == len(sizes) - 1
