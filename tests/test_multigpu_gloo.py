"""Host logic of the multi-process path on CPU with gloo (world_size 2).

Checks that chains shard exactly as MPI ranks would (chain c uses seeds row
c), that the cross-rank bin average equals MPI_REDUCE(SUM)/ISIZE over all
chains, and that the per-chain gather keeps chain order.
"""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from bafqmc_b200.multigpu import chain_average, shard


def test_shard_covers_all_chains_in_order():
    for n in (1, 7, 8, 4096, 4099):
        for world in (1, 2, 3, 8):
            if world > n:
                continue
            parts = [shard(n, r, world) for r in range(world)]
            assert parts[0][0] == 0
            for (s0, c0), (s1, _) in zip(parts, parts[1:]):
                assert s0 + c0 == s1
            assert sum(c for _, c in parts) == n
            assert max(c for _, c in parts) - min(c for _, c in parts) <= 1


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from bafqmc_b200.multigpu import chain_average, gather_rows, shard, torch_all_reduce
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        nchains, width = 5, 30
        rng = np.random.default_rng(1234)
        per_chain = rng.standard_normal((nchains, width))   # same table on every rank
        start, count = shard(nchains, rank, world)
        mine = per_chain[start:start + count]
        avg = chain_average(mine.sum(axis=0), count, torch_all_reduce())
        rows = gather_rows(mine)
        out[rank] = (avg, rows)
    finally:
        dist.destroy_process_group()


def test_two_rank_reduce_and_gather_match_single_process():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = 29500 + os.getpid() % 1000
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    rng = np.random.default_rng(1234)
    per_chain = rng.standard_normal((5, 30))
    expect = per_chain.sum(axis=0) / 5.0
    for r in (0, 1):
        avg, rows = out[r]
        np.testing.assert_allclose(avg, expect, rtol=1e-15, atol=1e-15)
        np.testing.assert_array_equal(rows, per_chain)


def test_single_rank_average_is_plain_mean():
    x = np.arange(12.0).reshape(3, 4)
    np.testing.assert_allclose(chain_average(x.sum(axis=0), 3, lambda b: b), x.mean(axis=0))


def _launched(rank, world, out):
    import torch
    import torch.distributed as dist
    from bafqmc_b200.multigpu import chain_average, shard, torch_all_reduce
    dist.init_process_group("gloo")   # env:// from the launcher, as bench.py's ranks do with NCCL
    try:
        assert dist.get_rank() == rank and dist.get_world_size() == world
        assert int(os.environ["LOCAL_RANK"]) == rank and os.environ["MASTER_ADDR"] == "127.0.0.1"
        nchains = 4099
        start, count = shard(nchains, rank, world)
        local = np.arange(start, start + count, dtype=np.float64)
        t = torch.tensor([float(count)])
        dist.all_reduce(t)
        out[rank] = (start, count, float(t.item()), chain_average(np.array([local.sum()]), count, torch_all_reduce()))
    finally:
        dist.destroy_process_group()


def test_launcher_spawns_ranks_like_torchrun():
    """bench.py --gpus N without torchrun uses multigpu.launch_ranks: each spawned
    rank sees the torchrun environment, takes its shard of the job's chains and
    joins the per-bin reduction."""
    from bafqmc_b200.multigpu import launch_ranks
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    launch_ranks(_launched, 3, out)
    assert sorted(out.keys()) == [0, 1, 2]
    assert sum(out[r][1] for r in range(3)) == 4099
    for r in range(3):
        assert out[r][2] == 4099.0
        np.testing.assert_allclose(out[r][3], [np.arange(4099).mean()], rtol=1e-14)
