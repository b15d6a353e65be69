"""Chains across GPUs: one process per GPU, chains sharded by rank.

The reference runs one Markov chain per MPI rank and averages each bin over
ranks with MPI_REDUCE (fourier_trans.f90:350-457; pole diagnostics with
MPI_GATHER, pole_diagnostics.f90:158-187).  Here each process owns a
contiguous shard of the job's chains on its GPU; chain c of the job uses row c
of seeds.txt (or block c of confin.txt), exactly as MPI rank c does.  The
per-bin exchange is one all-reduce of the chain-summed bin record (a few
hundred bytes), so the data path has no other collective.
"""
from __future__ import annotations

import numpy as np


def shard(nchains: int, rank: int, world: int) -> tuple[int, int]:
    """(first chain, count) of `rank`'s contiguous share of `nchains` chains."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    base, extra = divmod(nchains, world)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def chain_average(local_sum: np.ndarray, local_count: int, all_reduce) -> np.ndarray:
    """Job-wide chain average of a bin record from per-rank chain sums.

    all_reduce(x) must sum a float64 array over ranks in place and return it
    (torch.distributed.all_reduce on a tensor view, or the identity on one
    rank).  Equivalent to MPI_REDUCE(SUM) followed by division by ISIZE.
    """
    buf = np.concatenate([np.asarray(local_sum, dtype=np.float64).ravel(), [float(local_count)]])
    buf = all_reduce(buf)
    return buf[:-1].reshape(np.shape(local_sum)) / buf[-1]


def torch_all_reduce(group=None, device=None):
    """all_reduce callable over a torch.distributed process group."""
    import torch
    import torch.distributed as dist

    def f(x: np.ndarray) -> np.ndarray:
        t = torch.from_numpy(np.ascontiguousarray(x))
        if device is not None:
            t = t.to(device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        return t.cpu().numpy()

    return f


def gather_rows(local_rows: np.ndarray, group=None) -> np.ndarray:
    """All ranks' per-chain rows in chain order (the MPI_GATHER of the pole files)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    t = torch.from_numpy(np.ascontiguousarray(local_rows, dtype=np.float64))
    n = torch.tensor([t.shape[0]], dtype=torch.int64)
    ns = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(ns, n, group=group)
    m = int(max(int(x) for x in ns))
    pad = torch.zeros((m,) + tuple(t.shape[1:]), dtype=t.dtype)
    pad[: t.shape[0]] = t
    out = [torch.zeros_like(pad) for _ in range(world)]
    dist.all_gather(out, pad, group=group)
    return torch.cat([o[: int(k)] for o, k in zip(out, ns)]).numpy()


def free_port() -> int:
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def _rank_entry(rank, fn, world, port, args):
    import os
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    fn(rank, world, *args)


def launch_ranks(fn, world: int, *args) -> None:
    """Run fn(rank, world, *args) in `world` spawned processes on this node, one
    per GPU, with RANK / LOCAL_RANK / WORLD_SIZE / MASTER_ADDR (127.0.0.1) /
    MASTER_PORT set as torchrun sets them, so that fn may call
    torch.distributed.init_process_group() with the env:// defaults.  Raises if
    any rank fails."""
    import torch.multiprocessing as mp
    mp.start_processes(_rank_entry, args=(fn, world, free_port(), args), nprocs=world, join=True,
                       start_method="spawn")
