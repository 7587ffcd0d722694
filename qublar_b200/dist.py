"""Branches of one problem spread over several GPUs (one process per GPU).

Branches are independent (ising_recon.hpp:153-159): rank r anneals a
contiguous range of them on its own GPU with the reference's seed convention
(branch b uses seed b + 1 + seed_offset), so no collective touches the anneal.
The only exchange is the per-bit count of branches with x = 1, summed over
ranks (one all-reduce of n int32) to form the void fractions -- the same float
division as the single-GPU result, hence the same fractions bit for bit.
"""
from __future__ import annotations

import numpy as np


def branch_range(n_branches: int, world: int, rank: int) -> tuple[int, int]:
    """[b0, b1): the branches rank `rank` of `world` anneals (contiguous,
    sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    base, extra = divmod(int(n_branches), int(world))
    b0 = rank * base + min(rank, extra)
    return b0, b0 + base + (1 if rank < extra else 0)


def fractions_from_counts(counts, n_branches: int) -> np.ndarray:
    """branch_fractions' division (ising_recon.hpp:160-163) of exact counts."""
    c = np.asarray(counts)
    return (c.astype(np.float32) / np.float32(n_branches)).astype(np.float32)


def allreduce_counts(local_branches: np.ndarray, group=None) -> np.ndarray:
    """Sum over ranks of the per-bit count of x = 1 (torch.distributed
    all-reduce; NCCL on GPUs, gloo on CPU)."""
    import torch
    import torch.distributed as dist
    cnt = np.asarray(local_branches, dtype=np.uint8).sum(axis=0, dtype=np.int64).astype(np.int32)
    backend = dist.get_backend(group)
    dev = "cuda" if backend == "nccl" else "cpu"
    t = torch.from_numpy(cnt).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def sharded_branch_fractions(problem, schedule, n_branches: int, seed_offset: int = 0, group=None):
    """branch_fractions of one problem with its branches spread over the
    ranks of `group`: each rank solves its range on its current GPU; the
    counts are summed. Returns (fractions, this rank's branches, (b0, b1))."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    b0, b1 = branch_range(n_branches, world, rank)
    if b1 > b0:
        r = problem.solve(schedule, b1 - b0, seed_offset + b0)
        X = r.branches()
        r.close()
    else:
        X = np.zeros((0, problem.n), np.uint8)
    counts = allreduce_counts(X, group)
    return fractions_from_counts(counts, n_branches), X, (b0, b1)
