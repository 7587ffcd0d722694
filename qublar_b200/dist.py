"""Branches of one problem spread over several GPUs (one process per GPU).

Branches are independent (ising_recon.hpp:153-159): rank r anneals a
contiguous range of them on its own GPU with the reference's seed convention
(branch b uses seed b + 1 + seed_offset), so no collective touches the anneal.
A range starts on a multiple of the kind's draw granule (integer Ising: pairs
of replicas share a Philox key; weighted QUBO: launches of 64 replicas do), so
a rank's solve with seed_offset + b0 draws what the single solve draws.
The only exchange is the per-bit count of branches with x = 1, summed over
ranks (one all-reduce of n int32) to form the void fractions -- the same float
division as the single-GPU result, hence the same fractions bit for bit.
"""
from __future__ import annotations

import numpy as np


def branch_range(n_branches: int, world: int, rank: int, granule: int = 1) -> tuple[int, int]:
    """[b0, b1): the branches rank `rank` of `world` anneals: contiguous, b0 a
    multiple of `granule`, the counts of whole granules differing by at most
    one."""
    if world < 1 or not 0 <= rank < world or granule < 1:
        raise ValueError("bad world/rank/granule")
    units = -(-int(n_branches) // int(granule))
    base, extra = divmod(units, int(world))
    u0 = rank * base + min(rank, extra)
    u1 = u0 + base + (1 if rank < extra else 0)
    return min(u0 * granule, int(n_branches)), min(u1 * granule, int(n_branches))


def draw_granule(problem) -> int:
    """Branches per Philox key group of the problem's kind: 2 for integer
    Ising (replicas 2k, 2k + 1), 64 for the weighted QUBO (a launch of 64
    replicas), 1 for residual problems."""
    from . import KIND_ISING, KIND_QUBO
    return {KIND_ISING: 2, KIND_QUBO: 64}.get(int(problem.kind), 1)


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
    b0, b1 = branch_range(n_branches, world, rank, draw_granule(problem))
    if b1 > b0:
        r = problem.solve(schedule, b1 - b0, seed_offset + b0)
        X = r.branches()
        r.close()
    else:
        X = np.zeros((0, problem.n), np.uint8)
    counts = allreduce_counts(X, group)
    return fractions_from_counts(counts, n_branches), X, (b0, b1)
