"""Rank plumbing for one process per GPU (torch.distributed: NCCL on the GPUs, gloo in the CPU
tests). The single-problem Newton step does not shard in this build: N ranks run N replicas and
the job's time is the slowest rank's. The batched form shards naturally: its instances are
split over the ranks with no collective on the data path."""
from __future__ import annotations

import os


def world_info():
    """(rank, local_rank, world_size) from the launcher's environment (torchrun)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def max_over_ranks(value: float, device="cpu") -> float:
    """The largest value over all ranks (the job's time is its slowest rank's); the value itself
    without an initialised process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(n: int, rank: int, world: int) -> range:
    """Contiguous, balanced share of n items for `rank` (sizes differ by at most one)."""
    q, r = divmod(n, world)
    lo = rank * q + min(rank, r)
    return range(lo, lo + q + (1 if rank < r else 0))


def shard_by_cost(costs, world: int):
    """Items split over ranks largest first, each to the least-loaded rank (LPT); returns the
    sorted item indices of every rank. Deterministic: ties go to the lower rank and item."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        k = min(range(world), key=lambda w: (load[w], w))
        parts[k].append(i)
        load[k] += costs[i]
    return [sorted(p) for p in parts]


def batched_share(problems, rank: int, world: int, ctx, schedule=None, coarse_slabs: int = 0, **solver_opts):
    """This rank's share of independent instances (LPT by element count) as one batched solver.
    Ranks exchange nothing on the data path: each solves its own instances; the caller gathers
    results or times. schedule: (cluster, threads), or None to autotune on the share's
    tangent at u = 0, lambda = 0.2. Returns (instance ids of this rank, BatchGpu)."""
    from . import api
    mine = shard_by_cost([q.n_elem for q in problems], world)[rank]
    b = api.BatchGpu([problems[i] for i in mine], ctx, **solver_opts)
    b.set_coarse(coarse_slabs)
    if schedule is not None:
        b.set_schedule(*schedule)
    else:
        import numpy as np
        import torch
        u = b.union
        b.solver.calcStiffnessAndResidual(torch.zeros(u.n_dof, dtype=torch.float64, device=f"cuda:{ctx.device}"))
        b.solver.addExternalForces(torch.tensor(np.asarray(u.fnodal), device=f"cuda:{ctx.device}"), 0.2)
        b.autotune(maxit=0)
    return mine, b
