"""Host-side multi-rank logic of the projector path (one process per GPU,
torch.distributed).

The path shards without a data exchange when whole frames, studies or
subsets go to different ranks (replicas: `shard`), and has exactly one
exchange when the rays of one subset are split across ranks: the
backprojection is a sum over rays, so each rank backprojects its share and
an all-reduce (sum) of the partial images (and sensitivity images) gives the
subset's backprojection (`allreduce_backprojection`); the EM / PDHG update is
then replicated.  Timing takes the slowest rank (`max_over_ranks`).
"""
from __future__ import annotations


def shard(n, rank, world):
    """Contiguous share [lo, hi) of n units for `rank` of `world`: the first
    n % world ranks take one unit more, so the shares cover 0..n-1 once."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in 0..world-1")
    q, r = divmod(int(n), int(world))
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


def max_over_ranks(values, device=None):
    """Element-wise maximum over ranks of a list of floats (the per-phase
    times of a timed region); the values themselves when not distributed."""
    import torch
    import torch.distributed as dist
    vals = [float(v) for v in values]
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return vals
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def allreduce_backprojection(*images):
    """Sums partial backprojections (and sensitivity images) in place over
    ranks: the one exchange step of a subset whose rays are split across
    ranks.  Every rank calls it with tensors of the same shapes."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return images
    for t in images:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return images
