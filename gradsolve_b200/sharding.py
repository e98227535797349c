"""Ensemble sharding across GPUs: one process per GPU, trajectories split between ranks.

Trajectories are independent (no coupling anywhere in the forward solve, the record, the
checkpoints or the reverse pass), so a multi-GPU solve is a partition of the batch: each
rank records, checkpoints and differentiates its own trajectories in its own HBM, and the
data path has no collective.  The only cross-rank steps are host-side bookkeeping:

* the step time of a multi-GPU job is the maximum over ranks (``max_over_ranks``);
* a loss that averages over the whole ensemble needs the global count and, for reporting,
  the global sum (``global_sum``) -- 8 bytes, not a data-path exchange;
* uneven batches (per-trajectory horizons, stiff/non-stiff mixes) are balanced by
  assigning trajectories to ranks from estimated costs (``balanced_assignment``), e.g.
  the attempt counts of a forward-only pilot solve.

The reference (gradsolve) is single-device; this module has no counterpart there.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np


def contiguous_slices(n: int, world: int) -> List[Tuple[int, int]]:
    """Split range(n) into ``world`` contiguous slices whose sizes differ by at most one
    (the first ``n % world`` ranks take one extra trajectory)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    if n < 0:
        raise ValueError("n must be >= 0")
    q, r = divmod(n, world)
    out, start = [], 0
    for k in range(world):
        stop = start + q + (1 if k < r else 0)
        out.append((start, stop))
        start = stop
    return out


def balanced_assignment(cost: Sequence[float], world: int) -> List[np.ndarray]:
    """Assign trajectories to ranks so that the summed cost per rank is nearly equal.

    Trajectories are sorted by decreasing cost and dealt to ranks in a serpentine order
    (0, 1, ..., W-1, W-1, ..., 1, 0, 0, 1, ...), which bounds the spread of the per-rank
    sums by the largest single cost.  Each rank's indices are returned sorted ascending,
    so its slice of the inputs keeps the caller's order.  Ties are broken by index, so the
    assignment is deterministic and identical on every rank."""
    c = np.asarray(cost, dtype=np.float64).reshape(-1)
    if world < 1:
        raise ValueError("world must be >= 1")
    if np.any(~np.isfinite(c)) or np.any(c < 0):
        raise ValueError("costs must be finite and non-negative")
    order = np.lexsort((np.arange(c.size), -c))
    cycle = np.concatenate([np.arange(world), np.arange(world)[::-1]])
    owner = cycle[np.arange(c.size) % (2 * world)]
    return [np.sort(order[owner == k]) for k in range(world)]


def rank_and_world(group=None) -> Tuple[int, int]:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def max_over_ranks(x: float, device=None, group=None) -> float:
    """The maximum of a per-rank scalar (a step time) over the process group; the value
    itself when no group is initialised."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def global_sum(x, device=None, group=None):
    """Sum of a per-rank scalar or small tensor over the process group (a loss numerator,
    a trajectory count); the value itself when no group is initialised."""
    import torch
    import torch.distributed as dist
    t = torch.as_tensor(x, dtype=torch.float64, device=device).clone()
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t
