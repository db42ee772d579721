"""Host logic of the multi-GPU runs: which views a rank renders, the max over
ranks of a device time, and the whole-job rate.

The frame loop does not shard within a view (spatial reuse needs a halo of
reservoirs, the final-gather endpoint search is global in world space), so N
GPUs run N independent view replicas: weak scaling, no collective on the data
path.  The collectives are the timing reductions here (an all-reduce of one
float per measurement) and, for inverse rendering over views split across
ranks, one all-reduce of the gradient vector per step (sum_gradients), over
NCCL on GPUs or gloo on CPU.
"""
from __future__ import annotations

from typing import List, Optional, Sequence


def orbit_offset(rank: int, world: int, frames: int = 60) -> int:
    """First orbit frame of `rank`: ranks start evenly spaced along the
    `frames`-frame camera orbit, so each renders a different view."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    return rank * frames // world


def assign_views(pixels: Sequence[int], world: int) -> List[List[int]]:
    """Longest-processing-time greedy: views in decreasing pixel count, each to
    the rank with the fewest pixels so far (ties to the lower rank).  Returns
    the view indices of every rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for v in sorted(range(len(pixels)), key=lambda i: (-int(pixels[i]), i)):
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(v)
        load[r] += int(pixels[v])
    return out


def max_over_ranks(value: float, dist=None, device: Optional[str] = None) -> float:
    """Max of `value` over all ranks (identity without a process group).  Every
    rank must call this at the same point."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_gradients(g_mat, g_em, dist=None):
    """Inverse rendering over views split across ranks (assign_views): each rank
    adds its own views' dLoss/dparameter into g_mat (materials x 7) and g_em
    (emitters x 3); this sums them over all ranks in place, as one all-reduce
    of the two flattened into one buffer (992 values for the inverse-rendering
    config's parameters, 321 x 7 + 256 x 3 floats as stored).  Identity
    without a process group.  Every rank must call this at the same point."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return g_mat, g_em
    import torch

    flat = torch.cat([g_mat.reshape(-1), g_em.reshape(-1)])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM)
    n = g_mat.numel()
    g_mat.copy_(flat[:n].view_as(g_mat))
    g_em.copy_(flat[n:].view_as(g_em))
    return g_mat, g_em


def whole_job_rate(units_per_rank_step: float, steps: int, world: int, ms: float) -> float:
    """Units per second of the whole job: all ranks' units over the slowest
    rank's time (`ms`, the max over ranks)."""
    if ms <= 0.0:
        raise ValueError("time must be positive")
    return units_per_rank_step * steps * world / (ms / 1000.0)
