"""Whole-instance placement of an ensemble over GPUs, one process per GPU.

The instances of an ensemble are independent simulations (each its own
grid, electrodes, particles and Poisson system), so an ensemble shards
without any exchange on the data path: each rank builds a
`pic_b200.Ensemble` of the instances placed on it and advances them alone.
The only cross-rank traffic is on the host, before and after the run: the
placement is computed identically on every rank (no message), and the
per-instance results are gathered to rank 0 afterwards.

Placement: longest-processing-time-first greedy on a per-instance weight
(the cell count, which the particle count and the solve cost follow):
instances in decreasing weight order (ties by index) each go to the rank
with the smallest load so far (ties to the lowest rank).  Every rank's load
is then within one instance's weight of every other's.
"""
from __future__ import annotations

from typing import Sequence


def assign(weights: Sequence[float], world: int) -> list[int]:
    """Rank of every instance (same result on every rank)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    if any(w < 0 for w in weights):
        raise ValueError("weights must be non-negative")
    load = [0.0] * world
    rank_of = [0] * len(weights)
    for i in sorted(range(len(weights)), key=lambda i: (-weights[i], i)):
        r = min(range(world), key=lambda r: (load[r], r))
        rank_of[i] = r
        load[r] += weights[i]
    return rank_of


def local(weights: Sequence[float], world: int, rank: int) -> list[int]:
    """The instances placed on `rank`, in increasing index order."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return [i for i, r in enumerate(assign(weights, world)) if r == rank]


def loads(weights: Sequence[float], world: int) -> list[float]:
    out = [0.0] * world
    for i, r in enumerate(assign(weights, world)):
        out[r] += weights[i]
    return out


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def max_over_ranks(x: float) -> float:
    """Max of a host number over the ranks (x itself without a process group)."""
    dist = _dist()
    if dist is None or dist.get_world_size() == 1:
        return float(x)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float) -> float:
    dist = _dist()
    if dist is None or dist.get_world_size() == 1:
        return float(x)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_metrics(mine: dict) -> dict | None:
    """Per-instance results {instance index: metrics} of every rank, on rank
    0 (None elsewhere).  Each instance must be reported by exactly one rank."""
    dist = _dist()
    if dist is None or dist.get_world_size() == 1:
        return dict(mine)
    parts = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(dict(mine), parts, dst=0)
    if dist.get_rank() != 0:
        return None
    out = {}
    for p in parts:
        for k, v in p.items():
            if k in out:
                raise RuntimeError(f"instance {k} reported by two ranks")
            out[k] = v
    return out
