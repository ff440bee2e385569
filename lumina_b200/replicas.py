"""Replica (data-parallel) execution over independent solve units.

The units of a CDA sweep -- wavelengths, polarisations, clusters -- are
independent solves, so N GPUs run N replicas with no collective on the data
path.  Rank r takes units r, r+N, r+2N, ...  Timing is the maximum over ranks
of each rank's device time, and throughput counts the units all ranks solved.
The only collectives are a barrier and these two reductions.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple


def assign(units: Sequence, rank: int, world: int) -> List:
    """Round-robin share of ``units`` for ``rank`` (disjoint, covering)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} / world {world}")
    return list(units[rank::world])


def rotated(units: Sequence, rank: int, world: int) -> List:
    """Every unit, starting at this rank's share (weak scaling: each rank
    runs the full list, offset so that ranks start on different units)."""
    n = len(units)
    return [units[(rank + i * world) % n] for i in range(n)]


def reduce_job(local_units: float, local_seconds: float, dist=None, device=None) -> Tuple[float, float]:
    """(total units over ranks, max seconds over ranks)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(local_units), float(local_seconds)
    import torch
    u = torch.tensor([float(local_units)], dtype=torch.float64, device=device)
    t = torch.tensor([float(local_seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(u.item()), float(t.item())
