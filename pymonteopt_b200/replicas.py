"""Replicas across GPUs: every rank traces its own photon-id range.

Photons are independent, and a photon's random numbers depend only on
(seed, photon id) through the Philox counter layout. A run of N photons split
into disjoint id ranges, one per rank, therefore traces exactly the photons of
the single run, and the summed tallies are that run's tallies:
- ledger and counters agree up to FP64 summation order;
- histograms agree up to fp32 order;
- the fixed-point absorbed grid agrees exactly.

There is no collective on the data path. The only exchanges are the optional
final sum of the tally buffers and the benchmark's max-over-ranks timing.
These work on any ``torch.distributed`` backend: NCCL for device tensors,
gloo for host tensors.
"""
from __future__ import annotations

from typing import Iterable, Optional

import torch
import torch.distributed as dist

__all__ = ["photon_range", "rank_offset", "reduce_tallies", "max_over_ranks"]


def photon_range(rank: int, world: int, n_photons: int) -> tuple:
    """(begin, count) of rank ``rank``'s share of photons ``[0, n_photons)``:
    contiguous ranges whose sizes differ by at most one."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    base, extra = divmod(int(n_photons), int(world))
    begin = rank * base + min(rank, extra)
    return begin, base + (1 if rank < extra else 0)


def rank_offset(rank: int, photons_per_rank: int, slots: int = 1) -> int:
    """First photon id of ``rank`` when every rank runs ``slots`` launches of
    ``photons_per_rank`` photons (weak scaling): ranks and launches never
    share a photon id."""
    return int(rank) * int(photons_per_rank) * int(slots)


def reduce_tallies(tensors: Iterable[Optional[torch.Tensor]], group=None) -> None:
    """Sum each tally buffer over the ranks, in place (None entries skipped).
    Buffers must have the same shape and dtype on every rank."""
    if not (dist.is_available() and dist.is_initialized()):
        return
    for t in tensors:
        if t is not None:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)


def max_over_ranks(value: float, device=None, group=None) -> float:
    """The maximum of ``value`` over the ranks (the benchmark's timing rule)."""
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
