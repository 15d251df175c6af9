"""Particle sharding over ranks (one process per GPU, torch.distributed).

The particle side of a PIC step partitions by particle: every rank pushes its
own particles and deposits them onto the full node vectors; the only exchange
is the sum of the per-rank rho and j (one all-reduce each), after which every
rank holds the global densities (the reference is single-process; its
deposition is a sum over particles, dep_target.hpp:203-273, so any partition
of the particles gives the same sum up to the order of the additions).
"""

from __future__ import annotations


def shard_slice(n: int, rank: int, world: int) -> slice:
    """Contiguous block of particles [start, stop) owned by `rank`."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


def allreduce_densities(rho, j, group=None):
    """Sum rho [Nn] and j [3, Nn] over the ranks, in place (either may be
    None). Every rank must call it, in the same order, once per deposition."""
    import torch.distributed as dist
    for t in (rho, j):
        if t is not None:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return rho, j


def max_over_ranks(value: float, device, group=None) -> float:
    """The largest of the ranks' values (a time, for the slowest rank)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
