"""Multi-GPU plumbing of the search path: one process per GPU.

Nets are independent within a routing round, so a batch shards by nets with no
data-path collective: every rank searches its own nets over a replicated
lattice (weak scaling).  The only collectives are the timing and count
reductions of a measurement, and, in a negotiated-congestion round, one
integer sum of per-cell usage.  After that sum every rank applies the same
price update locally.  Integer sums are order independent, so every rank sees
identical prices.

Everything here works over any torch.distributed backend (nccl on GPUs, gloo
on CPU for tests).
"""

from __future__ import annotations

import numpy as np

from . import synth


def rank_nets(lat, seed: int, rank: int, count: int) -> np.ndarray:
    """The net batch of one rank: rank 0 gets the canonical medium batch of
    ``seed``; rank r > 0 gets its own seeded batch of the same distribution."""
    if rank == 0:
        return synth.make_nets(lat, seed + 1000, count, hpwl_median=200.0, hpwl_sigma=1.0)
    return synth.make_nets(lat, seed + 1000 + 7919 * rank, count, hpwl_median=200.0,
                           hpwl_sigma=1.0)


def split_nets(nets: np.ndarray, rank: int, world: int) -> np.ndarray:
    """Strong-scaling split of one batch: rank r takes every world-th net
    starting at r (keeps the size mix of the batch on every rank)."""
    return np.ascontiguousarray(nets[rank::world])


def window_work(nets: np.ndarray, layers: int) -> np.ndarray:
    """Estimated search work of each net: its window cells over all layers
    (W x L)."""
    return nets["win_w"].astype(np.int64) * nets["win_h"].astype(np.int64) * int(layers)


def balanced_split(nets: np.ndarray, world: int, layers: int) -> list:
    """Static partition of one batch over ranks by estimated window work:
    longest-processing-time first, each net to the rank with the least work
    so far (ties to the lower rank).  Returns each rank's net indices,
    ascending; every rank computes the same partition."""
    work = window_work(nets, layers)
    order = np.lexsort((np.arange(len(nets)), -work))  # largest first, stable
    loads = np.zeros(world, dtype=np.int64)
    owner = np.empty(len(nets), dtype=np.int64)
    for i in order:
        r = int(np.argmin(loads))
        owner[i] = r
        loads[r] += work[i]
    return [np.flatnonzero(owner == r) for r in range(world)]


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Maximum of a per-rank value (step time) over all ranks."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: int, dist=None, device=None) -> int:
    """Sum of a per-rank count (certified nets) over all ranks."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return int(value)
    import torch

    t = torch.tensor([int(value)], dtype=torch.int64, device=device)
    dist.all_reduce(t)
    return int(t.item())


def allreduce_usage(usage, dist=None):
    """In-place integer sum of a per-cell usage tensor over all ranks (the one
    exchange of a negotiated-congestion round)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return usage
    dist.all_reduce(usage)
    return usage


def negotiate_ranked(negotiation, rounds: int, dist=None, partial: bool = True, stream: int = 0,
                     device: str = "cuda"):
    """Runs one rank's share of a negotiated-congestion run: ``negotiation``
    holds this rank's segments (for example ``split_nets`` of the whole set);
    each round sums the per-cell usage over all ranks with one all-reduce
    (``allreduce_usage``) between the rank's ROUTE and PRICE steps."""
    import torch

    usage = torch.zeros(negotiation.cells, dtype=torch.int32, device=device)
    negotiation.run_ranked(rounds, usage, lambda u: allreduce_usage(u, dist), stream=stream,
                           partial=partial)
    return usage

