"""CPU restatement of one rank's share of the Jacobi negotiated-congestion
loop, in the ROUTE / PRICE steps of the split-round form (test
infrastructure; the oracle's exact search stands in for the GPU search).

ROUTE of round r searches the rank's nets under the frozen snapshot: from
round 1 on, a net's own previous cells are priced from the other nets' usage
(the reference removes a net's incumbent uses before pricing its query,
src/allocator/cpu_sequential_negotiated_routing.cc:1023-1034), and with
partial rip-up only nets that missed their goal or cross a cell overused in
round r - 1 are searched again.  It returns the per-cell usage of the rank's
reached paths.  PRICE of round r takes the usage summed over all ranks: the
allocator epoch history update (src/allocator/negotiated_regeneration_plan.cc
:676-760) and the CS-RR next-pass snapshot (cpu_sequential_negotiated_routing.cc
:299-505), saturated to 2^31 - 1, for the net's view with and without its own
use."""

import numpy as np

import oracle


def snapshot32(usage, history, pol, epoch):
    rc, snap = oracle.price_snapshot(usage, history, pol.capacity, epoch,
                                     pol.initial_present_factor, pol.present_factor_increment,
                                     pol.maximum_value)
    assert rc == 0
    return np.minimum(snap, 0x7FFFFFFF).astype(np.uint32)


class CpuRank:
    def __init__(self, lat, nets, pol):
        self.lat, self.nets, self.pol = lat, nets, pol
        self.cells = lat.layers * lat.height * lat.width
        self.history = np.zeros(self.cells, np.uint64)
        self.cost = np.zeros(self.cells, np.uint32)
        self.cost_own = self.cost
        self.costs = self.paths = None
        self.usage = None  # the last summed usage
        self.per_round = []

    def route(self, r, partial):
        nets = self.nets
        if r == 0:
            self.costs, self.paths = oracle.dijkstra_batch(self.lat, nets, cell_cost=self.cost)
        else:
            if partial:
                idx = [i for i, (c, p) in enumerate(zip(self.costs, self.paths))
                       if c == oracle.lo_inf() or (self.usage[p.astype(np.int64)] > self.pol.capacity).any()]
            else:
                idx = range(len(nets))
            idx = list(idx)
            self.costs = self.costs.copy()
            self.paths = list(self.paths)
            if idx:
                own = [self.paths[i] if self.costs[i] != oracle.lo_inf() else None for i in idx]
                c, p = oracle.dijkstra_batch(self.lat, nets[idx], cell_cost=self.cost,
                                             cell_cost_own=self.cost_own, own=own)
                for k, i in enumerate(idx):
                    self.costs[i] = c[k]
                    self.paths[i] = p[k]
        reached = [p for c, p in zip(self.costs, self.paths) if c != oracle.lo_inf()]
        cells = np.concatenate(reached).astype(np.int64) if reached else np.zeros(0, np.int64)
        return np.bincount(cells, minlength=self.cells).astype(np.uint64)

    def price(self, r, usage):
        pol = self.pol
        self.usage = usage
        rc, _, self.history, _ = oracle.price_epoch_update(
            usage, self.history, pol.capacity, r, pol.initial_present_factor,
            pol.present_factor_increment, pol.historical_price_increment)
        assert rc == 0
        self.cost = snapshot32(usage, self.history, pol, r + 1)
        self.cost_own = snapshot32(np.where(usage > 0, usage - 1, 0).astype(np.uint64),
                                   self.history, pol, r + 1)
        over = np.where(usage > pol.capacity, usage - pol.capacity, 0)
        self.per_round.append((int((over > 0).sum()), int(over.sum())))


def cpu_rounds(lat, nets, pol, rounds, partial=False):
    """One rank over all nets: (usage, history, snapshot, costs, paths,
    per-round (overused cells, total overuse))."""
    rank = CpuRank(lat, nets, pol)
    for r in range(rounds):
        rank.price(r, rank.route(r, partial))
    return (rank.usage.astype(np.uint32), rank.history, rank.cost, rank.costs, rank.paths,
            rank.per_round)
