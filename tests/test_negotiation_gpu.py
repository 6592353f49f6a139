"""GPU negotiated-congestion rounds against a CPU restatement of the same
Jacobi rip-up-and-reroute loop: per round, the priced oracle search of every
net under the frozen snapshot, with the cells of the net's own previous route
priced from the other nets' usage (the reference removes a net's incumbent
uses before pricing its query, cpu_sequential_negotiated_routing.cc:1023-1034),
per-cell usage of the reached paths, the allocator epoch history update and
the CS-RR next-pass snapshot (price oracle).  Bit-exact usage, history, snapshot prices, per-round overuse and the
last round's costs and canonical paths; the CUDA-graph form replays to the
same result."""

import numpy as np
import pytest

import apgar_b200
import oracle
from apgar_b200 import negotiate, prices, synth
from tests.negotiation_cpu import cpu_rounds

pytestmark = pytest.mark.gpu


def _cpu_rounds(lat, nets, pol, rounds, partial=False):
    return cpu_rounds(lat, nets, pol, rounds, partial)


@pytest.mark.parametrize("partial", [False, True])
@pytest.mark.parametrize("use_graph", [False, True])
def test_rounds_match_cpu_restatement(use_graph, partial):
    lat = synth.make_lattice(61, 2, 128, 0.15, via_mask=True)
    nets = synth.make_nets(lat, 62, 48, hpwl_median=50.0, hpwl_sigma=0.5, margin=12)
    pol = prices.policy(initial=20, increment=20, history_increment=5, capacity=1)
    rounds = 4
    usage_c, history_c, cost_c, costs_c, paths_c, per_round_c = _cpu_rounds(lat, nets, pol, rounds,
                                                                            partial)
    assert per_round_c[0][0] > 0  # the batch is congested in the first round
    dev = apgar_b200.DeviceLattice(lat)
    try:
        plan = dev.plan(nets, generator="frontier")
        neg = negotiate.Negotiation(plan, pol)
        for _ in range(2 if use_graph else 1):  # the second graph run is a replay
            neg.run(rounds, use_graph=use_graph, partial=partial)
            usage, history, cost, rows = neg.readback()
            res, paths = plan.readback()
            assert np.array_equal(usage, usage_c)
            assert np.array_equal(history, history_c)
            assert np.array_equal(cost, cost_c)
            assert [(r["overused_cells"], r["total_overuse"]) for r in rows] == per_round_c
            assert all(r["price_status"] == 0 for r in rows)
            assert np.array_equal(res["cost"], costs_c)
            per = apgar_b200.split_paths(res, paths)
            for i in range(len(nets)):
                if costs_c[i] != oracle.lo_inf():
                    assert np.array_equal(per[i], paths_c[i]), i
        neg.close()
        plan.close()
    finally:
        dev.close()


def test_negotiation_needs_a_frontier_plan():
    lat, nets = synth.config_small(1)
    dev = apgar_b200.DeviceLattice(lat)
    try:
        plan = dev.plan(nets[:4].copy())
        with pytest.raises(ValueError):
            negotiate.Negotiation(plan, prices.policy())
        plan.close()
    finally:
        dev.close()
