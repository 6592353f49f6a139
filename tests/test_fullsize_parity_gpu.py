"""Parity at the benchmarked sizes, against the oracle.

* The medium configuration exactly as the bench runs it (4 layers of
  2048 x 2048, 25% blocked, 4096 nets, seed 2): the plain sweep, the
  persistent frontier and the learned-corridor form each return every net's
  cost and canonical path equal to the oracle's exact Dijkstra
  (``oracle.dijkstra_batch``), net for net.
* The negotiated configuration's lattice (6 layers of 4096 x 4096, 25%
  blocked) with a seeded 2048-segment share of its multi-terminal nets: round
  0 and one priced round with partial rip-up, bit-exact against the CPU
  restatement of the same Jacobi rounds (usage, history, snapshot prices,
  per-round overuse, the last round's costs and canonical paths).
"""

import numpy as np
import pytest

import apgar_b200
import oracle
from apgar_b200 import negotiate, prices, synth
from tests.negotiation_cpu import cpu_rounds

pytestmark = pytest.mark.gpu

PATH_CAP = 1 << 15


@pytest.fixture(scope="module")
def medium():
    lat, nets = synth.config_medium()
    costs, paths = oracle.dijkstra_batch(lat, nets, path_cap_per_net=PATH_CAP)
    assert all(p is not None for c, p in zip(costs, paths) if c != oracle.lo_inf())
    dev = apgar_b200.DeviceLattice(lat)
    yield lat, nets, costs, paths, dev
    dev.close()


def _same_as_oracle(results, packed, costs, paths):
    assert np.array_equal(results["cost"], costs)
    per = apgar_b200.split_paths(results, packed)
    bad = [i for i in range(len(costs))
           if costs[i] != oracle.lo_inf() and not np.array_equal(per[i], paths[i])]
    assert not bad, f"{len(bad)} canonical paths differ, first at net {bad[0]}"
    reached = int((costs != oracle.lo_inf()).sum())
    assert reached > 0.9 * len(costs)
    return reached


@pytest.mark.parametrize("generator", ["sweep", "frontier"])
def test_medium_batch_every_path_equals_the_oracle(medium, generator):
    lat, nets, costs, paths, dev = medium
    results, packed = dev.route(nets, generator=generator)
    _same_as_oracle(results, packed, costs, paths)


def test_medium_batch_learned_form_every_path_equals_the_oracle(medium):
    from apgar_b200 import learned

    lat, nets, costs, paths, dev = medium
    plan = dev.plan(nets, generator="frontier")
    try:
        router = learned.LearnedRouter(plan)
        router.execute()
        router.net.check_error()
        results, packed = plan.readback()
        _same_as_oracle(results, packed, costs, paths)
        status = plan.corridor_status()
        assert (status == 1).mean() > 0.5  # most nets certified inside their corridor
    finally:
        plan.close()


def test_negotiated_lattice_rounds_equal_the_cpu_restatement():
    lat, segs, _ = synth.config_negotiated()
    rng = np.random.default_rng(2048)
    segs = np.ascontiguousarray(segs[np.sort(rng.choice(len(segs), 2048, replace=False))])
    pol = prices.policy(capacity=1)
    rounds = 2
    usage_c, history_c, cost_c, costs_c, paths_c, per_round_c = cpu_rounds(
        lat, segs, pol, rounds, partial=True)
    assert per_round_c[0][0] > 0  # congested in round 0, so round 1 is priced
    dev = apgar_b200.DeviceLattice(lat)
    try:
        plan = dev.plan(segs, generator="frontier")
        neg = negotiate.Negotiation(plan, pol)
        neg.run(rounds, use_graph=True, partial=True)
        usage, history, cost, rows = neg.readback()
        res, packed = plan.readback()
        assert [(r["overused_cells"], r["total_overuse"]) for r in rows] == per_round_c
        assert all(r["price_status"] == 0 for r in rows)
        assert np.array_equal(usage, usage_c)
        assert np.array_equal(history, history_c)
        assert np.array_equal(cost, cost_c)
        assert np.array_equal(res["cost"], costs_c)
        per = apgar_b200.split_paths(res, packed)
        bad = [i for i in range(len(segs))
               if costs_c[i] != oracle.lo_inf() and not np.array_equal(per[i], paths_c[i])]
        assert not bad, f"{len(bad)} canonical paths differ, first at segment {bad[0]}"
        neg.close()
        plan.close()
    finally:
        dev.close()
