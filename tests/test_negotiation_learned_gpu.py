"""Negotiated rounds with learned corridor proposals in the priced rounds.

Before every priced round the corridor CNN reads the negotiation's current
snapshot as its congestion raster and proposes each net's corridor; the
priced corridor search certifies a net's route or searches its window again.
Routes, usage, history, prices and per-round overuse must equal the plain
negotiation's bit for bit."""

import numpy as np
import pytest

import apgar_b200
from apgar_b200 import learned, negotiate, prices, synth

pytestmark = pytest.mark.gpu


def _negotiate(lat, nets, pol, rounds, learned_form):
    dev = apgar_b200.DeviceLattice(lat)
    try:
        plan = dev.plan(nets, generator="frontier")
        neg = negotiate.Negotiation(plan, pol)
        status = []
        if learned_form:
            router = learned.LearnedRouter(plan)
            prices_ptr = neg.device_prices()
            for r in range(rounds):
                if r >= 1:
                    router.propose(cell_costs=prices_ptr)
                else:
                    router.clear()
                neg.step(r, neg.ROUTE, partial=True)
                neg.step(r, neg.PRICE, partial=True)
                status.append(plan.corridor_status().copy())
            router.net.check_error()
        else:
            neg.run(rounds, partial=True)
        usage, history, cost, rows = neg.readback()
        res, paths = plan.readback()
        neg.close()
        plan.close()
        return usage, history, cost, rows, res, paths, status
    finally:
        dev.close()


def test_learned_rounds_equal_plain_rounds():
    lat = synth.make_lattice(71, 4, 512, 0.22, pads=True)
    nets = synth.make_nets(lat, 72, 400, hpwl_median=80.0, hpwl_sigma=0.8, margin=32)
    pol = prices.policy(capacity=1)
    rounds = 4
    plain = _negotiate(lat, nets, pol, rounds, False)
    got = _negotiate(lat, nets, pol, rounds, True)
    for a, b, name in zip(plain[:3], got[:3], ("usage", "history", "prices")):
        assert np.array_equal(a, b), name
    assert plain[3] == got[3]
    assert plain[3][0]["overused_cells"] > 0  # congested, so later rounds are priced
    assert np.array_equal(plain[4]["cost"], got[4]["cost"])
    assert np.array_equal(plain[4]["completion"], got[4]["completion"])
    pa = apgar_b200.split_paths(plain[4], plain[5])
    pb = apgar_b200.split_paths(got[4], got[5])
    assert all(np.array_equal(x, y) for x, y in zip(pa, pb))
    status = got[6]
    assert (status[0] == 0).all()  # round 0: no corridor
    # priced rounds: some nets are certified inside their corridor
    assert any((s == 1).any() for s in status[1:])
