"""GPU parity of lattice mode against the CPU oracle, through the C ABI.

Bit-exact: costs, reverse canonical paths (reference tie-break), and the
per-net schedule counters (sweeps, row steps, row stores) against the CPU
restatement of the same sweep schedule."""

import numpy as np
import pytest

import apgar_b200
import oracle
from apgar_b200 import synth

pytestmark = pytest.mark.gpu


def _gpu_route(lat, nets, max_sweeps=4096):
    dev = apgar_b200.DeviceLattice(lat)
    try:
        res, paths = dev.route(nets, max_sweeps=max_sweeps)
    finally:
        dev.close()
    return res, apgar_b200.split_paths(res, paths)


def _assert_parity(lat, nets, check_counters=True):
    res, paths = _gpu_route(lat, nets)
    cost_o, paths_o = oracle.dijkstra_batch(lat, nets)
    cs, st = oracle.sweep_batch(lat, nets)
    assert np.array_equal(cost_o, cs)
    reached = res["completion"] == apgar_b200.COMPLETION_REACHED
    assert np.array_equal(res["cost"], cost_o), np.flatnonzero(res["cost"] != cost_o)[:10]
    assert np.array_equal(reached, cost_o != oracle.lo_inf())
    for i in range(len(nets)):
        if reached[i]:
            assert np.array_equal(paths[i], paths_o[i]), i
    if check_counters:
        admitted = res["completion"] != apgar_b200.COMPLETION_REJECTED
        endpoints_ok = st[:, 0] > 0
        sel = admitted & endpoints_ok
        assert np.array_equal(res["sweeps"][sel], st[sel, 0].astype(np.uint32))
        assert np.array_equal(res["row_steps"][sel], st[sel, 1].astype(np.uint32))
        assert np.array_equal(res["row_stores"][sel], st[sel, 2].astype(np.uint32))
        assert np.array_equal(res["row_loads"][sel], st[sel, 5].astype(np.uint32))
    return res


@pytest.mark.parametrize("seed", [1, 2])
def test_small_config_parity(seed):
    lat, nets = synth.config_small(seed)
    _assert_parity(lat, nets)


def test_medium_like_parity():
    lat, nets = synth.config_medium(3, nets=160, size=512)
    _assert_parity(lat, nets)


def test_every_width_class_and_via_mask():
    lat = synth.make_lattice(11, 3, 2048, 0.18, via_mask=True)
    rng = np.random.default_rng(5)
    nets = synth.make_nets(lat, 12, 40, hpwl_median=60.0, hpwl_sigma=0.5, margin=16)
    # widen windows to hit every class (<=128, 256, 512, 1024, 2048 cells)
    widths = [100, 200, 400, 900, 2048]
    for i in range(len(nets)):
        w = widths[i % len(widths)]
        x_lo = int(min(nets["start_x"][i], nets["goal_x"][i]))
        x_hi = int(max(nets["start_x"][i], nets["goal_x"][i]))
        x0 = int(max(0, min(x_lo, 2048 - w)))
        if x_hi >= x0 + w:
            x0 = int(x_hi - w + 1)
        nets["win_x0"][i] = x0
        nets["win_w"][i] = w
        y_lo = int(min(nets["start_y"][i], nets["goal_y"][i]))
        y_hi = int(max(nets["start_y"][i], nets["goal_y"][i]))
        y0 = max(0, y_lo - int(rng.integers(0, 20)))
        top = min(2047, y_hi + int(rng.integers(1, 20)))
        nets["win_y0"][i] = y0
        nets["win_h"][i] = top + 1 - y0
    _assert_parity(lat, nets)


def test_disconnected_blocked_endpoints_and_borders():
    dense = np.zeros((2, 64, 64), bool)
    dense[:, :, 30] = True
    dense[0, 5, 5] = True
    lat = synth.Lattice(2, 64, 64, synth.pack_bits(dense), None)
    nets = np.array([
        (0, 2, 3, 1, 60, 5, 0, 0, 64, 64),    # walled: disconnected
        (0, 5, 5, 0, 10, 10, 0, 0, 64, 64),   # blocked start
        (0, 0, 0, 1, 29, 63, 0, 0, 64, 64),   # corner to border
        (1, 63, 63, 0, 31, 0, 31, 0, 33, 64), # window touching the right border
    ], dtype=synth.NET_DTYPE)
    res = _assert_parity(lat, nets)
    assert res["completion"][0] == apgar_b200.COMPLETION_DISCONNECTED
    assert res["completion"][1] == apgar_b200.COMPLETION_DISCONNECTED


def test_budget_exhaustion_and_rejection():
    lat, nets = synth.config_small(4)
    res, _ = _gpu_route(lat, nets, max_sweeps=1)
    assert (res["completion"] == apgar_b200.COMPLETION_BUDGET_EXHAUSTED).all()
    bad = nets[:2].copy()
    bad["win_w"][0] = 10_000  # window outside the lattice
    res, _ = _gpu_route(lat, bad)
    assert res["completion"][0] == apgar_b200.COMPLETION_REJECTED
    assert res["completion"][1] == apgar_b200.COMPLETION_REACHED


def test_repeatable_and_plan_matches_route():
    lat, nets = synth.config_medium(6, nets=96, size=512)
    dev = apgar_b200.DeviceLattice(lat)
    r1, p1 = dev.route(nets)
    r2, p2 = dev.route(nets)
    plan = dev.plan(nets)
    plan.execute()
    r3, p3 = plan.readback()
    plan.execute()
    r4, p4 = plan.readback()
    for r, p in ((r2, p2), (r3, p3), (r4, p4)):
        assert np.array_equal(r1, r) and np.array_equal(p1, p)
    plan.close()
    dev.close()
