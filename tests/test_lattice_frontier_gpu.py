"""GPU parity of the lattice frontier generator (bucketed A*) against the CPU
oracle, through the C ABI.

Bit-exact costs and identical canonical reverse paths (reference tie-break)
against full-window exact labels.  The frontier form's own counters (rounds,
expansions) are not compared: they depend on the order of concurrent
relaxations within a round, while costs and paths do not."""

import numpy as np
import pytest

import apgar_b200
import oracle
from apgar_b200 import synth

pytestmark = pytest.mark.gpu


def _route(lat, nets, **kw):
    dev = apgar_b200.DeviceLattice(lat)
    try:
        res, paths = dev.route(nets, generator="frontier", **kw)
    finally:
        dev.close()
    return res, apgar_b200.split_paths(res, paths)


def _assert_parity(lat, nets, **kw):
    res, paths = _route(lat, nets, **kw)
    cost_o, paths_o = oracle.dijkstra_batch(lat, nets)
    admitted = res["completion"] != apgar_b200.COMPLETION_REJECTED
    assert admitted.all()
    assert np.array_equal(res["cost"], cost_o), np.flatnonzero(res["cost"] != cost_o)[:10]
    reached = res["completion"] == apgar_b200.COMPLETION_REACHED
    assert np.array_equal(reached, cost_o != oracle.lo_inf())
    for i in range(len(nets)):
        if reached[i]:
            assert np.array_equal(paths[i], paths_o[i]), i
    return res


@pytest.mark.parametrize("seed", [1, 2])
def test_small_config_parity(seed):
    lat, nets = synth.config_small(seed)
    _assert_parity(lat, nets)


def test_medium_like_parity():
    lat, nets = synth.config_medium(3, nets=160, size=512)
    res = _assert_parity(lat, nets)
    assert (res["sweeps"][res["completion"] == apgar_b200.COMPLETION_REACHED] > 0).all()


@pytest.mark.parametrize("bucket_width", [1, 100, 150, 400, 5000])
def test_bucket_width_does_not_change_results(bucket_width):
    # widths below twice the largest move (100 here) are raised to it
    lat, nets = synth.config_medium(8, nets=48, size=512)
    _assert_parity(lat, nets, bucket_width=bucket_width)


@pytest.mark.parametrize("layers", [1, 2, 3, 6, 8])
def test_layer_counts_and_via_masks(layers):
    lat = synth.make_lattice(20 + layers, layers, 256, 0.2, via_mask=layers > 1)
    nets = synth.make_nets(lat, 30 + layers, 24, hpwl_median=80.0, hpwl_sigma=0.6, margin=24)
    _assert_parity(lat, nets)


def test_every_warp_class():
    # windows from ~10^4 to ~10^7 cells (1 to 16 warps per net)
    lat = synth.make_lattice(41, 4, 2048, 0.18, via_mask=True)
    nets = synth.make_nets(lat, 42, 12, hpwl_median=100.0, hpwl_sigma=0.3, margin=16)
    sizes = [(64, 64), (150, 120), (300, 200), (700, 600), (1500, 1200), (2048, 1200)]
    for i in range(len(nets)):
        w, h = sizes[i % len(sizes)]
        for axis, extent, dim in (("x", w, 2048), ("y", h, 2048)):
            lo = int(min(nets[f"start_{axis}"][i], nets[f"goal_{axis}"][i]))
            hi = int(max(nets[f"start_{axis}"][i], nets[f"goal_{axis}"][i]))
            extent = max(extent, hi - lo + 1)
            o = max(0, min(lo, dim - extent))
            if hi >= o + extent:
                o = hi - extent + 1
            nets[f"win_{axis}0"][i] = o
            nets[f"win_{'w' if axis == 'x' else 'h'}"][i] = extent
    _assert_parity(lat, nets)


def test_disconnected_and_blocked_endpoints():
    dense = np.zeros((2, 64, 64), bool)
    dense[:, :, 30] = True
    dense[0, 5, 5] = True
    lat = synth.Lattice(2, 64, 64, synth.pack_bits(dense), None)
    nets = np.array([
        (0, 2, 3, 1, 60, 5, 0, 0, 64, 64),    # walled: disconnected
        (0, 5, 5, 0, 10, 10, 0, 0, 64, 64),   # blocked start
        (0, 0, 0, 1, 29, 63, 0, 0, 64, 64),   # corner to border
        (1, 63, 63, 0, 31, 0, 31, 0, 33, 64), # window touching the right border
        (0, 7, 7, 0, 7, 7, 0, 0, 64, 64),     # start == goal
    ], dtype=synth.NET_DTYPE)
    res = _assert_parity(lat, nets)
    assert res["completion"][0] == apgar_b200.COMPLETION_DISCONNECTED
    assert res["completion"][1] == apgar_b200.COMPLETION_DISCONNECTED
    assert res["cost"][4] == 0 and res["path_len"][4] == 1


def test_round_budget_is_reported():
    lat, nets = synth.config_small(4)
    res, _ = _route(lat, nets, max_rounds=1)
    far = res["cost"] == apgar_b200.UNREACHABLE
    assert (res["completion"][far] == apgar_b200.COMPLETION_BUDGET_EXHAUSTED).all()
    assert far.sum() > 0


def test_plan_matches_route_and_sweep():
    lat, nets = synth.config_medium(6, nets=96, size=512)
    dev = apgar_b200.DeviceLattice(lat)
    try:
        r_sweep, p_sweep = dev.route(nets)
        r1, p1 = dev.route(nets, generator="frontier")
        plan = dev.plan(nets, generator="frontier")
        for _ in range(2):
            plan.execute()
            r2, p2 = plan.readback()
            assert np.array_equal(r1["cost"], r2["cost"]) and np.array_equal(p1, p2)
            assert np.array_equal(r1["path_offset"], r2["path_offset"])
        plan.close()
        assert np.array_equal(r1["cost"], r_sweep["cost"])
        assert np.array_equal(r1["completion"], r_sweep["completion"])
        assert np.array_equal(p1, p_sweep)
    finally:
        dev.close()


def test_tiny_windows_one_warp_per_net():
    # windows of a few hundred cells (the one-warp class), many nets per CTA
    lat = synth.make_lattice(51, 2, 256, 0.2, via_mask=True)
    nets = synth.make_nets(lat, 52, 200, hpwl_median=10.0, hpwl_sigma=0.4, margin=6)
    assert (2 * nets["win_w"].astype(int) * nets["win_h"] <= 4096).mean() > 0.9
    _assert_parity(lat, nets)


def test_per_cell_prices_match_the_priced_oracle():
    import torch

    rng = np.random.default_rng(77)
    lat, nets = synth.config_medium(5, nets=96, size=512)
    price = rng.integers(0, 60, size=(lat.layers, lat.height, lat.width)).astype(np.uint32)
    price[:, 100:140, :] += 400  # an expensive band that paths route around
    dev = apgar_b200.DeviceLattice(lat)
    try:
        plan = dev.plan(nets, generator="frontier")
        plan.set_cell_costs(torch.from_numpy(price.ravel().view(np.int32)).cuda())
        plan.execute()
        res, paths = plan.readback()
        plan.close()
    finally:
        dev.close()
    cost_o, paths_o = oracle.dijkstra_batch(lat, nets, cell_cost=price)
    assert (res["completion"] != apgar_b200.COMPLETION_REJECTED).all()
    assert np.array_equal(res["cost"], cost_o)
    per = apgar_b200.split_paths(res, paths)
    for i in range(len(nets)):
        if cost_o[i] != oracle.lo_inf():
            assert np.array_equal(per[i], paths_o[i]), i


def test_price_overflow_is_rejected_not_wrong():
    import torch

    lat, nets = synth.config_small(2)
    price = np.full((lat.layers, lat.height, lat.width), 0x3FFFFFFF, np.uint32)
    dev = apgar_b200.DeviceLattice(lat)
    try:
        plan = dev.plan(nets[:8].copy(), generator="frontier")
        plan.set_cell_costs(torch.from_numpy(price.ravel().view(np.int32)).cuda())
        plan.execute()
        res, _ = plan.readback()
        plan.close()
    finally:
        dev.close()
    # two entries already pass 2^31: every net with a path of 2+ moves is rejected
    moved = (nets["start_x"][:8] != nets["goal_x"][:8]) | (nets["start_y"][:8] != nets["goal_y"][:8])
    assert (res["completion"][moved] == apgar_b200.COMPLETION_REJECTED).all()


@pytest.mark.parametrize("chain", [1, 2, 4, 9, 16])
def test_chained_expansions_do_not_change_results(chain):
    # chain n: up to n - 1 chained expansions per queued cell in every class
    lat, nets = synth.config_medium(10, nets=64, size=640)
    _assert_parity(lat, nets, chain=chain)


def test_chain_above_sixteen_is_refused():
    lat, nets = synth.config_small(1)
    with pytest.raises(apgar_b200.BackendError):
        _route(lat, nets[:4].copy(), chain=17)


def test_slot_workspace_gives_the_per_net_results(monkeypatch):
    """The persistent slot workspace (used when per-net slabs exceed their
    budget), with its full slot count and with slots cut to fit a small
    budget, gives exactly the per-net workspace's (and the oracle's) costs
    and paths."""
    lat = synth.make_lattice(51, 2, 512, 0.2, pads=True)
    nets = synth.make_nets(lat, 52, 300, hpwl_median=120.0, hpwl_sigma=1.0)
    cost_o, paths_o = oracle.dijkstra_batch(lat, nets)
    dev = apgar_b200.DeviceLattice(lat)
    try:
        outs = []
        for per_net, slot in ((None, None), ("1", None), ("1", str(64 << 20))):
            if per_net is not None:
                monkeypatch.setenv("APGAR_B200_FRONTIER_PER_NET_BYTES", per_net)
            if slot is not None:
                monkeypatch.setenv("APGAR_B200_FRONTIER_SLOT_BYTES", slot)
            plan = dev.plan(nets, generator="frontier")
            plan.execute()
            res, paths = plan.readback()
            outs.append((res, paths, plan.info()["workspace_bytes"]))
            plan.close()
        monkeypatch.delenv("APGAR_B200_FRONTIER_PER_NET_BYTES")
        monkeypatch.delenv("APGAR_B200_FRONTIER_SLOT_BYTES")
        assert len({w for _, _, w in outs}) == 3  # three different workspaces
        assert outs[2][2] < outs[1][2]
        for res, paths, _ in outs:
            assert (res["completion"] != apgar_b200.COMPLETION_REJECTED).all()
            assert np.array_equal(res["cost"], cost_o)
            per = apgar_b200.split_paths(res, paths)
            for i in range(len(nets)):
                if cost_o[i] != oracle.lo_inf():
                    assert np.array_equal(per[i], paths_o[i]), i
    finally:
        dev.close()
