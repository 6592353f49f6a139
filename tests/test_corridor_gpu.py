"""GPU corridor mode of the frontier generator, through the C ABI.

Results never depend on the corridor: every net's cost and canonical path
equal the full-window oracle's, whether its corridor result was certified or
it fell back to the whole window.  Each net's corridor outcome equals the CPU
restatement of the certificate (oracle.corridor_certificate)."""

import numpy as np
import pytest
import torch

import apgar_b200
import oracle
from apgar_b200 import corridor, synth

pytestmark = pytest.mark.gpu


def _run(lat, nets, masks, cell_cost=None):
    dev = apgar_b200.DeviceLattice(lat)
    try:
        plan = dev.plan(nets, generator="frontier")
        bits = torch.from_numpy(corridor.pack(masks).view(np.int32)).cuda().view(torch.uint32)
        plan.set_corridors(bits)
        if cell_cost is not None:
            prices = torch.from_numpy(cell_cost.view(np.int32)).cuda().view(torch.uint32)
            plan.set_cell_costs(prices)
        plan.execute()
        res, paths = plan.readback()
        status = plan.corridor_status()
        plan.close()
    finally:
        dev.close()
    return res, apgar_b200.split_paths(res, paths), status


def _check(lat, nets, masks, cell_cost=None):
    res, paths, status = _run(lat, nets, masks, cell_cost)
    cost_o, paths_o = oracle.dijkstra_batch(lat, nets, cell_cost=cell_cost)
    assert (res["completion"] != apgar_b200.COMPLETION_REJECTED).all()
    assert np.array_equal(res["cost"], cost_o), np.flatnonzero(res["cost"] != cost_o)[:10]
    for i in range(len(nets)):
        if cost_o[i] != oracle.lo_inf():
            assert np.array_equal(paths[i], paths_o[i]), i
    want = np.array([oracle.corridor_certificate(lat, nets[i], masks[i], cell_cost)[0]
                     for i in range(len(nets))])
    assert np.array_equal(status, want), (np.flatnonzero(status != want)[:10], status[:10], want[:10])
    return status


def _case(seed, count=48, layers=2, size=192):
    lat = synth.make_lattice(seed, layers, size, 0.22, via_mask=True)
    nets = synth.make_nets(lat, seed + 1, count, hpwl_median=60.0, hpwl_sigma=0.7, margin=16)
    return lat, nets


def test_full_corridor_certifies_everything():
    lat, nets = _case(21)
    status = _check(lat, nets, corridor.full_corridor(len(nets)))
    assert (status == corridor.CERTIFIED).all()


def test_empty_corridor_is_no_proposal():
    lat, nets = _case(22, 24)
    status = _check(lat, nets, np.zeros((len(nets), 64, 64), bool))
    assert (status == corridor.NONE).all()


def test_corridor_missing_a_terminal_falls_back():
    lat, nets = _case(27, 24)
    masks = corridor.full_corridor(len(nets))
    for i, n in enumerate(nets):  # drop the start's coarse cell only
        s = corridor.coarse_shift(int(n["win_w"]), int(n["win_h"]))
        masks[i, (int(n["start_y"]) - int(n["win_y0"])) >> s, (int(n["start_x"]) - int(n["win_x0"])) >> s] = False
    status = _check(lat, nets, masks)
    assert (status == corridor.FALLBACK_UNREACHED).all()


@pytest.mark.parametrize("radius", [0, 1, 2])
def test_segment_corridors_mixed_outcomes(radius):
    lat, nets = _case(23 + radius, 64, layers=3)
    rng = np.random.default_rng(radius)
    masks = corridor.segment_corridor(nets, radius) & (rng.random((len(nets), 64, 64)) < 0.95)
    status = _check(lat, nets, masks)
    assert (status == corridor.CERTIFIED).any()


def test_corridor_mode_on_medium_windows():
    # windows of several coarse scales and every warp class
    lat, nets = synth.config_medium(9, nets=96, size=768)
    masks = corridor.segment_corridor(nets, 2)
    status = _check(lat, nets, masks)
    assert (status == corridor.CERTIFIED).mean() > 0.3


def test_repeated_executions_do_not_read_stale_labels():
    # corridor passes never clear cells outside the corridor; a second
    # execution with a different corridor must still match the oracle
    lat, nets = _case(27, 32)
    dev = apgar_b200.DeviceLattice(lat)
    try:
        plan = dev.plan(nets, generator="frontier")
        plan.execute()  # full windows first: every slab holds labels
        for radius in (3, 0):
            masks = corridor.segment_corridor(nets, radius)
            bits = torch.from_numpy(corridor.pack(masks).view(np.int32)).cuda().view(torch.uint32)
            plan.set_corridors(bits)
            plan.execute()
            res, paths = plan.readback()
            cost_o, paths_o = oracle.dijkstra_batch(lat, nets)
            assert np.array_equal(res["cost"], cost_o)
            per = apgar_b200.split_paths(res, paths)
            for i in range(len(nets)):
                if cost_o[i] != oracle.lo_inf():
                    assert np.array_equal(per[i], paths_o[i]), (radius, i)
        plan.close()
    finally:
        dev.close()


@pytest.mark.parametrize("radius", [1, 2])
def test_priced_corridors_match_the_priced_oracle(radius):
    """Corridor mode under per-cell entry prices (the negotiated rounds'
    snapshot): costs and canonical paths equal the priced full-window oracle,
    and each outcome equals the priced certificate restatement."""
    lat, nets = _case(31 + radius, 64, layers=3)
    rng = np.random.default_rng(40 + radius)
    cells = lat.layers * lat.height * lat.width
    # sparse congestion prices, as a negotiation's snapshot has them
    cell_cost = np.where(rng.random(cells) < 0.15, rng.integers(1, 120, cells), 0).astype(np.uint32)
    masks = corridor.segment_corridor(nets, radius) & (rng.random((len(nets), 64, 64)) < 0.95)
    status = _check(lat, nets, masks, cell_cost)
    assert (status == corridor.CERTIFIED).any()
