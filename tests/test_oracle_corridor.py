"""CPU checks of the corridor certificate restatement (oracle.corridor_certificate):
soundness against the full-window oracle on seeded lattices and corridors,
and the corridor helpers' bitmap layout."""

import numpy as np
import pytest

import oracle
from apgar_b200 import corridor, synth


def _case(seed, count=24):
    lat = synth.make_lattice(seed, 2, 160, 0.22, via_mask=True)
    nets = synth.make_nets(lat, seed + 1, count, hpwl_median=50.0, hpwl_sigma=0.6, margin=12)
    return lat, nets


def test_pack_roundtrip_and_layout():
    rng = np.random.default_rng(5)
    masks = rng.random((3, 64, 64)) < 0.3
    words = corridor.pack(masks)
    assert words.shape == (3, 128) and words.dtype == np.uint32
    assert np.array_equal(corridor.unpack(words), masks)
    # bit cx % 32 of word 2 * cy + cx // 32
    one = np.zeros((1, 64, 64), bool)
    one[0, 7, 37] = True
    w = corridor.pack(one)[0]
    assert np.flatnonzero(w).tolist() == [2 * 7 + 1] and w[15] == 1 << (37 - 32)


@pytest.mark.parametrize("w,h,s", [(1, 1, 2), (252, 10, 2), (253, 10, 3), (256, 10, 3),
                                   (512, 600, 4), (2016, 9, 5), (2017, 9, 6)])
def test_coarse_shift(w, h, s):
    assert corridor.coarse_shift(w, h) == s
    assert -(-max(w, h) // (1 << s)) <= 63


@pytest.mark.parametrize("seed", [11, 12])
def test_certificate_is_sound(seed):
    lat, nets = _case(seed)
    cost_full, paths_full = oracle.dijkstra_batch(lat, nets)
    rng = np.random.default_rng(seed)
    seen = set()
    for radius in (0, 1, 3):
        masks = corridor.segment_corridor(nets, radius)
        masks &= rng.random(masks.shape) < 0.97  # knock a few coarse cells out
        for i in range(len(nets)):
            status, cost, bound = oracle.corridor_certificate(lat, nets[i], masks[i])
            seen.add(status)
            if status == oracle.CORRIDOR_CERTIFIED and cost is not None:
                assert cost == cost_full[i]
                _, path, _ = oracle.dijkstra(lat, nets[i], cell_cost=_priced_out(lat, nets[i], masks[i]))
                assert np.array_equal(path, paths_full[i]), i
            if status == oracle.CORRIDOR_FALLBACK_EXIT:
                assert bound is not None and bound <= cost
    assert oracle.CORRIDOR_CERTIFIED in seen
    assert seen - {oracle.CORRIDOR_CERTIFIED}


def test_full_corridor_always_certifies():
    lat, nets = _case(13, 16)
    masks = corridor.full_corridor(len(nets))
    for i in range(len(nets)):
        status, _, bound = oracle.corridor_certificate(lat, nets[i], masks[i])
        assert status == oracle.CORRIDOR_CERTIFIED and bound is None


def test_empty_corridor_is_no_proposal_and_a_missing_terminal_falls_back():
    lat, nets = _case(14, 8)
    masks = np.zeros((len(nets), 64, 64), bool)
    for i in range(len(nets)):
        assert oracle.corridor_certificate(lat, nets[i], masks[i])[0] == oracle.CORRIDOR_NONE
    masks = np.ones((len(nets), 64, 64), bool)
    for i, n in enumerate(nets):
        s = corridor.coarse_shift(int(n["win_w"]), int(n["win_h"]))
        masks[i, (int(n["goal_y"]) - int(n["win_y0"])) >> s, (int(n["goal_x"]) - int(n["win_x0"])) >> s] = False
        assert oracle.corridor_certificate(lat, nets[i], masks[i])[0] == \
            oracle.CORRIDOR_FALLBACK_UNREACHED


def _priced_out(lat, net, mask):
    w, h = int(net["win_w"]), int(net["win_h"])
    x0, y0 = int(net["win_x0"]), int(net["win_y0"])
    s = corridor.coarse_shift(w, h)
    inside = mask[(np.arange(h) >> s)[:, None], (np.arange(w) >> s)[None, :]]
    price = np.zeros((lat.layers, lat.height, lat.width), np.uint32)
    price[:, y0:y0 + h, x0:x0 + w][:, ~inside] = 1 << 30
    return price.reshape(-1)


@pytest.mark.parametrize("seed", [15, 16])
def test_priced_certificate_is_sound(seed):
    """Under non-negative entry prices (a negotiated round's snapshot) a
    certified corridor cost is the priced full-window optimum and its path the
    priced canonical path."""
    lat, nets = _case(seed)
    rng = np.random.default_rng(seed + 7)
    cells = lat.layers * lat.height * lat.width
    cell_cost = np.where(rng.random(cells) < 0.2, rng.integers(1, 80, cells), 0).astype(np.uint32)
    cost_full, paths_full = oracle.dijkstra_batch(lat, nets, cell_cost=cell_cost)
    seen = set()
    for radius in (0, 1, 3):
        masks = corridor.segment_corridor(nets, radius)
        for i in range(len(nets)):
            status, cost, bound = oracle.corridor_certificate(lat, nets[i], masks[i], cell_cost)
            seen.add(status)
            if status == oracle.CORRIDOR_CERTIFIED and cost is not None:
                assert cost == cost_full[i]
                priced = _priced_out(lat, nets[i], masks[i]) + cell_cost
                _, path, _ = oracle.dijkstra(lat, nets[i], cell_cost=priced)
                assert np.array_equal(path, paths_full[i]), i
    assert oracle.CORRIDOR_CERTIFIED in seen
