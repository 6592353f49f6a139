"""GPU geometry compile through the C ABI: the exact swept-trace clearance
predicate against the reference's own verdicts, the legal-edge masks of
every corpus device view, and seeded boards with many boxes against the
restatement (oracle.compile_legal_edges, which tests every box per move, so
the GPU's per-layer binning is checked too)."""

import numpy as np
import pytest

import oracle
from apgar_b200 import geometry
from tests.golden import ref_corpus

pytestmark = pytest.mark.gpu


def test_clearance_predicate_matches_the_reference():
    cases = ref_corpus.load_clearance()
    flat = np.concatenate([cases["start"], cases["end"], cases["box_min"], cases["box_max"],
                           cases["width"][:, None], cases["clearance"][:, None]], axis=1)
    err, sat = geometry.swept_clearance(flat)
    assert np.array_equal(err, cases["error"])
    assert np.array_equal(sat, cases["satisfied"])


def test_corpus_legal_edges_match_the_reference():
    geo = ref_corpus.load_geometry()
    for case in ref_corpus.load_all():
        g = geo[case.name]
        n = case.nodes
        obstacles = np.zeros(len(g["obstacles"]), geometry.OBSTACLE_DTYPE)
        for f_new, f_old in zip(geometry.OBSTACLE_DTYPE.names, ref_corpus.OBSTACLE_DTYPE.names):
            obstacles[f_new] = g["obstacles"][f_old]
        masks = geometry.compile_legal_edges(n["lattice_x"], n["lattice_y"], n["layer"], g["origin"],
                                             g["step"], g["heading_mask"], g["width"], g["clearance"],
                                             obstacles)
        assert np.array_equal(masks, n["legal_edges"]), case.name


@pytest.mark.parametrize("seed,heading", [(1, 7), (2, 3), (3, 5)])
def test_seeded_boards_match_the_restatement(seed, heading):
    rng = np.random.default_rng(seed)
    step, width, clearance = 10, int(rng.integers(2, 12)), int(rng.integers(0, 8))
    origin = (int(rng.integers(-500, 500)), int(rng.integers(-500, 500)))
    xs, ys, ls = [], [], []
    for layer in (0, 3):
        gx, gy = np.meshgrid(np.arange(-5, 25), np.arange(2, 30))
        keep = rng.random(gx.shape) < 0.9  # a few unrepresented nodes
        xs.append(gx[keep]); ys.append(gy[keep]); ls.append(np.full(int(keep.sum()), layer))
    x, y, layers = np.concatenate(xs), np.concatenate(ys), np.concatenate(ls)
    k = 30
    obstacles = np.zeros(k, geometry.OBSTACLE_DTYPE)
    cx = origin[0] + rng.integers(-5, 25, k) * step + rng.integers(-step, step, k)
    cy = origin[1] + rng.integers(2, 30, k) * step + rng.integers(-step, step, k)
    hw, hh = rng.integers(0, 25, k), rng.integers(0, 25, k)
    obstacles["min_x"], obstacles["max_x"] = cx - hw, cx + hw
    obstacles["min_y"], obstacles["max_y"] = cy - hh, cy + hh
    obstacles["layer"] = rng.choice([0, 3, 5], k)
    obstacles["owned_by_net"] = rng.random(k) < 0.2
    got = geometry.compile_legal_edges(x, y, layers, origin, step, heading, width, clearance, obstacles)
    want = oracle.compile_legal_edges(x, y, layers, origin, step, heading, width, clearance,
                                      [tuple(o) for o in obstacles])
    assert np.array_equal(got, want)
    free = oracle.compile_legal_edges(x, y, layers, origin, step, heading, width, clearance, [])
    assert (got != free).any() and (got == free).any()  # boxes block some moves, not all
