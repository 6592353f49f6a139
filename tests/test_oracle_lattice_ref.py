"""The lattice oracle pinned to the reference itself.

tests/golden/ref_lattice/ holds planar 256 x 256 boards with seeded rectangle
obstacles (about 20% of cells, the small configuration's model), 12 queries
each, and the reference's own verdicts (tests/golden/make_ref_lattice.py
running oracle/ref_lattice.cc over the reference compiled from its sources):
the legal-edge masks of CompileBoard's swept-trace compile
(src/geometry_compiler/compiled_board.cc:427-476) and the cost, expanded-state
count and path of RouteWithCpuAStar (src/routing/cpu_astar.cc:323-638).

Checked here:
  * the lattice move rule (orthogonal: both cells free; diagonal: both cells
    and both side cells free) equals the reference's compiled legal edges at
    every node and heading;
  * ``lo_dijkstra`` and ``lo_astar`` give the reference's costs;
  * ``lo_astar``'s expanded-state count and path equal the reference A*'s, so
    the restatement pops states in the reference's order.
"""

import os
import subprocess
import sys

import numpy as np
import pytest

import oracle
from apgar_b200 import synth

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "ref_lattice")
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_ref_lattice as mrl  # noqa: E402

SEEDS = [seed for seed, _ in mrl.CASES]
DX = [1, 1, 0, -1, -1, -1, 0, 1]
DY = [0, 1, 1, 1, 0, -1, -1, -1]


def _blocked(rects, size):
    b = np.zeros((size, size), dtype=bool)
    for x0, y0, x1, y1 in rects:
        b[y0:y1 + 1, x0:x1 + 1] = True
    return b


def _rule_masks(blocked):
    size = blocked.shape[0]
    pad = np.ones((size + 2, size + 2), dtype=bool)
    pad[1:-1, 1:-1] = blocked
    free = ~pad

    def f(dx, dy):
        return free[1 + dy:size + 1 + dy, 1 + dx:size + 1 + dx]

    masks = np.zeros((size, size), dtype=np.uint8)
    for d in range(8):
        ok = f(0, 0) & f(DX[d], DY[d])
        if d & 1:
            ok &= f(DX[d], 0) & f(0, DY[d])
        masks |= ok.astype(np.uint8) << d
    return masks


def _lattice(blocked):
    size = blocked.shape[0]
    return synth.Lattice(layers=1, height=size, width=size,
                         blocked=synth.pack_bits(blocked[None]), via_ok=None)


def _net(q, size):
    net = np.zeros(1, dtype=synth.NET_DTYPE)
    sx, sy, gx, gy = (int(v) for v in q)
    net[0] = (0, sx, sy, 0, gx, gy, 0, 0, size, size)
    return net


@pytest.mark.parametrize("seed", SEEDS)
def test_lattice_rule_equals_the_reference_compile(seed):
    rects, _, legal, _ = mrl.load(GOLDEN, seed)
    blocked = _blocked(rects, legal.shape[0])
    assert 0.19 <= blocked.mean() <= 0.23
    want = _rule_masks(blocked)
    assert np.array_equal(legal, want), int((legal != want).sum())
    # the rule is not vacuous: diagonals are cut by side cells on this board
    assert ((want & 0xAA) != 0).any() and (((want >> 1) & 1) != (want & 1)).any()


@pytest.mark.parametrize("seed", SEEDS)
def test_astar_and_dijkstra_equal_the_reference_astar(seed):
    rects, queries, legal, routes = mrl.load(GOLDEN, seed)
    size = legal.shape[0]
    lat = _lattice(_blocked(rects, size))
    reached = 0
    for q, (status, cost, expanded, _pops, path) in zip(queries, routes):
        net = _net(q, size)
        a_cost, a_expanded, a_path = oracle.astar_path(lat, net)
        d_cost, _, _ = oracle.dijkstra(lat, net)
        if status == 1:
            assert a_cost == oracle.lo_inf() and d_cost == oracle.lo_inf()
            continue
        assert status == 0
        reached += 1
        assert a_cost == cost and d_cost == cost, (q, cost, a_cost, d_cost)
        assert a_expanded == expanded, (q, expanded, a_expanded)
        ids = path[:, 1].astype(np.int64) * size + path[:, 0]
        assert np.array_equal(a_path, ids), q
    assert reached >= 10


def test_fixtures_regenerate_from_the_reference(tmp_path):
    """Where the reference is built (oracle/build_ref.sh), its own compiler
    and A* reproduce the committed fixtures byte for byte."""
    exe = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "ref_lattice")
    if oracle.reference_root() is None or not os.path.exists(exe):
        pytest.skip("the compiled reference is absent (set APGAR_REFERENCE or run "
                    "oracle/build_ref.sh)")
    subprocess.run([sys.executable, os.path.join(HERE, "golden", "make_ref_lattice.py"),
                    str(tmp_path)], check=True)
    for seed in SEEDS:
        for ext in ("in", "out"):
            name = f"board{seed}.{ext}"
            with open(os.path.join(GOLDEN, name), "rb") as a, open(tmp_path / name, "rb") as b:
                assert a.read() == b.read(), name
