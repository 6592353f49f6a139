"""CPU checks of the lattice-mode oracle: three independent restatements
(Dijkstra, reference-key A*, row-sweep schedule) agree, and the canonical
path obeys the tie-break rule and the move model."""

import numpy as np
import pytest

import oracle
from apgar_b200 import synth

DX = [1, 1, 0, -1, -1, -1, 0, 1]
DY = [0, 1, 1, 1, 0, -1, -1, -1]


def _free(dense, net, l, x, y):
    if not (0 <= l < dense.shape[0]):
        return False
    if not (net["win_x0"] <= x < net["win_x0"] + net["win_w"]):
        return False
    if not (net["win_y0"] <= y < net["win_y0"] + net["win_h"]):
        return False
    return not dense[l, y, x]


def _check_path(lat, net, cost, path):
    """Reverse path legality + exact cost (move model of oracle.h)."""
    dense = lat.blocked_dense()
    H, W = lat.height, lat.width
    cells = [(int(c) // (H * W), (int(c) % (H * W)) // W, int(c) % W) for c in path]
    assert cells[0] == (net["goal_layer"], net["goal_y"], net["goal_x"])
    assert cells[-1] == (net["start_layer"], net["start_y"], net["start_x"])
    total = 0
    for (l1, y1, x1), (l0, y0, x0) in zip(cells[:-1], cells[1:]):
        assert _free(dense, net, l0, x0, y0) and _free(dense, net, l1, x1, y1)
        if l1 != l0:
            assert (x1, y1) == (x0, y0) and abs(l1 - l0) == 1
            total += lat.via
        else:
            dx, dy = x1 - x0, y1 - y0
            assert max(abs(dx), abs(dy)) == 1
            if dx and dy:
                assert _free(dense, net, l0, x1, y0) and _free(dense, net, l0, x0, y1)
                total += lat.diag
            else:
                total += lat.orth
    assert total == cost


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_small_config_restatements_agree(seed):
    lat, nets = synth.config_small(seed)
    cd, paths = oracle.dijkstra_batch(lat, nets)
    ca = oracle.astar_batch(lat, nets)
    cs, _ = oracle.sweep_batch(lat, nets)
    assert np.array_equal(cd, ca)
    assert np.array_equal(cd, cs)
    for i in range(len(nets)):
        if cd[i] != oracle.lo_inf():
            _check_path(lat, nets[i], int(cd[i]), paths[i])


def test_medium_like_restatements_agree():
    lat, nets = synth.config_medium(5, nets=48, size=512)
    cd, paths = oracle.dijkstra_batch(lat, nets)
    ca = oracle.astar_batch(lat, nets)
    cs, st = oracle.sweep_batch(lat, nets)
    assert np.array_equal(cd, ca) and np.array_equal(cd, cs)
    assert (st[:, 0] >= 2).all()
    for i in range(len(nets)):
        if cd[i] != oracle.lo_inf():
            _check_path(lat, nets[i], int(cd[i]), paths[i])


def test_via_mask_and_single_layer():
    lat = synth.make_lattice(7, 3, 96, 0.22, via_mask=True)
    nets = synth.make_nets(lat, 70, 24, hpwl_median=40.0, hpwl_sigma=0.6, margin=8)
    cd, _ = oracle.dijkstra_batch(lat, nets)
    assert np.array_equal(cd, oracle.astar_batch(lat, nets))
    assert np.array_equal(cd, oracle.sweep_batch(lat, nets)[0])
    lat1 = synth.make_lattice(8, 1, 64, 0.3)
    nets1 = synth.make_nets(lat1, 80, 20, hpwl_median=None, margin=None)
    cd1, _ = oracle.dijkstra_batch(lat1, nets1)
    assert np.array_equal(cd1, oracle.astar_batch(lat1, nets1))
    assert np.array_equal(cd1, oracle.sweep_batch(lat1, nets1)[0])


def test_known_answers_open_field():
    # Open 1-layer field: octile distance, canonical path prefers east/north-east first.
    lat = synth.Lattice(1, 32, 32, np.zeros((1, 32, 1), np.uint32), None)
    net = np.array([(0, 2, 3, 0, 9, 5, 0, 0, 32, 32)], dtype=synth.NET_DTYPE)
    cost, path, _ = oracle.dijkstra(lat, net[0])
    assert cost == 2 * 14 + 5 * 10  # dx=7, dy=2
    _check_path(lat, net[0], cost, path)
    # blocked start -> disconnected
    dense = np.zeros((1, 32, 32), bool)
    dense[0, 3, 2] = True
    lat2 = synth.Lattice(1, 32, 32, synth.pack_bits(dense), None)
    cost2, _, _ = oracle.dijkstra(lat2, net[0])
    assert cost2 == oracle.lo_inf()


def test_disconnected_by_wall():
    dense = np.zeros((2, 32, 32), bool)
    dense[:, :, 16] = True  # full wall on both layers
    lat = synth.Lattice(2, 32, 32, synth.pack_bits(dense), None)
    net = np.array([(0, 2, 3, 1, 30, 5, 0, 0, 32, 32)], dtype=synth.NET_DTYPE)
    assert oracle.dijkstra(lat, net[0])[0] == oracle.lo_inf()
    assert oracle.astar_batch(lat, net)[0] == oracle.lo_inf()
    assert oracle.sweep_batch(lat, net)[0][0] == oracle.lo_inf()
    # a via hole does not help when both layers are walled; open one layer's wall
    dense[1, 10, 16] = False
    lat = synth.Lattice(2, 32, 32, synth.pack_bits(dense), None)
    c = oracle.dijkstra(lat, net[0])[0]
    assert c != oracle.lo_inf()
    assert c == oracle.astar_batch(lat, net)[0] == oracle.sweep_batch(lat, net)[0][0]


def _lattice_as_graph(dense):
    """Single-layer lattice as DeviceCompiledBoardV1 node records (node id
    y*W + x), with legal-edge masks from the lattice move rule: orthogonal moves
    need both cells free, diagonal moves also both side cells."""
    from tests.golden import ref_corpus

    _, h, w = dense.shape
    nodes = np.zeros(h * w, dtype=ref_corpus.NODE_DTYPE)
    nodes["neighbors"] = 0xFFFFFFFF

    def free(x, y):
        return 0 <= x < w and 0 <= y < h and not dense[0, y, x]

    for y in range(h):
        for x in range(w):
            n = nodes[y * w + x]
            n["lattice_x"], n["lattice_y"] = x, y
            legal = 0
            for d in range(8):
                nx, ny = x + DX[d], y + DY[d]
                if not (0 <= nx < w and 0 <= ny < h):
                    continue
                n["neighbors"][d] = ny * w + nx
                ok = free(x, y) and free(nx, ny)
                if d & 1:
                    ok = ok and free(x + DX[d], y) and free(x, y + DY[d])
                if ok:
                    legal |= 1 << d
            n["legal_edges"] = legal
    return nodes


@pytest.mark.parametrize("seed", [3, 4])
def test_pinned_to_reference_graph_oracle_on_single_layer(seed):
    """Transitive pin: the graph oracle reproduces the reference CPU A* on
    every fixture query (test_oracle_graph.py); on single-layer lattices
    (no vias, bend 0) the lattice oracle must give the same costs and the same
    canonical reverse paths as the graph oracle's compact heading-state path."""
    rng = np.random.default_rng(seed)
    h, w = 40, 64
    dense = np.zeros((1, h, w), bool)
    for _ in range(30):
        x0, y0 = rng.integers(0, w - 4), rng.integers(0, h - 4)
        dense[0, y0:y0 + rng.integers(2, 9), x0:x0 + rng.integers(2, 9)] = True
    lat = synth.Lattice(1, h, w, synth.pack_bits(dense), None)
    nodes = _lattice_as_graph(dense)
    free = np.argwhere(~dense[0])
    compared = reached = 0
    for _ in range(40):
        (sy, sx), (gy, gx) = free[rng.integers(len(free), size=2)]
        net = np.array([(0, sx, sy, 0, gx, gy, 0, 0, w, h)], dtype=synth.NET_DTYPE)
        cost, path, _ = oracle.dijkstra(lat, net[0])
        ok, gcost, _, gpath, _ = oracle.graph_search(nodes, (10, 14, 0), int(sy * w + sx),
                                                     int(gy * w + gx))
        compared += 1
        if cost == oracle.lo_inf():
            assert not ok
            continue
        reached += 1
        assert ok and gcost == cost
        graph_cells = (gpath // 9).astype(np.uint32)  # node ids are y*W + x = cell ids
        assert np.array_equal(graph_cells, path), (sx, sy, gx, gy)
    assert compared == 40 and reached >= 20


def test_priced_dijkstra_against_brute_force_relaxation():
    """Per-cell entry prices: the oracle's labels equal a Bellman-Ford fixed
    point computed here, and its canonical path pays move + entry costs."""
    rng = np.random.default_rng(9)
    lat = synth.make_lattice(9, 2, 32, 0.15, via_mask=False)
    price = rng.integers(0, 40, size=(2, 32, 32)).astype(np.uint32)
    dense = synth.unpack_bits(np.asarray(lat.blocked).reshape(2, 32, 1), 32)
    free = np.argwhere(~dense)
    for _ in range(4):
        (sl, sy, sx), (gl, gy, gx) = free[rng.integers(len(free), size=2)]
        net = np.array([(sl, sx, sy, gl, gx, gy, 0, 0, 32, 32)], dtype=synth.NET_DTYPE)
        cost, path, dist = oracle.dijkstra(lat, net[0], full=True, want_dist=True, cell_cost=price)
        # Bellman-Ford over the same move model
        INF = 1 << 40
        d = np.full((2, 32, 32), INF, dtype=np.int64)
        d[sl, sy, sx] = 0
        for _ in range(400):
            changed = False
            for l in range(2):
                for y in range(32):
                    for x in range(32):
                        if d[l, y, x] >= INF:
                            continue
                        for h in range(10):
                            if h < 8:
                                nl, nx, ny = l, x + DX[h], y + DY[h]
                                if not (_free(dense, net[0], l, x, y) and _free(dense, net[0], l, nx, ny)):
                                    continue
                                if h & 1 and not (_free(dense, net[0], l, nx, y) and _free(dense, net[0], l, x, ny)):
                                    continue
                                c = 14 if h & 1 else 10
                            else:
                                nl, nx, ny = l + (1 if h == 8 else -1), x, y
                                if not (_free(dense, net[0], l, x, y) and _free(dense, net[0], nl, x, y)):
                                    continue
                                c = 50
                            v = d[l, y, x] + c + int(price[nl, ny, nx])
                            if v < d[nl, ny, nx]:
                                d[nl, ny, nx] = v
                                changed = True
            if not changed:
                break
        want = d[gl, gy, gx]
        assert (cost == oracle.lo_inf()) == (want >= INF)
        if want < INF:
            assert cost == want
            # the path pays exactly its cost
            total = 0
            cells = [(int(c) // (32 * 32), (int(c) // 32) % 32, int(c) % 32) for c in path[::-1]]
            for (l0, y0, x0), (l1, y1, x1) in zip(cells, cells[1:]):
                step = 50 if l0 != l1 else (14 if (x0 != x1 and y0 != y1) else 10)
                total += step + int(price[l1, y1, x1])
            assert total == cost
