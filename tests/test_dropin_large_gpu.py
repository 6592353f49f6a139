"""GPU parity of the drop-in search on boards too large for its shared-memory
form (about 880 nodes): synthetic single-layer boards of 1,296 and 2,304
nodes, built as DeviceCompiledBoardV1 records that pass the upload checks,
with wall segments cut out of the edge set.  The compact paths and, in the
full-workspace form, every label and canonical predecessor must equal the
exact heading-state oracle's (oracle.graph_search / graph_predecessors)."""

import numpy as np
import pytest

import apgar_b200
import oracle
from apgar_b200 import dropin
from tests.golden import ref_corpus

pytestmark = pytest.mark.gpu

DX = (1, 1, 0, -1, -1, -1, 0, 1)
DY = (0, 1, 1, 1, 0, -1, -1, -1)
U64_MAX = (1 << 64) - 1


def _board(side: int, seed: int, bend: int):
    """A side x side grid, every move legal except those crossing a wall."""
    rng = np.random.default_rng(seed)
    cut = np.zeros((side, side), bool)  # cells whose edges are removed (walls)
    for _ in range(side // 3):
        x, y = rng.integers(2, side - 2, size=2)
        if rng.integers(2):
            cut[y, max(0, x - side // 4):x + side // 4] = True
        else:
            cut[max(0, y - side // 4):y + side // 4, x] = True
    n = side * side
    nodes = np.zeros(n, dtype=ref_corpus.NODE_DTYPE)
    nodes["neighbors"] = 0xFFFFFFFF
    for y in range(side):
        for x in range(side):
            rec = nodes[y * side + x]
            rec["lattice_x"], rec["lattice_y"] = x, y
            legal = 0
            for d in range(8):
                nx, ny = x + DX[d], y + DY[d]
                if 0 <= nx < side and 0 <= ny < side and not cut[y, x] and not cut[ny, nx]:
                    rec["neighbors"][d] = ny * side + nx
                    legal |= 1 << d
            rec["legal_edges"] = legal
    # maximal directed runs, one per chain of legal edges in each direction
    runs, run_nodes = [], []
    for d in range(8):
        back = (d + 4) % 8
        for i in range(n):
            if not (nodes[i]["legal_edges"] >> d) & 1 or (nodes[i]["legal_edges"] >> back) & 1:
                continue
            chain = [i]
            while (nodes[chain[-1]]["legal_edges"] >> d) & 1:
                chain.append(int(nodes[chain[-1]]["neighbors"][d]))
            runs.append((len(run_nodes), len(chain), d))
            run_nodes.extend(chain)
    run = np.zeros(len(runs), dtype=ref_corpus.RUN_DTYPE)
    for k, (off, cnt, d) in enumerate(runs):
        run[k]["node_offset"], run[k]["node_count"], run[k]["direction"] = off, cnt, d
    run_nodes = np.array(run_nodes, dtype=np.uint32)
    layers = np.zeros(1, dtype=ref_corpus.LAYER_DTYPE)
    layers[0]["node_count"] = n
    layers[0]["maximum_lattice_x"] = layers[0]["maximum_lattice_y"] = side - 1
    header = np.zeros(1, dtype=ref_corpus.HEADER_DTYPE)
    h = header[0]
    h["schema_version"], h["compiler_version"] = 1, 1
    h["represented_nodes"], h["represented_states"] = n, 9 * n
    h["lattice_step"], h["orthogonal_step"], h["diagonal_step"], h["bend"] = 1, 10, 14, bend
    h["heading_mask"] = 7
    h["estimated_persistent_device_bytes"] = 112 + 48 + 56 * n + 12 * len(run) + 4 * len(run_nodes)
    return header, layers, nodes, run, run_nodes, cut


def _queries(nodes, cut, seed, count):
    rng = np.random.default_rng(seed)
    free = np.flatnonzero(~cut.ravel())
    diag = np.flatnonzero((nodes["legal_edges"] >> 1) & 1)  # nodes with a legal +x+y edge
    entries = []
    for i in range(count):
        s, g = rng.choice(free, size=2, replace=False)
        e = dict(start_node=int(s), goal_node=int(g))
        if i % 3 == 1:
            e.update(orthogonal_step_surcharge=2, bend_surcharge=5)
        if i % 3 == 2:
            # a few penalised and one banned legal edge (node * 8 + d, d < 4)
            picks = np.sort(rng.choice(diag, size=6, replace=False))
            pol = np.zeros(6, dtype=ref_corpus.POLICY_EDGE_DTYPE)
            pol["physical_edge_index"] = picks.astype(np.uint32) * 8 + 1
            pol["adjustment"] = 40
            pol["adjustment"][0] = U64_MAX
            e.update(policy=pol)
        entries.append(e)
    return entries


@pytest.mark.parametrize("side,bend", [(36, 0), (48, 7)])
@pytest.mark.parametrize("generator", [dropin.GENERATOR_SWEEP, dropin.GENERATOR_PERSISTENT])
def test_large_board_compact_paths_match_the_oracle(side, bend, generator):
    header, layers, nodes, runs, run_nodes, cut = _board(side, side + bend, bend)
    assert len(nodes) * (9 * 8 + 12) > 100 * 1024  # beyond the shared-memory form
    view = dropin.View(header, layers, nodes, runs, run_nodes)
    entries = _queries(nodes, cut, side, 24)
    queries, edges = dropin.make_queries(view.node_count, entries, generator=generator)
    pending = view.execute_batch(queries, edges, generator=generator)
    results, compact, states, _ = pending.readback()
    pending.close()
    reached = 0
    for i, e in enumerate(entries):
        ok, cost, goal_state, path, _ = oracle.graph_search(
            nodes, (10, 14, bend), e["start_node"], e["goal_node"],
            e.get("orthogonal_step_surcharge", 0), 0, e.get("bend_surcharge", 0), e.get("policy"))
        r, c = results[i], compact[i]
        if not ok:
            assert r["completion"] == apgar_b200.COMPLETION_DISCONNECTED, i
            continue
        reached += 1
        assert r["completion"] == apgar_b200.COMPLETION_REACHED, i
        assert r["goal_state"] == goal_state, i
        got = states[int(c["state_offset"]): int(c["state_offset"]) + int(c["state_count"])]
        assert np.array_equal(got, path), i
    assert reached > 0
    view.close()


def test_large_board_full_workspace_labels_and_predecessors():
    side, bend = 36, 3
    header, layers, nodes, runs, run_nodes, cut = _board(side, 11, bend)
    view = dropin.View(header, layers, nodes, runs, run_nodes)
    entries = _queries(nodes, cut, 5, 6)
    queries, edges = dropin.make_queries(view.node_count, entries, generator=dropin.GENERATOR_FRONTIER)
    pending = view.execute_batch(queries, edges, generator=dropin.GENERATOR_FRONTIER)
    pending.readback()
    labels, preds, _, _ = pending.readback_workspace()
    pending.close()
    S = 9 * view.node_count
    for i, e in enumerate(entries):
        args = (e.get("orthogonal_step_surcharge", 0), 0, e.get("bend_surcharge", 0), e.get("policy"))
        _, _, _, _, exact = oracle.graph_search(nodes, (10, 14, bend), e["start_node"], e["goal_node"],
                                                *args, want_labels=True)
        sl = slice(i * S, (i + 1) * S)
        assert np.array_equal(labels[sl], exact), i
        canon = oracle.graph_predecessors(nodes, (10, 14, bend), e["start_node"], exact, *args)
        assert np.array_equal(preds[sl], canon), i
    view.close()
