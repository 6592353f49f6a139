"""CPU pin of the graph-mode oracle: on every query of the reference's own
corpus, the oracle's exact heading-state search reproduces the reference CPU
A* outcome (cost, or disconnected) bit for bit, and its canonical compact
path is a legal, cost-consistent reverse path."""

import numpy as np
import pytest

import oracle
from tests.golden import ref_corpus

CASES = ref_corpus.load_all()
U64_MAX = (1 << 64) - 1


def test_fixture_set_is_complete():
    names = {c.name for c in CASES}
    assert {"dense_corridors", "sparse_regions", "fragmented_runs", "high_turn_maze",
            "cross_tile_edges", "negative_coordinates", "disconnected_fields",
            "kicad_fixture"} <= names
    # the reference's published Phase-2 costs (base policy, forward request)
    published = {"dense_corridors": 140, "sparse_regions": 149, "fragmented_runs": 454,
                 "high_turn_maze": 1148, "cross_tile_edges": 50, "negative_coordinates": 370,
                 "kicad_fixture": 37168}
    for c in CASES:
        if c.name in published:
            assert c.queries[0].cpu_status == 0 and c.queries[0].cpu_cost == published[c.name]
        if c.name == "disconnected_fields":
            assert c.queries[0].cpu_status == 1


def _transition(nodes, costs, q, src, d, h_in):
    """Reference DeviceBatchTransitionCost (planar_router.cu:557-583) in Python."""
    orth, diag, bend = costs
    if d < 4:
        edge = src * 8 + d
    else:
        canon = int(nodes["neighbors"][src][d])
        edge = canon * 8 + d - 4
    adj = 0
    idx = np.searchsorted(q.policy["physical_edge_index"], edge) if len(q.policy) else 0
    if len(q.policy) and idx < len(q.policy) and q.policy["physical_edge_index"][idx] == edge:
        adj = int(q.policy["adjustment"][idx])
    if adj == U64_MAX:
        return None
    v = (diag + q.diagonal_surcharge) if d & 1 else (orth + q.orthogonal_surcharge)
    if h_in != 8 and h_in != d:
        v += bend + q.bend_surcharge
    v += adj
    return v if v < U64_MAX else None


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_graph_oracle_matches_reference_cpu_astar(case):
    costs = case.costs
    for qi, q in enumerate(case.queries):
        reached, cost, goal_state, path, _ = oracle.graph_search(
            case.nodes, costs, q.start_node, q.goal_node, q.orthogonal_surcharge,
            q.diagonal_surcharge, q.bend_surcharge, q.policy)
        if q.cpu_status == 0:
            assert reached and cost == q.cpu_cost, (qi, cost, q.cpu_cost)
            # reverse path: goal state first, start state (heading 8) last
            assert path[0] == goal_state and path[-1] == q.start_node * 9 + 8
            total = 0
            for a, b in zip(path[::-1][:-1], path[::-1][1:]):
                node_a, h_a = divmod(int(a), 9)
                node_b, h_b = divmod(int(b), 9)
                assert int(case.nodes["neighbors"][node_a][h_b]) == node_b
                t = _transition(case.nodes, costs, q, node_a, h_b, h_a)
                assert t is not None
                total += t
            assert total == cost
        elif q.cpu_status == 1:
            assert not reached, qi


def test_fixtures_regenerate_from_the_reference(tmp_path):
    """Where the reference sources are present and built (oracle/build_ref.sh),
    its own corpus builders and CPU A* reproduce the committed fixtures byte
    for byte."""
    import filecmp
    import os
    import subprocess

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(root, "oracle", "_ref", "ref_fixtures")
    ref = oracle.reference_root()
    if ref is None or not os.path.exists(exe):
        pytest.skip("reference sources or the compiled reference checker are absent "
                    "(set APGAR_REFERENCE or run oracle/build_ref.sh)")
    pcb = os.path.join(ref, "tests", "fixtures", "m1_exactness.kicad_pcb")
    subprocess.run([exe, pcb, str(tmp_path)], check=True, stdout=subprocess.DEVNULL)
    committed = os.path.join(root, "tests", "golden", "ref_corpus")
    names = sorted(os.listdir(committed))
    assert sorted(os.listdir(tmp_path)) == names
    for name in names:
        assert filecmp.cmp(os.path.join(committed, name), os.path.join(tmp_path, name),
                           shallow=False), name


def _mutations(case, q, path):
    """(label, mutated reverse path, policy, expected code) for one reached path."""
    n = len(case.nodes)
    out = [("valid", path, q.policy, "ok")]
    out.append(("truncated start", path[:-1], q.policy, "endpoint"))
    out.append(("wrong goal", np.concatenate([[path[0] ^ 1], path[1:]]).astype(np.uint32), q.policy,
                "endpoint"))
    if len(path) > 3:
        rep = path.copy()
        rep[1] = rep[3]
        out.append(("repeated state", rep, q.policy, None))  # cycle, edge or heading
        hd = path.copy()
        node, h = divmod(int(hd[1]), 9)
        hd[1] = node * 9 + (h + 1) % 8
        out.append(("turned heading", hd, q.policy, None))
        oob = path.copy()
        oob[1] = 9 * n + 3
        out.append(("state out of range", oob, q.policy, "bounds"))
    if len(path) > 2:
        # ban the physical edge of the first move
        s0, s1 = int(path[-1]), int(path[-2])
        d = s1 % 9
        src = s0 // 9
        edge = src * 8 + d if d < 4 else int(case.nodes[src]["neighbors"][d]) * 8 + d - 4
        ban = np.zeros(1, dtype=ref_corpus.POLICY_EDGE_DTYPE)
        ban[0] = (edge, 0, U64_MAX)
        pol = ban if not len(q.policy) else np.sort(
            np.concatenate([q.policy[q.policy["physical_edge_index"] != edge], ban]),
            order="physical_edge_index")
        out.append(("banned first edge", path, pol, "banned"))
    return out


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_compact_path_validation_pins_the_reference_cost(case):
    """Valid canonical paths validate with exactly the reference CPU A* cost;
    each kind of corruption is reported with the reference's invariant."""
    for q in case.queries:
        if q.cpu_status != 0:
            continue
        ok, cost, goal_state, path, _ = oracle.graph_search(
            case.nodes, case.costs, q.start_node, q.goal_node, q.orthogonal_surcharge,
            q.diagonal_surcharge, q.bend_surcharge, q.policy)
        assert ok and cost == q.cpu_cost
        for label, rev, pol, want in _mutations(case, q, path):
            code, total, _ = oracle.validate_compact(
                case.nodes, case.costs, q.start_node, q.goal_node, rev, goal_state, 0,
                q.orthogonal_surcharge, q.diagonal_surcharge, q.bend_surcharge, pol)
            if want is None:
                assert code in ("cycle", "heading", "edge"), (label, code)
            else:
                assert code == want, (case.name, label, code)
            if label == "valid":
                assert total == q.cpu_cost
