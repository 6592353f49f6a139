"""CPU pin of the disconnected-confirmation restatement: on every query of the
reference's own corpus its verdict is the reference CPU A* outcome
("confirmed" exactly where the reference reported disconnected, "reachable"
where it found a route), it agrees with the oracle's exact heading-state
search under added bans, and the overflow bound turns "confirmed" into
"unbounded" exactly at the edge of the finite range."""

import numpy as np
import pytest

import oracle
from tests.golden import ref_corpus

CASES = ref_corpus.load_all()
U64_MAX = (1 << 64) - 1


def _isolating_bans(case, node, policy):
    """The query's policy plus a ban on every legal edge of `node`."""
    edges = []
    nd = case.nodes[node]
    for d in range(8):
        if (int(nd["legal_edges"]) >> d) & 1:
            v = int(nd["neighbors"][d])
            edges.append(node * 8 + d if d < 4 else v * 8 + d - 4)
    keep = policy[~np.isin(policy["physical_edge_index"], edges)] if len(policy) else policy
    ban = np.zeros(len(edges), dtype=ref_corpus.POLICY_EDGE_DTYPE)
    ban["physical_edge_index"] = edges
    ban["adjustment"] = U64_MAX
    return np.sort(np.concatenate([keep, ban]), order="physical_edge_index")


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_verdict_is_reference_cpu_outcome(case):
    for q in case.queries:
        code, reached = oracle.disconnect_verdict(
            case.nodes, case.costs, q.start_node, q.goal_node, q.orthogonal_surcharge,
            q.diagonal_surcharge, q.bend_surcharge, q.policy)
        assert code == {0: "reachable", 1: "confirmed"}[q.cpu_status], (case.name, q.start_node)
        assert 1 <= reached <= len(case.nodes)


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_verdict_agrees_with_exact_search_under_bans(case):
    for q in case.queries:
        if q.start_node == q.goal_node:
            continue
        pol = _isolating_bans(case, q.start_node, q.policy)
        code, reached = oracle.disconnect_verdict(
            case.nodes, case.costs, q.start_node, q.goal_node, q.orthogonal_surcharge,
            q.diagonal_surcharge, q.bend_surcharge, pol)
        ok, *_ = oracle.graph_search(case.nodes, case.costs, q.start_node, q.goal_node,
                                     q.orthogonal_surcharge, q.diagonal_surcharge,
                                     q.bend_surcharge, pol)
        assert not ok and code == "confirmed" and reached == 1


def test_overflow_bound_edge():
    case = next(c for c in CASES if c.name == "disconnected_fields")
    q = case.queries[0]
    _, reached = oracle.disconnect_verdict(case.nodes, case.costs, q.start_node, q.goal_node,
                                           policy=q.policy)
    orth, diag, bend = case.costs
    base = max(orth, diag) + bend
    limit = (U64_MAX - 1) // (8 * reached + 1)  # the largest bounded transition
    for extra, want in ((limit - base, "confirmed"), (limit - base + 1, "unbounded")):
        # a finite penalty on an edge nobody takes raises the transition bound
        pen = np.zeros(1, dtype=ref_corpus.POLICY_EDGE_DTYPE)
        pen[0] = (len(case.nodes) * 8 + 7, 0, extra)
        pol = np.sort(np.concatenate([q.policy, pen]), order="physical_edge_index")
        code, _ = oracle.disconnect_verdict(case.nodes, case.costs, q.start_node, q.goal_node,
                                            policy=pol)
        assert code == want
