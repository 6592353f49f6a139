"""CPU pin of the full-workspace predecessor validation restatement: the
oracle's exact labels with their canonical predecessors validate on every
query of the reference corpus, and each corruption gets its code at the
first failing state."""

import numpy as np
import pytest

import oracle
from tests.golden import ref_corpus

CASES = ref_corpus.load_all()
U64 = (1 << 64) - 1
INV = 0xFFFFFFFF


def workspace(case, q):
    _, _, _, _, labels = oracle.graph_search(
        case.nodes, case.costs, q.start_node, q.goal_node, q.orthogonal_surcharge,
        q.diagonal_surcharge, q.bend_surcharge, q.policy, want_labels=True)
    preds = oracle.graph_predecessors(case.nodes, case.costs, q.start_node, labels,
                                      q.orthogonal_surcharge, q.diagonal_surcharge,
                                      q.bend_surcharge, q.policy)
    return labels.copy(), preds.copy()


def corruptions(case, q, labels, preds):
    """(kind, labels, preds, expected code, expected failing state)."""
    out = []
    finite = [s for s in range(len(labels)) if labels[s] != U64 and preds[s] != INV]
    if not finite:
        return out
    s = finite[len(finite) // 2]
    L, P = labels.copy(), preds.copy()
    P[s] = s
    out.append(("self", L, P, "self_reference", s))
    L, P = labels.copy(), preds.copy()
    P[s] = len(labels) + 3
    out.append(("bounds", L, P, "bounds", s))
    L, P = labels.copy(), preds.copy()
    L[s] += 1
    first = min([s] + [t for t in finite if P[t] == s])  # s and every state that follows it
    out.append(("cost", L, P, "cost", first))
    L, P = labels.copy(), preds.copy()
    unreach = [t for t in range(len(labels)) if labels[t] == U64 and t % 9 != 8]
    if unreach:
        P[unreach[0]] = finite[0]
        out.append(("unreachable", L, P, "unreachable", unreach[0]))
    L, P = labels.copy(), preds.copy()
    start_state = 9 * q.start_node + 8
    L[start_state] = 5
    out.append(("start", L, P, "start", start_state))
    return out


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_exact_workspaces_validate_and_corruptions_are_caught(case):
    for q in case.queries[:6]:
        labels, preds = workspace(case, q)
        code, _ = oracle.validate_predecessors(case.nodes, case.costs, q.start_node, labels, preds,
                                               q.orthogonal_surcharge, q.diagonal_surcharge,
                                               q.bend_surcharge, q.policy)
        assert code == "ok", (case.name, q.start_node, code)
        for kind, L, P, want, state in corruptions(case, q, labels, preds):
            code, idx = oracle.validate_predecessors(case.nodes, case.costs, q.start_node, L, P,
                                                     q.orthogonal_surcharge, q.diagonal_surcharge,
                                                     q.bend_surcharge, q.policy)
            assert (code, idx) == (want, state), (case.name, kind, code, idx)
