"""GPU confirmation of DISCONNECTED results (the device counterpart of the
reference's ConfirmDisconnectedWithCpuOracle) against the CPU restatement, on
the reference corpus: the engine's own disconnected results are confirmed,
forged claims on reachable queries are caught with the same count of nodes
reached, bans that isolate the start are confirmed, and the overflow bound
flips to "unbounded" at the same penalty as in the oracle."""

import numpy as np
import pytest

import oracle
from apgar_b200 import dropin
from tests.golden import ref_corpus
from tests.test_oracle_disconnect import _isolating_bans

pytestmark = pytest.mark.gpu

CASES = ref_corpus.load_all()
U64_MAX = (1 << 64) - 1
DISCONNECTED = 1


def _entries(case, policies=None):
    return [dict(start_node=q.start_node, goal_node=q.goal_node,
                 orthogonal_step_surcharge=q.orthogonal_surcharge,
                 diagonal_step_surcharge=q.diagonal_surcharge, bend_surcharge=q.bend_surcharge,
                 policy=q.policy if policies is None else policies[i],
                 policy_identity=q.policy_identity) for i, q in enumerate(case.queries)]


def _expect(case, policies, claimed):
    out = []
    for i, q in enumerate(case.queries):
        if not claimed[i]:
            out.append(("not_claimed", 0))
            continue
        out.append(oracle.disconnect_verdict(
            case.nodes, case.costs, q.start_node, q.goal_node, q.orthogonal_surcharge,
            q.diagonal_surcharge, q.bend_surcharge, policies[i]))
    return out


def _got(verdicts):
    return [(dropin.DISCONNECT_CODES[int(v["code"])], int(v["reachable_nodes"])) for v in verdicts]


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_engine_disconnected_results_are_confirmed(case):
    view = dropin.View(case.header, case.layers, case.nodes, case.runs, case.run_nodes)
    queries, edges = dropin.make_queries(view.node_count, _entries(case))
    pending = view.execute_batch(queries, edges)
    results, _, _, _ = pending.readback()
    pending.close()
    claimed = results["completion"] == DISCONNECTED
    got = _got(view.confirm_disconnected(queries, edges, results))
    assert got == _expect(case, [q.policy for q in case.queries], claimed)
    for i, q in enumerate(case.queries):
        if claimed[i]:
            assert got[i][0] == "confirmed" and q.cpu_status == 1
    # every result forged as DISCONNECTED: reachable queries are caught
    forged = results.copy()
    forged["completion"] = DISCONNECTED
    got = _got(view.confirm_disconnected(queries, edges, forged))
    assert got == _expect(case, [q.policy for q in case.queries], [True] * len(case.queries))
    assert [g[0] for g in got] == [{0: "reachable", 1: "confirmed"}[q.cpu_status]
                                   for q in case.queries]
    view.close()


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_isolated_starts_are_confirmed(case):
    view = dropin.View(case.header, case.layers, case.nodes, case.runs, case.run_nodes)
    pols = [q.policy if q.start_node == q.goal_node else _isolating_bans(case, q.start_node, q.policy)
            for q in case.queries]
    queries, edges = dropin.make_queries(view.node_count, _entries(case, pols))
    pending = view.execute_batch(queries, edges)
    results, _, _, _ = pending.readback()
    pending.close()
    claimed = results["completion"] == DISCONNECTED
    for i, q in enumerate(case.queries):
        assert claimed[i] == (q.start_node != q.goal_node)
    got = _got(view.confirm_disconnected(queries, edges, results))
    assert got == _expect(case, pols, claimed)
    view.close()


def test_overflow_bound_matches_oracle():
    case = next(c for c in CASES if c.name == "disconnected_fields")
    view = dropin.View(case.header, case.layers, case.nodes, case.runs, case.run_nodes)
    q = case.queries[0]
    _, reached = oracle.disconnect_verdict(case.nodes, case.costs, q.start_node, q.goal_node,
                                           q.orthogonal_surcharge, q.diagonal_surcharge,
                                           q.bend_surcharge, q.policy)
    orth, diag, bend = case.costs
    base = max(orth + q.orthogonal_surcharge, diag + q.diagonal_surcharge) + bend + q.bend_surcharge
    limit = (U64_MAX - 1) // (8 * reached + 1)
    for extra, want in ((limit - base, "confirmed"), (limit - base + 1, "unbounded")):
        pen = np.zeros(1, dtype=ref_corpus.POLICY_EDGE_DTYPE)
        pen[0] = (len(case.nodes) * 8 + 7, 0, extra)
        pol = np.sort(np.concatenate([q.policy, pen]), order="physical_edge_index")
        queries, edges = dropin.make_queries(view.node_count, _entries(case, [pol] * len(case.queries)))
        results = np.zeros(len(queries), dtype=dropin.RESULT_DTYPE)
        results["completion"] = DISCONNECTED
        got = _got(view.confirm_disconnected(queries, edges, results))
        assert got[0] == (want, reached)
        assert got == _expect(case, [pol] * len(case.queries), [True] * len(case.queries))
    view.close()


def test_empty_and_unclaimed_batches():
    case = CASES[0]
    view = dropin.View(case.header, case.layers, case.nodes, case.runs, case.run_nodes)
    queries, edges = dropin.make_queries(view.node_count, _entries(case))
    results = np.zeros(len(queries), dtype=dropin.RESULT_DTYPE)  # all REACHED (0)
    got = _got(view.confirm_disconnected(queries, edges, results))
    assert got == [("not_claimed", 0)] * len(queries)
    assert len(view.confirm_disconnected(queries[:0], edges, results[:0])) == 0
    view.close()
