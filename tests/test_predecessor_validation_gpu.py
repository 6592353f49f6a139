"""GPU validation of full-workspace results (the checks of the reference's
ValidateAllPredecessors) against the CPU restatement: the engine's own
workspaces validate, every corruption gets the oracle's code and first
failing state, and the reference's goal-predecessor self-cycle replay fault
raises its invariant (gpu.predecessor.self_reference.v1)."""

import json
import os

import numpy as np
import pytest

import oracle
from apgar_b200 import dropin
from tests.golden import ref_corpus
from tests.test_oracle_predecessors import corruptions

pytestmark = pytest.mark.gpu

CASES = ref_corpus.load_all()
HERE = os.path.dirname(os.path.abspath(__file__))


def _entries(case):
    return [dict(start_node=q.start_node, goal_node=q.goal_node,
                 orthogonal_step_surcharge=q.orthogonal_surcharge,
                 diagonal_step_surcharge=q.diagonal_surcharge, bend_surcharge=q.bend_surcharge,
                 policy=q.policy, policy_identity=q.policy_identity) for q in case.queries]


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_workspaces_validate_and_corruptions_match_the_oracle(case):
    view = dropin.View(case.header, case.layers, case.nodes, case.runs, case.run_nodes)
    try:
        queries, edges = dropin.make_queries(view.node_count, _entries(case),
                                             generator=dropin.GENERATOR_FRONTIER)
        pending = view.execute_batch(queries, edges, generator=dropin.GENERATOR_FRONTIER)
        labels, preds, _, _ = pending.readback_workspace()
        pending.close()
        S = 9 * view.node_count
        labels = labels.reshape(len(queries), S)
        preds = preds.reshape(len(queries), S)
        v = view.validate_predecessors(queries, edges, labels, preds)
        assert (v["code"] == 0).all(), v["code"]
        # corruptions, one per query row, checked against the oracle
        rows_l, rows_p, rows_q, want = [], [], [], []
        for i, q in enumerate(case.queries):
            for _, L, P, _, _ in corruptions(case, q, labels[i], preds[i]):
                rows_l.append(L)
                rows_p.append(P)
                rows_q.append(i)
                want.append(oracle.validate_predecessors(
                    case.nodes, case.costs, q.start_node, L, P, q.orthogonal_surcharge,
                    q.diagonal_surcharge, q.bend_surcharge, q.policy))
        if not rows_q:
            return
        v = view.validate_predecessors(queries[rows_q], edges, np.stack(rows_l), np.stack(rows_p))
        got = [(dropin.PRED_CODES[int(x["code"])], int(x["failing_index"])) for x in v]
        assert got == want
    finally:
        view.close()


def test_goal_predecessor_self_cycle_replay():
    with open(os.path.join(HERE, "golden", "replay_invariants.json")) as f:
        replays = [r for r in json.load(f) if r["fault"] == "goal_predecessor_self_cycle"]
    assert len(replays) == 2
    case = next(c for c in CASES if c.name == "kicad_fixture")
    q = case.queries[0]
    view = dropin.View(case.header, case.layers, case.nodes, case.runs, case.run_nodes)
    try:
        pending = view.execute_route(q.start_node, q.goal_node)
        _, completion, goal_state, labels, preds, _ = pending.readback()
        pending.close()
        assert completion == 0
        queries, edges = dropin.make_queries(view.node_count, [dict(start_node=q.start_node,
                                                                    goal_node=q.goal_node)])
        assert int(view.validate_predecessors(queries, edges, labels[None], preds[None])[0]["code"]) == 0
        preds = preds.copy()
        preds[goal_state] = goal_state  # the reference's fault: the goal points at itself
        v = view.validate_predecessors(queries, edges, labels[None], preds[None])[0]
        assert dropin.PRED_CODES[int(v["code"])] == "self_reference"
        assert int(v["failing_index"]) == goal_state
        for r in replays:
            assert r["expected_invariant"] == "gpu.predecessor.self_reference.v1"
    finally:
        view.close()
