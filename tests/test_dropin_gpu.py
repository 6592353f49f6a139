"""GPU parity of the drop-in seam (reference device view, heading states,
policies) through the C ABI, against the reference's own corpus.

Per query: reached / disconnected as the reference CPU A*; the compact reverse
path equal to the canonical path of the exact labels (oracle) and its cost
equal to the reference CPU A* cost; in the full-workspace form every label
equal to the exact label and every predecessor equal to the canonical rule."""

import numpy as np
import pytest

import apgar_b200
import oracle
from apgar_b200 import dropin
from tests.golden import ref_corpus

pytestmark = pytest.mark.gpu

CASES = ref_corpus.load_all()
U64_MAX = (1 << 64) - 1


def _view(case):
    return dropin.View(case.header, case.layers, case.nodes, case.runs, case.run_nodes)


def _entries(case):
    return [dict(start_node=q.start_node, goal_node=q.goal_node,
                 orthogonal_step_surcharge=q.orthogonal_surcharge,
                 diagonal_step_surcharge=q.diagonal_surcharge, bend_surcharge=q.bend_surcharge,
                 policy=q.policy, policy_identity=q.policy_identity) for q in case.queries]


@pytest.mark.parametrize("generator", [dropin.GENERATOR_SWEEP, dropin.GENERATOR_PERSISTENT])
@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_compact_paths_match_reference(case, generator):
    view = _view(case)
    queries, edges = dropin.make_queries(view.node_count, _entries(case), generator=generator)
    pending = view.execute_batch(queries, edges, generator=generator)
    results, compact, states, tel = pending.readback()
    pending.close()
    assert tel.kernel_launch_count == 3 and tel.blocking_status_readback_count == 0
    offset = 0
    for i, q in enumerate(case.queries):
        r, c = results[i], compact[i]
        assert r["query_id"] == i + 1 and r["workspace_owner"] == i + 1 and r["generator"] == generator
        assert c["state_offset"] == offset
        offset += int(c["state_count"])
        reached, cost, goal_state, path, _ = oracle.graph_search(
            case.nodes, case.costs, q.start_node, q.goal_node, q.orthogonal_surcharge,
            q.diagonal_surcharge, q.bend_surcharge, q.policy)
        if q.cpu_status == 1:
            assert r["completion"] == apgar_b200.COMPLETION_DISCONNECTED and c["state_count"] == 0
            continue
        assert q.cpu_status == 0
        assert r["completion"] == apgar_b200.COMPLETION_REACHED, i
        assert r["goal_state"] == goal_state, i
        got = states[int(c["state_offset"]): int(c["state_offset"]) + int(c["state_count"])]
        assert np.array_equal(got, path), i
        assert cost == q.cpu_cost
    assert offset == len(states)
    view.close()


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_full_workspace_labels_and_predecessors(case):
    view = _view(case)
    queries, edges = dropin.make_queries(view.node_count, _entries(case),
                                         generator=dropin.GENERATOR_FRONTIER)
    pending = view.execute_batch(queries, edges, generator=dropin.GENERATOR_FRONTIER)
    results, _, _, tel = pending.readback()
    labels, preds, owners, powners = pending.readback_workspace()
    pending.close()
    S = 9 * view.node_count
    for i, q in enumerate(case.queries):
        _, _, _, _, exact = oracle.graph_search(
            case.nodes, case.costs, q.start_node, q.goal_node, q.orthogonal_surcharge,
            q.diagonal_surcharge, q.bend_surcharge, q.policy, want_labels=True)
        sl = slice(i * S, (i + 1) * S)
        assert np.array_equal(labels[sl], exact), i
        canon = oracle.graph_predecessors(case.nodes, case.costs, q.start_node, exact,
                                          q.orthogonal_surcharge, q.diagonal_surcharge,
                                          q.bend_surcharge, q.policy)
        assert np.array_equal(preds[sl], canon), i
        assert (owners[sl] == i + 1).all() and (powners[sl] == i + 1).all()
    view.close()


def test_single_route_pair_matches_exact_labels():
    case = next(c for c in CASES if c.name == "kicad_fixture")
    view = _view(case)
    q = case.queries[0]
    pending = view.execute_route(q.start_node, q.goal_node, generator=dropin.GENERATOR_SWEEP,
                                 routing_profile_fingerprint=77)
    header, completion, goal_state, labels, preds, _ = pending.readback()
    pending.close()
    _, cost, exact_goal, _, exact = oracle.graph_search(case.nodes, case.costs, q.start_node,
                                                        q.goal_node, want_labels=True)
    assert completion == apgar_b200.COMPLETION_REACHED and goal_state == exact_goal
    assert np.array_equal(labels, exact)
    assert header["routing_profile_fingerprint"] == 77 and header["start_node"] == q.start_node
    assert cost == 37168
    view.close()


def test_budget_exhaustion_and_admission_errors():
    case = next(c for c in CASES if c.name == "dense_corridors")
    view = _view(case)
    queries, edges = dropin.make_queries(view.node_count, _entries(case)[:3], maximum_rounds=1)
    pending = view.execute_batch(queries, edges, maximum_rounds=1)
    results, compact, _, _ = pending.readback()
    pending.close()
    assert (results["completion"] == apgar_b200.COMPLETION_BUDGET_EXHAUSTED).all()
    assert (compact["state_count"] == 0).all()
    # non-ascending query ids are rejected before any launch
    bad, edges = dropin.make_queries(view.node_count, _entries(case)[:2])
    bad["query_id"] = [5, 3]
    with pytest.raises(apgar_b200.BackendError) as err:
        view.execute_batch(bad, edges)
    assert err.value.code == 4
    # a device budget below the workspace is resource exhaustion
    ok, edges = dropin.make_queries(view.node_count, _entries(case)[:2])
    with pytest.raises(apgar_b200.BackendError) as err:
        view.execute_batch(ok, edges, maximum_device_bytes=1024)
    assert err.value.code == 2
    view.close()
