"""The reference's GPU replay artifacts (replays/gpu/*.replay, summarised in
tests/golden/replay_invariants.json) name the invariant id its host
validation raises for each injected fault.  For the faults that the device
validators of this backend cover, the same corruption (restated from the
reference's fault-injecting backend, src/gpu/fault_injecting_backend.cc:
161-233) of this engine's result for the replays' KiCad query raises the same
invariant id."""

import json
import os

import numpy as np
import pytest

from apgar_b200 import dropin
from tests.golden import ref_corpus

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "replay_invariants.json")) as _f:
    REPLAYS = json.load(_f)
DEVICE_FAULTS = ("compact_path_bounds", "compact_path_endpoint", "compact_path_cycle",
                 "compact_path_heading", "compact_path_edge", "false_disconnected")
INVARIANT = {1: "gpu.batch.compact_path.bounds.v1", 2: "gpu.batch.compact_path.endpoint.v1",
             3: "gpu.batch.compact_path.cycle.v1", 4: "gpu.batch.compact_path.heading.v1",
             5: "gpu.batch.compact_path.edge.v1", 6: "gpu.policy.banned_predecessor.v1"}
INVALID_STATE = 0xFFFFFFFF


def inject(fault, results, compact, states, start_node):
    """One fault of the reference's fault-injecting backend on query 0."""
    results, compact, states = results.copy(), compact.copy(), states.copy()
    o, n = int(compact[0]["state_offset"]), int(compact[0]["state_count"])
    s = states[o:o + n]  # a view: edits land in `states`
    if fault == "false_disconnected":
        results[0]["completion"] = 1
        results[0]["goal_state"] = INVALID_STATE
    elif fault == "compact_path_bounds":
        v = int(compact[0]["schema_version"])
        compact[0]["schema_version"] = v - 1 if v == 0xFFFFFFFF else v + 1
    elif fault == "compact_path_endpoint":
        if n:
            s[0] = INVALID_STATE
    elif fault == "compact_path_cycle":
        if n >= 4:
            s[1] = s[2]
    elif fault == "compact_path_heading":
        for i in range(1, n - 1):
            node = int(s[i]) // 9
            repl = node * 9 + 8
            if node != start_node and repl not in s:
                s[i] = repl
                break
    elif fault == "compact_path_edge":
        done = False
        for i in range(1, n - 1):
            node, h = divmod(int(s[i]), 9)
            for heading in range(8):
                repl = node * 9 + heading
                if heading != h and repl not in s:
                    s[i] = repl
                    done = True
                    break
            if done:
                break
    return results, compact, states


@pytest.mark.parametrize("replay", [r for r in REPLAYS if r["fault"] in DEVICE_FAULTS],
                         ids=lambda r: r["replay"])
def test_device_validation_raises_the_replay_invariant(replay):
    case = next(c for c in ref_corpus.load_all() if c.name == "kicad_fixture")
    q = case.queries[0]
    assert q.cpu_status == 0 and q.cpu_cost == 37168  # the replays' base request
    view = dropin.View(case.header, case.layers, case.nodes, case.runs, case.run_nodes)
    try:
        queries, edges = dropin.make_queries(view.node_count, [dict(
            start_node=q.start_node, goal_node=q.goal_node, policy=q.policy,
            policy_identity=q.policy_identity)])
        pending = view.execute_batch(queries, edges)
        results, compact, states, _ = pending.readback()
        pending.close()
        ok = view.validate_compact_paths(queries, edges, results, compact, states)
        assert int(ok[0]["code"]) == 0 and int(ok[0]["total_cost"]) == 37168
        results, compact, states = inject(replay["fault"], results, compact, states, q.start_node)
        if replay["fault"] == "false_disconnected":
            v = view.confirm_disconnected(queries, edges, results)
            assert dropin.DISCONNECT_CODES[int(v[0]["code"])] == "reachable"
            assert replay["expected_invariant"] == "gpu.disconnected.cpu_reachable.v1"
        else:
            v = view.validate_compact_paths(queries, edges, results, compact, states)
            assert INVARIANT.get(int(v[0]["code"])) == replay["expected_invariant"], int(v[0]["code"])
        assert replay["expected_failure"] == "internal_invariant"
    finally:
        view.close()
