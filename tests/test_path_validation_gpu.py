"""GPU structural validation of compact paths (the device-view checks of the
reference's ValidateAndReconstructCompactGpuPath) against the CPU
restatement, on the reference corpus: the engine's own paths validate with
exactly the reference CPU A* cost, and corrupted paths and policies get the
same invariant code and failing index as the oracle."""

import numpy as np
import pytest

import oracle
from apgar_b200 import dropin
from tests.golden import ref_corpus

pytestmark = pytest.mark.gpu

CASES = ref_corpus.load_all()
U64_MAX = (1 << 64) - 1


def _entries(case):
    return [dict(start_node=q.start_node, goal_node=q.goal_node,
                 orthogonal_step_surcharge=q.orthogonal_surcharge,
                 diagonal_step_surcharge=q.diagonal_surcharge, bend_surcharge=q.bend_surcharge,
                 policy=q.policy, policy_identity=q.policy_identity) for q in case.queries]


def _corrupt(case, kind, rev, policy):
    """One corruption of a reverse path (or of its policy)."""
    n = len(case.nodes)
    rev = rev.copy()
    if kind == 0 or len(rev) < 4:
        return rev[:-1], policy                      # start state missing
    if kind == 1:
        rev[1] = rev[3]                              # repeated state
    elif kind == 2:
        node, h = divmod(int(rev[1]), 9)
        rev[1] = node * 9 + (h + 3) % 8              # wrong incoming heading
    elif kind == 3:
        rev[2] = 9 * n + 1                           # state out of range
    elif kind == 4:
        s0, s1 = int(rev[-1]), int(rev[-2])          # ban the first move's edge
        d, src = s1 % 9, s0 // 9
        edge = src * 8 + d if d < 4 else int(case.nodes[src]["neighbors"][d]) * 8 + d - 4
        ban = np.zeros(1, dtype=ref_corpus.POLICY_EDGE_DTYPE)
        ban[0] = (edge, 0, U64_MAX)
        keep = policy[policy["physical_edge_index"] != edge] if len(policy) else policy
        policy = np.sort(np.concatenate([keep, ban]), order="physical_edge_index")
    return rev, policy


@pytest.mark.parametrize("corrupt", [False, True])
@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_validation_matches_oracle(case, corrupt):
    view = dropin.View(case.header, case.layers, case.nodes, case.runs, case.run_nodes)
    queries, edges = dropin.make_queries(view.node_count, _entries(case))
    pending = view.execute_batch(queries, edges)
    results, compact, states, _ = pending.readback()
    pending.close()
    # per-query reverse paths and policies, optionally corrupted, then repacked
    revs, pols = [], []
    for i, q in enumerate(case.queries):
        c = compact[i]
        rev = states[int(c["state_offset"]): int(c["state_offset"]) + int(c["state_count"])]
        pol = q.policy
        if corrupt and results[i]["completion"] == 0:
            rev, pol = _corrupt(case, i % 5, rev, pol)
        revs.append(np.asarray(rev, np.uint32))
        pols.append(pol)
    q2 = queries.copy()
    c2 = compact.copy()
    off = poff = 0
    for i in range(len(revs)):
        c2[i]["state_offset"] = off
        c2[i]["state_count"] = len(revs[i])
        off += len(revs[i])
        q2[i]["policy_offset"] = poff
        q2[i]["policy_count"] = len(pols[i])
        poff += len(pols[i])
    packed = np.concatenate(revs) if off else np.zeros(0, np.uint32)
    pol_all = (np.concatenate([p for p in pols if len(p)]).astype(ref_corpus.POLICY_EDGE_DTYPE)
               if poff else np.zeros(0, ref_corpus.POLICY_EDGE_DTYPE))
    verdicts = view.validate_compact_paths(q2, pol_all, results, c2, packed)
    view.close()
    for i, q in enumerate(case.queries):
        code, total, index = oracle.validate_compact(
            case.nodes, case.costs, q.start_node, q.goal_node, revs[i], int(results[i]["goal_state"]),
            int(results[i]["completion"]), q.orthogonal_surcharge, q.diagonal_surcharge,
            q.bend_surcharge, pols[i])
        v = verdicts[i]
        assert dropin.PATH_CODES[int(v["code"])] == code, (case.name, i)
        if code == "ok":
            assert int(v["total_cost"]) == total
            if not corrupt:
                assert total == q.cpu_cost  # the reference CPU A* cost
        elif code not in ("not_reached", "bounds", "endpoint"):
            assert int(v["failing_index"]) == index, (case.name, i)
    if corrupt:
        reached = results["completion"] == 0
        assert (verdicts["code"][reached] != 0).all()
