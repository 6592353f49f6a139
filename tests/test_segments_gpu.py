"""GPU route reconstruction (apgar_b200_path_segments, apgar_b200_lattice_segments)
through the C ABI.

V1 form: the reference CPU A* routes of the golden corpus, fed as compact
paths, come back as exactly the reference's routing::CoalesceSegments output.
Lattice form: the frontier's paths on multi-layer lattices with vias give the
segments of the restatement oracle.coalesce_segments, bit for bit."""

import numpy as np
import pytest

import apgar_b200
import oracle
from apgar_b200 import dropin, synth
from tests.golden import ref_corpus

pytestmark = pytest.mark.gpu


def test_v1_paths_give_the_reference_segments():
    cases = {c.name: c for c in ref_corpus.load_all()}
    records = ref_corpus.load_segments()
    by_case = {}
    for rec in records:
        by_case.setdefault(rec[0], []).append(rec)
    checked = 0
    for name, recs in by_case.items():
        case = cases[name]
        view = dropin.View(case.header, case.layers, case.nodes, case.runs, case.run_nodes)
        try:
            compact = np.zeros(len(recs), dtype=dropin.COMPACT_DTYPE)
            states, at = [], 0
            for i, (_, _, nodes, _) in enumerate(recs):
                rev = nodes[::-1].astype(np.uint32) * 9 + 8  # goal first; heading unused
                compact[i]["state_count"] = len(rev)
                compact[i]["state_offset"] = at
                states.append(rev)
                at += len(rev)
            segs, counts = view.path_segments(compact, np.concatenate(states))
            for i, (_, q, _, ref) in enumerate(recs):
                got = segs[int(compact[i]["state_offset"]):][: int(counts[i])]
                assert counts[i] == len(ref), (name, q)
                for f in ("x0", "y0", "x1", "y1"):
                    assert np.array_equal(got[f], ref[f]), (name, q, f)
                assert np.array_equal(got["layer0"], ref["layer"])
                assert np.array_equal(got["layer1"], ref["layer"])
                checked += 1
        finally:
            view.close()
    assert checked == len(records)


def test_v1_paths_outside_the_view_fail():
    case = ref_corpus.load_all()[0]
    view = dropin.View(case.header, case.layers, case.nodes, case.runs, case.run_nodes)
    try:
        compact = np.zeros(2, dtype=dropin.COMPACT_DTYPE)
        compact[0]["state_count"], compact[0]["state_offset"] = 2, 0
        compact[1]["state_count"], compact[1]["state_offset"] = 3, 5  # past the states
        states = np.array([9 * len(case.nodes) + 1, 8], np.uint32)  # first state out of range
        _, counts = view.path_segments(compact, states)
        assert counts.tolist() == [dropin.SEGMENT_FAILURE, dropin.SEGMENT_FAILURE]
    finally:
        view.close()


@pytest.mark.parametrize("origin,step", [((0, 0), 1), ((-12345, 678), 25)])
def test_lattice_paths_match_the_restatement(origin, step):
    lat = synth.make_lattice(81, 3, 256, 0.2, via_mask=True)
    nets = synth.make_nets(lat, 82, 96, hpwl_median=60.0, hpwl_sigma=0.7, margin=16)
    dev = apgar_b200.DeviceLattice(lat)
    try:
        plan = dev.plan(nets, generator="frontier")
        plan.execute()
        res, paths = plan.readback()
        segs_t, counts_t = plan.segments(origin[0], origin[1], step)
        segs = segs_t.cpu().numpy().view(dropin.SEGMENT_DTYPE)
        counts = counts_t.cpu().numpy().view(np.uint32)
        per = apgar_b200.split_paths(res, paths)
        vias = 0
        for i in range(len(nets)):
            if res["completion"][i] != apgar_b200.COMPLETION_REACHED:
                assert counts[i] == 0
                continue
            fwd = per[i][::-1].astype(np.int64)
            x = fwd % lat.width
            y = (fwd // lat.width) % lat.height
            layer = fwd // (lat.width * lat.height)
            pts = oracle.exact_points(origin[0], origin[1], step, x, y)
            want = oracle.coalesce_segments(pts[0], pts[1], layer)
            got = segs[int(res["path_offset"][i]):][: int(counts[i])]
            assert len(got) == len(want), i
            assert got.tolist() == want.tolist(), i
            vias += int((want["layer0"] != want["layer1"]).sum())
        assert vias > 0  # the batch exercises via runs
        plan.close()
    finally:
        dev.close()
