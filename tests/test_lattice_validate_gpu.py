"""GPU validation of lattice route results against the CPU restatement: the
engine's own frontier and sweep paths validate at exactly their cost, and
every corruption (of a path or its result record) gets the oracle's code and
failing index."""

import numpy as np
import pytest

import apgar_b200
import oracle
from apgar_b200 import synth
from tests.test_oracle_lattice_validate import _case, corrupt

pytestmark = pytest.mark.gpu

CODES = apgar_b200.LATTICE_PATH_CODES


@pytest.mark.parametrize("generator", ["frontier", "sweep"])
def test_engine_paths_validate(generator):
    lat, nets, costs, _ = _case()
    dev = apgar_b200.DeviceLattice(lat)
    try:
        res, paths = dev.route(nets, generator=generator)
        v = dev.validate(nets, res, paths)
        for i in range(len(nets)):
            if costs[i] == oracle.lo_inf():
                assert CODES[int(v[i]["code"])] == "not_reached"
            else:
                assert CODES[int(v[i]["code"])] == "ok", i
                assert int(v[i]["total_cost"]) == int(costs[i])
    finally:
        dev.close()


def test_medium_batch_validates():
    lat, nets = synth.config_medium(2, nets=512)
    dev = apgar_b200.DeviceLattice(lat)
    try:
        res, paths = dev.route(nets, generator="frontier")
        v = dev.validate(nets, res, paths)
        reached = res["completion"] == 0
        assert reached.sum() > 400
        assert (v["code"][reached] == 0).all()
        assert np.array_equal(v["total_cost"][reached], res["cost"][reached].astype(np.uint64))
    finally:
        dev.close()


def test_corruptions_match_the_oracle():
    lat, nets, costs, paths = _case()
    dev = apgar_b200.DeviceLattice(lat)
    try:
        recs, revs, sel = [], [], []
        for i, (net, c, p) in enumerate(zip(nets, costs, paths)):
            if c == oracle.lo_inf() or len(p) < 6:
                continue
            for kind in range(5):
                r, rev, _, _ = corrupt(lat, net, int(c), p, kind)
                recs.append(r)
                revs.append(np.asarray(rev, np.uint32))
                sel.append(i)
        results = np.array(recs, dtype=apgar_b200.RESULT_DTYPE)
        off = 0
        for k, rev in enumerate(revs):
            results[k]["path_offset"] = off
            results[k]["path_len"] = len(rev)
            off += len(rev)
        packed = np.concatenate(revs)
        # one more record whose path lies outside the packed array
        extra = results[:1].copy()
        extra[0]["path_offset"] = len(packed)
        results = np.concatenate([results, extra])
        sel.append(sel[0])
        v = dev.validate(np.ascontiguousarray(nets[sel]), results, packed)
        for k in range(len(revs)):
            code, idx, _ = oracle.validate_lattice_path(lat, nets[sel[k]], results[k], revs[k])
            assert CODES[int(v[k]["code"])] == code, (k, code)
            if code != "cost":
                assert int(v[k]["failing_index"]) == idx, (k, idx)
        assert CODES[int(v[-1]["code"])] == "bounds"
    finally:
        dev.close()
