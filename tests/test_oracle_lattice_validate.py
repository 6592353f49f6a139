"""CPU pin of the lattice-path validation restatement: the oracle's own exact
paths validate at exactly their cost, and each corruption of a path or its
result record gets its code at the right forward index."""

import numpy as np

import apgar_b200
import oracle
from apgar_b200 import synth


def _case():
    lat = synth.make_lattice(31, 2, 128, 0.15, via_mask=True)
    nets = synth.make_nets(lat, 32, 24, hpwl_median=40.0, hpwl_sigma=0.5, margin=8)
    costs, paths = oracle.dijkstra_batch(lat, nets)
    return lat, nets, costs, paths


def _result(cost, n):
    r = np.zeros(1, dtype=apgar_b200.RESULT_DTYPE)[0]
    r["completion"] = 0 if cost != oracle.lo_inf() else 1
    r["cost"] = cost if cost != oracle.lo_inf() else 0xFFFFFFFF
    r["path_len"] = n
    return r


def corrupt(lat, net, cost, rev, kind):
    """One corruption of a reverse path (goal first) or of its cost; returns
    (result record, reverse path, expected code, expected forward index)."""
    rev = [int(c) for c in rev]
    n = len(rev)
    if kind == 0:                                   # start cell missing
        rev = rev[:-1]
        return _result(cost, len(rev)), rev, "endpoint", 0
    if kind == 1:                                   # goal replaced
        rev[0] = rev[1] if n > 1 else rev[0] + 1
        return _result(cost, n), rev, "endpoint", n - 1
    if kind == 2:                                   # a middle cell jumps away
        k = n // 2
        W = lat.width
        l, rem = divmod(rev[k], lat.width * lat.height)
        y, x = divmod(rem, W)
        x2 = x + 3 if x + 3 < int(net["win_x0"]) + int(net["win_w"]) else x - 3
        rev[k] = (l * lat.height + y) * W + x2
        return _result(cost, n), rev, "edge", n - 1 - k
    if kind == 3:                                   # wrong cost
        return _result(cost + 1, n), rev, "cost", 0
    # a cell outside the window
    k = n // 2
    l, rem = divmod(rev[k], lat.width * lat.height)
    rev[k] = (l * lat.height + int(net["win_y0"])) * lat.width + (int(net["win_x0"]) - 1) \
        if int(net["win_x0"]) > 0 else rev[k] + lat.width * lat.height * lat.layers
    return _result(cost, n), rev, "bounds", n - 1 - k


def test_oracle_paths_validate_at_their_cost():
    lat, nets, costs, paths = _case()
    reached = 0
    for net, c, p in zip(nets, costs, paths):
        if c == oracle.lo_inf():
            code, _, _ = oracle.validate_lattice_path(lat, net, _result(c, 0), [])
            assert code == "not_reached"
            continue
        reached += 1
        code, idx, total = oracle.validate_lattice_path(lat, net, _result(c, len(p)), p)
        assert (code, idx, total) == ("ok", 0, int(c))
    assert reached >= 20


def test_corruptions_get_their_codes():
    lat, nets, costs, paths = _case()
    seen = set()
    for i, (net, c, p) in enumerate(zip(nets, costs, paths)):
        if c == oracle.lo_inf() or len(p) < 6:
            continue
        for kind in range(5):
            r, rev, want, index = corrupt(lat, net, int(c), p, kind)
            code, idx, _ = oracle.validate_lattice_path(lat, net, r, rev)
            assert code == want, (i, kind, code)
            if want != "cost":
                assert idx == index, (i, kind, idx, index)
            seen.add(code)
    assert seen == {"endpoint", "edge", "cost", "bounds"}
