"""CPU pin of the segment restatement (oracle.coalesce_segments) to the
reference's own routing::CoalesceSegments outputs on the golden corpus
(tests/golden/ref_corpus/segments.bin, written by oracle/ref_fixtures.cc)."""

import numpy as np

import oracle
from golden import ref_corpus as rc


def test_restatement_reproduces_reference_segments():
    cases = {c.name: c for c in rc.load_all()}
    records = rc.load_segments()
    assert len(records) > 100
    for name, query, nodes, segs in records:
        case = cases[name]
        h = case.header[0]
        nd = case.nodes[nodes]
        pts = oracle.exact_points(h["lattice_origin_x"], h["lattice_origin_y"], h["lattice_step"],
                                  nd["lattice_x"], nd["lattice_y"])
        assert pts is not None
        got = oracle.coalesce_segments(pts[0], pts[1], nd["layer"])
        assert len(got) == len(segs), (name, query)
        for field_got, field_ref in (("x0", "x0"), ("y0", "y0"), ("x1", "x1"), ("y1", "y1")):
            assert np.array_equal(got[field_got], segs[field_ref]), (name, query)
        assert np.array_equal(got["layer0"], segs["layer"])


def test_coalesce_splits_on_layer_steps():
    xs = np.array([0, 10, 20, 20, 20, 30], np.int64)
    ys = np.zeros(6, np.int64)
    layers = np.array([0, 0, 0, 1, 2, 2])
    segs = oracle.coalesce_segments(xs, ys, layers)
    assert segs[["layer0", "layer1", "x0", "x1"]].tolist() == [(0, 0, 0, 20), (0, 2, 20, 20),
                                                                (2, 2, 20, 30)]
    assert len(oracle.coalesce_segments(xs[:1], ys[:1], layers[:1])) == 0
