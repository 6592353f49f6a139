"""CPU pins of the geometry-compile restatement: the exact swept-trace
clearance predicate against the reference's own verdicts on seeded cases,
and the legal-edge masks of every corpus device view."""

import oracle
from golden import ref_corpus as rc


def test_clearance_predicate_matches_the_reference():
    cases = rc.load_clearance()
    assert len(cases) >= 10000 and 0.2 < cases["satisfied"].mean() < 0.8
    for c in cases:
        err, sat = oracle.swept_clearance(tuple(c["start"]), tuple(c["end"]), tuple(c["box_min"]),
                                          tuple(c["box_max"]), int(c["width"]), int(c["clearance"]))
        assert (err, int(sat)) == (int(c["error"]), int(c["satisfied"])), c


def test_corpus_legal_edges_are_reproduced():
    geo = rc.load_geometry()
    for case in rc.load_all():
        g = geo[case.name]
        n = case.nodes
        masks = oracle.compile_legal_edges(n["lattice_x"], n["lattice_y"], n["layer"], g["origin"],
                                           g["step"], g["heading_mask"], g["width"], g["clearance"],
                                           [tuple(o) for o in g["obstacles"]])
        assert (masks == n["legal_edges"]).all(), case.name
