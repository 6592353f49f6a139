"""The frontier schedule autotuner on a B200: every candidate schedule gives
the same costs and paths (the oracle's), the chosen one is a candidate, and
invalid class limits are refused."""

import numpy as np
import pytest

import apgar_b200
import oracle
from apgar_b200 import autotune, synth

pytestmark = pytest.mark.gpu


def test_tuned_schedule_keeps_results():
    lat = synth.make_lattice(21, 4, 512, 0.25, pads=True)
    nets = synth.make_nets(lat, 22, 256, hpwl_median=120.0, hpwl_sigma=1.0)
    cost_o, paths_o = oracle.dijkstra_batch(lat, nets)
    dev = apgar_b200.DeviceLattice(lat)
    try:
        best, table = autotune.tune(dev, nets, use_cache=False)
        assert 1 + 3 + (len(autotune.BOUND_SETS) - 1) + 1 <= len(table) <= 1 + 3 + (
            len(autotune.BOUND_SETS) - 1) + 8 * autotune.REFINE_STEPS + 1
        assert best.describe() in [row[0] for row in table]
        assert autotune.tune(dev, nets)[0] == best  # cached
        for s in (best, autotune.Schedule(bucket_width=400, chain=3,
                                          class_bounds=apgar_b200.class_bounds(10, 12, 14, 16))):
            res, paths = dev.route(nets, generator="frontier", schedule=s)
            assert np.array_equal(res["cost"], cost_o)
            per = apgar_b200.split_paths(res, paths)
            for i in range(len(nets)):
                if cost_o[i] != oracle.lo_inf():
                    assert np.array_equal(per[i], paths_o[i]), i
        for bad in (apgar_b200.class_bounds(12, 12, 17, 20), apgar_b200.class_bounds(12, 15, 17, 32),
                    apgar_b200.class_bounds(0, 15, 17, 20)):
            with pytest.raises(apgar_b200.BackendError):
                dev.plan(nets[:4].copy(), generator="frontier", class_bounds=bad)
    finally:
        dev.close()
