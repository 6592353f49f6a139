"""Host logic of the frontier schedule autotuner: the packed class limits,
workload signatures, the stratified sample and the saved choices."""

import numpy as np
import pytest

import apgar_b200
from apgar_b200 import autotune, synth


def test_class_bounds_packing():
    assert apgar_b200.class_bounds() == 0
    word = apgar_b200.class_bounds(12, 15, 17, 20)
    assert word == 0x14110F0C
    assert autotune.Schedule(class_bounds=word).describe()["class_log2_limits"] == [12, 15, 17, 20]
    assert autotune.DEFAULT.describe() == {"bucket_width": 0, "chain": 0, "class_log2_limits": None,
                                           "wide_bucket_width": 0, "wide_chain": 0}
    with pytest.raises(ValueError):
        apgar_b200.class_bounds(12, 15)
    for bounds in autotune.BOUND_SETS:
        assert list(bounds) == sorted(set(bounds)) and 1 <= bounds[0] and bounds[-1] <= 31


class _Lat:
    layers, height, width = 4, 512, 512


def test_signature_and_sample():
    lat = synth.make_lattice(3, 2, 256, 0.2)
    nets = synth.make_nets(lat, 4, 300, hpwl_median=60.0, hpwl_sigma=1.0, margin=16)
    assert autotune.signature(_Lat, nets) == autotune.signature(_Lat, nets.copy())
    assert autotune.signature(_Lat, nets) != autotune.signature(_Lat, nets[:200])
    sample = autotune._sample(nets, 50, seed=1)
    assert len(sample) == 50
    assert np.array_equal(sample, autotune._sample(nets, 50, seed=1))
    # every sampled net is a net of the batch, and the size range is kept
    cells = lambda a: a["win_w"].astype(np.int64) * a["win_h"].astype(np.int64)
    assert set(map(bytes, sample.view(np.uint8).reshape(len(sample), -1))) <= \
        set(map(bytes, nets.view(np.uint8).reshape(len(nets), -1)))
    assert cells(sample).max() == cells(nets).max() or cells(sample).max() >= np.quantile(cells(nets), 0.95)
    assert autotune._sample(nets, None, 0) is not None and len(autotune._sample(nets, 1000, 0)) == len(nets)


def test_save_and_load(tmp_path):
    key = "test-key"
    autotune._CACHE[key] = (autotune.Schedule(bucket_width=200, chain=2,
                                              class_bounds=apgar_b200.class_bounds(12, 15, 18, 21)), [])
    path = str(tmp_path / "schedules.json")
    autotune.save(path)
    del autotune._CACHE[key]
    autotune.load(path)
    assert autotune._CACHE[key][0] == autotune.Schedule(200, 2, apgar_b200.class_bounds(12, 15, 18, 21))
    del autotune._CACHE[key]


class _FakeLattice:
    layers, height, width = 4, 512, 512
    orth, diag, via = 10, 14, 50


def _fake_timer(table):
    """time_schedule stand-in: ms from `table` keyed by the schedule's
    describe(), the same costs for every schedule."""
    def timer(lattice, nets, s, warmup=1, reps=5):
        d = s.describe()
        key = (d["bucket_width"], d["chain"], tuple(d["class_log2_limits"] or ()))
        return table.get(key, 20.0), np.arange(len(nets), dtype=np.uint32)
    return timer


def test_coordinate_descent_keeps_gains_above_the_noise(monkeypatch):
    lat = synth.make_lattice(3, 2, 256, 0.2)
    nets = synth.make_nets(lat, 4, 50, hpwl_median=40.0, hpwl_sigma=1.0, margin=16)
    table = {
        (0, 0, ()): 20.0,
        (200, 0, ()): 19.9,                 # 0.5% better: noise, not taken
        (400, 0, ()): 25.0,
        (0, 0, (12, 15, 18, 21)): 18.0,     # 10% better: taken
        (0, 0, (12, 15, 18, 20)): 17.0,     # one refinement step further
        (0, 2, (12, 15, 18, 20)): 16.9,     # chaining within the noise: not taken
    }
    monkeypatch.setattr(autotune, "time_schedule", _fake_timer(table))
    best, rows = autotune.tune(_FakeLattice, nets, use_cache=False)
    assert best == autotune.Schedule(0, 0, apgar_b200.class_bounds(12, 15, 18, 20))
    assert rows[0][0] == autotune.DEFAULT.describe()
    assert len(rows) >= 1 + 3 + len(autotune.BOUND_SETS) - 1 + 1


def test_a_schedule_that_changes_a_result_raises(monkeypatch):
    lat = synth.make_lattice(3, 2, 256, 0.2)
    nets = synth.make_nets(lat, 4, 20, hpwl_median=40.0, hpwl_sigma=1.0, margin=16)
    calls = []

    def timer(lattice, nets_, s, warmup=1, reps=5):
        calls.append(s)
        cost = np.zeros(len(nets_), np.uint32)
        if len(calls) == 3:
            cost[0] = 1  # the third candidate disagrees
        return 20.0, cost

    monkeypatch.setattr(autotune, "time_schedule", timer)
    with pytest.raises(RuntimeError):
        autotune.tune(_FakeLattice, nets, use_cache=False)
