"""GPU checks of the allocation-free lattice route (apgar_b200_lattice_route_noalloc).

The entry point must return exactly what apgar_b200_lattice_route returns on
the same nets, on consecutive calls through the same fixed scratch, and must
refuse batches larger than the scratch with a clear error.  This file is named
to be collected last, so it also runs after every other GPU test has used the
device."""

import numpy as np
import pytest

import apgar_b200
from apgar_b200 import synth

pytestmark = pytest.mark.gpu


def _same(a, b):
    res_a, paths_a = a
    res_b, paths_b = b
    assert np.array_equal(res_a, res_b)
    assert np.array_equal(paths_a, paths_b)


def _check_against_route(lat, batches):
    dev = apgar_b200.DeviceLattice(lat)
    try:
        expected = [dev.route(nets) for nets in batches]
        # two calls in a row through the same scratch, each against route()
        for nets, want in zip(batches, expected):
            _same(dev.route_noalloc(nets), want)
        for nets, want in zip(batches, expected):
            _same(dev.route_noalloc(nets), want)
    finally:
        dev.close()
    return expected


def test_matches_route_on_consecutive_calls():
    lat, nets = synth.config_medium(7, nets=64, size=256)
    small_lat, small_nets = synth.config_small(1)
    expected = _check_against_route(lat, [nets, nets[::-1].copy()])
    reached = expected[0][0]["completion"] == apgar_b200.COMPLETION_REACHED
    assert reached.sum() > len(nets) // 2
    _check_against_route(small_lat, [small_nets[:24].copy(), small_nets[24:40].copy()])


def test_no_device_memory_is_allocated():
    torch = pytest.importorskip("torch")
    lat, nets = synth.config_medium(7, nets=64, size=256)
    dev = apgar_b200.DeviceLattice(lat)
    try:
        results = np.empty(len(nets), dtype=apgar_b200.RESULT_DTYPE)
        paths = np.empty(1 << 20, dtype=np.uint32)
        first = dev.route_noalloc(nets, out=(results, paths))
        first = (first[0].copy(), first[1].copy())
        free_before, _ = torch.cuda.mem_get_info()
        for _ in range(3):
            _same(dev.route_noalloc(nets, out=(results, paths)), first)
        free_after, _ = torch.cuda.mem_get_info()
        assert free_after == free_before
    finally:
        dev.close()


def test_batch_beyond_scratch_is_refused():
    lat, nets = synth.config_small(1)  # about 34 MiB of label slabs and arena
    dev = apgar_b200.DeviceLattice(lat)
    try:
        with pytest.raises(apgar_b200.BackendError) as err:
            dev.route_noalloc(nets)
        assert err.value.code == 2
        assert "scratch" in err.value.detail
        too_many = np.repeat(nets[:1], apgar_b200.NOALLOC_MAX_NETS + 1)
        with pytest.raises(apgar_b200.BackendError) as err:
            dev.route_noalloc(too_many)
        assert err.value.code == 2
        # the scratch is still usable after a refusal
        _same(dev.route_noalloc(nets[:8].copy()), dev.route(nets[:8].copy()))
    finally:
        dev.close()
