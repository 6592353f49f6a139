"""GPU parity of the fused price kernel and the usage accumulation against
the CPU oracle (checked uint64 arithmetic; bit-exact)."""

import numpy as np
import pytest

import apgar_b200
import oracle
from apgar_b200 import prices, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("epoch", [0, 1, 7])
def test_price_update_matches_oracle(epoch):
    rng = np.random.default_rng(epoch)
    n = 100_003
    usage = rng.integers(0, 5, n).astype(np.uint32)
    history = rng.integers(0, 1000, n).astype(np.uint64)
    pol = prices.policy(capacity=1)
    present, hist, total, nxt, status = prices.update(usage, history, pol, epoch)
    assert status == 0
    rc, p_o, h_o, t_o = oracle.price_epoch_update(usage, history, 1, epoch)
    assert rc == 0
    assert np.array_equal(present, p_o) and np.array_equal(hist, h_o) and np.array_equal(total, t_o)
    rc, c_o = oracle.price_snapshot(usage, h_o, 1, epoch + 1, 100, 100, (1 << 64) - 1)
    assert rc == 0 and np.array_equal(nxt, c_o)


def test_price_known_answers_and_flags_on_gpu():
    pol = prices.policy(capacity=1)
    p, h, t, _, st = prices.update([2, 2], [0, 0], pol, 0)
    assert st == 0 and list(p) == [100, 100] and list(h) == [10, 10] and list(t) == [110, 110]
    p, h, t, _, st = prices.update([2, 2], h, pol, 1)
    assert list(p) == [200, 200] and list(h) == [20, 20] and list(t) == [220, 220]
    p, h, t, _, st = prices.update([1, 0], [10, 10], pol, 1)
    assert list(p) == [0, 0] and list(h) == [10, 10] and list(t) == [10, 10]
    # bound and overflow are reported, never silent
    _, _, _, _, st = prices.update([3], [0], prices.policy(capacity=1, maximum=5), 0)
    assert st & prices.PRICE_BOUND
    _, _, _, _, st = prices.update([3], [0], prices.policy(initial=2**63, capacity=1), 0)
    assert st & prices.PRICE_OVERFLOW


def test_usage_accumulation_matches_paths():
    lat, nets = synth.config_medium(9, nets=128, size=256)
    dev = apgar_b200.DeviceLattice(lat)
    plan = dev.plan(nets)
    plan.execute()
    results, paths = plan.readback()
    cells = lat.layers * lat.height * lat.width
    usage = prices.accumulate_usage(plan, cells)
    ok = results["completion"] == apgar_b200.COMPLETION_REACHED
    expect = oracle.accumulate_cells(results["path_offset"][ok], results["path_len"][ok], paths, cells)
    assert np.array_equal(usage, expect) and usage.sum() == results["path_len"][ok].sum()
    plan.close()
    dev.close()
