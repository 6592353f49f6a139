"""CPU pin of the congestion-price oracle against the reference's own
known-answer tests (values, not code):
  tests/allocator/negotiated_regeneration_plan_test.cc:816-845 (epoch 0:
  present 100 / history 10 / total 110; epoch 1: 200 / 20 / 220),
  :847-874 (history 10 persists when overuse drops to 0),
  tests/allocator/cpu_sequential_negotiated_routing_test.cc:787-831
  (zero-capacity snapshot: present 7, merged with the base penalty 5 -> 12;
  a bound of 11 is exceeded)."""

import numpy as np

import oracle


def test_epoch_schedule_known_answers():
    usage = np.array([2, 2, 2], np.uint64)  # two users of capacity-1 resources
    rc, p0, h0, t0 = oracle.price_epoch_update(usage, np.zeros(3), 1, 0)
    assert rc == 0 and (p0 == 100).all() and (h0 == 10).all() and (t0 == 110).all()
    rc, p1, h1, t1 = oracle.price_epoch_update(usage, h0, 1, 1)
    assert rc == 0 and (p1 == 200).all() and (h1 == 20).all() and (t1 == 220).all()


def test_history_persists_without_overuse():
    rc, p, h, t = oracle.price_epoch_update(np.array([1, 0], np.uint64), np.array([10, 10]), 1, 1)
    assert rc == 0 and (p == 0).all() and (h == 10).all() and (t == 10).all()


def test_zero_capacity_snapshot_known_answer():
    rc, cost = oracle.price_snapshot(np.array([0], np.uint64), np.array([0], np.uint64), 0, 0, 7, 0, 12)
    assert rc == 0 and cost[0] == 7
    assert cost[0] + 5 == 12  # merged with the request's base penalty
    assert cost[0] + 5 > 11


def test_overflow_is_reported():
    big = np.array([3], np.uint64)
    rc, *_ = oracle.price_epoch_update(big, np.zeros(1), 0, 1, init=2**62, inc=2**62)
    assert rc == 1
