"""The replay-invariant fixture (from the reference's replays/gpu/*.replay)
holds every artifact, and the faults the device validators cover."""

from tests.test_replay_invariants_gpu import DEVICE_FAULTS, REPLAYS


def test_fixture_holds_the_device_faults():
    assert len(REPLAYS) == 16
    faults = {r["fault"] for r in REPLAYS}
    assert set(DEVICE_FAULTS) <= faults
    for r in REPLAYS:
        assert r["expected_invariant"] and r["expected_failure"] in ("internal_invariant", "unsupported")
