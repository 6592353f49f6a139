"""Host-side pieces of bench.py that need no GPU: the clock sampler's
parsing of nvidia-smi rows (only rows written after timing began count;
throttle reasons are collected), the algorithmic byte counts, and the
reference arm's JSON line."""

import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture
def bench(monkeypatch):
    """bench.py as a module, imported without leaving its process-wide CUDA
    setting behind in this test process."""
    monkeypatch.setenv("CUDA_DEVICE_MAX_CONNECTIONS", os.environ.get("CUDA_DEVICE_MAX_CONNECTIONS", "8"))
    monkeypatch.syspath_prepend(ROOT)
    import bench as module

    return module


def test_clock_summary_skips_rows_before_timing(tmp_path, bench):
    s = bench.ClockSampler(0)
    s.path = str(tmp_path / "clocks.csv")
    rows = [
        "0, 345, 1965, 120.0, 0x0, Not Active, Not Active, Not Active, Not Active",  # idle, before timing
        "0, 1965, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
        "0, 1965, 1965, 800.0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ]
    with open(s.path, "w") as f:
        f.write("\n".join(rows) + "\n")
    s.proc = object()  # as if nvidia-smi ran
    s.skip = 1
    out = s.summary()
    assert out["samples"] == 3 and out["sm_mhz"] == 1965.0 and out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"]


def test_frontier_bytes_follow_the_expansion_count(bench):
    res = np.zeros(3, dtype=[("row_steps", "<u4"), ("path_len", "<u4")])
    res["row_steps"] = [10, 0, 5]
    res["path_len"] = [4, 0, 2]
    assert bench.frontier_bytes(res) == 15 * (4 + 11 * 8) + 4 * 6


def test_reference_arm_prints_one_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "1", "--ref-sample", "8", "--size", "256",
                          "--nets", "32"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "nets/s"
    for key in ("metric", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "cpu_baseline", "e2e", "config"):
        assert key in line
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
