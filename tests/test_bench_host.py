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


def test_frontier_bytes_come_from_the_oracle_expansions(bench):
    """The frontier's algorithmic bytes count the oracle A*'s distinct expanded
    cells, not the GPU's own expansions (which are reported beside them)."""
    import oracle
    from apgar_b200 import synth

    lat, nets = synth.config_small(1)
    nets = nets[:6].copy()
    _, _, cells = oracle.astar_batch(lat, nets, counts=True)
    res = np.zeros(len(nets), dtype=[("row_steps", "<u4"), ("path_len", "<u4")])
    res["row_steps"] = 1000
    res["path_len"] = 3
    alg, gpu = bench.frontier_bytes(lat, nets, res)
    assert cells.sum() > 0
    assert alg == cells.sum() * (4 + 11 * 8) + 4 * 3 * len(nets)
    assert gpu == 1000 * len(nets) * (4 + 11 * 8) + 4 * 3 * len(nets)


def test_oracle_expanded_cells_are_distinct_cells_of_expanded_states():
    """Expanded states count every (cell, heading) the A* pops and expands;
    distinct cells are at most that and at least one per expanded cell."""
    import oracle
    from apgar_b200 import synth

    lat, nets = synth.config_small(1)
    costs, states, cells = oracle.astar_batch(lat, nets[:8].copy(), counts=True)
    assert np.array_equal(costs, oracle.astar_batch(lat, nets[:8].copy()))
    assert (cells <= states).all() and (cells[states > 0] > 0).all()
    for i in range(3):
        _, expanded, _ = oracle.astar_path(lat, nets[i:i + 1].copy())
        assert expanded == states[i]


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
    # the same static config dict as the device arm's line (medium_config)
    assert line["config"] == {
        "workload": line["config"]["workload"], "nets_per_gpu": 32, "lattice": [4, 256, 256],
        "seed": 2, "parallelism": "weak x1 (independent net batches)",
        "l2": "label words (5.4 GB) larger than L2 (126 MB) and cleared every step"}
