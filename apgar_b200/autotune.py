"""Schedule autotuner for the frontier generator.

The frontier's results do not depend on its schedule: the key-level width
(bucket width), chained expansions and the width-class limits that give a net
1, 2, 4, 8 or 16 warps only change how the same exact search is laid out on
the GPU.  So the tuner times candidate schedules on the caller's own batch
(or a seeded sample with the batch's window-size mix) and keeps the fastest.
Every candidate's costs are compared with the first candidate's, and a
mismatch raises: a schedule that changed a result would be a bug.

The search is a coordinate descent over the three knobs, starting from the
library default: bucket width first, then the class limits (a few preset
sets, then one limit at a time by one step while that helps), then
chaining.
Choices are cached per workload signature (lattice shape, batch size and
window-size quantiles) for the life of the process, and can be saved to and
loaded from a JSON file.
"""

from __future__ import annotations

import dataclasses
import json
import os

import numpy as np

from . import class_bounds


@dataclasses.dataclass(frozen=True)
class Schedule:
    bucket_width: int = 0  # 0 = twice the largest move cost
    chain: int = 0         # 0 = the per-class default (no chaining)
    class_bounds: int = 0  # 0 = the library default limits
    # the 16-warp class (the batch's longest searches, its critical path):
    # its own level width and chain, 0 = as the other classes
    wide_bucket_width: int = 0
    wide_chain: int = 0

    def describe(self) -> dict:
        bounds = [(self.class_bounds >> (8 * k)) & 0xFF for k in range(4)] if self.class_bounds else None
        return {"bucket_width": self.bucket_width, "chain": self.chain, "class_log2_limits": bounds,
                "wide_bucket_width": self.wide_bucket_width, "wide_chain": self.wide_chain}


DEFAULT = Schedule()

# width-class limit sets tried first, the library default (12, 15, 17, 19)
# leading; the best of them is then refined one limit at a time
BOUND_SETS = ((12, 15, 17, 19), (12, 15, 17, 20), (12, 15, 18, 21), (13, 16, 18, 20),
              (11, 14, 17, 19), (12, 14, 16, 18))
REFINE_STEPS = 3

_CACHE: dict = {}


def signature(lattice, nets) -> str:
    """Workload key: lattice shape, move costs, batch size and the window-size
    quartiles (log2, rounded)."""
    cells = (nets["win_w"].astype(np.float64) * nets["win_h"].astype(np.float64) * lattice.layers)
    q = np.round(np.log2(np.maximum(np.quantile(cells, [0.25, 0.5, 0.75, 1.0]), 1.0)), 1) if len(nets) else []
    return json.dumps([lattice.layers, lattice.height, lattice.width, int(len(nets)),
                       [float(x) for x in q]])


def _sample(nets, max_nets, seed):
    if max_nets is None or len(nets) <= max_nets:
        return np.ascontiguousarray(nets)
    rng = np.random.default_rng(seed)
    # stratified by window size, so the sample keeps the batch's class mix
    order = np.argsort(nets["win_w"].astype(np.int64) * nets["win_h"].astype(np.int64), kind="stable")
    strata = np.array_split(order, max_nets)
    pick = np.array([s[rng.integers(len(s))] for s in strata if len(s)])
    return np.ascontiguousarray(nets[np.sort(pick)])


def time_schedule(lattice, nets, schedule: Schedule, warmup: int = 1, reps: int = 5):
    """(ms per execution, per-net costs) of one schedule: the mean over
    `reps` back-to-back executions, as a resident plan runs them."""
    import torch

    plan = lattice.plan(nets, generator="frontier", schedule=schedule)
    try:
        stream = torch.cuda.current_stream()
        for _ in range(warmup):
            plan.execute(stream.cuda_stream)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            plan.execute(stream.cuda_stream)
        b.record(stream)
        b.synchronize()
        res, _ = plan.readback(want_paths=False)
        return a.elapsed_time(b) / reps, res["cost"].copy()
    finally:
        plan.close()


# a candidate replaces the best only when it is faster by this fraction (run
# to run noise of one batch is a few percent)
MIN_GAIN = 0.03


def tune(lattice, nets, max_nets: int | None = None, warmup: int = 1, reps: int = 5, seed: int = 0,
         use_cache: bool = True):
    """Tunes the frontier schedule for ``nets`` on ``lattice`` (a
    DeviceLattice).  Returns (best Schedule, list of (schedule dict, ms))."""
    key = signature(lattice, nets)
    if use_cache and key in _CACHE:
        return _CACHE[key]
    sample = _sample(nets, max_nets, seed)
    min_width = 2 * max(lattice.orth, lattice.diag, lattice.via)
    table = []
    reference = None

    def measure(s: Schedule) -> float:
        nonlocal reference
        ms, cost = time_schedule(lattice, sample, s, warmup, reps)
        if reference is None:
            reference = cost
        elif not np.array_equal(cost, reference):
            raise RuntimeError(f"schedule {s.describe()} changed a result")
        table.append((s.describe(), round(ms, 3)))
        return ms

    best, best_ms = DEFAULT, measure(DEFAULT)
    for width in (min_width * 3 // 2, min_width * 2, min_width * 4):
        s = dataclasses.replace(best, bucket_width=width)
        ms = measure(s)
        if ms < best_ms * (1.0 - MIN_GAIN):
            best, best_ms = s, ms
    base = best
    best_bounds = BOUND_SETS[0]
    tried = {BOUND_SETS[0]}
    for bounds in BOUND_SETS[1:]:
        tried.add(bounds)
        s = dataclasses.replace(base, class_bounds=class_bounds(*bounds))
        ms = measure(s)
        if ms < best_ms * (1.0 - MIN_GAIN):
            best, best_ms, best_bounds = s, ms, bounds
    # refinement: move one limit by one step while that helps
    for _ in range(REFINE_STEPS):
        step = None
        for k in range(4):
            for d in (-1, 1):
                b = list(best_bounds)
                b[k] += d
                b = tuple(b)
                if b in tried or not (1 <= b[0] and b[3] <= 31 and all(x < y for x, y in zip(b, b[1:]))):
                    continue
                tried.add(b)
                s = dataclasses.replace(best, class_bounds=class_bounds(*b))
                ms = measure(s)
                if ms < best_ms * (1.0 - MIN_GAIN):
                    step, best_ms = (s, b), ms
        if step is None:
            break
        best, best_bounds = step
    s = dataclasses.replace(best, chain=2)
    ms = measure(s)
    if ms < best_ms * (1.0 - MIN_GAIN):
        best, best_ms = s, ms
    # the widest class alone: wider levels mean fewer level openings on its
    # nets' round chains (the batch's critical path) at the price of extra
    # expansions, which the other classes' throughput cannot afford
    # (a chain for the widest class alone measured 2-4x slower on the medium
    # batch, depths 4-16, so it is not searched; the option stays available)
    base = best
    for factor in (2, 4):
        s = dataclasses.replace(base, wide_bucket_width=min_width * factor)
        ms = measure(s)
        if ms < best_ms * (1.0 - MIN_GAIN):
            best, best_ms = s, ms
    out = (best, table)
    _CACHE[key] = out
    return out


def save(path: str) -> None:
    """Writes the cached choices to a JSON file."""
    data = {k: dataclasses.asdict(v[0]) for k, v in _CACHE.items()}
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def load(path: str) -> None:
    """Adds the choices of a JSON file written by ``save`` to the cache."""
    with open(path) as f:
        data = json.load(f)
    for k, v in data.items():
        _CACHE[k] = (Schedule(**v), [])
