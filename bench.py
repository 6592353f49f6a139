#!/usr/bin/env python
"""Benchmark: certified-optimal nets/s of the batched lattice search on B200.

Workload (the medium lattice configuration, the largest that is quoted on one
GPU): 4 layers of 2048x2048 cells, 25% blocked (rectangles + pad keep-outs),
4096 two-terminal nets with lognormal(200, 1.0) half-perimeter, each searched
in its bbox + 32 window with uint32 labels and bit-packed masks.  Synthetic,
seeded inputs (no public dataset exists for this path).

One step = one batched search of all nets of the batch: exact labels on every
cell the canonical reverse path needs, plus that path, for every net.  A net is
certified when its search converged (reached or proved disconnected inside its
window).  The headline form is the persistent work-stealing frontier search
(bucketed A*); the plain batched sweep is measured beside it on the same nets
and reported under "plain_sweep", with the ratio of the two, and so is the
learned form (CNN corridors with the exact certificate and full-window
fallback, trained weights under apgar_b200/weights) under "learned_corridor".

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun every rank searches its own batch (same lattice, rank-specific
net seed): weak scaling, no data-path collective; the timed region is
bracketed by a barrier and synchronize and reported as the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

# One hardware work queue per process (read when the CUDA context is created,
# so before torch touches the GPU).  The plain sweep runs its width classes as
# concurrent kernels on forked streams; with several queues their CTAs reach
# the SMs in any order and its time per batch varies by about 7%.  (The
# frontier runs all its classes in one launch and does not depend on it.)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "1")

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "certified-optimal nets/sec on 1 B200: learned+batched vs plain sweep"
UNIT = "nets/s"
WORKLOAD = ("medium lattice: 4 layers x 2048x2048, 25% blocked (rectangles + 4x4 pad keep-outs "
            "on a 20-cell pitch), 4096 two-terminal nets, half-perimeter lognormal(median 200, "
            "sigma 1.0), bbox+32 windows, costs orth 10 / diag 14 / via 50, bend 0")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--size", type=int, default=2048)
    ap.add_argument("--nets", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--cpu-sample", type=int, default=4096,
                    help="nets timed by the CPU baseline (bounded sample)")
    ap.add_argument("--ref-sample", type=int, default=512,
                    help="nets per step of the reference arm")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true",
                    help="skip the learned-corridor form (reported beside the headline)")
    ap.add_argument("--workload", choices=["medium", "negotiated", "full", "dropin"],
                    default="medium",
                    help="medium: the headline batch; negotiated: 10 rip-up/reroute rounds "
                         "on the 6 x 4096^2 lattice with multi-terminal nets (one CUDA graph); "
                         "full: 20 rounds on the 8 x 8192^2 full-scale configuration; dropin: "
                         "the reference's corpus at 4..512 candidate queries per case through "
                         "the reference's own prepared batch path over this backend, beside the "
                         "reference's CPU A*")
    ap.add_argument("--no-tune", action="store_true",
                    help="medium workload: skip the (untimed) frontier schedule autotuner and use "
                         "the library's default schedule")
    ap.add_argument("--ranked", action="store_true",
                    help="negotiated workloads: the multi-GPU split-round form (per-round NCCL "
                         "all-reduce of usage) even on one GPU; it is the form used for N > 1")
    ap.add_argument("--rounds", type=int, default=None,
                    help="negotiated rounds (default 10, or 20 for the full workload)")
    ap.add_argument("--neg-sample", type=int, default=2048,
                    help="negotiated workloads: segments of the round-0 comparison (frontier, "
                         "sweep, oracle bytes and CPU baseline)")
    ap.add_argument("--learned-rounds", action="store_true",
                    help="negotiated workloads: also run the negotiation with learned corridor "
                         "proposals in every priced round and report it beside the line")
    ap.add_argument("--full-ripup", action="store_true",
                    help="negotiated: reroute every net each round (default: only nets "
                         "crossing overused cells after round 0)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic():
    """DRAM bytes per sweep launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "lattice_traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return None


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during timing."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.skip = 0
        self.path = os.path.join("/tmp", f"apgar_b200_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return self
        # nvidia-smi takes a moment to start: wait for its first row, then
        # count only the rows written after this point (the timed region)
        deadline = time.monotonic() + 3.0
        while time.monotonic() < deadline and self._rows_written() == 0:
            time.sleep(0.01)
        self.skip = self._rows_written()
        return self

    def _rows_written(self) -> int:
        try:
            with open(self.path) as f:
                return sum(1 for line in f if line.count(",") >= 8)
        except OSError:
            return 0

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.out.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return None
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                rows.append(parts)
        os.unlink(self.path)
        rows = rows[self.skip:] or rows[-1:]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# Bytes one cell expansion of the frontier moves: its queue entry (4 B), its
# label word and the words of its 10 neighbours (11 x 8 B).
EXPANSION_BYTES = 4.0 + 11 * 8.0


def frontier_bytes(lat, nets, results):
    """Algorithmic bytes of one frontier batch, from the oracle, not from the
    GPU's own work: the distinct cells the A* restatement of RouteWithCpuAStar
    expands per net (the cell expansions an exact search needs) times the
    bytes of an expansion, plus 4 B per emitted path cell.  Returns (those
    bytes, the bytes of the GPU's own expansions, re-expansions included)."""
    import oracle

    _, _, cells = oracle.astar_batch(lat, nets, counts=True)
    path = 4.0 * results["path_len"].astype(np.float64).sum()
    gpu = results["row_steps"].astype(np.float64).sum() * EXPANSION_BYTES + path
    return cells.astype(np.float64).sum() * EXPANSION_BYTES + path, gpu


def certified(results):
    import apgar_b200

    c = results["completion"]
    return int(np.count_nonzero((c == apgar_b200.COMPLETION_REACHED)
                                | (c == apgar_b200.COMPLETION_DISCONNECTED)))


def algorithmic_bytes(lat, nets, results):
    """Bytes the sweep schedule must move.

    Per processed frame row: the layer rows read and written (4 B per cell of
    the row, which runs along the window's longer side) plus the obstacle and
    via bits (2 bits per cell per layer); plus 4 B per emitted path cell.  The
    per-net row counters are the CPU restatement's counts (the GPU tests check
    they are identical)."""
    w = np.maximum(nets["win_w"], nets["win_h"]).astype(np.float64)
    rows_moved = results["row_loads"].astype(np.float64) + results["row_stores"].astype(np.float64)
    label_bytes = (4.0 * w * rows_moved).sum()
    mask_bytes = (results["row_steps"].astype(np.float64) * lat.layers * w * 2.0 / 8.0).sum()
    path_bytes = 4.0 * results["path_len"].astype(np.float64).sum()
    one_pass = (nets["win_w"].astype(np.float64) * nets["win_h"] * lat.layers * 4.25).sum()
    return label_bytes + mask_bytes + path_bytes, one_pass


def cpu_baseline(lat, nets, sample: int):
    """The CPU A* port (reference RouteWithCpuAStar restated with vias), all host
    threads, on a bounded sample of the same nets."""
    import oracle

    threads = os.cpu_count() or 1
    sub = np.ascontiguousarray(nets[:sample])
    t0 = time.perf_counter()
    costs = oracle.astar_batch(lat, sub, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": len(sub) / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"first {len(sub)} of the {len(nets)} nets, A* port of RouteWithCpuAStar "
                      f"(cpu_astar.cc:323-638) extended with vias, {threads} threads, {dt:.2f} s"}, costs


def round0_sample(args, lat, segs, dev):
    """Round 0 of a negotiation (zero prices) on a bounded sample of its
    segments, untimed by the negotiation itself: the frontier (the search every
    round runs) against the plain sweep on the same segments, the frontier
    launch's roofline from the oracle's expansions, and the CPU A* port on all
    host threads over the same sample (one oracle run gives both)."""
    import torch

    import apgar_b200
    import oracle

    sample = np.ascontiguousarray(segs[: min(args.neg_sample, len(segs))])
    stream = torch.cuda.current_stream()

    def timed(plan, reps=3):
        for _ in range(3):
            plan.execute(stream.cuda_stream)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            plan.execute(stream.cuda_stream)
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    fp = dev.plan(sample, generator="frontier")
    f_ms = timed(fp)
    fres, _ = fp.readback(want_paths=False)
    fp.close()
    sp = dev.plan(sample, generator="sweep")
    s_ms = timed(sp)
    sres, _ = sp.readback(want_paths=False)
    sp.close()
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    cpu_costs, _, cells = oracle.astar_batch(lat, sample, threads=threads, counts=True)
    cpu_s = time.perf_counter() - t0
    ok = fres["completion"] != apgar_b200.COMPLETION_REJECTED
    both = (fres["completion"] == apgar_b200.COMPLETION_REACHED) & \
        (sres["completion"] == apgar_b200.COMPLETION_REACHED)
    peak, peak_kind = load_peaks()
    fbytes = cells.astype(np.float64).sum() * EXPANSION_BYTES + 4.0 * fres["path_len"].astype(np.float64).sum()
    achieved = fbytes / (f_ms / 1000.0) / 1e9
    n = len(sample)
    return {
        "round0_sample": {
            "segments": n, "frontier_ms": f_ms, "sweep_ms": s_ms, "frontier_over_sweep": s_ms / f_ms,
            "frontier_routes_per_s": n / (f_ms / 1000.0), "sweep_routes_per_s": n / (s_ms / 1000.0),
            # over the segments both forms reached (a form rejects a segment
            # when its window or queue bound is exceeded)
            "same_costs": bool(np.array_equal(fres["cost"][both], sres["cost"][both])),
            "both_reached": int(both.sum()),
            "frontier_completion": np.bincount(fres["completion"], minlength=5).tolist(),
            "sweep_completion": np.bincount(sres["completion"], minlength=5).tolist(),
        },
        "roofline": {
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
            "kernel": f"lattice_frontier_kernel, round 0 (zero prices) of the first {n} segments",
            "bytes_alg_per_launch": fbytes,
            "bytes_alg_source": "oracle A* expanded cells x 92 B + 4 B per path cell",
        },
        "cpu_baseline": {
            "value": n / cpu_s, "unit": "routes/s", "cores": threads, "kind": "port",
            "sample": f"round 0 of the first {n} segments, A* port of RouteWithCpuAStar "
                      f"(cpu_astar.cc:323-638) extended with vias, {threads} threads, {cpu_s:.2f} s",
            "costs_match_gpu": bool(np.array_equal(cpu_costs[ok], fres["cost"][ok])),
        },
    }


def medium_config(args, world, lat):
    """The medium workload's `config`, the same dict in both arms (what
    differs between runs, such as the frontier schedule, is reported beside
    it)."""
    return {
        "workload": WORKLOAD, "nets_per_gpu": args.nets,
        "lattice": [lat.layers, lat.height, lat.width], "seed": args.seed,
        "parallelism": f"weak x{world} (independent net batches)",
        "l2": "label words (5.4 GB) larger than L2 (126 MB) and cleared every step",
    }


def run_reference(args, rank, world):
    if rank != 0:
        return
    import oracle
    from apgar_b200 import synth

    lat, nets = synth.config_medium(args.seed, nets=args.nets, size=args.size)
    threads = os.cpu_count() or 1
    sample = np.ascontiguousarray(nets[: args.ref_sample])
    for _ in range(args.warmup):
        oracle.astar_batch(lat, sample[:64], threads=threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.astar_batch(lat, sample, threads=threads)
    dt = time.perf_counter() - t0
    value = len(sample) * args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1000.0 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic",
        "config": medium_config(args, world, lat),
        "form": f"CPU A* port over {len(sample)} nets of the batch per step",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{len(sample)} nets per step, all {threads} host threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


NEG_METRIC = "2-pin segment routes/sec over negotiated rip-up/reroute rounds on 1 B200"
NEG_WORKLOAD = ("negotiated lattice: 6 layers x 4096x4096, 25% blocked (rectangles + pad keep-outs), "
                "16384 nets with 2-6 terminals split into 2-pin segments along a Manhattan MST, "
                "half-perimeter lognormal(median 300, sigma 1.2), bbox+32 windows, cell capacity 1, "
                "prices 100/+100/+10 (reference defaults)")
FULL_WORKLOAD = ("full-scale lattice: 8 layers x 8192x8192, 30% blocked (rectangles + pad keep-outs), "
                 "32768 nets with 2-8 terminals split into 2-pin segments along a Manhattan MST, "
                 "half-perimeter lognormal(median 400, sigma 1.3), bbox+32 windows, cell capacity 1, "
                 "prices 100/+100/+10 (reference defaults)")


def run_negotiated(args, rank, world, local):
    """One step = a whole negotiation from zero prices: args.rounds Jacobi
    rip-up/reroute rounds of every segment, replayed as one CUDA graph."""
    import torch

    torch.cuda.set_device(local)
    import apgar_b200
    from apgar_b200 import negotiate, prices, synth

    full = args.workload == "full"
    rounds = args.rounds if args.rounds is not None else (20 if full else 10)
    args.rounds = rounds
    lat, segs, _ = synth.config_full(args.seed + 3) if full else synth.config_negotiated(args.seed + 1)
    dev = apgar_b200.DeviceLattice(lat)
    plan = dev.plan(segs, generator="frontier")
    neg = negotiate.Negotiation(plan, prices.policy(capacity=1))
    stream = torch.cuda.current_stream()
    partial = not args.full_ripup
    for _ in range(max(args.warmup, 3)):
        neg.run(args.rounds, use_graph=True, stream=stream.cuda_stream, partial=partial)
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            neg.run(args.rounds, use_graph=True, stream=stream.cuda_stream, partial=partial)
        end.record(stream)
        torch.cuda.synchronize()
    ms = start.elapsed_time(end) / args.steps
    usage, history, cost, rows = neg.readback()
    res, paths = plan.readback()
    routes = len(segs) * args.rounds
    # end to end: segments from the host, plan, negotiation, results + paths back
    import time as _t

    torch.cuda.synchronize()
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    e_start.record()
    for _ in range(max(1, args.steps // 2)):
        p2 = dev.plan(segs, generator="frontier")
        n2 = negotiate.Negotiation(p2, prices.policy(capacity=1))
        n2.run(args.rounds, use_graph=False, stream=0, partial=partial)
        r2, pa2 = p2.readback()
        n2.close()
        p2.close()
    e_end.record()
    torch.cuda.synchronize()
    e2e_ms = e_start.elapsed_time(e_end) / max(1, args.steps // 2)
    c = res["completion"]
    line = {
        "metric": NEG_METRIC, "value": routes / (ms / 1000.0), "unit": "routes/s", "n_gpus": 1,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic",
        "config": {"workload": FULL_WORKLOAD if full else NEG_WORKLOAD, "segments": len(segs),
                   "rounds": args.rounds,
                   "form": "frontier search + fused snapshot prices, Jacobi rounds, one CUDA graph",
                   "rip_up": "full" if args.full_ripup else "partial (nets crossing overused cells)",
                   "workspace_bytes": plan.info()["workspace_bytes"]},
        "gpu_launches": args.rounds * (plan.info()["kernel_launches"] + 2) * args.steps,
        "e2e": {"value": routes / (e2e_ms / 1000.0), "unit": "routes/s",
                "h2d_bytes_per_step": int(segs.nbytes),
                "d2h_bytes_per_step": int(len(segs) * apgar_b200.RESULT_DTYPE.itemsize + 4 * len(pa2)),
                "ms_per_step": e2e_ms},
        "clocks": clocks.summary(),
        "last_round": {"reached": int((c == 0).sum()), "disconnected": int((c == 1).sum()),
                       "rejected": int((c == 4).sum())},
        "overuse_per_round": [[r["overused_cells"], r["total_overuse"]] for r in rows],
    }
    neg.close()
    plan.close()
    if args.learned_rounds:
        line["learned_rounds"] = learned_negotiation(args, segs, dev, res, ms)
    line.update(round0_sample(args, lat, segs, dev))
    dev.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


# activations of the corridor CNN take ~0.6 MB per segment (two ping-pong
# buffers and the rasters): larger negotiations would not fit beside the plan
LEARNED_ROUNDS_MAX_SEGMENTS = 65536


def learned_negotiation(args, segs, dev, plain_results, plain_ms):
    """The same negotiation with a learned corridor proposal before every
    priced round (round 0 searches without corridors), one warm-up and one
    timed run; its routes must equal the plain negotiation's."""
    import torch

    from apgar_b200 import learned, negotiate, prices

    if len(segs) > LEARNED_ROUNDS_MAX_SEGMENTS:
        return {"skipped": f"{len(segs)} segments: the CNN's activations would not fit beside the "
                           f"plan (limit {LEARNED_ROUNDS_MAX_SEGMENTS})"}
    partial = not args.full_ripup
    plan = dev.plan(segs, generator="frontier")
    neg = negotiate.Negotiation(plan, prices.policy(capacity=1))
    router = learned.LearnedRouter(plan)
    stream = torch.cuda.current_stream()
    neg.run_learned(args.rounds, router, stream.cuda_stream, partial)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    neg.run_learned(args.rounds, router, stream.cuda_stream, partial)
    b.record(stream)
    torch.cuda.synchronize()
    l_ms = a.elapsed_time(b)
    router.net.check_error()
    res, _ = plan.readback(want_paths=False)
    status = plan.corridor_status()
    neg.close()
    plan.close()
    return {"value": len(segs) * args.rounds / (l_ms / 1000.0), "unit": "routes/s",
            "ms_per_negotiation": l_ms, "plain_over_learned": l_ms / plain_ms,
            "same_results": bool(np.array_equal(res["cost"], plain_results["cost"]) and
                                 np.array_equal(res["completion"], plain_results["completion"])),
            "last_round_certified": float((status == 1).mean()),
            "last_round_fallback": float((status >= 2).mean())}


def run_negotiated_ranked(args, rank, world, local):
    """The negotiated workload on `world` GPUs: rank r takes every world-th
    segment, and every round sums the per-cell usage over the ranks with one
    NCCL all-reduce between its ROUTE and PRICE steps (strong scaling: the
    total work is the single-GPU run's, and the routes are identical to it)."""
    import datetime

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                            device_id=torch.device("cuda", local))
    import apgar_b200
    from apgar_b200 import negotiate, prices, shard, synth

    full = args.workload == "full"
    rounds = args.rounds if args.rounds is not None else (20 if full else 10)
    lat, segs, _ = synth.config_full(args.seed + 3) if full else synth.config_negotiated(args.seed + 1)
    # static partition by estimated window work (every rank computes the same)
    mine = np.ascontiguousarray(segs[shard.balanced_split(segs, world, lat.layers)[rank]])
    dev = apgar_b200.DeviceLattice(lat)
    plan = dev.plan(mine, generator="frontier")
    neg = negotiate.Negotiation(plan, prices.policy(capacity=1))
    stream = torch.cuda.current_stream()
    partial = not args.full_ripup
    usage = torch.zeros(neg.cells, dtype=torch.int32, device="cuda")

    def one_run(n):
        n.run_ranked(rounds, usage, lambda u: shard.allreduce_usage(u, dist),
                     stream=stream.cuda_stream, partial=partial)

    for _ in range(max(args.warmup, 3)):
        one_run(neg)
    torch.cuda.synchronize()
    dist.barrier()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            one_run(neg)
        end.record(stream)
        torch.cuda.synchronize()
    ms = shard.max_over_ranks(start.elapsed_time(end) / args.steps, dist, device="cuda")
    _, _, _, rows = neg.readback()
    res, _ = plan.readback()
    # end to end: this rank's segments from the host, plan, ranked negotiation,
    # results and paths back
    dist.barrier()
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    e_runs = max(1, args.steps // 2)
    e_start.record(stream)
    for _ in range(e_runs):
        p2 = dev.plan(mine, generator="frontier")
        n2 = negotiate.Negotiation(p2, prices.policy(capacity=1))
        one_run(n2)
        r2, pa2 = p2.readback()
        n2.close()
        p2.close()
    e_end.record(stream)
    torch.cuda.synchronize()
    e2e_ms = shard.max_over_ranks(e_start.elapsed_time(e_end) / e_runs, dist, device="cuda")
    reached = shard.sum_over_ranks(int((res["completion"] == 0).sum()), dist, device="cuda")
    d2h = shard.sum_over_ranks(int(len(mine) * apgar_b200.RESULT_DTYPE.itemsize + 4 * len(pa2)), dist,
                               device="cuda")
    routes = len(segs) * rounds
    line = {
        "metric": NEG_METRIC if world == 1 else NEG_METRIC.replace("on 1 B200", f"on {world} B200s"),
        "value": routes / (ms / 1000.0), "unit": "routes/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic",
        "config": {"workload": FULL_WORKLOAD if full else NEG_WORKLOAD, "segments": len(segs),
                   "rounds": rounds,
                   "parallelism": f"segments split over {world} ranks, balanced by window work",
                   "form": "frontier search + fused snapshot prices, Jacobi rounds; one int32 "
                           "all-reduce of per-cell usage per round (NCCL)",
                   "rip_up": "full" if args.full_ripup else "partial (nets crossing overused cells)"},
        "gpu_launches": rounds * (plan.info()["kernel_launches"] + 2) * args.steps,
        "e2e": {"value": routes / (e2e_ms / 1000.0), "unit": "routes/s",
                "h2d_bytes_per_step": int(segs.nbytes),
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms},
        "clocks": clocks.summary(),
        "last_round_reached": reached,
        "overuse_per_round": [[r["overused_cells"], r["total_overuse"]] for r in rows],
    }
    neg.close()
    plan.close()
    dev.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    dist.barrier()
    dist.destroy_process_group()


DROPIN_METRIC = ("prepared end-to-end candidate queries/s on the reference's corpus "
                 "(drop-in through the reference's prepared batch path)")


def run_dropin(args, rank):
    """The drop-in on the reference's own workload: every case of its parity
    corpus (BuildPhase3CandidateCorpus) at k = 4..512 candidate policies, the
    prepared end-to-end scope of the reference's report (the view upload once,
    then per batch: H2D, search, D2H and the reference's host validation and
    sealing), timed by apgar_b200/adapter/_build/dropin_bench (built with the
    reference sources), beside the reference's own CPU A* on all host threads
    and on one.  Pooled throughput = queries over summed medians."""
    if rank != 0:
        return
    exe = os.path.join(ROOT, "apgar_b200", "adapter", "_build", "dropin_bench")
    if not os.path.exists(exe):
        raise SystemExit("dropin_bench is not built (apgar_b200/adapter/build_adapter.sh needs the "
                         "reference sources)")
    out = subprocess.run([exe], capture_output=True, text=True, timeout=1800)
    if out.returncode != 0:
        raise SystemExit("dropin_bench failed: " + out.stderr[-2000:])
    data = json.loads(out.stdout)
    ks = [row["k"] for row in data["cases"][0]["k"]]
    per_k = []
    tot = {"q": 0, "gpu": 0.0, "par": 0.0, "ser": 0.0, "best": 0.0}
    for k in ks:
        rows = [next(r for r in c["k"] if r["k"] == k) for c in data["cases"]]
        q = k * len(rows)
        g = sum(r["gpu_ms"] for r in rows)
        p = sum(r["cpu_par_ms"] for r in rows)
        s = sum(r["cpu_ser_ms"] for r in rows)
        best = sum(min(r["cpu_par_ms"], r["cpu_ser_ms"]) for r in rows)
        tot["q"] += q
        tot["gpu"] += g
        tot["par"] += p
        tot["ser"] += s
        tot["best"] += best
        kern = sum(r.get("gpu_kernel_ms", 0.0) for r in rows)
        per_k.append({"k": k, "gpu_qps": q / (g / 1e3), "cpu_parallel_qps": q / (p / 1e3),
                      "cpu_serial_qps": q / (s / 1e3), "gpu_over_faster_cpu": best / g,
                      "gpu_ms_per_batch": g / len(rows), "gpu_kernel_ms_per_batch": kern / len(rows),
                      "cases_gpu_slower": [c["name"] for c, r in zip(data["cases"], rows)
                                           if r["gpu_ms"] > min(r["cpu_par_ms"], r["cpu_ser_ms"])]})
    value = tot["q"] / (tot["gpu"] / 1e3)
    line = {
        "metric": DROPIN_METRIC, "value": value, "unit": "queries/s", "n_gpus": 1,
        "steps": data["repetitions"], "warmup": 1, "ms_per_step": tot["gpu"] / len(ks),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "the reference's own parity corpus (generated boards and its KiCad fixture)",
        "config": {"workload": "BuildPhase3CandidateCorpus, 11 cases, k = " +
                               ",".join(map(str, ks)) + " candidate policies per batch "
                               "(BuildDeterministicAlternativePolicies over the base route)",
                   "generator": "kB200Persistent (compact paths)",
                   "scope": "prepared end to end: H2D, search, D2H, host validation and sealing; "
                            "the view upload excluded"},
        "per_k": per_k,
        "gpu_over_faster_cpu_pooled": tot["best"] / tot["gpu"],
        "cpu_baseline": {"value": tot["q"] / (tot["par"] / 1e3), "unit": "queries/s",
                         "cores": data["threads"], "kind": "reference",
                         "sample": "the same batches, the reference's RouteWithCpuAStar "
                                   "compiled from its sources, one query per task",
                         "serial_value": tot["q"] / (tot["ser"] / 1e3)},
        "costs_match_cpu": data["costs_match"],
        "cases": data["cases"],
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "dropin":
        run_dropin(args, rank)
        return
    if args.workload in ("negotiated", "full"):
        if world > 1 or args.ranked:
            run_negotiated_ranked(args, rank, world, local)
        else:
            run_negotiated(args, rank, world, local)
        return

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    import apgar_b200
    from apgar_b200 import shard, synth

    lat, _ = synth.config_medium(args.seed, nets=0, size=args.size)
    nets = shard.rank_nets(lat, args.seed, rank, args.nets)  # weak scaling: a batch per rank
    dev = apgar_b200.DeviceLattice(lat)
    stream = torch.cuda.current_stream()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(ms):
        return shard.max_over_ranks(ms, dist, device="cuda")

    def sum_over_ranks(n):
        return shard.sum_over_ranks(n, dist, device="cuda")

    # ---------------- frontier schedule (autotuned, untimed) ----------------
    from apgar_b200 import autotune

    if args.no_tune:
        schedule, tuning = autotune.DEFAULT, []
    else:
        schedule, tuning = autotune.tune(dev, nets)
    barrier()

    def device_resident(generator, sample_clocks):
        """K executions of a resident plan, CUDA events on torch's stream."""
        plan = dev.plan(nets, generator=generator,
                        schedule=schedule if generator == "frontier" else None)
        info = plan.info()
        for _ in range(max(args.warmup, 3)):
            plan.execute(stream.cuda_stream)
        barrier()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        sampler = ClockSampler(local) if sample_clocks else None
        if sampler:
            sampler.__enter__()
        barrier()
        for i in range(args.steps):
            starts[i].record(stream)
            plan.execute(stream.cuda_stream)
            ends[i].record(stream)
        barrier()
        if sampler:
            sampler.__exit__(None, None, None)
        step_ms = [a.elapsed_time(b) for a, b in zip(starts, ends)]
        total_ms = max_over_ranks(starts[0].elapsed_time(ends[-1]))
        results, _ = plan.readback()
        plan.close()
        return dict(info=info, step_ms=step_ms, total_ms=total_ms, results=results,
                    clocks=sampler.summary() if sampler else None)

    # ---------------- device-resident throughput (value) ----------------
    front = device_resident("frontier", sample_clocks=True)
    sweep = device_resident("sweep", sample_clocks=False)
    cert_all = sum_over_ranks(certified(front["results"]))
    value = cert_all * args.steps / (front["total_ms"] / 1000.0)
    sweep_value = sum_over_ranks(certified(sweep["results"])) * args.steps / (sweep["total_ms"] / 1000.0)
    same = bool(np.array_equal(front["results"]["cost"], sweep["results"]["cost"]) and
                np.array_equal(front["results"]["completion"], sweep["results"]["completion"]))

    # -------- learned corridor + persistent batched form (same nets) --------
    learned_form = None
    if not args.no_learned:
        from apgar_b200 import learned

        lplan = dev.plan(nets, generator="frontier", schedule=schedule)
        router = learned.LearnedRouter(lplan)
        for _ in range(max(args.warmup, 3)):
            router.execute(stream.cuda_stream)
        barrier()
        l_start = torch.cuda.Event(enable_timing=True)
        l_mid = torch.cuda.Event(enable_timing=True)
        l_end = torch.cuda.Event(enable_timing=True)
        l_start.record(stream)
        for _ in range(args.steps):
            router.execute(stream.cuda_stream)
        l_end.record(stream)
        barrier()
        l_ms = max_over_ranks(l_start.elapsed_time(l_end))
        # the proposal alone (rasters, CNN, corridor extraction)
        l_start.record(stream)
        for _ in range(args.steps):
            router.propose(stream.cuda_stream)
        l_mid.record(stream)
        barrier()
        p_ms = max_over_ranks(l_start.elapsed_time(l_mid))
        # and stage by stage
        stage_ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        stage_ms = [0.0, 0.0, 0.0]
        for _ in range(args.steps):
            stage_ev[0].record(stream)
            router.rasterize(stream.cuda_stream)
            stage_ev[1].record(stream)
            router.infer(stream.cuda_stream)
            stage_ev[2].record(stream)
            router.extract(stream.cuda_stream)
            stage_ev[3].record(stream)
            stream.synchronize()
            for i in range(3):
                stage_ms[i] += stage_ev[i].elapsed_time(stage_ev[i + 1]) / args.steps
        router.net.check_error()
        l_res, _ = lplan.readback(want_paths=False)
        status = lplan.corridor_status()
        l_cert = sum_over_ranks(certified(l_res))
        learned_form = {
            "value": l_cert * args.steps / (l_ms / 1000.0), "unit": UNIT,
            "ms_per_step": l_ms / args.steps, "proposal_ms_per_step": p_ms / args.steps,
            "proposal_stage_ms": {"rasters": stage_ms[0], "cnn": stage_ms[1], "corridors": stage_ms[2]},
            "corridor_certified": float((status == 1).mean()),
            "fallback_exit": float((status == 2).mean()),
            "fallback_unreached": float((status == 3).mean()),
            "no_corridor": float((status == 0).mean()),  # windows above the policy's limit
            "same_costs_as_frontier": bool(np.array_equal(l_res["cost"], front["results"]["cost"])),
            "policy": router.policy,
            "form": "6-layer 3x3 CNN (tcgen05, bf16/f32) corridors + certified corridor frontier, "
                    "full-window fallback in the same kernel; windows above the policy's "
                    "max_window_cells get no corridor",
        }
        lplan.close()

    # ---------------- end to end through the public API (e2e) ----------------
    info = front["info"]
    pinned_nets = torch.from_numpy(nets.view(np.uint8)).pin_memory()
    nets_host = pinned_nets.numpy().view(synth.NET_DTYPE)
    res_host = torch.empty(len(nets) * apgar_b200.RESULT_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
    res_arr = res_host.numpy().view(apgar_b200.RESULT_DTYPE)
    path_host = torch.empty(int(info["path_arena_capacity"]), dtype=torch.int32).pin_memory()
    path_arr = path_host.numpy().view(np.uint32)
    for _ in range(2):
        dev.route(nets_host, out=(res_arr, path_arr), generator="frontier", schedule=schedule)
    barrier()
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    path_cells = 0
    validated = None
    e_start.record()
    for _ in range(args.steps):
        # route from host buffers, then validate the untrusted results on the
        # device, as a caller does before trusting them
        r, p = dev.route(nets_host, out=(res_arr, path_arr), generator="frontier",
                         schedule=schedule)
        validated = dev.validate(nets_host, r, p)
        path_cells = len(p)
    e_end.record()
    barrier()
    reached = r["completion"] == apgar_b200.COMPLETION_REACHED
    if not (validated["code"][reached] == 0).all():
        raise RuntimeError("a routed path failed validation")
    e2e_ms = max_over_ranks(e_start.elapsed_time(e_end))
    e2e_value = cert_all * args.steps / (e2e_ms / 1000.0)
    verdict_bytes = len(nets) * validated.dtype.itemsize
    result_bytes = len(nets) * apgar_b200.RESULT_DTYPE.itemsize
    h2d = 2 * nets.nbytes + result_bytes + 4 * path_cells
    d2h = result_bytes + 4 * path_cells + 8 + verdict_bytes
    results = front["results"]
    step_ms = front["step_ms"]
    total_ms = front["total_ms"]
    clocks = front["clocks"]

    if rank == 0:
        peak, peak_kind = load_peaks()
        avg_ms = total_ms / args.steps
        fbytes, gpu_fbytes = frontier_bytes(lat, nets, results)
        achieved = fbytes / (avg_ms / 1000.0) / 1e9
        one_pass_f = (nets["win_w"].astype(np.float64) * nets["win_h"] * lat.layers * 4.25).sum()
        traffic = load_traffic()
        sweep_ms = sweep["total_ms"] / args.steps
        sbytes, one_pass = algorithmic_bytes(lat, nets, sweep["results"])
        sweep_achieved = sbytes / (sweep_ms / 1000.0) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": avg_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": medium_config(args, world, lat),
            "form": "persistent work-stealing frontier (bucketed A*)",
            "certified_per_step": cert_all,
            "schedule": dict(schedule.describe(),
                             chosen_by="autotuner (untimed, on this batch)" if tuning else "default"),
            "tuning_ms": [[row[0], row[1]] for row in tuning],
            "gpu_launches": int(info["kernel_launches"]) * args.steps,
            "roofline": {
                "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": (traffic or {}).get("frontier_dram_bytes_per_step"),
                "kernel": "lattice_frontier_kernel (all width classes of one execution)",
                "bytes_alg_per_step": fbytes,
                "bytes_alg_source": "oracle A* expanded cells x 92 B + 4 B per path cell",
                "gpu_expansion_bytes_per_step": gpu_fbytes,
                "one_pass_bytes_per_step": one_pass_f,
                "one_pass_frac": one_pass_f / (avg_ms / 1000.0) / 1e9 / peak,
            },
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms / args.steps,
                    "scope": "host nets -> route (H2D, search, D2H results and paths) -> "
                             "device validation of every path (H2D, check, D2H verdicts)",
                    "validated_ok": int((validated["code"] == 0).sum())},
            "clocks": clocks,
            "step_ms_min_max": [min(step_ms), max(step_ms)],
            "plain_sweep": {
                "value": sweep_value, "unit": UNIT, "ms_per_step": sweep_ms,
                "frontier_over_sweep": value / sweep_value, "same_costs": same,
                "roofline": {"bound": "hbm", "achieved": sweep_achieved, "peak": peak,
                             "unit": "GB/s", "frac": sweep_achieved / peak,
                             "traffic": (traffic or {}).get("dram_bytes_per_step"),
                             "bytes_alg_per_step": sbytes, "one_pass_bytes_per_step": one_pass},
                "sweeps_mean": float(sweep["results"]["sweeps"].mean()),
            },
        }
        if learned_form is not None:
            learned_form["learned_over_sweep"] = learned_form["value"] / sweep_value
            line["learned_corridor"] = learned_form
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"], cpu_costs = cpu_baseline(lat, nets, args.cpu_sample)
            ok = results["completion"][: args.cpu_sample] != apgar_b200.COMPLETION_REJECTED
            line["cpu_baseline"]["costs_match_gpu"] = bool(
                np.array_equal(cpu_costs[ok], results["cost"][: args.cpu_sample][ok]))
        print(json.dumps(line), flush=True)
    dev.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
