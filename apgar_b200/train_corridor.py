"""Trains the corridor CNN on the GPU and evaluates it on held-out nets.

    python -m apgar_b200.train_corridor [--paths 200000] [--epochs 3]
        [--out apgar_b200/weights/corridor_net.f32] [--report FILE]
    python -m apgar_b200.train_corridor --priced [--paths 200000]
        [--out apgar_b200/weights/corridor_net_priced.f32] [--report FILE]

Training data: optimal paths of the plain batched sweep on seeded lattices of
the medium distribution (4 layers of 2048^2, 25% blocked with pad keep-outs,
lognormal(200, 1.0) half-perimeters, bbox + 32 windows), 4096 nets per batch,
several net batches per lattice.  The coarse label of a net is 1 where its
path has a cell.  Training runs the project's own forward, backward and Adam
kernels (apgar_b200.learned).

Evaluation: the 4096 nets of the medium workload (lattice seed 2, never
trained on), through the frontier's corridor mode for a few corridor policies
(logit threshold, coarse dilation).  It reports, per policy, the certificate
pass rate, the fallback rates, whether every cost equals the plain frontier's,
the mean corridor area as a fraction of the window, and the execution time;
the fastest policy is written next to the weights.

With --priced the network is trained for negotiated congestion rounds: the
data are the priced-optimal paths of full rip-up negotiation rounds on seeded
lattices of the negotiated distribution (2-6 terminal nets split into 2-pin
segments, lognormal(300, 1.2) half-perimeters, capacity 1), each raster
carrying the round's snapshot prices as its congestion channel (round 0
unpriced).  Evaluation: the negotiated workload (6 layers of 4096^2, 49,544
segments, 10 rounds with partial rip-up, never trained on), timed with
corridors proposed before every priced round against the plain negotiation,
per corridor policy; the results must be identical, and the fastest policy
is written next to the weights (corridor_policy_priced.json).
"""

from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

import apgar_b200
from apgar_b200 import corridor, learned, synth

POLICY_PATH = os.path.join(os.path.dirname(learned.WEIGHTS_PATH), "corridor_policy.json")
# Windows above 2^19 cells get no corridor: measured on the medium batch, a
# corridor never shortens a frontier search's rounds, and the widest nets
# (the batch's critical path) fall back more often (18% of them), which
# searches them twice (32.1 ms per batch with corridors on every net, 25.6
# ms without them above 2^19 cells).
MAX_WINDOW_CELLS = 1 << 19


def training_batches(paths: int, nets_per_batch: int = 4096, batches_per_lattice: int = 7,
                     size: int = 2048, first_seed: int = 100):
    """Yields (lattice, nets) batches until `paths` nets are produced."""
    produced, k = 0, 0
    while produced < paths:
        lat = synth.make_lattice(first_seed + k, 4, size, 0.25, pads=True)
        for b in range(batches_per_lattice):
            if produced >= paths:
                break
            n = min(nets_per_batch, paths - produced)
            nets = synth.make_nets(lat, 10_000 + 97 * k + b, n, hpwl_median=200.0,
                                   hpwl_sigma=1.0)
            produced += n
            yield lat, nets
        k += 1


def build_dataset(paths: int, log=print):
    """Rasters, dims and labels of `paths` sweep-routed nets, resident on the GPU."""
    import torch

    rasters, dims, labels = [], [], []
    t0 = time.time()
    for lat, nets in training_batches(paths):
        dev = apgar_b200.DeviceLattice(lat)
        plan = dev.plan(nets, generator="sweep")
        plan.execute()
        r, d = learned.rasters(plan)
        lab = learned.labels(plan, d)
        torch.cuda.synchronize()
        rasters.append(r)
        dims.append(d)
        labels.append(lab)
        plan.close()
        dev.close()
        log(f"dataset: {sum(x.shape[0] for x in rasters)} paths ({time.time() - t0:.1f} s)")
    return torch.cat(rasters), torch.cat(dims), torch.cat(labels)


PRICED_WEIGHTS_PATH = os.path.join(os.path.dirname(learned.WEIGHTS_PATH), "corridor_net_priced.f32")
PRICED_POLICY_PATH = os.path.join(os.path.dirname(learned.WEIGHTS_PATH), "corridor_policy_priced.json")


def priced_dataset(samples: int, rounds: int = 6, size: int = 2048, first_seed: int = 300,
                   log=print):
    """Rasters with the snapshot's congestion channel, dims and labels of the
    priced-optimal paths of full rip-up negotiation rounds, resident on the
    GPU.  Each lattice contributes every segment of every round."""
    import ctypes

    import torch

    from . import _check, lib, negotiate, prices

    rasters, dims, labels = [], [], []
    got, k = 0, 0
    t0 = time.time()
    while got < samples:
        lat = synth.make_lattice(first_seed + k, 4, size, 0.25, pads=True)
        segs, _ = synth.make_multi_terminal_nets(lat, 5000 + k, 4096, 300.0, 1.2)
        dev = apgar_b200.DeviceLattice(lat)
        plan = dev.plan(segs, generator="frontier")
        neg = negotiate.Negotiation(plan, prices.policy(capacity=1))
        snapshot = neg.device_prices()
        n = len(segs)
        for r in range(rounds):
            if got >= samples:
                break
            ras = torch.zeros((n, learned.PADDED_ROWS, learned.GRID, learned.RASTER_CHANNELS),
                              dtype=torch.bfloat16, device="cuda")
            dim = torch.empty(n, dtype=torch.uint32, device="cuda")
            # the snapshot the round's search is priced by (round 0: none)
            _check(lib().apgar_b200_corridor_rasters(
                plan.handle, ctypes.c_void_p(snapshot) if r > 0 else None,
                ctypes.c_void_p(ras.data_ptr()), ctypes.c_void_p(dim.data_ptr()), None))
            neg.step(r, neg.ROUTE, 0, partial=False)
            lab = learned.labels(plan, dim)
            neg.step(r, neg.PRICE, 0, partial=False)
            torch.cuda.synchronize()
            take = min(n, samples - got)
            rasters.append(ras[:take])
            dims.append(dim[:take])
            labels.append(lab[:take])
            got += take
        neg.close()
        plan.close()
        dev.close()
        k += 1
        log(f"priced dataset: {got} paths ({time.time() - t0:.1f} s)")
    return torch.cat(rasters), torch.cat(dims), torch.cat(labels)


def evaluate_priced(net, policies, rounds: int = 10, log=print):
    """Negotiated workload: plain negotiation against learned proposals before
    every priced round, per policy (threshold, dilate); ms per negotiation,
    identical results, and the last round's corridor outcomes."""
    import torch

    from . import negotiate, prices

    lat, segs, _ = synth.config_negotiated()
    dev = apgar_b200.DeviceLattice(lat)
    pol = prices.policy(capacity=1)
    stream = torch.cuda.current_stream()

    def timed(fn):
        fn()  # warm-up
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        fn()
        e.record(stream)
        e.synchronize()
        return s.elapsed_time(e)

    plan = dev.plan(segs, generator="frontier")
    neg = negotiate.Negotiation(plan, pol)
    plain_ms = timed(lambda: neg.run(rounds, stream=stream.cuda_stream, partial=True))
    base = neg.readback()
    base_res, _ = plan.readback(want_paths=False)
    neg.close()
    plan.close()
    rows = []
    for threshold, dilate in policies:
        plan = dev.plan(segs, generator="frontier")
        neg = negotiate.Negotiation(plan, pol)
        router = learned.LearnedRouter(plan, net=net, policy={
            "threshold": threshold, "dilate": dilate, "max_window_cells": MAX_WINDOW_CELLS})
        ms = timed(lambda: neg.run_learned(rounds, router, stream.cuda_stream, partial=True))
        got = neg.readback()
        res, _ = plan.readback(want_paths=False)
        st = plan.corridor_status()
        same = (all(np.array_equal(a, b) for a, b in zip(base[:3], got[:3])) and base[3] == got[3]
                and np.array_equal(base_res["cost"], res["cost"]))
        row = {"threshold": threshold, "dilate": dilate, "ms": round(ms, 1), "same_results": bool(same),
               "last_round_certified": float((st == corridor.CERTIFIED).mean()),
               "last_round_fallback": float(((st == corridor.FALLBACK_EXIT)
                                             | (st == corridor.FALLBACK_UNREACHED)).mean())}
        rows.append(row)
        log(json.dumps(row))
        neg.close()
        plan.close()
    dev.close()
    return plain_ms, rows


def train(net, rasters, dims, labels, epochs: int, batch: int = 1024, lr: float = 2e-3,
          pos_weight: float = 8.0, seed: int = 0, log=print):
    import torch

    n = rasters.shape[0]
    g = torch.Generator(device="cpu").manual_seed(seed)
    acts = net.activations(batch, distinct=True)
    history = []
    steps = epochs * (n // batch)
    step = 0
    for epoch in range(epochs):
        order = torch.randperm(n, generator=g).cuda()
        total = 0.0
        for b in range(n // batch):
            idx = order[b * batch:(b + 1) * batch]
            # cosine decay of the step size
            rate = lr * 0.5 * (1.0 + np.cos(np.pi * step / max(steps, 1)))
            d = dims.view(torch.int32)[idx].contiguous().view(torch.uint32)
            loss = net.train_step(rasters[idx].contiguous(), d, labels[idx].contiguous(), rate,
                                  pos_weight, acts=acts)
            total += loss.item()
            step += 1
        net.check_error()
        history.append(total / max(1, n // batch))
        log(f"epoch {epoch}: mean loss {history[-1]:.5f}")
    return history


def evaluate(net, policies, log=print):
    """Corridor-mode outcomes on the medium workload's 4096 nets."""
    import torch

    lat, nets = synth.config_medium(2)
    dev = apgar_b200.DeviceLattice(lat)
    plan = dev.plan(nets, generator="frontier")

    def timed(k=5):
        for _ in range(2):
            plan.execute()
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(k):
            plan.execute()
        e.record()
        torch.cuda.synchronize()
        return s.elapsed_time(e) / k

    plain_ms = timed()
    base, _ = plan.readback(want_paths=False)
    r, d = learned.rasters(plan)
    logits = net.forward(r, d)
    torch.cuda.synchronize()
    net.check_error()
    dims = d.view(torch.int32).cpu().numpy().view(np.uint32)
    cw, ch = (dims & 0xFF).astype(np.float64), ((dims >> 8) & 0xFF).astype(np.float64)
    rows = []
    for threshold, dilate in policies:
        bits = learned.corridors(plan, logits, d, threshold=threshold, dilate=dilate,
                                 max_window_cells=MAX_WINDOW_CELLS)
        plan.set_corridors(bits)
        ms = timed()
        st = plan.corridor_status()
        res, _ = plan.readback(want_paths=False)
        area = corridor.unpack(bits.view(torch.int32).cpu().numpy().view(np.uint32)).sum(axis=(1, 2))
        row = {
            "threshold": threshold, "dilate": dilate, "ms": round(ms, 3),
            "certified": float((st == corridor.CERTIFIED).mean()),
            "fallback_exit": float((st == corridor.FALLBACK_EXIT).mean()),
            "fallback_unreached": float((st == corridor.FALLBACK_UNREACHED).mean()),
            "costs_equal_plain": bool(np.array_equal(res["cost"], base["cost"])),
            "area_fraction": float((area / (cw * ch)).mean()),
        }
        rows.append(row)
        log(json.dumps(row))
        plan.set_corridors(None)
    plan.close()
    dev.close()
    return plain_ms, rows


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--paths", type=int, default=200_000)
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--batch", type=int, default=1024)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=None)
    ap.add_argument("--report", default=None)
    ap.add_argument("--priced", action="store_true",
                    help="train on priced negotiation rounds and evaluate on the negotiated workload")
    args = ap.parse_args(argv)

    import torch

    if args.priced:
        return main_priced(args)
    args.out = args.out or learned.WEIGHTS_PATH
    t0 = time.time()
    rasters, dims, labels = build_dataset(args.paths)
    t1 = time.time()
    net = learned.CorridorNet(seed=0)
    history = train(net, rasters, dims, labels, args.epochs, batch=args.batch, lr=args.lr)
    torch.cuda.synchronize()
    t2 = time.time()
    net.save(args.out)
    policies = [(t, r) for t in (-2.0, -1.0, 0.0) for r in (1, 2, 3)]
    plain_ms, rows = evaluate(net, policies)
    ok = [row for row in rows if row["costs_equal_plain"]]
    best = min(ok, key=lambda row: row["ms"]) if ok else None
    if best is not None:
        with open(os.path.join(os.path.dirname(args.out), "corridor_policy.json"), "w") as f:
            json.dump({"threshold": best["threshold"], "dilate": best["dilate"],
                       "max_window_cells": MAX_WINDOW_CELLS}, f)
    report = {
        "paths": int(rasters.shape[0]), "epochs": args.epochs, "batch": args.batch, "lr": args.lr,
        "dataset_s": round(t1 - t0, 1), "train_s": round(t2 - t1, 1), "loss": history,
        "plain_frontier_ms": round(plain_ms, 3), "policies": rows, "chosen": best,
    }
    print(json.dumps(report))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1)


def main_priced(args):
    import torch

    out = args.out or PRICED_WEIGHTS_PATH
    t0 = time.time()
    rasters, dims, labels = priced_dataset(args.paths)
    t1 = time.time()
    net = learned.CorridorNet(seed=0)
    history = train(net, rasters, dims, labels, args.epochs, batch=args.batch, lr=args.lr)
    torch.cuda.synchronize()
    t2 = time.time()
    samples = int(rasters.shape[0])
    del rasters, dims, labels
    torch.cuda.empty_cache()
    net.save(out)
    policies = [(-2.0, 3), (-2.0, 5), (-3.0, 4), (-3.0, 6), (-4.0, 6)]
    plain_ms, rows = evaluate_priced(net, policies)
    ok = [row for row in rows if row["same_results"]]
    best = min(ok, key=lambda row: row["ms"]) if ok else None
    if best is not None:
        with open(os.path.join(os.path.dirname(out), os.path.basename(PRICED_POLICY_PATH)), "w") as f:
            json.dump({"threshold": best["threshold"], "dilate": best["dilate"],
                       "max_window_cells": MAX_WINDOW_CELLS}, f)
    report = {
        "paths": samples, "epochs": args.epochs, "batch": args.batch, "lr": args.lr,
        "dataset_s": round(t1 - t0, 1), "train_s": round(t2 - t1, 1), "loss": history,
        "plain_negotiation_ms": round(plain_ms, 1), "policies": rows, "chosen": best,
    }
    print(json.dumps(report))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1)


if __name__ == "__main__":
    main()
