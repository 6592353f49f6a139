"""World-size-2 checks of the multi-GPU plumbing on CPU (gloo): net sharding,
the timing / count reductions bench.py uses, the usage sum of a
negotiated-congestion round followed by identical price updates on every
rank, and a whole ranked negotiation (split-round driver, CPU restatement in
place of the GPU steps) equal to one plan over all nets."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from apgar_b200 import negotiate, prices, shard, synth
from tests.negotiation_cpu import CpuRank, cpu_rounds


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        lat, _ = synth.config_small(3)
        nets = shard.rank_nets(lat, 5, rank, 6)
        # each rank certifies its own nets (the oracle stands in for the search)
        costs, _ = oracle.dijkstra_batch(lat, nets)
        certified = int((costs != oracle.lo_inf()).sum())
        total = shard.sum_over_ranks(certified, dist)
        slowest = shard.max_over_ranks(10.0 + rank, dist)
        # negotiated round: per-rank usage of its own paths, summed
        usage = torch.zeros(64, dtype=torch.int64)
        usage[rank * 8:(rank + 1) * 8] += 1
        usage[0] += 1  # both ranks use cell 0
        shard.allreduce_usage(usage, dist)
        rc, present, history, total_cost = oracle.price_epoch_update(
            usage.numpy(), np.zeros(64, np.uint64), 1, epoch=1)
        assert rc == 0
        out[rank] = dict(nets=nets.tobytes(), certified=certified, total=total, slowest=slowest,
                         usage=usage.numpy().copy(), price=total_cost.copy())
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_and_reduce():
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    r0, r1 = out[0], out[1]
    assert r0["nets"] != r1["nets"]  # each rank has its own batch
    assert r0["total"] == r1["total"] == r0["certified"] + r1["certified"]
    assert r0["slowest"] == r1["slowest"] == 11.0
    assert np.array_equal(r0["usage"], r1["usage"])
    assert r0["usage"][0] == 3 and r0["usage"][1:16].tolist() == [1] * 15
    assert np.array_equal(r0["price"], r1["price"])  # identical prices on every rank
    # capacity 1: only the shared cell is overused and priced
    assert r0["price"][0] > 0 and (r0["price"][1:] == 0).all()


def test_rank_batches_are_deterministic_and_splits_cover_the_batch():
    lat, _ = synth.config_small(3)
    a = shard.rank_nets(lat, 5, 1, 10)
    b = shard.rank_nets(lat, 5, 1, 10)
    assert np.array_equal(a, b)
    nets = shard.rank_nets(lat, 5, 0, 11)
    parts = [shard.split_nets(nets, r, 3) for r in range(3)]
    assert sum(len(p) for p in parts) == len(nets)
    assert np.array_equal(np.sort(np.concatenate(parts), order="start_x"),
                          np.sort(nets, order="start_x"))


def test_single_process_reductions_are_identities():
    assert shard.max_over_ranks(3.5) == 3.5
    assert shard.sum_over_ranks(7) == 7
    u = torch.arange(4)
    assert shard.allreduce_usage(u) is u


class _CpuRankNegotiation(negotiate.Negotiation):
    """The split-round negotiation of one rank with the CPU restatement in
    place of the GPU steps, so the ranked driver (Negotiation.run_ranked and
    shard.negotiate_ranked, the same code the GPU ranks run) is exercised over
    gloo."""

    def __init__(self, rank_state):
        self.state = rank_state
        self.cells = rank_state.cells
        self.rounds = 0
        self.handle = None
        self.calls = []

    def set_usage_buffer(self, usage):
        self.buffer = usage

    def step(self, round_index, phase, stream=0, partial=False):
        self.calls.append((round_index, phase))
        if phase == self.ROUTE:
            self.buffer.copy_(torch.from_numpy(self.state.route(round_index, partial).astype(np.int32)))
        else:
            self.state.price(round_index, self.buffer.numpy().astype(np.uint64))
            self.rounds = round_index + 1


def _negotiation_case():
    lat = synth.make_lattice(71, 2, 64, 0.15)
    nets = synth.make_nets(lat, 72, 16, hpwl_median=30.0, hpwl_sigma=0.5, margin=8)
    return lat, nets, prices.policy(initial=20, increment=20, history_increment=5, capacity=1)


def _negotiation_worker(rank, world, port, rounds, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        lat, nets, pol = _negotiation_case()
        state = CpuRank(lat, shard.split_nets(nets, rank, world), pol)
        neg = _CpuRankNegotiation(state)
        usage = shard.negotiate_ranked(neg, rounds, dist, partial=True, device="cpu")
        out[rank] = dict(usage=usage.numpy().copy(), history=state.history.copy(),
                         cost=state.cost.copy(), per_round=list(state.per_round),
                         costs=np.asarray(state.costs).copy(), calls=list(neg.calls))
    finally:
        dist.destroy_process_group()


def test_two_ranks_negotiate_like_one_plan():
    world, rounds = 2, 3
    out = mp.Manager().dict()
    mp.spawn(_negotiation_worker, args=(world, _free_port(), rounds, out), nprocs=world, join=True)
    lat, nets, pol = _negotiation_case()
    usage, history, cost, costs, _, per_round = cpu_rounds(lat, nets, pol, rounds, partial=True)
    assert per_round[0][0] > 0  # congested
    for rank in range(world):
        r = out[rank]
        assert np.array_equal(r["usage"].view(np.uint32), usage)
        assert np.array_equal(r["history"], history)
        assert np.array_equal(r["cost"], cost)
        assert r["per_round"] == per_round
        assert np.array_equal(r["costs"], costs[rank::world])
        assert r["calls"] == [(i, p) for i in range(rounds) for p in (0, 1)]


def test_balanced_split_covers_the_batch_and_balances_work():
    lat = synth.make_lattice(5, 2, 256, 0.2)
    nets = synth.make_nets(lat, 6, 500, hpwl_median=40.0, hpwl_sigma=1.0, margin=16)
    work = shard.window_work(nets, lat.layers)
    for world in (1, 2, 3, 8):
        parts = shard.balanced_split(nets, world, lat.layers)
        assert len(parts) == world
        allidx = np.concatenate(parts)
        assert np.array_equal(np.sort(allidx), np.arange(len(nets)))
        loads = np.array([work[p].sum() for p in parts])
        # LPT: no rank exceeds the mean by more than the largest single net
        assert loads.max() - loads.mean() <= work.max()
        again = shard.balanced_split(nets.copy(), world, lat.layers)  # deterministic
        assert all(np.array_equal(a, b) for a, b in zip(parts, again))

