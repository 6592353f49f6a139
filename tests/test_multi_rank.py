"""World-size-2 checks of the multi-GPU plumbing on CPU (gloo): net sharding,
the timing / count reductions bench.py uses, and the usage sum of a
negotiated-congestion round followed by identical price updates on every
rank."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from apgar_b200 import shard, synth


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
