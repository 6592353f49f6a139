"""The split-round negotiation (one rank's share of a multi-GPU run): ranks
emulated one after another on one GPU, each with its own plan over its share
of the nets, and the per-round usage sum done between the ROUTE and PRICE
steps (the one collective of a multi-GPU round).  Jacobi rounds make every
rank's routes, usage, history, prices and per-round overuse bit-identical to
one plan over all nets and to the CPU restatement."""

import numpy as np
import pytest
import torch

import apgar_b200
import oracle
from apgar_b200 import negotiate, prices, shard, synth
from tests.negotiation_cpu import cpu_rounds as _cpu_rounds

pytestmark = pytest.mark.gpu


def _case():
    lat = synth.make_lattice(61, 2, 128, 0.15, via_mask=True)
    nets = synth.make_nets(lat, 62, 48, hpwl_median=50.0, hpwl_sigma=0.5, margin=12)
    pol = prices.policy(initial=20, increment=20, history_increment=5, capacity=1)
    return lat, nets, pol


@pytest.mark.parametrize("split", ["round_robin", "balanced"])
@pytest.mark.parametrize("partial", [False, True])
@pytest.mark.parametrize("world", [1, 2, 3])
def test_emulated_ranks_match_one_plan(world, partial, split):
    lat, nets, pol = _case()
    rounds = 4
    usage_c, history_c, cost_c, costs_c, paths_c, per_round_c = _cpu_rounds(lat, nets, pol, rounds,
                                                                            partial)
    dev = apgar_b200.DeviceLattice(lat)
    try:
        if split == "balanced":
            shares = shard.balanced_split(nets, world, lat.layers)
        else:
            shares = [np.arange(len(nets))[r::world] for r in range(world)]
        plans = [dev.plan(np.ascontiguousarray(nets[shares[r]]), generator="frontier")
                 for r in range(world)]
        negs = [negotiate.Negotiation(p, pol) for p in plans]
        usages = [torch.zeros(negs[0].cells, dtype=torch.int32, device="cuda") for _ in range(world)]
        for n, u in zip(negs, usages):
            n.set_usage_buffer(u)
        for r in range(rounds):
            for n in negs:
                n.step(r, n.ROUTE, partial=partial)
            total = torch.stack(usages).sum(0, dtype=torch.int32)
            for u in usages:
                u.copy_(total)
            for n in negs:
                n.step(r, n.PRICE, partial=partial)
        torch.cuda.synchronize()
        for rank, (n, p) in enumerate(zip(negs, plans)):
            usage, history, cost, rows = n.readback()
            assert np.array_equal(usage, usage_c)
            assert np.array_equal(history, history_c)
            assert np.array_equal(cost, cost_c)
            assert [(x["overused_cells"], x["total_overuse"]) for x in rows] == per_round_c
            res, paths = p.readback()
            per = apgar_b200.split_paths(res, paths)
            for k, i in enumerate(shares[rank]):
                assert res["cost"][k] == costs_c[i]
                if costs_c[i] != oracle.lo_inf():
                    assert np.array_equal(per[k], paths_c[i]), (rank, i)
        for n in negs:
            n.close()
        for p in plans:
            p.close()
    finally:
        dev.close()


def test_single_rank_steps_equal_the_whole_run():
    lat, nets, pol = _case()
    dev = apgar_b200.DeviceLattice(lat)
    try:
        plan = dev.plan(nets, generator="frontier")
        neg = negotiate.Negotiation(plan, pol)
        neg.run(5, use_graph=True, partial=True)
        whole = neg.readback()
        whole_res, whole_paths = plan.readback()
        usage = shard.negotiate_ranked(neg, 5, dist=None, partial=True)
        torch.cuda.synchronize()
        steps = neg.readback()
        res, paths = plan.readback()
        for a, b in zip(whole[:3], steps[:3]):
            assert np.array_equal(a, b)
        assert whole[3] == steps[3]
        assert np.array_equal(usage.cpu().numpy().view(np.uint32), steps[0])
        assert np.array_equal(whole_res["cost"], res["cost"])
        assert np.array_equal(whole_paths, paths)
        # back on its own buffer, the graph form runs again unchanged
        neg.set_usage_buffer(None)
        neg.run(5, use_graph=True, partial=True)
        again = neg.readback()
        for a, b in zip(whole[:3], again[:3]):
            assert np.array_equal(a, b)
        neg.close()
        plan.close()
    finally:
        dev.close()


def test_steps_are_checked():
    lat, nets, pol = _case()
    dev = apgar_b200.DeviceLattice(lat)
    try:
        plan = dev.plan(nets[:8].copy(), generator="frontier")
        neg = negotiate.Negotiation(plan, pol)
        with pytest.raises(apgar_b200.BackendError):
            neg.step(0, neg.PRICE)                 # PRICE before ROUTE
        neg.step(0, neg.ROUTE)
        with pytest.raises(apgar_b200.BackendError):
            neg.step(1, neg.ROUTE)                 # round 0 not priced
        neg.step(0, neg.PRICE)
        with pytest.raises(apgar_b200.BackendError):
            neg.step(2, neg.ROUTE)                 # skips round 1
        neg.step(1, neg.ROUTE)
        neg.step(0, neg.ROUTE)                     # round 0 restarts
        neg.step(0, neg.PRICE)
        with pytest.raises(apgar_b200.BackendError):
            neg.step(1000, neg.ROUTE)
        with pytest.raises(ValueError):
            neg.set_usage_buffer(torch.zeros(7, dtype=torch.int32, device="cuda"))
        with pytest.raises(ValueError):
            neg.set_usage_buffer(torch.zeros(neg.cells, dtype=torch.int32))
        host = torch.zeros(neg.cells, dtype=torch.int32)
        with pytest.raises(apgar_b200.BackendError):    # host memory, through the C ABI
            apgar_b200._check(apgar_b200.lib().apgar_b200_negotiation_set_usage_buffer(
                neg.handle, apgar_b200.ctypes.c_void_p(host.data_ptr())))
        neg.close()
        plan.close()
    finally:
        dev.close()
