"""Python mirror of the congestion-price entry points (C ABI section C).

``update`` runs the fused integer price pass on the GPU over host arrays;
``accumulate_usage`` adds the path cells of a planned lattice batch to a
usage array on the device (returned as numpy).
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _check, lib

PRICE_OVERFLOW = 1
PRICE_BOUND = 2
U64_MAX = (1 << 64) - 1


class PricePolicy(ctypes.Structure):
    _fields_ = [
        ("initial_present_factor", ctypes.c_uint64),
        ("present_factor_increment", ctypes.c_uint64),
        ("historical_price_increment", ctypes.c_uint64),
        ("capacity", ctypes.c_uint64),
        ("maximum_value", ctypes.c_uint64),
    ]


def policy(initial=100, increment=100, history_increment=10, capacity=1, maximum=U64_MAX):
    """Reference defaults: NegotiatedPriceUpdatePolicyV1 (100 / +100 / +10)."""
    return PricePolicy(initial, increment, history_increment, capacity, maximum)


def update(usage, history, pol: PricePolicy, epoch: int, want_next=True):
    """Returns (present, history', total, next_cost or None, status bits)."""
    usage = np.ascontiguousarray(usage, dtype=np.uint32)
    hist = np.ascontiguousarray(history, dtype=np.uint64).copy()
    n = len(usage)
    present = np.zeros(n, np.uint64)
    total = np.zeros(n, np.uint64)
    nxt = np.zeros(n, np.uint64) if want_next else None
    status = ctypes.c_uint32(0)
    vp = lambda a: None if a is None else ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    _check(lib().apgar_b200_price_update(ctypes.c_uint32(n), vp(usage), ctypes.byref(pol),
                                         ctypes.c_uint64(epoch), vp(present), vp(hist), vp(total),
                                         vp(nxt), ctypes.byref(status)))
    return present, hist, total, nxt, status.value


def accumulate_usage(plan, cell_count: int, usage=None):
    """Usage counts (uint32 per global cell id) of a planned batch's paths."""
    import torch

    dev = torch.zeros(cell_count, dtype=torch.int32, device="cuda") if usage is None else usage
    _check(lib().apgar_b200_lattice_accumulate_usage(plan.handle, ctypes.c_void_p(dev.data_ptr()),
                                                     ctypes.c_uint64(cell_count), None))
    torch.cuda.synchronize()
    return dev.cpu().numpy().view(np.uint32)
