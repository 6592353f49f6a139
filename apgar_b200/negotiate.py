"""Negotiated-congestion rounds (rip-up and reroute) on a frontier plan.

Host mirror of the apgar_b200_negotiation_* C ABI: every round reroutes all
nets of the plan (or, with partial rip-up, only those crossing overused
cells) against frozen per-cell snapshot prices, with each net's own previous
cells priced from the other nets' usage; then it counts per-cell usage and
runs the fused price pass (history and the next snapshot).  The whole run can
be captured once as a CUDA graph and replayed.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _check, lib
from .prices import PricePolicy


class RoundStats(ctypes.Structure):
    _fields_ = [
        ("overused_cells", ctypes.c_uint64),
        ("total_overuse", ctypes.c_uint64),
        ("price_status", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]


class Negotiation:
    def __init__(self, plan, policy: PricePolicy):
        if plan.generator != "frontier":
            raise ValueError("negotiated rounds need a frontier plan")
        self.plan = plan
        self.policy = policy
        self.cells = plan.lattice.layers * plan.lattice.height * plan.lattice.width
        self.rounds = 0
        self._usage_buffer = None
        handle = ctypes.c_void_p()
        _check(lib().apgar_b200_negotiation_create(plan.handle, ctypes.byref(policy),
                                                   ctypes.byref(handle)))
        self.handle = handle

    def run(self, rounds: int, use_graph: bool = False, stream: int = 0,
            partial: bool = False) -> None:
        """A whole negotiation from zero prices.  ``partial``: from round 1 on,
        reroute only nets whose route crosses an overused cell."""
        flags = (1 if use_graph else 0) | (2 if partial else 0)
        _check(lib().apgar_b200_negotiation_run_ex(self.handle, ctypes.c_uint32(rounds),
                                                   ctypes.c_uint32(flags), ctypes.c_void_p(stream)))
        self.rounds = rounds

    ROUTE, PRICE = 0, 1

    def step(self, round_index: int, phase: int, stream: int = 0, partial: bool = False) -> None:
        """One phase of one round of the split-round form: ROUTE (reroute this
        plan's nets, count their usage; round 0 first zeroes history and
        prices) or PRICE (the fused price pass over the usage buffer)."""
        _check(lib().apgar_b200_negotiation_step(self.handle, ctypes.c_uint32(round_index),
                                                 ctypes.c_uint32(phase),
                                                 ctypes.c_uint32(2 if partial else 0),
                                                 ctypes.c_void_p(stream)))
        if phase == self.PRICE:
            self.rounds = round_index + 1

    def set_usage_buffer(self, usage) -> None:
        """Counts usage into ``usage`` (a CUDA int32 tensor of one element per
        lattice cell on the plan's device), or back into the negotiation's own
        buffer with None."""
        if usage is not None:
            if (not usage.is_cuda or usage.numel() != self.cells or usage.element_size() != 4
                    or not usage.is_contiguous()):
                raise ValueError("usage buffer must be a contiguous 32-bit CUDA tensor of one entry per cell")
        self._usage_buffer = usage  # kept alive while the negotiation uses it
        _check(lib().apgar_b200_negotiation_set_usage_buffer(
            self.handle, ctypes.c_void_p(usage.data_ptr() if usage is not None else None)))

    def run_ranked(self, rounds: int, usage, sum_usage, stream: int = 0,
                   partial: bool = False) -> None:
        """This rank's share of a multi-GPU negotiation: the plan holds the
        rank's segments; after each round's ROUTE, ``sum_usage(usage)`` sums
        the usage tensor over all ranks in place (one integer all-reduce),
        then every rank runs the same PRICE pass.  Jacobi rounds make the
        ranks' routes exactly those of one plan over all segments."""
        self.set_usage_buffer(usage)
        for r in range(rounds):
            self.step(r, self.ROUTE, stream, partial)
            sum_usage(usage)
            self.step(r, self.PRICE, stream, partial)

    def device_prices(self) -> int:
        """Device address of the current snapshot prices (uint32 per cell)."""
        ptr = ctypes.c_void_p()
        _check(lib().apgar_b200_negotiation_device_prices(self.handle, ctypes.byref(ptr)))
        return ptr.value

    def run_learned(self, rounds: int, router, stream: int = 0, partial: bool = False,
                    from_round: int = 1) -> None:
        """A whole negotiation in split-round steps with a learned corridor
        proposal before each priced round: ``router`` (a
        ``learned.LearnedRouter`` on this negotiation's plan) reads the
        current snapshot as its congestion raster and sets every net's
        corridor; rounds before ``from_round`` search without corridors.
        Corridor results are certified or searched again over the window, so
        the routes, usage and prices equal those of ``run``."""
        prices = self.device_prices()
        for r in range(rounds):
            if r >= from_round:
                router.propose(stream, cell_costs=prices)
            else:
                router.clear(stream)
            self.step(r, self.ROUTE, stream, partial)
            self.step(r, self.PRICE, stream, partial)

    def readback(self):
        """(usage, history, next snapshot prices, per-round stats list)."""
        usage = np.empty(self.cells, np.uint32)
        history = np.empty(self.cells, np.uint64)
        costs = np.empty(self.cells, np.uint32)
        stats = (RoundStats * max(self.rounds, 1))()
        _check(lib().apgar_b200_negotiation_readback(
            self.handle, usage.ctypes.data_as(ctypes.c_void_p), history.ctypes.data_as(ctypes.c_void_p),
            costs.ctypes.data_as(ctypes.c_void_p), stats, ctypes.c_uint32(self.rounds)))
        rows = [dict(overused_cells=s.overused_cells, total_overuse=s.total_overuse,
                     price_status=s.price_status) for s in stats[: self.rounds]]
        return usage, history, costs, rows

    def close(self):
        if self.handle:
            lib().apgar_b200_negotiation_release(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
