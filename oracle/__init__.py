"""ctypes binding for the CPU oracle.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm
may import this package; the product (apgar_b200) never does.  See oracle.h for
what each routine restates and which reference file:line it follows.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

U32P = ctypes.POINTER(ctypes.c_uint32)
U64P = ctypes.POINTER(ctypes.c_uint64)


class LoLattice(ctypes.Structure):
    _fields_ = [
        ("layers", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("width", ctypes.c_int32),
        ("blocked", U32P),
        ("via_ok", U32P),
        ("orth", ctypes.c_uint32),
        ("diag", ctypes.c_uint32),
        ("via", ctypes.c_uint32),
        ("cell_cost", U32P),
    ]


class LoSweepStats(ctypes.Structure):
    _fields_ = [
        ("sweeps", ctypes.c_uint32),
        ("row_visits", ctypes.c_uint64),
        ("row_stores", ctypes.c_uint64),
        ("cells_loaded", ctypes.c_uint64),
        ("cells_stored", ctypes.c_uint64),
        ("row_loads", ctypes.c_uint64),
    ]


class GoCosts(ctypes.Structure):
    _fields_ = [
        ("orthogonal_step", ctypes.c_uint32),
        ("diagonal_step", ctypes.c_uint32),
        ("bend", ctypes.c_uint32),
    ]


class GoQuery(ctypes.Structure):
    _fields_ = [
        ("start_node", ctypes.c_uint32),
        ("goal_node", ctypes.c_uint32),
        ("orthogonal_step_surcharge", ctypes.c_uint64),
        ("diagonal_step_surcharge", ctypes.c_uint64),
        ("bend_surcharge", ctypes.c_uint64),
        ("policy", ctypes.c_void_p),
        ("policy_count", ctypes.c_uint32),
    ]


def lo_inf() -> int:
    return 0xFFFFFFFF


def build() -> str:
    """Compile the oracle with make (gcc); returns the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.lo_dijkstra.restype = ctypes.c_uint32
        _lib.lo_astar.restype = ctypes.c_uint32
        _lib.lo_sweep_schedule.restype = ctypes.c_uint32
        _lib.go_search.restype = ctypes.c_int
        _lib.go_validate_compact.restype = ctypes.c_int
        _lib.po_epoch_update.restype = ctypes.c_int
        _lib.po_snapshot_costs.restype = ctypes.c_int
        _lib.po_history_update.restype = ctypes.c_int
    return _lib


def _ptr(a, t=U32P):
    return a.ctypes.data_as(t)


class LatticeRef:
    """Keeps the numpy buffers alive while the C struct points at them."""

    def __init__(self, lat, cell_cost=None):
        self.blocked = np.ascontiguousarray(lat.blocked, dtype=np.uint32)
        self.via_ok = None if lat.via_ok is None else np.ascontiguousarray(lat.via_ok, np.uint32)
        self.cell_cost = None if cell_cost is None else np.ascontiguousarray(cell_cost, np.uint32)
        if self.cell_cost is not None:
            assert self.cell_cost.size == lat.layers * lat.height * lat.width
        self.c = LoLattice(
            lat.layers, lat.height, lat.width, _ptr(self.blocked),
            _ptr(self.via_ok) if self.via_ok is not None else U32P(),
            lat.orth, lat.diag, lat.via,
            _ptr(self.cell_cost) if self.cell_cost is not None else U32P())


def _net_ptr(nets):
    return nets.ctypes.data_as(ctypes.c_void_p)


def dijkstra(lat, net_row, full=False, want_dist=False, path_cap=1 << 22, cell_cost=None):
    """Returns (cost, reverse canonical path as uint32 array, dist or None)."""
    L = lib()
    ref = LatticeRef(lat, cell_cost)
    net = np.array([net_row], dtype=net_row.dtype) if not isinstance(net_row, np.ndarray) else net_row
    net = np.ascontiguousarray(net.reshape(1))
    cells = lat.layers * int(net["win_w"][0]) * int(net["win_h"][0])
    dist = np.empty(cells, dtype=np.uint32) if want_dist else None
    path = np.empty(path_cap, dtype=np.uint32)
    plen = ctypes.c_uint32(0)
    cost = L.lo_dijkstra(ctypes.byref(ref.c), _net_ptr(net), int(full),
                         _ptr(dist) if dist is not None else U32P(), _ptr(path),
                         ctypes.c_uint32(path_cap), ctypes.byref(plen))
    n = plen.value
    return cost, (path[:n].copy() if n != 0xFFFFFFFF else None), dist


def dijkstra_batch(lat, nets, threads=None, path_cap_per_net=None, cell_cost=None):
    """Exact costs and canonical reverse paths of every net; ``cell_cost``
    (optional, uint32 [layers][height][width]) adds a per-cell entry price."""
    L = lib()
    ref = LatticeRef(lat, cell_cost)
    nets = np.ascontiguousarray(nets)
    count = len(nets)
    threads = threads or os.cpu_count() or 1
    # canonical paths are bounded by window cells; use the Chebyshev-bounded
    # estimate w*h*layers capped to keep memory small for tests
    caps = (nets["win_w"].astype(np.uint64) * nets["win_h"].astype(np.uint64) * lat.layers)
    if path_cap_per_net is not None:
        caps = np.minimum(caps, np.uint64(path_cap_per_net))
    offsets = np.zeros(count, dtype=np.uint64)
    offsets[1:] = np.cumsum(caps)[:-1]
    total = int(caps.sum())
    paths = np.empty(total, dtype=np.uint32)
    costs = np.empty(count, dtype=np.uint32)
    lens = np.empty(count, dtype=np.uint32)
    L.lo_dijkstra_batch(ctypes.byref(ref.c), _net_ptr(nets), ctypes.c_uint32(count),
                        ctypes.c_int(threads), _ptr(costs), _ptr(lens), _ptr(offsets, U64P),
                        _ptr(paths), ctypes.c_uint64(total))
    out = []
    for i in range(count):
        n = int(lens[i])
        if n == 0xFFFFFFFF:
            out.append(None)
        else:
            o = int(offsets[i])
            out.append(paths[o:o + n].copy())
    return costs, out


def astar_batch(lat, nets, threads=None):
    L = lib()
    ref = LatticeRef(lat)
    nets = np.ascontiguousarray(nets)
    costs = np.empty(len(nets), dtype=np.uint32)
    L.lo_astar_batch(ctypes.byref(ref.c), _net_ptr(nets), ctypes.c_uint32(len(nets)),
                     ctypes.c_int(threads or os.cpu_count() or 1), _ptr(costs))
    return costs


def sweep_batch(lat, nets, threads=None, max_sweeps=100000):
    L = lib()
    ref = LatticeRef(lat)
    nets = np.ascontiguousarray(nets)
    costs = np.empty(len(nets), dtype=np.uint32)
    stats = (LoSweepStats * len(nets))()
    L.lo_sweep_batch(ctypes.byref(ref.c), _net_ptr(nets), ctypes.c_uint32(len(nets)),
                     ctypes.c_int(threads or os.cpu_count() or 1), ctypes.c_uint32(max_sweeps),
                     _ptr(costs), stats)
    rows = [(s.sweeps, s.row_visits, s.row_stores, s.cells_loaded, s.cells_stored, s.row_loads)
            for s in stats]
    return costs, np.array(rows, dtype=np.uint64).reshape(len(nets), 6)


def sweep_one(lat, net_row, max_sweeps=100000):
    L = lib()
    ref = LatticeRef(lat)
    net = np.ascontiguousarray(np.asarray(net_row).reshape(1))
    cells = lat.layers * int(net["win_w"][0]) * int(net["win_h"][0])
    dist = np.empty(cells, dtype=np.uint32)
    st = LoSweepStats()
    cost = L.lo_sweep_schedule(ctypes.byref(ref.c), _net_ptr(net), ctypes.c_uint32(max_sweeps),
                               _ptr(dist), ctypes.byref(st))
    return cost, dist, st


def graph_search(nodes, costs, start, goal, orth_s=0, diag_s=0, bend_s=0, policy=None,
                 want_labels=False, path_cap=None):
    """Exact heading-state search over DeviceCompiledBoardV1 node records.

    Returns (reached, goal_cost, goal_state, reverse compact path, labels)."""
    L = lib()
    nodes = np.ascontiguousarray(nodes)
    n = len(nodes)
    labels = np.empty(9 * n, dtype=np.uint64) if want_labels else None
    cap = path_cap or 9 * n
    path = np.empty(cap, dtype=np.uint32)
    pol = np.ascontiguousarray(policy) if policy is not None and len(policy) else None
    q = GoQuery(start, goal, orth_s, diag_s, bend_s,
                pol.ctypes.data_as(ctypes.c_void_p) if pol is not None else None,
                len(pol) if pol is not None else 0)
    gc = ctypes.c_uint64(0)
    gs = ctypes.c_uint32(0)
    plen = ctypes.c_uint32(0)
    reached = L.go_search(nodes.ctypes.data_as(ctypes.c_void_p), ctypes.c_uint32(n),
                          GoCosts(*costs), ctypes.byref(q),
                          labels.ctypes.data_as(U64P) if labels is not None else U64P(),
                          ctypes.byref(gc), ctypes.byref(gs), _ptr(path), ctypes.c_uint32(cap),
                          ctypes.byref(plen))
    return bool(reached), gc.value, gs.value, path[: plen.value].copy(), labels


PATH_CODES = {0: "ok", 1: "bounds", 2: "endpoint", 3: "cycle", 4: "heading", 5: "edge",
              6: "banned", 7: "not_reached"}


def validate_compact(nodes, costs, start, goal, reverse_states, goal_state, completion=0,
                     orth_s=0, diag_s=0, bend_s=0, policy=None):
    """Structural validation of one compact reverse path.  Returns
    (code name, total cost, failing forward index)."""
    L = lib()
    nodes = np.ascontiguousarray(nodes)
    rev = np.ascontiguousarray(reverse_states, dtype=np.uint32)
    pol = np.ascontiguousarray(policy) if policy is not None and len(policy) else None
    q = GoQuery(start, goal, orth_s, diag_s, bend_s,
                pol.ctypes.data_as(ctypes.c_void_p) if pol is not None else None,
                len(pol) if pol is not None else 0)
    total = ctypes.c_uint64(0)
    index = ctypes.c_uint64(0)
    code = L.go_validate_compact(nodes.ctypes.data_as(ctypes.c_void_p), ctypes.c_uint32(len(nodes)),
                                 GoCosts(*costs), ctypes.byref(q), ctypes.c_uint8(completion),
                                 ctypes.c_uint32(goal_state), _ptr(rev), ctypes.c_uint64(len(rev)),
                                 ctypes.byref(total), ctypes.byref(index))
    return PATH_CODES[code], total.value, index.value


def graph_predecessors(nodes, costs, start, labels, orth_s=0, diag_s=0, bend_s=0, policy=None):
    """Canonical predecessor of every state from exact labels."""
    L = lib()
    nodes = np.ascontiguousarray(nodes)
    labels = np.ascontiguousarray(labels, dtype=np.uint64)
    pol = np.ascontiguousarray(policy) if policy is not None and len(policy) else None
    q = GoQuery(start, 0, orth_s, diag_s, bend_s,
                pol.ctypes.data_as(ctypes.c_void_p) if pol is not None else None,
                len(pol) if pol is not None else 0)
    preds = np.empty(len(labels), dtype=np.uint32)
    L.go_predecessors(nodes.ctypes.data_as(ctypes.c_void_p), ctypes.c_uint32(len(nodes)),
                      GoCosts(*costs), ctypes.byref(q), labels.ctypes.data_as(U64P), _ptr(preds))
    return preds


def price_epoch_update(usage, history, capacity, epoch, init=100, inc=100, hinc=10):
    """Allocator epoch prices (checked). Returns (rc, present, history', total)."""
    L = lib()
    usage = np.ascontiguousarray(usage, dtype=np.uint64)
    hist = np.ascontiguousarray(history, dtype=np.uint64).copy()
    n = len(usage)
    present = np.zeros(n, np.uint64)
    total = np.zeros(n, np.uint64)
    rc = L.po_epoch_update(ctypes.c_uint32(n), usage.ctypes.data_as(U64P), ctypes.c_uint64(capacity),
                           ctypes.c_uint64(epoch), ctypes.c_uint64(init), ctypes.c_uint64(inc),
                           ctypes.c_uint64(hinc), present.ctypes.data_as(U64P),
                           hist.ctypes.data_as(U64P), total.ctypes.data_as(U64P))
    return rc, present, hist, total


def price_snapshot(usage, history, capacity, pass_index, init, inc, max_value):
    """CS-RR-v1 snapshot costs. Returns (rc, costs)."""
    L = lib()
    usage = np.ascontiguousarray(usage, dtype=np.uint64)
    hist = np.ascontiguousarray(history, dtype=np.uint64)
    cost = np.zeros(len(usage), np.uint64)
    rc = L.po_snapshot_costs(ctypes.c_uint32(len(usage)), usage.ctypes.data_as(U64P),
                             hist.ctypes.data_as(U64P), ctypes.c_uint64(capacity),
                             ctypes.c_uint32(pass_index), ctypes.c_uint64(init),
                             ctypes.c_uint64(inc), ctypes.c_uint64(max_value),
                             cost.ctypes.data_as(U64P))
    return rc, cost


def accumulate_cells(offsets, lengths, cells, cell_count):
    L = lib()
    offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
    lengths = np.ascontiguousarray(lengths, dtype=np.uint32)
    cells = np.ascontiguousarray(cells, dtype=np.uint32)
    usage = np.zeros(cell_count, np.uint32)
    L.po_accumulate_cells(ctypes.c_uint32(len(lengths)), offsets.ctypes.data_as(U64P), _ptr(lengths),
                          _ptr(cells), ctypes.c_uint32(cell_count), _ptr(usage))
    return usage
