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


def reference_root():
    """Root of the reference source tree, or None where it is absent.

    ``APGAR_REFERENCE`` names it; otherwise the tree that ``oracle/build_ref.sh``
    last compiled into ``oracle/_ref`` (recorded there in
    ``reference_root.txt``).  Tests that read reference sources or run the
    compiled reference skip with a message when this is None."""
    root = os.environ.get("APGAR_REFERENCE")
    if not root:
        stamp = os.path.join(_HERE, "_ref", "reference_root.txt")
        if os.path.exists(stamp):
            with open(stamp) as f:
                root = f.read().strip()
    if root and os.path.isdir(os.path.join(root, "src")):
        return root
    return None


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


def dijkstra_batch(lat, nets, threads=None, path_cap_per_net=None, cell_cost=None,
                   cell_cost_own=None, own=None):
    """Exact costs and canonical reverse paths of every net; ``cell_cost``
    (optional, uint32 [layers][height][width]) adds a per-cell entry price.
    Rip-up pricing: with ``own`` (one array of global cell ids per net, the
    net's previous route, or None) those cells enter at ``cell_cost_own``
    instead."""
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
    if own is None:
        L.lo_dijkstra_batch(ctypes.byref(ref.c), _net_ptr(nets), ctypes.c_uint32(count),
                            ctypes.c_int(threads), _ptr(costs), _ptr(lens), _ptr(offsets, U64P),
                            _ptr(paths), ctypes.c_uint64(total))
    else:
        assert cell_cost is not None and cell_cost_own is not None and len(own) == count
        cost_own = np.ascontiguousarray(cell_cost_own, dtype=np.uint32)
        assert cost_own.size == lat.layers * lat.height * lat.width
        sizes = np.array([0 if o is None else len(o) for o in own], dtype=np.uint64)
        own_offsets = np.zeros(count + 1, dtype=np.uint64)
        own_offsets[1:] = np.cumsum(sizes)
        parts = [np.asarray(o, dtype=np.uint32) for o in own if o is not None and len(o)]
        own_cells = np.ascontiguousarray(np.concatenate(parts) if parts else np.zeros(1, np.uint32))
        L.lo_dijkstra_batch_own(ctypes.byref(ref.c), _net_ptr(nets), ctypes.c_uint32(count),
                                ctypes.c_int(threads), _ptr(cost_own), _ptr(own_offsets, U64P),
                                _ptr(own_cells), _ptr(costs), _ptr(lens), _ptr(offsets, U64P),
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


def astar_path(lat, net_row, path_cap=1 << 22):
    """(cost, expanded states, forward A* path as global cell ids or None) of
    the restatement of RouteWithCpuAStar for one net."""
    L = lib()
    ref = LatticeRef(lat)
    net = np.ascontiguousarray(np.asarray(net_row).reshape(1))
    path = np.empty(path_cap, dtype=np.uint32)
    plen = ctypes.c_uint32(0)
    expanded = ctypes.c_uint64(0)
    L.lo_astar_path.restype = ctypes.c_uint32
    cost = L.lo_astar_path(ctypes.byref(ref.c), _net_ptr(net), ctypes.byref(expanded), _ptr(path),
                           ctypes.c_uint32(path_cap), ctypes.byref(plen))
    n = plen.value
    return cost, expanded.value, (path[:n].copy() if 0 < n != 0xFFFFFFFF else None)


def astar_batch(lat, nets, threads=None, counts=False):
    """A* restatement costs of every net; with ``counts`` also (expanded
    states, distinct expanded cells) per net as uint64 arrays."""
    L = lib()
    ref = LatticeRef(lat)
    nets = np.ascontiguousarray(nets)
    costs = np.empty(len(nets), dtype=np.uint32)
    if not counts:
        L.lo_astar_batch(ctypes.byref(ref.c), _net_ptr(nets), ctypes.c_uint32(len(nets)),
                         ctypes.c_int(threads or os.cpu_count() or 1), _ptr(costs))
        return costs
    states = np.empty(len(nets), dtype=np.uint64)
    cells = np.empty(len(nets), dtype=np.uint64)
    L.lo_astar_batch_ex(ctypes.byref(ref.c), _net_ptr(nets), ctypes.c_uint32(len(nets)),
                        ctypes.c_int(threads or os.cpu_count() or 1), _ptr(costs),
                        _ptr(states, U64P), _ptr(cells, U64P))
    return costs, states, cells


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


DISCONNECT_CODES = {0: "confirmed", 1: "reachable", 2: "unbounded", 3: "not_claimed"}
_U64_MAX = (1 << 64) - 1


def disconnect_verdict(nodes, costs, start, goal, orth_s=0, diag_s=0, bend_s=0, policy=None):
    """Confirmation of a DISCONNECTED claim for one query, restating what the
    CPU A* rerun of ConfirmDisconnectedWithCpuOracle decides
    (src/gpu/planar_router.cc:629-667; the search src/routing/cpu_astar.cc:
    413-512): its queue empties without the goal exactly when the goal node
    is unreachable over compiled legal edges whose canonical resource the
    policy does not ban.  Level-by-level breadth-first search, stopping after
    the level that reaches the goal.  An unreachable goal is "unbounded" when
    (8 * reachable nodes + 1) x the largest transition (StepCostUnderPolicy,
    src/routing/candidate_policy.cc:419-438) can leave the finite range
    (CheckedAddFiniteRouteCost, src/routing/planar_route.cc:154-161).

    Returns (code name, nodes reached)."""
    orth, diag, bend = int(costs[0]), int(costs[1]), int(costs[2])
    bans, penalty = set(), 0
    if policy is not None:
        for e in policy:
            adj = int(e["adjustment"])
            if adj == _U64_MAX:
                bans.add(int(e["physical_edge_index"]))
            else:
                penalty = max(penalty, adj)
    seen = {int(start)}
    level = [int(start)]
    found = int(start) == int(goal)
    while level and not found:
        nxt = []
        for u in level:
            legal = int(nodes[u]["legal_edges"])
            for d in range(8):
                if not (legal >> d) & 1:
                    continue
                v = int(nodes[u]["neighbors"][d])
                edge = u * 8 + d if d < 4 else v * 8 + d - 4
                if edge in bans or v in seen:
                    continue
                seen.add(v)
                nxt.append(v)
                found = found or v == int(goal)
        level = nxt
    if found:
        return "reachable", len(seen)
    t = max(orth + orth_s, diag + diag_s) + bend + bend_s + penalty
    bounded = (8 * len(seen) + 1) * t <= _U64_MAX - 1
    return ("confirmed" if bounded else "unbounded"), len(seen)


LATTICE_PATH_CODES = {0: "ok", 1: "bounds", 2: "endpoint", 5: "edge", 7: "not_reached", 8: "cost"}


def validate_lattice_path(lat, net, result, path):
    """Structural validation of one lattice route result, restating the checks
    a host applies to an untrusted GPU path (src/gpu/planar_router.cc:969-1067)
    for lattice paths: bounds, endpoints (start first, goal last in forward
    order), every cell inside the lattice and the net's window, every step a
    legal move by the lattice rule (orthogonal: both cells free; diagonal: both
    cells and both side cells free; via: same column, adjacent layer, both
    cells free, via bit set), and the move costs summing to the reported cost.
    ``path`` is the reverse path of global cell ids (goal first).  Returns
    (code name, failing forward index, cost sum)."""
    if int(result["completion"]) != 0:
        return "not_reached", 0, 0
    path = [int(c) for c in path]
    if not path:
        return "bounds", 0, 0
    free = ~lat.blocked_dense()
    via_ok = None if lat.via_ok is None else unpack_bits_dense(lat.via_ok, lat.width)
    L, H, W = lat.layers, lat.height, lat.width

    def cell(c):
        return c // (W * H), c % W, (c // W) % H

    fwd = path[::-1]
    start = (int(net["start_layer"]) * H + int(net["start_y"])) * W + int(net["start_x"])
    goal = (int(net["goal_layer"]) * H + int(net["goal_y"])) * W + int(net["goal_x"])
    if fwd[0] != start:
        return "endpoint", 0, 0
    if fwd[-1] != goal:
        return "endpoint", len(fwd) - 1, 0
    x0, y0 = int(net["win_x0"]), int(net["win_y0"])
    x1, y1 = x0 + int(net["win_w"]), y0 + int(net["win_h"])
    total = 0
    for f, c in enumerate(fwd):
        if c >= L * H * W:
            return "bounds", f, 0
        l, x, y = cell(c)
        if not (x0 <= x < x1 and y0 <= y < y1):
            return "bounds", f, 0
        if f == 0:
            continue
        pl, px, py = cell(fwd[f - 1])
        dx, dy, dl = x - px, y - py, l - pl
        cost = 0
        if dl != 0:
            if dx == 0 and dy == 0 and abs(dl) == 1 and free[pl, py, px] and free[l, y, x] and \
                    (via_ok is None or via_ok[min(l, pl), y, x]):
                cost = lat.via
        elif max(abs(dx), abs(dy)) == 1 and free[pl, py, px] and free[l, y, x]:
            if dx != 0 and dy != 0:
                if free[l, py, x] and free[l, y, px]:
                    cost = lat.diag
            else:
                cost = lat.orth
        if cost == 0:
            return "edge", f, 0
        total += cost
    if total != int(result["cost"]):
        return "cost", 0, total
    return "ok", 0, total


def unpack_bits_dense(words, width):
    """uint32 [..., width // 32] -> bool [..., width] (bit x % 32 of word x // 32)."""
    shifts = np.arange(32, dtype=np.uint32)
    bits = (np.asarray(words)[..., None] >> shifts) & np.uint32(1)
    return bits.reshape(np.asarray(words).shape[:-1] + (width,)).astype(bool)


PRED_CODES = {0: "ok", 1: "start", 2: "no_heading", 3: "unreachable", 4: "bounds",
              5: "self_reference", 6: "edge", 7: "sentinel", 8: "infinite", 9: "banned", 10: "cost"}


def validate_predecessors(nodes, costs, start, labels, preds, orth_s=0, diag_s=0, bend_s=0,
                          policy=None, partial=False):
    """The checks of ValidateAllPredecessors (src/gpu/planar_router.cc:492-611)
    over one query's heading-state labels and predecessors, in state order;
    returns (code name, failing state) of the first failure, ("ok", 0) if
    none."""
    U64 = (1 << 64) - 1
    INV = 0xFFFFFFFF
    orth, diag, bend = (int(c) for c in costs)
    n = len(nodes)
    S = 9 * n
    labels = [int(x) for x in labels]
    preds = [int(x) for x in preds]
    adj = {}
    if policy is not None:
        for e in policy:
            adj[int(e["physical_edge_index"])] = int(e["adjustment"])
    if start >= n:
        return "start", 9 * start + 8
    start_state = 9 * start + 8
    if labels[start_state] != 0 or preds[start_state] != INV:
        return "start", start_state
    dxs = (1, 1, 0, -1, -1, -1, 0, 1)
    dys = (0, 1, 1, 1, 0, -1, -1, -1)
    for state in range(S):
        if state == start_state:
            continue
        label, pred, inc = labels[state], preds[state], state % 9
        if inc == 8:
            if label != U64 or pred != INV:
                return "no_heading", state
            continue
        if label == U64:
            if pred != INV:
                return "unreachable", state
            continue
        if pred == INV and partial:
            continue
        if pred >= S:
            return "bounds", state
        if pred == state:
            return "self_reference", state
        node, pnode = state // 9, pred // 9
        a, b = nodes[pnode], nodes[node]
        if (int(a["layer"]) != int(b["layer"]) or int(b["lattice_x"]) - int(a["lattice_x"]) != dxs[inc]
                or int(b["lattice_y"]) - int(a["lattice_y"]) != dys[inc]
                or int(a["neighbors"][inc]) != node or not (int(a["legal_edges"]) >> inc) & 1):
            return "edge", state
        ph = pred % 9
        if ph == 8 and pred != start_state:
            return "sentinel", state
        if labels[pred] == U64:
            return "infinite", state
        edge = pnode * 8 + inc if inc < 4 else node * 8 + inc - 4
        pen = adj.get(edge, 0)
        if pen == U64:
            return "banned", state
        t = (diag + diag_s) if inc & 1 else (orth + orth_s)
        if ph != 8 and ph != inc:
            t += bend + bend_s
        t += pen
        expected = labels[pred] + t if t < U64 else None
        if expected is None or expected > U64 - 1 or (expected > label if partial else expected != label):
            return "cost", state
    return "ok", 0


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


# ---------------------------------------------------------------------------
# Corridor certificate (no reference counterpart): the exact restatement of
# the frontier corridor mode's decision.  A net is searched in its corridor
# only (cells outside it priced out of reach); every legal planar move from a
# reached corridor cell u to a window cell v outside the corridor is an exit
# with key d(u) + move + h(v), h the octile-plus-via bound.  The corridor
# result is certified when its cost is strictly below every exit key.
CORRIDOR_NONE, CORRIDOR_CERTIFIED, CORRIDOR_FALLBACK_EXIT, CORRIDOR_FALLBACK_UNREACHED = 0, 1, 2, 3
_STEPS = ((1, 0), (1, 1), (0, 1), (-1, 1), (-1, 0), (-1, -1), (0, -1), (1, -1))


def _window_free(lat, net):
    x0, y0 = int(net["win_x0"]), int(net["win_y0"])
    w, h = int(net["win_w"]), int(net["win_h"])
    words = np.ascontiguousarray(lat.blocked, dtype=np.uint32).reshape(lat.layers, lat.height, -1)
    bits = np.unpackbits(words.view(np.uint8).reshape(lat.layers, lat.height, -1), axis=2,
                         bitorder="little")
    return bits[:, y0:y0 + h, x0:x0 + w] == 0


def corridor_certificate(lat, net, mask, cell_cost=None):
    """(status, corridor cost or None, least exit key or None) of one net
    for a bool [64][64] coarse corridor (coarse scale as in
    apgar_b200.corridor.coarse_shift).  ``cell_cost`` (optional, uint32
    [layers][height][width]): per-cell entry prices, paid inside the
    corridor; an exit's key leaves out its outside cell's price, a lower bound
    because prices are non-negative."""
    net = np.ascontiguousarray(np.asarray(net).reshape(1))
    n0 = net[0]
    w, h = int(n0["win_w"]), int(n0["win_h"])
    x0, y0 = int(n0["win_x0"]), int(n0["win_y0"])
    span = max(w, h)
    s = 2
    while ((span - 1) >> s) >= 63:
        s += 1
    inside = np.asarray(mask, dtype=bool)[(np.arange(h) >> s)[:, None], (np.arange(w) >> s)[None, :]]
    sx, sy = int(n0["start_x"]) - x0, int(n0["start_y"]) - y0
    gx, gy = int(n0["goal_x"]) - x0, int(n0["goal_y"]) - y0
    sl, gl = int(n0["start_layer"]), int(n0["goal_layer"])
    if not np.asarray(mask).any():
        return CORRIDOR_NONE, None, None  # no corridor proposed: the window is searched
    if not (inside[sy, sx] and inside[gy, gx]):
        return CORRIDOR_FALLBACK_UNREACHED, None, None
    free = _window_free(lat, n0)
    if not (free[sl, sy, sx] and free[gl, gy, gx]):
        return CORRIDOR_CERTIFIED, None, None  # disconnected either way
    big = 1 << 30
    if cell_cost is None:
        price = np.zeros((lat.layers, lat.height, lat.width), dtype=np.uint32)
    else:
        price = np.array(cell_cost, dtype=np.uint32).reshape(lat.layers, lat.height, lat.width)
    price[:, y0:y0 + h, x0:x0 + w][:, ~inside] = big
    cost, _, dist = dijkstra(lat, net, full=True, want_dist=True, cell_cost=price.reshape(-1))
    if cost >= big:
        return CORRIDOR_FALLBACK_UNREACHED, None, None
    d = dist.reshape(lat.layers, h, w).astype(np.uint64)
    reached = inside[None] & (d < big)
    layer_term = (np.abs(np.arange(lat.layers) - gl) * lat.via).astype(np.uint64)[:, None, None]
    best = None
    for dx, dy in _STEPS:
        # u at (y, x) and v at (y + dy, x + dx), both inside the window
        uy = slice(max(0, -dy), h - max(0, dy))
        ux = slice(max(0, -dx), w - max(0, dx))
        vy = slice(uy.start + dy, uy.stop + dy)
        vx = slice(ux.start + dx, ux.stop + dx)
        legal = free[:, uy, ux] & free[:, vy, vx]
        if dx != 0 and dy != 0:
            legal &= free[:, uy, vx] & free[:, vy, ux]
        exits = reached[:, uy, ux] & ~inside[None, vy, vx] & legal
        if not exits.any():
            continue
        move = lat.diag if (dx != 0 and dy != 0) else lat.orth
        adx = np.abs(np.arange(w)[vx] - gx)[None, :]
        ady = np.abs(np.arange(h)[vy] - gy)[:, None]
        lo, hi = np.minimum(adx, ady), np.maximum(adx, ady)
        if lat.diag >= lat.orth:
            planar = lo * min(lat.diag, 2 * lat.orth) + (hi - lo) * lat.orth
        else:
            planar = hi * lat.diag
        key = d[:, uy, ux] + np.uint64(move) + planar.astype(np.uint64)[None] + layer_term
        m = int(key[exits].min())
        best = m if best is None else min(best, m)
    status = CORRIDOR_CERTIFIED if best is None or cost < best else CORRIDOR_FALLBACK_EXIT
    return status, int(cost), best


# ---------------------------------------------------------------------------
# Route reconstruction: exact points and coalesced segments.
SEGMENT_DTYPE = np.dtype([("layer0", "<u4"), ("layer1", "<u4"), ("x0", "<i8"), ("y0", "<i8"),
                          ("x1", "<i8"), ("y1", "<i8")])
MAX_ABS_DB_COORD = 1_000_000_000_000  # board_ir::kMaxAbsDbCoord (include/apgar/board_ir/board.h:20)


def exact_points(origin_x, origin_y, step, lattice_x, lattice_y):
    """origin + index * step per axis (LatticeIndexToExactPoint,
    src/geometry_compiler/compiled_board.cc:219-238); None if a point leaves
    the exact coordinate envelope."""
    xs = [int(origin_x) + int(x) * int(step) for x in lattice_x]
    ys = [int(origin_y) + int(y) * int(step) for y in lattice_y]
    if any(abs(v) > MAX_ABS_DB_COORD for v in xs + ys):
        return None
    return np.array(xs, np.int64), np.array(ys, np.int64)


def coalesce_segments(xs, ys, layers):
    """Segments of a forward point sequence: a new segment starts wherever the
    step (dx, dy, dlayer) changes (routing::CoalesceSegments,
    src/routing/planar_route.cc:188-215, with the layer step added for vias;
    on one layer the two agree).  Fewer than two points give no segment."""
    n = len(xs)
    out = []
    if n < 2:
        return np.zeros(0, SEGMENT_DTYPE)
    start = 0
    prev = (xs[1] - xs[0], ys[1] - ys[0], int(layers[1]) - int(layers[0]))
    for i in range(2, n):
        step = (xs[i] - xs[i - 1], ys[i] - ys[i - 1], int(layers[i]) - int(layers[i - 1]))
        if step != prev:
            out.append((layers[start], layers[i - 1], xs[start], ys[start], xs[i - 1], ys[i - 1]))
            start = i - 1
            prev = step
    out.append((layers[start], layers[n - 1], xs[start], ys[start], xs[n - 1], ys[n - 1]))
    return np.array(out, SEGMENT_DTYPE)


# ---------------------------------------------------------------------------
# Exact edge legality of the geometry compile (pure-Python integers; small
# cases only).  A one-step lattice move is legal when the swept trace of
# width w keeps clearance c from every obstacle box on its layer that the
# routed net does not own (geometry::SweptTraceClearanceAtLeast,
# src/geometry/exact.cc:165-216 and :325-360; CompileBoard's edge loop,
# src/geometry_compiler/compiled_board.cc:427-476).  Coordinates are doubled
# so that the required distance w + 2c stays integral.
CLEARANCE_OK, CLEARANCE_OUT_OF_RANGE, CLEARANCE_BAD_BOX, CLEARANCE_BAD_DISTANCE = 0, 1, 2, 3


def _orient(a, b, c):
    return (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0])


def _on_segment(a, b, p):
    return (_orient(a, b, p) == 0 and min(a[0], b[0]) <= p[0] <= max(a[0], b[0])
            and min(a[1], b[1]) <= p[1] <= max(a[1], b[1]))


def _sign(v):
    return (v > 0) - (v < 0)


def _segments_touch(a, b, c, d):
    o1, o2 = _orient(a, b, c), _orient(a, b, d)
    o3, o4 = _orient(c, d, a), _orient(c, d, b)
    if _sign(o1) * _sign(o2) < 0 and _sign(o3) * _sign(o4) < 0:
        return True
    return ((o1 == 0 and _on_segment(a, b, c)) or (o2 == 0 and _on_segment(a, b, d))
            or (o3 == 0 and _on_segment(c, d, a)) or (o4 == 0 and _on_segment(c, d, b)))


def _point_segment_at_least(p, a, b, req):
    vx, vy = b[0] - a[0], b[1] - a[1]
    wx, wy = p[0] - a[0], p[1] - a[1]
    len2 = vx * vx + vy * vy
    if len2 == 0:
        return wx * wx + wy * wy >= req * req
    proj = wx * vx + wy * vy
    if proj <= 0:
        return wx * wx + wy * wy >= req * req
    if proj >= len2:
        ex, ey = p[0] - b[0], p[1] - b[1]
        return ex * ex + ey * ey >= req * req
    cross = vx * wy - vy * wx
    return cross * cross >= req * req * len2


def swept_clearance(start, end, box_min, box_max, width, clearance):
    """(error code, satisfied) of a centreline segment against one box."""
    lim = MAX_ABS_DB_COORD
    if any(abs(int(v)) > lim for v in (*start, *end, *box_min, *box_max)):
        return CLEARANCE_OUT_OF_RANGE, False
    if box_min[0] > box_max[0] or box_min[1] > box_max[1]:
        return CLEARANCE_BAD_BOX, False
    if width <= 0 or width > lim or clearance < 0 or clearance > lim:
        return CLEARANCE_BAD_DISTANCE, False
    req = int(width) + 2 * int(clearance)
    s = (2 * int(start[0]), 2 * int(start[1]))
    e = (2 * int(end[0]), 2 * int(end[1]))
    lo = (2 * int(box_min[0]), 2 * int(box_min[1]))
    hi = (2 * int(box_max[0]), 2 * int(box_max[1]))
    if (max(s[0], e[0]) <= lo[0] - req or min(s[0], e[0]) >= hi[0] + req
            or max(s[1], e[1]) <= lo[1] - req or min(s[1], e[1]) >= hi[1] + req):
        return CLEARANCE_OK, True
    inside = lambda p: lo[0] <= p[0] <= hi[0] and lo[1] <= p[1] <= hi[1]  # noqa: E731
    if inside(s) or inside(e):
        return CLEARANCE_OK, False
    corners = [lo, (hi[0], lo[1]), hi, (lo[0], hi[1])]
    for k in range(4):
        c, d = corners[k], corners[(k + 1) % 4]
        if _segments_touch(s, e, c, d):
            return CLEARANCE_OK, False
        if not (_point_segment_at_least(s, c, d, req) and _point_segment_at_least(e, c, d, req)
                and _point_segment_at_least(c, s, e, req) and _point_segment_at_least(d, s, e, req)):
            return CLEARANCE_OK, False
    return CLEARANCE_OK, True


_DIR = ((1, 0), (1, 1), (0, 1), (-1, 1), (-1, 0), (-1, -1), (0, -1), (1, -1))
_HEADING = (1, 4, 2, 4, 1, 4, 2, 4)  # horizontal 1, vertical 2, diagonal 4


def compile_legal_edges(lattice_x, lattice_y, layers, origin, step, heading_mask, width, clearance,
                        obstacles):
    """8-bit legal-edge masks of the given lattice nodes: a direction is legal
    when its neighbour is a given node on the same layer, the heading is in the
    compiler's mask, and the move clears every obstacle (minx, miny, maxx, maxy,
    layer, owned_by_net) on the layer that the net does not own."""
    index = {(int(l), int(x), int(y)): i for i, (x, y, l) in enumerate(zip(lattice_x, lattice_y, layers))}
    out = np.zeros(len(lattice_x), np.uint8)
    for i, (x, y, l) in enumerate(zip(lattice_x, lattice_y, layers)):
        x, y, l = int(x), int(y), int(l)
        for d, (dx, dy) in enumerate(_DIR):
            if (l, x + dx, y + dy) not in index or not (heading_mask & _HEADING[d]):
                continue
            a = (origin[0] + x * step, origin[1] + y * step)
            b = (origin[0] + (x + dx) * step, origin[1] + (y + dy) * step)
            ok = True
            for (minx, miny, maxx, maxy, ol, owned) in obstacles:
                if int(ol) != l or owned:
                    continue
                err, sat = swept_clearance(a, b, (minx, miny), (maxx, maxy), width, clearance)
                if err != CLEARANCE_OK or not sat:
                    ok = False
                    break
            if ok:
                out[i] |= 1 << d
    return out
