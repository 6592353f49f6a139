"""Python mirror of the drop-in seam (IPlanarRouteBackend over the C ABI).

Mirrors the reference backend interface (include/apgar/gpu/planar_router.h:
543-560): ``View.upload`` = UploadCompiledView, ``View.execute_batch`` /
``PendingBatch.readback`` = ExecuteCandidateBatch / ReadbackCandidateBatch,
``View.execute_route`` / ``PendingRoute.readback`` = ExecuteRoute /
ReadbackRoute.  Records are numpy structured arrays with the V1 layouts;
failures raise ``apgar_b200.BackendError`` whose ``code`` mirrors
BackendErrorCode.  All searching happens in the CUDA library.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import BackendError, _check, lib  # noqa: F401

GENERATOR_FRONTIER = 0
GENERATOR_SWEEP = 1
GENERATOR_PERSISTENT = 2
GENERATOR_PERSISTENT_WORKSPACE = 3

HEADER_DTYPE = np.dtype([
    ("schema_version", "<u4"), ("compiler_version", "<u4"),
    ("source_board_content_hash", "<u8"), ("compiler_profile_fingerprint", "<u8"),
    ("rule_bucket_identity", "<u8"), ("device_view_fingerprint", "<u8"),
    ("represented_nodes", "<u8"), ("represented_states", "<u8"),
    ("estimated_persistent_device_bytes", "<u8"),
    ("lattice_origin_x", "<i8"), ("lattice_origin_y", "<i8"), ("lattice_step", "<i8"),
    ("orthogonal_step", "<u4"), ("diagonal_step", "<u4"), ("bend", "<u4"),
    ("heading_mask", "u1"), ("reserved", "u1", (7,)), ("padding", "u1", (4,)),
])
QUERY_DTYPE = np.dtype([
    ("schema_version", "<u4"), ("input_ordinal", "<u4"), ("batch_id", "<u8"), ("query_id", "<u8"),
    ("workspace_owner", "<u8"), ("policy_identity", "<u8"), ("routing_profile_fingerprint", "<u8"),
    ("start_node", "<u4"), ("goal_node", "<u4"), ("policy_offset", "<u4"), ("policy_count", "<u4"),
    ("workspace_offset", "<u8"), ("workspace_state_count", "<u8"), ("frontier_state_capacity", "<u8"),
    ("orthogonal_step_surcharge", "<u8"), ("diagonal_step_surcharge", "<u8"), ("bend_surcharge", "<u8"),
    ("maximum_rounds", "<u4"), ("generator", "u1"), ("reserved", "u1", (3,)),
])
RESULT_DTYPE = np.dtype([
    ("schema_version", "<u4"), ("compiler_version", "<u4"), ("input_ordinal", "<u4"),
    ("start_node", "<u4"), ("goal_node", "<u4"), ("goal_state", "<u4"), ("rounds", "<u4"),
    ("generator", "u1"), ("completion", "u1"), ("reserved", "u1", (2,)),
    ("batch_id", "<u8"), ("query_id", "<u8"), ("workspace_owner", "<u8"), ("policy_identity", "<u8"),
    ("routing_profile_fingerprint", "<u8"), ("source_board_content_hash", "<u8"),
    ("compiler_profile_fingerprint", "<u8"), ("rule_bucket_identity", "<u8"),
    ("device_view_fingerprint", "<u8"), ("examined_work", "<u8"), ("heading_turn_relaxations", "<u8"),
])
COMPACT_DTYPE = np.dtype([("schema_version", "<u4"), ("state_count", "<u4"), ("query_id", "<u8"),
                          ("workspace_owner", "<u8"), ("state_offset", "<u8")])
POLICY_EDGE_DTYPE = np.dtype([("physical_edge_index", "<u4"), ("reserved", "<u4"), ("adjustment", "<u8")])
VERDICT_DTYPE = np.dtype([("code", "<u4"), ("reserved", "<u4"), ("failing_index", "<u8"),
                          ("total_cost", "<u8")])
PATH_CODES = {0: "ok", 1: "bounds", 2: "endpoint", 3: "cycle", 4: "heading", 5: "edge",
              6: "banned", 7: "not_reached"}
PRED_CODES = {0: "ok", 1: "start", 2: "no_heading", 3: "unreachable", 4: "bounds",
              5: "self_reference", 6: "edge", 7: "sentinel", 8: "infinite", 9: "banned", 10: "cost"}
DISCONNECT_VERDICT_DTYPE = np.dtype([("code", "<u4"), ("reserved", "<u4"), ("reachable_nodes", "<u8")])
DISCONNECT_CODES = {0: "confirmed", 1: "reachable", 2: "unbounded", 3: "not_claimed"}
ROUTE_HEADER_DTYPE = np.dtype([
    ("schema_version", "<u4"), ("compiler_version", "<u4"), ("start_node", "<u4"), ("goal_node", "<u4"),
    ("source_board_content_hash", "<u8"), ("compiler_profile_fingerprint", "<u8"),
    ("routing_profile_fingerprint", "<u8"), ("rule_bucket_identity", "<u8"),
    ("device_view_fingerprint", "<u8"), ("generator", "u1"), ("reserved", "u1", (7,)),
])
for _d, _n in ((HEADER_DTYPE, 112), (QUERY_DTYPE, 120), (RESULT_DTYPE, 120), (COMPACT_DTYPE, 32),
               (POLICY_EDGE_DTYPE, 16), (ROUTE_HEADER_DTYPE, 64)):
    assert _d.itemsize == _n


class BatchRequest(ctypes.Structure):
    _fields_ = [
        ("schema_version", ctypes.c_uint32), ("generator", ctypes.c_uint8),
        ("reserved", ctypes.c_uint8 * 3), ("batch_id", ctypes.c_uint64),
        ("maximum_rounds", ctypes.c_uint32), ("padding", ctypes.c_uint32),
        ("maximum_workspace_states_per_query", ctypes.c_uint64),
        ("maximum_frontier_states_per_query", ctypes.c_uint64),
        ("maximum_device_bytes", ctypes.c_uint64), ("maximum_host_bytes", ctypes.c_uint64),
    ]


class BatchTelemetry(ctypes.Structure):
    _fields_ = [
        ("persistent_device_bytes", ctypes.c_uint64), ("batch_device_bytes", ctypes.c_uint64),
        ("workspace_capacity_device_bytes", ctypes.c_uint64), ("peak_device_bytes", ctypes.c_uint64),
        ("device_to_host_readback_bytes", ctypes.c_uint64), ("kernel_launch_count", ctypes.c_uint64),
        ("blocking_status_readback_count", ctypes.c_uint64), ("dispatched_rounds", ctypes.c_uint32),
        ("finalization_launch_count", ctypes.c_uint32), ("kernel_milliseconds", ctypes.c_double),
    ]


def _vp(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _as(a, dtype):
    return np.ascontiguousarray(np.asarray(a).view(dtype) if a.dtype != dtype else a)


def make_queries(view_nodes: int, entries, batch_id: int = 7, generator: int = GENERATOR_SWEEP,
                 maximum_rounds: int = 100_000):
    """Builds canonical batch query records and the packed policy-edge array.

    ``entries``: iterable of dicts with start_node, goal_node and optional
    orthogonal/diagonal/bend surcharges, policy (POLICY_EDGE_DTYPE array),
    policy_identity."""
    entries = list(entries)
    S = 9 * view_nodes
    q = np.zeros(len(entries), dtype=QUERY_DTYPE)
    edges = []
    offset = 0
    for i, e in enumerate(entries):
        pol = e.get("policy")
        count = 0 if pol is None else len(pol)
        q[i] = (1, i, batch_id, i + 1, i + 1, e.get("policy_identity", 0), e.get("routing_profile_fingerprint", 0),
                e["start_node"], e["goal_node"], offset, count, i * S, S,
                S if generator in (GENERATOR_FRONTIER, GENERATOR_PERSISTENT_WORKSPACE) else 0,
                e.get("orthogonal_step_surcharge", 0), e.get("diagonal_step_surcharge", 0),
                e.get("bend_surcharge", 0), maximum_rounds, generator, (0, 0, 0))
        if count:
            edges.append(np.asarray(pol).astype(POLICY_EDGE_DTYPE))
        offset += count
    edge_arr = np.concatenate(edges) if edges else np.zeros(0, dtype=POLICY_EDGE_DTYPE)
    return q, np.ascontiguousarray(edge_arr)


# apgar_b200_segment (40 bytes)
SEGMENT_DTYPE = np.dtype([("layer0", "<u4"), ("layer1", "<u4"), ("x0", "<i8"), ("y0", "<i8"),
                          ("x1", "<i8"), ("y1", "<i8")])
SEGMENT_FAILURE = 0xFFFFFFFF


class View:
    """UploadCompiledView: the reference flattened device view on this GPU."""

    def __init__(self, header, layers, nodes, runs, run_nodes):
        self.header = np.ascontiguousarray(header).view(np.uint8)
        self.layers = np.ascontiguousarray(layers)
        self.nodes = np.ascontiguousarray(nodes)
        self.runs = np.ascontiguousarray(runs)
        self.run_nodes = np.ascontiguousarray(run_nodes, dtype=np.uint32)
        handle = ctypes.c_void_p()
        _check(lib().apgar_b200_view_upload(
            _vp(self.header), _vp(self.layers), ctypes.c_uint64(len(self.layers)),
            _vp(self.nodes), ctypes.c_uint64(len(self.nodes)), _vp(self.runs),
            ctypes.c_uint64(len(self.runs)), _vp(self.run_nodes), ctypes.c_uint64(len(self.run_nodes)),
            ctypes.byref(handle)))
        self.handle = handle
        self.node_count = len(self.nodes)

    def close(self):
        if self.handle:
            lib().apgar_b200_view_release(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def execute_batch(self, queries, policy_edges, generator=GENERATOR_SWEEP, batch_id=7,
                      maximum_rounds=100_000, maximum_device_bytes=(1 << 64) - 1, cancel=None):
        req = BatchRequest()
        req.schema_version = 1
        req.generator = generator
        req.batch_id = batch_id
        req.maximum_rounds = maximum_rounds
        req.maximum_workspace_states_per_query = (1 << 64) - 1
        req.maximum_frontier_states_per_query = (1 << 64) - 1
        req.maximum_device_bytes = maximum_device_bytes
        req.maximum_host_bytes = (1 << 64) - 1
        queries = np.ascontiguousarray(queries)
        policy_edges = np.ascontiguousarray(policy_edges)
        handle = ctypes.c_void_p()
        _check(lib().apgar_b200_execute_batch(
            self.handle, ctypes.byref(req), _vp(queries), ctypes.c_uint32(len(queries)),
            _vp(policy_edges) if len(policy_edges) else None, ctypes.c_uint64(len(policy_edges)),
            _vp(cancel), ctypes.byref(handle)))
        return PendingBatch(handle, len(queries), 9 * self.node_count)

    def validate_compact_paths(self, queries, policy_edges, results, compact, states):
        """Device-side structural validation of read-back compact paths; one
        (code, failing forward index, total cost) record per query."""
        queries = np.ascontiguousarray(queries)
        policy_edges = np.ascontiguousarray(policy_edges)
        results = np.ascontiguousarray(results)
        compact = np.ascontiguousarray(compact)
        states = np.ascontiguousarray(states, dtype=np.uint32)
        out = np.zeros(len(queries), dtype=VERDICT_DTYPE)
        _check(lib().apgar_b200_validate_compact_paths(
            self.handle, _vp(queries), ctypes.c_uint32(len(queries)),
            _vp(policy_edges) if len(policy_edges) else None, ctypes.c_uint64(len(policy_edges)),
            _vp(results), _vp(compact), _vp(states) if len(states) else None,
            ctypes.c_uint64(len(states)), _vp(out)))
        return out

    def validate_predecessors(self, queries, policy_edges, labels, predecessors, partial=None):
        """Device validation of full-workspace results (labels [Q][9N] uint64,
        predecessors [Q][9N] uint32): one (code, reserved, first failing
        state, 0) record per query, codes in PRED_CODES."""
        queries = np.ascontiguousarray(queries)
        policy_edges = np.ascontiguousarray(policy_edges)
        labels = np.ascontiguousarray(labels, dtype=np.uint64)
        predecessors = np.ascontiguousarray(predecessors, dtype=np.uint32)
        part = None if partial is None else np.ascontiguousarray(partial, dtype=np.uint8)
        out = np.zeros(len(queries), dtype=VERDICT_DTYPE)
        _check(lib().apgar_b200_validate_predecessors(
            self.handle, _vp(queries), ctypes.c_uint32(len(queries)),
            _vp(policy_edges) if len(policy_edges) else None, ctypes.c_uint64(len(policy_edges)),
            _vp(part) if part is not None else None, _vp(labels), _vp(predecessors), _vp(out)))
        return out

    def confirm_disconnected(self, queries, policy_edges, results):
        """Device confirmation of every DISCONNECTED result: one (code,
        reachable nodes) record per query (codes in DISCONNECT_CODES)."""
        queries = np.ascontiguousarray(queries)
        policy_edges = np.ascontiguousarray(policy_edges)
        results = np.ascontiguousarray(results)
        out = np.zeros(len(queries), dtype=DISCONNECT_VERDICT_DTYPE)
        _check(lib().apgar_b200_confirm_disconnected(
            self.handle, _vp(queries), ctypes.c_uint32(len(queries)),
            _vp(policy_edges) if len(policy_edges) else None, ctypes.c_uint64(len(policy_edges)),
            _vp(results), _vp(out)))
        return out

    def path_segments(self, compact, states):
        """Exact-coordinate segments of read-back compact paths (GPU):
        (segments record array indexed like the states, per-path counts;
        path i's segments are segments[compact[i].state_offset:][:count])."""
        compact = np.ascontiguousarray(compact)
        states = np.ascontiguousarray(states, dtype=np.uint32)
        segments = np.zeros(max(len(states), 1), dtype=SEGMENT_DTYPE)
        counts = np.zeros(max(len(compact), 1), dtype=np.uint32)
        _check(lib().apgar_b200_path_segments(
            self.handle, _vp(compact), ctypes.c_uint32(len(compact)),
            _vp(states) if len(states) else None, ctypes.c_uint64(len(states)), _vp(segments),
            ctypes.c_uint64(len(segments)), _vp(counts)))
        return segments, counts[: len(compact)]

    def execute_route(self, start_node, goal_node, generator=GENERATOR_SWEEP, maximum_rounds=100_000,
                      routing_profile_fingerprint=0, maximum_device_bytes=(1 << 64) - 1):
        handle = ctypes.c_void_p()
        _check(lib().apgar_b200_execute_route(
            self.handle, ctypes.c_uint8(generator), ctypes.c_uint32(start_node),
            ctypes.c_uint32(goal_node), ctypes.c_uint64(routing_profile_fingerprint),
            ctypes.c_uint32(maximum_rounds), ctypes.c_uint64(maximum_device_bytes), None,
            ctypes.byref(handle)))
        return PendingRoute(handle, 9 * self.node_count)


class PendingBatch:
    def __init__(self, handle, query_count, states):
        self.handle = handle
        self.query_count = query_count
        self.states = states

    def readback(self):
        """Compact form: (results, compact path headers, packed states, telemetry)."""
        results = np.zeros(self.query_count, dtype=RESULT_DTYPE)
        compact = np.zeros(self.query_count, dtype=COMPACT_DTYPE)
        cap = self.query_count * self.states
        states = np.zeros(cap, dtype=np.uint32)
        total = ctypes.c_uint64(0)
        tel = BatchTelemetry()
        _check(lib().apgar_b200_readback_batch(self.handle, _vp(results), _vp(compact), _vp(states),
                                               ctypes.c_uint64(cap), ctypes.byref(total),
                                               ctypes.byref(tel)))
        return results, compact, states[: total.value], tel

    def readback_workspace(self):
        """Full-workspace form: (labels, predecessors, state owners, predecessor owners)."""
        total = self.query_count * self.states
        labels = np.zeros(total, dtype=np.uint64)
        preds = np.zeros(total, dtype=np.uint32)
        owners = np.zeros(total, dtype=np.uint64)
        powners = np.zeros(total, dtype=np.uint64)
        _check(lib().apgar_b200_readback_batch_workspace(self.handle, _vp(labels), _vp(preds),
                                                         _vp(owners), _vp(powners)))
        return labels, preds, owners, powners

    def close(self):
        if self.handle:
            lib().apgar_b200_release_batch(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PendingRoute:
    def __init__(self, handle, states):
        self.handle = handle
        self.states = states

    def readback(self):
        header = np.zeros(1, dtype=ROUTE_HEADER_DTYPE)
        completion = ctypes.c_uint8(0)
        goal_state = ctypes.c_uint32(0)
        labels = np.zeros(self.states, dtype=np.uint64)
        preds = np.zeros(self.states, dtype=np.uint32)
        tel = BatchTelemetry()
        _check(lib().apgar_b200_readback_route(self.handle, _vp(header), ctypes.byref(completion),
                                               ctypes.byref(goal_state), _vp(labels), _vp(preds),
                                               ctypes.byref(tel)))
        return header[0], completion.value, goal_state.value, labels, preds, tel

    def close(self):
        if self.handle:
            lib().apgar_b200_release_route(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
