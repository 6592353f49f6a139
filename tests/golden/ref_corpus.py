"""Reader for tests/golden/ref_corpus/*.bin (written by oracle/ref_fixtures.cc).

Layout (little endian): u64 magic "AGRFTIX1"; DeviceCompiledHeaderV1 (112 B);
then u64-counted arrays of DeviceLayerRangeV1 (48 B), DeviceNodeV1 (56 B),
DeviceRunV1 (12 B) and run-node u32; then u64 query count and per query:
u32 start node, u32 goal node, u64 orthogonal / diagonal / bend surcharges,
u64 policy identity, u32 CPU status (0 reached, 1 disconnected, 2 failed),
u32 pad, u64 CPU A* cost, u64-counted DeviceCandidatePolicyEdgeV1 (16 B).
"""

from __future__ import annotations

import dataclasses
import glob
import json
import os

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_corpus")

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
LAYER_DTYPE = np.dtype([("layer", "<u4"), ("node_offset", "<u4"), ("node_count", "<u4"),
                        ("padding", "<u4"), ("minimum_lattice_x", "<i8"), ("maximum_lattice_x", "<i8"),
                        ("minimum_lattice_y", "<i8"), ("maximum_lattice_y", "<i8")])
NODE_DTYPE = np.dtype([("lattice_x", "<i8"), ("lattice_y", "<i8"), ("layer", "<u4"),
                       ("legal_edges", "u1"), ("reserved", "u1", (3,)), ("neighbors", "<u4", (8,))])
RUN_DTYPE = np.dtype([("node_offset", "<u4"), ("node_count", "<u4"), ("direction", "u1"),
                      ("reserved", "u1", (3,))])
POLICY_EDGE_DTYPE = np.dtype([("physical_edge_index", "<u4"), ("reserved", "<u4"), ("adjustment", "<u8")])
assert HEADER_DTYPE.itemsize == 112 and LAYER_DTYPE.itemsize == 48
assert NODE_DTYPE.itemsize == 56 and RUN_DTYPE.itemsize == 12 and POLICY_EDGE_DTYPE.itemsize == 16


@dataclasses.dataclass
class Query:
    start_node: int
    goal_node: int
    orthogonal_surcharge: int
    diagonal_surcharge: int
    bend_surcharge: int
    policy_identity: int
    cpu_status: int
    cpu_cost: int
    policy: np.ndarray


@dataclasses.dataclass
class Case:
    name: str
    header: np.ndarray
    layers: np.ndarray
    nodes: np.ndarray
    runs: np.ndarray
    run_nodes: np.ndarray
    queries: list

    @property
    def costs(self):
        h = self.header[0]
        return int(h["orthogonal_step"]), int(h["diagonal_step"]), int(h["bend"])


class _Reader:
    def __init__(self, data: bytes):
        self.data = data
        self.pos = 0

    def take(self, n: int) -> bytes:
        b = self.data[self.pos:self.pos + n]
        self.pos += n
        return b

    def u32(self) -> int:
        return int(np.frombuffer(self.take(4), "<u4")[0])

    def u64(self) -> int:
        return int(np.frombuffer(self.take(8), "<u8")[0])

    def array(self, dtype) -> np.ndarray:
        n = self.u64()
        return np.frombuffer(self.take(n * np.dtype(dtype).itemsize), dtype).copy()


def load_case(path: str) -> Case:
    r = _Reader(open(path, "rb").read())
    assert r.u64() == 0x3158495446524741, "bad fixture magic"
    header = np.frombuffer(r.take(112), HEADER_DTYPE).copy()
    layers = r.array(LAYER_DTYPE)
    nodes = r.array(NODE_DTYPE)
    runs = r.array(RUN_DTYPE)
    run_nodes = r.array("<u4")
    queries = []
    for _ in range(r.u64()):
        s, g = r.u32(), r.u32()
        o, d, b, ident = r.u64(), r.u64(), r.u64(), r.u64()
        status = r.u32()
        r.u32()
        cost = r.u64()
        policy = r.array(POLICY_EDGE_DTYPE)
        queries.append(Query(s, g, o, d, b, ident, status, cost, policy))
    return Case(os.path.basename(path)[:-4], header, layers, nodes, runs, run_nodes, queries)


def load_all() -> list:
    return [load_case(p) for p in sorted(glob.glob(os.path.join(HERE, "*.bin")))
            if os.path.basename(p) not in _NOT_CASES]


# reference outputs beside the cases (not device views)
_NOT_CASES = ("segments.bin", "clearance.bin", "geometry.bin")


SEGMENT_DTYPE = np.dtype([("layer", "<u4"), ("pad", "<u4"), ("x0", "<i8"), ("y0", "<i8"),
                          ("x1", "<i8"), ("y1", "<i8")])


def load_segments() -> list:
    """Reference routing::CoalesceSegments outputs: one (case name, query
    index, forward device nodes of the reference CPU A* route, segments)
    tuple per reached route of the corpus (written by oracle/ref_fixtures.cc)."""
    r = _Reader(open(os.path.join(HERE, "segments.bin"), "rb").read())
    assert r.u64() == 0x3147455354524741, "bad segments magic"
    names = [c["name"] for c in manifest()["cases"]]
    out = []
    for _ in range(r.u64()):
        case, query = r.u32(), r.u32()
        nodes = r.array("<u4")
        segs = r.array(SEGMENT_DTYPE)
        out.append((names[case], query, nodes, segs))
    return out


def manifest() -> dict:
    with open(os.path.join(HERE, "manifest.json")) as f:
        return json.load(f)


CLEARANCE_DTYPE = np.dtype([("start", "<i8", 2), ("end", "<i8", 2), ("box_min", "<i8", 2),
                            ("box_max", "<i8", 2), ("width", "<i8"), ("clearance", "<i8"),
                            ("error", "<u4"), ("satisfied", "<u4")])
OBSTACLE_DTYPE = np.dtype([("min_x", "<i8"), ("min_y", "<i8"), ("max_x", "<i8"), ("max_y", "<i8"),
                           ("layer", "<u4"), ("owned", "<u4")])


def load_clearance() -> np.ndarray:
    """Reference geometry::SweptTraceClearanceAtLeast verdicts on seeded
    one-step segments and nearby boxes (oracle/ref_fixtures.cc)."""
    r = _Reader(open(os.path.join(HERE, "clearance.bin"), "rb").read())
    assert r.u64() == 0x3143524c43524741, "bad clearance magic"
    n = r.u64()
    return np.frombuffer(r.take(n * CLEARANCE_DTYPE.itemsize), CLEARANCE_DTYPE).copy()


def load_geometry() -> dict:
    """Per case name: the compile inputs of edge legality (heading mask,
    routing width and clearance, lattice placement, obstacle boxes)."""
    r = _Reader(open(os.path.join(HERE, "geometry.bin"), "rb").read())
    assert r.u64() == 0x314f454754524741, "bad geometry magic"
    names = [c["name"] for c in manifest()["cases"]]
    out = {}
    for _ in range(r.u64()):
        case, heading = r.u32(), r.u32()
        vals = np.frombuffer(r.take(40), "<i8")
        obstacles = r.array(OBSTACLE_DTYPE)
        out[names[case]] = dict(heading_mask=heading, width=int(vals[0]), clearance=int(vals[1]),
                                origin=(int(vals[2]), int(vals[3])), step=int(vals[4]),
                                obstacles=obstacles)
    return out
