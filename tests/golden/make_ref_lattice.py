"""Writes tests/golden/ref_lattice/: single-layer 256 x 256 lattices whose
obstacles are seeded axis-aligned rectangles (sides uniform in 2-16 cells,
about 20% of cells blocked, the small configuration's obstacle model), a set
of two-terminal queries on free cells, and the reference's own verdicts on
them: the legal-edge masks of its geometry compiler (CompileBoard) and the
cost, expansion count and path of its CPU A* (RouteWithCpuAStar), produced by
oracle/_ref/ref_lattice (oracle/ref_lattice.cc, compiled from the reference
sources by oracle/build_ref.sh).

usage: python tests/golden/make_ref_lattice.py [out_dir]
"""

from __future__ import annotations

import os
import struct
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
SIZE = 256
CASES = ((31, 12), (32, 12))  # (seed, queries)


def rectangles(seed: int, size: int = SIZE, target: float = 0.20):
    """Seeded rectangles (inclusive cell bounds) and the blocked mask they make."""
    rng = np.random.default_rng(seed)
    blocked = np.zeros((size, size), dtype=bool)
    rects = []
    while blocked.mean() < target:
        w, h = rng.integers(2, 17, size=2)
        x0, y0 = rng.integers(0, size, size=2)
        x1, y1 = min(x0 + w, size) - 1, min(y0 + h, size) - 1
        rects.append((int(x0), int(y0), int(x1), int(y1)))
        blocked[y0:y1 + 1, x0:x1 + 1] = True
    return np.array(rects, dtype=np.uint32).reshape(-1, 4), blocked


def queries(seed: int, blocked: np.ndarray, count: int):
    rng = np.random.default_rng(seed + 1000)
    free = np.argwhere(~blocked)  # (y, x)
    out = []
    while len(out) < count:
        a, b = free[rng.integers(len(free), size=2)]
        if (a == b).all():
            continue
        out.append((int(a[1]), int(a[0]), int(b[1]), int(b[0])))
    return np.array(out, dtype=np.uint32)


def case_input(seed: int, count: int) -> bytes:
    rects, blocked = rectangles(seed)
    q = queries(seed, blocked, count)
    return (struct.pack("<II", SIZE, len(rects)) + rects.tobytes() + struct.pack("<I", len(q))
            + q.tobytes())


def main(out_dir: str) -> None:
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_lattice")
    if not os.path.exists(exe):
        sys.exit("oracle/_ref/ref_lattice is not built (run oracle/build_ref.sh)")
    os.makedirs(out_dir, exist_ok=True)
    for seed, count in CASES:
        inp = os.path.join(out_dir, f"board{seed}.in")
        with open(inp, "wb") as f:
            f.write(case_input(seed, count))
        subprocess.run([exe, inp, os.path.join(out_dir, f"board{seed}.out")], check=True)


def load(out_dir: str, seed: int):
    """(rects, queries, legal masks [size][size] u8, routes) of one case;
    routes: list of (status, cost, expanded, queue_pops, path [(x, y)])."""
    with open(os.path.join(out_dir, f"board{seed}.in"), "rb") as f:
        data = f.read()
    size, nrect = struct.unpack_from("<II", data, 0)
    rects = np.frombuffer(data, np.uint32, nrect * 4, 8).reshape(-1, 4)
    at = 8 + nrect * 16
    (nq,) = struct.unpack_from("<I", data, at)
    q = np.frombuffer(data, np.uint32, nq * 4, at + 4).reshape(-1, 4)
    with open(os.path.join(out_dir, f"board{seed}.out"), "rb") as f:
        out = f.read()
    magic, osize = struct.unpack_from("<QI", out, 0)
    assert magic == 0x3154414C54524741 and osize == size
    legal = np.frombuffer(out, np.uint8, size * size, 12).reshape(size, size)
    at = 12 + size * size
    (n,) = struct.unpack_from("<I", out, at)
    at += 4
    routes = []
    for _ in range(n):
        status, cost, expanded, pops, plen = struct.unpack_from("<IQQQI", out, at)
        at += 32
        path = np.frombuffer(out, np.uint32, plen * 2, at).reshape(-1, 2)
        at += plen * 8
        routes.append((status, cost, expanded, pops, path))
    return rects, q, legal, routes


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_lattice"))
