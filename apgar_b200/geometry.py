"""Host mirror of the GPU geometry compile (apgar_b200_swept_clearance,
apgar_b200_compile_legal_edges): exact swept-trace clearance and the
legal-edge masks of lattice nodes against obstacle boxes."""

from __future__ import annotations

import ctypes

import numpy as np

from . import _check, _vp, lib

OBSTACLE_DTYPE = np.dtype([("min_x", "<i8"), ("min_y", "<i8"), ("max_x", "<i8"), ("max_y", "<i8"),
                           ("layer", "<u4"), ("owned_by_net", "<u4")])
assert OBSTACLE_DTYPE.itemsize == 40

HORIZONTAL, VERTICAL, DIAGONAL45 = 1, 2, 4


class EdgeRules(ctypes.Structure):
    _fields_ = [
        ("nominal_width", ctypes.c_int64),
        ("clearance", ctypes.c_int64),
        ("lattice_origin_x", ctypes.c_int64),
        ("lattice_origin_y", ctypes.c_int64),
        ("lattice_step", ctypes.c_int64),
        ("heading_mask", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]


def swept_clearance(cases: np.ndarray):
    """cases: int64 [n][10] (start x, y, end x, y, box min x, y, max x, y,
    width, clearance) -> (error codes, satisfied) as uint32 arrays."""
    cases = np.ascontiguousarray(cases, dtype=np.int64).reshape(-1, 10)
    out = np.zeros((max(len(cases), 1), 2), np.uint32)
    _check(lib().apgar_b200_swept_clearance(_vp(cases), ctypes.c_uint64(len(cases)), _vp(out)))
    return out[: len(cases), 0], out[: len(cases), 1]


def compile_legal_edges(lattice_x, lattice_y, layers, origin, step: int, heading_mask: int,
                        width: int, clearance: int, obstacles) -> np.ndarray:
    """8-bit legal-edge masks (Direction order E, NE, N, NW, W, SW, S, SE)."""
    xy = np.ascontiguousarray(np.stack([np.asarray(lattice_x, np.int64),
                                        np.asarray(lattice_y, np.int64)], axis=1))
    layers = np.ascontiguousarray(layers, dtype=np.uint32)
    obstacles = np.ascontiguousarray(np.asarray(obstacles, dtype=OBSTACLE_DTYPE))
    rules = EdgeRules(int(width), int(clearance), int(origin[0]), int(origin[1]), int(step),
                      int(heading_mask), 0)
    out = np.zeros(max(len(layers), 1), np.uint8)
    _check(lib().apgar_b200_compile_legal_edges(
        ctypes.byref(rules), _vp(obstacles) if len(obstacles) else None,
        ctypes.c_uint64(len(obstacles)), _vp(xy), _vp(layers), ctypes.c_uint32(len(layers)),
        _vp(out)))
    return out[: len(layers)]
