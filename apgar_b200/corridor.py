"""Search corridors for the frontier generator's corridor mode.

A corridor is a 64 x 64 bitmap of coarse cells over a net's window: coarse
cell (cx, cy) covers window cells x in [cx << s, (cx + 1) << s) and y in
[cy << s, (cy + 1) << s) on every layer, where s = coarse_shift(win_w, win_h)
is the least value >= 2 that keeps both window sides within 63 coarse cells.
The device layout is 128 uint32 words per net, bit cx % 32 of word
2 * cy + cx // 32 (``apgar_b200_lattice_plan_set_corridors``).

Results never depend on the corridor: a net whose corridor result is not
certified is searched again over its whole window.  The corridor only decides
how much of the window the search touches.
"""

from __future__ import annotations

import numpy as np

COARSE = 64
MAX_SPAN = 63  # coarse cells a window may span per side (the CNN's layout keeps column 63 empty)
WORDS_PER_NET = 128

NONE, CERTIFIED, FALLBACK_EXIT, FALLBACK_UNREACHED = 0, 1, 2, 3
STATUS_NAMES = {NONE: "none", CERTIFIED: "certified", FALLBACK_EXIT: "fallback_exit",
                FALLBACK_UNREACHED: "fallback_unreached"}


def coarse_shift(win_w: int, win_h: int) -> int:
    """Coarse scale s of a window (the kernel's rule)."""
    span = max(int(win_w), int(win_h))
    s = 2
    while ((span - 1) >> s) >= MAX_SPAN:
        s += 1
    return s


def coarse_dims(win_w: int, win_h: int) -> tuple[int, int, int]:
    """(s, coarse width, coarse height) of a window."""
    s = coarse_shift(win_w, win_h)
    return s, -(-int(win_w) // (1 << s)), -(-int(win_h) // (1 << s))


def pack(masks: np.ndarray) -> np.ndarray:
    """Bool coarse masks [n][64 rows][64 cols] -> uint32 words [n][128]."""
    m = np.ascontiguousarray(masks, dtype=bool).reshape(len(masks), COARSE * COARSE)
    return np.packbits(m, axis=1, bitorder="little").view(np.uint32).reshape(len(masks),
                                                                              WORDS_PER_NET)


def unpack(words: np.ndarray) -> np.ndarray:
    """uint32 words [n][128] -> bool coarse masks [n][64][64]."""
    w = np.ascontiguousarray(words, dtype=np.uint32)
    bits = np.unpackbits(w.view(np.uint8).reshape(len(w), -1), axis=1, bitorder="little")
    return bits.astype(bool).reshape(len(w), COARSE, COARSE)


def terminals_coarse(nets: np.ndarray):
    """Coarse (x, y) of each net's start and goal, and each net's shift."""
    sx = (nets["start_x"].astype(np.int64) - nets["win_x0"])
    sy = (nets["start_y"].astype(np.int64) - nets["win_y0"])
    gx = (nets["goal_x"].astype(np.int64) - nets["win_x0"])
    gy = (nets["goal_y"].astype(np.int64) - nets["win_y0"])
    shifts = np.array([coarse_shift(w, h) for w, h in zip(nets["win_w"], nets["win_h"])],
                      dtype=np.int64)
    return (sx >> shifts, sy >> shifts), (gx >> shifts, gy >> shifts), shifts


def segment_corridor(nets: np.ndarray, radius: int | np.ndarray = 1) -> np.ndarray:
    """The fixed, unlearned corridor: coarse cells within Chebyshev distance
    ``radius`` of the coarse segment from start to goal.  Bool [n][64][64]."""
    (sx, sy), (gx, gy), shifts = terminals_coarse(nets)
    n = len(nets)
    radius = np.broadcast_to(np.asarray(radius, dtype=np.int64), (n,))
    out = np.zeros((n, COARSE, COARSE), dtype=bool)
    for i in range(n):
        steps = int(max(abs(gx[i] - sx[i]), abs(gy[i] - sy[i]), 1))
        t = np.linspace(0.0, 1.0, 2 * steps + 1)
        px = np.rint(sx[i] + t * (gx[i] - sx[i])).astype(np.int64)
        py = np.rint(sy[i] + t * (gy[i] - sy[i])).astype(np.int64)
        r = int(radius[i])
        for dy in range(-r, r + 1):
            for dx in range(-r, r + 1):
                x = np.clip(px + dx, 0, COARSE - 1)
                y = np.clip(py + dy, 0, COARSE - 1)
                out[i, y, x] = True
    return out


def full_corridor(n: int) -> np.ndarray:
    return np.ones((n, COARSE, COARSE), dtype=bool)
