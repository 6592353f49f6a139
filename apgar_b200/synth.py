"""Seeded synthetic routing lattices and nets for the lattice configurations.

No public benchmark suite exists for this path; these generators stand in for
the named lattice shapes.  Everything is derived from one integer seed through
numpy's PCG64 generator, so the GPU run, the CPU oracle and the CPU baseline all
see identical inputs.

Lattice rule (shared with the kernels and the oracle):
  * ``blocked`` is bit-packed per layer: word ``[l, y, x // 32]`` bit ``x % 32``.
  * orthogonal move legal iff both cells are free; diagonal move legal iff both
    cells and both side cells are free; via legal iff the cell is free on both
    layers and the via bit of that layer pair is set.
  * A net is searched inside its window: the terminal bounding box plus a
    margin (32 cells), clipped to the lattice, spanning every layer.

Obstacle model: axis-aligned rectangles with sides uniform in [2, 16] cells,
added independently per layer until the target blocked fraction is reached.
The medium/large configurations also carry pad keep-outs: 4x4-cell squares on
a 20-cell pitch (0.5 mm pitch at an assumed 25 um cell) on the outer layers.
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np

PAD_PITCH = 20
PAD_SIZE = 4
WINDOW_MARGIN = 32


@dataclasses.dataclass
class Lattice:
    layers: int
    height: int
    width: int
    blocked: np.ndarray  # uint32 [layers, height, width // 32]
    via_ok: np.ndarray | None  # uint32 [layers - 1, height, width // 32] or None
    orth: int = 10
    diag: int = 14
    via: int = 50

    def blocked_dense(self) -> np.ndarray:
        """bool [layers, height, width] view of the blocked bits."""
        return unpack_bits(self.blocked, self.width)

    @property
    def blocked_fraction(self) -> float:
        return float(self.blocked_dense().mean())


# Net record: start (layer, x, y), goal (layer, x, y), window (x0, y0, w, h).
NET_DTYPE = np.dtype(
    [
        ("start_layer", "<u4"),
        ("start_x", "<u4"),
        ("start_y", "<u4"),
        ("goal_layer", "<u4"),
        ("goal_x", "<u4"),
        ("goal_y", "<u4"),
        ("win_x0", "<u4"),
        ("win_y0", "<u4"),
        ("win_w", "<u4"),
        ("win_h", "<u4"),
    ]
)


def pack_bits(dense: np.ndarray) -> np.ndarray:
    """bool [..., width] -> uint32 [..., width // 32], bit x % 32 of word x // 32."""
    width = dense.shape[-1]
    if width % 32:
        raise ValueError("width must be a multiple of 32")
    bits = dense.reshape(dense.shape[:-1] + (width // 32, 32)).astype(np.uint64)
    weights = (np.uint64(1) << np.arange(32, dtype=np.uint64)).astype(np.uint64)
    return (bits * weights).sum(axis=-1).astype(np.uint32)


def unpack_bits(words: np.ndarray, width: int) -> np.ndarray:
    shifts = np.arange(32, dtype=np.uint32)
    bits = (words[..., None] >> shifts) & np.uint32(1)
    return bits.reshape(words.shape[:-1] + (width,)).astype(bool)


def _paint_rectangles(rng: np.random.Generator, height: int, width: int, target: float,
                      base: np.ndarray) -> np.ndarray:
    """Add random rectangles (sides U[2,16]) to ``base`` until ``target`` is met."""
    blocked = base.copy()
    cells = height * width
    while blocked.mean() < target:
        deficit = (target - blocked.mean()) * cells
        count = max(16, int(deficit / 81.0 * 1.15))
        w = rng.integers(2, 17, size=count)
        h = rng.integers(2, 17, size=count)
        x0 = rng.integers(0, width, size=count)
        y0 = rng.integers(0, height, size=count)
        x1 = np.minimum(x0 + w, width)
        y1 = np.minimum(y0 + h, height)
        diff = np.zeros((height + 1, width + 1), dtype=np.int32)
        np.add.at(diff, (y0, x0), 1)
        np.add.at(diff, (y0, x1), -1)
        np.add.at(diff, (y1, x0), -1)
        np.add.at(diff, (y1, x1), 1)
        cover = diff.cumsum(0).cumsum(1)[:height, :width] > 0
        candidate = blocked | cover
        if candidate.mean() > target + 0.01 and count > 16:
            # add in smaller portions near the target to land close to it
            order = rng.permutation(count)
            for chunk in np.array_split(order, 8):
                d = np.zeros((height + 1, width + 1), dtype=np.int32)
                np.add.at(d, (y0[chunk], x0[chunk]), 1)
                np.add.at(d, (y0[chunk], x1[chunk]), -1)
                np.add.at(d, (y1[chunk], x0[chunk]), -1)
                np.add.at(d, (y1[chunk], x1[chunk]), 1)
                blocked |= d.cumsum(0).cumsum(1)[:height, :width] > 0
                if blocked.mean() >= target:
                    break
        else:
            blocked = candidate
    return blocked


def make_lattice(seed: int, layers: int, size: int, blocked_fraction: float,
                 pads: bool = False, via_mask: bool = False) -> Lattice:
    """Seeded lattice of ``layers`` x ``size`` x ``size`` cells."""
    rng = np.random.default_rng(seed)
    dense = np.zeros((layers, size, size), dtype=bool)
    for layer in range(layers):
        base = np.zeros((size, size), dtype=bool)
        if pads and layer in (0, layers - 1):
            grid = np.zeros((size, size), dtype=bool)
            offsets = np.arange(PAD_PITCH // 2 - PAD_SIZE // 2, size, PAD_PITCH)
            for dy in range(PAD_SIZE):
                for dx in range(PAD_SIZE):
                    ys = offsets + dy
                    xs = offsets + dx
                    ys = ys[ys < size]
                    xs = xs[xs < size]
                    grid[np.ix_(ys, xs)] = True
            base |= grid
        dense[layer] = _paint_rectangles(rng, size, size, blocked_fraction, base)
    via_ok = None
    if via_mask and layers > 1:
        # optional via keep-outs: a sparse random subset of cells forbids vias
        forbid = rng.random((layers - 1, size, size)) < 0.05
        via_ok = pack_bits(~forbid)
    return Lattice(layers, size, size, pack_bits(dense), via_ok)


def _window(lat: Lattice, sx, sy, gx, gy, margin):
    x0 = max(0, min(sx, gx) - margin)
    y0 = max(0, min(sy, gy) - margin)
    x1 = min(lat.width - 1, max(sx, gx) + margin)
    y1 = min(lat.height - 1, max(sy, gy) + margin)
    return x0, y0, x1 - x0 + 1, y1 - y0 + 1


def make_nets(lat: Lattice, seed: int, count: int, hpwl_median: float | None = None,
              hpwl_sigma: float = 1.0, margin: int | None = WINDOW_MARGIN) -> np.ndarray:
    """Two-terminal nets on free cells.

    With ``hpwl_median`` None both terminals are uniform over free cells (the
    small configuration); otherwise the bounding-box half-perimeter is
    lognormal(ln median, sigma), split uniformly between dx and dy.  With
    ``margin`` None the window is the whole lattice.
    """
    rng = np.random.default_rng(seed)
    free = ~lat.blocked_dense()
    nets = np.zeros(count, dtype=NET_DTYPE)
    free_idx = np.flatnonzero(free.ravel())
    plane = lat.height * lat.width
    made = 0
    while made < count:
        a = int(free_idx[rng.integers(0, free_idx.size)])
        sl, rem = divmod(a, plane)
        sy, sx = divmod(rem, lat.width)
        if hpwl_median is None:
            b = int(free_idx[rng.integers(0, free_idx.size)])
            gl, rem = divmod(b, plane)
            gy, gx = divmod(rem, lat.width)
        else:
            hp = int(round(math.exp(math.log(hpwl_median) + hpwl_sigma * rng.standard_normal())))
            hp = max(hp, 1)
            dx = int(round(hp * rng.random()))
            dy = hp - dx
            gx = sx + (dx if rng.random() < 0.5 else -dx)
            gy = sy + (dy if rng.random() < 0.5 else -dy)
            gl = int(rng.integers(0, lat.layers))
            if not (0 <= gx < lat.width and 0 <= gy < lat.height):
                continue
            if not free[gl, gy, gx]:
                continue
        if (sl, sx, sy) == (gl, gx, gy):
            continue
        if margin is None:
            x0, y0, w, h = 0, 0, lat.width, lat.height
        else:
            x0, y0, w, h = _window(lat, sx, sy, gx, gy, margin)
        nets[made] = (sl, sx, sy, gl, gx, gy, x0, y0, w, h)
        made += 1
    return nets


# ---------------------------------------------------------------------------
# Named configurations (sizes from the reference-facing benchmark description)
# ---------------------------------------------------------------------------

def config_small(seed: int = 1):
    """2 layers of 256x256, ~20% blocked, 64 nets uniform over free cells,
    whole-lattice search."""
    lat = make_lattice(seed, 2, 256, 0.20)
    nets = make_nets(lat, seed + 1000, 64, hpwl_median=None, margin=None)
    return lat, nets


def config_medium(seed: int = 2, nets: int = 4096, size: int = 2048):
    """4 layers of 2048x2048, 25% blocked (rectangles + pad keep-outs), 4096
    nets with lognormal(200, 1.0) half-perimeter, bbox + 32 windows."""
    lat = make_lattice(seed, 4, size, 0.25, pads=True)
    net_arr = make_nets(lat, seed + 1000, nets, hpwl_median=200.0, hpwl_sigma=1.0)
    return lat, net_arr


def window_cells(lat: Lattice, nets: np.ndarray) -> np.ndarray:
    return nets["win_w"].astype(np.int64) * nets["win_h"].astype(np.int64) * lat.layers


def make_multi_terminal_nets(lat: Lattice, seed: int, count: int, hpwl_median: float,
                             hpwl_sigma: float, min_terminals: int = 2, max_terminals: int = 6,
                             margin: int = WINDOW_MARGIN) -> tuple[np.ndarray, np.ndarray]:
    """Nets with ``min_terminals``..``max_terminals`` terminals (uniform) on free
    cells inside a bounding box whose half-perimeter is lognormal(ln median,
    sigma), split into 2-pin segments along a Manhattan minimum spanning tree
    of the terminals (Prim).  Returns (segments as two-terminal net records
    with bbox + margin windows, owning net index per segment)."""
    rng = np.random.default_rng(seed)
    free = ~lat.blocked_dense()
    segs, owner = [], []
    made = 0
    while made < count:
        hp = max(2, int(round(math.exp(math.log(hpwl_median) + hpwl_sigma * rng.standard_normal()))))
        bw = min(lat.width, max(1, int(round(hp * rng.random()))) + 1)
        bh = min(lat.height, max(1, hp - bw + 1) + 1)
        bx = int(rng.integers(0, lat.width - bw + 1))
        by = int(rng.integers(0, lat.height - bh + 1))
        k = int(rng.integers(min_terminals, max_terminals + 1))
        terms = []
        for _ in range(64 * k):
            x = bx + int(rng.integers(0, bw))
            y = by + int(rng.integers(0, bh))
            l = int(rng.integers(0, lat.layers))
            if free[l, y, x] and (l, x, y) not in terms:
                terms.append((l, x, y))
                if len(terms) == k:
                    break
        if len(terms) < 2:
            continue
        # Prim's MST under Manhattan distance (ties by terminal order)
        in_tree = [0]
        rest = list(range(1, len(terms)))
        while rest:
            best = None
            for a in in_tree:
                for b in rest:
                    d = abs(terms[a][1] - terms[b][1]) + abs(terms[a][2] - terms[b][2])
                    if best is None or d < best[0]:
                        best = (d, a, b)
            _, a, b = best
            (sl, sx, sy), (gl, gx, gy) = terms[a], terms[b]
            x0, y0, w, h = _window(lat, sx, sy, gx, gy, margin)
            segs.append((sl, sx, sy, gl, gx, gy, x0, y0, w, h))
            owner.append(made)
            in_tree.append(b)
            rest.remove(b)
        made += 1
    return np.array(segs, dtype=NET_DTYPE), np.array(owner, dtype=np.int64)


def config_full(seed: int = 5, nets: int = 32768, size: int = 8192, layers: int = 8):
    """8 layers of 8192x8192 (30% blocked, rectangles + pad keep-outs), 32768
    nets with 2-8 terminals split into 2-pin segments, half-perimeter
    lognormal(400, 1.3), bbox + 32 windows; one routing resource per cell with
    capacity 1 (the full-scale combined configuration)."""
    lat = make_lattice(seed, layers, size, 0.30, pads=True)
    segs, owner = make_multi_terminal_nets(lat, seed + 1000, nets, 400.0, 1.3, max_terminals=8)
    return lat, segs, owner


def config_negotiated(seed: int = 3, nets: int = 16384, size: int = 4096, layers: int = 6):
    """6 layers of 4096x4096 (25% blocked, rectangles + pad keep-outs as in the
    medium configuration), 16384 nets with 2-6 terminals split into 2-pin
    segments, half-perimeter lognormal(300, 1.2), bbox + 32 windows; one
    routing resource per cell with capacity 1."""
    lat = make_lattice(seed, layers, size, 0.25, pads=True)
    segs, owner = make_multi_terminal_nets(lat, seed + 1000, nets, 300.0, 1.2)
    return lat, segs, owner
