"""numpy restatement of the corridor CNN (forward and backward).  TEST
INFRASTRUCTURE ONLY: the GPU kernels (apgar_b200/csrc/corridor_net.cu) are
checked against it layer by layer.

It follows the kernels' arithmetic: bf16 weights and activations (round to
nearest even), f32 accumulation, 3x3 "same" convolution over each net's
cw x ch window cells of a 64 x 64 grid with zero padding at the window border,
cells outside the window are zero.  Parameter layout: per layer l
w[32][9][cin_l] (tap = (dy + 1) * 3 + dx + 1) then b[32]; head w6[9][32], b6.
"""

from __future__ import annotations

import numpy as np

GRID = 64
CIN0 = 16
CH = 32

# Exact mode (``exact()``): every rounding point is the identity and the
# arithmetic is float64, so the backward can be checked against central finite
# differences of the forward.  The kernels' arithmetic is the default mode.
_EXACT = False


class exact:
    """Context manager: run the restatement in float64 without bf16 rounding."""

    def __enter__(self):
        global _EXACT
        self._prev, _EXACT = _EXACT, True
        return self

    def __exit__(self, *exc):
        global _EXACT
        _EXACT = self._prev
        return False


def _ft():
    return np.float64 if _EXACT else np.float32


def bf16(x):
    """Round float32 to bfloat16 (nearest even), returned as float32 (in
    exact mode: the value itself, as float64)."""
    if _EXACT:
        return np.asarray(x, dtype=np.float64)
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def from_bf16_bits(bits):
    return (np.asarray(bits, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


def offsets():
    o, at = {}, 0
    for layer in range(5):
        cin = CIN0 if layer == 0 else CH
        o[f"w{layer}"] = (at, (CH, 9, cin))
        at += CH * 9 * cin
        o[f"b{layer}"] = (at, (CH,))
        at += CH
    o["w6"] = (at, (9, CH))
    at += 9 * CH
    o["b6"] = (at, (1,))
    at += 1
    return o, at


def unflatten(params):
    o, total = offsets()
    assert params.size == total
    return {k: params[a:a + int(np.prod(s))].reshape(s) for k, (a, s) in o.items()}


def flatten(parts):
    o, total = offsets()
    out = np.zeros(total, _ft())
    for k, (a, s) in o.items():
        out[a:a + int(np.prod(s))] = parts[k].reshape(-1)
    return out


def valid_mask(dims):
    """bool [n][64][64]: cells inside each net's window (dims = cw | ch << 8)."""
    dims = np.asarray(dims, dtype=np.uint32)
    cw, ch = dims & 0xFF, (dims >> 8) & 0xFF
    ys, xs = np.arange(GRID)[None, :, None], np.arange(GRID)[None, None, :]
    return (xs < cw[:, None, None]) & (ys < ch[:, None, None])


def _shift(x, dy, dx):
    """out[y][x] = x[y + dy][x + dx], zero beyond the grid."""
    out = np.zeros_like(x)
    ys = slice(max(0, -dy), GRID - max(0, dy))
    xs = slice(max(0, -dx), GRID - max(0, dx))
    yt = slice(ys.start + dy, ys.stop + dy)
    xt = slice(xs.start + dx, xs.stop + dx)
    out[:, ys, xs] = x[:, yt, xt]
    return out


def conv(x, w, mask):
    """acc[cell][co] = sum_{tap, ci} x[cell + tap][ci] * w[co][tap][ci] over
    window cells (x zero outside the window), f32; zero outside the window."""
    x = np.where(mask[..., None], x, 0.0).astype(_ft())
    acc = np.zeros(x.shape[:3] + (w.shape[0],), _ft())
    for t in range(9):
        dy, dx = t // 3 - 1, t % 3 - 1
        acc += np.einsum("nyxc,oc->nyxo", _shift(x, dy, dx), w[:, t, :], optimize=True)
    return np.where(mask[..., None], acc, 0.0)


def conv_layer(x, params, layer, mask):
    p = unflatten(params)
    acc = conv(x, bf16(p[f"w{layer}"]), mask) + p[f"b{layer}"]
    return np.where(mask[..., None], bf16(np.maximum(acc, 0.0)), 0.0)


def head(a5, params, mask):
    p = unflatten(params)
    a5 = np.where(mask[..., None], a5, 0.0)
    z = np.zeros(a5.shape[:3], _ft())
    for t in range(9):
        dy, dx = t // 3 - 1, t % 3 - 1
        z += _shift(a5, dy, dx) @ p["w6"][t]
    return np.where(mask, z + p["b6"][0], 0.0)


def loss_grad(logits, labels, mask, pos_weight):
    """(loss, dlogit) of the kernels' weighted cross-entropy."""
    n = logits.shape[0]
    cells = mask.reshape(n, -1).sum(axis=1).astype(_ft())
    norm = (1.0 / (cells * n))[:, None, None]
    t = labels.astype(_ft())
    wgt = np.where(labels != 0, pos_weight, 1.0).astype(_ft())
    z = logits.astype(_ft())
    sig = 1.0 / (1.0 + np.exp(-z))
    g = np.where(mask, wgt * (sig - t) * norm, 0.0)
    l = np.where(mask, wgt * (np.maximum(z, 0) - z * t + np.log1p(np.exp(-np.abs(z)))) * norm, 0.0)
    return float(l.sum()), g.astype(_ft())


def head_backward(a5, params, dlogit, mask):
    """(gradient at layer 5's pre-activation, dw6, db6)."""
    p = unflatten(params)
    a5 = np.where(mask[..., None], a5, 0.0)
    da = np.zeros_like(a5)
    dw6 = np.zeros((9, CH), _ft())
    for t in range(9):
        dy, dx = t // 3 - 1, t % 3 - 1
        da += _shift(dlogit, -dy, -dx)[..., None] * p["w6"][t][None, None, None, :]
        dw6[t] = np.einsum("nyx,nyxc->c", dlogit, _shift(a5, dy, dx))
    dpre = np.where(mask[..., None] & (a5 > 0), bf16(da), 0.0)
    return dpre, dw6, np.array([dlogit.sum()], _ft())


def input_grad(dpre, params, layer, gate, mask):
    """Gradient at layer (layer - 1)'s pre-activation from the gradient at
    layer `layer`'s pre-activation: the flipped-kernel convolution, gated by
    the ReLU of the layer's input, rounded to bf16."""
    p = unflatten(params)
    w = bf16(p[f"w{layer}"])  # [co][tap][ci]
    wt = np.transpose(w[:, ::-1, :], (2, 1, 0))  # [ci][tap'][co], tap' = 8 - tap
    acc = conv(dpre, wt, mask)
    return np.where(mask[..., None] & (gate > 0), bf16(acc), 0.0)


def weight_grad(x, dpre, mask):
    """(dw[co][tap][ci], db[co]) = sums over window cells."""
    x = np.where(mask[..., None], x, 0.0)
    dpre = np.where(mask[..., None], dpre, 0.0)
    dw = np.zeros((CH, 9, x.shape[-1]), _ft())
    for t in range(9):
        dy, dx = t // 3 - 1, t % 3 - 1
        dw[:, t, :] = np.einsum("nyxo,nyxc->oc", dpre, _shift(x, dy, dx), optimize=True)
    return dw, dpre.sum(axis=(0, 1, 2)).astype(_ft())
