"""The corridor CNN restatement's backward against central finite differences.

The GPU training kernels are checked against ``oracle/corridor_net.py``'s
analytic backward; this test pins that backward itself.  In the restatement's
exact mode (float64, no bf16 rounding) the gradient of the weighted
cross-entropy with respect to every layer's weights and biases, the head's,
and the input rasters must equal central differences of the forward, to a
relative error of 1e-5: per tensor along a random direction (all entries at
once) and at sampled single entries.  The grid is shrunk to 8 x 8 cells to
keep the check fast; the windows (5 x 4 and 3 x 6 cells) lie inside it.
"""

import numpy as np
import pytest

from oracle import corridor_net as ref

TOL = 1e-5


@pytest.fixture()
def small_grid():
    old = ref.GRID
    ref.GRID = 8
    try:
        with ref.exact():
            yield
    finally:
        ref.GRID = old


def _problem(seed=3):
    rng = np.random.default_rng(seed)
    dims = np.array([5 | (4 << 8), 3 | (6 << 8)], np.uint32)
    mask = ref.valid_mask(dims)
    n = len(dims)
    x0 = np.where(mask[..., None], rng.normal(0.0, 1.0, (n, ref.GRID, ref.GRID, ref.CIN0)), 0.0)
    parts = {}
    for layer in range(5):
        cin = ref.CIN0 if layer == 0 else ref.CH
        parts[f"w{layer}"] = rng.normal(0.0, 1.0 / np.sqrt(9 * cin), (ref.CH, 9, cin))
        parts[f"b{layer}"] = rng.normal(0.05, 0.1, ref.CH)
    parts["w6"] = rng.normal(0.0, 1.0 / np.sqrt(9 * ref.CH), (9, ref.CH))
    parts["b6"] = rng.normal(0.0, 0.1, 1)
    params = ref.flatten(parts)
    labels = (rng.random((n, ref.GRID, ref.GRID)) < 0.3) & mask
    return params, x0, mask, labels.astype(np.uint8)


def _loss(params, x0, mask, labels):
    a = x0
    for layer in range(5):
        a = ref.conv_layer(a, params, layer, mask)
    return ref.loss_grad(ref.head(a, params, mask), labels, mask, 3.0)[0]


def _analytic(params, x0, mask, labels):
    x = [x0]
    for layer in range(5):
        x.append(ref.conv_layer(x[-1], params, layer, mask))
    z = ref.head(x[5], params, mask)
    _, dlogit = ref.loss_grad(z, labels, mask, 3.0)
    grads = {}
    dpre, grads["w6"], grads["b6"] = ref.head_backward(x[5], params, dlogit, mask)
    for layer in range(4, -1, -1):
        grads[f"w{layer}"], grads[f"b{layer}"] = ref.weight_grad(x[layer], dpre, mask)
        gate = x[layer] if layer > 0 else np.ones_like(x[0])
        dpre = ref.input_grad(dpre, params, layer, gate, mask)
    return ref.flatten(grads), dpre  # dpre is now d loss / d input rasters


def test_exact_mode_is_float64_without_rounding(small_grid):
    v = np.array([1.0 + 2.0 ** -20], np.float64)
    assert ref.bf16(v)[0] == v[0]
    assert ref.bf16(v).dtype == np.float64


@pytest.mark.parametrize("seed", [3, 11])
def test_parameter_gradients_equal_central_differences(small_grid, seed):
    params, x0, mask, labels = _problem(seed)
    g, _ = _analytic(params, x0, mask, labels)
    rng = np.random.default_rng(seed + 100)
    offsets, _ = ref.offsets()
    eps = 1e-6
    for name, (at, shape) in offsets.items():
        size = int(np.prod(shape))
        # directional derivative over the whole tensor
        v = np.zeros_like(params)
        v[at:at + size] = rng.normal(size=size)
        fd = (_loss(params + eps * v, x0, mask, labels) - _loss(params - eps * v, x0, mask, labels)) / (2 * eps)
        an = float(g @ v)
        assert abs(fd - an) <= TOL * max(abs(an), 1e-8), (name, fd, an)
        # sampled single entries
        for k in rng.choice(size, size=min(size, 4), replace=False):
            e = np.zeros_like(params)
            e[at + k] = 1.0
            fd = (_loss(params + eps * e, x0, mask, labels) - _loss(params - eps * e, x0, mask, labels)) / (2 * eps)
            an = g[at + k]
            assert abs(fd - an) <= TOL * max(abs(an), 1e-6), (name, int(k), fd, an)


def test_input_gradient_equals_central_differences(small_grid):
    params, x0, mask, labels = _problem(5)
    _, dx = _analytic(params, x0, mask, labels)
    rng = np.random.default_rng(7)
    eps = 1e-6
    v = np.where(mask[..., None], rng.normal(size=x0.shape), 0.0)
    fd = (_loss(params, x0 + eps * v, mask, labels) - _loss(params, x0 - eps * v, mask, labels)) / (2 * eps)
    an = float((dx * v).sum())
    assert abs(fd - an) <= TOL * max(abs(an), 1e-8), (fd, an)
    cells = np.argwhere(mask)
    for i in rng.choice(len(cells), size=6, replace=False):
        n, y, x = cells[i]
        c = int(rng.integers(ref.CIN0))
        e = np.zeros_like(x0)
        e[n, y, x, c] = 1.0
        fd = (_loss(params, x0 + eps * e, mask, labels) - _loss(params, x0 - eps * e, mask, labels)) / (2 * eps)
        an = dx[n, y, x, c]
        assert abs(fd - an) <= TOL * max(abs(an), 1e-6), (int(n), int(y), int(x), c, fd, an)
