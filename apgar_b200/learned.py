"""The learned corridor: a small CNN that proposes each net's search corridor.

Host mirror of the apgar_b200_cnn_* / apgar_b200_corridor_* C ABI.  The
network (6 layers of 3x3 convolutions, 32 channels, bf16 weights and
activations with f32 accumulation on the tensor cores) reads 64 x 64 coarse
rasters of each net's window (obstacle density, congestion, terminals and
their geometry) and outputs a corridor logit per coarse cell.  It is trained
on the GPU by the project's own forward and backward kernels, on the optimal
paths the exact plain sweep finds.

A corridor only decides how much of the window the frontier search touches:
a net whose corridor result is not certified by the exact integer
certificate is searched again over its whole window, so costs and paths
never depend on the network.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _check, lib

GRID = 64
PADDED_ROWS = GRID + 2  # rasters and activations carry a zero row above and below the grid
RASTER_CHANNELS = 16
CHANNELS = 32
WEIGHTS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "corridor_net.f32")


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def param_count() -> int:
    return int(lib().apgar_b200_cnn_param_count())


def operand_count() -> int:
    return int(lib().apgar_b200_cnn_operand_count())


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal convolution weights, zero biases, a small head biased
    towards "outside the corridor" (positives are rare)."""
    rng = np.random.default_rng(seed)
    parts = []
    for layer in range(5):
        cin = RASTER_CHANNELS if layer == 0 else CHANNELS
        parts.append(rng.normal(0.0, np.sqrt(2.0 / (9 * cin)), CHANNELS * 9 * cin))
        parts.append(np.zeros(CHANNELS))
    parts.append(rng.normal(0.0, np.sqrt(1.0 / (9 * CHANNELS)), 9 * CHANNELS))
    parts.append(np.array([-3.0]))
    out = np.concatenate(parts).astype(np.float32)
    assert out.size == param_count()
    return out


class CorridorNet:
    """Parameters, Adam state and bf16 operands of the corridor CNN on the
    current CUDA device."""

    def __init__(self, params: np.ndarray | None = None, seed: int = 0):
        import torch

        self.torch = torch
        p = init_params(seed) if params is None else np.asarray(params, np.float32)
        if p.size != param_count():
            raise ValueError(f"expected {param_count()} parameters, got {p.size}")
        self.params = torch.from_numpy(p.copy()).cuda()
        self.operands = torch.empty(operand_count(), dtype=torch.bfloat16, device="cuda")
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grads = torch.zeros_like(self.params)
        self.error = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.step = 0
        self.prepare()

    @classmethod
    def load(cls, path: str = WEIGHTS_PATH) -> "CorridorNet":
        return cls(np.fromfile(path, dtype=np.float32))

    def save(self, path: str = WEIGHTS_PATH) -> None:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        self.params.cpu().numpy().astype(np.float32).tofile(path)

    def prepare(self, stream: int = 0) -> None:
        _check(lib().apgar_b200_cnn_prepare(_ptr(self.params), _ptr(self.operands),
                                            ctypes.c_void_p(stream)))

    def check_error(self) -> None:
        if int(self.error.item()) != 0:
            raise RuntimeError(f"corridor CNN kernels reported error bits {int(self.error.item())}")

    def activations(self, count: int, distinct: bool):
        t = self.torch
        n = 5 if distinct else 2
        bufs = [t.zeros((count, PADDED_ROWS, GRID, CHANNELS), dtype=t.bfloat16, device="cuda")
                for _ in range(n)]
        return bufs if distinct else [bufs[i % 2] for i in range(5)]

    def forward(self, rasters, dims, acts=None, logits=None, stream: int = 0):
        t = self.torch
        count = int(dims.numel())
        if acts is None:
            acts = self.activations(count, distinct=False)
        if logits is None:
            logits = t.empty((count, GRID, GRID), dtype=t.float32, device="cuda")
        arr = (ctypes.c_void_p * 5)(*[a.data_ptr() for a in acts])
        _check(lib().apgar_b200_cnn_forward(_ptr(self.params), _ptr(self.operands), _ptr(rasters),
                                            _ptr(dims), ctypes.c_uint32(count), arr, _ptr(logits),
                                            _ptr(self.error), ctypes.c_void_p(stream)))
        return logits

    def backward(self, rasters, dims, acts, logits, labels, pos_weight: float, stream: int = 0):
        """Fills self.grads; returns the loss as a device scalar."""
        t = self.torch
        count = int(dims.numel())
        dlogit = t.empty_like(logits)
        s0 = t.empty_like(acts[0])
        s1 = t.empty_like(acts[0])
        loss = t.zeros(1, dtype=t.float32, device="cuda")
        arr = (ctypes.c_void_p * 5)(*[a.data_ptr() for a in acts])
        _check(lib().apgar_b200_cnn_backward(
            _ptr(self.params), _ptr(self.operands), _ptr(rasters), _ptr(dims), ctypes.c_uint32(count),
            arr, _ptr(logits), _ptr(labels), ctypes.c_float(pos_weight), _ptr(dlogit), _ptr(s0),
            _ptr(s1), _ptr(self.grads), _ptr(loss), _ptr(self.error), ctypes.c_void_p(stream)))
        return loss

    def adam(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8,
             stream: int = 0) -> None:
        self.step += 1
        _check(lib().apgar_b200_cnn_adam(_ptr(self.params), _ptr(self.grads), _ptr(self.m),
                                         _ptr(self.v), ctypes.c_uint32(self.step), ctypes.c_float(lr),
                                         ctypes.c_float(beta1), ctypes.c_float(beta2),
                                         ctypes.c_float(eps), ctypes.c_void_p(stream)))
        self.prepare(stream)

    def train_step(self, rasters, dims, labels, lr: float, pos_weight: float = 8.0, acts=None):
        if acts is None:
            acts = self.activations(int(dims.numel()), distinct=True)
        logits = self.forward(rasters, dims, acts=acts)
        loss = self.backward(rasters, dims, acts, logits, labels, pos_weight)
        self.adam(lr)
        return loss


def rasters(plan, cell_costs=None, stream: int = 0, out=None):
    """(rasters bf16 [n][66][64][16], dims uint32 [n]) of every net of a plan
    (into `out` = (rasters, dims) when given).  Only the pad row and grid rows
    0 .. ch of each net are written; a buffer allocated here starts zeroed."""
    import torch

    n = len(plan.nets)
    if out is not None:
        r, d = out
    else:
        r = torch.zeros((n, PADDED_ROWS, GRID, RASTER_CHANNELS), dtype=torch.bfloat16, device="cuda")
        d = torch.empty(n, dtype=torch.uint32, device="cuda")
    costs = None if cell_costs is None else _ptr(cell_costs)
    _check(lib().apgar_b200_corridor_rasters(plan.handle, costs, _ptr(r), _ptr(d), ctypes.c_void_p(stream)))
    return r, d


def labels(plan, dims, stream: int = 0):
    """Coarse path labels uint8 [n][64][64] from the plan's last execution."""
    import torch

    out = torch.empty((len(plan.nets), GRID, GRID), dtype=torch.uint8, device="cuda")
    _check(lib().apgar_b200_corridor_labels(plan.handle, _ptr(dims), _ptr(out), ctypes.c_void_p(stream)))
    return out


def corridors(plan, logits, dims, threshold: float = 0.0, dilate: int = 1, out=None,
              stream: int = 0, max_window_cells: int = 0):
    """Corridor bitmaps uint32 [n][128] from logits; nets whose window holds
    more than ``max_window_cells`` cells (0 = no limit) get no corridor."""
    import torch

    if out is None:
        out = torch.empty((len(plan.nets), 128), dtype=torch.uint32, device="cuda")
    _check(lib().apgar_b200_corridor_from_logits(plan.handle, _ptr(logits), _ptr(dims),
                                                 ctypes.c_float(threshold), ctypes.c_int32(dilate),
                                                 ctypes.c_uint64(max_window_cells), _ptr(out),
                                                 ctypes.c_void_p(stream)))
    return out


POLICY_PATH = os.path.join(os.path.dirname(WEIGHTS_PATH), "corridor_policy.json")


def load_policy(path: str = POLICY_PATH) -> dict:
    """The corridor policy: logit threshold and dilation (chosen at training
    time) and the largest window that gets a corridor (0 = all; chosen by
    measuring the learned form)."""
    import json

    with open(path) as f:
        return json.load(f)


class LearnedRouter:
    """The learned + persistent batched form on one frontier plan: per
    execution, rasters -> CNN -> corridors -> corridor-mode frontier search,
    all on one stream with buffers allocated once."""

    def __init__(self, plan, net: CorridorNet | None = None, policy: dict | None = None):
        import torch

        self.plan = plan
        self.net = net if net is not None else CorridorNet.load()
        self.policy = policy if policy is not None else load_policy()
        n = len(plan.nets)
        self.rasters = torch.zeros((n, PADDED_ROWS, GRID, RASTER_CHANNELS), dtype=torch.bfloat16,
                                   device="cuda")
        self.dims = torch.empty(n, dtype=torch.uint32, device="cuda")
        self.acts = self.net.activations(n, distinct=False)
        self.logits = torch.empty((n, GRID, GRID), dtype=torch.float32, device="cuda")
        self.bits = torch.empty((n, 128), dtype=torch.uint32, device="cuda")
        plan.set_corridors(self.bits)

    def propose(self, stream: int = 0, cell_costs=None) -> None:
        """Rasters -> CNN -> corridors.  ``cell_costs``: device address (int)
        or CUDA uint32 tensor of per-cell prices for the congestion channel
        (a negotiation's snapshot), or None."""
        self.rasterize(stream, cell_costs)
        self.infer(stream)
        self.extract(stream)

    def rasterize(self, stream: int = 0, cell_costs=None) -> None:
        """The proposal's first stage: every net's coarse raster and dims."""
        if cell_costs is not None and not isinstance(cell_costs, int):
            cell_costs = cell_costs.data_ptr()
        _check(lib().apgar_b200_corridor_rasters(
            self.plan.handle, ctypes.c_void_p(cell_costs) if cell_costs else None,
            _ptr(self.rasters), _ptr(self.dims), ctypes.c_void_p(stream)))

    def infer(self, stream: int = 0) -> None:
        """The second stage: the CNN's logits from the rasters."""
        self.net.forward(self.rasters, self.dims, acts=self.acts, logits=self.logits, stream=stream)

    def extract(self, stream: int = 0) -> None:
        """The third stage: the corridor bitmaps from the logits."""
        corridors(self.plan, self.logits, self.dims, threshold=float(self.policy["threshold"]),
                  dilate=int(self.policy["dilate"]), out=self.bits, stream=stream,
                  max_window_cells=int(self.policy.get("max_window_cells", 0)))

    def clear(self, stream: int = 0) -> None:
        """No corridor for any net (every window searched at once)."""
        import torch

        with torch.cuda.stream(torch.cuda.ExternalStream(stream)) if stream else _null():
            self.bits.zero_()

    def execute(self, stream: int = 0) -> None:
        self.propose(stream)
        self.plan.execute(stream)


class _null:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False
