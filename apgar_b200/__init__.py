"""apgar_b200: B200-native batched routing search behind a C ABI.

This package is a thin Python host mirror over ``libapgar_b200.so`` (the C ABI
declared in include/apgar_b200.h).  Every search runs in the CUDA kernels of
that library; there is no CPU fallback.  Importing works without a GPU (so the
ABI can be inspected), but every call that needs the device raises
``BackendError`` when the library or the device is missing.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import synth  # noqa: F401  (seeded inputs for tests and benchmarks)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libapgar_b200.so")

STATUS_NAMES = {
    0: "ok",
    1: "unsupported",
    2: "resource_exhausted",
    3: "backend_failure",
    4: "internal_invariant",
}

COMPLETION_REACHED = 0
COMPLETION_DISCONNECTED = 1
COMPLETION_BUDGET_EXHAUSTED = 2
COMPLETION_CANCELLED = 3
COMPLETION_REJECTED = 4
UNREACHABLE = 0xFFFFFFFF
NOALLOC_SCRATCH_BYTES = 32 * 1024 * 1024  # APGAR_B200_NOALLOC_SCRATCH_BYTES
NOALLOC_MAX_NETS = 4096  # APGAR_B200_NOALLOC_MAX_NETS


class BackendError(RuntimeError):
    """A C-ABI call failed; ``code`` mirrors the reference BackendErrorCode."""

    def __init__(self, code: int, detail: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {detail}")
        self.code = code
        self.detail = detail


class LatticeDesc(ctypes.Structure):
    _fields_ = [
        ("layers", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("width", ctypes.c_int32),
        ("blocked", ctypes.c_void_p),
        ("via_ok", ctypes.c_void_p),
        ("orth", ctypes.c_uint32),
        ("diag", ctypes.c_uint32),
        ("via", ctypes.c_uint32),
    ]


GENERATORS = {"sweep": 0, "frontier": 1}
LATTICE_PATH_CODES = {0: "ok", 1: "bounds", 2: "endpoint", 5: "edge", 7: "not_reached", 8: "cost"}


class LatticeOptions(ctypes.Structure):
    _fields_ = [
        ("generator", ctypes.c_uint32),
        ("max_iterations", ctypes.c_uint32),
        ("bucket_width", ctypes.c_uint32),
        ("chain", ctypes.c_uint32),
        ("class_bounds", ctypes.c_uint32),
        ("wide_bucket_width", ctypes.c_uint32),
        ("wide_chain", ctypes.c_uint32),
    ]


def class_bounds(*log2_limits: int) -> int:
    """Packs the frontier width-class limits (log2 of the largest window, in
    cells over all layers, of the 1-, 2-, 4- and 8-warp classes) into the
    options word; no argument gives 0, the library default."""
    if not log2_limits:
        return 0
    if len(log2_limits) != 4:
        raise ValueError("four class limits (1, 2, 4 and 8 warps per net)")
    return sum(int(b) << (8 * k) for k, b in enumerate(log2_limits))


def _options(generator: str, max_iterations: int, bucket_width: int, chain: int = 0,
             bounds: int = 0, wide_bucket_width: int = 0, wide_chain: int = 0) -> LatticeOptions:
    if generator not in GENERATORS:
        raise BackendError(1, f"unknown lattice generator {generator!r}")
    return LatticeOptions(GENERATORS[generator], max_iterations, bucket_width, chain, bounds,
                          wide_bucket_width, wide_chain)


def _schedule_fields(schedule):
    """(bucket_width, chain, class_bounds, wide_bucket_width, wide_chain) of a
    tuned schedule (``apgar_b200.autotune.Schedule``)."""
    return (schedule.bucket_width, schedule.chain, schedule.class_bounds,
            getattr(schedule, "wide_bucket_width", 0), getattr(schedule, "wide_chain", 0))


class PlanInfo(ctypes.Structure):
    _fields_ = [
        ("net_count", ctypes.c_uint32),
        ("kernel_launches", ctypes.c_uint32),
        ("class_count", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
        ("workspace_bytes", ctypes.c_uint64),
        ("label_cells", ctypes.c_uint64),
        ("path_arena_capacity", ctypes.c_uint64),
    ]


class Metadata(ctypes.Structure):
    _fields_ = [
        ("device_name", ctypes.c_char * 256),
        ("device_uuid", ctypes.c_char * 40),
        ("compute_capability_major", ctypes.c_uint32),
        ("compute_capability_minor", ctypes.c_uint32),
        ("runtime_version", ctypes.c_uint32),
        ("driver_version", ctypes.c_uint32),
        ("global_memory_bytes", ctypes.c_uint64),
        ("multiprocessor_count", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]


RESULT_DTYPE = np.dtype(
    [
        ("cost", "<u4"),
        ("completion", "<u4"),
        ("sweeps", "<u4"),
        ("path_len", "<u4"),
        ("path_offset", "<u8"),
        ("arena_offset", "<u8"),
        ("row_steps", "<u4"),
        ("row_stores", "<u4"),
        ("row_loads", "<u4"),
        ("reserved", "<u4"),
    ]
)
assert RESULT_DTYPE.itemsize == 48

_lib = None


def library_path() -> str:
    return LIB_PATH


def lib():
    """Loads libapgar_b200.so; raises BackendError if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise BackendError(3, f"CUDA library not built: {LIB_PATH} (run python -m apgar_b200.build)")
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.apgar_b200_last_error.restype = ctypes.c_size_t
        _lib.apgar_b200_abi_version.restype = ctypes.c_uint32
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        buf = ctypes.create_string_buffer(1024)
        lib().apgar_b200_last_error(buf, ctypes.c_size_t(len(buf)))
        raise BackendError(rc, buf.value.decode(errors="replace"))


def query_metadata() -> dict:
    m = Metadata()
    _check(lib().apgar_b200_query_metadata(ctypes.byref(m)))
    return {f: (getattr(m, f).decode() if isinstance(getattr(m, f), bytes) else getattr(m, f))
            for f, _ in Metadata._fields_ if f != "reserved"}


def _vp(a: np.ndarray | None):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


class DeviceLattice:
    """A lattice uploaded to the current CUDA device (the prepared view)."""

    def __init__(self, lat):
        self.layers, self.height, self.width = lat.layers, lat.height, lat.width
        self.orth, self.diag, self.via = int(lat.orth), int(lat.diag), int(lat.via)
        self._blocked = np.ascontiguousarray(lat.blocked, dtype=np.uint32)
        self._via = None if lat.via_ok is None else np.ascontiguousarray(lat.via_ok, np.uint32)
        desc = LatticeDesc(lat.layers, lat.height, lat.width, _vp(self._blocked), _vp(self._via),
                           lat.orth, lat.diag, lat.via)
        handle = ctypes.c_void_p()
        _check(lib().apgar_b200_lattice_upload(ctypes.byref(desc), ctypes.byref(handle)))
        self.handle = handle

    def close(self):
        if self.handle:
            lib().apgar_b200_lattice_release(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def route(self, nets: np.ndarray, max_sweeps: int = 4096, cancel: np.ndarray | None = None,
              want_paths: bool = True, path_capacity: int | None = None, out=None,
              generator: str = "sweep", max_rounds: int = 1 << 30, bucket_width: int = 0,
              chain: int = 0, class_bounds: int = 0, schedule=None, wide_bucket_width: int = 0,
              wide_chain: int = 0):
        """Searches every net; returns (results record array, packed paths).

        ``generator`` is "sweep" (budget ``max_sweeps``) or "frontier"
        (budget ``max_rounds``, key level width ``bucket_width``, 0 = twice
        the largest move; ``chain``, 0 = the default per width class, n = up
        to n - 1 chained expansions per queued cell; ``class_bounds``, the
        packed width-class limits of ``class_bounds()``, 0 = the default;
        ``wide_bucket_width`` and ``wide_chain``, the 16-warp class's own level
        width and chain, 0 = as the others; or a tuned ``schedule`` holding
        all five).  ``out`` may supply
        preallocated (results, paths) host arrays (pinned memory makes the
        transfers faster)."""
        nets = np.ascontiguousarray(nets)
        count = len(nets)
        if out is not None:
            results, paths = out
            # the C side writes count records and up to paths.size cells
            if not (isinstance(results, np.ndarray) and results.dtype == RESULT_DTYPE
                    and results.flags.c_contiguous and results.size >= count):
                raise ValueError("out[0] must be a C-contiguous RESULT_DTYPE array of at least "
                                 f"{count} records")
            if not (isinstance(paths, np.ndarray) and paths.dtype == np.uint32
                    and paths.flags.c_contiguous):
                raise ValueError("out[1] must be a C-contiguous uint32 array")
        else:
            results = np.empty(count, dtype=RESULT_DTYPE)
            cap = path_capacity or int(8 * (nets["win_w"].astype(np.int64)
                                            + nets["win_h"].astype(np.int64)).sum() + 64 * self.layers * count + 64)
            paths = np.empty(cap if want_paths else 0, dtype=np.uint32)
        total = ctypes.c_uint64(0)
        if generator == "sweep":
            _check(lib().apgar_b200_lattice_route(
                self.handle, _vp(nets), ctypes.c_uint32(count), ctypes.c_uint32(max_sweeps),
                _vp(cancel), _vp(results), _vp(paths) if want_paths else None,
                ctypes.c_uint64(paths.size if want_paths else 0), ctypes.byref(total)))
        else:
            if schedule is not None:
                bucket_width, chain, class_bounds, wide_bucket_width, wide_chain = \
                    _schedule_fields(schedule)
            opts = _options(generator, max_rounds, bucket_width, chain, class_bounds,
                            wide_bucket_width, wide_chain)
            _check(lib().apgar_b200_lattice_route_ex(
                self.handle, _vp(nets), ctypes.c_uint32(count), ctypes.byref(opts),
                _vp(cancel), _vp(results), _vp(paths) if want_paths else None,
                ctypes.c_uint64(paths.size if want_paths else 0), ctypes.byref(total)))
        return results, (paths[: total.value] if want_paths else None)

    def validate(self, nets: np.ndarray, results: np.ndarray, paths: np.ndarray) -> np.ndarray:
        """Device validation of read-back route results (packed reverse paths):
        one (code, reserved, failing forward index, cost sum) record per net,
        codes as in ``LATTICE_PATH_CODES``."""
        from .dropin import VERDICT_DTYPE

        nets = np.ascontiguousarray(nets)
        results = np.ascontiguousarray(results)
        paths = np.ascontiguousarray(paths, dtype=np.uint32)
        out = np.zeros(len(nets), dtype=VERDICT_DTYPE)
        _check(lib().apgar_b200_lattice_validate(
            self.handle, _vp(nets), ctypes.c_uint32(len(nets)), _vp(results),
            _vp(paths) if len(paths) else None, ctypes.c_uint64(len(paths)), _vp(out)))
        return out

    def route_noalloc(self, nets: np.ndarray, max_sweeps: int = 4096, stream: int = 0,
                      out=None):
        """``route`` without device allocation: the library's fixed scratch
        (``NOALLOC_SCRATCH_BYTES`` per device, at most ``NOALLOC_MAX_NETS``
        nets) holds the workspace, and work goes to ``stream``.  Calls share
        that scratch and take one process-wide lock, so concurrent calls run
        one after another.  ``out`` may supply preallocated (results, paths)
        host arrays so that the call allocates nothing in Python either."""
        nets = np.ascontiguousarray(nets)
        count = len(nets)
        if out is not None:
            results, paths = out
            # the C side writes count records and up to paths.size cells
            if not (isinstance(results, np.ndarray) and results.dtype == RESULT_DTYPE
                    and results.flags.c_contiguous and results.size >= count):
                raise ValueError("out[0] must be a C-contiguous RESULT_DTYPE array of at least "
                                 f"{count} records")
            if not (isinstance(paths, np.ndarray) and paths.dtype == np.uint32
                    and paths.flags.c_contiguous):
                raise ValueError("out[1] must be a C-contiguous uint32 array")
        else:
            results = np.empty(count, dtype=RESULT_DTYPE)
            cap = int(8 * (nets["win_w"].astype(np.int64) + nets["win_h"].astype(np.int64)).sum()
                      + 64 * self.layers * count + 64)
            paths = np.empty(cap, dtype=np.uint32)
        total = ctypes.c_uint64(0)
        _check(lib().apgar_b200_lattice_route_noalloc(
            self.handle, _vp(nets), ctypes.c_uint32(count), ctypes.c_uint32(max_sweeps),
            ctypes.c_void_p(stream), _vp(results), _vp(paths), ctypes.c_uint64(paths.size),
            ctypes.byref(total)))
        return results, paths[: total.value]

    def plan(self, nets: np.ndarray, max_sweeps: int = 4096, generator: str = "sweep",
             max_rounds: int = 1 << 30, bucket_width: int = 0, chain: int = 0,
             class_bounds: int = 0, schedule=None) -> "Plan":
        """``schedule``: a frontier schedule (for example from
        ``apgar_b200.autotune.tune``) whose bucket width, chain and class bounds
        replace the three arguments."""
        if schedule is not None:
            bucket_width, chain, class_bounds, wide_bucket_width, wide_chain = _schedule_fields(schedule)
        else:
            wide_bucket_width = wide_chain = 0
        return Plan(self, nets, max_sweeps, generator, max_rounds, bucket_width, chain, class_bounds,
                    wide_bucket_width, wide_chain)


class Plan:
    """A planned batch resident on the device (execute may be graph-captured)."""

    def __init__(self, lattice: DeviceLattice, nets: np.ndarray, max_sweeps: int,
                 generator: str = "sweep", max_rounds: int = 1 << 30, bucket_width: int = 0,
                 chain: int = 0, class_bounds: int = 0, wide_bucket_width: int = 0,
                 wide_chain: int = 0):
        self.lattice = lattice
        self.nets = np.ascontiguousarray(nets)
        self.generator = generator
        handle = ctypes.c_void_p()
        if generator == "sweep":
            _check(lib().apgar_b200_lattice_plan(lattice.handle, _vp(self.nets),
                                                 ctypes.c_uint32(len(self.nets)),
                                                 ctypes.c_uint32(max_sweeps), ctypes.byref(handle)))
        else:
            opts = _options(generator, max_rounds, bucket_width, chain, class_bounds,
                            wide_bucket_width, wide_chain)
            _check(lib().apgar_b200_lattice_plan_ex(lattice.handle, _vp(self.nets),
                                                    ctypes.c_uint32(len(self.nets)),
                                                    ctypes.byref(opts), ctypes.byref(handle)))
        self.handle = handle

    def set_cell_costs(self, costs) -> None:
        """Per-cell entry prices for later executes: a CUDA uint32 tensor of
        layers*height*width cells (kept referenced here), or None."""
        self._cell_costs = costs
        ptr = None if costs is None else ctypes.c_void_p(costs.data_ptr())
        _check(lib().apgar_b200_lattice_plan_set_cell_costs(self.handle, ptr))

    def set_corridors(self, bits) -> None:
        """Corridor mode for later executes: a CUDA uint32 tensor [nets][128]
        of coarse corridor bitmaps (see ``apgar_b200.corridor``; kept
        referenced here), or None."""
        import torch

        if bits is not None and (bits.dtype != torch.uint32 or bits.numel() != 128 * len(self.nets)
                                 or not bits.is_cuda or not bits.is_contiguous()):
            raise ValueError("corridors are a contiguous CUDA uint32 tensor of 128 words per net")
        self._corridors = bits
        ptr = None if bits is None else ctypes.c_void_p(bits.data_ptr())
        _check(lib().apgar_b200_lattice_plan_set_corridors(self.handle, ptr))

    def segments(self, origin_x: int = 0, origin_y: int = 0, step: int = 1, stream: int = 0):
        """Exact-coordinate segments of the last execution's paths (GPU):
        (segments as a CUDA int64 tensor viewed by apgar_b200.dropin.SEGMENT_DTYPE
        after .cpu().numpy(), per-net counts as a CUDA int32 tensor); net i's
        segments start at its result's path_offset."""
        import torch

        cap = max(int(self.info()["path_arena_capacity"]), 1)
        segs = torch.empty(cap * 5, dtype=torch.int64, device="cuda")  # 40 B per segment
        counts = torch.empty(max(len(self.nets), 1), dtype=torch.int32, device="cuda")
        _check(lib().apgar_b200_lattice_segments(self.handle, ctypes.c_int64(origin_x),
                                                 ctypes.c_int64(origin_y), ctypes.c_int64(step),
                                                 ctypes.c_void_p(segs.data_ptr()),
                                                 ctypes.c_void_p(counts.data_ptr()),
                                                 ctypes.c_void_p(stream)))
        return segs, counts

    def corridor_status(self) -> np.ndarray:
        """Per-net corridor outcomes of the last corridor-mode execute
        (``apgar_b200.corridor`` CERTIFIED / FALLBACK_*)."""
        out = np.empty(len(self.nets), dtype=np.uint8)
        _check(lib().apgar_b200_lattice_plan_corridor_status(self.handle, _vp(out)))
        return out

    def execute(self, stream: int = 0) -> None:
        _check(lib().apgar_b200_lattice_execute(self.handle, ctypes.c_void_p(stream)))

    def info(self) -> dict:
        info = PlanInfo()
        _check(lib().apgar_b200_lattice_plan_info(self.handle, ctypes.byref(info)))
        return {f: getattr(info, f) for f, _ in PlanInfo._fields_ if f != "reserved"}

    def readback(self, want_paths: bool = True):
        count = len(self.nets)
        results = np.empty(count, dtype=RESULT_DTYPE)
        cap = int(self.info()["path_arena_capacity"]) if want_paths else 0
        paths = np.empty(cap, dtype=np.uint32)
        total = ctypes.c_uint64(0)
        _check(lib().apgar_b200_lattice_readback(self.handle, _vp(results),
                                                 _vp(paths) if want_paths else None,
                                                 ctypes.c_uint64(cap), ctypes.byref(total)))
        return results, (paths[: total.value] if want_paths else None)

    def close(self):
        if self.handle:
            lib().apgar_b200_lattice_plan_release(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def split_paths(results: np.ndarray, paths: np.ndarray) -> list:
    """Per-net reverse paths (goal first) from the packed array."""
    out = []
    for r in results:
        if r["completion"] == COMPLETION_REACHED:
            o = int(r["path_offset"])
            out.append(paths[o:o + int(r["path_len"])])
        else:
            out.append(None)
    return out
