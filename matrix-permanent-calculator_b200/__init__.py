"""Python mirror of the B200 permanent engine's C ABI (include/perman_b200.h).

The compute lives in ``libperman_b200.so`` (hand-written sm_100a CUDA kernels
behind ``extern "C"`` entry points); this module only binds it with ctypes so
that tests, the benchmark and Python callers use the same entry points a C,
C++ or ctypes caller would.  There is no CPU fallback: if the library is
missing or no B200 is usable, every compute call raises ``PermError``.

The reference (berkyaglioglu/matrix-permanent-calculator) exposes its GPU path
as C++ templates taking a row-major ``T* mat`` and returning a double
(gpu_exact_dense.cu:641, gpu_exact_sparse.cu:1124,
gpu_approximation_dense.cu:374 and :528, gpu_approximation_sparse.cu:455 and
:608).  Functions with the same names and argument meaning are provided at the
bottom of this module; they dispatch on the numpy dtype like the templates do
on ``T``.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libperman_b200.so"
CLI_PATH = PKG_DIR / "bin" / "perman"

PERM_OK, PERM_EINVAL, PERM_ECUDA, PERM_ENOMEM, PERM_EUNSUPPORTED, PERM_ETIMEOUT, PERM_EIO = 0, -1, -2, -3, -4, -5, -6
PERM_F64, PERM_F32, PERM_I32 = 0, 1, 2
PERM_KERNEL_DENSE, PERM_KERNEL_SKIPPER, PERM_KERNEL_DENSE_INT = 1, 2, 3
MAX_EXACT_N = 64
MAX_MC_N = 64

# Every extern "C" symbol declared in include/perman_b200.h.
EXPORTED_SYMBOLS = (
    "perm_version", "perm_device_count", "perm_ctx_create", "perm_ctx_destroy", "perm_ctx_last_error",
    "perm_status_string", "perm_exact_dense", "perm_exact_dense_shard", "perm_exact_dense_ex",
    "perm_exact_sparse", "perm_exact_sparse_ex", "perm_matrix_create_dense", "perm_matrix_create_dense_ex", "perm_matrix_destroy",
    "perm_exact_dense_resident",
    "perm_approx_rasmussen", "perm_approx_scaling", "perm_approx_rasmussen_sparse",
    "perm_approx_scaling_sparse", "perm_read_matrix", "perm_compress", "perm_fp64_peak",
    "gpu_perman64_xshared_coalescing_mshared_int", "gpu_perman64_xshared_coalescing_mshared_float",
    "gpu_perman64_xshared_coalescing_mshared_double",
    "gpu_perman64_xshared_coalescing_mshared_skipper_int",
    "gpu_perman64_xshared_coalescing_mshared_skipper_float",
    "gpu_perman64_xshared_coalescing_mshared_skipper_double",
    "gpu_perman64_rasmussen_int", "gpu_perman64_rasmussen_float", "gpu_perman64_rasmussen_double",
    "gpu_perman64_approximation_int", "gpu_perman64_approximation_float",
    "gpu_perman64_approximation_double", "gpu_perman64_rasmussen_sparse",
    "gpu_perman64_approximation_sparse",
)


class PermError(RuntimeError):
    """A failed engine call: status code and the context's message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class PermResult(ctypes.Structure):
    _fields_ = [("value", ctypes.c_double), ("hi", ctypes.c_double), ("lo", ctypes.c_double),
                ("steps", ctypes.c_double), ("total_steps", ctypes.c_double),
                ("kernel_ms", ctypes.c_double), ("kernel", ctypes.c_int), ("n", ctypes.c_int)]


class PermEstimate(ctypes.Structure):
    _fields_ = [("mean", ctypes.c_double), ("std_error", ctypes.c_double), ("trials", ctypes.c_double),
                ("zero_trials", ctypes.c_double), ("sum", ctypes.c_double), ("sum_sq", ctypes.c_double),
                ("kernel_ms", ctypes.c_double)]


_P = ctypes.c_void_p
_lib = None


def load_library(path: str | os.PathLike | None = None) -> ctypes.CDLL:
    """Load libperman_b200.so (raises PermError if it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise PermError(PERM_ECUDA, f"{p} is missing: run python matrix-permanent-calculator_b200/build.py")
    lib = ctypes.CDLL(str(p))
    i, d, u64, i64 = ctypes.c_int, ctypes.c_double, ctypes.c_uint64, ctypes.c_int64
    sig = {
        "perm_version": (i, []), "perm_device_count": (i, []),
        "perm_ctx_create": (i, [i, ctypes.POINTER(_P)]), "perm_ctx_destroy": (None, [_P]),
        "perm_ctx_last_error": (ctypes.c_char_p, [_P]), "perm_status_string": (ctypes.c_char_p, [i]),
        "perm_exact_dense": (i, [_P, _P, i, i, ctypes.POINTER(PermResult)]),
        "perm_exact_dense_shard": (i, [_P, _P, i, i, i, i, ctypes.POINTER(PermResult)]),
        "perm_exact_dense_ex": (i, [_P, _P, i, i, i, i, i, ctypes.POINTER(PermResult)]),
        "perm_matrix_create_dense_ex": (i, [_P, _P, i, i, i, ctypes.POINTER(_P)]),
        "perm_exact_sparse": (i, [_P, i, _P, _P, _P, _P, _P, _P, ctypes.POINTER(PermResult)]),
        "perm_exact_sparse_ex": (i, [_P, i, _P, _P, _P, _P, _P, _P, i, ctypes.POINTER(PermResult)]),
        "perm_matrix_create_dense": (i, [_P, _P, i, i, ctypes.POINTER(_P)]),
        "perm_matrix_destroy": (None, [_P, _P]),
        "perm_exact_dense_resident": (i, [_P, _P, ctypes.POINTER(PermResult)]),
        "perm_approx_rasmussen": (i, [_P, _P, i, i, i64, u64, _P, ctypes.POINTER(PermEstimate)]),
        "perm_approx_scaling": (i, [_P, _P, i, i, i64, i, i, u64, _P, ctypes.POINTER(PermEstimate)]),
        "perm_approx_rasmussen_sparse": (i, [_P, i, _P, _P, i64, u64, _P, ctypes.POINTER(PermEstimate)]),
        "perm_approx_scaling_sparse": (i, [_P, i, _P, _P, _P, _P, i64, i, i, u64, _P,
                                           ctypes.POINTER(PermEstimate)]),
        "perm_read_matrix": (i, [ctypes.c_char_p, i, i, _P, ctypes.POINTER(i), ctypes.POINTER(i),
                                 ctypes.c_char_p]),
        "perm_compress": (i, [i, _P, i, _P, _P, _P, _P, _P, _P]),
        "perm_fp64_peak": (i, [_P, ctypes.POINTER(d), ctypes.POINTER(d)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    for name in EXPORTED_SYMBOLS:
        if name.startswith("gpu_perman64"):
            getattr(lib, name).restype = d
    if path is None:
        _lib = lib
    return lib


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(_P)


def _as_matrix(mat) -> tuple[np.ndarray, int]:
    a = np.asarray(mat)
    if a.ndim != 2 or a.shape[0] != a.shape[1]:
        raise PermError(PERM_EINVAL, f"need a square matrix, got shape {a.shape}")
    if a.dtype == np.float32:
        return np.ascontiguousarray(a), PERM_F32
    if a.dtype.kind in "iub" and a.dtype.itemsize <= 4 and a.dtype != np.uint32:
        return np.ascontiguousarray(a, dtype=np.int32), PERM_I32
    return np.ascontiguousarray(a, dtype=np.float64), PERM_F64


@dataclass
class ExactResult:
    value: float
    hi: float
    lo: float
    steps: float
    total_steps: float
    kernel_ms: float
    kernel: int
    n: int


@dataclass
class Estimate:
    mean: float
    std_error: float
    trials: float
    zero_trials: float
    kernel_ms: float
    trial_values: np.ndarray | None = None


def _exact(r: PermResult) -> ExactResult:
    return ExactResult(r.value, r.hi, r.lo, r.steps, r.total_steps, r.kernel_ms, r.kernel, r.n)


class Engine:
    """One device context (stream + scratch) of libperman_b200.so."""

    def __init__(self, device: int = 0, lib_path=None):
        self.lib = load_library(lib_path)
        h = _P()
        rc = self.lib.perm_ctx_create(device, ctypes.byref(h))
        if rc != PERM_OK:
            raise PermError(rc, f"cannot create a context on device {device} "
                                f"({self.lib.perm_status_string(rc).decode()})")
        self.ctx = h
        self.device = device

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.perm_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int):
        if rc != PERM_OK:
            raise PermError(rc, self.lib.perm_ctx_last_error(self.ctx).decode())

    # ---- exact ----
    def exact_dense(self, mat, variant: int = 0) -> ExactResult:
        """Dense Ryser; variant 0 = automatic, PERM_KERNEL_DENSE = FP64 X, PERM_KERNEL_DENSE_INT = int32 X."""
        a, dt = _as_matrix(mat)
        r = PermResult()
        if variant:
            self._check(self.lib.perm_exact_dense_ex(self.ctx, _ptr(a), a.shape[0], dt, variant, 0, 1,
                                                     ctypes.byref(r)))
        else:
            self._check(self.lib.perm_exact_dense(self.ctx, _ptr(a), a.shape[0], dt, ctypes.byref(r)))
        return _exact(r)

    def exact_dense_shard(self, mat, shard: int, nshards: int, variant: int = 0) -> ExactResult:
        a, dt = _as_matrix(mat)
        r = PermResult()
        self._check(self.lib.perm_exact_dense_ex(self.ctx, _ptr(a), a.shape[0], dt, variant, shard, nshards,
                                                 ctypes.byref(r)))
        return _exact(r)

    def exact_sparse(self, n: int, rptrs, cols, rvals, cptrs, rows, cvals, variant: int = 0) -> ExactResult:
        """Sparse exact permanent; variant 0 = automatic, PERM_KERNEL_SKIPPER forces SkipPer."""
        ar = [np.ascontiguousarray(x, dtype=np.int32) for x in (rptrs, cols, cptrs, rows)]
        rv = np.ascontiguousarray(rvals, dtype=np.float64)
        cv = np.ascontiguousarray(cvals, dtype=np.float64)
        r = PermResult()
        self._check(self.lib.perm_exact_sparse_ex(self.ctx, n, _ptr(ar[0]), _ptr(ar[1]), _ptr(rv), _ptr(ar[2]),
                                                  _ptr(ar[3]), _ptr(cv), variant, ctypes.byref(r)))
        return _exact(r)

    def exact_sparse_matrix(self, mat, order: int = 2, variant: int = 0) -> ExactResult:
        """Sparse exact permanent of a dense matrix after the reference's -r <order> preprocessing."""
        c = compress(order, mat)
        return self.exact_sparse(c["n"], c["rptrs"], c["cols"], c["rvals"], c["cptrs"], c["rows"], c["cvals"],
                                 variant)

    def upload_dense(self, mat, variant: int = 0) -> "ResidentMatrix":
        a, dt = _as_matrix(mat)
        h = _P()
        self._check(self.lib.perm_matrix_create_dense_ex(self.ctx, _ptr(a), a.shape[0], dt, variant,
                                                         ctypes.byref(h)))
        return ResidentMatrix(self, h, a.shape[0])

    # ---- Monte Carlo ----
    def _estimate(self, e: PermEstimate, tv) -> Estimate:
        return Estimate(e.mean, e.std_error, e.trials, e.zero_trials, e.kernel_ms, tv)

    def rasmussen(self, mat, trials: int, seed: int = 1, keep_trials: bool = False) -> Estimate:
        a, dt = _as_matrix(mat)
        tv = np.empty(trials, dtype=np.float64) if keep_trials else None
        e = PermEstimate()
        self._check(self.lib.perm_approx_rasmussen(self.ctx, _ptr(a), a.shape[0], dt, trials, seed, _ptr(tv),
                                                   ctypes.byref(e)))
        return self._estimate(e, tv)

    def scaling(self, mat, trials: int, scale_intervals: int = 4, scale_times: int = 5, seed: int = 1,
                keep_trials: bool = False) -> Estimate:
        a, dt = _as_matrix(mat)
        tv = np.empty(trials, dtype=np.float64) if keep_trials else None
        e = PermEstimate()
        self._check(self.lib.perm_approx_scaling(self.ctx, _ptr(a), a.shape[0], dt, trials, scale_intervals,
                                                 scale_times, seed, _ptr(tv), ctypes.byref(e)))
        return self._estimate(e, tv)

    def rasmussen_sparse(self, n, rptrs, cols, trials, seed=1, keep_trials=False) -> Estimate:
        rp = np.ascontiguousarray(rptrs, dtype=np.int32)
        cl = np.ascontiguousarray(cols, dtype=np.int32)
        tv = np.empty(trials, dtype=np.float64) if keep_trials else None
        e = PermEstimate()
        self._check(self.lib.perm_approx_rasmussen_sparse(self.ctx, n, _ptr(rp), _ptr(cl), trials, seed,
                                                          _ptr(tv), ctypes.byref(e)))
        return self._estimate(e, tv)

    def scaling_sparse(self, n, rptrs, cols, cptrs, rows, trials, scale_intervals=4, scale_times=5, seed=1,
                       keep_trials=False) -> Estimate:
        arrs = [np.ascontiguousarray(x, dtype=np.int32) for x in (rptrs, cols, cptrs, rows)]
        tv = np.empty(trials, dtype=np.float64) if keep_trials else None
        e = PermEstimate()
        self._check(self.lib.perm_approx_scaling_sparse(self.ctx, n, *map(_ptr, arrs), trials, scale_intervals,
                                                        scale_times, seed, _ptr(tv), ctypes.byref(e)))
        return self._estimate(e, tv)

    def fp64_peak(self) -> tuple[float, float]:
        ops, ms = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.perm_fp64_peak(self.ctx, ctypes.byref(ops), ctypes.byref(ms)))
        return ops.value, ms.value


class ResidentMatrix:
    """A dense matrix kept in device memory; run() launches with no host copy."""

    def __init__(self, engine: Engine, handle, n: int):
        self.engine, self.handle, self.n = engine, handle, n

    def run(self) -> ExactResult:
        r = PermResult()
        self.engine._check(self.engine.lib.perm_exact_dense_resident(self.engine.ctx, self.handle,
                                                                     ctypes.byref(r)))
        return _exact(r)

    def free(self):
        if self.handle:
            self.engine.lib.perm_matrix_destroy(self.engine.ctx, self.handle)
            self.handle = None


# ---- host-only helpers (no device needed) -------------------------------------

def read_matrix(path, binary: bool = False, cap_n: int = 4096) -> tuple[np.ndarray, str, int]:
    """Read the reference text format; returns (row-major float64 matrix, type, header nnz)."""
    lib = load_library()
    with open(path) as f:
        head = f.readline().split()
    n_hdr = int(head[0]) if head else 0
    cap = max(1, min(cap_n, n_hdr))
    buf = np.zeros(cap * cap, dtype=np.float64)
    n, nnz = ctypes.c_int(), ctypes.c_int()
    typ = ctypes.create_string_buffer(8)
    rc = lib.perm_read_matrix(str(path).encode(), int(binary), cap, _ptr(buf), ctypes.byref(n), ctypes.byref(nnz),
                              typ)
    if rc != PERM_OK:
        raise PermError(rc, f"cannot read matrix file {path}")
    k = n.value
    return buf[: k * k].reshape(k, k).copy(), typ.value.decode(), nnz.value


def compress(mode: int, mat) -> dict:
    """CRS/CCS of the positive entries after the reference's -r <mode> ordering.

    Returns the arrays and the (possibly permuted) dense matrix under "mat"."""
    lib = load_library()
    a = np.array(mat, dtype=np.float64, order="C", copy=True)
    n = a.shape[0]
    cptrs = np.zeros(n + 1, np.int32)
    rptrs = np.zeros(n + 1, np.int32)
    rows = np.zeros(n * n, np.int32)
    cols = np.zeros(n * n, np.int32)
    cvals = np.zeros(n * n, np.float64)
    rvals = np.zeros(n * n, np.float64)
    nnz = lib.perm_compress(mode, _ptr(a), n, _ptr(cptrs), _ptr(rows), _ptr(cvals), _ptr(rptrs), _ptr(cols),
                            _ptr(rvals))
    if nnz < 0:
        raise PermError(nnz, "perm_compress failed")
    return {"n": n, "nnz": nnz, "mat": a, "cptrs": cptrs, "rows": rows[:nnz], "cvals": cvals[:nnz],
            "rptrs": rptrs, "cols": cols[:nnz], "rvals": rvals[:nnz]}


# ---- reference-named entry points (argument meaning as in the reference) ------
_default_engine: Engine | None = None


def default_engine() -> Engine:
    global _default_engine
    if _default_engine is None:
        _default_engine = Engine(int(os.environ.get("PERM_DEVICE", "0")))
    return _default_engine


def gpu_perman64_xshared_coalescing_mshared(mat, nov: int | None = None, grid_dim: int = 2048,
                                            block_dim: int = 256) -> float:
    """Dense exact permanent (gpu_exact_dense.cu:641); grid/block are ignored."""
    a = np.asarray(mat)
    if nov is not None and nov != a.shape[0]:
        a = a.reshape(nov, nov)
    return default_engine().exact_dense(a).value


def gpu_perman64_xshared_coalescing_mshared_skipper(mat, rptrs, cols, cptrs, rows, cvals, nov: int,
                                                    grid_dim: int = 2048, block_dim: int = 256) -> float:
    """SkipPer exact permanent (gpu_exact_sparse.cu:1124); CRS values taken from mat."""
    a = np.asarray(mat, dtype=np.float64).reshape(nov, nov)
    rptrs = np.asarray(rptrs, np.int32)
    cols = np.asarray(cols, np.int32)
    rvals = np.array([a[i, cols[p]] for i in range(nov) for p in range(rptrs[i], rptrs[i + 1])], np.float64)
    return default_engine().exact_sparse(nov, rptrs, cols, rvals, cptrs, rows, cvals).value


def gpu_perman64_rasmussen(mat, nov: int, number_of_times: int, seed: int = 1) -> float:
    """Rasmussen estimate (gpu_approximation_dense.cu:374)."""
    return default_engine().rasmussen(np.asarray(mat).reshape(nov, nov), number_of_times, seed).mean


def gpu_perman64_approximation(mat, nov: int, number_of_times: int, scale_intervals: int, scale_times: int,
                               seed: int = 1) -> float:
    """Scaling-based estimate (gpu_approximation_dense.cu:528)."""
    return default_engine().scaling(np.asarray(mat).reshape(nov, nov), number_of_times, scale_intervals,
                                    scale_times, seed).mean


def gpu_perman64_rasmussen_sparse(rptrs, cols, nov: int, nnz: int, number_of_times: int,
                                  grid_graph: bool = False, seed: int = 1) -> float:
    """Sparse Rasmussen estimate (gpu_approximation_sparse.cu:455)."""
    return default_engine().rasmussen_sparse(nov, rptrs, cols, number_of_times, seed).mean


def gpu_perman64_approximation_sparse(cptrs, rows, rptrs, cols, nov: int, nnz: int, number_of_times: int,
                                      scale_intervals: int, scale_times: int, grid_graph: bool = False,
                                      seed: int = 1) -> float:
    """Sparse scaling-based estimate (gpu_approximation_sparse.cu:608)."""
    return default_engine().scaling_sparse(nov, rptrs, cols, cptrs, rows, number_of_times, scale_intervals,
                                           scale_times, seed).mean
