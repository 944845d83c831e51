"""Python mirror of the B200 permanent engine's C ABI (include/perman_b200.h).

The compute lives in ``libperman_b200.so`` (hand-written sm_100a CUDA kernels
behind ``extern "C"`` entry points); this module only binds it with ctypes so
that tests, the benchmark and Python callers use the same entry points a C,
C++ or ctypes caller would.  There is no CPU fallback: if the library is
missing or no B200 is usable, every compute call raises ``PermError``.

The reference (berkyaglioglu/matrix-permanent-calculator) exposes its GPU path
as C++ templates taking a row-major ``T* mat`` and returning a double
(gpu_exact_dense.cu:641 and :702, gpu_exact_sparse.cu:1124,
gpu_approximation_dense.cu:374 and :528, gpu_approximation_sparse.cu:455 and
:608).  Functions with the same names and argument meaning are provided at the
bottom of this module; they dispatch on the numpy dtype like the templates do
on ``T``.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libperman_b200.so"
CLI_PATH = PKG_DIR / "bin" / "perman"

PERM_OK, PERM_EINVAL, PERM_ECUDA, PERM_ENOMEM, PERM_EUNSUPPORTED, PERM_ETIMEOUT, PERM_EIO = 0, -1, -2, -3, -4, -5, -6
PERM_F64, PERM_F32, PERM_I32 = 0, 1, 2
PERM_KERNEL_DENSE, PERM_KERNEL_SKIPPER, PERM_KERNEL_DENSE_INT, PERM_KERNEL_DENSE_DD = 1, 2, 3, 4
PERM_KERNEL_DENSE_TC = 5
PERM_KERNEL_DENSE_SPLIT = 6
PERM_KERNEL_DENSE_INT_DD = 7
PERM_KERNEL_DENSE_SDD = 8
MAX_EXACT_N = 64
MAX_MC_N = 64
MAX_MC_SPARSE_N = 2047

# Every extern "C" symbol declared in include/perman_b200.h.
EXPORTED_SYMBOLS = (
    "perm_version", "perm_device_count", "perm_ctx_create", "perm_ctx_destroy", "perm_ctx_last_error",
    "perm_status_string", "perm_exact_dense", "perm_exact_dense_shard", "perm_shard_range", "perm_exact_dense_multi",
    "perm_exact_dense_ex",
    "perm_exact_sparse", "perm_exact_sparse_ex", "perm_matrix_create_dense", "perm_matrix_create_dense_ex", "perm_matrix_destroy",
    "perm_exact_dense_resident", "perm_exact_dense_resident_shard", "perm_exact_dense_refine", "perm_sdd_layout", "perm_sdd_levels", "perm_fp64_layout", "perm_fp64_levels", "perm_int_layout", "perm_intc_layout", "perm_exact_dense_plan", "perm_exact_dense_tc_rounds", "perm_exact_dense_noalloc", "perm_dense_autotune", "perm_ctx_set_rel_target", "perm_ctx_inject_wait_timeout",
    "perm_batch_create", "perm_batch_run", "perm_batch_run_ex", "perm_batch_destroy", "perm_batch_exact", "perm_batch_autotune", "perm_batch_variant", "perm_batch_use_variant",
    "perm_server_create", "perm_server_submit", "perm_server_wait", "perm_server_stats", "perm_server_destroy",
    "perm_approx_rasmussen", "perm_approx_scaling", "perm_approx_rasmussen_range", "perm_approx_scaling_range",
    "perm_approx_rasmussen_sparse_range", "perm_approx_scaling_sparse_range", "perm_approx_rasmussen_sparse",
    "perm_approx_scaling_sparse", "perm_read_matrix", "perm_compress", "perm_grid_graph", "perm_fp64_peak",
    "gpu_perman64_xshared_coalescing_mshared_int", "gpu_perman64_xshared_coalescing_mshared_float",
    "gpu_perman64_xshared_coalescing_mshared_double",
    "gpu_perman64_xshared_coalescing_mshared_multigpu_int", "gpu_perman64_xshared_coalescing_mshared_multigpu_float",
    "gpu_perman64_xshared_coalescing_mshared_multigpu_double",
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
                ("kernel_ms", ctypes.c_double), ("kernel", ctypes.c_int), ("n", ctypes.c_int),
                ("abs_term_sum", ctypes.c_double), ("rel_error_estimate", ctypes.c_double)]


class PermRequest(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("n", ctypes.c_int), ("mat", ctypes.c_void_p), ("trials", ctypes.c_int64),
                ("scale_intervals", ctypes.c_int), ("scale_times", ctypes.c_int), ("seed", ctypes.c_uint64)]


class PermResponse(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("kernel", ctypes.c_int), ("value", ctypes.c_double),
                ("hi", ctypes.c_double), ("lo", ctypes.c_double), ("std_error", ctypes.c_double),
                ("t_submit_ms", ctypes.c_double), ("t_admit_ms", ctypes.c_double), ("t_done_ms", ctypes.c_double),
                ("device_ms", ctypes.c_double), ("message", ctypes.c_char * 160)]


PERM_REQ_EXACT_DENSE, PERM_REQ_EXACT_SPARSE, PERM_REQ_RASMUSSEN, PERM_REQ_SCALING = 0, 1, 2, 3


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
        "perm_shard_range": (i, [i, i, i, ctypes.POINTER(u64), ctypes.POINTER(u64)]),
        "perm_exact_dense_multi": (i, [_P, i, i, i, i, _P, ctypes.POINTER(PermResult)]),
        "perm_sdd_layout": (i, [_P, i]),
        "perm_sdd_levels": (i, [_P, i, _P]),
        "perm_intc_layout": (i, [_P, i, ctypes.POINTER(ctypes.c_int), _P]),
        "perm_int_layout": (i, [_P, i, _P]),
        "perm_fp64_layout": (i, [_P, i]),
        "perm_fp64_levels": (i, [_P, i, _P]),
        "perm_exact_dense_plan": (i, [_P, _P, i, i, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]),
        "perm_matrix_create_dense_ex": (i, [_P, _P, i, i, i, ctypes.POINTER(_P)]),
        "perm_exact_sparse": (i, [_P, i, _P, _P, _P, _P, _P, _P, ctypes.POINTER(PermResult)]),
        "perm_exact_sparse_ex": (i, [_P, i, _P, _P, _P, _P, _P, _P, i, ctypes.POINTER(PermResult)]),
        "perm_matrix_create_dense": (i, [_P, _P, i, i, ctypes.POINTER(_P)]),
        "perm_matrix_destroy": (None, [_P, _P]),
        "perm_exact_dense_resident": (i, [_P, _P, ctypes.POINTER(PermResult)]),
        "perm_exact_dense_resident_shard": (i, [_P, _P, i, i, ctypes.POINTER(PermResult)]),
        "perm_exact_dense_refine": (i, [_P, _P, i, i, ctypes.POINTER(PermResult)]),
        "perm_exact_dense_tc_rounds": (i, [_P, _P, i, i, u64, u64, ctypes.POINTER(PermResult)]),
        "perm_approx_rasmussen": (i, [_P, _P, i, i, i64, u64, _P, ctypes.POINTER(PermEstimate)]),
        "perm_approx_scaling": (i, [_P, _P, i, i, i64, i, i, u64, _P, ctypes.POINTER(PermEstimate)]),
        "perm_approx_rasmussen_range": (i, [_P, _P, i, i, i64, i64, u64, _P, ctypes.POINTER(PermEstimate)]),
        "perm_approx_scaling_range": (i, [_P, _P, i, i, i64, i64, i, i, u64, _P, ctypes.POINTER(PermEstimate)]),
        "perm_approx_rasmussen_sparse_range": (i, [_P, i, _P, _P, i64, i64, u64, _P, ctypes.POINTER(PermEstimate)]),
        "perm_approx_scaling_sparse_range": (i, [_P, i, _P, _P, i64, i64, i, i, u64, _P,
                                                 ctypes.POINTER(PermEstimate)]),
        "perm_approx_rasmussen_sparse": (i, [_P, i, _P, _P, i64, u64, _P, ctypes.POINTER(PermEstimate)]),
        "perm_approx_scaling_sparse": (i, [_P, i, _P, _P, _P, _P, i64, i, i, u64, _P,
                                           ctypes.POINTER(PermEstimate)]),
        "perm_read_matrix": (i, [ctypes.c_char_p, i, i, _P, ctypes.POINTER(i), ctypes.POINTER(i),
                                 ctypes.c_char_p]),
        "perm_compress": (i, [i, _P, i, _P, _P, _P, _P, _P, _P]),
        "perm_grid_graph": (i, [i, i, i, _P, ctypes.POINTER(i)]),
        "perm_fp64_peak": (i, [_P, ctypes.POINTER(d), ctypes.POINTER(d)]),
        "perm_batch_create": (i, [_P, i, _P, _P, ctypes.POINTER(_P)]),
        "perm_batch_run": (i, [_P, _P, _P, ctypes.POINTER(d)]),
        "perm_batch_run_ex": (i, [_P, _P, _P, _P, ctypes.POINTER(i), ctypes.POINTER(d)]),
        "perm_batch_destroy": (None, [_P, _P]),
        "perm_batch_exact": (i, [_P, i, _P, _P, _P, ctypes.POINTER(d)]),
        "perm_batch_autotune": (i, [_P, i, i, _P]),
        "perm_batch_variant": (i, [_P, _P, _P, _P, _P, _P]),
        "perm_batch_use_variant": (i, [_P, i]),
        "perm_dense_autotune": (i, [_P, i, i, _P]),
        "perm_ctx_set_rel_target": (i, [_P, d]),
        "perm_ctx_inject_wait_timeout": (i, [_P, i]),
        "perm_server_create": (i, [i, i, ctypes.c_size_t, u64, ctypes.POINTER(_P)]),
        "perm_server_submit": (i, [_P, ctypes.POINTER(PermRequest), ctypes.POINTER(u64)]),
        "perm_server_wait": (i, [_P, u64, i, ctypes.POINTER(PermResponse)]),
        "perm_server_stats": (i, [_P, _P]),
        "perm_server_destroy": (None, [_P]),
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
    abs_term_sum: float = 0.0
    rel_error_estimate: float = 0.0


@dataclass
class Estimate:
    mean: float
    std_error: float
    trials: float
    zero_trials: float
    kernel_ms: float
    trial_values: np.ndarray | None = None
    sum: float = 0.0      # sum of the trial weights (mean = sum / trials)
    sum_sq: float = 0.0   # sum of their squares


def _exact(r: PermResult) -> ExactResult:
    return ExactResult(r.value, r.hi, r.lo, r.steps, r.total_steps, r.kernel_ms, r.kernel, r.n, r.abs_term_sum,
                       r.rel_error_estimate)


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
        """Dense Ryser; variant 0 = automatic, PERM_KERNEL_DENSE = FP64 X, PERM_KERNEL_DENSE_INT = int32 X,
        PERM_KERNEL_DENSE_TC = tensor-core row sums, PERM_KERNEL_DENSE_DD = double-double,
        PERM_KERNEL_DENSE_SPLIT = split X (exact coarse row sums, orders 4..40),
        PERM_KERNEL_DENSE_INT_DD / PERM_KERNEL_DENSE_SDD = the certified int32-X /
        split-dd walks."""
        a, dt = _as_matrix(mat)
        r = PermResult()
        if variant:
            self._check(self.lib.perm_exact_dense_ex(self.ctx, _ptr(a), a.shape[0], dt, variant, 0, 1,
                                                     ctypes.byref(r)))
        else:
            self._check(self.lib.perm_exact_dense(self.ctx, _ptr(a), a.shape[0], dt, ctypes.byref(r)))
        return _exact(r)

    def dense_plan(self, mat) -> tuple[int, float]:
        """(kernel, predicted FP64-X bound) the accuracy policy starts a
        whole-walk call with (perm_exact_dense_plan): PERM_KERNEL_DENSE_INT_DD
        or PERM_KERNEL_DENSE_SDD when a certified walk is the whole
        evaluation, 0 when the FP64-X / int32-X walk goes first; the bound is
        0 where no prediction ran."""
        a, dt = _as_matrix(mat)
        k, b = ctypes.c_int(0), ctypes.c_double(0.0)
        self._check(self.lib.perm_exact_dense_plan(self.ctx, _ptr(a), a.shape[0], dt, ctypes.byref(k), ctypes.byref(b)))
        return k.value, b.value

    def refine_dense(self, mat, hi: float, lo: float, kernel_ms: float = 0.0) -> ExactResult:
        """Accuracy policy and error estimate for a whole-walk value assembled
        from shards (perm_exact_dense_refine)."""
        a, dt = _as_matrix(mat)
        r = PermResult()
        r.hi, r.lo, r.kernel_ms = hi, lo, kernel_ms
        self._check(self.lib.perm_exact_dense_refine(self.ctx, _ptr(a), a.shape[0], dt, ctypes.byref(r)))
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

    def exact_dense_tc_rounds(self, mat, round0: int, nrounds: int) -> ExactResult:
        """Tensor-core kernel over a range of its rounds (partial, scaled sum)."""
        a, dt = _as_matrix(mat)
        r = PermResult()
        self._check(self.lib.perm_exact_dense_tc_rounds(self.ctx, _ptr(a), a.shape[0], dt, round0, nrounds,
                                                        ctypes.byref(r)))
        return _exact(r)

    def upload_dense(self, mat, variant: int = 0) -> "ResidentMatrix":
        a, dt = _as_matrix(mat)
        h = _P()
        self._check(self.lib.perm_matrix_create_dense_ex(self.ctx, _ptr(a), a.shape[0], dt, variant,
                                                         ctypes.byref(h)))
        return ResidentMatrix(self, h, a.shape[0])

    # ---- Monte Carlo ----
    def _estimate(self, e: PermEstimate, tv) -> Estimate:
        return Estimate(e.mean, e.std_error, e.trials, e.zero_trials, e.kernel_ms, tv, e.sum, e.sum_sq)

    def rasmussen(self, mat, trials: int, seed: int = 1, keep_trials: bool = False, trial0: int = 0) -> Estimate:
        """Rasmussen estimate over trials [trial0, trial0 + trials) of the
        streams keyed by `seed` (trial0 > 0: perm_approx_rasmussen_range)."""
        a, dt = _as_matrix(mat)
        tv = np.empty(trials, dtype=np.float64) if keep_trials else None
        e = PermEstimate()
        if trial0:
            self._check(self.lib.perm_approx_rasmussen_range(self.ctx, _ptr(a), a.shape[0], dt, trial0, trials, seed,
                                                             _ptr(tv), ctypes.byref(e)))
        else:
            self._check(self.lib.perm_approx_rasmussen(self.ctx, _ptr(a), a.shape[0], dt, trials, seed, _ptr(tv),
                                                       ctypes.byref(e)))
        return self._estimate(e, tv)

    def scaling(self, mat, trials: int, scale_intervals: int = 4, scale_times: int = 5, seed: int = 1,
                keep_trials: bool = False, trial0: int = 0) -> Estimate:
        """Sinkhorn-scaled estimate over trials [trial0, trial0 + trials)
        (trial0 > 0: perm_approx_scaling_range)."""
        a, dt = _as_matrix(mat)
        tv = np.empty(trials, dtype=np.float64) if keep_trials else None
        e = PermEstimate()
        if trial0:
            self._check(self.lib.perm_approx_scaling_range(self.ctx, _ptr(a), a.shape[0], dt, trial0, trials,
                                                           scale_intervals, scale_times, seed, _ptr(tv),
                                                           ctypes.byref(e)))
        else:
            self._check(self.lib.perm_approx_scaling(self.ctx, _ptr(a), a.shape[0], dt, trials, scale_intervals,
                                                     scale_times, seed, _ptr(tv), ctypes.byref(e)))
        return self._estimate(e, tv)

    def rasmussen_sparse(self, n, rptrs, cols, trials, seed=1, keep_trials=False, trial0: int = 0) -> Estimate:
        rp = np.ascontiguousarray(rptrs, dtype=np.int32)
        cl = np.ascontiguousarray(cols, dtype=np.int32)
        tv = np.empty(trials, dtype=np.float64) if keep_trials else None
        e = PermEstimate()
        if trial0:
            self._check(self.lib.perm_approx_rasmussen_sparse_range(self.ctx, n, _ptr(rp), _ptr(cl), trial0, trials,
                                                                    seed, _ptr(tv), ctypes.byref(e)))
        else:
            self._check(self.lib.perm_approx_rasmussen_sparse(self.ctx, n, _ptr(rp), _ptr(cl), trials, seed,
                                                              _ptr(tv), ctypes.byref(e)))
        return self._estimate(e, tv)

    def scaling_sparse(self, n, rptrs, cols, cptrs, rows, trials, scale_intervals=4, scale_times=5, seed=1,
                       keep_trials=False, trial0: int = 0) -> Estimate:
        arrs = [np.ascontiguousarray(x, dtype=np.int32) for x in (rptrs, cols, cptrs, rows)]
        tv = np.empty(trials, dtype=np.float64) if keep_trials else None
        e = PermEstimate()
        if trial0:
            self._check(self.lib.perm_approx_scaling_sparse_range(self.ctx, n, _ptr(arrs[0]), _ptr(arrs[1]), trial0,
                                                                  trials, scale_intervals, scale_times, seed,
                                                                  _ptr(tv), ctypes.byref(e)))
        else:
            self._check(self.lib.perm_approx_scaling_sparse(self.ctx, n, *map(_ptr, arrs), trials, scale_intervals,
                                                            scale_times, seed, _ptr(tv), ctypes.byref(e)))
        return self._estimate(e, tv)

    # ---- batches ----
    def batch(self, mats) -> "Batch":
        """Upload a list of square matrices (orders 1..40) as one resident batch."""
        orders = np.array([np.asarray(m).shape[0] for m in mats], dtype=np.int32)
        vals = np.ascontiguousarray(np.concatenate([np.asarray(m, dtype=np.float64).ravel() for m in mats]))
        h = _P()
        self._check(self.lib.perm_batch_create(self.ctx, len(mats), _ptr(orders), _ptr(vals), ctypes.byref(h)))
        return Batch(self, h, len(mats))

    def batch_exact(self, mats) -> tuple[np.ndarray, float]:
        b = self.batch(mats)
        try:
            return b.run()
        finally:
            b.free()

    def batch_autotune(self, n_lo: int, n_hi: int) -> dict:
        """Per-order lane-range exponents (and, kept in the context, the
        fastest batch kernel variant: see batch_variant())."""
        out = np.zeros(n_hi - n_lo + 1, dtype=np.int32)
        self._check(self.lib.perm_batch_autotune(self.ctx, n_lo, n_hi, _ptr(out)))
        return {n_lo + i: int(m) for i, m in enumerate(out)}

    def batch_use_variant(self, variant: int):
        """Later batches run kernel variant `variant` (perm_batch_use_variant)."""
        self._check(self.lib.perm_batch_use_variant(self.ctx, variant))

    def batch_variant(self) -> dict:
        """The batch kernel variant later batches use (perm_batch_variant)."""
        v = np.zeros(5, dtype=np.int32)
        self._check(self.lib.perm_batch_variant(self.ctx, *[_ptr(v[i:i + 1]) for i in range(5)]))
        return {"variant": int(v[0]), "max_order": int(v[1]), "threads_per_block": int(v[2]),
                "ctas_per_sm_compiled_for": int(v[3]), "shared_memory_x": bool(v[4])}

    def set_rel_target(self, target: float):
        """Relative-error target of the automatic dense path's accuracy policy
        (exact zeros, transpose cross-check, double-double); 0 keeps the
        estimate without the policy, < 0 skips the estimate too."""
        self._check(self.lib.perm_ctx_set_rel_target(self.ctx, target))

    def inject_wait_timeout(self, launches: int = 1):
        """Failure injection for tests (perm_ctx_inject_wait_timeout): the next
        `launches` FP64-X or tensor-core dense launches wait on a barrier that
        never completes, give up after their bounded wait and fail with
        PERM_ETIMEOUT; the context stays usable."""
        self._check(self.lib.perm_ctx_inject_wait_timeout(self.ctx, launches))

    def dense_autotune(self, n_lo: int, n_hi: int) -> dict:
        """Per order: which register kernel the automatic choice uses for integer inputs."""
        out = np.zeros(n_hi - n_lo + 1, dtype=np.int32)
        self._check(self.lib.perm_dense_autotune(self.ctx, n_lo, n_hi, _ptr(out)))
        return {n_lo + i: int(k) for i, k in enumerate(out)}

    def fp64_peak(self) -> tuple[float, float]:
        ops, ms = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.perm_fp64_peak(self.ctx, ctypes.byref(ops), ctypes.byref(ms)))
        return ops.value, ms.value


class Batch:
    """A resident batch; run() replays its captured CUDA graph."""

    def __init__(self, engine: Engine, handle, count: int):
        self.engine, self.handle, self.count = engine, handle, count

    def run(self) -> tuple[np.ndarray, float]:
        """Returns (values, device ms) of one graph replay; values[i] = hi + lo
        of matrix i (plain FP64-X walk, no accuracy policy)."""
        res = np.zeros(2 * self.count, dtype=np.float64)
        ms = ctypes.c_double()
        self.engine._check(self.engine.lib.perm_batch_run(self.engine.ctx, self.handle, _ptr(res),
                                                          ctypes.byref(ms)))
        return res[0::2] + res[1::2], ms.value

    def run_ex(self) -> tuple[np.ndarray, np.ndarray, int, float]:
        """(values, relative-error estimates, matrices re-evaluated by the
        accuracy policy, device ms of the graph plus those re-evaluations)."""
        res = np.zeros(2 * self.count, dtype=np.float64)
        est = np.zeros(self.count, dtype=np.float64)
        ms = ctypes.c_double()
        reruns = ctypes.c_int()
        self.engine._check(self.engine.lib.perm_batch_run_ex(self.engine.ctx, self.handle, _ptr(res), _ptr(est),
                                                             ctypes.byref(reruns), ctypes.byref(ms)))
        return res[0::2] + res[1::2], est, reruns.value, ms.value

    def free(self):
        if self.handle:
            self.engine.lib.perm_batch_destroy(self.engine.ctx, self.handle)
            self.handle = None


class ResidentMatrix:
    """A dense matrix kept in device memory; run() launches with no host copy."""

    def __init__(self, engine: Engine, handle, n: int):
        self.engine, self.handle, self.n = engine, handle, n

    def run(self) -> ExactResult:
        r = PermResult()
        self.engine._check(self.engine.lib.perm_exact_dense_resident(self.engine.ctx, self.handle,
                                                                     ctypes.byref(r)))
        return _exact(r)

    def run_shard(self, shard: int, nshards: int) -> ExactResult:
        """Shard `shard` of `nshards` of the walk (perm_exact_dense_resident_shard)."""
        r = PermResult()
        self.engine._check(self.engine.lib.perm_exact_dense_resident_shard(self.engine.ctx, self.handle, shard,
                                                                           nshards, ctypes.byref(r)))
        return _exact(r)

    def free(self):
        if self.handle:
            self.engine.lib.perm_matrix_destroy(self.engine.ctx, self.handle)
            self.handle = None


class Server:
    """Request loop on one GPU (continuous batching over `slots` contexts)."""

    def __init__(self, device: int = 0, slots: int = 4, memory_budget: int = 0, slice_steps: int = 0, lib_path=None):
        self.lib = load_library(lib_path)
        h = _P()
        rc = self.lib.perm_server_create(device, slots, memory_budget, slice_steps, ctypes.byref(h))
        if rc != PERM_OK:
            raise PermError(rc, f"cannot create a server on device {device}")
        self.handle = h

    def submit(self, kind: int, mat, trials: int = 0, scale_intervals: int = 4, scale_times: int = 5,
               seed: int = 1) -> int:
        a = np.ascontiguousarray(mat, dtype=np.float64)
        req = PermRequest(kind, a.shape[0], a.ctypes.data, trials, scale_intervals, scale_times, seed)
        t = ctypes.c_uint64()
        rc = self.lib.perm_server_submit(self.handle, ctypes.byref(req), ctypes.byref(t))
        if rc != PERM_OK:
            raise PermError(rc, "submit failed")
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1) -> dict:
        r = PermResponse()
        rc = self.lib.perm_server_wait(self.handle, ticket, timeout_ms, ctypes.byref(r))
        if rc != PERM_OK:
            raise PermError(rc, f"wait for ticket {ticket} failed")
        return {"status": r.status, "kernel": r.kernel, "value": r.value, "hi": r.hi, "lo": r.lo,
                "std_error": r.std_error, "t_submit_ms": r.t_submit_ms, "t_admit_ms": r.t_admit_ms,
                "t_done_ms": r.t_done_ms, "device_ms": r.device_ms, "message": r.message.decode(errors="replace")}

    def stats(self) -> dict:
        out = np.zeros(5)
        self.lib.perm_server_stats(self.handle, _ptr(out))
        return dict(zip(("submitted", "completed", "in_flight", "queued", "bytes_in_use"), out.tolist()))

    def close(self):
        if getattr(self, "handle", None):
            self.lib.perm_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


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


def grid_graph(m: int, n: int) -> np.ndarray:
    """The reference's grid-graph matrix of an m x n board (util.h:403-520)."""
    lib = load_library()
    nov = m * n // 2
    buf = np.zeros(max(nov, 1) ** 2, dtype=np.float64)
    k = ctypes.c_int()
    rc = lib.perm_grid_graph(m, n, max(nov, 1), _ptr(buf), ctypes.byref(k))
    if rc != PERM_OK:
        raise PermError(rc, f"no grid graph for a {m}x{n} board")
    return buf[: k.value * k.value].reshape(k.value, k.value).copy()


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


def sdd_layout(mat) -> int:
    """Rows the split-dd kernel keeps in registers for this matrix
    (perm_sdd_layout; host only): the sparse layout's inner rows (6 .. 28)
    or the three-level layout's second level (16 .. 28), 0 for the dense
    layout, negative where the kernel does not apply."""
    a = np.ascontiguousarray(mat, dtype=np.float64)
    return int(load_library().perm_sdd_layout(_ptr(a), a.shape[0]))


def sdd_levels(mat) -> tuple[int, int]:
    """(first level R1 of the three-level layout, 0 for the other layouts;
    the sdd_layout value) of the split-dd walk for this matrix
    (perm_sdd_levels; host only); (negative status, 0) where the kernel does
    not apply."""
    a = np.ascontiguousarray(mat, dtype=np.float64)
    lv = np.zeros(2, dtype=np.int32)
    rc = int(load_library().perm_sdd_levels(_ptr(a), a.shape[0], _ptr(lv)))
    return (rc, 0) if rc else (int(lv[0]), int(lv[1]))


def fp64_layout(mat) -> int:
    """Inner rows of the FP64-X walk's two-level row layout for this matrix
    (perm_fp64_layout; host only): 16, 20, 24 or 28, or the second level
    (20..36) of its three-level layout; 0 for one level."""
    a = np.ascontiguousarray(mat, dtype=np.float64)
    return int(load_library().perm_fp64_layout(_ptr(a), a.shape[0]))


def fp64_levels(mat) -> tuple[int, int]:
    """(first level R1 of the FP64-X walk's three-level layout, 0 for the
    other layouts; the fp64_layout value) for this matrix (perm_fp64_levels;
    host only)."""
    a = np.ascontiguousarray(mat, dtype=np.float64)
    lv = np.zeros(2, dtype=np.int32)
    rc = int(load_library().perm_fp64_levels(_ptr(a), a.shape[0], _ptr(lv)))
    return (rc, 0) if rc else (int(lv[0]), int(lv[1]))


def int_layout(mat) -> tuple[int, int, int, int]:
    """(G, outer groups of the two-level layout, first- and second-level
    groups of the three-level layout) of the int32-X walk for this matrix
    (perm_int_layout; host only): all zero beside G for the one-level walk;
    (negative status, 0, 0, 0) where int32 X does not apply."""
    a = np.ascontiguousarray(mat, dtype=np.float64)
    lv = np.zeros(3, dtype=np.int32)
    g = int(load_library().perm_int_layout(_ptr(a), a.shape[0], _ptr(lv)))
    return g, int(lv[0]), int(lv[1]), int(lv[2])


def intc_layout(mat) -> tuple[int, bool, int, int, int]:
    """(G, exact int64 pairing, outer groups of the two-level layout, first-
    and second-level groups of the three-level layout) of the certified
    int32-X walk for this matrix (perm_intc_layout; host only): the last
    three zero for the one-level walk; (negative status, False, 0, 0, 0)
    where the kernel does not apply."""
    a = np.ascontiguousarray(mat, dtype=np.float64)
    pair = ctypes.c_int(0)
    lv = np.zeros(3, dtype=np.int32)
    g = int(load_library().perm_intc_layout(_ptr(a), a.shape[0], ctypes.byref(pair), _ptr(lv)))
    return g, bool(pair.value), int(lv[0]), int(lv[1]), int(lv[2])


def shard_range(n: int, shard: int, nshards: int) -> tuple[int, int]:
    """Gray-index range [first, last) of one shard (host only, device independent)."""
    lib = load_library()
    a, b = ctypes.c_uint64(), ctypes.c_uint64()
    rc = lib.perm_shard_range(n, shard, nshards, ctypes.byref(a), ctypes.byref(b))
    if rc != PERM_OK:
        raise PermError(rc, f"bad shard request n={n} shard={shard}/{nshards}")
    return a.value, b.value


def exact_dense_multi(mat, devices=None, nshards: int | None = None, variant: int = 0) -> ExactResult:
    """One permanent sharded over devices of this process
    (perm_exact_dense_multi; gpu_exact_dense.cu:702): shard s runs on
    devices[s] (default: devices 0 .. nshards-1) in its own host thread, the
    shards' (hi, lo) are added in shard order.  One evaluation, no error
    estimate."""
    a, dtype = _as_matrix(mat)
    n = a.shape[0]
    if devices is not None:
        dev = np.ascontiguousarray(devices, dtype=np.int32)
        nshards = len(dev)
    else:
        dev = None
        nshards = nshards or 1
    r = PermResult()
    rc = load_library().perm_exact_dense_multi(_ptr(a), n, dtype, variant, nshards, _ptr(dev), ctypes.byref(r))
    if rc != PERM_OK:
        raise PermError(rc, f"perm_exact_dense_multi failed for n={n} over {nshards} shards (see stderr)")
    return _exact(r)


def dd_sum(pairs) -> tuple[float, float]:
    """Double-double sum of (hi, lo) pairs in the given order."""
    hi = lo = 0.0
    for h, l in pairs:
        s = hi + h
        bb = s - hi
        lo += ((hi - (s - bb)) + (h - bb)) + l
        hi = s
    s = hi + lo
    return s, lo - (s - hi)


def distributed_exact_dense(mat, group=None, engine: Engine | None = None, shard_fn=None) -> tuple[float, float]:
    """Exact permanent of one matrix over all ranks of a torch.distributed group.

    Rank r computes shard r of world (perm_exact_dense_shard on its own GPU),
    the 16-byte (hi, lo) partials are all-gathered -- the only collective --
    and every rank adds them in rank order (double-double, deterministic).
    `shard_fn(mat, rank, world) -> (hi, lo)` replaces the device call; it
    exists so that the host logic can be exercised without a GPU."""
    import torch
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    if shard_fn is None:
        eng = engine or default_engine()
        r = eng.exact_dense_shard(mat, rank, world)
        part = (r.hi, r.lo)
    else:
        part = shard_fn(mat, rank, world)
    backend = dist.get_backend(group)
    dev = f"cuda:{torch.cuda.current_device()}" if backend == "nccl" else "cpu"
    t = torch.tensor([part[0], part[1]], dtype=torch.float64, device=dev)
    gathered = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(gathered, t, group=group)
    return dd_sum((float(g[0]), float(g[1])) for g in gathered)


# calls of distributed_exact_dense_dynamic so far, per process group (keyed
# by its sorted global ranks): every member makes the same calls in the same
# order, so (group, call number) names one queue on all of them
_queue_calls: dict[tuple[int, ...], int] = {}


def distributed_exact_dense_dynamic(mat, chunks: int | None = None, group=None, engine: Engine | None = None,
                                    shard_fn=None, store=None, claims_out: list | None = None
                                    ) -> tuple[float, float]:
    """Exact permanent of one matrix over all ranks with a dynamic chunk queue
    (the reference's hybrid multi-GPU chunk queue, gpu_exact_dense.cu:777-904,
    restated over torch.distributed ranks instead of host threads).

    The Gray walk is cut into `chunks` device-independent shards
    (perm_shard_range; default 8 per rank).  Each rank repeatedly claims the
    next chunk from an atomic counter in the process group's key-value store
    (`store`, default: the group's rendezvous store) and runs it on its own
    GPU, so faster or less loaded GPUs take more chunks.  One all-reduce of a
    chunks x 3 table (claimed flag, hi, lo; each row written by exactly one
    rank, so the sum is exact) gives every rank all partials, which are added
    in chunk order (double-double): the result does not depend on who ran
    what.  `shard_fn(mat, chunk, chunks) -> (hi, lo)` replaces the device
    call (host-logic tests without a GPU); `claims_out` receives this rank's
    chunk ids."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    chunks = chunks or 8 * world
    if store is None:
        store = dist.distributed_c10d._get_default_store()
    members = tuple(sorted(dist.get_process_group_ranks(group if group is not None else dist.group.WORLD)))
    call = _queue_calls.get(members, 0)
    _queue_calls[members] = call + 1
    # the key names the group and the call, so concurrent subgroups and later
    # world calls never share a counter
    key = f"perm_b200_queue_{'-'.join(map(str, members))}_{call}"
    eng = None if shard_fn is not None else (engine or default_engine())
    table = torch.zeros((chunks, 3), dtype=torch.float64)
    while True:
        c = int(store.add(key, 1)) - 1
        if c >= chunks:
            break
        if shard_fn is None:
            r = eng.exact_dense_shard(mat, c, chunks)
            hi, lo = r.hi, r.lo
        else:
            hi, lo = shard_fn(mat, c, chunks)
        table[c, 0], table[c, 1], table[c, 2] = 1.0, hi, lo
        if claims_out is not None:
            claims_out.append(c)
    backend = dist.get_backend(group)
    if backend == "nccl":
        table = table.to(f"cuda:{torch.cuda.current_device()}")
    dist.all_reduce(table, op=dist.ReduceOp.SUM, group=group)
    table = table.cpu()
    if not bool((table[:, 0] == 1.0).all()):
        raise PermError(PERM_EINVAL, "chunk queue: a chunk was not computed exactly once")
    return dd_sum((float(table[c, 1]), float(table[c, 2])) for c in range(chunks))


CHECKPOINT_FORMAT = "perm_b200_checkpoint_v1"


def _fingerprint(a: np.ndarray) -> str:
    import hashlib

    h = hashlib.sha256()
    h.update(f"{a.shape[0]}:{a.dtype.str}:".encode())
    h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def _read_checkpoint(path, fingerprint: str, n: int, chunks: int, variant: int) -> dict[int, tuple[float, float]]:
    import json

    try:
        with open(path) as f:
            state = json.load(f)
    except FileNotFoundError:
        return {}
    except (OSError, ValueError) as e:
        raise PermError(PERM_EIO, f"checkpoint {path} is unreadable ({e}); remove it to start over") from e
    want = {"format": CHECKPOINT_FORMAT, "matrix_sha256": fingerprint, "n": n, "chunks": chunks,
            "variant": variant}
    for k, v in want.items():
        if state.get(k) != v:
            raise PermError(PERM_EINVAL, f"checkpoint {path} belongs to another run ({k}: {state.get(k)!r}, "
                                         f"this run: {v!r}); remove it or pass another path")
    done = {}
    try:
        for key, (h, l) in state.get("done", {}).items():
            c = int(key)
            if not 0 <= c < chunks:
                raise PermError(PERM_EINVAL, f"checkpoint {path}: chunk {c} outside [0, {chunks})")
            done[c] = (float.fromhex(h), float.fromhex(l))
    except (AttributeError, TypeError, ValueError) as e:
        raise PermError(PERM_EIO, f"checkpoint {path} is unreadable ({e}); remove it to start over") from e
    return done


def _write_checkpoint(path, fingerprint: str, n: int, chunks: int, variant: int,
                      done: dict[int, tuple[float, float]]) -> None:
    import json

    state = {"format": CHECKPOINT_FORMAT, "matrix_sha256": fingerprint, "n": n, "chunks": chunks,
             "variant": variant,
             "done": {str(c): [h.hex(), l.hex()] for c, (h, l) in sorted(done.items())}}
    tmp = f"{path}.tmp"
    with open(tmp, "w") as f:
        json.dump(state, f)
        f.flush()
        os.fsync(f.fileno())
    os.replace(tmp, path)  # atomic: a crash leaves the old file or the new one, never half of one


def checkpointed_exact_dense(mat, path, chunks: int = 64, variant: int = 0, engine: Engine | None = None,
                             shard_fn=None, keep: bool = False) -> tuple[float, float]:
    """Exact permanent of one long walk that survives interruption
    (checkpoint / resume; the reference has none: a killed run starts over).

    The Gray walk is cut into `chunks` device-independent shards
    (perm_shard_range) and walked one after another with
    perm_exact_dense_ex(variant) on `engine` (default: the process default
    engine).  After every shard the checkpoint file `path` is rewritten
    atomically (temporary file, fsync, rename) with the matrix fingerprint
    (order, dtype, SHA-256 of the values), the chunk count, the variant and
    the exact bits of every finished shard's (hi, lo).  A later call with
    the same matrix, chunks and variant resumes: it walks only the shards the
    file lacks.  The shards are added in chunk order in double-double, so an
    interrupted and resumed run returns the uninterrupted run's value bit
    for bit.  A file written for another matrix, chunk count or variant is
    refused (PermError) instead of being mixed in.  The file is removed
    after success unless `keep`.  One process at a time per file: two runs
    sharing a path would overwrite each other's progress.  One evaluation, like the shard API: pass
    the sum to Engine.refine_dense for the accuracy policy.  `shard_fn(mat,
    chunk, chunks) -> (hi, lo)` replaces the device call (host-logic tests
    without a GPU)."""
    a = np.ascontiguousarray(np.asarray(mat, dtype=np.float64))
    if a.ndim != 2 or a.shape[0] != a.shape[1]:
        raise PermError(PERM_EINVAL, f"need a square matrix, got shape {a.shape}")
    n = a.shape[0]
    if not 1 <= chunks <= (1 << 20):
        raise PermError(PERM_EINVAL, f"chunks must be in [1, 2^20], got {chunks}")
    fp = _fingerprint(a)
    done = _read_checkpoint(path, fp, n, chunks, variant)
    eng = None if shard_fn is not None else (engine or default_engine())
    for c in range(chunks):
        if c in done:
            continue
        if shard_fn is None:
            r = eng.exact_dense_shard(a, c, chunks, variant=variant)
            done[c] = (r.hi, r.lo)
        else:
            hi, lo = shard_fn(a, c, chunks)
            done[c] = (float(hi), float(lo))
        _write_checkpoint(path, fp, n, chunks, variant, done)
    result = dd_sum(done[c] for c in range(chunks))
    if not keep:
        try:
            os.remove(path)
        except FileNotFoundError:
            pass
    return result


def _gather_rows(row, group):
    """All-gather of one float64 row per rank (rank order), on the device for
    NCCL groups and on the host for gloo."""
    import torch
    import torch.distributed as dist

    backend = dist.get_backend(group)
    dev = f"cuda:{torch.cuda.current_device()}" if backend == "nccl" else "cpu"
    t = torch.tensor(row, dtype=torch.float64, device=dev)
    out = [torch.zeros_like(t) for _ in range(dist.get_world_size(group))]
    dist.all_gather(out, t, group=group)
    return [g.cpu().numpy() for g in out]


def distributed_estimate(mat, trials: int, method: str = "rasmussen", scale_intervals: int = 4,
                         scale_times: int = 5, seed: int = 1, group=None, engine: Engine | None = None,
                         range_fn=None) -> Estimate:
    """Monte-Carlo estimate of one matrix over all ranks of a torch.distributed
    group, split by trial id (the reference's multi-GPU estimators,
    gpu_approximation_dense.cu:412, 574, with static ranges instead of its
    chunk queue: trials cost alike).

    Rank r runs trials [r T / W, (r + 1) T / W) of the streams keyed by `seed`
    (perm_approx_*_range), so the union of the ranks' trials is exactly the
    single-device run's; one all-gather of (sum, sum of squares, zero trials,
    device ms) per rank -- the only collective -- and every rank adds them in
    rank order.  `range_fn(mat, trial0, count) -> (sum, sum_sq, zeros)`
    replaces the device call (host-logic tests without a GPU)."""
    import torch.distributed as dist

    if trials < 1:
        raise PermError(PERM_EINVAL, f"trials must be >= 1 (got {trials})")
    if method not in ("rasmussen", "scaling"):
        raise PermError(PERM_EINVAL, f"unknown estimator {method!r}")
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    t0, t1 = trials * rank // world, trials * (rank + 1) // world
    row = [0.0, 0.0, 0.0, 0.0]
    if t1 > t0:
        if range_fn is not None:
            s, s2, z = range_fn(mat, t0, t1 - t0)
            row = [s, s2, z, 0.0]
        else:
            eng = engine or default_engine()
            if method == "rasmussen":
                e = eng.rasmussen(mat, t1 - t0, seed=seed, trial0=t0)
            else:
                e = eng.scaling(mat, t1 - t0, scale_intervals, scale_times, seed=seed, trial0=t0)
            row = [e.sum, e.sum_sq, e.zero_trials, e.kernel_ms]
    rows = _gather_rows(row, group)
    s = s2 = z = 0.0
    ms = 0.0
    for g in rows:
        s += float(g[0])
        s2 += float(g[1])
        z += float(g[2])
        ms = max(ms, float(g[3]))
    T = float(trials)
    mean = s / T
    var = (s2 - s * mean) / (T - 1) if T > 1 else 0.0
    return Estimate(mean, math.sqrt(max(var, 0.0) / T), T, z, ms, None, s, s2)


def batch_assignment(orders, world: int) -> list[int]:
    """Owner rank of every matrix of a batch split over `world` ranks: longest
    walk first to the least-loaded rank (cost 2^(n-1) Gray steps; ties to the
    lower index and rank), the same on every rank."""
    load = [0.0] * world
    owner = [0] * len(orders)
    for i in sorted(range(len(orders)), key=lambda i: (-int(orders[i]), i)):
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += 2.0 ** (int(orders[i]) - 1)
    return owner


def distributed_batch_exact(mats, group=None, engine: Engine | None = None, batch_fn=None) -> np.ndarray:
    """Exact permanents of a list of matrices over all ranks: each rank runs
    one resident batch (perm_batch_*) of the matrices batch_assignment gives
    it, and one all-reduce of a count x 2 table (owner flag, value; every row
    written by exactly one rank, so the sum is exact) gives every rank all
    values, in the caller's order.  `batch_fn(list_of_matrices) -> values`
    replaces the device call (host-logic tests without a GPU)."""
    import torch
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    orders = [np.asarray(m).shape[0] for m in mats]
    owner = batch_assignment(orders, world)
    mine = [i for i in range(len(mats)) if owner[i] == rank]
    table = torch.zeros((len(mats), 2), dtype=torch.float64)
    if mine:
        sub = [mats[i] for i in mine]
        vals = batch_fn(sub) if batch_fn is not None else (engine or default_engine()).batch_exact(sub)[0]
        for i, v in zip(mine, vals):
            table[i, 0], table[i, 1] = 1.0, float(v)
    if dist.get_backend(group) == "nccl":
        table = table.to(f"cuda:{torch.cuda.current_device()}")
    dist.all_reduce(table, op=dist.ReduceOp.SUM, group=group)
    table = table.cpu()
    if not bool((table[:, 0] == 1.0).all()):
        raise PermError(PERM_EINVAL, "batch split: a matrix was not computed exactly once")
    return table[:, 1].numpy().copy()


# ---- reference-named entry points (argument meaning as in the reference) ------
_default_engine: Engine | None = None


def default_engine() -> Engine:
    """Engine of the reference-named functions below.  Like the reference they
    evaluate once (no error estimate, no accuracy policy) unless
    PERM_REL_TARGET sets a target; PERM_DEVICE picks the device."""
    global _default_engine
    if _default_engine is None:
        _default_engine = Engine(int(os.environ.get("PERM_DEVICE", "0")))
        _default_engine.set_rel_target(float(os.environ.get("PERM_REL_TARGET", "-1")))
    return _default_engine


def gpu_perman64_xshared_coalescing_mshared(mat, nov: int | None = None, grid_dim: int = 2048,
                                            block_dim: int = 256) -> float:
    """Dense exact permanent (gpu_exact_dense.cu:641); grid/block are ignored."""
    a = np.asarray(mat)
    if nov is not None and nov != a.shape[0]:
        a = a.reshape(nov, nov)
    return default_engine().exact_dense(a).value


def gpu_perman64_xshared_coalescing_mshared_multigpu(mat, nov: int | None = None, gpu_num: int = 2,
                                                     grid_dim: int = 2048, block_dim: int = 256) -> float:
    """Dense exact permanent over devices 0 .. gpu_num - 1 of this process
    (gpu_exact_dense.cu:702; at most the visible devices): one shard per
    device through perm_exact_dense_multi, one evaluation; grid/block are
    ignored."""
    a = np.asarray(mat)
    if nov is not None and nov != a.shape[0]:
        a = a.reshape(nov, nov)
    avail = int(load_library().perm_device_count())
    if avail < 1:
        raise PermError(PERM_ECUDA, "no CUDA device")
    return exact_dense_multi(a, nshards=max(1, min(gpu_num, avail))).value


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
