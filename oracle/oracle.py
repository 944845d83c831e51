"""ctypes binding of the oracle -- TEST INFRASTRUCTURE ONLY.

liboracle.so is the CPU restatement of the reference's algorithms
(oracle/oracle.c); libperman_ref.so is the reference itself, compiled from its
own sources by oracle/build_ref.sh.  Only tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / --impl reference legs import this module; the
product library never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libperman_ref.so"
_P = ctypes.c_void_p


def build_oracle() -> Path:
    """Compile liboracle.so (gcc) if it is missing or older than its source."""
    src = HERE / "oracle.c"
    if not ORACLE_SO.exists() or ORACLE_SO.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), "liboracle.so"], check=True, capture_output=True)
    return ORACLE_SO


def reference_sources() -> Path:
    """Where the reference's sources are read from: $REF_SRC, else a
    `reference` directory beside this repository."""
    return Path(os.environ.get("REF_SRC", HERE.parents[1] / "reference"))


def build_reference() -> Path | None:
    """Compile the reference into oracle/_ref when its sources are present."""
    if not (reference_sources() / "main.cu").exists():
        return REF_SO if REF_SO.exists() else None
    if not REF_SO.exists():
        subprocess.run([str(HERE / "build_ref.sh")], check=True, capture_output=True)
    return REF_SO


def _ptr(a):
    return a.ctypes.data_as(_P)


class Oracle:
    def __init__(self):
        self.lib = ctypes.CDLL(str(build_oracle()))
        L = self.lib
        i, d, i64, u64 = ctypes.c_int, ctypes.c_double, ctypes.c_int64, ctypes.c_uint64
        L.orc_ryser_dd_range.argtypes = [_P, i, i64, i64, i, _P]
        L.orc_perm_dd.argtypes = [_P, i, i, _P]
        L.orc_perm_q.argtypes = [_P, i, i, _P]
        L.orc_perm_dp.argtypes = [_P, i, _P]
        L.orc_perm_exact_int.argtypes = [_P, i, i, ctypes.c_char_p, i, ctypes.POINTER(d)]
        L.orc_skipper.argtypes = [_P, _P, _P, _P, _P, _P, i, i, i, ctypes.POINTER(d)]
        L.orc_skipper.restype = d
        L.orc_philox4x32_10.argtypes = [_P, _P, _P]
        L.orc_rasmussen_trials.argtypes = [_P, i, u64, i64, i64, _P]
        L.orc_scaling_trials.argtypes = [_P, i, i, i, u64, i64, i64, _P]
        L.orc_rasmussen_sparse_trials.argtypes = [_P, _P, _P, _P, i, u64, i64, i64, _P]
        L.orc_scaling_sparse_trials.argtypes = [_P, _P, _P, _P, i, i, i, u64, i64, i64, _P]
        L.orc_grid_graph.argtypes = [i, i, _P, i]

    @staticmethod
    def _mat(a):
        return np.ascontiguousarray(a, dtype=np.float64)

    def perm_dd(self, a, threads: int = os.cpu_count() or 1) -> tuple[float, float]:
        a = self._mat(a)
        out = np.zeros(2)
        self.lib.orc_perm_dd(_ptr(a), a.shape[0], threads, _ptr(out))
        return float(out[0]), float(out[1])

    def ryser_dd_range(self, a, i0: int, i1: int, threads: int = os.cpu_count() or 1) -> tuple[float, float]:
        a = self._mat(a)
        out = np.zeros(2)
        self.lib.orc_ryser_dd_range(_ptr(a), a.shape[0], i0, i1, threads, _ptr(out))
        return float(out[0]), float(out[1])

    def perm_q(self, a, threads: int = os.cpu_count() or 1) -> tuple[float, float]:
        a = self._mat(a)
        out = np.zeros(2)
        self.lib.orc_perm_q(_ptr(a), a.shape[0], threads, _ptr(out))
        return float(out[0]), float(out[1])

    def perm_dp(self, a) -> tuple[float, float]:
        a = self._mat(a)
        out = np.zeros(2)
        self.lib.orc_perm_dp(_ptr(a), a.shape[0], _ptr(out))
        return float(out[0]), float(out[1])

    def perm_exact_int(self, a, threads: int = os.cpu_count() or 1) -> tuple[int, float]:
        a = np.ascontiguousarray(a, dtype=np.int64)
        buf = ctypes.create_string_buffer(1024)
        approx = ctypes.c_double()
        rc = self.lib.orc_perm_exact_int(_ptr(a), a.shape[0], threads, buf, 1024, ctypes.byref(approx))
        if rc != 0:
            raise RuntimeError(f"orc_perm_exact_int failed ({rc})")
        return int(buf.value.decode()), approx.value

    def skipper(self, c: dict, chunks: int = 512, threads: int = os.cpu_count() or 1) -> tuple[float, float]:
        vis = ctypes.c_double()
        arrs = {k: np.ascontiguousarray(c[k], dtype=np.int32) for k in ("rptrs", "cols", "cptrs", "rows")}
        rv = np.ascontiguousarray(c["rvals"], dtype=np.float64)
        cv = np.ascontiguousarray(c["cvals"], dtype=np.float64)
        v = self.lib.orc_skipper(_ptr(arrs["rptrs"]), _ptr(arrs["cols"]), _ptr(rv), _ptr(arrs["cptrs"]),
                                 _ptr(arrs["rows"]), _ptr(cv), c["n"], chunks, threads, ctypes.byref(vis))
        return v, vis.value

    def philox(self, ctr, key) -> list[int]:
        c = np.array(ctr, dtype=np.uint32)
        k = np.array(key, dtype=np.uint32)
        o = np.zeros(4, dtype=np.uint32)
        self.lib.orc_philox4x32_10(_ptr(c), _ptr(k), _ptr(o))
        return [int(x) for x in o]

    def rasmussen_trials(self, a, seed: int, t0: int, count: int) -> np.ndarray:
        a = self._mat(a)
        out = np.zeros(count)
        self.lib.orc_rasmussen_trials(_ptr(a), a.shape[0], seed, t0, count, _ptr(out))
        return out

    def scaling_trials(self, a, y: int, z: int, seed: int, t0: int, count: int) -> np.ndarray:
        a = self._mat(a)
        out = np.zeros(count)
        self.lib.orc_scaling_trials(_ptr(a), a.shape[0], y, z, seed, t0, count, _ptr(out))
        return out


def tc_rounds_sum(a, round0: int, nrounds: int):
    """Exact (fractions.Fraction) partial Ryser sum over the subsets that the
    tensor-core kernel assigns to rounds [round0, round0 + nrounds): every
    choice of columns 0 .. 8 and the remaining columns 9 .. n - 2 by the Gray
    code of the round index, each term (-1)^|S| prod_j y_j(S) with y = 2x (the
    Nijenhuis-Wilf form of the reference's Ryser sum, gpu_exact_dense.cu:
    330-399), scaled by (4(n&1) - 2) / 2^n like the whole sum.  Returns
    (sum, sum of |terms|), both scaled.  Pure-Python integers: small round
    counts only."""
    from fractions import Fraction
    a = np.asarray(a, dtype=np.int64)
    n = a.shape[0]
    low = 9
    rb = n - 1 - low
    cols = [[2 * int(a[j, k]) for j in range(n)] for k in range(n)]
    y0 = [2 * int(a[j, n - 1]) - int(a[j].sum()) for j in range(n)]
    total = abs_total = 0
    for r in range(round0, round0 + nrounds):
        g = r ^ (r >> 1)
        base = list(y0)
        for k in range(rb):
            if (g >> k) & 1:
                base = [b + c for b, c in zip(base, cols[low + k])]
        for s in range(1 << low):
            y = list(base)
            for k in range(low):
                if (s >> k) & 1:
                    y = [v + c for v, c in zip(y, cols[k])]
            t = 1
            for v in y:
                t *= v
            total += -t if (bin(s).count("1") + bin(g).count("1")) & 1 else t
            abs_total += abs(t)
    return Fraction(total * (2 if n & 1 else -2), 2 ** n), Fraction(abs_total * 2, 2 ** n)


def _crs_ccs(a):
    a = np.asarray(a) != 0
    n = a.shape[0]
    rptrs = np.concatenate([[0], np.cumsum(a.sum(1))]).astype(np.int32)
    cols = np.nonzero(a)[1].astype(np.int32)
    cptrs = np.concatenate([[0], np.cumsum(a.sum(0))]).astype(np.int32)
    rows = np.nonzero(a.T)[1].astype(np.int32)
    return n, rptrs, cols, cptrs, rows


def _oracle_sparse(self, a, seed, t0, count, y=None, z=None):
    n, rp, cl, cp, rw = _crs_ccs(a)
    out = np.zeros(count)
    if y is None:
        self.lib.orc_rasmussen_sparse_trials(_ptr(rp), _ptr(cl), _ptr(cp), _ptr(rw), n, seed, t0, count, _ptr(out))
    else:
        self.lib.orc_scaling_sparse_trials(_ptr(rp), _ptr(cl), _ptr(cp), _ptr(rw), n, y, z, seed, t0, count,
                                           _ptr(out))
    return out


def _grid_graph(self, m, n):
    cap = max(1, m * n // 2)
    out = np.zeros(cap * cap)
    k = self.lib.orc_grid_graph(m, n, _ptr(out), cap)
    if k < 0:
        raise ValueError("both sides odd")
    return out[: k * k].reshape(k, k).copy()


Oracle.rasmussen_sparse_trials = lambda self, a, seed, t0, count: _oracle_sparse(self, a, seed, t0, count)
Oracle.scaling_sparse_trials = lambda self, a, y, z, seed, t0, count: _oracle_sparse(self, a, seed, t0, count, y, z)
Oracle.grid_graph = _grid_graph


class Reference:
    """The reference's own functions (oracle/_ref/libperman_ref.so)."""

    def __init__(self):
        so = build_reference()
        if so is None or not Path(so).exists():
            raise FileNotFoundError("oracle/_ref/libperman_ref.so not built")
        self.lib = ctypes.CDLL(str(so))
        L = self.lib
        i, d, ll = ctypes.c_int, ctypes.c_double, ctypes.c_longlong
        for name in ("ref_parallel_perman64_f64", "ref_parallel_perman64_i32", "ref_perman64_f64",
                     "ref_parallel_perman64_sparse_f64", "ref_parallel_skip_balanced_f64",
                     "ref_cpu_perman64_range_f64", "ref_rasmussen_f64", "ref_approximation_f64",
                     "ref_rasmussen_sparse_f64", "ref_approximation_sparse", "ref_gpu_dense_mshared_f64",
                     "ref_gpu_dense_mshared_i32", "ref_gpu_skipper_f64", "ref_gpu_rasmussen_f64",
                     "ref_gpu_approximation_f64"):
            getattr(L, name).restype = d
        L.ref_cpu_perman64_range_f64.argtypes = [_P, i, ll, ll, i]
        L.ref_read_matrix_f64.argtypes = [ctypes.c_char_p, i, _P, i, ctypes.POINTER(i)]
        L.ref_compress_f64.argtypes = [i, _P, i, i, _P, _P, _P, _P, _P, _P]
        L.ref_grid_graph.argtypes = [i, i, _P, i]
        L.ref_last_cuda_error.restype = ctypes.c_char_p

    def parallel_perman64(self, a, threads: int) -> float:
        a = np.ascontiguousarray(a, dtype=np.float64)
        return self.lib.ref_parallel_perman64_f64(_ptr(a), a.shape[0], threads)

    def perman64(self, a) -> float:
        a = np.ascontiguousarray(a, dtype=np.float64)
        return self.lib.ref_perman64_f64(_ptr(a), a.shape[0])

    def cpu_perman64_range(self, a, start: int, end: int, threads: int) -> float:
        a = np.ascontiguousarray(a, dtype=np.float64)
        return self.lib.ref_cpu_perman64_range_f64(_ptr(a), a.shape[0], start, end, threads)

    def skip_balanced(self, c: dict, threads: int) -> float:
        arrs = [np.ascontiguousarray(c[k], dtype=np.int32) for k in ("rptrs", "cols")]
        rv = np.ascontiguousarray(c["rvals"], dtype=np.float64)
        carrs = [np.ascontiguousarray(c[k], dtype=np.int32) for k in ("cptrs", "rows")]
        cv = np.ascontiguousarray(c["cvals"], dtype=np.float64)
        return self.lib.ref_parallel_skip_balanced_f64(_ptr(arrs[0]), _ptr(arrs[1]), _ptr(rv), _ptr(carrs[0]),
                                                       _ptr(carrs[1]), _ptr(cv), c["n"], threads)

    def rasmussen(self, a, times: int, threads: int) -> float:
        a = np.ascontiguousarray(a, dtype=np.float64)
        return self.lib.ref_rasmussen_f64(_ptr(a), a.shape[0], times, threads)

    def approximation(self, a, times: int, y: int, z: int, threads: int) -> float:
        a = np.ascontiguousarray(a, dtype=np.float64)
        return self.lib.ref_approximation_f64(_ptr(a), a.shape[0], times, y, z, threads)

    def read_matrix(self, path, binary: bool, cap: int = 128) -> np.ndarray:
        buf = np.zeros(cap * cap)
        nnz = ctypes.c_int()
        n = self.lib.ref_read_matrix_f64(str(path).encode(), 0 if binary else 1, _ptr(buf), cap, ctypes.byref(nnz))
        if n < 0:
            raise RuntimeError(f"reference reader failed ({n})")
        return buf[: n * n].reshape(n, n).copy()

    def grid_graph(self, m: int, n: int) -> np.ndarray:
        cap = max(1, m * n // 2)
        out = np.zeros(cap * cap)
        k = self.lib.ref_grid_graph(m, n, _ptr(out), cap)
        if k < 0:
            raise ValueError("both sides odd")
        return out[: k * k].reshape(k, k).copy()

    def compress(self, mode: int, a) -> dict:
        a = np.array(a, dtype=np.float64, order="C", copy=True)
        n = a.shape[0]
        cap = n * n
        cp, rp = np.zeros(n + 1, np.int32), np.zeros(n + 1, np.int32)
        rows, cols = np.zeros(cap, np.int32), np.zeros(cap, np.int32)
        cv, rv = np.zeros(cap), np.zeros(cap)
        nnz = int((a > 0).sum()) if mode != 2 else int((a != 0).sum())
        used = self.lib.ref_compress_f64(mode, _ptr(a), n, max(nnz, 1), _ptr(cp), _ptr(rows), _ptr(cv), _ptr(rp),
                                         _ptr(cols), _ptr(rv))
        return {"n": n, "nnz": used, "mat": a, "cptrs": cp, "rows": rows[:used], "cvals": cv[:used], "rptrs": rp,
                "cols": cols[:used], "rvals": rv[:used]}
