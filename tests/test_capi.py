"""The C-ABI library loads and exports every symbol include/perman_b200.h declares
(no compute calls: runs without a GPU)."""
import ctypes
import math
import re
import subprocess

import numpy as np
import pytest
from conftest import ROOT


def declared_symbols():
    text = (ROOT / "include" / "perman_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"\b((?:perm|gpu_perman64)_\w+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "perm_exact_dense" in names and "perm_exact_sparse" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol(pb):
    lib = pb.load_library()
    out = subprocess.run(["nm", "-D", "--defined-only", str(pb.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT\s+(\w+)", out))
    missing = [n for n in declared_symbols() if n not in exported]
    assert not missing, f"declared but not exported: {missing}"
    for n in declared_symbols():
        assert getattr(lib, n) is not None
    assert set(pb.EXPORTED_SYMBOLS) <= exported


def test_version_and_status_strings(pb):
    lib = pb.load_library()
    assert lib.perm_version() >= 10000
    assert lib.perm_status_string(0) == b"ok"
    assert b"invalid" in lib.perm_status_string(-1)


def test_no_device_fails_loudly(pb):
    lib = pb.load_library()
    if lib.perm_device_count() > 0:
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    rc = lib.perm_ctx_create(0, ctypes.byref(h))
    assert rc != 0 and not h.value
    with pytest.raises(pb.PermError):
        pb.Engine(0)


def test_missing_library_raises(pb, tmp_path):
    with pytest.raises(pb.PermError):
        pb.load_library(tmp_path / "nope.so")


def test_header_constants_match_the_binding(pb):
    """Every PERM_* integer #define in the header has the same value in the
    Python binding (status codes, dtypes, kernel ids, request kinds)."""
    text = (ROOT / "include" / "perman_b200.h").read_text()
    defines = dict(re.findall(r"^#define\s+(PERM_\w+)\s+(-?\d+)\b", text, flags=re.M))
    assert "PERM_KERNEL_DENSE_SPLIT" in defines and "PERM_KERNEL_DENSE_TC" in defines
    checked = 0
    for name, value in defines.items():
        if name.startswith("PERM_MAX") or not hasattr(pb, name):
            continue
        assert getattr(pb, name) == int(value), (name, getattr(pb, name), value)
        checked += 1
    assert checked >= 10
    for name in defines:
        if name.startswith(("PERM_KERNEL_", "PERM_E", "PERM_F", "PERM_I", "PERM_REQ_")):
            assert hasattr(pb, name), name


def test_int_layout_query(pb):
    """Host-only layout of the int32-X walk: the order-40 bench matrix walks
    in the three-level row layout (column 0's rows in 3 groups of 5, the
    further rows of columns 1 and 2 in 2 more); order 24 takes two levels;
    small orders keep one level; non-integer matrices are refused."""
    import bench

    assert pb.int_layout(bench.make_matrix(0)) == (5, 0, 3, 2)
    rng = np.random.default_rng(4)
    assert pb.int_layout((rng.random((16, 16)) < 0.5).astype(float))[1:] == (0, 0, 0)
    g, ngo, ng1, ng2 = pb.int_layout((rng.random((24, 24)) < 0.5) * rng.integers(1, 5, (24, 24)).astype(float))
    assert g in (4, 5, 6) and ngo in (1, 2, 3) and ng1 == ng2 == 0
    assert pb.int_layout(rng.random((20, 20)))[0] == pb.PERM_EUNSUPPORTED


def test_intc_layout_query(pb):
    """Host-only layout of the certified int32-X walk: product groups that
    fit int32, consecutive groups paired (exact int64 products) from order 16
    when every run of 2G rows stays below 2^53, and from order 20 the
    two-level row layout and from order 28 the three-level one where they
    are cheaper -- the layout with the fewest instructions per Gray step."""
    rng = np.random.default_rng(3)
    A = ((rng.random((40, 40)) < 0.5) * rng.integers(1, 5, (40, 40))).astype(float)
    g, pair, ngo, ng1, ng2 = pb.intc_layout(A)
    # several levels at order 40: two (outer groups) or three (first, second level)
    assert (g, pair) in ((4, True), (5, False), (6, True))
    assert (ngo in (1, 2, 3) and ng1 == ng2 == 0) or (ngo == 0 and ng1 in (2, 3, 4) and ng2 in (1, 2))
    B = (rng.random((40, 40)) < 0.5).astype(float)
    assert pb.intc_layout(B)[0] in (4, 5, 6)
    assert pb.intc_layout(B[:12, :12])[1:] == (False, 0, 0, 0)  # pairs from order 16, levels from 20
    Bs = B[:24, :24]
    assert pb.intc_layout(Bs)[3:] == (0, 0)  # three levels from order 28
    C = rng.integers(0, 60, (24, 24)).astype(float)
    assert pb.intc_layout(C) == (3, False, 0, 0, 0)  # large entries: groups of 3, no pairs
    assert pb.intc_layout(rng.random((20, 20)))[0] == pb.PERM_EUNSUPPORTED
    assert pb.intc_layout(np.ones((7, 7)))[0] == pb.PERM_EUNSUPPORTED


def test_sdd_layout_query(pb):
    """Host-only layout query: dense matrices keep the dense layout, sparse
    ones get the smallest inner-row count that holds their three sparsest
    columns' rows, orders outside 4..40 are refused."""
    rng = np.random.default_rng(1)
    assert pb.sdd_layout(1.0 - rng.random((30, 30))) == 0
    P = np.eye(20)[rng.permutation(20)] + np.eye(20)
    assert pb.sdd_layout(P) == 6
    assert pb.sdd_layout(np.ones((41, 41))) == pb.PERM_EUNSUPPORTED
    assert pb.sdd_layout(np.ones((3, 3))) == pb.PERM_EUNSUPPORTED
    assert pb.sdd_levels(P) == (0, 6)


def test_fp64_levels_query(pb):
    """Density-1/2 real matrices of orders 28..48 take the FP64-X walk's
    three-level layout (first level 8..20 rows, second ending at 20..36);
    orders 20..27 the two-level one."""
    for n in (28, 34, 40, 48):
        rng = np.random.default_rng(n)
        A = (rng.random((n, n)) < 0.5) * (1.0 - rng.random((n, n)))
        r1, r2 = pb.fp64_levels(A)
        assert r1 in (8, 12, 16, 20) and r2 in (20, 24, 28, 32, 36) and r1 < r2, (n, r1, r2)
        assert pb.fp64_layout(A) == r2
    rng = np.random.default_rng(7)
    A = (rng.random((24, 24)) < 0.5) * 1.0
    assert pb.fp64_levels(A) == (0, pb.fp64_layout(A))
    assert pb.fp64_levels(1.0 - rng.random((30, 30))) == (0, 0)  # no zeros: one level


def test_sdd_levels_query(pb):
    """Density-1/2 real matrices of orders 24..40 take the split-dd walk's
    three-level layout (first level 8..20 rows, second ending at 16..28);
    below order 24 they do not."""
    for n in (24, 30, 34, 40):
        rng = np.random.default_rng(n)
        A = (rng.random((n, n)) < 0.5) * (1.0 - rng.random((n, n)))
        r1, r2 = pb.sdd_levels(A)
        assert r1 in (8, 12, 16, 20) and r2 in (16, 20, 24, 28) and r1 < r2, (n, r1, r2)
        assert pb.sdd_layout(A) == r2
    rng = np.random.default_rng(5)
    assert pb.sdd_levels((rng.random((22, 22)) < 0.5) * 1.0)[0] == 0
    assert pb.sdd_levels(np.ones((41, 41)))[0] == pb.PERM_EUNSUPPORTED


def test_multi_device_arguments_and_no_device(pb):
    """perm_exact_dense_multi checks its arguments on the host (1..64 shards,
    orders 1..64) and, without a GPU, fails loudly instead of computing."""
    lib = pb.load_library()
    A = np.ones((5, 5))
    r = pb.PermResult()
    p = A.ctypes.data_as(ctypes.c_void_p)
    assert lib.perm_exact_dense_multi(p, 5, pb.PERM_F64, 0, 0, None, ctypes.byref(r)) == pb.PERM_EINVAL
    assert lib.perm_exact_dense_multi(p, 5, pb.PERM_F64, 0, 65, None, ctypes.byref(r)) == pb.PERM_EINVAL
    assert lib.perm_exact_dense_multi(p, 65, pb.PERM_F64, 0, 2, None, ctypes.byref(r)) == pb.PERM_EINVAL
    assert lib.perm_exact_dense_multi(None, 5, pb.PERM_F64, 0, 2, None, ctypes.byref(r)) == pb.PERM_EINVAL
    if lib.perm_device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(pb.PermError):
        pb.exact_dense_multi(A, nshards=2)
    assert math.isnan(lib.gpu_perman64_xshared_coalescing_mshared_multigpu_double(p, 5, 2, 2048, 128))


def test_multigpu_python_mirror_fails_loudly_without_gpu(pb):
    if pb.load_library().perm_device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(pb.PermError):
        pb.gpu_perman64_xshared_coalescing_mshared_multigpu(np.ones((4, 4)), 4, 2)
