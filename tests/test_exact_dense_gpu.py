"""Dense exact Ryser kernel on the B200 against the oracle (tolerance 1e-10
relative, the exact-algorithm bar; integer inputs that fit are compared exactly)."""
import math
from fractions import Fraction

import numpy as np
import pytest
from conftest import bernoulli, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.mark.parametrize("n", list(range(1, 25)))
def test_orders_1_to_24_vs_oracle(engine, orc, n):
    rng = np.random.default_rng(1000 + n)
    for kind in ("binary", "int", "real", "signed"):
        if kind == "binary":
            A = bernoulli(rng, n, 0.5) if n > 1 else np.ones((1, 1))
        elif kind == "int":
            A = rng.integers(0, 5, (n, n)).astype(float)
        elif kind == "real":
            A = 1.0 - rng.random((n, n))
        else:
            A = rng.standard_normal((n, n))
        r = engine.exact_dense(A)
        want = orc.perm_dd(A)
        if kind in ("binary", "int"):
            exact = orc.perm_exact_int(A)[0]
            assert rel_err(r.value, exact) < 1e-13, (kind, r.value, exact)
        else:
            # signed matrices cancel heavily: compare against the oracle's scale
            scale = max(abs(want[0]), 1e-300)
            assert abs(r.value - want[0]) / scale < (TOL if kind == "real" else 1e-8), (kind, r.value, want)
        assert r.total_steps == 2.0 ** (n - 1)


def test_golden_vectors(engine, golden):
    for name, c in golden.items():
        r = engine.exact_dense(c["A"])
        want = int(c["exact"]) if "exact" in c else c["dd"][0] + c["dd"][1]
        assert rel_err(r.value, want) < TOL, (name, r.value, want)


def test_dtypes_agree(engine):
    rng = np.random.default_rng(3)
    A = rng.integers(0, 5, (20, 20))
    v64 = engine.exact_dense(A.astype(np.float64)).value
    assert engine.exact_dense(A.astype(np.int32)).value == v64
    assert engine.exact_dense(A.astype(np.float32)).value == v64


@pytest.mark.parametrize("n", [1, 2, 3, 4, 12, 18, 22])
def test_all_ones_factorial(engine, n):
    # small orders are exact; beyond ~2^53 in the intermediate terms, 1e-13
    for variant in (1, 3):
        if variant == 3 and n < 8:
            continue
        v = engine.exact_dense(np.ones((n, n)), variant=variant).value
        assert rel_err(v, math.factorial(n)) <= (0 if n <= 12 else 1e-13)


def test_identity_permutation_zero_row(engine):
    rng = np.random.default_rng(4)
    for n in (5, 17, 26):
        P = np.eye(n)[rng.permutation(n)]
        assert engine.exact_dense(P).value == 1.0
        Z = rng.random((n, n))
        Z[rng.integers(n)] = 0
        assert engine.exact_dense(Z).value == 0.0


@pytest.mark.parametrize("nshards", [2, 3, 7])
def test_shards_sum_to_whole(engine, nshards):
    rng = np.random.default_rng(5)
    A = bernoulli(rng, 27, 0.5) * rng.integers(1, 5, (27, 27))
    whole = engine.exact_dense(A)
    hi = lo = 0.0
    for s in range(nshards):
        r = engine.exact_dense_shard(A, s, nshards)
        hi, lo = hi + r.hi, lo + r.lo
    # a different thread decomposition rounds differently: compare at 1e-12
    assert rel_err(hi + lo, whole.value) < 1e-12


def test_resident_matrix_matches_one_shot(engine, pb):
    rng = np.random.default_rng(6)
    A = 1.0 - rng.random((25, 25))
    m = engine.upload_dense(A)
    try:
        # same kernel both ways (the automatic path may rerun this real matrix in double-double)
        assert m.run().value == engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE).value
    finally:
        m.free()


@pytest.mark.slow
@pytest.mark.parametrize("n", [36, 40])
def test_full_size_invariances(engine, n):
    """At the benchmark sizes the oracle is too slow; use size-independent
    properties: row/column permutation and transpose invariance, and exact
    scaling of a row by 2 on an integer matrix."""
    rng = np.random.default_rng(n)
    A = bernoulli(rng, n, 0.5) * rng.integers(1, 5, (n, n))
    base = engine.exact_dense(A).value
    assert rel_err(engine.exact_dense(A, variant=1).value, base) < TOL  # FP64-X and int32-X agree
    Pm = A[rng.permutation(n)][:, rng.permutation(n)]
    assert rel_err(engine.exact_dense(Pm).value, base) < TOL
    assert rel_err(engine.exact_dense(A.T.copy()).value, base) < TOL
    B = A.copy()
    B[3] *= 2
    assert rel_err(engine.exact_dense(B).value, 2 * base) < TOL


def test_errors_are_reported(engine, pb):
    with pytest.raises(pb.PermError) as e:
        engine.exact_dense(np.ones((65, 65)))
    assert e.value.status == pb.PERM_EUNSUPPORTED
    with pytest.raises(pb.PermError):
        engine.exact_dense(np.ones((3, 4)))
    # the context stays usable after an error
    assert engine.exact_dense(np.ones((5, 5))).value == 120.0


def test_reference_signature_entry_points(pb):
    rng = np.random.default_rng(8)
    A = bernoulli(rng, 15, 0.5)
    want = pb.default_engine().exact_dense(A).value
    assert pb.gpu_perman64_xshared_coalescing_mshared(A, 15, 2048, 256) == want
    lib = pb.load_library()
    Ai = np.ascontiguousarray(A, dtype=np.int32)
    assert lib.gpu_perman64_xshared_coalescing_mshared_int(Ai.ctypes.data_as(pb._P), 15, 2048, 256) == want


def test_reference_gpu_kernel_same_inputs(engine, ref):
    """The reference's own -p4 kernel (built for sm_100a) on the same binary
    matrix; its FP32 X is exact for small integer inputs."""
    rng = np.random.default_rng(9)
    A = bernoulli(rng, 20, 0.5)
    import ctypes
    Ac = np.ascontiguousarray(A)
    theirs = ref.lib.ref_gpu_dense_mshared_f64(Ac.ctypes.data_as(ctypes.c_void_p), 20, 2048, 128)
    assert rel_err(engine.exact_dense(A).value, theirs) < 1e-12


# ---- int32-X kernel ---------------------------------------------------------------

@pytest.mark.parametrize("n", [8, 9, 13, 17, 21, 24, 27])
def test_int_kernel_exact_vs_oracle(engine, orc, pb, n):
    rng = np.random.default_rng(500 + n)
    for hi in (2, 5, 30):  # binary, small and larger integers -> different group sizes
        A = bernoulli(rng, n, 0.5) * rng.integers(1, hi, (n, n))
        exact = orc.perm_exact_int(A)[0]
        r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_INT)
        assert r.kernel == pb.PERM_KERNEL_DENSE_INT
        assert rel_err(r.value, exact) < 1e-12, (hi, r.value, exact)
        f = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE)
        assert rel_err(f.value, r.value) < 1e-12


@pytest.mark.parametrize("n", [20, 23, 27])
def test_int_kernel_two_level_layout_vs_exact(engine, orc, pb, n):
    """The int32-X walk in the two-level row layout (the rows that the three
    sparsest columns never touch keep their group product for seven of
    every eight steps) against the exact multi-modular oracle, on dense
    U{1..4}, 0/1 and signed matrices; shards and a resident matrix of the
    same layout add up to the whole walk."""
    rng = np.random.default_rng(600 + n)
    cases = {"u1to4": bernoulli(rng, n, 0.5) * rng.integers(1, 5, (n, n)),
             "binary": bernoulli(rng, n, 0.5),
             "signed": bernoulli(rng, n, 0.5) * rng.integers(-3, 4, (n, n))}
    for kind, A in cases.items():
        g, ngo, _, _ = pb.int_layout(A)
        assert ngo >= 1, (kind, g, ngo)
        exact = orc.perm_exact_int(A)[0]
        r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_INT)
        assert r.kernel == pb.PERM_KERNEL_DENSE_INT
        assert abs(r.value - exact) <= 1e-12 * max(abs(exact), 1.0) + 1e-12 * r.abs_term_sum, (kind, r.value, exact)
    A = cases["u1to4"]
    whole = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_INT).value
    parts = [engine.exact_dense_shard(A, s, 3, variant=pb.PERM_KERNEL_DENSE_INT) for s in range(3)]
    assert rel_err(sum(p.hi + p.lo for p in parts), whole) < 1e-13
    res = engine.upload_dense(A, variant=pb.PERM_KERNEL_DENSE_INT)
    try:
        assert res.run().value == whole
    finally:
        res.free()


def _fp64_layout_case(engine, orc, pb, A, tol=1e-10):
    r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE)
    hi, lo = orc.perm_dd(A)
    want = hi + lo
    assert abs(r.value - want) <= r.rel_error_estimate * abs(want), (r.value, want, r.rel_error_estimate)
    if tol:
        assert rel_err(r.value, want) < tol
    # shards re-anchor X at other indices: same bound, different roundings
    parts = [engine.exact_dense_shard(A, s, 3, variant=pb.PERM_KERNEL_DENSE) for s in range(3)]
    assert abs(sum(p.hi + p.lo for p in parts) - r.value) <= 2 * r.rel_error_estimate * abs(r.value)
    res = engine.upload_dense(A, variant=pb.PERM_KERNEL_DENSE)
    try:
        assert res.run().value == r.value
    finally:
        res.free()


@pytest.mark.parametrize("n,seed,levels", [(28, 0, (8, 20)), (29, 1, (12, 20)), (30, 2, (12, 20))])
def test_fp64_three_level_layout_vs_oracle(engine, orc, pb, n, seed, levels):
    """The FP64-X walk in the three-level row layout (column 0's rows at
    half of the steps, columns 1-2's at three in eight) on real density-1/2
    matrices: against the CPU double-double Ryser within the walk's own
    bound; shards and a resident matrix of that layout add up to it."""
    rng = np.random.default_rng(seed)
    A = (rng.random((n, n)) < 0.5) * (1.0 - rng.random((n, n)))
    assert pb.fp64_levels(A) == levels
    _fp64_layout_case(engine, orc, pb, A)


def test_fp64_three_level_layout_signed_and_wide(engine, orc, pb):
    """Signed entries (cancellation) in the three-level layout, and a
    second level of 24 rows at order 30 (constructed supports)."""
    rng = np.random.default_rng(31)
    n = 30
    mask = rng.random((n, n)) < 0.9
    mask[12:, 0] = False
    mask[:12, 0] = True
    mask[24:, 1:3] = False
    mask[12:24, 1] = True
    A = mask * rng.standard_normal((n, n))
    r1, r2 = pb.fp64_levels(A)
    assert r1 == 12 and r2 == 24, (r1, r2)
    _fp64_layout_case(engine, orc, pb, A, tol=None)  # cancellation: the bound alone


@pytest.mark.parametrize("n", [22, 25])
def test_fp64_two_level_layout_vs_oracle(engine, orc, pb, n):
    """The FP64-X walk in the two-level row layout on real density-1/2
    matrices: against the CPU double-double Ryser within the walk's own
    bound, and shards and a resident matrix of that layout add up to it."""
    rng = np.random.default_rng(700 + n)
    A = (rng.random((n, n)) < 0.5) * (1.0 - rng.random((n, n)))
    assert pb.fp64_layout(A) in (16, 20, 24, 28) and pb.fp64_levels(A)[0] == 0
    _fp64_layout_case(engine, orc, pb, A)


@pytest.mark.parametrize("n", [28, 30])
def test_int_kernel_three_level_layout_vs_exact(engine, orc, pb, n):
    """The int32-X walk in the three-level row layout (column 0's rows, the
    further rows of columns 1 and 2, the rest) against the exact
    multi-modular oracle on dense U{1..4} and 0/1 matrices."""
    rng = np.random.default_rng(650 + n)
    for kind, A in (("u1to4", bernoulli(rng, n, 0.5) * rng.integers(1, 5, (n, n))), ("binary", bernoulli(rng, n, 0.5))):
        g, ngo, ng1, ng2 = pb.int_layout(A)
        assert ng1 >= 2 and ng2 >= 1, (kind, g, ngo, ng1, ng2)
        exact = orc.perm_exact_int(A)[0]
        r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_INT)
        assert rel_err(r.value, exact) < 1e-12, (kind, r.value, exact)


def test_int_kernel_signed_entries(engine, orc, pb):
    rng = np.random.default_rng(17)
    A = rng.integers(-4, 5, (18, 18)).astype(float)
    exact = orc.perm_exact_int(A)[0]
    r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_INT)
    assert abs(r.value - exact) <= 1e-10 * max(abs(exact), 1.0) * 1e3


def test_automatic_kernel_choice(engine, pb):
    """With the accuracy policy on, integer matrices start with the certified
    int32-X walk; with it off (one evaluation) the plain int32-X walk runs;
    non-integer and large-entry matrices take FP64 X (dense real matrices
    keep their FP64-X value when its bound meets the target)."""
    rng = np.random.default_rng(18)
    A = bernoulli(rng, 20, 0.5)
    assert engine.exact_dense(A).kernel == pb.PERM_KERNEL_DENSE_INT_DD
    engine.set_rel_target(0.0)
    try:
        assert engine.exact_dense(A).kernel == pb.PERM_KERNEL_DENSE_INT
        assert engine.exact_dense(A * 0.5).kernel == pb.PERM_KERNEL_DENSE
        big = A * 100000  # row products no longer fit int32 in groups of 3
        assert engine.exact_dense(big).kernel == pb.PERM_KERNEL_DENSE
    finally:
        engine.set_rel_target(1e-10)
    with pytest.raises(pb.PermError):
        engine.exact_dense(A * 0.5, variant=pb.PERM_KERNEL_DENSE_INT)


def test_int_kernel_golden(engine, golden, pb):
    for name, c in golden.items():
        if c["kind"] == "real" or c["n"] < 8 or "exact" not in c:
            continue
        r = engine.exact_dense(c["A"], variant=pb.PERM_KERNEL_DENSE_INT)
        assert rel_err(r.value, int(c["exact"])) < TOL, name


def test_int_kernel_shards(engine, pb):
    rng = np.random.default_rng(19)
    A = bernoulli(rng, 26, 0.5) * rng.integers(1, 5, (26, 26))
    whole = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_INT).value
    parts = [engine.exact_dense_shard(A, s, 5, variant=pb.PERM_KERNEL_DENSE_INT) for s in range(5)]
    assert rel_err(sum(p.hi + p.lo for p in parts), whole) < 1e-12


def test_multi_device_entry_point(engine, orc, pb):
    """perm_exact_dense_multi (gpu_exact_dense.cu:702): shards on device 0
    listed two and three times (one host thread and context each, kernels
    running side by side) add up to the one-walk value -- exactly for the
    integer matrix (oracle), within 1e-12 of the FP64-X walk for the real
    one -- and the reference-signature shim clamps gpu_num to the visible
    devices."""
    import ctypes

    rng = np.random.default_rng(702)
    A = bernoulli(rng, 26, 0.5) * rng.integers(1, 5, (26, 26))
    exact = orc.perm_exact_int(A)[0]
    for devices in ([0, 0], [0, 0, 0]):
        r = pb.exact_dense_multi(A, devices=devices)
        assert rel_err(r.value, exact) < 1e-13, (devices, r.value, exact)
        assert r.total_steps == 2.0**25 and r.rel_error_estimate == 0.0
    R = 1.0 - rng.random((23, 23))
    want = engine.exact_dense(R, variant=pb.PERM_KERNEL_DENSE).value
    assert rel_err(pb.exact_dense_multi(R, devices=[0, 0, 0, 0]).value, want) < 1e-12
    lib = pb.load_library()
    Ai = np.ascontiguousarray(A, dtype=np.int32)
    got = lib.gpu_perman64_xshared_coalescing_mshared_multigpu_int(Ai.ctypes.data_as(ctypes.c_void_p), 26,
                                                                    lib.perm_device_count() + 3, 2048, 256)
    assert rel_err(got, exact) < 1e-13
    Rd = np.ascontiguousarray(R)
    got = lib.gpu_perman64_xshared_coalescing_mshared_multigpu_double(Rd.ctypes.data_as(ctypes.c_void_p), 23, 1,
                                                                       2048, 128)
    assert rel_err(got, want) < 1e-12
    with pytest.raises(pb.PermError):
        pb.exact_dense_multi(A, devices=[0, 10**6])  # no such device: the failing shard's status


def test_dense_autotune_sets_the_automatic_choice(pb):
    """The autotuned kernel is the automatic choice for single evaluations
    (policy off); with the policy on, integer inputs take the certified walk."""
    with pb.Engine(0) as eng:
        eng.set_rel_target(0.0)
        table = eng.dense_autotune(8, 22)
        assert set(table.values()) <= {pb.PERM_KERNEL_DENSE, pb.PERM_KERNEL_DENSE_INT, pb.PERM_KERNEL_DENSE_TC}
        rng = np.random.default_rng(1)
        for n, k in table.items():
            A = bernoulli(rng, n, 0.5)
            assert eng.exact_dense(A).kernel == k


# ---- double-double kernel and per-result error estimates ------------------------------

@pytest.mark.parametrize("n", [1, 2, 3, 5, 12, 19, 24])
def test_dd_kernel_vs_oracle(engine, orc, pb, n):
    rng = np.random.default_rng(700 + n)
    for A in (rng.standard_normal((n, n)), 1.0 - rng.random((n, n))):
        r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_DD)
        assert r.kernel == pb.PERM_KERNEL_DENSE_DD
        hi, lo = orc.perm_dd(A)
        # both are double-double evaluations: agree far below FP64 roundoff
        assert abs((r.hi - hi) + (r.lo - lo)) <= 1e-24 * abs(hi) + 1e-300, (r.hi, r.lo, hi, lo)


def test_dd_kernel_exact_on_integers(engine, orc, pb):
    rng = np.random.default_rng(31)
    A = bernoulli(rng, 22, 0.5) * rng.integers(1, 5, (22, 22))
    r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_DD)
    exact = orc.perm_exact_int(A)[0]
    assert int(r.hi) + int(r.lo) == exact


def test_error_estimate_bounds_the_fp64_error(engine, orc, pb):
    rng = np.random.default_rng(32)
    for n in (14, 18, 22):
        for _ in range(3):
            A = rng.standard_normal((n, n))
            r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE)
            hi, lo = orc.perm_dd(A)
            actual = abs(r.value - hi - lo) / abs(hi)
            assert r.rel_error_estimate > 0 and r.abs_term_sum > 0
            assert actual <= r.rel_error_estimate, (n, actual, r.rel_error_estimate)


def test_automatic_double_double_rerun(pb, orc):
    rng = np.random.default_rng(33)
    A = rng.standard_normal((20, 20))
    with pb.Engine(0) as eng:
        eng.set_rel_target(1e-16)  # unreachable in FP64: forces the certified (split-dd) rerun
        r = eng.exact_dense(A)
        assert r.kernel == pb.PERM_KERNEL_DENSE_SDD
        hi, lo = orc.perm_dd(A)
        assert abs((r.hi - hi) + (r.lo - lo)) <= max(r.rel_error_estimate, 1e-24) * abs(hi)
        assert r.rel_error_estimate < 1e-20
        eng.set_rel_target(0.0)  # no reruns
        assert eng.exact_dense(A).kernel in (pb.PERM_KERNEL_DENSE, pb.PERM_KERNEL_DENSE_INT)


def test_fp64_error_grows_and_double_double_fixes_it(engine, pb):
    """Dense positive real matrices cancel more with n: the FP64-X result's
    estimate flags it and the automatic path returns the double-double value."""
    rng = np.random.default_rng(4)
    A = 1.0 - rng.random((30, 30))
    f = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE)
    d = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_DD)
    auto = engine.exact_dense(A)
    actual = abs(f.value - d.value) / abs(d.value)
    assert actual <= f.rel_error_estimate
    if f.rel_error_estimate > 1e-10:
        # kept after the transpose cross-check, or recomputed by the certified split-dd walk
        if auto.kernel == pb.PERM_KERNEL_DENSE_SDD:
            assert abs(auto.value - d.value) <= (auto.rel_error_estimate + d.rel_error_estimate + 2.3e-16) * abs(d.value)
        else:
            assert auto.kernel == pb.PERM_KERNEL_DENSE
            assert abs(auto.value - d.value) / abs(d.value) <= auto.rel_error_estimate <= 1e-10


@pytest.mark.parametrize("n", [28, 32])
def test_transpose_cross_check_meets_the_target(engine, pb, n):
    """Positive real matrices: the worst-case bound exceeds 1e-10 at these
    orders; whatever the automatic path returns is within 1e-10 of the
    double-double value."""
    rng = np.random.default_rng(40 + n)
    A = 1.0 - rng.random((n, n))
    d = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_DD)
    auto = engine.exact_dense(A)
    assert abs(auto.value - d.value) <= 1e-10 * abs(d.value)
    assert auto.rel_error_estimate <= 1e-10


def test_int_kernel_estimate_covers_signed_cancellation(engine, orc, pb):
    """Signed integer entries cancel heavily; the int32-X estimate (independent
    roundings of exact group products) still covers the actual error."""
    rng = np.random.default_rng(41)
    for n in (16, 20, 24):
        A = rng.integers(-2, 3, (n, n)).astype(np.float64)
        r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_INT)
        exact = orc.perm_exact_int(A)[0]
        if exact == 0:
            continue
        actual = float(abs(Fraction(r.hi) + Fraction(r.lo) - exact) / abs(exact))
        assert actual <= max(r.rel_error_estimate, 2.0 ** -52), (n, actual, r.rel_error_estimate)


@pytest.mark.parametrize("n", [32, 36, 40])
def test_int_kernel_estimate_at_headline_distribution(engine, pb, n):
    """U{1..4} entries at density 0.5 (the headline workload's distribution):
    the int32-X result's estimate covers its distance to the double-double
    value, and the automatic path returns a result within the 1e-10 target."""
    rng = np.random.default_rng(900 + n)
    A = bernoulli(rng, n, 0.5) * rng.integers(1, 5, (n, n))
    r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_INT)
    d = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_DD)
    actual = abs(r.value - d.value) / abs(d.value)
    assert actual <= max(r.rel_error_estimate, 2.0 ** -52), (actual, r.rel_error_estimate)
    auto = engine.exact_dense(A)
    assert abs(auto.value - d.value) <= 1e-10 * abs(d.value)


def test_structural_zero_is_exact(engine, pb):
    """A zero pattern without a perfect matching (rows 0 and 1 share one
    nonzero column) has permanent exactly 0 on the automatic path."""
    rng = np.random.default_rng(42)
    A = rng.random((24, 24))
    A[0, :] = 0.0
    A[1, :] = 0.0
    A[0, 5] = A[1, 5] = 1.0
    r = engine.exact_dense(A)
    assert r.value == 0.0 and r.hi == 0.0 and r.lo == 0.0 and r.rel_error_estimate == 0.0
    f = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE)
    assert abs(f.value) <= 1e-12 * f.abs_term_sum


# ---- tensor-core kernel (kind::i8 row sums, int32 products) ----------------------------

@pytest.mark.parametrize("n", [16, 17, 20, 23, 24, 27])
def test_tc_kernel_vs_oracle(engine, orc, pb, n):
    rng = np.random.default_rng(1100 + n)
    A = bernoulli(rng, n, 0.5) * rng.integers(1, 5, (n, n))
    r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_TC)
    assert r.kernel == pb.PERM_KERNEL_DENSE_TC and r.steps == r.total_steps == 2.0 ** (n - 1)
    exact = orc.perm_exact_int(A)[0]
    assert rel_err(r.value, exact) < 1e-12, (r.value, exact)


@pytest.mark.parametrize("n", [32, 33, 36])
def test_tc_kernel_vs_int_kernel(engine, pb, n):
    """Orders where the CPU oracle is slow: against the int32-X kernel (pinned
    to the oracle up to n = 30)."""
    rng = np.random.default_rng(1150 + n)
    A = bernoulli(rng, n, 0.5) * rng.integers(1, 5, (n, n))
    t = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_TC)
    i = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_INT)
    assert t.kernel == pb.PERM_KERNEL_DENSE_TC
    assert rel_err(t.value, i.value) < 1e-11, (t.value, i.value)


@pytest.mark.parametrize("n,round0,nrounds", [(16, 0, 64), (31, 5, 6), (33, 0, 5), (40, 12345, 6),
                                              (48, 2 ** 35 - 2, 4), (49, 3, 5), (57, 2 ** 40 - 3, 5),
                                              (64, 2 ** 50 - 2, 4), (64, 2 ** 53 + 2 ** 52 + 11, 3)])
def test_tc_kernel_round_ranges_vs_oracle(engine, pb, n, round0, nrounds):
    """Every operand layout (16, 32, 48, 64 columns per block) up to order
    64, on round ranges that one CTA walks (from-scratch first rounds, then
    in-place updates, including round columns >= 32 at 2^35 and 2^50) and
    the oracle sums exactly."""
    from oracle import tc_rounds_sum
    rng = np.random.default_rng(1170 + n)
    lim = 63 if n <= 33 else 20  # keeps the int32 product grouping available
    A = rng.integers(-lim, lim + 1, (n, n)).astype(np.float64) * (rng.random((n, n)) < 0.5)
    A[0, 0], A[1, 1] = 63, -63  # int8 operand limits (2a = +-126)
    r = engine.exact_dense_tc_rounds(A, round0, nrounds)
    want, abs_sum = tc_rounds_sum(A, round0, nrounds)
    assert r.steps == nrounds * 512.0
    got = Fraction(r.hi) + Fraction(r.lo)
    # group products are exact int32; only the <= 21 FP64 products across
    # groups round: |error| <= (21 + 16) u sum |terms|
    assert abs(got - want) <= Fraction(37, 2 ** 53) * abs_sum, (float(got), float(want), float(abs_sum))


def test_tc_kernel_signed_and_extreme_entries(engine, orc, pb):
    """Entries at the int8 limits of the operands (|2a| = 126) and mixed signs."""
    rng = np.random.default_rng(1200)
    for n, vals in ((18, (-63, 63)), (21, (-1, 1)), (24, (-5, 5))):
        A = rng.integers(vals[0], vals[1] + 1, (n, n)).astype(np.float64)
        A[0, 0] = vals[1]
        r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_TC)
        exact = orc.perm_exact_int(A)[0]
        assert abs(r.value - exact) <= 1e-12 * max(abs(exact), r.abs_term_sum), (n, r.value, exact)


def test_tc_kernel_matches_int_kernel_at_40(engine, pb):
    rng = np.random.default_rng(1300)
    A = bernoulli(rng, 40, 0.5) * rng.integers(1, 5, (40, 40))
    t = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_TC)
    i = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_INT)
    assert rel_err(t.value, i.value) < 1e-10


def test_tc_kernel_eligibility(engine, pb):
    rng = np.random.default_rng(1400)
    A = bernoulli(rng, 24, 0.5) * rng.integers(1, 5, (24, 24))
    assert engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_TC).kernel == pb.PERM_KERNEL_DENSE_TC
    B = A.copy()
    B[0, 0] = 64  # beyond int8 operands
    with pytest.raises(pb.PermError):
        engine.exact_dense(B, variant=pb.PERM_KERNEL_DENSE_TC)
    with pytest.raises(pb.PermError):
        engine.exact_dense(A[:15, :15], variant=pb.PERM_KERNEL_DENSE_TC)
    with pytest.raises(pb.PermError):
        engine.exact_dense(A + 0.5, variant=pb.PERM_KERNEL_DENSE_TC)


def test_tc_kernel_resident_and_shards(engine, pb):
    rng = np.random.default_rng(1500)
    A = bernoulli(rng, 26, 0.5) * rng.integers(1, 5, (26, 26))
    whole = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_TC).value
    res = engine.upload_dense(A, variant=pb.PERM_KERNEL_DENSE_TC)
    try:
        assert res.run().value == whole
    finally:
        res.free()
    parts = [engine.exact_dense_shard(A, s, 3, variant=pb.PERM_KERNEL_DENSE_TC) for s in range(3)]
    assert all(p.kernel == pb.PERM_KERNEL_DENSE_INT for p in parts)
    assert rel_err(pb.dd_sum([(p.hi, p.lo) for p in parts])[0], whole) < 1e-12


def test_refine_assembled_shards(engine, pb):
    """perm_exact_dense_refine gives a value assembled from shards the same
    estimate and policy as a whole call: within 1e-10 of double-double."""
    rng = np.random.default_rng(92)
    A = 1.0 - rng.random((29, 29))
    parts = [engine.exact_dense_shard(A, s, 4) for s in range(4)]
    hi, lo = pb.dd_sum([(p.hi, p.lo) for p in parts])
    r = engine.refine_dense(A, hi, lo, sum(p.kernel_ms for p in parts))
    d = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_DD).value
    assert abs(r.value - d) <= 1e-10 * abs(d)
    assert 0 < r.rel_error_estimate <= 1e-10
    assert r.kernel_ms >= sum(p.kernel_ms for p in parts)


# ---- split-X kernel ---------------------------------------------------------------------

@pytest.mark.parametrize("n", [4, 5, 9, 12, 19, 24])
def test_split_kernel_vs_oracle(engine, orc, pb, n):
    rng = np.random.default_rng(950 + n)
    for kind in ("real", "signed", "wide"):
        if kind == "real":
            A = 1.0 - rng.random((n, n))
        elif kind == "signed":
            A = rng.standard_normal((n, n))
        else:  # entries over many binades: the small ones live mostly in the remainder part;
            # Ryser's terms cancel heavily here, so only the estimate is checked
            A = rng.random((n, n)) * np.exp2(rng.integers(-30, 4, (n, n)))
        r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_SPLIT)
        assert r.kernel == pb.PERM_KERNEL_DENSE_SPLIT
        hi, lo = orc.perm_dd(A)
        actual = abs(r.value - hi - lo) / abs(hi)
        assert 0 < r.rel_error_estimate and actual <= r.rel_error_estimate, (kind, actual, r.rel_error_estimate)
        if kind == "real":
            assert actual <= 1e-13, (kind, actual)


def test_split_kernel_rows_of_different_scales(engine, orc, pb):
    """Each row gets its own coarse grid: rows scaled over 10 orders of
    magnitude keep the split result at the unscaled matrix's accuracy."""
    n = 22
    rng = np.random.default_rng(961)
    A = (1.0 - rng.random((n, n))) * (7.3 ** (np.arange(n) % 11 - 5.0))[:, None]
    r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_SPLIT)
    hi, lo = orc.perm_dd(A)
    assert abs(r.value - hi - lo) / abs(hi) <= 1e-13


def test_split_kernel_integer_and_binary_inputs(engine, orc, pb):
    rng = np.random.default_rng(960)
    for A in (bernoulli(rng, 21, 0.5), rng.integers(-3, 4, (18, 18)).astype(float), np.ones((13, 13))):
        r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_SPLIT)
        exact = orc.perm_exact_int(A)[0]
        assert abs(r.value - exact) <= max(r.rel_error_estimate * abs(exact), 2.0 ** -52 * abs(exact))


@pytest.mark.parametrize("n", [30, 34])
def test_split_kernel_vs_double_double(engine, pb, n):
    """Positive real matrices, where the FP64-X walk's correlated roundings
    reach 1e-10..1e-9: the split-X result stays far inside the target."""
    rng = np.random.default_rng(970 + n)
    A = 1.0 - rng.random((n, n))
    s = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_SPLIT)
    d = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_DD)
    actual = abs(s.value - d.value) / abs(d.value)
    assert actual <= 1e-11, actual
    assert actual <= s.rel_error_estimate


def test_split_kernel_shards_and_resident(engine, pb):
    rng = np.random.default_rng(980)
    A = 1.0 - rng.random((25, 25))
    whole = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_SPLIT)
    parts = [engine.exact_dense_shard(A, s, 5, variant=pb.PERM_KERNEL_DENSE_SPLIT) for s in range(5)]
    assert all(p.kernel == pb.PERM_KERNEL_DENSE_SPLIT for p in parts)
    assert sum(p.steps for p in parts) == 2.0 ** 24
    assert rel_err(pb.dd_sum([(p.hi, p.lo) for p in parts])[0], whole.value) < 1e-13
    res = engine.upload_dense(A, variant=pb.PERM_KERNEL_DENSE_SPLIT)
    try:
        assert res.run().value == whole.value
    finally:
        res.free()


def test_split_kernel_order_limits(engine, pb):
    for n in (3, 41):
        with pytest.raises(pb.PermError) as ei:
            engine.exact_dense(np.ones((n, n)), variant=pb.PERM_KERNEL_DENSE_SPLIT)
        assert ei.value.status == pb.PERM_EUNSUPPORTED


@pytest.mark.parametrize("n", [31, 33])
def test_policy_certified_stage_meets_the_target(engine, pb, n):
    """Where the FP64-X bound misses the target (and the cross-check, where
    it runs, fails), positive real requests end on the certified split-dd
    walk; whichever kernel the policy ends on, the value is within 1e-10 of
    double-double and no split-X pass runs."""
    rng = np.random.default_rng(990 + n)
    A = 1.0 - rng.random((n, n))
    d = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_DD)
    auto = engine.exact_dense(A)
    assert auto.kernel in (pb.PERM_KERNEL_DENSE, pb.PERM_KERNEL_DENSE_SDD)
    assert abs(auto.value - d.value) <= 1e-10 * abs(d.value)
    assert auto.rel_error_estimate <= 1e-10


def test_split_kernel_exact_term_moments(engine, pb):
    """The split walk sums |term| over its own terms: abs_term_sum is the exact
    sum of |2 prod_j x_j(S)| over all 2^(n-1) subsets S (numpy, order 13)."""
    n = 13
    rng = np.random.default_rng(995)
    A = rng.standard_normal((n, n))
    x0 = A[:, n - 1] - A.sum(axis=1) / 2
    S = ((np.arange(2 ** (n - 1))[:, None] >> np.arange(n - 1)) & 1).astype(float)
    X = x0[None, :] + S @ A[:, : n - 1].T
    want = 2.0 * np.abs(np.prod(X, axis=1)).sum()
    r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_SPLIT)
    assert rel_err(r.abs_term_sum, want) < 1e-12, (r.abs_term_sum, want)


def test_term_moment_sample_is_exact_for_small_orders(engine, pb):
    """Every subset-size class of an order-16 walk fits the per-class sample
    (C(15, k) <= 6435), so the stratified sample enumerates all 2^15 terms."""
    n = 16
    rng = np.random.default_rng(996)
    for A in (rng.standard_normal((n, n)), 1.0 - rng.random((n, n))):
        x0 = A[:, n - 1] - A.sum(axis=1) / 2
        S = ((np.arange(2 ** (n - 1))[:, None] >> np.arange(n - 1)) & 1).astype(float)
        want = 2.0 * np.abs(np.prod(x0[None, :] + S @ A[:, : n - 1].T, axis=1)).sum()
        r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE)
        assert rel_err(r.abs_term_sum, want) < 1e-12, (r.abs_term_sum, want)


@pytest.mark.parametrize("n", [22, 28, 33])
def test_term_moment_sample_tracks_the_exact_sum(engine, pb, n):
    """The stratified sample's sum |term| against the split walk's exact one:
    within 10% on positive, sparse positive and sparse integer matrices,
    whose term sizes are set mostly by the subset size.  (Signed Gaussian
    matrices have heavy-tailed terms within each class: there the sample is
    only an order-of-magnitude estimate, and the policy's transpose
    cross-check carries the decision.)"""
    rng = np.random.default_rng(997 + n)
    kinds = (1.0 - rng.random((n, n)), (rng.random((n, n)) < 0.5) * (1.0 - rng.random((n, n))),
             bernoulli(rng, n, 0.5) * rng.integers(1, 5, (n, n)))
    for A in kinds:
        f = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE)
        s = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_SPLIT)
        assert abs(f.abs_term_sum / s.abs_term_sum - 1.0) < 0.1, (f.abs_term_sum, s.abs_term_sum)
    G = rng.standard_normal((n, n))
    f = engine.exact_dense(G, variant=pb.PERM_KERNEL_DENSE)
    s = engine.exact_dense(G, variant=pb.PERM_KERNEL_DENSE_SPLIT)
    assert 0.1 < f.abs_term_sum / s.abs_term_sum < 10.0


def test_policy_predicts_the_fp64_bound_before_the_walk(engine, pb):
    """Nonnegative real matrices of order 28..40: the policy predicts the
    FP64-X walk's bound before any walk (stratified sample of sum|term| and a
    weighted-Rasmussen size estimate of perm) and, above 1.5x the target,
    runs the certified split-dd walk alone.  The prediction is checked
    against the bound of the FP64-X walk itself; the routing against the
    planned kernel; the value against the FP64-X value within its bound.
    Density-0.5 U(0,1] matrices: at order 28 the FP64-X bound is near
    0.8-0.9e-10 (FP64 X goes first and passes), at order 33 near 1e-9."""
    rng = np.random.default_rng(5555)
    mats = {}
    for n in (26, 28, 30, 31, 32, 33):
        for rep in range(3):
            A = (rng.random((n, n)) < 0.5) * (1.0 - rng.random((n, n)))
            if rep == 0 and n in (28, 33):
                mats[n] = A
    for n, A in mats.items():
        kernel, predicted = engine.dense_plan(A)
        f = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE)
        assert predicted > 0.0
        assert f.rel_error_estimate / 3.0 <= predicted <= 3.0 * f.rel_error_estimate, (n, predicted, f)
        assert kernel == (pb.PERM_KERNEL_DENSE_SDD if predicted > 1.5e-10 else 0)
        assert kernel == (0 if n == 28 else pb.PERM_KERNEL_DENSE_SDD), (n, predicted)
        auto = engine.exact_dense(A)
        assert auto.kernel == (pb.PERM_KERNEL_DENSE if n == 28 else pb.PERM_KERNEL_DENSE_SDD)
        if n == 33:
            assert auto.kernel_ms < 1.5 * engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_SDD).kernel_ms
        assert auto.rel_error_estimate <= 1e-10
        assert abs(auto.value - f.value) <= (f.rel_error_estimate + auto.rel_error_estimate) * abs(f.value)
    # no prediction: below order 28, signed entries, integer matrices (certified first)
    assert engine.dense_plan(1.0 - rng.random((24, 24))) == (0, 0.0)
    assert engine.dense_plan(rng.standard_normal((30, 30))) == (0, 0.0)
    assert engine.dense_plan(rng.integers(0, 4, (30, 30)).astype(float)) == (pb.PERM_KERNEL_DENSE_INT_DD, 0.0)
