"""Certified kernels on the B200: int32 X with double-double products and sum
(PERM_KERNEL_DENSE_INT_DD) and split-dd (PERM_KERNEL_DENSE_SDD, dense and
sparse layouts).  Each result carries a worst-case bound (rel_error_estimate)
built from the walk's own sum |term|; the tests check that the bound covers
the actual error against the oracle -- the exact multi-modular integer
permanent, the CPU double-double Ryser -- and that the automatic path with the
1e-10 target ends on these kernels where the policy says it should."""
import numpy as np
import pytest
from conftest import bernoulli, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _covers(r, want, slack=0.0):
    """|value - want| <= bound * |want| (+ slack for the oracle's own rounding)."""
    err = abs(r.value - want)
    return err <= r.rel_error_estimate * abs(want) + slack, (r.value, want, err / abs(want), r.rel_error_estimate)


@pytest.mark.parametrize("n", [8, 9, 13, 17, 20, 24, 27])
def test_int_dd_vs_exact(engine, orc, pb, n):
    rng = np.random.default_rng(700 + n)
    cases = {
        "u1to4": bernoulli(rng, n, 0.5) * rng.integers(1, 5, (n, n)),
        "signed": rng.integers(-3, 4, (n, n)).astype(float),
        "binary": bernoulli(rng, n, 0.5),
        "large": rng.integers(0, 60, (n, n)).astype(float),  # small product groups
    }
    layouts, levels = set(), set()
    for kind, A in cases.items():
        g, pair, ngo, _, _ = pb.intc_layout(A)
        layouts.add((g, pair))
        levels.add(ngo > 0)
        exact = orc.perm_exact_int(A)[0]
        r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_INT_DD)
        assert r.kernel == pb.PERM_KERNEL_DENSE_INT_DD
        if exact == 0:
            assert abs(r.value) <= r.rel_error_estimate * max(r.abs_term_sum, 1.0), (kind, r.value)
            continue
        ok, info = _covers(r, exact)
        assert ok, (kind, info)
        assert r.rel_error_estimate < 1e-20, (kind, r.rel_error_estimate)  # u^2-level bound
        assert rel_err(r.value, exact) <= 1.2e-16  # value is the pair rounded once (<= 2^-53)
    if n >= 16:  # both product layouts ran: exact int64 pairs of groups and the plain chain
        assert {p for _, p in layouts} == {True, False}, layouts
    if n >= 20:  # and the two-level row layout beside the one-level walk
        assert True in levels, levels


@pytest.mark.parametrize("n,d,seed", [(24, 0.3, 1), (26, 0.3, 0), (27, 0.4, 2)])
def test_int_dd_two_level_groups_of_6_vs_exact(engine, orc, pb, n, d, seed):
    """Sparse 0/1 matrices whose certified walk takes the two-level row
    layout with groups of 6 in int64 pairs: exact against the multi-modular
    oracle within the walk's own bound."""
    rng = np.random.default_rng(seed)
    A = bernoulli(rng, n, d)
    g, pair, ngo, _, _ = pb.intc_layout(A)
    assert g == 6 and pair and ngo >= 2
    exact = orc.perm_exact_int(A)[0]
    r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_INT_DD)
    if exact == 0:
        assert abs(r.value) <= r.rel_error_estimate * max(r.abs_term_sum, 1.0)
    else:
        ok, info = _covers(r, exact)
        assert ok, info
        assert rel_err(r.value, exact) <= 1.2e-16


@pytest.mark.parametrize("n", [28, 30])
def test_int_dd_three_level_vs_exact(engine, orc, pb, n):
    """The certified walk in the three-level row layout (column 0's rows,
    the further rows of columns 1 and 2, the rest) on dense U{1..4} and 0/1
    matrices: the exact permanent inside the walk's bound, the value the
    exact one rounded once."""
    rng = np.random.default_rng(650 + n)
    for kind, A in (("u1to4", bernoulli(rng, n, 0.5) * rng.integers(1, 5, (n, n))), ("binary", bernoulli(rng, n, 0.5))):
        g, pair, ngo, ng1, ng2 = pb.intc_layout(A)
        assert ngo == 0 and ng1 >= 2 and ng2 >= 1, (kind, g, pair, ngo, ng1, ng2)
        exact = orc.perm_exact_int(A)[0]
        r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_INT_DD)
        ok, info = _covers(r, exact)
        assert ok, (kind, info)
        # u^2-level: dominated by K^2 u^2 S1 / |perm|, K ~ 2^n / threads terms per thread
        assert r.rel_error_estimate < 1e-18, (kind, r.rel_error_estimate)
        assert rel_err(r.value, exact) <= 1.2e-16, kind


def test_int_dd_golden_n32(engine, golden, pb):
    """The headline distribution at the oracle's largest size (n=32, exact)."""
    c = golden["cfg3_int_n32_d050"]
    exact = int(c["exact"])
    r = engine.exact_dense(c["A"], variant=pb.PERM_KERNEL_DENSE_INT_DD)
    ok, info = _covers(r, exact)
    assert ok, info
    assert r.rel_error_estimate <= TOL
    # the automatic path with the 1e-10 target runs this kernel first
    a = engine.exact_dense(c["A"])
    assert a.kernel == pb.PERM_KERNEL_DENSE_INT_DD and a.value == r.value


@pytest.mark.slow
@pytest.mark.parametrize("n", [36, 40])
def test_int_dd_full_size_vs_double_double(engine, pb, n):
    """At the benchmark sizes: the certified int32-X value against the
    double-double kernel (itself pinned to the CPU double-double oracle), both
    bounds covering the difference; the automatic path certifies 1e-10 with
    this one kernel."""
    rng = np.random.default_rng(303 if n == 40 else n)
    while True:
        m = rng.random((n, n)) < 0.5
        if m.any(0).all() and m.any(1).all():
            break
    A = (m * rng.integers(1, 5, (n, n))).astype(np.int32)
    c = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_INT_DD)
    d = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_DD)
    assert c.rel_error_estimate <= TOL
    assert abs(c.value - d.value) <= (c.rel_error_estimate + d.rel_error_estimate) * abs(d.value) + 1e-15 * abs(d.value)
    a = engine.exact_dense(A)
    assert a.kernel == pb.PERM_KERNEL_DENSE_INT_DD and a.rel_error_estimate <= TOL
    assert a.value == c.value


@pytest.mark.parametrize("n", [4, 5, 7, 11, 16, 20, 24])
def test_sdd_dense_vs_oracle_dd(engine, orc, pb, n):
    rng = np.random.default_rng(800 + n)
    for kind in ("real", "signed", "sparse"):
        if kind == "real":
            A = 1.0 - rng.random((n, n))
        elif kind == "signed":
            A = rng.standard_normal((n, n))
        else:
            A = bernoulli(rng, n, 0.3) * (1.0 - rng.random((n, n)))
        r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_SDD)
        assert r.kernel == pb.PERM_KERNEL_DENSE_SDD
        hi, lo = orc.perm_dd(A)
        want = hi + lo
        # the oracle's own double-double error: (4n + 32) u^2 sum|t|
        slack = (4 * n + 32) * 2.0 ** -106 * r.abs_term_sum
        ok, info = _covers(r, want, slack)
        assert ok, (kind, info)
        assert r.rel_error_estimate < 1e-18 or abs(want) < 1e-12 * r.abs_term_sum, (kind, r.rel_error_estimate)
        assert abs(r.value - want) <= 1.2e-16 * abs(want) + slack + r.rel_error_estimate * abs(want)


@pytest.mark.parametrize("n,d", [(12, 0.2), (16, 0.2), (20, 0.25), (24, 0.2), (26, 0.3), (28, 0.2)])
def test_sdd_sparse_layout_vs_oracle_dd(engine, orc, pb, n, d):
    """Sparse real matrices: the layout that walks only the rows of the three
    sparsest columns at seven of eight steps, against the CPU double-double
    Ryser; the automatic path (dense and CRS/CCS entry points) runs it first
    where its FP64 operations per Gray step are no more than FP64 X's, and
    meets 1e-10 either way."""
    rng = np.random.default_rng(900 + n)
    # a Bernoulli pattern plus a random permutation: a perfect matching exists,
    # so the permanent is positive and the relative bound is meaningful
    mask = (bernoulli(rng, n, d) + np.eye(n)[rng.permutation(n)]) > 0
    A = mask * (1.0 - rng.random((n, n)))
    inner = pb.sdd_layout(A)
    assert inner in (6, 8, 12, 16), inner
    r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_SDD)
    hi, lo = orc.perm_dd(A)
    want = hi + lo
    slack = (4 * n + 32) * 2.0 ** -106 * r.abs_term_sum
    ok, info = _covers(r, want, slack)
    assert ok, info
    assert r.rel_error_estimate <= TOL
    a = engine.exact_dense(A)
    if 7 * (6 * inner + 9) + 6 * n + 5 <= 16 * n:
        assert engine.dense_plan(A)[0] == pb.PERM_KERNEL_DENSE_SDD
    if a.kernel == pb.PERM_KERNEL_DENSE_SDD:
        assert a.value == r.value
    else:
        assert a.kernel == pb.PERM_KERNEL_DENSE
    assert a.rel_error_estimate <= TOL and rel_err(a.value, want) <= TOL
    s = engine.exact_sparse_matrix(A)
    assert s.kernel in (pb.PERM_KERNEL_DENSE, pb.PERM_KERNEL_DENSE_SDD, pb.PERM_KERNEL_SKIPPER)
    assert rel_err(s.value, want) < TOL


def _sdd_vs_oracle(engine, orc, pb, A):
    n = A.shape[0]
    r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_SDD)
    hi, lo = orc.perm_dd(A)
    want = hi + lo
    slack = (4 * n + 32) * 2.0 ** -106 * r.abs_term_sum
    ok, info = _covers(r, want, slack)
    assert ok, info
    assert r.rel_error_estimate <= TOL
    a = engine.exact_dense(A)
    assert a.rel_error_estimate <= TOL and rel_err(a.value, want) <= TOL


@pytest.mark.parametrize("n,seed,levels", [(24, 1, (12, 16)), (26, 0, (8, 20)), (27, 2, (12, 20)), (28, 10, (8, 16)),
                                           (30, 11, (12, 24))])
def test_sdd_three_level_vs_oracle_dd(engine, orc, pb, n, seed, levels):
    """Dense real matrices (density 1/2): split-dd walks column 0's rows
    (R1) at half of the steps and those of columns 0..2 (R2) at three in
    eight -- the three-level layout; against the CPU double-double Ryser,
    and the automatic path certifies 1e-10."""
    rng = np.random.default_rng(seed)
    A = (rng.random((n, n)) < 0.5) * (1.0 - rng.random((n, n)))
    assert pb.sdd_levels(A) == levels
    _sdd_vs_oracle(engine, orc, pb, A)


@pytest.mark.parametrize("seed", [0, 2])
def test_sdd_three_level_second_level_28_vs_oracle_dd(engine, orc, pb, seed):
    """Order 30, column 0 on rows 0..15, columns 1 and 2 on rows 0..27, the
    rest dense: the three-level layout with 28 rows in registers (2 CTAs per
    SM)."""
    rng = np.random.default_rng(seed)
    n = 30
    mask = rng.random((n, n)) < 0.9
    mask[16:, 0] = False
    mask[:16, 0] = True
    mask[:, 1:3] = False
    mask[16:28, 1:3] = rng.random((12, 2)) < 0.7
    mask[16:28, 1] |= ~mask[16:28, 2]
    mask[:16, 1:3] = rng.random((16, 2)) < 0.25
    A = mask * (1.0 - rng.random((n, n)))
    r1, r2 = pb.sdd_levels(A)
    assert r1 in (8, 12, 16) and r2 == 28, (r1, r2)
    _sdd_vs_oracle(engine, orc, pb, A)


@pytest.mark.parametrize("n,seed", [(27, 1), (28, 2)])
def test_sdd_two_level_rolled_vs_oracle_dd(engine, orc, pb, n, seed):
    """Three columns on the same 20 rows and every other column on 21 or
    more (no cheaper three-level layout): split-dd walks 20 inner rows at
    seven of eight steps (the rolled two-level loop); against the CPU
    double-double Ryser, and the automatic path certifies 1e-10."""
    rng = np.random.default_rng(seed)
    mask = rng.random((n, n)) < 0.9
    mask[20:, :3] = False
    mask[:20, :3] |= rng.random((20, 3)) < 0.5
    A = mask * (1.0 - rng.random((n, n)))
    assert pb.sdd_levels(A) == (0, 20)
    inner = pb.sdd_layout(A)
    assert inner == 20, inner
    r = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_SDD)
    hi, lo = orc.perm_dd(A)
    want = hi + lo
    slack = (4 * n + 32) * 2.0 ** -106 * r.abs_term_sum
    ok, info = _covers(r, want, slack)
    assert ok, info
    assert r.rel_error_estimate <= TOL
    a = engine.exact_dense(A)
    assert a.rel_error_estimate <= TOL and rel_err(a.value, want) <= TOL


def test_cfg2_full_size_against_golden(engine, golden, pb, orc):
    """The sparse exact configuration at its stated size (n=36, density 0.20,
    values U(0,1]) against the CPU double-double oracle's value recorded in
    the golden file: the automatic SkipPer entry point certifies 1e-10 with
    the split-dd sparse layout; forced SkipPer (FP64 X) is within 1e-10 too.
    The reference's own SkipPer value, recorded beside it, is reported."""
    if "cfg2_sparse_real_n36_d020" not in golden:
        pytest.skip("n=36 golden case not generated")
    c = golden["cfg2_sparse_real_n36_d020"]
    A = c["A"]
    want = c["dd"][0] + c["dd"][1]
    cmp = pb.compress(2, A)
    auto = engine.exact_sparse(cmp["n"], cmp["rptrs"], cmp["cols"], cmp["rvals"], cmp["cptrs"], cmp["rows"],
                               cmp["cvals"])
    assert auto.kernel == pb.PERM_KERNEL_DENSE_SDD
    assert auto.rel_error_estimate <= TOL
    assert rel_err(auto.value, want) <= max(auto.rel_error_estimate, 1e-15)
    sk = engine.exact_sparse(cmp["n"], cmp["rptrs"], cmp["cols"], cmp["rvals"], cmp["cptrs"], cmp["rows"],
                             cmp["cvals"], variant=pb.PERM_KERNEL_SKIPPER)
    assert rel_err(sk.value, want) < TOL
    ref = c.get("ref_skip_balanced_skiporder")
    if ref is not None:
        print(f"reference SkipPer (CPU, double X) rel error vs dd: {rel_err(ref, want):.3e}")


def test_policy_integer_goes_certified_directly(engine, orc, pb):
    rng = np.random.default_rng(31)
    A = bernoulli(rng, 26, 0.5) * rng.integers(1, 5, (26, 26))
    exact = orc.perm_exact_int(A)[0]
    r = engine.exact_dense(A)
    assert r.kernel == pb.PERM_KERNEL_DENSE_INT_DD
    assert r.rel_error_estimate <= TOL
    ok, info = _covers(r, exact)
    assert ok, info
    # with the policy off the plain int32-X walk runs (one evaluation)
    engine.set_rel_target(0.0)
    try:
        p = engine.exact_dense(A)
        assert p.kernel == pb.PERM_KERNEL_DENSE_INT
        assert rel_err(p.value, exact) < 1e-12
    finally:
        engine.set_rel_target(1e-10)


def test_certified_shards_and_sparse_variants(engine, pb):
    """Forced certified variants through the sparse entry point and as shards
    (shards sum to the whole walk)."""
    rng = np.random.default_rng(41)
    A = bernoulli(rng, 22, 0.3) * rng.integers(1, 4, (22, 22))
    whole = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_INT_DD)
    hi = lo = 0.0
    for s in range(3):
        r = engine.exact_dense_shard(A, s, 3, variant=pb.PERM_KERNEL_DENSE_INT_DD)
        hi, lo = hi + r.hi, lo + r.lo
    assert rel_err(hi + lo, whole.value) < 1e-14
    for v in (pb.PERM_KERNEL_DENSE_INT_DD, pb.PERM_KERNEL_DENSE_SDD):
        s = engine.exact_sparse_matrix(A.astype(float), variant=v)
        assert s.kernel == v and rel_err(s.value, whole.value) < 1e-14


def test_bounded_wait_expires_and_context_survives(pb):
    """Failure detection without a GPU fault: an injected barrier that never
    completes makes the FP64-X kernel's staging wait and the tensor-core
    kernel's pipeline wait give up after their limit; the call fails with
    PERM_ETIMEOUT and a message naming the wait, and the next normal call on
    the same context returns the right permanent."""
    rng = np.random.default_rng(77)
    A = bernoulli(rng, 24, 0.5) * rng.integers(1, 5, (24, 24))
    with pb.Engine(0) as eng:
        eng.set_rel_target(-1.0)  # one evaluation per call
        want = eng.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_INT).value
        for variant, what in ((pb.PERM_KERNEL_DENSE, "staging"), (pb.PERM_KERNEL_DENSE_TC, "tensor-core pipeline")):
            eng.inject_wait_timeout(1)
            with pytest.raises(pb.PermError) as ei:
                eng.exact_dense(A, variant=variant)
            assert ei.value.status == pb.PERM_ETIMEOUT
            assert what in str(ei.value) and "timed out" in str(ei.value)
            again = eng.exact_dense(A, variant=variant)
            assert rel_err(again.value, want) < 1e-13, (variant, again.value, want)
