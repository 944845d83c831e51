"""Batched persistent kernel: every matrix of a mixed-order batch equals the
single-matrix kernel's result and the oracle within 1e-10 relative (the two
kernels cut the Gray walk differently, so real-valued matrices with heavy
cancellation differ in the last ~12 digits)."""
import numpy as np
import pytest
from conftest import bernoulli, rel_err

pytestmark = pytest.mark.gpu


def mixed_batch(rng, count, lo, hi):
    mats = []
    for i in range(count):
        n = int(rng.integers(lo, hi + 1))
        d = rng.uniform(0.2, 0.9)
        m = bernoulli(rng, n, d) if n > 1 else np.ones((1, 1))
        if i % 2:
            m = m * (1.0 - rng.random((n, n)))
        mats.append(m)
    return mats


def test_batch_matches_single_matrix_kernel(engine, pb):
    rng = np.random.default_rng(404)
    mats = mixed_batch(rng, 300, 1, 26) + [np.ones((n, n)) for n in (1, 2, 3, 8, 9)]
    vals, ms = engine.batch_exact(mats)
    assert ms > 0
    for m, v in zip(mats, vals):
        want = engine.exact_dense(m, variant=pb.PERM_KERNEL_DENSE).value
        # a binary matrix without a perfect matching has permanent 0; both
        # kernels then return rounding noise of order 1e-17
        assert rel_err(v, want) < 1e-10 or abs(v - want) < 1e-12, (m.shape, v, want)


def test_batch_vs_oracle_and_golden(engine, orc, golden):
    cases = [c for c in golden.values() if c["n"] <= 40]
    vals, _ = engine.batch_exact([c["A"] for c in cases])
    for c, v in zip(cases, vals):
        want = int(c["exact"]) if "exact" in c else c["dd"][0] + c["dd"][1]
        assert rel_err(v, want) < 1e-10, c["name"]
    rng = np.random.default_rng(5)
    mats = [rng.standard_normal((n, n)) for n in (10, 13, 17)]
    vals, _ = engine.batch_exact(mats)
    for m, v in zip(mats, vals):
        hi, lo = orc.perm_dd(m)
        assert abs(v - (hi + lo)) <= 1e-9 * max(abs(hi), 1e-300)


def test_batch_is_deterministic_and_replayable(engine):
    rng = np.random.default_rng(9)
    b = engine.batch(mixed_batch(rng, 200, 9, 24))
    try:
        v1, _ = b.run()
        v2, _ = b.run()
        np.testing.assert_array_equal(v1, v2)
    finally:
        b.free()


def test_autotune_keeps_results(engine, pb):
    rng = np.random.default_rng(10)
    mats = mixed_batch(rng, 64, 12, 22)
    before, _ = engine.batch_exact(mats)
    table = engine.batch_autotune(12, 22)
    assert all(3 <= m <= n - 6 for n, m in table.items())
    after, _ = engine.batch_exact(mats)
    for a, b in zip(before, after):
        assert rel_err(a, b) < 1e-12


def test_batch_rejects_large_order(engine, pb):
    with pytest.raises(pb.PermError):
        engine.batch_exact([np.ones((41, 41))])


def test_batch_error_estimates_and_reruns(engine, orc, pb):
    rng = np.random.default_rng(12)
    mats = [rng.standard_normal((n, n)) for n in (12, 15, 18, 20)]
    b = engine.batch(mats)
    try:
        vals, est, reruns, _ = b.run_ex()
        for m, v, e in zip(mats, vals, est):
            hi, lo = orc.perm_dd(m)
            assert abs(v - hi - lo) / abs(hi) <= max(e, 1e-15)
        # a zero pattern without a perfect matching: exactly 0, estimate 0
        Z = rng.random((16, 16))
        Z[:, 3] = 0.0
        bz = engine.batch([Z])
        try:
            vz, ez, _, _ = bz.run_ex()
            assert vz[0] == 0.0 and ez[0] == 0.0
        finally:
            bz.free()
        engine.set_rel_target(1e-16)  # unreachable in FP64: every matrix reruns in double-double
        vals, est, reruns, _ = b.run_ex()
        assert reruns == len(mats)
        for m, v, e in zip(mats, vals, est):
            hi, lo = orc.perm_dd(m)
            assert abs(v - hi - lo) <= 1e-15 * abs(hi) and e < 1e-20
    finally:
        engine.set_rel_target(1e-10)
        b.free()


def test_integer_matrices_take_int32_x_exactly(engine, orc):
    """0/1 and small-integer matrices (groups of 5-6 rows fit in int32) walk
    y = 2x in int32 inside the batch; larger entries stay in FP64 X.  All
    agree with the exact oracle, including integer permanents above 2^53."""
    rng = np.random.default_rng(77)
    mats = []
    for n in (9, 12, 17, 22, 26):
        mats.append((rng.random((n, n)) < 0.5).astype(np.float64))
    for n in (10, 16, 24):
        mats.append(rng.integers(-2, 3, (n, n)).astype(np.float64))
    mats.append(rng.integers(0, 200, (14, 14)).astype(np.float64))  # groups do not fit: FP64 X
    b = engine.batch(mats)
    try:
        vals, est, _, _ = b.run_ex()
    finally:
        b.free()
    for A, v, e in zip(mats, vals, est):
        exact = orc.perm_exact_int(A)[0]
        if exact == 0:
            assert abs(v) <= 1e-9
        else:
            assert abs(v - exact) <= max(1e-10, e) * abs(exact), (A.shape[0], v, exact, e)


def test_order_35_binary_in_batch_matches_single_kernel(engine, pb):
    """Groups of 6 rows still fit at order 35 (35^6 < 2^31): the batch's int32
    walk against the single-matrix int32-X kernel (the CPU oracle is too slow
    at this order)."""
    rng = np.random.default_rng(78)
    A = (rng.random((35, 35)) < 0.5).astype(np.float64)
    vals, _ = engine.batch_exact([A])
    single = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_INT).value
    assert abs(vals[0] - single) <= 1e-12 * abs(single)


def test_sparse_layout_in_the_batch(engine, orc, pb):
    """Sparse matrices walk the two-level layout inside the batch (FP64 X with
    8 or 16 inner rows, int32 X with 6 or 12 and vanishing-group skips):
    every result agrees with the oracle (exact for integers, double-double for
    reals) exactly as the dense walk's would."""
    rng = np.random.default_rng(91)
    mats = []
    for n in (12, 14, 17, 20, 23, 26):
        for d in (0.15, 0.25):
            P = (bernoulli(rng, n, d) + np.eye(n)[rng.permutation(n)]) > 0
            mats.append(P.astype(np.float64))                          # 0/1
            mats.append(P * rng.integers(1, 4, (n, n)).astype(float))   # small integers
            mats.append(P * (1.0 - rng.random((n, n))))                 # real
    assert sum(pb.sdd_layout(m) > 0 for m in mats) >= len(mats) // 2
    # sparse matrices cancel heavily (small permanents, large terms): the
    # batch's plain int32-X / FP64-X walks are accurate to ~1e-13 here; a
    # layout bookkeeping error would be of order 1
    vals, _ = engine.batch_exact(mats)
    for m, v in zip(mats, vals):
        if np.all(m == np.round(m)):
            want = orc.perm_exact_int(m)[0]
        else:
            hi, lo = orc.perm_dd(m)
            want = hi + lo
        assert rel_err(v, want) < 1e-11, (m.shape, v, want)


def test_dense_two_level_layout_in_the_batch(engine, orc, pb):
    """Dense matrices (density 1/2) whose three sparsest columns still miss a
    quarter or more of the rows walk the two-level layout with 18..24 inner
    rows inside the batch: against the oracle at orders 25..28 and against
    single-matrix walks at 30..32."""
    rng = np.random.default_rng(92)
    small, large = [], []
    for n in (25, 27, 28, 30, 31, 32):
        P = (rng.random((n, n)) < 0.5) | (np.eye(n)[rng.permutation(n)] > 0)
        trio = [P.astype(np.float64), P * rng.integers(1, 4, (n, n)).astype(float), P * (1.0 - rng.random((n, n)))]
        (small if n <= 28 else large).extend(trio)
    vals, _ = engine.batch_exact(small + large)
    for m, v in zip(small, vals[:len(small)]):
        if np.all(m == np.round(m)):
            want = orc.perm_exact_int(m)[0]
        else:
            hi, lo = orc.perm_dd(m)
            want = hi + lo
        assert rel_err(v, want) < 1e-11, (m.shape, v, want)
    for m, v in zip(large, vals[len(small):]):
        one = engine.exact_dense(m, variant=pb.PERM_KERNEL_DENSE)
        assert rel_err(v, one.value) < 1e-10 + 2 * one.rel_error_estimate, (m.shape, v, one.value)


def test_every_batch_variant_agrees(pb, orc):
    """Each compiled batch kernel variant (threads per block, register budget,
    shared-memory X) returns the same permanents, to rounding, on a batch of
    dense and sparse, 0/1 and real matrices of orders 9..28."""
    rng = np.random.default_rng(93)
    mats = mixed_batch(rng, 80, 9, 22)
    for n in (24, 26, 28):
        mats.append(bernoulli(rng, n, 0.3) * (1.0 - rng.random((n, n))))
        mats.append(bernoulli(rng, n, 0.7))
    with pb.Engine(0) as eng:
        eng.set_rel_target(-1.0)
        ref = [eng.exact_dense(m, variant=pb.PERM_KERNEL_DENSE).value for m in mats]
        for v in range(6):
            eng.batch_use_variant(v)
            vals, _ = eng.batch_exact(mats)
            assert eng.batch_variant()["variant"] == v
            for m, a, b in zip(mats, vals, ref):
                assert abs(a - b) <= 1e-10 * abs(b) or abs(a - b) < 1e-12, (v, m.shape, a, b)


def test_batch_variants_agree_and_autotune_picks_one(pb):
    """The autotuner measures the compiled batch kernel variants (threads per
    block, register budget, shared-memory X), keeps one, and later batches
    run it with the same permanents (to rounding) as the general variant."""
    rng = np.random.default_rng(92)
    mats = mixed_batch(rng, 120, 9, 24)
    with pb.Engine(0) as eng:
        base, _ = eng.batch_exact(mats)
        table = eng.batch_autotune(9, 24)
        assert set(table) == set(range(9, 25))
        v = eng.batch_variant()
        assert 0 <= v["variant"] < 6 and v["max_order"] >= 24
        tuned, _ = eng.batch_exact(mats)
        for a, b in zip(base, tuned):
            assert abs(a - b) <= 1e-11 * abs(b) or abs(a - b) < 1e-12
