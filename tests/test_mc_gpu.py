"""Monte-Carlo trial kernels on the B200: per-trial weights bit-identical to the
oracle's CPU restatement (same Philox streams, same FP64 operation order), and
estimates within the stated standard error of the exact permanent."""
import math

import numpy as np
import pytest
from conftest import bernoulli

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 7, 20, 33, 64])
def test_rasmussen_trials_bit_identical(engine, orc, n):
    rng = np.random.default_rng(n)
    A = bernoulli(rng, n, 0.5) if n > 1 else np.ones((1, 1))
    e = engine.rasmussen(A, 3000, seed=42, keep_trials=True)
    want = orc.rasmussen_trials(A, 42, 0, 3000)
    np.testing.assert_array_equal(e.trial_values, want)


@pytest.mark.parametrize("n,y,z", [(6, 1, 1), (20, 4, 5), (40, 4, 5), (64, 2, 3)])
def test_scaling_trials_bit_identical(engine, orc, n, y, z):
    rng = np.random.default_rng(100 + n)
    A = bernoulli(rng, n, 0.5)
    e = engine.scaling(A, 1000, y, z, seed=7, keep_trials=True)
    want = orc.scaling_trials(A, y, z, 7, 0, 1000)
    np.testing.assert_array_equal(e.trial_values, want)


@pytest.mark.parametrize("n", [9, 33, 64])
def test_scaling_trials_bit_identical_weighted(engine, orc, n):
    """Entries other than 0/1 take the general scaling kernel (Sinkhorn sums
    over the values); 0/1 matrices take the mask kernel: both match the oracle
    bit for bit."""
    rng = np.random.default_rng(300 + n)
    A = bernoulli(rng, n, 0.5) * rng.integers(1, 4, (n, n))
    e = engine.scaling(A, 500, 3, 4, seed=11, keep_trials=True)
    np.testing.assert_array_equal(e.trial_values, orc.scaling_trials(A, 3, 4, 11, 0, 500))


def test_estimates_within_standard_error(engine, orc):
    rng = np.random.default_rng(5)
    A = bernoulli(rng, 16, 0.5)
    exact = orc.perm_exact_int(A)[0]
    r = engine.rasmussen(A, 200000, seed=1)
    s = engine.scaling(A, 200000, 4, 5, seed=2)
    for est in (r, s):
        assert est.std_error > 0
        assert abs(est.mean - exact) < 5 * est.std_error
    assert s.std_error < r.std_error  # scaling reduces the variance


def test_mean_matches_trial_values(engine):
    rng = np.random.default_rng(6)
    A = bernoulli(rng, 30, 0.5)
    e = engine.scaling(A, 5000, seed=3, keep_trials=True)
    assert abs(e.mean - e.trial_values.mean()) <= 1e-12 * abs(e.mean)
    assert e.zero_trials == float((e.trial_values == 0).sum())


def test_streams_independent_of_trial_count(engine):
    rng = np.random.default_rng(7)
    A = bernoulli(rng, 25, 0.5)
    a = engine.rasmussen(A, 1000, seed=9, keep_trials=True).trial_values
    b = engine.rasmussen(A, 77777, seed=9, keep_trials=True).trial_values
    np.testing.assert_array_equal(a, b[:1000])


def test_trial_ranges_are_the_whole_runs_trials(engine, pb):
    """perm_approx_*_range: trials [t0, t0 + k) of the same streams give the
    whole run's weights bit for bit, and ranges' sums add up to its sums
    (the multi-GPU split by trial id)."""
    rng = np.random.default_rng(8)
    A = bernoulli(rng, 30, 0.5)
    whole = engine.rasmussen(A, 3000, seed=4, keep_trials=True)
    lo = engine.rasmussen(A, 1234, seed=4, keep_trials=True)
    hi = engine.rasmussen(A, 1766, seed=4, keep_trials=True, trial0=1234)
    np.testing.assert_array_equal(np.concatenate([lo.trial_values, hi.trial_values]), whole.trial_values)
    assert abs((lo.sum + hi.sum) - whole.sum) <= 1e-13 * abs(whole.sum)
    s_whole = engine.scaling(A, 600, 4, 5, seed=6, keep_trials=True)
    s_hi = engine.scaling(A, 250, 4, 5, seed=6, keep_trials=True, trial0=350)
    np.testing.assert_array_equal(s_hi.trial_values, s_whole.trial_values[350:])
    # the sparse forms: below and above order 64 (bitset kernel)
    for n in (30, 100):
        B = bernoulli(rng, n, 0.3 if n == 30 else 0.05)
        c = pb.compress(0, B)
        w = engine.rasmussen_sparse(n, c["rptrs"], c["cols"], 900, seed=2, keep_trials=True)
        h = engine.rasmussen_sparse(n, c["rptrs"], c["cols"], 400, seed=2, keep_trials=True, trial0=500)
        np.testing.assert_array_equal(h.trial_values, w.trial_values[500:])
        sw = engine.scaling_sparse(n, c["rptrs"], c["cols"], c["cptrs"], c["rows"], 300, 4, 5, seed=3,
                                   keep_trials=True)
        sh = engine.scaling_sparse(n, c["rptrs"], c["cols"], c["cptrs"], c["rows"], 100, 4, 5, seed=3,
                                   keep_trials=True, trial0=200)
        np.testing.assert_array_equal(sh.trial_values, sw.trial_values[200:])


def test_sparse_equals_dense_pattern(engine, pb):
    rng = np.random.default_rng(8)
    A = bernoulli(rng, 24, 0.4)
    c = pb.compress(0, A)
    d = engine.rasmussen(A, 4000, seed=5, keep_trials=True).trial_values
    s = engine.rasmussen_sparse(24, c["rptrs"], c["cols"], 4000, seed=5, keep_trials=True).trial_values
    np.testing.assert_array_equal(d, s)
    d = engine.scaling(A, 2000, 4, 5, seed=5, keep_trials=True).trial_values
    s = engine.scaling_sparse(24, c["rptrs"], c["cols"], c["cptrs"], c["rows"], 2000, 4, 5, seed=5,
                              keep_trials=True).trial_values
    np.testing.assert_array_equal(d, s)


def test_agrees_with_reference_estimator(engine, ref, orc):
    """The reference's own CPU estimators (different RNG) and ours estimate the
    same quantity: both within combined standard error of the exact value."""
    rng = np.random.default_rng(9)
    A = bernoulli(rng, 12, 0.5)
    exact = orc.perm_exact_int(A)[0]
    ours = engine.rasmussen(A, 100000, seed=11)
    theirs = ref.rasmussen(A, 100000, 4)
    assert abs(ours.mean - exact) < 5 * ours.std_error
    assert abs(theirs - exact) < 5 * ours.std_error * 1.5
    ours_s = engine.scaling(A, 50000, 4, 5, seed=12)
    theirs_s = ref.approximation(A, 50000, 4, 5, 4)
    assert abs(theirs_s - exact) < 6 * ours_s.std_error * 1.5


def test_bad_arguments(engine, pb):
    A = np.ones((5, 5))
    with pytest.raises(pb.PermError):
        engine.rasmussen(A, 0)
    with pytest.raises(pb.PermError):
        engine.scaling(A, 10, scale_intervals=0)
    with pytest.raises(pb.PermError):
        engine.rasmussen(np.ones((65, 65)), 10)


def test_reference_signature_mc(pb):
    A = np.ones((8, 8))
    # every trial of J_n gives exactly n!
    assert pb.gpu_perman64_rasmussen(A, 8, 1000) == math.factorial(8)
    v = pb.gpu_perman64_approximation(A, 8, 1000, 4, 5)
    assert abs(v - math.factorial(8)) < 1e-6 * math.factorial(8)


# ---- sparse estimators above order 64 (bitset kernel) -------------------------------

def _crs(pb, A):
    c = pb.compress(0, A)
    return c["n"], c["rptrs"], c["cols"], c["cptrs"], c["rows"]


@pytest.mark.parametrize("board", [(10, 14), (18, 20), (36, 36)])
def test_grid_graph_trials_bit_identical_above_64(engine, orc, pb, board):
    G = pb.grid_graph(*board)
    n, rp, cl, cp, rw = _crs(pb, G)
    assert n > 64
    e = engine.rasmussen_sparse(n, rp, cl, 600, seed=4, keep_trials=True)
    np.testing.assert_array_equal(e.trial_values, orc.rasmussen_sparse_trials(G, 4, 0, 600))
    s = engine.scaling_sparse(n, rp, cl, cp, rw, 100, 4, 5, seed=6, keep_trials=True)
    np.testing.assert_array_equal(s.trial_values, orc.scaling_sparse_trials(G, 4, 5, 6, 0, 100))


def test_random_sparse_above_64(engine, orc, pb):
    rng = np.random.default_rng(88)
    A = bernoulli(rng, 150, 0.05)
    n, rp, cl, cp, rw = _crs(pb, A)
    e = engine.rasmussen_sparse(n, rp, cl, 500, seed=9, keep_trials=True)
    np.testing.assert_array_equal(e.trial_values, orc.rasmussen_sparse_trials(A, 9, 0, 500))
    s = engine.scaling_sparse(n, rp, cl, cp, rw, 80, 2, 3, seed=9, keep_trials=True)
    np.testing.assert_array_equal(s.trial_values, orc.scaling_sparse_trials(A, 2, 3, 9, 0, 80))


def test_estimators_agree_above_64(engine, pb):
    G = pb.grid_graph(10, 14)
    n, rp, cl, cp, rw = _crs(pb, G)
    r = engine.rasmussen_sparse(n, rp, cl, 400000, seed=1)
    s = engine.scaling_sparse(n, rp, cl, cp, rw, 100000, 4, 5, seed=2)
    assert abs(r.mean - s.mean) < 5 * math.hypot(r.std_error, s.std_error)


def test_large_order_limits(engine, pb):
    rp = np.zeros(2049, np.int32)
    with pytest.raises(pb.PermError):
        engine.rasmussen_sparse(2048, rp, np.zeros(0, np.int32), 10)


def test_n64_estimators_agree_at_bench_size(engine):
    """Order 64, 2e5 trials each (the serving workload's approximate size):
    the two estimators agree within their combined standard error."""
    rng = np.random.default_rng(55)
    A = (rng.random((64, 64)) < 0.5).astype(np.float64)
    r = engine.rasmussen(A, 200000, seed=1)
    s = engine.scaling(A, 200000, 4, 5, seed=2)
    assert abs(r.mean - s.mean) < 5 * math.hypot(r.std_error, s.std_error)
