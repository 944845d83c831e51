"""The oracle is pinned before it is trusted (CPU only).

The reference ships no known-answer tests, so the pins are: published
Philox4x32-10 vectors, closed forms, agreement of four independent algorithms
(dd Ryser, __float128 Ryser, subset DP, exact multi-modular integer Ryser),
and the reference's own functions compiled from its sources (values recorded
in tests/golden/golden.json by tests/golden/make_golden.py, re-checked live
when the reference build is present).
"""
import math

import numpy as np
import pytest
from conftest import bernoulli, rel_err


def test_philox_known_answers(orc):
    # Random123 kat_vectors, philox4x32 with 10 rounds
    assert orc.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert orc.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert orc.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == [
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 12])
def test_all_ones_is_factorial(orc, n):
    J = np.ones((n, n))
    f = math.factorial(n)
    assert orc.perm_dd(J)[0] == f
    assert orc.perm_q(J)[0] == f
    assert orc.perm_dp(J)[0] == f
    assert orc.perm_exact_int(J)[0] == f


def test_identity_permutation_zero_row(orc):
    rng = np.random.default_rng(0)
    for n in (4, 9, 13):
        I = np.eye(n)
        P = I[rng.permutation(n)]
        assert orc.perm_dd(I)[0] == 1.0
        assert orc.perm_exact_int(P)[0] == 1
        Z = rng.integers(1, 4, (n, n)).astype(float)
        Z[n // 2] = 0
        assert orc.perm_exact_int(Z)[0] == 0
        assert orc.perm_dd(Z)[0] == 0.0


def test_block_diagonal_is_product(orc):
    rng = np.random.default_rng(1)
    A = rng.integers(0, 4, (6, 6)).astype(float)
    B = rng.integers(0, 4, (7, 7)).astype(float)
    M = np.zeros((13, 13))
    M[:6, :6] = A
    M[6:, 6:] = B
    assert orc.perm_exact_int(M)[0] == orc.perm_exact_int(A)[0] * orc.perm_exact_int(B)[0]


@pytest.mark.parametrize("seed", range(6))
def test_four_algorithms_agree(orc, seed):
    rng = np.random.default_rng(100 + seed)
    n = 8 + seed
    A = rng.integers(-3, 5, (n, n)).astype(float)
    exact = orc.perm_exact_int(A)[0]
    hi, lo = orc.perm_dd(A)
    qh, ql = orc.perm_q(A)
    dh, dl = orc.perm_dp(A)
    assert int(hi) + int(lo) == exact
    assert int(qh) + int(ql) == exact
    assert int(dh) + int(dl) == exact
    R = rng.random((n, n))
    assert rel_err(orc.perm_dd(R)[0], orc.perm_dp(R)[0]) < 1e-15
    assert rel_err(orc.perm_q(R)[0], orc.perm_dp(R)[0]) < 1e-15


def test_dd_range_sums_to_whole(orc):
    rng = np.random.default_rng(7)
    A = rng.random((12, 12))
    total = 1 << 11
    parts = [orc.ryser_dd_range(A, a, b) for a, b in [(0, 5), (5, 700), (700, total)]]
    s = sum(p[0] + p[1] for p in parts) * -2.0  # even n: factor -2
    assert rel_err(s, orc.perm_dd(A)[0]) < 1e-14


def test_skipper_restatement_matches_ryser(orc, pb):
    rng = np.random.default_rng(11)
    for n, d in [(10, 0.3), (14, 0.25), (16, 0.5)]:
        A = bernoulli(rng, n, d)
        c = pb.compress(2, A)
        v, vis = orc.skipper(c, chunks=64)
        exact = orc.perm_exact_int(c["mat"].astype(np.int64))[0]
        assert rel_err(v, exact) < 1e-12
        assert vis < (1 << (n - 1))  # binary sparse matrices do skip


def test_golden_values_consistent(golden):
    for name, c in golden.items():
        hi, lo = c["dd"]
        if "exact" in c:
            ex = int(c["exact"])
            assert rel_err(hi + lo, ex) < 1e-15 or ex == 0, name
        if "dp" in c:
            assert rel_err(c["dp"][0], hi) < 1e-14, name


def test_golden_reference_values_match_oracle(golden):
    """The reference's own outputs (recorded by make_golden.py) agree with the
    oracle where the reference is accurate: double-X paths on every input, and
    the FP32-X parallel_perman64 on integer inputs."""
    for name, c in golden.items():
        want = c["dd"][0]
        if want == 0:
            continue
        if c.get("ref_perman64") is not None:
            # serial double-X walk with an uncompensated sum: ~1e-9 on n=30 reals
            assert rel_err(c["ref_perman64"], want) < (1e-8 if c["kind"] == "real" else 1e-9), name
        # the reference's CRS/CCS keep positive entries only (util.h:537), so its
        # SkipPer computes the permanent of the positive part: compare on
        # non-negative matrices
        if c.get("ref_skip_balanced_skiporder") is not None and (c["A"] >= 0).all():
            assert rel_err(c["ref_skip_balanced_skiporder"], want) < 1e-9, name
        if c["kind"] in ("binary", "int") and c["n"] <= 24:
            assert rel_err(c["ref_parallel_perman64"], want) < 1e-9, name


def test_reference_live_agrees_with_oracle(orc, ref):
    rng = np.random.default_rng(5)
    for n in (6, 11, 15):
        A = rng.integers(0, 5, (n, n)).astype(float)
        ex = orc.perm_exact_int(A)[0]
        assert rel_err(ref.perman64(A), ex) < 1e-12
        assert rel_err(ref.parallel_perman64(A, 4), ex) < 1e-9
        c = ref.compress(2, A)
        assert rel_err(ref.skip_balanced(c, 4), ex) < 1e-12


def test_mc_oracle_is_unbiased(orc):
    rng = np.random.default_rng(3)
    A = bernoulli(rng, 10, 0.5)
    exact = orc.perm_exact_int(A)[0]
    for fn in (lambda: orc.rasmussen_trials(A, 9, 0, 40000), lambda: orc.scaling_trials(A, 2, 3, 9, 0, 40000)):
        v = fn()
        mean, se = v.mean(), v.std(ddof=1) / math.sqrt(len(v))
        assert abs(mean - exact) < 5 * se + 1e-12


# domino tilings of small boards (OEIS A004003 for n x n; 2 x n are Fibonacci numbers)
TILINGS = {(2, 2): 2, (2, 3): 3, (2, 4): 5, (3, 4): 11, (4, 4): 36, (4, 5): 95, (6, 6): 6728, (4, 6): 281,
           (6, 5): 1183}


def test_grid_graph_counts_domino_tilings(orc, pb):
    for (m, n), t in TILINGS.items():
        G = orc.grid_graph(m, n)
        np.testing.assert_array_equal(G, pb.grid_graph(m, n))
        assert orc.perm_exact_int(G)[0] == t, (m, n)


def test_grid_graph_matches_reference(ref, pb):
    for m, n in [(2, 2), (3, 4), (6, 5), (8, 8), (5, 6), (10, 12)]:
        np.testing.assert_array_equal(pb.grid_graph(m, n), ref.grid_graph(m, n))
    with pytest.raises(pb.PermError):
        pb.grid_graph(3, 5)


def test_sparse_estimator_restatement_equals_dense_on_patterns(orc):
    rng = np.random.default_rng(12)
    A = bernoulli(rng, 30, 0.4)
    np.testing.assert_array_equal(orc.rasmussen_sparse_trials(A, 5, 0, 500), orc.rasmussen_trials(A, 5, 0, 500))
    np.testing.assert_array_equal(orc.scaling_sparse_trials(A, 4, 5, 5, 0, 300), orc.scaling_trials(A, 4, 5, 5, 0, 300))


def test_sparse_estimators_large_order_unbiased(orc):
    G = orc.grid_graph(8, 8)  # order 32: 12988816 tilings
    for v in (orc.rasmussen_sparse_trials(G, 3, 0, 20000), orc.scaling_sparse_trials(G, 4, 5, 3, 0, 5000)):
        mean, se = v.mean(), v.std(ddof=1) / math.sqrt(len(v))
        assert abs(mean - 12988816) < 5 * se


def test_tc_round_restatement_sums_to_the_permanent(orc):
    """The tensor-core kernel's subset split (rounds x 4 blocks x 128 lanes),
    restated exactly in the oracle, covers every subset once with the right
    signs: all rounds together give the permanent (orders 16, 17, 18)."""
    from oracle import tc_rounds_sum
    rng = np.random.default_rng(77)
    for n in (16, 17, 18):
        A = rng.integers(-3, 4, (n, n)).astype(np.float64)
        total, _ = tc_rounds_sum(A, 0, 2 ** (n - 10))
        assert total == orc.perm_exact_int(A)[0]
