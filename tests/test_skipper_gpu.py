"""SkipPer kernel on the B200 against the oracle and the dense kernel."""
import numpy as np
import pytest
from conftest import bernoulli, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.mark.parametrize("n,d", [(2, 0.9), (5, 0.5), (9, 0.3), (14, 0.25), (18, 0.2), (22, 0.3), (24, 0.15)])
@pytest.mark.parametrize("order", [0, 2])
def test_binary_sparse_exact(engine, orc, pb, n, d, order):
    rng = np.random.default_rng(n * 10 + order)
    A = bernoulli(rng, n, d)
    c = pb.compress(order, A)
    r = engine.exact_sparse(c["n"], c["rptrs"], c["cols"], c["rvals"], c["cptrs"], c["rows"], c["cvals"],
                           variant=pb.PERM_KERNEL_SKIPPER)
    exact = orc.perm_exact_int(A)[0]
    assert rel_err(r.value, exact) < 1e-13
    assert r.kernel == pb.PERM_KERNEL_SKIPPER
    assert 0 < r.steps <= r.total_steps


def test_skips_happen_and_match_cpu_skipper(engine, orc, pb):
    rng = np.random.default_rng(77)
    A = bernoulli(rng, 22, 0.2)
    c = pb.compress(2, A)
    r = engine.exact_sparse(c["n"], c["rptrs"], c["cols"], c["rvals"], c["cptrs"], c["rows"], c["cvals"],
                           variant=pb.PERM_KERNEL_SKIPPER)
    v, _ = orc.skipper(c, chunks=512)
    assert rel_err(r.value, v) < 1e-12
    assert r.steps < 0.9 * r.total_steps


def test_real_valued_sparse(engine, orc, pb):
    rng = np.random.default_rng(12)
    for n in (12, 20, 24):
        A = bernoulli(rng, n, 0.25) * (1.0 - rng.random((n, n)))
        c = pb.compress(2, A)
        r = engine.exact_sparse(c["n"], c["rptrs"], c["cols"], c["rvals"], c["cptrs"], c["rows"], c["cvals"],
                           variant=pb.PERM_KERNEL_SKIPPER)
        want = orc.perm_dd(c["mat"])
        assert rel_err(r.value, want[0] + want[1]) < TOL


def test_golden_sparse_case(engine, golden, pb):
    c0 = golden["cfg2_sparse_real_n28_d020"]
    c = pb.compress(2, c0["A"])
    r = engine.exact_sparse(c["n"], c["rptrs"], c["cols"], c["rvals"], c["cptrs"], c["rows"], c["cvals"],
                           variant=pb.PERM_KERNEL_SKIPPER)
    assert rel_err(r.value, c0["dd"][0] + c0["dd"][1]) < TOL


def test_zero_row_gives_zero(engine, pb):
    A = np.ones((10, 10))
    A[4] = 0
    c = pb.compress(0, A)
    r = engine.exact_sparse(c["n"], c["rptrs"], c["cols"], c["rvals"], c["cptrs"], c["rows"], c["cvals"],
                           variant=pb.PERM_KERNEL_SKIPPER)
    assert r.value == 0.0


@pytest.mark.slow
def test_cfg2_full_size_matches_dense(engine, pb):
    """n=36, density 0.2, values U(0,1]: two independent kernels agree."""
    rng = np.random.default_rng(2026)
    A = bernoulli(rng, 36, 0.2) * (1.0 - rng.random((36, 36)))
    c = pb.compress(2, A)
    r = engine.exact_sparse(c["n"], c["rptrs"], c["cols"], c["rvals"], c["cptrs"], c["rows"], c["cvals"],
                           variant=pb.PERM_KERNEL_SKIPPER)
    d = engine.exact_dense(c["mat"])
    assert rel_err(r.value, d.value) < TOL


def test_reference_signature_skipper(pb):
    rng = np.random.default_rng(13)
    A = bernoulli(rng, 16, 0.3)
    c = pb.compress(2, A)
    v = pb.gpu_perman64_xshared_coalescing_mshared_skipper(c["mat"], c["rptrs"], c["cols"], c["cptrs"], c["rows"],
                                                           c["cvals"], 16)
    assert rel_err(v, pb.default_engine().exact_dense(c["mat"]).value) < 1e-13


def test_automatic_choice(engine, pb):
    """Real values never give exact zeros, so a register kernel runs under
    the accuracy policy (FP64 X, or the certified split-dd walk in its sparse
    layout where that costs no more or FP64 X would miss the target); sparse
    binary matrices mostly vanish, so SkipPer runs."""
    rng = np.random.default_rng(31)
    A = bernoulli(rng, 26, 0.2) * (1.0 - rng.random((26, 26)))
    c = pb.compress(2, A)
    r = engine.exact_sparse(c["n"], c["rptrs"], c["cols"], c["rvals"], c["cptrs"], c["rows"], c["cvals"])
    assert r.kernel in (pb.PERM_KERNEL_DENSE, pb.PERM_KERNEL_DENSE_SDD) and r.rel_error_estimate <= TOL
    s = engine.exact_sparse(c["n"], c["rptrs"], c["cols"], c["rvals"], c["cptrs"], c["rows"], c["cvals"],
                            variant=pb.PERM_KERNEL_SKIPPER)
    assert rel_err(r.value, s.value) < TOL
    # two ones per row (identity plus a permutation): almost every term vanishes
    B = ((np.eye(30) + np.eye(30)[rng.permutation(30)]) > 0).astype(float)
    cb = pb.compress(2, B)
    rb = engine.exact_sparse(cb["n"], cb["rptrs"], cb["cols"], cb["rvals"], cb["cptrs"], cb["rows"], cb["cvals"])
    assert rb.kernel == pb.PERM_KERNEL_SKIPPER
    assert rel_err(rb.value, engine.exact_dense(cb["mat"]).value) < 1e-13
