"""Request loop: every result is the same alone and in the mix (exact: 1e-12
relative -- large requests run as shards, which changes the rounding only --
or 1e-10 where the accuracy policy recomputed one in double-double;
Monte Carlo: bit-identical, same Philox streams), work of different slots
overlaps on the device, and a bad request fails alone."""
import numpy as np
import pytest
from conftest import bernoulli, rel_err

pytestmark = pytest.mark.gpu


def make_requests(pb, rng, count):
    reqs = []
    for i in range(count):
        kind = i % 4
        if kind in (0, 1):
            n = int(rng.integers(12, 27))
            A = bernoulli(rng, n, 0.5) * (1.0 - rng.random((n, n)))
            reqs.append((pb.PERM_REQ_EXACT_DENSE if kind == 0 else pb.PERM_REQ_EXACT_SPARSE, A, {}))
        else:
            n = int(rng.integers(20, 41))
            A = bernoulli(rng, n, 0.5)
            reqs.append((pb.PERM_REQ_RASMUSSEN if kind == 2 else pb.PERM_REQ_SCALING, A,
                         {"trials": 20000, "seed": 100 + i}))
    return reqs


def alone(engine, pb, kind, A, kw):
    """(value, kernel) of the request run alone through the engine."""
    if kind == pb.PERM_REQ_EXACT_DENSE:
        r = engine.exact_dense(A)
        return r.value, r.kernel
    if kind == pb.PERM_REQ_EXACT_SPARSE:
        r = engine.exact_sparse_matrix(A, order=0)
        return r.value, r.kernel
    if kind == pb.PERM_REQ_RASMUSSEN:
        return engine.rasmussen(A, kw["trials"], seed=kw["seed"]).mean, 0
    return engine.scaling(A, kw["trials"], 4, 5, seed=kw["seed"]).mean, 0


def test_results_same_alone_and_in_the_mix(engine, pb):
    rng = np.random.default_rng(77)
    reqs = make_requests(pb, rng, 48)
    with pb.Server(0, slots=4, slice_steps=1 << 20) as srv:
        tickets = [srv.submit(k, A, **kw) for k, A, kw in reqs]
        resps = [srv.wait(t) for t in tickets]
    overlap = 0
    for (k, A, kw), r in zip(reqs, resps):
        assert r["status"] == pb.PERM_OK, r["message"]
        want, kern = alone(engine, pb, k, A, kw)
        if k in (pb.PERM_REQ_RASMUSSEN, pb.PERM_REQ_SCALING):
            assert r["value"] == want
        elif {pb.PERM_KERNEL_DENSE_DD, pb.PERM_KERNEL_DENSE_SDD} & {kern, r["kernel"]}:
            # the accuracy policy recomputed one of them (split-dd or double-double): both meet 1e-10
            assert rel_err(r["value"], want) < 1e-10
        else:
            assert rel_err(r["value"], want) < 1e-12
    spans = sorted((r["t_admit_ms"], r["t_done_ms"]) for r in resps)
    for (a0, d0), (a1, d1) in zip(spans, spans[1:]):
        overlap += a1 < d0
    assert overlap > 0, "no two requests were ever in flight together"


def test_certified_requests_run_unsliced(engine, pb):
    """Requests whose policy starts with a certified walk (an integer matrix;
    a strongly cancelling real one, predicted on the device) run as that one
    walk even when they are longer than slice_steps: same kernel and the same
    bits as the call alone."""
    rng = np.random.default_rng(31)
    I = (bernoulli(rng, 24, 0.5) * rng.integers(1, 5, (24, 24))).astype(float)
    R = (rng.random((32, 32)) < 0.5) * (1.0 - rng.random((32, 32)))
    assert engine.dense_plan(I)[0] == pb.PERM_KERNEL_DENSE_INT_DD
    assert engine.dense_plan(R)[0] == pb.PERM_KERNEL_DENSE_SDD
    with pb.Server(0, slots=2, slice_steps=1 << 20) as srv:
        resps = [srv.wait(srv.submit(pb.PERM_REQ_EXACT_DENSE, M)) for M in (I, R)]
    for M, r in zip((I, R), resps):
        assert r["status"] == pb.PERM_OK, r["message"]
        alone = engine.exact_dense(M)
        assert r["kernel"] == alone.kernel and r["value"] == alone.value


def test_bad_request_fails_alone(pb):
    rng = np.random.default_rng(3)
    with pb.Server(0, slots=2) as srv:
        good = srv.submit(pb.PERM_REQ_EXACT_DENSE, bernoulli(rng, 14, 0.5))
        bad = srv.submit(pb.PERM_REQ_EXACT_DENSE, np.ones((70, 70)))
        mc_bad = srv.submit(pb.PERM_REQ_SCALING, np.ones((10, 10)), trials=0)
        assert srv.wait(good)["status"] == pb.PERM_OK
        assert srv.wait(bad)["status"] == pb.PERM_EUNSUPPORTED
        assert srv.wait(mc_bad)["status"] == pb.PERM_EINVAL


def test_memory_budget_admission(pb):
    """A budget smaller than two requests forces one-at-a-time admission."""
    rng = np.random.default_rng(4)
    mats = [bernoulli(rng, 20, 0.5) for _ in range(6)]
    with pb.Server(0, slots=4, memory_budget=6000) as srv:
        ts = [srv.submit(pb.PERM_REQ_EXACT_DENSE, m) for m in mats]
        rs = [srv.wait(t) for t in ts]
    spans = sorted((r["t_admit_ms"], r["t_done_ms"]) for r in rs)
    for (a0, d0), (a1, d1) in zip(spans, spans[1:]):
        assert a1 >= d0 - 1e-6


def test_sliced_request_gets_the_accuracy_policy(engine, pb):
    """A positive real order-28 matrix cancels enough that its FP64 bound
    misses 1e-10; run as 128 shards, the assembled value still goes through
    the policy and lands within 1e-10 of the double-double permanent."""
    rng = np.random.default_rng(91)
    A = 1.0 - rng.random((28, 28))
    with pb.Server(0, slots=2, slice_steps=1 << 20) as srv:
        r = srv.wait(srv.submit(pb.PERM_REQ_EXACT_DENSE, A))
    assert r["status"] == pb.PERM_OK, r["message"]
    d = engine.exact_dense(A, variant=pb.PERM_KERNEL_DENSE_DD).value
    assert abs(r["value"] - d) <= 1e-10 * abs(d)
