"""Checkpoint / resume of a long exact walk.  Host logic without a GPU: the
oracle stands in for perm_exact_dense_shard; a simulated crash after some
shards leaves a checkpoint from which a second call finishes the walk,
computing only the missing shards and returning the uninterrupted value bit
for bit.  One gpu-marked test runs the same on the B200's shard kernels."""
import json

import numpy as np
import pytest


def oracle_shard_fn(pb, orc, calls=None, crash_after=None):
    def fn(mat, c, chunks):
        if crash_after is not None and calls is not None and len(calls) >= crash_after:
            raise KeyboardInterrupt("simulated interruption")
        n = mat.shape[0]
        a, b = pb.shard_range(n, c, chunks)
        hi, lo = orc.ryser_dd_range(mat, a, b, threads=1)
        f = 2.0 if n & 1 else -2.0
        if calls is not None:
            calls.append(c)
        return hi * f, lo * f

    return fn


def test_uninterrupted_walk_matches_the_oracle(pb, orc, tmp_path):
    rng = np.random.default_rng(31)
    A = rng.random((15, 15))
    path = tmp_path / "walk.ckpt"
    hi, lo = pb.checkpointed_exact_dense(A, path, chunks=7, shard_fn=oracle_shard_fn(pb, orc))
    want = sum(orc.perm_dd(A))
    assert abs((hi + lo) - want) <= 1e-13 * abs(want)
    assert not path.exists()  # removed after success


def test_interrupted_walk_resumes_bit_for_bit(pb, orc, tmp_path):
    rng = np.random.default_rng(32)
    A = rng.standard_normal((16, 16))  # signed: cancellation makes summation order visible
    ref = pb.checkpointed_exact_dense(A, tmp_path / "ref.ckpt", chunks=9, shard_fn=oracle_shard_fn(pb, orc))
    path = tmp_path / "walk.ckpt"
    first = []
    with pytest.raises(KeyboardInterrupt):
        pb.checkpointed_exact_dense(A, path, chunks=9, shard_fn=oracle_shard_fn(pb, orc, first, crash_after=4))
    state = json.loads(path.read_text())
    assert sorted(int(c) for c in state["done"]) == [0, 1, 2, 3]
    second = []
    got = pb.checkpointed_exact_dense(A, path, chunks=9, shard_fn=oracle_shard_fn(pb, orc, second), keep=True)
    assert second == [4, 5, 6, 7, 8]  # only the missing shards
    assert got == ref  # the same chunk-ordered double-double sum
    # a completed checkpoint kept on disk answers without walking again
    third = []
    assert pb.checkpointed_exact_dense(A, path, chunks=9, shard_fn=oracle_shard_fn(pb, orc, third)) == ref
    assert third == []


def test_checkpoint_of_another_run_is_refused(pb, orc, tmp_path):
    rng = np.random.default_rng(33)
    A = rng.random((12, 12))
    path = tmp_path / "walk.ckpt"
    with pytest.raises(KeyboardInterrupt):
        pb.checkpointed_exact_dense(A, path, chunks=5, shard_fn=oracle_shard_fn(pb, orc, [], crash_after=2))
    B = A.copy()
    B[3, 4] += 1e-9
    fn = oracle_shard_fn(pb, orc)
    with pytest.raises(pb.PermError, match="matrix_sha256"):
        pb.checkpointed_exact_dense(B, path, chunks=5, shard_fn=fn)
    with pytest.raises(pb.PermError, match="chunks"):
        pb.checkpointed_exact_dense(A, path, chunks=6, shard_fn=fn)
    with pytest.raises(pb.PermError, match="variant"):
        pb.checkpointed_exact_dense(A, path, chunks=5, variant=pb.PERM_KERNEL_DENSE, shard_fn=fn)
    path.write_text('{"format": "perm_b200_checkpoint_v1", "done": ')  # torn by hand
    with pytest.raises(pb.PermError, match="unreadable"):
        pb.checkpointed_exact_dense(A, path, chunks=5, shard_fn=fn)
    with pytest.raises(pb.PermError):
        pb.checkpointed_exact_dense(A, path, chunks=0, shard_fn=fn)


class _OracleEngine:
    """Stands in for Engine: exact_dense_shard answers from the oracle, so
    the production branch (engine= instead of shard_fn=) runs without a GPU."""

    def __init__(self, pb, orc):
        self.fn = oracle_shard_fn(pb, orc, calls=[])
        self.variants = []

    def exact_dense_shard(self, mat, shard, nshards, variant=0):
        from types import SimpleNamespace

        self.variants.append(variant)
        hi, lo = self.fn(mat, shard, nshards)
        return SimpleNamespace(hi=hi, lo=lo)


def test_engine_branch_walks_every_shard_once(pb, orc, tmp_path):
    rng = np.random.default_rng(34)
    A = (rng.random((14, 14)) < 0.6) * rng.integers(1, 5, (14, 14))
    eng = _OracleEngine(pb, orc)
    hi, lo = pb.checkpointed_exact_dense(A, tmp_path / "w.ckpt", chunks=6, variant=pb.PERM_KERNEL_DENSE_INT,
                                         engine=eng)
    assert hi + lo == orc.perm_exact_int(A)[0]
    assert eng.variants == [pb.PERM_KERNEL_DENSE_INT] * 6


@pytest.mark.gpu
def test_checkpointed_walk_on_the_gpu(pb, orc, engine, tmp_path):
    """The same walk on the B200 (perm_exact_dense_ex shards): interrupted
    after three shards, resumed, equal to the oracle's exact value."""
    rng = np.random.default_rng(35)
    A = ((rng.random((24, 24)) < 0.5) * rng.integers(1, 5, (24, 24))).astype(np.float64)
    exact = orc.perm_exact_int(A)[0]
    path = tmp_path / "gpu.ckpt"

    class Crash(Exception):
        pass

    calls = []

    def crashing(mat, c, chunks):
        if len(calls) == 3:
            raise Crash()
        calls.append(c)
        r = engine.exact_dense_shard(mat, c, chunks)
        return r.hi, r.lo

    with pytest.raises(Crash):
        pb.checkpointed_exact_dense(A, path, chunks=8, shard_fn=crashing)
    hi, lo = pb.checkpointed_exact_dense(A, path, chunks=8, engine=engine)
    assert abs((hi + lo) - exact) <= 1e-12 * abs(exact)
    assert not path.exists()
    # deterministic shard kernels: the resumed sum is the uninterrupted one
    assert (hi, lo) == pb.checkpointed_exact_dense(A, tmp_path / "again.ckpt", chunks=8, engine=engine)


def test_checkpoint_with_bad_entries_is_refused(pb, orc, tmp_path):
    A = np.eye(6) + 0.5
    path = tmp_path / "walk.ckpt"
    state = {"format": pb.CHECKPOINT_FORMAT, "matrix_sha256": pb._fingerprint(np.ascontiguousarray(A)),
             "n": 6, "chunks": 3, "variant": 0, "done": {"0": [1.5, "0x0p+0"]}}
    path.write_text(json.dumps(state))
    with pytest.raises(pb.PermError, match="unreadable"):
        pb.checkpointed_exact_dense(A, path, chunks=3, shard_fn=oracle_shard_fn(pb, orc))
    state["done"] = {"7": ["0x1p+0", "0x0p+0"]}
    path.write_text(json.dumps(state))
    with pytest.raises(pb.PermError, match="outside"):
        pb.checkpointed_exact_dense(A, path, chunks=3, shard_fn=oracle_shard_fn(pb, orc))
