"""Multi-GPU host logic on CPU: shard ranges partition the Gray walk exactly
for any (n, world), and world_size-2 gloo ranks that each sum their shard
(with the oracle standing in for the device) recombine to the permanent."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


@pytest.mark.parametrize("n", [1, 2, 3, 4, 9, 17, 30, 40, 64])
@pytest.mark.parametrize("world", [1, 2, 3, 8, 13])
def test_shard_ranges_partition(pb, n, world):
    total = 1 << (n - 1)
    prev = 0
    for s in range(world):
        a, b = pb.shard_range(n, s, world)
        assert a == prev and b >= a
        if n >= 4:
            ms = max(3, n - 21)
            assert a % (1 << ms) == 0 and b % (1 << ms) == 0
        prev = b
    assert prev == total


def test_dd_sum_is_exactish(pb):
    parts = [(1e16, 1.0), (-1e16, 0.5), (3.0, 1e-17)]
    hi, lo = pb.dd_sum(parts)
    assert hi + lo == 4.5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, A, out_path):
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    sys.path.insert(0, str(root / "tests"))
    sys.path.insert(0, str(root / "oracle"))
    import torch.distributed as dist
    from conftest import load_package
    from oracle import Oracle

    pb = load_package()
    orc = Oracle()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    n = A.shape[0]
    factor = 2.0 if n & 1 else -2.0

    def shard_fn(mat, r, w):  # CPU stand-in for perm_exact_dense_shard
        a, b = pb.shard_range(n, r, w)
        hi, lo = orc.ryser_dd_range(mat, a, b, threads=1)
        return hi * factor, lo * factor

    hi, lo = pb.distributed_exact_dense(A, shard_fn=shard_fn)
    dist.barrier()
    dist.destroy_process_group()
    np.save(f"{out_path}.{rank}.npy", np.array([hi, lo]))


@pytest.mark.parametrize("n", [11, 16])
def test_gloo_two_ranks_recombine(pb, orc, tmp_path, n):
    rng = np.random.default_rng(n)
    A = rng.random((n, n))
    port = _free_port()
    out = str(tmp_path / "res")
    mp.start_processes(_rank_main, args=(2, port, A, out), nprocs=2, join=True, start_method="spawn")
    want = sum(orc.perm_dd(A))
    for r in range(2):
        hi, lo = np.load(f"{out}.{r}.npy")
        assert abs((hi + lo) - want) <= 1e-14 * abs(want)


def _rank_dynamic(rank, world, port, store_port, A, out_path):
    import sys
    import time
    from datetime import timedelta
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    sys.path.insert(0, str(root / "tests"))
    sys.path.insert(0, str(root / "oracle"))
    import torch.distributed as dist
    from conftest import load_package
    from oracle import Oracle

    pb = load_package()
    orc = Oracle()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    store = dist.TCPStore("127.0.0.1", store_port, world, rank == 0, timeout=timedelta(seconds=60))
    n = A.shape[0]
    factor = 2.0 if n & 1 else -2.0

    def shard_fn(mat, c, chunks):  # CPU stand-in; rank 0 is made slower
        if rank == 0:
            time.sleep(0.05)
        a, b = pb.shard_range(n, c, chunks)
        hi, lo = orc.ryser_dd_range(mat, a, b, threads=1)
        return hi * factor, lo * factor

    claims = []
    hi, lo = pb.distributed_exact_dense_dynamic(A, chunks=24, shard_fn=shard_fn, store=store, claims_out=claims)
    # a second call uses a fresh queue
    hi2, lo2 = pb.distributed_exact_dense_dynamic(A, chunks=5, shard_fn=shard_fn, store=store)
    dist.barrier()
    dist.destroy_process_group()
    np.save(f"{out_path}.{rank}.npy", np.array([hi, lo, len(claims), hi2, lo2]))


def test_gloo_dynamic_chunk_queue(pb, orc, tmp_path):
    """Two gloo ranks share a chunk queue: every chunk runs exactly once, the
    slower rank claims fewer chunks, and both ranks get the same permanent
    (independent of who ran what)."""
    rng = np.random.default_rng(5)
    A = rng.random((15, 15))
    port, store_port = _free_port(), _free_port()
    out = str(tmp_path / "dyn")
    mp.start_processes(_rank_dynamic, args=(2, port, store_port, A, out), nprocs=2, join=True,
                       start_method="spawn")
    want = sum(orc.perm_dd(A))
    r0, r1 = np.load(f"{out}.0.npy"), np.load(f"{out}.1.npy")
    for r in (r0, r1):
        assert abs((r[0] + r[1]) - want) <= 1e-14 * abs(want)
        assert abs((r[3] + r[4]) - want) <= 1e-14 * abs(want)
    assert r0[0] == r1[0] and r0[1] == r1[1]
    assert r0[2] + r1[2] == 24 and r1[2] > r0[2]


def _rank_subgroup_then_world(rank, world, port, store_port, A, out_path):
    import sys
    from datetime import timedelta
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    sys.path.insert(0, str(root / "tests"))
    sys.path.insert(0, str(root / "oracle"))
    import torch.distributed as dist
    from conftest import load_package
    from oracle import Oracle

    pb = load_package()
    orc = Oracle()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    store = dist.TCPStore("127.0.0.1", store_port, world, rank == 0, timeout=timedelta(seconds=60))
    n = A.shape[0]
    factor = 2.0 if n & 1 else -2.0

    def shard_fn(mat, c, chunks):
        a, b = pb.shard_range(n, c, chunks)
        hi, lo = orc.ryser_dd_range(mat, a, b, threads=1)
        return hi * factor, lo * factor

    # two disjoint subgroups run their own queues at the same time, then the
    # world group runs one: no queue is shared, every chunk runs exactly once
    g01, g23 = dist.new_group([0, 1]), dist.new_group([2, 3])
    mine = g01 if rank < 2 else g23
    sub = pb.distributed_exact_dense_dynamic(A, chunks=6, group=mine, shard_fn=shard_fn, store=store)
    whole = pb.distributed_exact_dense_dynamic(A, chunks=8, shard_fn=shard_fn, store=store)
    dist.barrier()
    dist.destroy_process_group()
    np.save(f"{out_path}.{rank}.npy", np.array([sub[0], sub[1], whole[0], whole[1]]))


def test_gloo_dynamic_queue_subgroups_then_world(pb, orc, tmp_path):
    """The queue's store key names the process group: two subgroups of a
    4-rank job and then the world group each drain a queue of their own."""
    rng = np.random.default_rng(9)
    A = rng.random((13, 13))
    port, store_port = _free_port(), _free_port()
    out = str(tmp_path / "sub")
    mp.start_processes(_rank_subgroup_then_world, args=(4, port, store_port, A, out), nprocs=4, join=True,
                       start_method="spawn")
    want = sum(orc.perm_dd(A))
    for r in range(4):
        v = np.load(f"{out}.{r}.npy")
        assert abs((v[0] + v[1]) - want) <= 1e-14 * abs(want)
        assert abs((v[2] + v[3]) - want) <= 1e-14 * abs(want)


def _rank_bench_sharded(rank, world, port, A, out_path):
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    sys.path.insert(0, str(root))
    sys.path.insert(0, str(root / "tests"))
    sys.path.insert(0, str(root / "oracle"))
    import torch.distributed as dist
    import bench
    from conftest import load_package
    from oracle import Oracle

    pb = load_package()
    orc = Oracle()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    n = A.shape[0]
    factor = 2.0 if n & 1 else -2.0

    def shard_fn(r, w):  # CPU stand-in for perm_exact_dense_resident_shard
        a, b = pb.shard_range(n, r, w)
        hi, lo = orc.ryser_dd_range(A, a, b, threads=1)
        return hi * factor, lo * factor, 0.0

    (hi, lo), ms = bench.sharded_step(pb, shard_fn, rank, world, dist, None)
    (hi1, lo1), _ = bench.sharded_step(pb, shard_fn, 0, 1)  # the one-rank step: the whole walk
    dist.barrier()
    dist.destroy_process_group()
    np.save(f"{out_path}.{rank}.npy", np.array([hi, lo, hi1, lo1, ms]))


def test_bench_sharded_step_two_ranks(pb, orc, tmp_path):
    """bench.py's distributed mode (one matrix, Gray-range shards per rank,
    16-byte all-gather, double-double sum) on two gloo ranks with the oracle
    as the device: the result equals the one-rank value within 1e-12 and is
    identical on both ranks."""
    rng = np.random.default_rng(12)
    A = (rng.random((17, 17)) < 0.5) * rng.integers(1, 5, (17, 17)).astype(float)
    A[np.arange(17), np.arange(17)] = 1.0
    port = _free_port()
    out = str(tmp_path / "bench")
    mp.start_processes(_rank_bench_sharded, args=(2, port, A, out), nprocs=2, join=True, start_method="spawn")
    r0, r1 = np.load(f"{out}.0.npy"), np.load(f"{out}.1.npy")
    exact = orc.perm_exact_int(A)[0]
    for r in (r0, r1):
        assert abs((r[0] + r[1]) - (r[2] + r[3])) <= 1e-12 * abs(r[2] + r[3])
        assert abs((r[0] + r[1]) - exact) <= 1e-12 * abs(exact)
    assert r0[0] == r1[0] and r0[1] == r1[1]


def _rank_estimate_and_batch(rank, world, port, A, mats, out_path):
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    sys.path.insert(0, str(root / "tests"))
    sys.path.insert(0, str(root / "oracle"))
    import torch.distributed as dist
    from conftest import load_package
    from oracle import Oracle

    pb = load_package()
    orc = Oracle()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)

    def ras_range(mat, t0, count):  # CPU stand-in for perm_approx_rasmussen_range
        w = orc.rasmussen_trials(mat, 77, t0, count)
        return float(w.sum()), float((w * w).sum()), float((w == 0).sum())

    def sca_range(mat, t0, count):  # ... and perm_approx_scaling_range
        w = orc.scaling_trials(mat, 3, 2, 77, t0, count)
        return float(w.sum()), float((w * w).sum()), float((w == 0).sum())

    e = pb.distributed_estimate(A, 1001, "rasmussen", seed=77, range_fn=ras_range)
    f = pb.distributed_estimate(A, 301, "scaling", 3, 2, seed=77, range_fn=sca_range)
    vals = pb.distributed_batch_exact(mats, batch_fn=lambda sub: [sum(orc.perm_dd(m)) for m in sub])
    dist.barrier()
    dist.destroy_process_group()
    np.save(f"{out_path}.{rank}.npy", np.concatenate([[e.mean, e.std_error, e.zero_trials, f.mean, f.std_error],
                                                      vals]))


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_estimates_and_batches_split_over_ranks(pb, orc, tmp_path, world):
    """Monte Carlo split by trial id: the ranks' trials are exactly the
    single-device run's (same Philox streams, the oracle standing in for the
    device), so the combined mean and standard error equal the whole run's;
    a batch split by walk length gives every rank every value, each computed
    once, in the caller's order."""
    rng = np.random.default_rng(11)
    A = (rng.random((12, 12)) < 0.6).astype(np.float64)
    mats = [rng.random((n, n)) for n in (4, 9, 7, 11, 5, 10, 8, 6)]
    port = _free_port()
    out = str(tmp_path / "mc")
    mp.start_processes(_rank_estimate_and_batch, args=(world, port, A, mats, out), nprocs=world, join=True,
                       start_method="spawn")
    w = orc.rasmussen_trials(A, 77, 0, 1001)
    v = orc.scaling_trials(A, 3, 2, 77, 0, 301)
    se = lambda x: np.sqrt(((x * x).sum() - x.sum() * x.mean()) / (len(x) - 1) / len(x))
    want_vals = [sum(orc.perm_dd(m)) for m in mats]
    rows = [np.load(f"{out}.{r}.npy") for r in range(world)]
    for r in rows:
        assert abs(r[0] - w.mean()) <= 1e-13 * abs(w.mean())
        assert abs(r[1] - se(w)) <= 1e-9 * se(w)
        assert r[2] == (w == 0).sum()
        assert abs(r[3] - v.mean()) <= 1e-13 * abs(v.mean())
        assert abs(r[4] - se(v)) <= 1e-9 * se(v)
        assert list(r[5:]) == want_vals
    assert all((rows[0] == r).all() for r in rows)


def test_batch_assignment_balances_walks(pb):
    """Longest walk first to the least-loaded rank: deterministic, every
    matrix owned once, loads within one largest walk of each other."""
    rng = np.random.default_rng(3)
    orders = rng.integers(12, 29, 500)
    for world in (1, 2, 3, 8):
        owner = pb.batch_assignment(orders, world)
        assert owner == pb.batch_assignment(list(orders), world)
        loads = [sum(2.0 ** (o - 1) for o, w in zip(orders, owner) if w == r) for r in range(world)]
        assert max(loads) - min(loads) <= 2.0 ** (orders.max() - 1)
