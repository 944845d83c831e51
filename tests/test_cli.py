"""The drop-in `perman` command line (main.cu:315-590 flags and output line)."""
import re
import subprocess

import numpy as np
import pytest
from conftest import bernoulli, rel_err


def write_matrix(path, A, typ="int"):
    n = A.shape[0]
    nz = [(i, j) for i in range(n) for j in range(n) if A[i, j] != 0]
    with open(path, "w") as f:
        f.write(f"{n} {len(nz)} {typ}\n")
        for i, j in nz:
            f.write(f"{i} {j} {int(A[i, j]) if typ == 'int' else repr(float(A[i, j]))}\n")


def run(pb, *args):
    return subprocess.run([str(pb.CLI_PATH), *map(str, args)], capture_output=True, text=True, timeout=300)


def result_value(out):
    m = re.search(r"^Result: (\S+) (\S+) in (\S+)$", out, re.M)
    assert m, out
    return m.group(1), float(m.group(2))


def test_missing_file_flag(pb):
    r = run(pb, "-g", "-p4")
    assert r.returncode == 1 and "required" in r.stderr


def test_cpu_algorithms_rejected(pb, tmp_path):
    p = tmp_path / "m.txt"
    write_matrix(p, np.ones((4, 4)))
    r = run(pb, "-f", p, "-c", "-t8")
    assert r.returncode != 0 and "CPU" in r.stderr


def test_grid_mode_odd_board(pb):
    r = run(pb, "-i", "-m", "3", "-n", "5")
    assert r.returncode == 0 and "should be positive" in r.stdout


def test_unreadable_file(pb, tmp_path):
    r = run(pb, "-f", tmp_path / "nope.txt")
    assert r.returncode != 0


@pytest.mark.gpu
@pytest.mark.parametrize("flag", ["-m", "-f"])
def test_dense_exact_output(pb, orc, tmp_path, flag):
    rng = np.random.default_rng(21)
    A = bernoulli(rng, 16, 0.5) * rng.integers(1, 5, (16, 16))
    p = tmp_path / "m.txt"
    write_matrix(p, A)
    r = run(pb, flag, p, "-g", "-p4")
    assert r.returncode == 0, r.stderr
    name, v = result_value(r.stdout)
    assert name == "gpu_perman64_xshared_coalescing_mshared"
    assert rel_err(v, orc.perm_exact_int(A)[0]) < 1e-13


@pytest.mark.gpu
def test_sparse_and_binary_flags(pb, orc, tmp_path):
    rng = np.random.default_rng(22)
    A = bernoulli(rng, 18, 0.3) * 3
    p = tmp_path / "m.txt"
    write_matrix(p, A)
    r = run(pb, "-f", p, "-s", "-p7", "-r2", "-b")
    assert r.returncode == 0, r.stderr
    name, v = result_value(r.stdout)
    assert name == "gpu_perman64_xshared_coalescing_mshared_skipper"
    assert rel_err(v, orc.perm_exact_int((A != 0).astype(float))[0]) < 1e-13


@pytest.mark.gpu
def test_approximation_flags(pb, orc, tmp_path):
    rng = np.random.default_rng(23)
    A = bernoulli(rng, 14, 0.5)
    p = tmp_path / "m.txt"
    write_matrix(p, A)
    exact = orc.perm_exact_int(A)[0]
    for algo in ("1", "2"):
        r = run(pb, "-f", p, "-b", "-a", "-p", algo, "-x", "100000", "-y", "4", "-z", "5", "--seed", "3")
        assert r.returncode == 0, r.stderr
        _, v = result_value(r.stdout)
        se = float(re.search(r"std error: (\S+)", r.stdout).group(1))
        assert abs(v - exact) < 5 * se


@pytest.mark.gpu
def test_multi_gpu_id_on_available_devices(pb, orc, tmp_path):
    rng = np.random.default_rng(24)
    A = bernoulli(rng, 20, 0.5)
    p = tmp_path / "m.txt"
    write_matrix(p, A)
    r = run(pb, "-f", p, "-p5", "-d", "2")
    assert r.returncode == 0, r.stderr
    _, v = result_value(r.stdout)
    assert rel_err(v, orc.perm_exact_int(A)[0]) < 1e-13


@pytest.mark.gpu
def test_grid_mode_estimates_tilings(pb):
    # 8 x 8 board: 12988816 domino tilings
    r = run(pb, "-i", "-m", "8", "-n", "8", "-p1", "-x", "200000", "--seed", "5")
    assert r.returncode == 0, r.stderr
    name, v = result_value(r.stdout)
    se = float(re.search(r"std error: (\S+)", r.stdout).group(1))
    assert name == "gpu_perman64_rasmussen_sparse" and abs(v - 12988816) < 5 * se
    r = run(pb, "-i", "-m", "20", "-n", "10", "-p2", "-x", "20000")
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_sparse_ccs_ids_run_the_sparse_walk(pb, orc, tmp_path):
    """-s -p1..-p6 (the reference's CCS walks; -p5/-p6 on -d devices) run the
    split-dd kernel, whose sparse layout walks only the rows of the three
    sparsest columns (the multi-GPU ids as Gray-range shards, one per
    device); the kernel that ran is named on its own line."""
    rng = np.random.default_rng(23)
    A = bernoulli(rng, 22, 0.2) * (1.0 - rng.random((22, 22)))
    p = tmp_path / "r.txt"
    write_matrix(p, A, "double")
    want = sum(orc.perm_dd(A))
    for pid in ("-p1", "-p4", "-p5", "-p6"):
        r = run(pb, "-f", p, "-s", pid)
        assert r.returncode == 0, r.stderr
        name, v = result_value(r.stdout)
        assert name.endswith("_sparse")
        assert "engine kernel: split-dd walk" in r.stdout
        assert rel_err(v, want) < 1e-10
