"""Matrix input and CRS/CCS builders against the reference's util.h (CPU only)."""
import os

import numpy as np
import pytest
from conftest import REF_SRC, bernoulli


def write_matrix(path, A, typ="double", extra_lines=()):
    n = A.shape[0]
    nz = [(i, j) for i in range(n) for j in range(n) if A[i, j] != 0]
    with open(path, "w") as f:
        f.write(f"{n} {len(nz)} {typ}\n")
        for i, j in nz:
            v = A[i, j]
            f.write(f"{i} {j} {int(v) if typ == 'int' else repr(float(v))}\n")
        for line in extra_lines:
            f.write(line + "\n")


@pytest.mark.parametrize("typ", ["int", "float", "double"])
@pytest.mark.parametrize("binary", [False, True])
def test_reader_matches_reference(pb, ref, tmp_path, typ, binary):
    rng = np.random.default_rng(42)
    A = bernoulli(rng, 17, 0.4) * (rng.integers(1, 6, (17, 17)) if typ == "int" else rng.random((17, 17)) * 5)
    p = tmp_path / "m.txt"
    write_matrix(p, A, typ, extra_lines=["garbage line", "3 4", "", "2 2 7"])
    mine, t, _ = pb.read_matrix(p, binary=binary)
    theirs = ref.read_matrix(p, binary=binary)
    assert t == typ
    np.testing.assert_array_equal(mine, theirs)


def test_reader_rejects_out_of_range(pb, tmp_path):
    p = tmp_path / "bad.txt"
    p.write_text("3 1 int\n5 0 1\n")
    with pytest.raises(pb.PermError):
        pb.read_matrix(p)


def test_reader_float_rounds_like_reference(pb, tmp_path):
    p = tmp_path / "f.txt"
    p.write_text("2 2 float\n0 0 0.1\n1 1 0.3\n")
    A, t, _ = pb.read_matrix(p)
    assert A[0, 0] == float(np.float32(0.1)) and A[1, 1] == float(np.float32(0.3))


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("seed", range(4))
def test_compress_matches_reference(pb, ref, mode, seed):
    rng = np.random.default_rng(seed)
    n = 9 + 5 * seed
    A = bernoulli(rng, n, 0.3 + 0.1 * seed) * (rng.random((n, n)) + 0.5)
    if seed == 3:  # negative entries: the reference drops them from CRS/CCS
        A[rng.random((n, n)) < 0.1] *= -1
    mine = pb.compress(mode, A)
    theirs = ref.compress(mode, A)
    for k in ("cptrs", "rows", "cvals", "rptrs", "cols", "rvals", "mat"):
        np.testing.assert_array_equal(mine[k], theirs[k], err_msg=f"mode {mode} field {k}")


@pytest.mark.skipif(not (REF_SRC / "int").is_dir(), reason="reference data files not present")
@pytest.mark.parametrize("rel", ["int/30_0.50_0", "float/32_0.30_1", "double/36_0.20_0", "real/d_ss.mtxzero"])
def test_reference_data_files(pb, ref, rel):
    path = REF_SRC / rel
    for binary in (False, True):
        mine, _, _ = pb.read_matrix(path, binary=binary)
        np.testing.assert_array_equal(mine, ref.read_matrix(path, binary=binary))
    mine, _, _ = pb.read_matrix(path)
    if "real" not in rel:  # d_ss has empty rows, where the reference skipOrder is undefined
        for mode in (0, 1, 2):
            a, b = pb.compress(mode, mine), ref.compress(mode, mine)
            for k in ("cptrs", "rows", "cvals", "rptrs", "cols", "rvals", "mat"):
                np.testing.assert_array_equal(a[k], b[k])
