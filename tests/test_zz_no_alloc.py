"""perm_exact_dense_noalloc: the entry point for callers that cannot allocate
device memory (code running inside another framework's allocator, plugins in
a host process that owns every device allocation, code paths where allocating
is forbidden).  The caller provides device input and output buffers -- here
they come from torch, standing in for such a caller's own memory -- and the
engine's scratch lives in a static device array.  The result must match the
context-based perm_exact_dense on two calls in a row.

This file is collected last on purpose (pytest orders files by name)."""
import ctypes

import numpy as np
import pytest
from conftest import bernoulli, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.fixture(scope="module")
def noalloc(pb):
    lib = pb.load_library()
    fn = lib.perm_exact_dense_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    return fn


def run_noalloc(fn, A):
    import torch

    d_mat = torch.tensor(A, dtype=torch.float64, device="cuda:0")
    d_out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda:0")
    stream = torch.cuda.current_stream(0)
    rc = fn(d_mat.data_ptr(), A.shape[0], d_out.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize(0)
    out = d_out.cpu().numpy()
    return rc, float(out[0]), float(out[1])


def test_noalloc_matches_context_entry_point_twice(pb, noalloc):
    rng = np.random.default_rng(99)
    cases = [1.0 - rng.random((22, 22)), bernoulli(rng, 27, 0.5) * rng.integers(1, 5, (27, 27)), np.ones((3, 3))]
    with pb.Engine(0) as eng:
        for A in cases:
            want = eng.exact_dense(A, variant=pb.PERM_KERNEL_DENSE).value
            for _ in range(2):  # two calls in a row share (and reuse) the scratch
                rc, hi, lo = run_noalloc(noalloc, A)
                assert rc == pb.PERM_OK
                assert rel_err(hi + lo, want) < TOL, (A.shape, hi + lo, want)


def test_noalloc_rejects_what_the_scratch_cannot_hold(pb, noalloc):
    import torch

    big = torch.zeros((65, 65), dtype=torch.float64, device="cuda:0")
    out = torch.zeros(2, dtype=torch.float64, device="cuda:0")
    assert noalloc(big.data_ptr(), 65, out.data_ptr(), None) == pb.PERM_EUNSUPPORTED
    assert noalloc(None, 10, out.data_ptr(), None) == pb.PERM_EINVAL
