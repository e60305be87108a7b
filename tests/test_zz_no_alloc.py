"""The allocation-free dense getrf (frank_getrf_dense_noalloc), for callers
that cannot call cudaMalloc (an allocator callback, an out-of-memory recovery
path, a pool that forbids growth).  It must give the same factor and pivots
as the plan-based path (frank_blr_getrf on a one-block plan) on two calls in a
row -- the calls share one fixed scratch array -- and reject orders above its
fixed maximum with a clear status.  Collected last so a first-failure run has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib, A_dev, n, lda, lu_dev, piv_dev):
    return lib.frank_getrf_dense_noalloc(C.c_void_p(A_dev.data_ptr()), lda, n, C.c_void_p(lu_dev.data_ptr()),
                                         n, C.c_void_p(piv_dev.data_ptr()), None)


def _plan_factor(A):
    from frank_b200 import BLRMatrix
    M = BLRMatrix(A.shape[0], 1, eps=1e-12)
    M.set_dense(0, 0, A)
    M.getrf()
    lu, piv = M.block(0, 0, which=1), M.pivots(0)
    M.close()
    return lu, piv


@pytest.mark.parametrize("n", [48, 256])
def test_noalloc_getrf_matches_plan_path_twice(gpu_lib, n):
    import torch
    from frank_b200._abi import FRANK_OK
    rng = np.random.default_rng(n)
    lda = n + 3
    for call in range(2):                      # two calls in a row share the scratch
        A = rng.standard_normal((n, n)) + (0.5 * n * np.eye(n) if call else 0.0)
        A_pad = np.zeros((n, lda))             # column-major with lda: rows of A_pad^T
        A_pad[:, :n] = A.T
        A_dev = torch.from_numpy(A_pad).cuda()
        lu_dev = torch.full((n, n), np.nan, dtype=torch.float64, device="cuda")
        piv_dev = torch.zeros(n, dtype=torch.int32, device="cuda")
        assert _noalloc(gpu_lib, A_dev, n, lda, lu_dev, piv_dev) == FRANK_OK, gpu_lib.frank_last_error()
        lu = lu_dev.cpu().numpy().T            # back to row-major (i, j)
        piv = piv_dev.cpu().numpy()
        ref_lu, ref_piv = _plan_factor(A)
        assert (piv == ref_piv).all()
        np.testing.assert_allclose(lu, ref_lu, rtol=0, atol=1e-11 * np.abs(ref_lu).max())
        # the input is left unchanged
        np.testing.assert_array_equal(A_dev.cpu().numpy()[:, :n], A.T)


def test_noalloc_getrf_rejects_oversize(gpu_lib):
    import torch
    from frank_b200._abi import FRANK_ERR_UNSUPPORTED
    n = 257
    A_dev = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    lu_dev = torch.zeros_like(A_dev)
    piv_dev = torch.zeros(n, dtype=torch.int32, device="cuda")
    assert _noalloc(gpu_lib, A_dev, n, n, lu_dev, piv_dev) == FRANK_ERR_UNSUPPORTED
    assert b"outside" in gpu_lib.frank_last_error()
