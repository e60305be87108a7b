"""GPU parity of the leaf operations through the C ABI (one dense block,
nb = 1): pivoted getrf against LAPACK dgetrf, and the two triangular solves
against the reference's dense_getrf / dense_trsm tests."""
import os

import numpy as np
import pytest
from scipy.linalg import lapack

import oracle.frank_oracle as fo

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _one_block(A, precision="fp64"):
    from frank_b200 import BLRMatrix
    M = BLRMatrix(A.shape[0], 1, eps=1e-12, precision=precision)
    M.set_dense(0, 0, A)
    return M


@pytest.mark.parametrize("m", [8, 16, 32])
def test_getrf_reference_grid(gpu_lib, m):
    """test/dense_getrf_test.cpp:12-43: L*U == A (diagonally boosted laplace)."""
    x = np.array([fo.get_sorted_random_vector(m)])
    A = fo.laplacend(x, 0, m, 0, m)
    d = m * m
    for i in range(m):
        A[i, i] += d
        d -= 1
    M = _one_block(A)
    M.getrf()
    LU = M.block(0, 0, which=1)
    L = np.tril(LU, -1) + np.eye(m)
    U = np.triu(LU)
    assert (M.pivots(0) == np.arange(1, m + 1)).all()
    np.testing.assert_allclose(L @ U, A, rtol=1e-15 * 8, atol=0)
    ref_lu, piv, _ = lapack.dgetrf(np.asfortranarray(A))
    np.testing.assert_allclose(LU, ref_lu, rtol=1e-13, atol=1e-13 * np.abs(ref_lu).max())


@pytest.mark.parametrize("n", [64, 100, 256, 512])
def test_getrf_pivoting_matches_lapack(gpu_lib, n):
    """Random (non-dominant) blocks: same pivots and packed LU as dgetrf."""
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n))
    M = _one_block(A)
    M.getrf()
    ref_lu, piv, _ = lapack.dgetrf(np.asfortranarray(A))
    assert (M.pivots(0) == piv + 1).all()
    LU = M.block(0, 0, which=1)
    np.testing.assert_allclose(LU, ref_lu, rtol=0, atol=1e-11 * np.abs(ref_lu).max())


@pytest.mark.parametrize("n", [8, 16, 32])
def test_solve_reference_grid(gpu_lib, n):
    """test/dense_trsm_test.cpp:10-29: |x - solve(A, A x)| <= 1e-12."""
    x = np.array([fo.get_sorted_random_vector(n)])
    A = fo.laplacend(x, 0, n, 0, n)
    xx = fo.random_uniform(n, 1)
    M = _one_block(A)
    M.getrf()
    s = M.solve(A @ xx)
    assert np.max(np.abs(s - xx)) <= 1e-12


def test_solve_matches_prototype_fixture(gpu_lib):
    g = np.load(os.path.join(GOLD, "prototype_dense_lu.npz"))
    for n in (8, 16, 32):
        M = _one_block(g["A%d" % n])
        M.getrf()
        s = M.solve(np.arange(1, n + 1, dtype=float))
        np.testing.assert_allclose(s, g["x%d" % n], rtol=1e-12, atol=0)


@pytest.mark.parametrize("n", [96, 512])
def test_transpose_solve(gpu_lib, n):
    import torch
    rng = np.random.default_rng(7)
    A = rng.standard_normal((n, n)) + n * np.eye(n) * 0.1
    M = _one_block(A)
    M.getrf()
    g = rng.standard_normal((n, 2))
    t = torch.tensor(np.asfortranarray(g).T.copy(), device="cuda", dtype=torch.float64)  # column-major n x 2
    M.solve_transpose_device(t.data_ptr(), 2)
    got = t.cpu().numpy().T
    want = np.linalg.solve(A.T, g)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-10 * np.abs(want).max())


def test_singular_block_reports_status(gpu_lib):
    from frank_b200._abi import FRANK_ERR_SINGULAR
    A = np.zeros((16, 16))
    M = _one_block(A)
    assert M.getrf(allow=(FRANK_ERR_SINGULAR,)) == FRANK_ERR_SINGULAR


def test_state_and_argument_errors(gpu_lib):
    from frank_b200 import BLRMatrix, FrankError
    from frank_b200._abi import FRANK_ERR_STATE, FRANK_ERR_INVALID
    M = _one_block(np.eye(8))
    with pytest.raises(FrankError) as e:
        M.solve(np.ones(8))
    assert e.value.code == FRANK_ERR_STATE
    with pytest.raises(FrankError) as e:
        BLRMatrix(8, 16, eps=1e-8)
    assert e.value.code == FRANK_ERR_INVALID
    with pytest.raises(FrankError) as e:
        M.set_dense(0, 1, np.eye(8))
    assert e.value.code == FRANK_ERR_INVALID
    # naive addition (FRANK_LRA=naive) grows ranks without bound: plans refuse it
    from frank_b200._abi import FRANK_ERR_UNSUPPORTED
    for name in ("naive", "no_such_addition"):
        with pytest.raises(FrankError) as e:
            M.set_lra(name)
        assert e.value.code == FRANK_ERR_UNSUPPORTED
