"""Per-operation entry points (qr, rq, svd, rsvd, id, rid, LowRank +=) through
the C ABI against the oracle's LAPACK calls (the reference's call sequence,
pinned to the reference's own outputs in test_oracle_vs_reference.py) and the
reference's known-answer criteria (test/dense_qr_test.cpp,
test/dense_svd_test.cpp, test/rsvd_test.cpp, test/dense_id_test.cpp,
test/lowrank_test.cpp).

Stated tolerances: factorizations reproduce A to 1e-13 relative and their
orthonormal factors to 1e-13; |R| equals LAPACK's |R| to 1e-12 relative
(signs of Householder reflectors may differ); singular values to 1e-12
relative; randomized and interpolative decompositions equal the oracle's
products to 1e-10 relative with the same selected rows / columns (the ID's
factors to 1e-7, the conditioning of R11); LowRank
additions equal the oracle's dense sum approximations to 1e-11 relative with
equal ranks."""
import ctypes as C

import numpy as np
import pytest

import oracle.frank_oracle as fo

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.asfortranarray(a).T.copy()).cuda()   # (cols, rows) row-major == column-major


def _host(t, m, n):
    return t.cpu().numpy().T[:m, :n].copy()


def _batch(mats):
    """Stack column-major matrices of equal shape: device (count, n, m)."""
    import torch
    return torch.stack([_dev(a) for a in mats])


def _p(t):
    return C.c_void_p(t.data_ptr())


def _ok(lib, rc):
    assert rc == 0, lib.frank_last_error()


SHAPES = [(64, 32), (33, 70), (300, 300), (512, 48)]


@pytest.mark.parametrize("m,n", SHAPES)
def test_qr_batched(gpu_lib, m, n):
    import torch
    rng = np.random.default_rng(m * 1000 + n)
    A = [rng.standard_normal((m, n)) for _ in range(3)]
    k = min(m, n)
    dA = _batch(A)
    dQ = torch.zeros((3, k, m), dtype=torch.float64, device="cuda")
    dR = torch.zeros((3, n, k), dtype=torch.float64, device="cuda")
    _ok(gpu_lib, gpu_lib.frank_qr_batched(m, n, 3, _p(dA), m, m * n, _p(dQ), m, m * k, _p(dR), k, k * n, None))
    for b in range(3):
        Q, R = dQ[b].cpu().numpy().T, dR[b].cpu().numpy().T
        np.testing.assert_allclose(Q @ R, A[b], rtol=0, atol=1e-13 * np.abs(A[b]).max() * max(m, n))
        np.testing.assert_allclose(Q.T @ Q, np.eye(k), rtol=0, atol=1e-13 * max(m, n))
        assert np.all(np.tril(R, -1) == 0)
        _, Rl = fo.qr_dense(A[b])
        np.testing.assert_allclose(np.abs(R), np.abs(Rl), rtol=0, atol=1e-12 * np.abs(Rl).max())


@pytest.mark.parametrize("m,n", SHAPES)
def test_rq_batched(gpu_lib, m, n):
    import torch
    rng = np.random.default_rng(7 * m + n)
    A = [rng.standard_normal((m, n)) for _ in range(2)]
    k = min(m, n)
    dA = _batch(A)
    dR = torch.zeros((2, k, m), dtype=torch.float64, device="cuda")
    dQ = torch.zeros((2, n, k), dtype=torch.float64, device="cuda")
    _ok(gpu_lib, gpu_lib.frank_rq_batched(m, n, 2, _p(dA), m, m * n, _p(dR), m, m * k, _p(dQ), k, k * n, None))
    for b in range(2):
        R, Q = dR[b].cpu().numpy().T, dQ[b].cpu().numpy().T
        np.testing.assert_allclose(R @ Q, A[b], rtol=0, atol=1e-13 * np.abs(A[b]).max() * max(m, n))
        np.testing.assert_allclose(Q @ Q.T, np.eye(k), rtol=0, atol=1e-13 * max(m, n))
        Rl, _ = fo.rq_dense(A[b])
        np.testing.assert_allclose(np.abs(R), np.abs(Rl), rtol=0, atol=1e-12 * np.abs(Rl).max())


@pytest.mark.parametrize("m,n", [(64, 32), (33, 70), (200, 200)])
def test_svd_batched(gpu_lib, m, n):
    """test/dense_svd_test.cpp:26 criterion (reconstruction) plus singular values vs dgesvd."""
    import torch
    rng = np.random.default_rng(m + 3 * n)
    x = np.array([fo.get_sorted_random_vector(2 * max(m, n))])
    A = [fo.laplacend(x, 0, m, max(m, n), n), rng.standard_normal((m, n))]
    k = min(m, n)
    dA = _batch(A)
    dU = torch.zeros((2, k, m), dtype=torch.float64, device="cuda")
    dS = torch.zeros((2, k), dtype=torch.float64, device="cuda")
    dV = torch.zeros((2, n, k), dtype=torch.float64, device="cuda")
    _ok(gpu_lib, gpu_lib.frank_svd_batched(m, n, 2, _p(dA), m, m * n, _p(dU), m, m * k, _p(dS), k, _p(dV), k, k * n,
                                           None))
    for b in range(2):
        U, s, Vt = dU[b].cpu().numpy().T, dS[b].cpu().numpy(), dV[b].cpu().numpy().T
        _, sl, _ = fo.svd_dense(A[b])
        np.testing.assert_allclose(s, sl, rtol=0, atol=1e-12 * sl[0])
        np.testing.assert_allclose((U * s) @ Vt, A[b], rtol=0, atol=1e-12 * sl[0])
        np.testing.assert_allclose(Vt @ Vt.T, np.eye(k), rtol=0, atol=1e-12)


@pytest.mark.parametrize("m,n,rank", [(256, 256, 16), (300, 200, 8)])
def test_rsvd_batched_matches_reference_construction(gpu_lib, m, n, rank):
    """LowRank(Dense, rank) = rsvd with oversample 5 and the reference's Omega
    (classes/low_rank.cpp:40-48): the same rank-`rank` approximation as the
    oracle; test/rsvd_test.cpp:22 criterion (< 1e-8 on a laplace block)."""
    import torch
    x = np.array([fo.get_sorted_random_vector(m + n)])
    A = fo.laplacend(x, 0, m, m, n)
    dA = _batch([A])
    dU = torch.zeros((1, rank, m), dtype=torch.float64, device="cuda")
    dS = torch.zeros((1, rank, rank), dtype=torch.float64, device="cuda")
    dV = torch.zeros((1, n, rank), dtype=torch.float64, device="cuda")
    _ok(gpu_lib, gpu_lib.frank_rsvd_batched(m, n, 1, rank, 5, 0, _p(dA), m, m * n, _p(dU), m, m * rank, _p(dS), rank,
                                            rank * rank, _p(dV), rank, rank * n, None))
    U, S, V = dU[0].cpu().numpy().T, dS[0].cpu().numpy().T, dV[0].cpu().numpy().T
    ref = fo.LowRank.from_rank(A, rank)
    np.testing.assert_allclose(U @ S @ V, ref.dense(), rtol=0, atol=1e-10 * np.linalg.norm(A))
    # singular values to 1e-13 of the largest (the small ones carry rounding)
    np.testing.assert_allclose(np.diag(S), np.diag(ref.S), rtol=0, atol=1e-13 * ref.S[0, 0])
    if rank == 16:
        assert fo.l2_error(A, U @ S @ V) < 1e-8
    # oversample 8 + one power iteration (the hierarchical workload's setting): no worse
    _ok(gpu_lib, gpu_lib.frank_rsvd_batched(m, n, 1, rank, 8, 1, _p(dA), m, m * n, _p(dU), m, m * rank, _p(dS), rank,
                                            rank * rank, _p(dV), rank, rank * n, None))
    U2, S2, V2 = dU[0].cpu().numpy().T, dS[0].cpu().numpy().T, dV[0].cpu().numpy().T
    assert fo.l2_error(A, U2 @ S2 @ V2) <= 1.01 * fo.l2_error(A, U @ S @ V)


def test_id_and_rid_reference_criterion(gpu_lib):
    """test/dense_id_test.cpp:25-60: the off-diagonal block A(0:n, n:2n) of
    laplacend on 2n sorted points, n = 2048, rank 16: id, rid (sample rank + 5)
    reproduce A to < 1e-7; the selected columns and rows and the factors equal
    the oracle's (operations/LAPACK/id.cpp)."""
    import torch
    n, k = 2048, 16
    x = np.array([fo.get_sorted_random_vector(2 * n)])
    A = fo.laplacend(x, 0, n, n, n)
    dA = _batch([A])
    dU = torch.zeros((1, k, n), dtype=torch.float64, device="cuda")
    dS = torch.zeros((1, k, k), dtype=torch.float64, device="cuda")
    dV = torch.zeros((1, n, k), dtype=torch.float64, device="cuda")
    rows = torch.zeros(k, dtype=torch.int32, device="cuda")
    cols = torch.zeros(k, dtype=torch.int32, device="cuda")
    _ok(gpu_lib, gpu_lib.frank_id_batched(n, n, 1, k, _p(dA), n, n * n, _p(dU), n, n * k, _p(dS), k, k * k, _p(dV), k,
                                          k * n, _p(rows), _p(cols), None))
    U, S, V = dU[0].cpu().numpy().T, dS[0].cpu().numpy().T, dV[0].cpu().numpy().T
    assert fo.l2_error(A, U @ S @ V) < 1e-7
    Uo, So, Vo, ro, co = fo.id_(A, k)
    assert list(cols.cpu().numpy()) == list(co)
    assert list(rows.cpu().numpy()) == list(ro)
    np.testing.assert_allclose(S, So, rtol=0, atol=1e-14 * np.abs(So).max())
    # V = R11^{-1} R12 and U carry the conditioning of R11 (its last pivot is
    # ~1e-7 of the first here): equal to the oracle's to 1e-7 relative
    np.testing.assert_allclose(V, Vo, rtol=0, atol=1e-7 * np.abs(Vo).max())
    np.testing.assert_allclose(U, Uo, rtol=0, atol=1e-7 * np.abs(Uo).max())
    _ok(gpu_lib, gpu_lib.frank_rid_batched(n, n, 1, k + 5, k, _p(dA), n, n * n, _p(dU), n, n * k, _p(dS), k, k * k,
                                           _p(dV), k, k * n, None))
    U, S, V = dU[0].cpu().numpy().T, dS[0].cpu().numpy().T, dV[0].cpu().numpy().T
    assert fo.l2_error(A, U @ S @ V) < 1e-7
    Ur, Sr, Vr = fo.rid(A, k + 5, k)
    np.testing.assert_allclose(U @ S @ V, Ur @ Sr @ Vr, rtol=0, atol=1e-10 * np.linalg.norm(A))


def _lr_add(lib, A, B, lra, eps, kmax):
    """One GPU LowRank += LowRank; A, B: oracle LowRank (U m x k, S, V k x n)."""
    import torch
    m, n = A.U.shape[0], A.V.shape[1]
    ka, kb = A.rank, B.rank
    Ua = np.zeros((m, kmax)); Ua[:, :ka] = A.U
    Sa = np.zeros((kmax, kmax)); Sa[:ka, :ka] = A.S
    Va = np.zeros((kmax, n)); Va[:ka] = A.V
    dUa, dSa, dVa = _dev(Ua), _dev(Sa), _dev(Va)
    dUb, dSb, dVb = _dev(B.U), _dev(B.S), _dev(B.V)
    dka = torch.tensor([ka], dtype=torch.int32, device="cuda")
    dkb = torch.tensor([kb], dtype=torch.int32, device="cuda")
    _ok(lib, lib.frank_lowrank_add_batched(m, n, 1, kmax, lra.encode(), eps, _p(dUa), m, 0, _p(dSa), kmax, 0, _p(dVa),
                                           kmax, 0, _p(dka), _p(dUb), m, 0, _p(dSb), kb, 0, _p(dVb), kb, 0, _p(dkb),
                                           kb, None))
    r = int(dka.cpu().item())
    U = _host(dUa, m, r)
    S = _host(dSa, r, r)
    V = _host(dVa, r, n)
    return U, S, V, r


@pytest.mark.parametrize("alg", ["rounded_addition", "fast_rounded_addition"])
@pytest.mark.parametrize("m,n", [(64, 64), (64, 21)])
@pytest.mark.parametrize("rank", [1, 4, 8])
def test_lowrank_add_fixed_rank_matches_oracle(gpu_lib, alg, m, n, rank):
    """test/lowrank_test.cpp:31-61 (fixed rank): A += B with B from the same
    block, then a LowRank of rank + 4 of it, then a LowRank of a random normal
    block; every step keeps the rank and equals the oracle's result on the
    same input (the GPU result of the previous step)."""
    x = np.array([fo.get_sorted_random_vector(2 * max(m, n))])
    DA = fo.laplacend(x, 0, m, n, n)
    A = fo.LowRank.from_rank(DA, rank)
    rng = np.random.default_rng(7)
    steps = [fo.LowRank.from_rank(DA.copy(), rank),
             fo.LowRank.from_rank(DA.copy(), min(rank + 4, min(m, n))),
             fo.LowRank.from_rank(rng.standard_normal((m, n)), rank)]
    for B in steps:
        U, S, V, r = _lr_add(gpu_lib, A, B, alg, 0.0, 2 * rank + 4)
        ref = A.copy()
        (fo.fast_rounded_addition if alg == "fast_rounded_addition" else fo.rounded_addition)(ref, B)
        assert r == ref.rank == rank
        np.testing.assert_allclose(U @ S @ V, ref.dense(), rtol=0,
                                   atol=1e-11 * (np.linalg.norm(A.dense()) + np.linalg.norm(B.dense())))
        A = fo.LowRank(U, S, V, r)


@pytest.mark.parametrize("m,n,ka,kb", [(64, 64, 4, 4), (64, 21, 8, 16), (48, 48, 20, 30)])
def test_lowrank_add_naive_matches_oracle(gpu_lib, m, n, ka, kb):
    """naive_addition (addition.cpp:68-89, FRANK_LRA=naive): concatenation when
    ka + kb < min(m, n) (exact, rank ka + kb), else LowRank(Dense(A) + Dense(B),
    ka) by rsvd with the reference's Omega -- equal to the oracle's."""
    x = np.array([fo.get_sorted_random_vector(3 * max(m, n))])
    DA = fo.laplacend(x, 0, m, n, n)
    DB = fo.laplacend(x, 0, m, 2 * n, n)
    A, B = fo.LowRank.from_rank(DA, ka), fo.LowRank.from_rank(DB, kb)
    U, S, V, r = _lr_add(gpu_lib, A, B, "naive", 0.0, ka + kb)
    ref = A.copy()
    fo.naive_addition(ref, B)
    assert r == ref.rank == (ka + kb if ka + kb < min(m, n) else ka)
    np.testing.assert_allclose(U @ S @ V, ref.dense(), rtol=0, atol=1e-10 * np.linalg.norm(DA + DB))


@pytest.mark.parametrize("m,n", [(64, 64), (64, 32)])
@pytest.mark.parametrize("eps", [1e-6, 1e-8, 1e-10])
def test_lowrank_add_fixed_accuracy_matches_oracle(gpu_lib, m, n, eps):
    """test/lowrank_test.cpp:63-115 (fixed accuracy, rounded_addition with
    find_svd_truncation_rank): same rank as the oracle, error within eps."""
    x = np.array([fo.get_sorted_random_vector(2 * max(m, n))])
    DA = fo.laplacend(x, 0, m, n, n)
    A = fo.LowRank.from_eps(DA, eps)
    B = fo.LowRank.from_eps(DA.copy(), eps)
    U, S, V, r = _lr_add(gpu_lib, A, B, "rounded_addition", eps, min(m, n))
    ref = A.copy()
    fo.rounded_addition(ref, B)
    assert r == ref.rank
    np.testing.assert_allclose(U @ S @ V, ref.dense(), rtol=0, atol=1e-11 * np.linalg.norm(DA))
    assert abs(fo.l2_error(DA + DA, U @ S @ V) - eps) <= 10 * eps
