"""CPU tests of the oracle: pinned against libstdc++ RNG outputs, the
reference's Python prototype (tests/golden) and the known-answer checks of
the reference's own GTest suites (grids and tolerances restated)."""
import os

import numpy as np
import pytest

import oracle.frank_oracle as fo

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _gold_rng(suffix=""):
    raw, uni, nor = [], [], []
    for line in open(os.path.join(GOLD, "libstdcxx_mt19937_seed0.txt")):
        k, v = line.split()
        d = {"raw" + suffix: raw, "uniform" + suffix: uni, "normal" + suffix: nor}.get(k)
        if d is not None:
            d.append(int(v) if k.startswith("raw") else float(v))
    return raw, uni, nor


def test_mt19937_streams_match_libstdcxx():
    raw, uni, nor = _gold_rng()
    assert list(fo.StdMT19937(0).raw(len(raw))) == [int(v) for v in raw]
    np.testing.assert_array_equal(fo.StdMT19937(0).uniform(len(uni)), np.array(uni))
    np.testing.assert_allclose(fo.StdMT19937(0).normal(len(nor)), np.array(nor), rtol=0, atol=1e-15)


def test_mt19937_64_streams_match_libstdcxx():
    """The benchmark's input streams (std::mt19937_64 seeded 2 for points, 3
    for right-hand sides) against g++ output."""
    from bench import MT19937_64
    raw, uni, nor = _gold_rng("64")
    assert [int(v) for v in MT19937_64(2).raw(len(raw))] == raw
    np.testing.assert_array_equal(MT19937_64(2).uniform(len(uni)), np.array(uni))
    np.testing.assert_allclose(MT19937_64(3).normal(len(nor)), np.array(nor), rtol=0, atol=1e-15)
    g = MT19937_64(3)          # drawn in pieces: the cached second variate carries over
    pieces = np.concatenate([g.normal(101), g.normal(300), g.normal(len(nor) - 401)])
    np.testing.assert_allclose(pieces, np.array(nor), rtol=0, atol=1e-15)


def test_prototype_dense_lu_fixture():
    g = np.load(os.path.join(GOLD, "prototype_dense_lu.npz"))
    for n in (8, 16, 32):
        A = g["A%d" % n]
        L, U = fo.getrf_dense(A.copy())
        LU = np.tril(L, -1) + U
        np.testing.assert_allclose(LU, g["LU%d" % n], rtol=1e-14, atol=0)
        b = np.arange(1, n + 1, dtype=float)[:, None]
        x = fo.trsm_dense(U, fo.trsm_dense(L, b, False, True), True, True)
        np.testing.assert_allclose(x, g["x%d" % n], rtol=1e-12, atol=0)


@pytest.mark.parametrize("m", [8, 16, 32])
def test_dense_getrf_reference_grid(m):
    """test/dense_getrf_test.cpp:12-43 (EXPECT_DOUBLE_EQ on L*U == A)."""
    x = np.array([fo.get_sorted_random_vector(m)])
    A = fo.laplacend(x, 0, m, 0, m)
    d = m * m
    for i in range(m):
        A[i, i] += d
        d -= 1
    L, U = fo.getrf_dense(A.copy())
    np.testing.assert_allclose(L @ U, A, rtol=4 * np.finfo(float).eps * 4, atol=0)


@pytest.mark.parametrize("n", [8, 16, 32])
def test_dense_trsm_reference_grid(n):
    """test/dense_trsm_test.cpp:10-29 (|x - b| <= 1e-12)."""
    x = np.array([fo.get_sorted_random_vector(n)])
    A = fo.laplacend(x, 0, n, 0, n)
    xx = fo.random_uniform(n, 1)
    b = A @ xx
    L, U = fo.getrf_dense(A.copy())
    s = fo.trsm_dense(U, fo.trsm_dense(L, b, False, True), True, True)
    assert np.max(np.abs(s - xx)) <= 1e-12


def test_rsvd_reference_case():
    """test/rsvd_test.cpp:12-23: LowRank(A, 16) of a 2048^2 laplace block, error < 1e-8."""
    n = 2048
    x = np.array([fo.get_sorted_random_vector(2 * n)])
    A = fo.laplacend(x, 0, n, n, n)
    LR = fo.LowRank.from_rank(A, 16)
    assert fo.l2_error(A, LR) < 1e-8


@pytest.mark.parametrize("alg", ["rounded_addition", "fast_rounded_addition"])
@pytest.mark.parametrize("m,n", [(64, 64), (64, 21), (32, 64), (32, 21)])
@pytest.mark.parametrize("rank", [1, 2, 4, 8])
def test_lowrank_fixed_rank_addition(alg, m, n, rank):
    """test/lowrank_test.cpp:31-61: the rank is preserved by +=."""
    fo.LRA_MODE["mode"] = alg
    try:
        x = np.array([fo.get_sorted_random_vector(2 * max(m, n))])
        DA = fo.laplacend(x, 0, m, n, n)
        A = fo.LowRank.from_rank(DA, rank)
        fo.add_into(A, fo.LowRank.from_rank(DA.copy(), rank))
        assert A.rank == rank and A.U.shape[1] == rank
        fo.add_into(A, fo.LowRank.from_rank(DA.copy(), min(rank + 4, min(m, n))))
        assert A.rank == rank
        DD = fo.random_normal(m, n)
        fo.add_into(A, fo.LowRank.from_rank(DD, rank))
        assert A.rank == rank
    finally:
        fo.LRA_MODE["mode"] = "rounded_addition"


@pytest.mark.parametrize("alg", ["rounded_addition", "fast_rounded_addition"])
@pytest.mark.parametrize("m,n", [(64, 64), (64, 32), (32, 64), (32, 32)])
@pytest.mark.parametrize("eps", [1e-6, 1e-8, 1e-10, 1e-12])
def test_lowrank_fixed_accuracy(alg, m, n, eps):
    """test/lowrank_test.cpp:63-115: construction and += keep the error within eps +- 10 eps."""
    fo.LRA_MODE["mode"] = alg
    try:
        x = np.array([fo.get_sorted_random_vector(2 * max(m, n))])
        DA = fo.laplacend(x, 0, m, n, n)
        A = fo.LowRank.from_eps(DA, eps)
        assert abs(fo.l2_error(DA, A) - eps) <= 10 * eps
        B = fo.LowRank.from_eps(DA.copy(), eps)
        fo.add_into(A, B)
        assert abs(fo.l2_error(DA + DA, A) - eps) <= 10 * eps
        C = fo.LowRank.from_eps(DA.copy(), eps * 1e-2)
        fo.add_into(A, C)
        assert abs(fo.l2_error(DA + DA + DA, A) - eps) <= 10 * eps
        DD = fo.random_normal(m, n)
        fo.add_into(A, fo.LowRank.from_eps(DD, eps))
        assert abs(fo.l2_error(DA + DA + DA + DD, A) - eps) <= 10 * eps
    finally:
        fo.LRA_MODE["mode"] = "rounded_addition"


BLR_GRID = [(n, eps, admis, at) for n in (128, 256) for eps in (1e-6, 1e-8, 1e-10)
            for admis in (0.0, 1.0, 4.0) for at in (fo.POSITION_BASED, fo.GEOMETRY_BASED)]


@pytest.mark.parametrize("n,eps,admis,at", BLR_GRID)
def test_blr_fixed_accuracy_lu(n, eps, admis, at):
    """test/blr_fixed_acc_test.cpp:46-83 with FRANK_LRA=rounded_addition:
    compression error <= eps and BLR-LU solve error <= eps."""
    x = np.array([fo.get_sorted_random_vector(n)])
    D = fo.laplacend(x, 0, n, 0, n)
    A = fo.build_hierarchical(fo.laplacend, x, n, 32, n // 32, eps=eps, admis=admis, admis_type=at)
    assert fo.l2_error(D, A) <= eps
    xv = fo.random_uniform(n, 1)
    b = fo.matvec(A, xv)
    L, U = fo.getrf(A)
    assert fo.l2_error(xv, fo.solve(L, U, b)) <= eps


@pytest.mark.parametrize("n,eps,admis,at", BLR_GRID)
def test_hierarchical_fixed_accuracy_lu(n, eps, admis, at):
    """test/hierarchical_fixed_acc_test.cpp:29-66 (nb = 2, recursive H-LU)."""
    x = np.array([fo.get_sorted_random_vector(n)])
    D = fo.laplacend(x, 0, n, 0, n)
    A = fo.build_hierarchical(fo.laplacend, x, n, 32, 2, eps=eps, admis=admis, admis_type=at)
    assert fo.l2_error(D, A) <= eps
    xv = fo.random_uniform(n, 1)
    b = fo.matvec(A, xv)
    L, U = fo.getrf(A)
    assert fo.l2_error(xv, fo.solve(L, U, b)) <= eps


@pytest.mark.parametrize("n", [128, 256])
@pytest.mark.parametrize("rank", [4, 8])
@pytest.mark.parametrize("admis", [0.0, 0.5, 1.0, 2.0])
def test_blr_fixed_rank_uniform(n, rank, admis):
    """test/blr_fixed_rank_test.cpp:44-55: every LowRank block has the rank."""
    x = np.array([fo.get_sorted_random_vector(n)])
    A = fo.build_hierarchical(fo.laplacend, x, n, 32, n // 32, rank=rank, admis=admis)
    assert all(k == rank for (_, _, k) in fo.blr_ranks(A))


def test_find_svd_truncation_rank_quirk():
    """misc.cpp:133-146: the tail sums S(rank,rank)^2 (min_dim - rank) times."""
    s = np.array([1.0, 1e-3, 1e-4, 1e-9])
    # threshold = 1e-6 * ||s||; rank 2: sqrt(2)*1e-4 > thr; rank 3: 1e-9 < thr
    assert fo.find_svd_truncation_rank(s, 1e-6) == 3
    assert fo.find_svd_truncation_rank(np.array([1.0]), 1e-6) == 1


def test_split_range_matches_index_range():
    """index_range.cpp:15-24 ceil-div split."""
    assert fo.split_range(0, 10, 3) == [(0, 4), (4, 4), (8, 2)]
    assert fo.split_range(0, 2048, 8) == [(256 * i, 256) for i in range(8)]
