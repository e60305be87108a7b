"""GPU parity of the multi-level H-LU (binary cluster tree, weak
admissibility, fixed rank) through the C ABI against the oracle's recursive
getrf_omm(Hierarchical), on the reference's hierarchical_fixed_rank_test grid
(n 128 / 256, nleaf 32, rank 4 / 8) and the h_lu example's defaults (n 256,
nleaf 16, rank 8).  Tolerances, stated per check:
  * construction: every block within 1e-9 (relative, Frobenius) of the
    oracle's LowRank(Dense, rank) with the same Omega;
  * factor blocks from identical inputs: leaves within 1e-10, LowRank
    blocks (U S V) within 1e-8 of the oracle's L and U;
  * solve (examples/h_lu.cpp: b = A_H x, trsm L, trsm U): error within a
    factor 10 of the oracle's plus 1e-13.
"""
import numpy as np
import pytest

import oracle.frank_oracle as fo

pytestmark = pytest.mark.gpu


def _points(n):
    return np.array([fo.get_sorted_random_vector(n)])


def _oracle_h(n, leaf, rank):
    return fo.build_hierarchical(fo.laplacend, _points(n), n, leaf, 2, rank=rank)


def _blocks(H, level=0, index=0, out=None):
    """{('D', p): array, ('L', l, c): LowRank} of a nested nb = 2 Hierarchical."""
    out = {} if out is None else out
    for i in range(2):
        for j in range(2):
            ch = H[i, j]
            if i == j:
                ci = 2 * index + i
                if isinstance(ch, np.ndarray):
                    out[("D", ci)] = ch
                else:
                    _blocks(ch, level + 1, ci, out)
            else:
                out[("L", level + 1, 2 * index + i)] = ch
    return out


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


CASES = [(128, 32, 4), (128, 32, 8), (256, 32, 4), (256, 32, 8), (256, 16, 8)]


@pytest.mark.parametrize("n,leaf,rank", CASES)
def test_hodlr_construction_matches_oracle(n, leaf, rank):
    from frank_b200 import HMatrix
    H = _oracle_h(n, leaf, rank)
    M = HMatrix(n, leaf, rank)
    M.build_kernel("laplace", _points(n))
    for key, blk in _blocks(H).items():
        if key[0] == "D":
            assert _rel(M.get_dense(key[1]), blk) < 1e-13, key
        else:
            U, S, V = M.get_lowrank(key[1], key[2])
            assert _rel(U @ S @ V, blk.dense()) < 1e-9, (key, _rel(U @ S @ V, blk.dense()))
            # orthonormal bases, as rsvd returns them
            assert np.abs(U.T @ U - np.eye(rank)).max() < 1e-12
            assert np.abs(V @ V.T - np.eye(rank)).max() < 1e-12
    M.close()


@pytest.mark.parametrize("lra", ["fast_rounded_addition", "rounded_addition"])
@pytest.mark.parametrize("n,leaf,rank", CASES)
def test_hodlr_factor_blocks_match_oracle(n, leaf, rank, lra):
    from frank_b200 import upload_hmatrix
    H = _oracle_h(n, leaf, rank)
    M = upload_hmatrix(H, n, leaf, rank, lra)
    M.getrf()
    old = fo.LRA_MODE["mode"]
    fo.LRA_MODE["mode"] = lra
    try:
        L, U = fo.getrf(fo.deep_copy(H))
    finally:
        fo.LRA_MODE["mode"] = old
    bl, bu = _blocks(L), _blocks(U)
    for p in range(n // leaf):
        assert (M.get_pivots(p) == np.arange(leaf)).all(), "leaf %d pivoted" % p
        lu = M.get_dense(p, factor=True)
        assert _rel(np.tril(lu, -1) + np.eye(leaf), bl[("D", p)]) < 1e-10
        assert _rel(np.triu(lu), bu[("D", p)]) < 1e-10
    for key in bl:
        if key[0] != "L":
            continue
        l, c = key[1], key[2]
        ref = (bl if c % 2 else bu)[key].dense()
        Uf, Sf, Vf = M.get_lowrank(l, c, factor=True)
        assert _rel(Uf @ Sf @ Vf, ref) < 1e-8, (key, _rel(Uf @ Sf @ Vf, ref))
    M.close()


@pytest.mark.parametrize("n,leaf,rank", CASES + [(2048, 64, 16)])
def test_hodlr_solve_matches_oracle(n, leaf, rank):
    """examples/h_lu.cpp:18-54: x = random_uniform(N), b = A_H x, getrf,
    trsm(L), trsm(U); the error l2_error(x, solution)."""
    from frank_b200 import HMatrix
    x = fo.random_uniform(n, 1)
    M = HMatrix(n, leaf, rank)
    M.build_kernel("laplace", _points(n))
    b = M.matvec(x)
    H = _oracle_h(n, leaf, rank)
    b_ref = fo.matvec(H, x)
    assert _rel(b, b_ref) < 1e-12
    M.getrf()
    sol = M.solve(b)
    L, U = fo.getrf(fo.deep_copy(H))
    sol_ref = fo.solve(L, U, b_ref)
    err, err_ref = fo.l2_error(x, sol), fo.l2_error(x, sol_ref)
    assert err <= 10.0 * err_ref + 1e-13, (err, err_ref)
    assert _rel(sol, sol_ref) < 1e-8
    # the two triangular solves one at a time, as trsm(L, b, Lower) and
    # trsm(U, b, Upper) (trsm.cpp:40-90 through the oracle's recursion)
    y = M.trsm(b, lower=True)
    y_ref = fo.trsm(L, np.array(b_ref, copy=True), upper=False, left=True)
    assert _rel(y, y_ref) < 1e-8
    z = M.trsm(y, lower=False)
    z_ref = fo.trsm(U, np.array(y_ref, copy=True), upper=True, left=True)
    assert _rel(z, z_ref) < 1e-8
    M.close()


def test_hodlr_refine_to_1e10():
    """Laplace-3D on Morton-ordered unit-cube points (n 8192, leaf 256,
    rank 32): the factorization preconditions FP64 refinement against A_H to
    a residual of 1e-10."""
    from frank_b200 import HMatrix
    import bench
    n = 8192
    pts = bench.make_points(n, 3, 5, 6)
    M = HMatrix(n, 256, 32)
    M.build_kernel("laplace", pts)
    M.getrf()
    rng = np.random.default_rng(0)
    b = rng.standard_normal((n, 8))
    x, it, res = M.refine(b, tol=1e-10, maxit=30)
    assert res <= 1e-10
    r = b - M.matvec(x)
    assert (np.linalg.norm(r, axis=0) / np.linalg.norm(b, axis=0)).max() < 1e-9
    # a second getrf replays the captured graph from A_H and gives the same factor
    lu0 = M.get_dense(3, factor=True)
    M.getrf()
    assert np.array_equal(lu0, M.get_dense(3, factor=True))
    M.close()


def test_hodlr_rejects_bad_shapes():
    from frank_b200 import HMatrix, FrankError
    with pytest.raises(FrankError):
        HMatrix(96 * 3, 32, 8)      # n / leaf not a power of two
    with pytest.raises(FrankError):
        HMatrix(256, 32, 40)        # rank above the leaf order
    M = HMatrix(256, 32, 8)
    with pytest.raises(FrankError):
        M.set_lra("naive")
    with pytest.raises(FrankError):
        M.solve(np.ones(256))       # before getrf
    M.close()
