"""The CPU oracle pinned to the reference's own outputs.

tests/golden/reference_blr.json and reference_vectors.npz were produced by
the reference itself (FRANK's C++ sources compiled unmodified into
oracle/_ref and driven through its public API; tests/golden/make_ref_golden.py).
Here the oracle (oracle/frank_oracle.py, the numpy restatement used as the
checker of the GPU path) runs the same cases and must agree with them:
per-block ranks of A_H and of the factors L and U (the rank decisions of
construction and of every recompression), and the solve / factorization
errors within a stated factor."""
import json
import os

import numpy as np
import pytest

import oracle.frank_oracle as fo

GOLD = os.path.join(os.path.dirname(__file__), "golden")
REF = json.load(open(os.path.join(GOLD, "reference_blr.json")))
VEC = np.load(os.path.join(GOLD, "reference_vectors.npz"))

# Errors of the oracle may differ from the reference's by roundoff in
# different BLAS kernels (row-major LAPACKE vs column-major Fortran calls):
# errors agree within this factor, plus an absolute floor at roundoff.
ERR_FACTOR, ERR_FLOOR = 3.0, 1e-13


def block_ranks(H):
    """Ranks of the blocks of a one-level block matrix, row-major (-1: not low rank)."""
    out = []
    for i in range(H.dim[0]):
        for j in range(H.dim[1]):
            b = H[i, j]
            out.append(b.rank if isinstance(b, fo.LowRank) else -1)
    return out


def run_case(c):
    n, nb = c["n"], c["n"] // c["nleaf"]
    at = fo.GEOMETRY_BASED if c["admis_type"] == "geometry" else fo.POSITION_BASED
    x = np.array([fo.get_sorted_random_vector(n)])
    kw = dict(rank=c["rank"]) if "rank" in c else dict(eps=c["eps"])
    A = fo.build_hierarchical(fo.laplacend, x, n, c["nleaf"], nb, admis=c["admis"], admis_type=at, **kw)
    ranks_h = block_ranks(A)
    xv = fo.random_uniform(n, 1)
    b = fo.matvec(A, xv)
    fo.LRA_MODE["mode"] = "fast_rounded_addition" if c["lra"] == "fast_rounded_addition" else c["lra"]
    try:
        L, U = fo.getrf(fo.deep_copy(A))
    finally:
        fo.LRA_MODE["mode"] = "rounded_addition"
    xs = fo.solve(L, U, b)
    return ranks_h, block_ranks(L), block_ranks(U), fo.l2_error(xv, xs)


CASES = REF["cases"]


@pytest.mark.parametrize("c", CASES, ids=["%s-%s-n%d-%s-a%g-%s" % (c["grid"], c["lra"], c["n"],
                                                                     ("e%g" % c["eps"]) if "eps" in c else
                                                                     ("k%d" % c["rank"]), c["admis"],
                                                                     c["admis_type"]) for c in CASES])
def test_oracle_matches_reference_grid(c):
    ranks_h, ranks_l, ranks_u, err = run_case(c)
    assert ranks_h == c["ranks_h"]
    assert ranks_l == c["ranks_l"]
    assert ranks_u == c["ranks_u"]
    assert err <= ERR_FACTOR * c["solve_error"] + ERR_FLOOR, (err, c["solve_error"])
    assert c["solve_error"] <= ERR_FACTOR * err + ERR_FLOOR, (err, c["solve_error"])


@pytest.mark.parametrize("lra", ["fast", "rounded_addition"])
def test_oracle_matches_reference_fixed_rank_2048(lra):
    """Fixed-rank Laplace-1D N=2048, 8 x 8 blocks of 256, rank 16: solution and
    the singular values of every low-rank factor block."""
    tag = "cfg1_" + lra
    n, nb = 2048, 8
    x = np.array([fo.get_sorted_random_vector(n)])
    A = fo.build_hierarchical(fo.laplacend, x, n, 256, nb, rank=16)
    xv = fo.random_uniform(n, 1)
    b = fo.matvec(A, xv)
    fo.LRA_MODE["mode"] = "fast_rounded_addition" if lra == "fast" else lra
    try:
        L, U = fo.getrf(fo.deep_copy(A))
    finally:
        fo.LRA_MODE["mode"] = "rounded_addition"
    xs = fo.solve(L, U, b)[:, 0]
    xr = VEC[tag + "/x"]
    assert np.linalg.norm(xs - xr) <= 1e-9 * np.linalg.norm(xr)
    for side, F in (("L", L), ("U", U)):
        for i in range(nb):
            for j in range(nb):
                key = "%s/sv/%s/%d/%d" % (tag, side, i, j)
                if key in VEC:
                    blk = F[i, j]
                    sv = np.linalg.svd(fo.to_dense(blk), compute_uv=False)[: len(VEC[key])]
                    np.testing.assert_allclose(sv, VEC[key], rtol=1e-8, atol=1e-12 * VEC[key][0])
