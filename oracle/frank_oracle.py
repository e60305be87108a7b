"""CPU oracle for FRANK's BLR / H-LU factor-and-solve path.

TEST INFRASTRUCTURE ONLY.  This module is the checker: `tests/`,
`__graft_entry__.smoke()` and the `cpu_baseline` / `--impl reference` legs of
`bench.py` may import it.  The product (`frank_b200`) never imports, calls or
links it, and has no CPU fallback.

What it is: a restatement of the reference algorithm in numpy, calling the
*same* LAPACK / BLAS routines the reference calls (dgetrf, dtrsm, dgemm,
dgeqrf + dorgqr, dgerqf + dorgrq, dgesvd, dlarfg, dnrm2 ...) through
`scipy.linalg.lapack` / `scipy.linalg.blas` on scipy's bundled OpenBLAS.
The reference calls them through LAPACKE/CBLAS in row-major mode; LAPACKE
transposes row-major input into a column-major copy of the *same* matrix,
so calling the Fortran routine on the same matrix reproduces the reference's
arithmetic up to BLAS-kernel roundoff.

Every function cites the reference file:line it restates (paths are within
the FRANK project).  The reference C++ cannot be compiled here: it needs
yomm2 (absent, fetched unpinned from GitHub master), CBLAS/LAPACKE headers
and libraries (absent) and a cmake build; so the oracle is a port ("kind":
"port"), pinned against the reference's own known-answer tests (test/*.cpp
grids and tolerances) and against std::mt19937 / libstdc++ distribution
outputs compiled from the C++ standard library here (tests/golden/).

Matrices are numpy float64 arrays in logical (row, col) order.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np
from scipy.linalg import blas, lapack

# --------------------------------------------------------------------------
# Random numbers: std::mt19937 + libstdc++ distributions
# --------------------------------------------------------------------------


class StdMT19937:
    """std::mt19937 seeded with `gen.seed(s)` (Knuth init_genrand), as used by
    random_uniform / random_normal (functions.cpp:36-66) and
    get_sorted_random_vector (util/experiment_setup.cpp:12-23).

    numpy's MT19937 `_legacy_seeding` is the same init_genrand routine, and
    `random_raw` returns the raw 32-bit outputs."""

    def __init__(self, seed: int):
        self._bg = np.random.MT19937()
        self._bg._legacy_seeding(seed)
        self._saved: Optional[float] = None

    def raw(self, n: int) -> np.ndarray:
        return self._bg.random_raw(n).astype(np.uint64)

    def canonical(self, n: int) -> np.ndarray:
        """std::generate_canonical<double, 53> for a 32-bit engine:
        two draws, (g1 + g2 * 2^32) / 2^64 in double, clamped below 1."""
        r = self.raw(2 * n).astype(np.float64)
        s = r[0::2] + r[1::2] * 4294967296.0
        out = s / 18446744073709551616.0
        out[out >= 1.0] = np.nextafter(1.0, 0.0)
        return out

    def uniform(self, n: int, a: float = 0.0, b: float = 1.0) -> np.ndarray:
        """std::uniform_real_distribution<double>(a, b): u * (b - a) + a."""
        return self.canonical(n) * (b - a) + a

    def normal(self, n: int) -> np.ndarray:
        """std::normal_distribution<double>(0, 1) of libstdc++: Marsaglia polar
        method, the second variate of each accepted pair cached."""
        out = np.empty(n)
        for i in range(n):
            if self._saved is not None:
                out[i] = self._saved
                self._saved = None
                continue
            while True:
                x = 2.0 * float(self.canonical(1)[0]) - 1.0
                y = 2.0 * float(self.canonical(1)[0]) - 1.0
                r2 = x * x + y * y
                if not (r2 > 1.0 or r2 == 0.0):
                    break
            mult = math.sqrt(-2.0 * math.log(r2) / r2)
            self._saved = x * mult
            out[i] = y * mult
        return out


def get_sorted_random_vector(n: int) -> np.ndarray:
    """util/experiment_setup.cpp:12-23: n uniform[0,1) draws of mt19937(0), sorted."""
    return np.sort(StdMT19937(0).uniform(n))


def random_uniform(rows: int, cols: int = 1) -> np.ndarray:
    """functions.cpp:52-66: row-major fill from a freshly seeded mt19937(0)."""
    return StdMT19937(0).uniform(rows * cols).reshape(rows, cols)


def random_normal(rows: int, cols: int = 1) -> np.ndarray:
    """functions.cpp:36-50: row-major fill from a freshly seeded mt19937(0)."""
    return StdMT19937(0).normal(rows * cols).reshape(rows, cols)


# --------------------------------------------------------------------------
# Kernel functions (functions.cpp) + the two kernels the workloads add
# --------------------------------------------------------------------------

Points = np.ndarray  # shape (dim, N), the reference's params[d][i] layout


def _dist(x: Points, r0: int, nr: int, c0: int, nc: int) -> np.ndarray:
    xi = x[:, r0:r0 + nr]
    xj = x[:, c0:c0 + nc]
    acc = np.zeros((nr, nc))
    for k in range(x.shape[0]):
        d = xi[k][:, None] - xj[k][None, :]
        acc += d * d
    return np.sqrt(acc)


def laplacend(x: Points, r0: int, nr: int, c0: int, nc: int) -> np.ndarray:
    """functions.cpp:92-109: 1 / (sqrt(sum_k (x_k[i]-x_k[j])^2) + 1e-3)."""
    return 1.0 / (_dist(x, r0, nr, c0, nc) + 1e-3)


def helmholtznd(x: Points, r0: int, nr: int, c0: int, nc: int) -> np.ndarray:
    """functions.cpp:111-128: exp(-r^2) / (r + 1e-3)."""
    r = _dist(x, r0, nr, c0, nc)
    return np.exp(-1.0 * r * r) / (r + 1e-3)


def cauchy2d(x: Points, r0: int, nr: int, c0: int, nc: int) -> np.ndarray:
    """functions.cpp:79-90: 1 / (x0[i] - x1[j] + 1e-2)."""
    return 1.0 / ((x[0][r0:r0 + nr][:, None] - x[1][c0:c0 + nc][None, :]) + 1e-2)


def _diag_mask(r0: int, nr: int, c0: int, nc: int) -> np.ndarray:
    return (np.arange(r0, r0 + nr)[:, None] == np.arange(c0, c0 + nc)[None, :])


def make_neglog_shift(shift: float):
    """-log(r + 1e-3) + shift * delta_ij: the 2-D log kernel of the batched
    workload, written in the reference's kernel plug-in form (dense.h:192-201)."""
    def k(x, r0, nr, c0, nc):
        return -np.log(_dist(x, r0, nr, c0, nc) + 1e-3) + shift * _diag_mask(r0, nr, c0, nc)
    return k


def make_exp_kernel(theta: float, nugget: float = 1e-2):
    """exp(-r / theta) + nugget * delta_ij: the kernel of the adjoint workload."""
    def k(x, r0, nr, c0, nc):
        return np.exp(-_dist(x, r0, nr, c0, nc) / theta) + nugget * _diag_mask(r0, nr, c0, nc)
    return k


def morton_sort(x: Points, level: int) -> Tuple[Points, np.ndarray]:
    """operations/misc/morton_index.cpp:36-98: normalise into a box padded by
    0.5, interleave `level` bits per axis (axis d at bit dim*lev + d), stable
    sort by box number."""
    dim, n = x.shape
    eps = 5e-1
    bmin = x.min(axis=1) - eps
    bsize = float((x.max(axis=1) - x.min(axis=1)).max()) + 2 * eps
    xn = (x - bmin[:, None]) / bsize
    nx = 1 << level
    ix = (xn * nx).astype(np.int64)
    code = np.zeros(n, dtype=np.int64)
    for lev in range(level):
        for d in range(dim):
            code += (ix[d] & 1) << (dim * lev + d)
            ix[d] >>= 1
    perm = np.argsort(code, kind="stable")
    return x[:, perm].copy(), perm


# --------------------------------------------------------------------------
# Index ranges, cluster tree, admissibility
# --------------------------------------------------------------------------


def split_range(start: int, n: int, n_splits: int) -> List[Tuple[int, int]]:
    """classes/initialization_helpers/index_range.cpp:15-24: ceil-div split,
    the last part takes the remainder."""
    out = []
    child = (n + n_splits - 1) // n_splits
    for i in range(n_splits):
        cn = child if i < n_splits - 1 else n - child * (n_splits - 1)
        out.append((start + child * i, cn))
    return out


POSITION_BASED = 0
GEOMETRY_BASED = 1


def is_admissible(rows, cols, abs_pos, admis, admis_type, x) -> bool:
    """classes/initialization_helpers/matrix_initializer.cpp:51-91."""
    ok = rows[1] > 1 and cols[1] > 1
    if admis_type == POSITION_BASED:
        ok = ok and (abs(abs_pos[0] - abs_pos[1]) > int(admis))
    else:
        rc = x[:, rows[0]:rows[0] + rows[1]]
        cc = x[:, cols[0]:cols[0] + cols[1]]
        off = 5e-1
        minr, maxr = rc.min(axis=1) - off, rc.max(axis=1) + off
        minc, maxc = cc.min(axis=1) - off, cc.max(axis=1) + off
        cr = minr + (maxr - minr) / 2.0
        ccen = minc + (maxc - minc) / 2.0
        dist = float(((cr - ccen) ** 2).sum())
        diam = max(float((maxr - minr).max()), float((maxc - minc).max()))
        ok = ok and (admis * admis * diam * diam < dist)
    return ok


# --------------------------------------------------------------------------
# Dense LAPACK / BLAS leaf operations
# --------------------------------------------------------------------------

DLAMCH_E = float(lapack.dlamch("e"))


def getrf_dense(A: np.ndarray, return_piv: bool = False):
    """operations/LAPACK/getrf.cpp:67-84: dgetrf, split into unit-L and U.
    The pivot vector is discarded, exactly as the reference does (so L·U = P·A;
    equal to A only when dgetrf swapped no rows)."""
    lu, piv, info = lapack.dgetrf(np.asfortranarray(A))
    n = A.shape[0]
    L = np.tril(lu, -1)[:, :n] + np.eye(A.shape[0], min(A.shape))
    U = np.triu(lu)
    if return_piv:
        return L, U, piv, info
    return L, U


def trsm_dense(A: np.ndarray, B: np.ndarray, upper: bool, left: bool) -> np.ndarray:
    """operations/BLAS/trsm.cpp:92-104: cblas_dtrsm, Upper -> NonUnit,
    Lower -> Unit diagonal. Returns the solved B."""
    return blas.dtrsm(1.0, np.asfortranarray(A), np.asfortranarray(B),
                      side=0 if left else 1, lower=0 if upper else 1,
                      trans_a=0, diag=0 if upper else 1)


def gemm(A, B, alpha=1.0, ta=False, tb=False):
    """operations/BLAS/gemm.cpp:126-146 (cblas_dgemm) for a new result."""
    return blas.dgemm(alpha, np.asfortranarray(A), np.asfortranarray(B), trans_a=ta, trans_b=tb)


def qr_dense(A: np.ndarray, q_cols: Optional[int] = None, r_rows: Optional[int] = None):
    """operations/LAPACK/qr.cpp:65-90: dgeqrf, R = upper part of the first
    r_rows rows, Q = dorgqr of the strictly-lower reflectors with q_cols
    columns and k = min(m, n) reflectors."""
    m, n = A.shape
    k = min(m, n)
    q_cols = k if q_cols is None else q_cols
    r_rows = k if r_rows is None else r_rows
    qr, tau, _, info = lapack.dgeqrf(np.asfortranarray(A))
    R = np.zeros((r_rows, n))
    for i in range(min(m, r_rows)):
        R[i, i:] = qr[i, i:]
    Q = np.zeros((m, q_cols))
    for i in range(m):
        c = min(i, n, q_cols)
        Q[i, :c] = qr[i, :c]
    q, _, info = lapack.dorgqr(np.asfortranarray(Q), tau[:min(k, q_cols)])
    return q, R


def rq_dense(A: np.ndarray):
    """operations/LAPACK/rq.cpp:43-70: dgerqf, R (m x min(m,n)) from the upper
    trapezoid, Q (min(m,n) x n) = dorgrq of the reflectors."""
    m, n = A.shape
    k = min(m, n)
    rq, tau, _, info = lapack.dgerqf(np.asfortranarray(A))
    R = np.zeros((m, k))
    for i in range(m):
        j0 = max(i + n - m, 0)
        for j in range(j0, n):
            R[i, j + k - n] = rq[i, j]
    Q = np.zeros((k, n))
    for i in range(max(m - n, 0), m):
        c = i + n - m
        if c > 0:
            Q[i + k - m, :c] = rq[i, :c]
    q, _, info = lapack.dorgrq(np.asfortranarray(Q), tau)
    return R, q


def svd_dense(A: np.ndarray):
    """operations/LAPACK/svd.cpp:23-44: dgesvd('S','S'); S returned as a
    diagonal Dense (here: the vector of singular values)."""
    u, s, vt, info = lapack.dgesvd(np.asfortranarray(A), compute_uv=1, full_matrices=0)
    return u, s, vt


def find_svd_truncation_rank(s: np.ndarray, eps: float) -> int:
    """operations/misc/misc.cpp:133-146, including its quirk: the tail error
    sums S(rank,rank)^2 (min_dim - rank) times rather than S(j,j)^2."""
    threshold = eps * math.sqrt(float((s * s).sum()))
    min_dim = len(s)
    rank = 0
    while True:
        rank += 1
        err = 0.0
        if rank < min_dim:
            v = float(s[rank]) * float(s[rank])
            for _ in range(rank, min_dim):
                err += v
        if not (rank < min_dim and math.sqrt(err) > threshold):
            break
    return rank


def truncated_geqp3(A0: np.ndarray, eps: float):
    """operations/LAPACK/geqp3.cpp:71-192: column-pivoted Householder QR that
    stops when the largest remaining (down-dated) column norm drops to
    eps * ||A||_F. Returns (Q m x r, R r x n with columns permuted back)."""
    A = np.array(A0, dtype=np.float64, copy=True)
    m, n = A.shape
    tol = DLAMCH_E
    tol3z = math.sqrt(tol)
    min_dim = min(m, n)
    tau = np.zeros(min_dim)
    ipiv = list(range(n))
    cnorm = np.array([blas.dnrm2(A[:, j]) for j in range(n)])
    partial = cnorm.copy()
    r = 0
    threshold = eps * math.sqrt(float((A * A).sum()))
    max_c = float(cnorm.max())
    if max_c <= tol:
        Q = np.zeros((m, 1)); Q[0, 0] = 1.0
        return Q, np.zeros((1, n))
    while r < min_dim and max_c > threshold:
        k = r + int(np.argmax(cnorm[r:]))
        A[:, [r, k]] = A[:, [k, r]]
        cnorm[[r, k]] = cnorm[[k, r]]
        partial[[r, k]] = partial[[k, r]]
        ipiv[r], ipiv[k] = ipiv[k], ipiv[r]
        if r < m - 1:
            beta, x, t = lapack.dlarfg(m - r, A[r, r], A[r + 1:, r].copy())
            A[r, r] = beta
            A[r + 1:, r] = x
            tau[r] = t
        else:
            # dlarfg with n = 1 is the identity reflector: tau = 0, beta = alpha
            tau[r] = 0.0
        if r < min_dim - 1:
            arr = A[r, r]
            A[r, r] = 1.0
            v = A[r:, r].copy()
            w = A[r:, r + 1:].T @ v
            A[r:, r + 1:] -= tau[r] * np.outer(v, w)
            A[r, r] = arr
        # LAPACK Working Note 176 norm down-date (geqp3.cpp:137-159),
        # elementwise over the remaining columns.
        js = np.arange(r + 1, n)
        js = js[cnorm[js] != 0.0]
        if len(js):
            temp = np.abs(A[r, js] / cnorm[js])
            temp = np.maximum(0.0, (1 - temp) * (1 + temp))
            ratio = cnorm[js] / partial[js]
            temp2 = temp * ratio * ratio
            keep = temp2 > tol3z
            cnorm[js[keep]] = cnorm[js[keep]] * np.sqrt(temp[keep])
            redo = js[~keep]
            for j in redo:
                if r < m - 1:
                    cnorm[j] = blas.dnrm2(A[r + 1:, j])
                    partial[j] = cnorm[j]
                else:
                    cnorm[j] = 0.0
                    partial[j] = 0.0
        r += 1
        max_c = float(cnorm[r:].max()) if r < n else 0.0
    Qr = np.zeros((m, r))
    for i in range(m):
        c = min(i, r)
        Qr[i, :c] = A[i, :c]
    if r > 0:
        Q, _, info = lapack.dorgqr(np.asfortranarray(Qr), tau[:r])
    else:
        Q = Qr
    R = np.triu(A[:r, :])
    ipivT = np.empty(n, dtype=np.int64)
    ipivT[np.array(ipiv)] = np.arange(n)
    return Q, R[:, ipivT]


def rsvd(A: np.ndarray, sample: int):
    """operations/randomized/rsvd.cpp:17-29: Omega = random_uniform(n, p)
    (the same mt19937(0) matrix on every call), Y = A Omega, Q = qr(Y),
    svd(Q^T A), U = Q Ub. No power iteration."""
    omega = random_uniform(A.shape[1], sample)
    Y = gemm(A, omega)
    Q, _ = qr_dense(Y, q_cols=Y.shape[1], r_rows=Y.shape[1])
    QtA = gemm(Q, A, ta=True)
    Ub, s, V = svd_dense(QtA)
    return gemm(Q, Ub), s, V


# --------------------------------------------------------------------------
# Matrix classes
# --------------------------------------------------------------------------


@dataclass
class LowRank:
    """classes/low_rank.h:37-71: U (m x k), S (k x k), V (k x n), rank, eps."""
    U: np.ndarray
    S: np.ndarray
    V: np.ndarray
    rank: int
    eps: float = 0.0

    @property
    def shape(self):
        return (self.U.shape[0], self.V.shape[1])

    def dense(self) -> np.ndarray:
        """classes/dense.cpp:73-75: gemm(gemm(U, S), V)."""
        return gemm(gemm(self.U, self.S), self.V)

    @staticmethod
    def from_rank(D: np.ndarray, rank: int) -> "LowRank":
        """classes/low_rank.cpp:40-48."""
        m, n = D.shape
        U, s, V = rsvd(D, min(rank + 5, m, n))
        return LowRank(U[:, :rank].copy(), np.diag(s)[:rank, :rank].copy(), V[:rank].copy(), rank)

    @staticmethod
    def from_eps(D: np.ndarray, eps: float) -> "LowRank":
        """classes/low_rank.cpp:50-59: truncated_geqp3, then rq of R so S is
        upper triangular."""
        U, R = truncated_geqp3(D, eps)
        S, V = rq_dense(R)
        return LowRank(U, S, V, U.shape[1], eps)

    def copy(self) -> "LowRank":
        return LowRank(self.U.copy(), self.S.copy(), self.V.copy(), self.rank, self.eps)


@dataclass
class Empty:
    """classes/empty.h:9-27: a placeholder block that only has dimensions."""
    shape: Tuple[int, int]


class Hierarchical:
    """classes/hierarchical.h:43-453: a dim[0] x dim[1] grid of children, each
    an ndarray (Dense), LowRank, Hierarchical or Empty."""

    def __init__(self, nr: int, nc: int):
        self.dim = (nr, nc)
        self.blocks = [[None] * nc for _ in range(nr)]

    def __getitem__(self, ij):
        return self.blocks[ij[0]][ij[1]]

    def __setitem__(self, ij, v):
        self.blocks[ij[0]][ij[1]] = v


def n_rows(M) -> int:
    if isinstance(M, np.ndarray):
        return M.shape[0]
    if isinstance(M, LowRank):
        return M.U.shape[0]
    if isinstance(M, Empty):
        return M.shape[0]
    return sum(n_rows(M[i, 0]) for i in range(M.dim[0]))


def n_cols(M) -> int:
    if isinstance(M, np.ndarray):
        return M.shape[1]
    if isinstance(M, LowRank):
        return M.V.shape[1]
    if isinstance(M, Empty):
        return M.shape[1]
    return sum(n_cols(M[0, j]) for j in range(M.dim[1]))


def build_hierarchical(kernel, x: Points, n: int, nleaf: int, nb: int,
                       rank: int = 0, eps: float = 0.0, admis: float = 0.0,
                       admis_type: int = POSITION_BASED,
                       rows=None, cols=None, abs_pos=(0, 0), is_root=True):
    """classes/hierarchical.cpp:49-109 with cluster_tree.cpp:14-45,75-82 and
    matrix_initializer.cpp:28-42: each child is LowRank if admissible
    (fixed rank when rank > 0, else fixed accuracy eps), Dense if a leaf,
    else recursed with the same nb x nb split."""
    rows = (0, n) if rows is None else rows
    cols = (0, n) if cols is None else cols
    H = Hierarchical(nb, nb)
    rs = split_range(rows[0], rows[1], nb)
    cs = split_range(cols[0], cols[1], nb)
    for i in range(nb):
        for j in range(nb):
            r, c = rs[i], cs[j]
            ap = (abs_pos[0] * nb + i, abs_pos[1] * nb + j)
            leaf = (r[1] <= nleaf and c[1] <= nleaf) or nleaf == 0
            if is_admissible(r, c, ap, admis, admis_type, x):
                D = kernel(x, r[0], r[1], c[0], c[1])
                H[i, j] = LowRank.from_rank(D, rank) if rank > 0 else LowRank.from_eps(D, eps)
            elif leaf:
                H[i, j] = kernel(x, r[0], r[1], c[0], c[1])
            else:
                H[i, j] = build_hierarchical(kernel, x, n, nleaf, nb, rank, eps, admis,
                                             admis_type, r, c, ap, False)
    return H


def to_dense(M) -> np.ndarray:
    if isinstance(M, np.ndarray):
        return M.copy()
    if isinstance(M, LowRank):
        return M.dense()
    if isinstance(M, Empty):
        return np.zeros(M.shape)
    return np.block([[to_dense(M[i, j]) for j in range(M.dim[1])] for i in range(M.dim[0])])


def deep_copy(M):
    if isinstance(M, np.ndarray):
        return M.copy()
    if isinstance(M, LowRank):
        return M.copy()
    H = Hierarchical(*M.dim)
    for i in range(M.dim[0]):
        for j in range(M.dim[1]):
            H[i, j] = deep_copy(M[i, j])
    return H


def split_rows(b: np.ndarray, like_rows: Sequence[int]) -> List[np.ndarray]:
    out, s = [], 0
    for n in like_rows:
        out.append(b[s:s + n])
        s += n
    return out


def split_lowrank(A: LowRank, rs, cs) -> Hierarchical:
    """operations/misc/misc.cpp:199-236: split U by rows and V by columns,
    S shared."""
    H = Hierarchical(len(rs), len(cs))
    for i, (r0, rn) in enumerate(rs):
        for j, (c0, cn) in enumerate(cs):
            H[i, j] = LowRank(A.U[r0:r0 + rn], A.S, A.V[:, c0:c0 + cn], A.S.shape[0], A.eps)
    return H


def _child_ranges(H: Hierarchical):
    rs, s = [], 0
    for i in range(H.dim[0]):
        n = n_rows(H[i, 0]); rs.append((s, n)); s += n
    cs, s = [], 0
    for j in range(H.dim[1]):
        n = n_cols(H[0, j]); cs.append((s, n)); s += n
    return rs, cs


# --------------------------------------------------------------------------
# LowRank addition (recompression)
# --------------------------------------------------------------------------

LRA_MODE = {"mode": "rounded_addition"}  # FRANK_LRA (global_key_value.cpp:10-22)


def rounded_addition(A: LowRank, B: LowRank) -> None:
    """operations/arithmetic/addition.cpp:93-127 (Bebendorf p.16)."""
    ka, kb = A.S.shape[1], B.S.shape[1]
    m = A.U.shape[0]
    Uc = np.zeros((m, ka + kb))
    Uc[:, :ka] = gemm(A.U, A.S)
    Uc[:, ka:] = gemm(B.U, B.S)
    s = min(Uc.shape)
    Qu, Ru = qr_dense(Uc, q_cols=s, r_rows=s)
    VcT = np.vstack([A.V, B.V])
    RvT, QvT = rq_dense(VcT)
    M = gemm(Ru, RvT)
    RRU, RRS, RRV = svd_dense(M)
    if A.eps != 0:
        A.rank = find_svd_truncation_rank(RRS, A.eps)
    r = A.rank
    A.S = np.diag(RRS)[:r, :r].copy()
    A.U = gemm(Qu, RRU[:, :r])
    A.V = gemm(RRV[:r, :], QvT)


def rounded_addition_rrqr(A: LowRank, B: LowRank) -> None:
    """Variant used by this engine's GPU path (NOT a reference algorithm):
    identical stacking to rounded_addition, but the core M = Ru RvT is
    truncated with the reference's own fixed-accuracy compressor
    (truncated_geqp3 + rq, low_rank.cpp:50-59) instead of dgesvd +
    find_svd_truncation_rank.  Used only to bound the deviation in tests."""
    if A.eps == 0:
        rounded_addition(A, B)
        return
    ka, kb = A.S.shape[1], B.S.shape[1]
    m = A.U.shape[0]
    Uc = np.zeros((m, ka + kb))
    Uc[:, :ka] = gemm(A.U, A.S)
    Uc[:, ka:] = gemm(B.U, B.S)
    s = min(Uc.shape)
    Qu, Ru = qr_dense(Uc, q_cols=s, r_rows=s)
    VcT = np.vstack([A.V, B.V])
    RvT, QvT = rq_dense(VcT)
    M = gemm(Ru, RvT)
    Qm, Rm = truncated_geqp3(M, A.eps)
    Sm, Vm = rq_dense(Rm)
    A.rank = Qm.shape[1]
    A.S = Sm
    A.U = gemm(Qu, Qm)
    A.V = gemm(Vm, QvT)


def fast_rounded_addition(A: LowRank, B: LowRank) -> None:
    """operations/arithmetic/addition.cpp:133-189 (Bebendorf p.17); falls back
    to rounded_addition for fixed accuracy."""
    if A.eps != 0.0:
        rounded_addition(A, B)
        return
    Zu = gemm(A.U, B.U, ta=True)
    Yu = B.U - gemm(A.U, Zu)
    Qu, Ru = qr_dense(Yu, q_cols=min(Yu.shape), r_rows=min(Yu.shape))
    Uc = np.hstack([A.U, Qu])
    ZvT = gemm(B.V, A.V, tb=True)
    YvT = B.V - gemm(ZvT, A.V)
    RvT, QvT = rq_dense(YvT)
    VcT = np.vstack([A.V, QvT])
    ka0, kb0 = A.S.shape[0], B.S.shape[0]
    ka1, kb1 = A.S.shape[1], B.S.shape[1]
    M = np.zeros((ka0 + Ru.shape[0], ka1 + RvT.shape[1]))
    ZuSb = gemm(Zu, B.S)
    RuSb = gemm(Ru, B.S)
    M[:ka0, :ka1] = A.S + gemm(ZuSb, ZvT)
    M[:ka0, ka1:] = gemm(ZuSb, RvT)
    M[ka0:, :ka1] = gemm(RuSb, ZvT)
    M[ka0:, ka1:] = gemm(RuSb, RvT)
    Um, Sm, VmT = svd_dense(M)
    r = A.rank
    A.S = np.diag(Sm)[:r, :r].copy()
    A.U = gemm(Uc, Um[:, :r])
    A.V = gemm(VmT[:r, :], VcT)


def naive_addition(A: LowRank, B: LowRank) -> None:
    """operations/arithmetic/addition.cpp:68-89."""
    m, n = A.shape
    if A.rank + B.rank >= min(m, n):
        N = LowRank.from_rank(A.dense() + B.dense(), A.rank)
        A.U, A.S, A.V = N.U, N.S, N.V
    else:
        S = np.zeros((A.rank + B.rank, A.rank + B.rank))
        S[:A.rank, :A.rank] = A.S
        S[A.rank:, A.rank:] = B.S
        A.U = np.hstack([A.U, B.U])
        A.V = np.vstack([A.V, B.V])
        A.S = S
        A.rank += B.rank


def lr_add(A: LowRank, B: LowRank) -> None:
    """operations/arithmetic/addition.cpp:191-203: algorithm by FRANK_LRA."""
    mode = LRA_MODE["mode"]
    if mode == "naive":
        naive_addition(A, B)
    elif mode == "rounded_addition_rrqr":
        rounded_addition_rrqr(A, B)
    elif mode == "rounded_addition":
        rounded_addition(A, B)
    else:
        fast_rounded_addition(A, B)


def add_into(C, B):
    """`C += B` (addition.cpp:39-66, 191-203); returns the (possibly new) C."""
    if isinstance(C, np.ndarray):
        if isinstance(B, np.ndarray):
            C += B
        elif isinstance(B, LowRank):
            C += gemm(gemm(B.U, B.S), B.V)          # addition.cpp:48-51
        else:
            C += to_dense(B)
        return C
    if isinstance(C, LowRank):
        if isinstance(B, LowRank):
            lr_add(C, B)
            return C
        raise TypeError("operator+= (LowRank, %s) unsupported" % type(B).__name__)
    # Hierarchical
    if isinstance(B, LowRank):
        rs, cs = _child_ranges(C)
        B = split_lowrank(B, rs, cs)                # addition.cpp:62-66
    for i in range(C.dim[0]):
        for j in range(C.dim[1]):
            C[i, j] = add_into(C[i, j], B[i, j])
    return C


# --------------------------------------------------------------------------
# gemm multimethod (the type triples the LU path reaches)
# --------------------------------------------------------------------------


def gemm_into(A, B, C, alpha: float, beta: float):
    """C = alpha * A * B + beta * C over Dense / LowRank / Hierarchical,
    no transposes (operations/BLAS/gemm.cpp). Returns the (possibly new) C."""
    dA, dB, dC = (isinstance(A, np.ndarray), isinstance(B, np.ndarray), isinstance(C, np.ndarray))
    lA, lB, lC = (isinstance(A, LowRank), isinstance(B, LowRank), isinstance(C, LowRank))
    hA, hB, hC = (isinstance(A, Hierarchical), isinstance(B, Hierarchical), isinstance(C, Hierarchical))
    if dA and dB and dC:                       # gemm.cpp:126-146
        C[...] = blas.dgemm(alpha, np.asfortranarray(A), np.asfortranarray(B), beta,
                            np.asfortranarray(C))
        return C
    if lA and dB and dC:                       # gemm.cpp:148-162
        t = gemm(A.S, gemm(A.V, B, alpha))
        C[...] = blas.dgemm(1.0, np.asfortranarray(A.U), np.asfortranarray(t), beta,
                            np.asfortranarray(C))
        return C
    if dA and lB and dC:                       # gemm.cpp:164-178
        t = gemm(gemm(A, B.U, alpha), B.S)
        C[...] = blas.dgemm(1.0, np.asfortranarray(t), np.asfortranarray(B.V), beta,
                            np.asfortranarray(C))
        return C
    if lA and lB and dC:                       # gemm.cpp:180-200
        inner = gemm(A.U, gemm(gemm(A.S, gemm(A.V, B.U, alpha)), B.S))
        C[...] = blas.dgemm(1.0, np.asfortranarray(inner), np.asfortranarray(B.V), beta,
                            np.asfortranarray(C))
        return C
    if lA and lB and (lC or hC):               # gemm.cpp:253-272, 374-393
        S = gemm(gemm(A.S, A.V), gemm(B.U, B.S), alpha)
        AxB = LowRank(A.U, S, B.V, S.shape[0])
        C = scale(C, beta)
        return add_into(C, AxB)
    if lA and dB and (lC or hC):               # gemm.cpp:219-234, 344-357
        AxB = LowRank(A.U, A.S, gemm(A.V, B, alpha), A.S.shape[0])
        C = scale(C, beta)
        return add_into(C, AxB)
    if dA and lB and (lC or hC):               # gemm.cpp:236-251, 330-342
        AxB = LowRank(gemm(A, B.U, alpha), B.S, B.V, B.S.shape[0])
        C = scale(C, beta)
        return add_into(C, AxB)
    if dA and dB and lC:                       # gemm.cpp:202-217
        C = scale(C, beta)
        P = gemm(A, B, alpha)
        N = LowRank.from_eps(P, C.eps) if C.eps != 0.0 else LowRank.from_rank(P, C.rank)
        return add_into(C, N)
    if hA and hB and hC:                       # gemm.cpp:431-449
        for i in range(C.dim[0]):
            for j in range(C.dim[1]):
                for k in range(A.dim[1]):
                    C[i, j] = gemm_into(A[i, k], B[k, j], C[i, j], alpha, beta if k == 0 else 1.0)
        return C
    if hA and dC and (dB or lB):               # gemm.cpp:581-615 (H x dense -> dense)
        if dB:
            rs, cs = _child_ranges(A)
            Bs = [B[c0:c0 + cn] for (c0, cn) in cs]
            if beta != 1.0:
                C *= beta
            for i, (r0, rn) in enumerate(rs):
                Ci = C[r0:r0 + rn]
                for k in range(A.dim[1]):
                    Ci = gemm_into(A[i, k], Bs[k], Ci, alpha, 1.0)
                C[r0:r0 + rn] = Ci
            return C
    if hA and (dB or lB) and hC:               # gemm.cpp:498-523 H D H / H LR H
        rs, cs = _child_ranges(A)
        _, ccs = _child_ranges(C)
        if dB:
            Bh = Hierarchical(A.dim[1], C.dim[1])
            for k, (r0, rn) in enumerate(cs):
                for j, (c0, cn) in enumerate(ccs):
                    Bh[k, j] = B[r0:r0 + rn, c0:c0 + cn]
        else:
            Bh = split_lowrank(B, cs, ccs)
        return gemm_into(A, Bh, C, alpha, beta)
    if (dA or lA) and hB and hC:               # gemm.cpp:472-496 D H H / LR H H
        rs, cs = _child_ranges(B)
        crs, _ = _child_ranges(C)
        if dA:
            Ah = Hierarchical(C.dim[0], B.dim[0])
            for i, (r0, rn) in enumerate(crs):
                for k, (c0, cn) in enumerate(rs):
                    Ah[i, k] = A[r0:r0 + rn, c0:c0 + cn]
        else:
            Ah = split_lowrank(A, crs, rs)
        return gemm_into(Ah, B, C, alpha, beta)
    if (dA or lA) and hB and dC:               # gemm.cpp:545-579 D H D / LR H D
        return gemm_into(A, to_dense(B), C, alpha, beta)
    if hA and hB and dC:                       # gemm.cpp:525-543
        return gemm_into(to_dense(A), to_dense(B), C, alpha, beta)
    if hA and lB and lC:                       # gemm.cpp:274-289 H LR LR
        AxB = LowRank(gemm_into(A, B.U, np.zeros((n_rows(A), B.U.shape[1])), alpha, 0.0),
                      B.S, B.V, B.S.shape[0])
        C = scale(C, beta)
        return add_into(C, AxB)
    if lA and hB and lC:                       # gemm.cpp:317-328 LR H LR
        VB = gemm(A.V, to_dense(B), alpha)
        AxB = LowRank(A.U, A.S, VB, A.S.shape[0])
        C = scale(C, beta)
        return add_into(C, AxB)
    raise TypeError("gemm(%s, %s, %s) unsupported" % tuple(type(t).__name__ for t in (A, B, C)))


def scale(C, beta: float):
    """operations/arithmetic/multiplication.cpp:30-52: LowRank scales S only."""
    if beta == 1.0:
        return C
    if isinstance(C, np.ndarray):
        C *= beta
    elif isinstance(C, LowRank):
        C.S = C.S * beta
    else:
        for i in range(C.dim[0]):
            for j in range(C.dim[1]):
                C[i, j] = scale(C[i, j], beta)
    return C


# --------------------------------------------------------------------------
# trsm multimethod
# --------------------------------------------------------------------------


def trsm(A, B, upper: bool, left: bool = True):
    """operations/BLAS/trsm.cpp:32-125. Returns the (in-place updated) B."""
    if isinstance(A, np.ndarray) and isinstance(B, np.ndarray):
        B[...] = trsm_dense(A, B, upper, left)
        return B
    if isinstance(B, LowRank):                  # trsm.cpp:106-115
        if left:
            B.U = trsm(A, B.U, upper, True)
        else:
            B.V = trsm(A, B.V, upper, False)
        return B
    if isinstance(A, Hierarchical) and isinstance(B, np.ndarray):   # trsm.cpp:117-125
        rs, cs = _child_ranges(A)
        if left:
            Bh = Hierarchical(A.dim[0], 1)
            for i, (r0, rn) in enumerate(rs):
                Bh[i, 0] = B[r0:r0 + rn]
        else:
            Bh = Hierarchical(1, A.dim[1])
            for j, (c0, cn) in enumerate(cs):
                Bh[0, j] = B[:, c0:c0 + cn]
        trsm(A, Bh, upper, left)
        return B
    if isinstance(A, Hierarchical) and isinstance(B, Hierarchical):  # trsm.cpp:40-90
        if upper and left:
            if B.dim[1] != 1:
                raise TypeError("Left upper with B.dim[1] != 1 trsm")
            for i in range(B.dim[0] - 1, -1, -1):
                for j in range(B.dim[0] - 1, i, -1):
                    B[i, 0] = gemm_into(A[i, j], B[j, 0], B[i, 0], -1.0, 1.0)
                B[i, 0] = trsm(A[i, i], B[i, 0], True, True)
        elif upper and not left:
            for i in range(B.dim[0]):
                for j in range(B.dim[1]):
                    for k in range(j):
                        B[i, j] = gemm_into(B[i, k], A[k, j], B[i, j], -1.0, 1.0)
                    B[i, j] = trsm(A[j, j], B[i, j], True, False)
        elif not upper and left:
            for j in range(B.dim[1]):
                for i in range(B.dim[0]):
                    for k in range(i):
                        B[i, j] = gemm_into(A[i, k], B[k, j], B[i, j], -1.0, 1.0)
                    B[i, j] = trsm(A[i, i], B[i, j], False, True)
        else:
            raise TypeError("Right lower trsm")
        return B
    raise TypeError("trsm(%s, %s) unsupported" % (type(A).__name__, type(B).__name__))


# --------------------------------------------------------------------------
# getrf multimethod, solve, matvec, errors
# --------------------------------------------------------------------------


def getrf(A, piv_log: Optional[list] = None):
    """operations/LAPACK/getrf.cpp:45-84: right-looking block LU. Consumes A;
    returns (L, U). `piv_log` collects whether each leaf dgetrf swapped rows."""
    if isinstance(A, np.ndarray):
        L, U, piv, info = getrf_dense(A, return_piv=True)
        if piv_log is not None:
            piv_log.append(bool(np.all(piv == np.arange(len(piv)))))
        return L, U
    L = Hierarchical(*A.dim)
    for i in range(A.dim[0]):
        L[i, i], A[i, i] = getrf(A[i, i], piv_log)
        for ic in range(i + 1, L.dim[0]):
            L[ic, i] = A[ic, i]
            A[ic, i] = Empty((n_rows(L[ic, i]), n_cols(L[ic, i])))
            L[ic, i] = trsm(A[i, i], L[ic, i], upper=True, left=False)
        for j in range(i + 1, A.dim[1]):
            L[i, j] = Empty((n_rows(A[i, j]), n_cols(A[i, j])))
            A[i, j] = trsm(L[i, i], A[i, j], upper=False, left=True)
        for ic in range(i + 1, L.dim[0]):
            for k in range(i + 1, A.dim[1]):
                A[ic, k] = gemm_into(L[ic, i], A[i, k], A[ic, k], -1.0, 1.0)
    return L, A


def solve(L, U, b: np.ndarray) -> np.ndarray:
    """examples/h_lu.cpp:45-48: trsm(L, b, Lower) then trsm(U, b, Upper)."""
    x = np.array(b, dtype=np.float64, copy=True)
    if x.ndim == 1:
        x = x[:, None]
    trsm(L, x, upper=False, left=True)
    trsm(U, x, upper=True, left=True)
    return x


def matvec(A, x: np.ndarray) -> np.ndarray:
    """gemm(A, x, b, 1, 1) with b = 0 (gemm.cpp:581-615 -> leaves): the
    H-matrix times a dense block of vectors."""
    xx = x if x.ndim == 2 else x[:, None]
    b = np.zeros((n_rows(A), xx.shape[1]))
    return gemm_into(A, np.ascontiguousarray(xx), b, 1.0, 1.0)


def norm2(M) -> float:
    """operations/misc/norm.cpp:24-44: the SQUARED Frobenius norm."""
    if isinstance(M, np.ndarray):
        return float((M * M).sum())
    if isinstance(M, LowRank):
        d = M.dense()
        return float((d * d).sum())
    return sum(norm2(M[i, j]) for i in range(M.dim[0]) for j in range(M.dim[1]))


def l2_error(A, B) -> float:
    """util/l2_error.cpp:35-41: sqrt(||A-B||^2 / (||A||^2 + DBL_EPSILON))."""
    a = to_dense(A)
    b = to_dense(B)
    return math.sqrt(float(((a - b) ** 2).sum()) / (float((a * a).sum()) + np.finfo(float).eps))


def lu_factor_error(A_dense: np.ndarray, L, U) -> float:
    """||A - L U||_F / ||A||_F (dense, small sizes)."""
    LU = to_dense(L) @ to_dense(U)
    return float(np.linalg.norm(A_dense - LU) / np.linalg.norm(A_dense))


def blr_ranks(H) -> List[Tuple[int, int, int]]:
    out = []
    for i in range(H.dim[0]):
        for j in range(H.dim[1]):
            if isinstance(H[i, j], LowRank):
                out.append((i, j, H[i, j].rank))
    return out


# --------------------------------------------------------------------------
# Interpolative decompositions (operations/LAPACK/id.cpp, randomized/rid.cpp)
# --------------------------------------------------------------------------


def geqp3(A: np.ndarray):
    """operations/LAPACK/geqp3.cpp:36-69: LAPACKE_dgeqp3 with jpvt = 0 (all
    columns free); returns R (the upper triangle of the factored matrix,
    n x n) and the 0-based column order."""
    m, n = A.shape
    # scipy's wrapper starts from jpvt = 0 (every column free), as the reference does
    qr_, jpvt, tau, work, info = lapack.dgeqp3(np.asfortranarray(A.copy()))
    R = np.zeros((n, n))
    k = min(m, n)
    R[:k, :] = np.triu(qr_[:k, :])
    return R, [int(j) - 1 for j in jpvt]


def one_sided_id(A: np.ndarray, k: int):
    """operations/LAPACK/id.cpp:49-73: V (k x n) with A ~= A[:, cols] V."""
    m, n = A.shape
    R, P = geqp3(A)
    if k < min(m, n) or n > m:
        T = trsm_dense(R[:k, :k], R[:k, k:], upper=True, left=True)
    else:
        T = np.zeros((k, 0))
    V = np.zeros((k, n))
    for j in range(n):                                   # interleave_id (id.cpp:29-39)
        V[:, P[j]] = np.eye(k)[:, j] if j < k else T[:, j - k]
    return V, P[:k]


def id_(A: np.ndarray, k: int):
    """operations/LAPACK/id.cpp:100-111: A ~= U S V with S = A[rows, cols]."""
    V, cols = one_sided_id(A.copy(), k)
    AC = A[:, cols]
    Ut, rows = one_sided_id(AC.T.copy(), k)
    return Ut.T.copy(), AC[rows, :].copy(), V, rows, cols


def rid(A: np.ndarray, sample: int, k: int):
    """operations/randomized/rid.cpp:18-31 with the reference's Omega."""
    m, n = A.shape
    RN = random_uniform(n, sample)
    Y = gemm(A, RN)
    Q, _ = qr_dense(Y)
    U, S, V, _, _ = id_(gemm(Q, A, 1.0, True, False), k)
    return gemm(Q, U), S, V
