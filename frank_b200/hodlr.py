"""Host mirror of FRANK's multi-level H-LU calls over the C ABI.

`HMatrix` is one H-matrix with a binary cluster tree and weak admissibility
(every off-diagonal child LowRank of a fixed rank, diagonal children recursed
down to dense leaves) resident on the current GPU (a `frank_hodlr`):

=========================================  ==========================================
FRANK (C++)                                here
=========================================  ==========================================
Hierarchical(kernel, x, n, n, rank,        HMatrix(n, leaf, rank).build_kernel(...)
  nleaf, 0, 2, 2)                          (or set_dense / set_lowrank per block)
std::tie(L, U) = getrf(A)                  A.getrf()
trsm(L, b, Lower); trsm(U, b, Upper)       A.solve(b)
gemm(A, x, b, 1, 0)                        A.matvec(x)
=========================================  ==========================================

Block (level l, index c) spans the rows of cluster c of level l and the
columns of its sibling c ^ 1.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import numpy as np

from ._abi import check, lib
from .blr import KERNELS, _dptr


class _DeviceBuffer:
    def __init__(self, count: int):
        self.ptr = C.c_void_p()
        check(lib().frank_device_alloc(C.c_size_t(8 * max(1, count)), C.byref(self.ptr)), "frank_device_alloc")

    def __del__(self):
        if self.ptr:
            lib().frank_device_free(self.ptr)
            self.ptr = C.c_void_p()

    def put(self, a: np.ndarray):
        check(lib().frank_copy(self.ptr, a.ctypes.data_as(C.c_void_p), C.c_size_t(a.nbytes), 1), "frank_copy")

    def get(self, a: np.ndarray):
        check(lib().frank_copy(a.ctypes.data_as(C.c_void_p), self.ptr, C.c_size_t(a.nbytes), 0), "frank_copy")


class HMatrix:
    """An n x n H-matrix on the GPU: leaves of order `leaf`, n / leaf a power
    of two, every off-diagonal block of every level LowRank of rank `rank`."""

    def __init__(self, n: int, leaf: int, rank: int, lra: str = "fast_rounded_addition"):
        self._h = C.c_void_p()
        check(lib().frank_hodlr_create(int(n), int(leaf), int(rank), C.byref(self._h)), "frank_hodlr_create")
        nn, lf, rk, lv = C.c_int64(), C.c_int(), C.c_int(), C.c_int()
        check(lib().frank_hodlr_shape(self._h, C.byref(nn), C.byref(lf), C.byref(rk), C.byref(lv)),
              "frank_hodlr_shape")
        self.n, self.leaf, self.rank, self.levels = nn.value, lf.value, rk.value, lv.value
        self.set_lra(lra)

    def close(self):
        if self._h:
            lib().frank_hodlr_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def block_size(self, level: int) -> int:
        return self.n >> level

    def set_lra(self, name: str):
        """fast_rounded_addition (the reference's default) or rounded_addition."""
        check(lib().frank_hodlr_set_lra(self._h, name.encode()), "frank_hodlr_set_lra")

    def build_kernel(self, kernel: str, points: np.ndarray, kparams: Optional[Tuple[float, float]] = None):
        x = np.ascontiguousarray(points, dtype=np.float64)
        if x.ndim == 1:
            x = x[None, :]
        kp = np.array(kparams if kparams is not None else (0.0, 0.0), dtype=np.float64)
        check(lib().frank_hodlr_build_kernel(self._h, KERNELS[kernel], _dptr(x), x.shape[0], _dptr(kp), None),
              "frank_hodlr_build_kernel")

    def set_dense(self, leaf: int, a: np.ndarray):
        aa = np.asfortranarray(a, dtype=np.float64)
        check(lib().frank_hodlr_set_dense(self._h, int(leaf), _dptr(aa), aa.shape[0]), "frank_hodlr_set_dense")

    def set_lowrank(self, level: int, index: int, U: np.ndarray, S: np.ndarray, V: np.ndarray):
        u, s, v = (np.asfortranarray(t, dtype=np.float64) for t in (U, S, V))
        check(lib().frank_hodlr_set_lowrank(self._h, int(level), int(index), _dptr(u), _dptr(s), _dptr(v)),
              "frank_hodlr_set_lowrank")

    def get_dense(self, leaf: int, factor: bool = False) -> np.ndarray:
        a = np.zeros((self.leaf, self.leaf), order="F")
        check(lib().frank_hodlr_get_dense(self._h, int(factor), int(leaf), _dptr(a), self.leaf),
              "frank_hodlr_get_dense")
        return a

    def get_lowrank(self, level: int, index: int, factor: bool = False):
        s = self.block_size(level)
        U = np.zeros((s, self.rank), order="F")
        S = np.zeros((self.rank, self.rank), order="F")
        V = np.zeros((self.rank, s), order="F")
        check(lib().frank_hodlr_get_lowrank(self._h, int(factor), int(level), int(index), _dptr(U), _dptr(S),
                                            _dptr(V)), "frank_hodlr_get_lowrank")
        return U, S, V

    def get_pivots(self, leaf: int) -> np.ndarray:
        """0-based pivots of leaf `leaf`'s getrf."""
        p = np.zeros(self.leaf, dtype=np.int32)
        check(lib().frank_hodlr_get_pivots(self._h, int(leaf), p.ctypes.data_as(C.POINTER(C.c_int))),
              "frank_hodlr_get_pivots")
        return p

    def getrf(self, stream: Optional[int] = None):
        check(lib().frank_hodlr_getrf(self._h, stream), "frank_hodlr_getrf")

    def stats(self) -> dict:
        la, ms = C.c_int64(), C.c_double()
        check(lib().frank_hodlr_stats(self._h, C.byref(la), C.byref(ms)), "frank_hodlr_stats")
        return {"launches": la.value, "factor_ms": ms.value}

    # host arrays (n x nrhs), through a device buffer
    def solve(self, b: np.ndarray) -> np.ndarray:
        bb = np.array(np.asarray(b, dtype=np.float64).reshape(self.n, -1), order="F", copy=True)
        d = _DeviceBuffer(bb.size)
        d.put(bb)
        check(lib().frank_hodlr_solve_device(self._h, d.ptr, self.n, bb.shape[1], None), "frank_hodlr_solve_device")
        d.get(bb)
        return bb if np.ndim(b) == 2 else bb[:, 0]

    def trsm(self, b: np.ndarray, lower: bool) -> np.ndarray:
        """trsm(L, b, Lower) (lower=True: b <- L^{-1} P b) or trsm(U, b, Upper)."""
        bb = np.array(np.asarray(b, dtype=np.float64).reshape(self.n, -1), order="F", copy=True)
        d = _DeviceBuffer(bb.size)
        d.put(bb)
        check(lib().frank_hodlr_trsm_device(self._h, 0 if lower else 1, d.ptr, self.n, bb.shape[1], None),
              "frank_hodlr_trsm_device")
        d.get(bb)
        return bb if np.ndim(b) == 2 else bb[:, 0]

    def matvec(self, x: np.ndarray) -> np.ndarray:
        xx = np.asfortranarray(np.asarray(x, dtype=np.float64).reshape(self.n, -1))
        dx, dy = _DeviceBuffer(xx.size), _DeviceBuffer(xx.size)
        dx.put(xx)
        check(lib().frank_hodlr_matvec_device(self._h, dx.ptr, self.n, dy.ptr, self.n, xx.shape[1], None),
              "frank_hodlr_matvec_device")
        y = np.zeros_like(xx, order="F")
        dy.get(y)
        return y if np.ndim(x) == 2 else y[:, 0]

    def refine(self, b: np.ndarray, tol: float = 1e-10, maxit: int = 50) -> Tuple[np.ndarray, int, float]:
        bb = np.asfortranarray(np.asarray(b, dtype=np.float64).reshape(self.n, -1))
        db, dx = _DeviceBuffer(bb.size), _DeviceBuffer(bb.size)
        db.put(bb)
        it, res = C.c_int(), C.c_double()
        check(lib().frank_hodlr_refine_device(self._h, db.ptr, self.n, dx.ptr, self.n, bb.shape[1], float(tol),
                                              int(maxit), C.byref(it), C.byref(res), None),
              "frank_hodlr_refine_device")
        x = np.zeros_like(bb, order="F")
        dx.get(x)
        return x, it.value, res.value

    # device pointers (e.g. torch tensors' data_ptr(), column-major n x nrhs)
    def solve_device(self, ptr: int, nrhs: int, ld: Optional[int] = None, stream: Optional[int] = None):
        check(lib().frank_hodlr_solve_device(self._h, C.c_void_p(ptr), ld or self.n, nrhs, stream),
              "frank_hodlr_solve_device")

    def matvec_device(self, xptr: int, yptr: int, nrhs: int, stream: Optional[int] = None):
        check(lib().frank_hodlr_matvec_device(self._h, C.c_void_p(xptr), self.n, C.c_void_p(yptr), self.n, nrhs,
                                              stream), "frank_hodlr_matvec_device")

    def refine_device(self, bptr: int, xptr: int, nrhs: int, tol: float = 1e-10, maxit: int = 50,
                      stream: Optional[int] = None) -> Tuple[int, float]:
        it, res = C.c_int(), C.c_double()
        check(lib().frank_hodlr_refine_device(self._h, C.c_void_p(bptr), self.n, C.c_void_p(xptr), self.n, nrhs,
                                              float(tol), int(maxit), C.byref(it), C.byref(res), stream),
              "frank_hodlr_refine_device")
        return it.value, res.value


def upload_hmatrix(H, n: int, leaf: int, rank: int, lra: str = "fast_rounded_addition") -> HMatrix:
    """An HMatrix holding the blocks of a nested Hierarchical `H` (nb = 2 at
    every level, LowRank off-diagonal children with attributes U, S, V, dense
    leaves as 2-D arrays), e.g. one built on the host."""
    M = HMatrix(n, leaf, rank, lra)

    def walk(node, level: int, index: int):
        for i in range(2):
            for j in range(2):
                child = node[i, j]
                if i == j:
                    ci = 2 * index + i
                    if isinstance(child, np.ndarray):
                        M.set_dense(ci, child)
                    else:
                        walk(child, level + 1, ci)
                else:
                    M.set_lowrank(level + 1, 2 * index + i, child.U, child.S, child.V)

    walk(H, 0, 0)
    return M
