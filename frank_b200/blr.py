"""Host mirror of FRANK's BLR factor-and-solve calls over the C ABI.

`BLRMatrix` is one block-low-rank matrix resident on the current GPU (a
`frank_blr` plan).  Its methods mirror the reference calls of the path:

=====================================  =============================================
FRANK (C++)                            here
=====================================  =============================================
Hierarchical(kernel, x, n, n, nleaf,   BLRMatrix(n, nb, ...).build_kernel(...)
  eps, admis, nb, nb)                  (or set_dense / set_lowrank per block)
std::tie(L, U) = getrf(A)              A.getrf()       (factors in place)
trsm(L, b, Lower); trsm(U, b, Upper)   A.solve(b)
gemm(A, x, b, 1, 0)                    A.matvec(x)
l2_error(x, b)                         numpy on the host
=====================================  =============================================

Errors are raised as `FrankError` carrying the C ABI status; there is no CPU
fallback: every call runs the sm_100a kernels of libfrank_b200.so.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence, Tuple

import numpy as np

from . import _abi
from ._abi import FrankError, check, lib

KERNELS = {"laplace": _abi.FRANK_KERNEL_LAPLACE, "helmholtz": _abi.FRANK_KERNEL_HELMHOLTZ,
           "neglog": _abi.FRANK_KERNEL_NEGLOG, "exp": _abi.FRANK_KERNEL_EXP}


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def split_offsets(n: int, nb: int) -> np.ndarray:
    """IndexRange::split (classes/initialization_helpers/index_range.cpp:15-24)."""
    child = (n + nb - 1) // nb
    off = [child * i for i in range(nb)] + [n]
    return np.array(off, dtype=np.int64)


class BLRMatrix:
    """A BLR matrix on the GPU: diagonal blocks dense, block (i, j) low rank iff
    |i - j| > admis (position-based admissibility, matrix_initializer.cpp:51-58)."""

    def __init__(self, n: int, nb: int, *, eps: float = 0.0, fixed_rank: int = 0, max_rank: int = 0,
                 precision: str = "fp64", admis: float = 0.0, admis_type: str = "position",
                 points: Optional[np.ndarray] = None):
        """admis_type "position": block (i, j) low rank iff |i - j| > admis;
        "geometry": from the bounding boxes of `points` (dim x n), as
        AdmisType::GeometryBased (matrix_initializer.cpp:51-91)."""
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        if admis_type not in ("position", "geometry"):
            raise ValueError("admis_type must be 'position' or 'geometry'")
        self.n, self.nb = int(n), int(nb)
        self.precision = precision
        d = _abi.BlrDesc(n=self.n, nb=self.nb, max_rank=int(max_rank),
                         precision=_abi.FRANK_PREC_FP64 if precision == "fp64" else _abi.FRANK_PREC_MIXED,
                         fixed_rank=int(fixed_rank), eps=float(eps), admis=float(admis))
        h = C.c_void_p()
        if admis_type == "geometry":
            if points is None:
                raise ValueError("geometry-based admissibility needs points")
            x = np.ascontiguousarray(np.atleast_2d(points), dtype=np.float64)
            check(lib().frank_blr_create_geometric(C.byref(d), _dptr(x), x.shape[0], C.byref(h)),
                  "frank_blr_create_geometric")
        else:
            check(lib().frank_blr_create(C.byref(d), C.byref(h)), "frank_blr_create")
        self._h = h
        off = np.zeros(self.nb + 1, dtype=np.int64)
        check(lib().frank_blr_offsets(self._h, off.ctypes.data_as(C.POINTER(C.c_int64))), "frank_blr_offsets")
        self.offsets = off
        self.admis = float(admis)

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            lib().frank_blr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- geometry ---------------------------------------------------------
    def block_size(self, i: int) -> int:
        return int(self.offsets[i + 1] - self.offsets[i])

    def is_lowrank(self, i: int, j: int) -> bool:
        t = C.c_int()
        check(lib().frank_blr_block_info(self._h, 0, i, j, C.byref(t), None), "frank_blr_block_info")
        return t.value == _abi.FRANK_BLOCK_LOWRANK

    def rank(self, i: int, j: int, which: int = 0) -> int:
        r = C.c_int()
        check(lib().frank_blr_block_info(self._h, which, i, j, None, C.byref(r)), "frank_blr_block_info")
        return r.value

    # -- filling A_H --------------------------------------------------------
    def set_dense(self, i: int, j: int, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.float64)
        check(lib().frank_blr_set_dense(self._h, i, j, _dptr(a), a.shape[1], 1), "frank_blr_set_dense")

    def set_lowrank(self, i: int, j: int, U: np.ndarray, S: np.ndarray, V: np.ndarray):
        U = np.ascontiguousarray(U, dtype=np.float64)
        S = np.ascontiguousarray(S, dtype=np.float64)
        V = np.ascontiguousarray(V, dtype=np.float64)
        k = S.shape[0]
        check(lib().frank_blr_set_lowrank(self._h, i, j, k, _dptr(U), U.shape[1], _dptr(S), S.shape[1],
                                          _dptr(V), V.shape[1], 1), "frank_blr_set_lowrank")

    def build_kernel(self, kernel: str, points: np.ndarray, eps: float, params: Sequence[float] = (0.0, 0.0)):
        """On-device construction from points (dim x n, axis-major)."""
        x = np.ascontiguousarray(points, dtype=np.float64)
        if x.ndim == 1:
            x = x[None, :]
        kp = np.zeros(2)
        kp[:len(params)] = params
        check(lib().frank_blr_build_kernel(self._h, KERNELS[kernel], _dptr(x), x.shape[0], _dptr(kp),
                                           float(eps), None), "frank_blr_build_kernel")

    # -- reading blocks -----------------------------------------------------
    def block(self, i: int, j: int, which: int = 0):
        """Dense ndarray, or (U, S, V) for a low-rank block; which = 0: A_H,
        1: the factor after getrf."""
        bi, bj = self.block_size(i), self.block_size(j)
        if self.is_lowrank(i, j):
            k = self.rank(i, j, which)
            U = np.zeros((bi, k)); S = np.zeros((k, k)); V = np.zeros((k, bj))
            check(lib().frank_blr_get_lowrank(self._h, which, i, j, _dptr(U), max(k, 1), _dptr(S), max(k, 1),
                                              _dptr(V), bj, 1), "frank_blr_get_lowrank")
            return U, S, V
        a = np.zeros((bi, bj))
        check(lib().frank_blr_get_dense(self._h, which, i, j, _dptr(a), bj, 1), "frank_blr_get_dense")
        return a

    def block_dense(self, i: int, j: int, which: int = 0) -> np.ndarray:
        b = self.block(i, j, which)
        if isinstance(b, tuple):
            U, S, V = b
            return U @ S @ V
        return b

    def to_dense(self, which: int = 0) -> np.ndarray:
        return np.block([[self.block_dense(i, j, which) for j in range(self.nb)] for i in range(self.nb)])

    def pivots(self, i: int) -> np.ndarray:
        p = np.zeros(self.block_size(i), dtype=np.int32)
        check(lib().frank_blr_get_pivots(self._h, i, p.ctypes.data_as(C.POINTER(C.c_int))), "frank_blr_get_pivots")
        return p

    # -- the path -----------------------------------------------------------
    def set_lra(self, name: str, core_scale: float = 0.1):
        """FRANK_LRA: "rounded_addition" (core SVD, the reference algorithm),
        "fast_rounded_addition" (default of fixed-rank plans; tolerance plans
        fall back to rounded_addition), "rounded_addition_rrqr"
        (truncated_geqp3 + rq of the core on stacked bases) or
        "rounded_addition_rrqr_proj" (the same on projected bases, default of
        tolerance plans)."""
        check(lib().frank_blr_set_lra(self._h, name.encode(), float(core_scale)), "frank_blr_set_lra")

    def getrf(self, stream: Optional[int] = None, allow=()):
        return check(lib().frank_blr_getrf(self._h, stream), "frank_blr_getrf", allow)

    def solve(self, b: np.ndarray) -> np.ndarray:
        x = np.asfortranarray(np.array(b, dtype=np.float64, copy=True).reshape(self.n, -1))
        check(lib().frank_blr_solve(self._h, _dptr(x), self.n, x.shape[1], None), "frank_blr_solve")
        return x

    def matvec(self, x: np.ndarray) -> np.ndarray:
        xx = np.asfortranarray(np.asarray(x, dtype=np.float64).reshape(self.n, -1))
        y = np.zeros_like(xx, order="F")
        check(lib().frank_blr_matvec(self._h, _dptr(xx), self.n, _dptr(y), self.n, xx.shape[1], None),
              "frank_blr_matvec")
        return y

    def refine(self, b: np.ndarray, tol: float = 1e-10, maxit: int = 50) -> Tuple[np.ndarray, int, float]:
        bb = np.asfortranarray(np.asarray(b, dtype=np.float64).reshape(self.n, -1))
        x = np.zeros_like(bb, order="F")
        it = C.c_int()
        res = C.c_double()
        check(lib().frank_blr_refine(self._h, _dptr(bb), self.n, _dptr(x), self.n, bb.shape[1], float(tol),
                                     int(maxit), C.byref(it), C.byref(res), None), "frank_blr_refine")
        return x, it.value, res.value

    # device-pointer variants (e.g. torch tensors' data_ptr(), column-major n x nrhs)
    def solve_device(self, ptr: int, nrhs: int, ld: Optional[int] = None, stream: Optional[int] = None):
        check(lib().frank_blr_solve_device(self._h, C.c_void_p(ptr), ld or self.n, nrhs, stream),
              "frank_blr_solve_device")

    def solve_transpose_device(self, ptr: int, nrhs: int, ld: Optional[int] = None, stream: Optional[int] = None):
        check(lib().frank_blr_solve_transpose_device(self._h, C.c_void_p(ptr), ld or self.n, nrhs, stream),
              "frank_blr_solve_transpose_device")

    def matvec_device(self, xptr: int, yptr: int, nrhs: int, stream: Optional[int] = None):
        check(lib().frank_blr_matvec_device(self._h, C.c_void_p(xptr), self.n, C.c_void_p(yptr), self.n, nrhs,
                                            stream), "frank_blr_matvec_device")

    def refine_device(self, bptr: int, xptr: int, nrhs: int, tol: float = 1e-10, maxit: int = 50,
                      stream: Optional[int] = None) -> Tuple[int, float]:
        it = C.c_int()
        res = C.c_double()
        check(lib().frank_blr_refine_device(self._h, C.c_void_p(bptr), self.n, C.c_void_p(xptr), self.n, nrhs,
                                            float(tol), int(maxit), C.byref(it), C.byref(res), stream),
              "frank_blr_refine_device")
        return it.value, res.value

    def autotune(self, force: bool = False, stream: Optional[int] = None) -> dict:
        """Pick the launch parameters by timing this plan's factorization
        (frank_blr_autotune); returns them."""
        check(lib().frank_blr_autotune(self._h, 1 if force else 0, stream), "frank_blr_autotune")
        return self.tuning()

    def set_tuning(self, band_rows: int = 128, split_rank: int = 32, projected: bool = False):
        check(lib().frank_blr_set_tuning(self._h, int(band_rows), int(split_rank), 1 if projected else 0),
              "frank_blr_set_tuning")

    def tuning(self) -> dict:
        v = [C.c_int() for _ in range(3)]
        check(lib().frank_blr_tuning(self._h, *[C.byref(t) for t in v]), "frank_blr_tuning")
        cs = C.c_int()
        check(lib().frank_blr_core_smem(self._h, C.byref(cs)), "frank_blr_core_smem")
        return {"band_rows": v[0].value, "split_rank": v[1].value, "projected": bool(v[2].value),
                "core_smem_doubles": cs.value}

    def set_core_smem(self, doubles: int):
        """Largest recompression core (doubles) kept in shared memory."""
        check(lib().frank_blr_set_core_smem(self._h, int(doubles)), "frank_blr_set_core_smem")

    def write_json(self, path: str, which: int = 0):
        """The block tree with per-block singular values, in the layout of
        FRANK's write_JSON (util/print.cpp:54-128)."""
        check(lib().frank_blr_write_json(self._h, int(which), str(path).encode()), "frank_blr_write_json")

    def set_grid(self, ctas: int):
        """Limit the update / recompression grids to `ctas` thread blocks
        (plans that run concurrently in a batch); every target then runs on
        one CTA."""
        check(lib().frank_blr_set_grid(self._h, int(ctas)), "frank_blr_set_grid")

    def set_timing(self, on: bool = True):
        """Record per-class kernel times inside the factorization graph (off
        by default: the event nodes serialise the graph's concurrent branches)."""
        check(lib().frank_blr_set_timing(self._h, 1 if on else 0), "frank_blr_set_timing")

    def kernel_times(self) -> dict:
        """Per-class device time (ms) and algorithmic FLOPs of the last getrf."""
        ms = np.zeros(4)
        fl = np.zeros(4)
        check(lib().frank_blr_kernel_times(self._h, _dptr(ms), _dptr(fl)), "frank_blr_kernel_times")
        names = ("getrf", "panel", "dense_update", "recompress")
        return {n: {"ms": float(ms[i]), "flops": float(fl[i])} for i, n in enumerate(names)}

    def stats(self) -> dict:
        v = [C.c_int64() for _ in range(4)]
        check(lib().frank_blr_stats(self._h, *[C.byref(t) for t in v]), "frank_blr_stats")
        return {"launches": v[0].value, "recompressions": v[1].value, "max_rank": v[2].value,
                "rank_overflows": v[3].value}


def upload_hierarchical(H, n: int, nb: int, **kw) -> BLRMatrix:
    """Create a BLRMatrix from a one-level block grid given as `H[i][j]` =
    ndarray (dense) or (U, S, V) tuple / object with U, S, V attributes."""
    A = BLRMatrix(n, nb, **kw)
    for i in range(nb):
        for j in range(nb):
            blk = H[i][j]
            if isinstance(blk, np.ndarray) and A.is_lowrank(i, j):
                raise ValueError("block (%d, %d) is dense but low rank under the plan's admissibility" % (i, j))
            if isinstance(blk, np.ndarray):
                A.set_dense(i, j, blk)
            else:
                U, S, V = (blk.U, blk.S, blk.V) if hasattr(blk, "U") else blk
                A.set_lowrank(i, j, U, S, V)
    return A
