"""Batches of independent BLR systems on one GPU (the batched uneven-systems
workload): all factorizations in one captured CUDA graph, one branch per
system, and a batched FP64 refinement."""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence, Tuple

import numpy as np

from ._abi import check, lib
from .blr import BLRMatrix


class BLRBatch:
    def __init__(self, plans: Sequence[BLRMatrix], grid: int = 0):
        self.plans = list(plans)
        if grid > 0:
            for p in self.plans:
                check(lib().frank_blr_set_grid(p._h, int(grid)), "frank_blr_set_grid")
        arr = (C.c_void_p * len(self.plans))(*[p._h.value for p in self.plans])
        h = C.c_void_p()
        check(lib().frank_batch_create(arr, len(self.plans), C.byref(h)), "frank_batch_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().frank_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def getrf(self):
        check(lib().frank_batch_getrf(self._h, None), "frank_batch_getrf")

    def refine_device(self, b_ptrs: Sequence[int], x_ptrs: Sequence[int], ld: int, nrhs: int, tol: float = 1e-10,
                      maxit: int = 50) -> Tuple[List[int], List[float]]:
        """Refine every system; b_ptrs / x_ptrs are device pointers to
        column-major (ld x nrhs) blocks, ld >= the largest order."""
        K = len(self.plans)
        bp = (C.c_void_p * K)(*b_ptrs)
        xp = (C.c_void_p * K)(*x_ptrs)
        its = np.zeros(K, dtype=np.int32)
        res = np.zeros(K)
        check(lib().frank_batch_refine_device(self._h, bp, int(ld), xp, int(ld), int(nrhs), float(tol), int(maxit),
                                              its.ctypes.data_as(C.POINTER(C.c_int)),
                                              res.ctypes.data_as(C.POINTER(C.c_double))), "frank_batch_refine_device")
        return its.tolist(), res.tolist()
