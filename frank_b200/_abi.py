"""ctypes binding of the C ABI in include/frank_b200.h.

Loading fails loudly if the sm_100a library has not been built: there is no
CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

from .build import LIB

FRANK_OK = 0
FRANK_ERR_INVALID = 1
FRANK_ERR_SINGULAR = 2
FRANK_ERR_UNSUPPORTED = 3
FRANK_ERR_NOT_CONVERGED = 4
FRANK_ERR_TIMEOUT = 5
FRANK_ERR_CUDA = 6
FRANK_ERR_RANK_OVERFLOW = 7
FRANK_ERR_STATE = 8

FRANK_PREC_FP64 = 0
FRANK_PREC_MIXED = 1
FRANK_BLOCK_DENSE = 0
FRANK_BLOCK_LOWRANK = 1
FRANK_KERNEL_LAPLACE = 0
FRANK_KERNEL_HELMHOLTZ = 1
FRANK_KERNEL_NEGLOG = 2
FRANK_KERNEL_EXP = 3

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_i64p = C.POINTER(C.c_int64)
_vp = C.c_void_p


class BlrDesc(C.Structure):
    _fields_ = [("n", C.c_int64), ("nb", C.c_int32), ("max_rank", C.c_int32),
                ("precision", C.c_int32), ("fixed_rank", C.c_int32),
                ("eps", C.c_double), ("admis", C.c_double)]


# name -> (restype, argtypes); one entry per declaration in include/frank_b200.h
SIGNATURES = {
    "frank_last_error": (C.c_char_p, []),
    "frank_device_info": (C.c_int, [C.c_char_p, C.c_int, _ip, _ip, _ip]),
    "frank_blr_create": (C.c_int, [C.POINTER(BlrDesc), C.POINTER(_vp)]),
    "frank_blr_create_geometric": (C.c_int, [C.POINTER(BlrDesc), _dp, C.c_int, C.POINTER(_vp)]),
    "frank_device_alloc": (C.c_int, [C.c_size_t, C.POINTER(_vp)]),
    "frank_device_free": (C.c_int, [_vp]),
    "frank_copy": (C.c_int, [_vp, _vp, C.c_size_t, C.c_int]),
    "frank_blr_autotune": (C.c_int, [_vp, C.c_int, _vp]),
    "frank_blr_tuning": (C.c_int, [_vp, _ip, _ip, _ip]),
    "frank_blr_core_smem": (C.c_int, [_vp, _ip]),
    "frank_blr_set_core_smem": (C.c_int, [_vp, C.c_int]),
    "frank_blr_set_tuning": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int]),
    "frank_blr_write_json": (C.c_int, [_vp, C.c_int, C.c_char_p]),
    "frank_blr_trsm": (C.c_int, [_vp, C.c_int, _dp, C.c_int64, C.c_int, _vp]),
    "frank_blr_gemv": (C.c_int, [_vp, C.c_double, _dp, C.c_int64, C.c_double, _dp, C.c_int64, C.c_int, _vp]),
    "frank_gemm_batched": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _vp, C.c_int64, C.c_int64,
                                     C.c_int, _vp, C.c_int64, C.c_int64, C.c_int, C.c_double, _vp, C.c_int64,
                                     C.c_int64, _vp]),
    "frank_qr_batched": (C.c_int, [C.c_int, C.c_int, C.c_int, _vp, C.c_int64, C.c_int64, _vp, C.c_int64, C.c_int64,
                                   _vp, C.c_int64, C.c_int64, _vp]),
    "frank_rq_batched": (C.c_int, [C.c_int, C.c_int, C.c_int, _vp, C.c_int64, C.c_int64, _vp, C.c_int64, C.c_int64,
                                   _vp, C.c_int64, C.c_int64, _vp]),
    "frank_svd_batched": (C.c_int, [C.c_int, C.c_int, C.c_int, _vp, C.c_int64, C.c_int64, _vp, C.c_int64, C.c_int64,
                                    _vp, C.c_int64, _vp, C.c_int64, C.c_int64, _vp]),
    "frank_rsvd_batched": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _vp, C.c_int64, C.c_int64,
                                     _vp, C.c_int64, C.c_int64, _vp, C.c_int64, C.c_int64, _vp, C.c_int64, C.c_int64,
                                     _vp]),
    "frank_id_batched": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _vp, C.c_int64, C.c_int64, _vp, C.c_int64,
                                   C.c_int64, _vp, C.c_int64, C.c_int64, _vp, C.c_int64, C.c_int64, _vp, _vp, _vp]),
    "frank_rid_batched": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _vp, C.c_int64, C.c_int64, _vp,
                                    C.c_int64, C.c_int64, _vp, C.c_int64, C.c_int64, _vp, C.c_int64, C.c_int64, _vp]),
    "frank_lowrank_add_batched": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_double,
                                            _vp, C.c_int64, C.c_int64, _vp, C.c_int64, C.c_int64, _vp, C.c_int64,
                                            C.c_int64, _vp, _vp, C.c_int64, C.c_int64, _vp, C.c_int64, C.c_int64,
                                            _vp, C.c_int64, C.c_int64, _vp, C.c_int, _vp]),
    "frank_blr_destroy": (C.c_int, [_vp]),
    "frank_blr_offsets": (C.c_int, [_vp, _i64p]),
    "frank_blr_set_dense": (C.c_int, [_vp, C.c_int, C.c_int, _dp, C.c_int64, C.c_int]),
    "frank_blr_set_lowrank": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _dp, C.c_int64, _dp, C.c_int64,
                                        _dp, C.c_int64, C.c_int]),
    "frank_blr_build_kernel": (C.c_int, [_vp, C.c_int, _dp, C.c_int, _dp, C.c_double, _vp]),
    "frank_blr_block_info": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _ip, _ip]),
    "frank_blr_get_dense": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _dp, C.c_int64, C.c_int]),
    "frank_blr_get_lowrank": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _dp, C.c_int64, _dp, C.c_int64,
                                        _dp, C.c_int64, C.c_int]),
    "frank_blr_get_pivots": (C.c_int, [_vp, C.c_int, _ip]),
    "frank_blr_set_lra": (C.c_int, [_vp, C.c_char_p, C.c_double]),
    "frank_blr_getrf": (C.c_int, [_vp, _vp]),
    "frank_blr_solve": (C.c_int, [_vp, _dp, C.c_int64, C.c_int, _vp]),
    "frank_blr_solve_device": (C.c_int, [_vp, C.c_void_p, C.c_int64, C.c_int, _vp]),
    "frank_blr_matvec": (C.c_int, [_vp, _dp, C.c_int64, _dp, C.c_int64, C.c_int, _vp]),
    "frank_blr_matvec_device": (C.c_int, [_vp, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int, _vp]),
    "frank_blr_refine": (C.c_int, [_vp, _dp, C.c_int64, _dp, C.c_int64, C.c_int, C.c_double, C.c_int,
                                   _ip, _dp, _vp]),
    "frank_blr_refine_device": (C.c_int, [_vp, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int,
                                          C.c_double, C.c_int, _ip, _dp, _vp]),
    "frank_blr_solve_transpose_device": (C.c_int, [_vp, C.c_void_p, C.c_int64, C.c_int, _vp]),
    "frank_blr_stats": (C.c_int, [_vp, _i64p, _i64p, _i64p, _i64p]),
    "frank_blr_kernel_times": (C.c_int, [_vp, _dp, _dp]),
    "frank_blr_set_grid": (C.c_int, [_vp, C.c_int]),
    "frank_blr_set_timing": (C.c_int, [_vp, C.c_int]),
    "frank_batch_create": (C.c_int, [C.POINTER(_vp), C.c_int, C.POINTER(_vp)]),
    "frank_batch_destroy": (C.c_int, [_vp]),
    "frank_batch_getrf": (C.c_int, [_vp, _vp]),
    "frank_batch_refine_device": (C.c_int, [_vp, C.POINTER(C.c_void_p), C.c_int64, C.POINTER(C.c_void_p), C.c_int64,
                                            C.c_int, C.c_double, C.c_int, _ip, _dp]),
    "frank_blr_matvec_transpose_device": (C.c_int, [_vp, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int,
                                                    _vp]),
    "frank_blr_refine_transpose_device": (C.c_int, [_vp, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int,
                                                    C.c_double, C.c_int, _ip, _dp, _vp]),
    "frank_kernel_dtheta_contract": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_int64, _dp, C.c_void_p, C.c_int64,
                                               C.c_void_p, C.c_int64, C.c_int, _dp, _vp]),
    "frank_getrf_dense_noalloc": (C.c_int, [C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.c_int64, C.c_void_p,
                                            _vp]),
    "frank_hodlr_create": (C.c_int, [C.c_int64, C.c_int, C.c_int, C.POINTER(_vp)]),
    "frank_hodlr_destroy": (C.c_int, [_vp]),
    "frank_hodlr_shape": (C.c_int, [_vp, _i64p, _ip, _ip, _ip]),
    "frank_hodlr_set_lra": (C.c_int, [_vp, C.c_char_p]),
    "frank_hodlr_set_dense": (C.c_int, [_vp, C.c_int, _dp, C.c_int64]),
    "frank_hodlr_set_lowrank": (C.c_int, [_vp, C.c_int, C.c_int, _dp, _dp, _dp]),
    "frank_hodlr_get_dense": (C.c_int, [_vp, C.c_int, C.c_int, _dp, C.c_int64]),
    "frank_hodlr_get_lowrank": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp]),
    "frank_hodlr_get_pivots": (C.c_int, [_vp, C.c_int, _ip]),
    "frank_hodlr_build_kernel": (C.c_int, [_vp, C.c_int, _dp, C.c_int, _dp, _vp]),
    "frank_hodlr_getrf": (C.c_int, [_vp, _vp]),
    "frank_hodlr_solve_device": (C.c_int, [_vp, C.c_void_p, C.c_int64, C.c_int, _vp]),
    "frank_hodlr_trsm_device": (C.c_int, [_vp, C.c_int, C.c_void_p, C.c_int64, C.c_int, _vp]),
    "frank_hodlr_matvec_device": (C.c_int, [_vp, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int, _vp]),
    "frank_hodlr_refine_device": (C.c_int, [_vp, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int,
                                            C.c_double, C.c_int, _ip, _dp, _vp]),
    "frank_hodlr_stats": (C.c_int, [_vp, _i64p, _dp]),
}

_lib = None


def lib():
    """Load and type the library once; raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError(
                "frank_b200 CUDA library not built (%s); run `python -m frank_b200.build`" % LIB)
        h = C.CDLL(LIB)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(h, name)
            f.restype = res
            f.argtypes = args
        _lib = h
    return _lib


class FrankError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = lib().frank_last_error().decode()
        super().__init__("%s failed (code %d): %s" % (where, code, msg))
        self.code = code


def check(code: int, where: str, allow=()):
    if code != FRANK_OK and code not in allow:
        raise FrankError(code, where)
    return code
