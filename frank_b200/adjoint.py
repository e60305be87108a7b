"""Differentiable solve x = A(theta)^{-1} b for the exponential kernel
A_ij = exp(-r_ij / theta) + nugget delta_ij on a BLR matrix on the GPU.

Forward: on-device construction of A_H(theta) (compression to eps), factor
(FP64 or mixed) and FP64 iterative refinement to `tol`.
Backward (hand-written adjoint): reuse the factors for the transposed solve
A^T lambda = g (refined against A_H^T), then
    dL/db = lambda,  dL/dtheta = -sum_h lambda_h^T (dA/dtheta) x_h,
with dA/dtheta = exp(-r/theta) r / theta^2 contracted on the fly by a CUDA
kernel (the kernel matrix is never formed).  No reference counterpart: this is
the adjoint the python/FRANK bindings expose.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _abi
from ._abi import check, lib
from .blr import BLRMatrix


def _colmajor(t: torch.Tensor) -> torch.Tensor:
    """(n,) or (n, k) -> contiguous (k, n) FP64 CUDA tensor (= column-major n x k)."""
    t = t.to(device="cuda", dtype=torch.float64)
    if t.dim() == 1:
        t = t[:, None]
    return t.t().contiguous()


class BLRSolveExp(torch.autograd.Function):
    @staticmethod
    def forward(ctx, b, theta, points, nb, eps, nugget, precision, factor_eps, tol, maxit):
        th = float(theta)
        pts = points.to(device="cuda", dtype=torch.float64).contiguous()
        dim, n = pts.shape
        M = BLRMatrix(n, nb, eps=factor_eps, precision=precision)
        M.build_kernel("exp", pts.cpu().numpy(), eps, params=(th, nugget))
        M.getrf()
        bc = _colmajor(b)
        xc = torch.zeros_like(bc)
        it, res = M.refine_device(bc.data_ptr(), xc.data_ptr(), bc.shape[0], tol=tol, maxit=maxit)
        ctx.M, ctx.tol, ctx.maxit = M, tol, maxit
        ctx.theta, ctx.nugget, ctx.dim, ctx.n = th, nugget, dim, n
        ctx.vec = b.dim() == 1
        ctx.save_for_backward(pts, xc)
        ctx.iters, ctx.resid = it, res
        x = xc.t()
        return (x[:, 0] if ctx.vec else x).to(b.dtype)

    @staticmethod
    def backward(ctx, g):
        pts, xc = ctx.saved_tensors
        M = ctx.M
        gc = _colmajor(g)
        lam = torch.zeros_like(gc)
        it = C.c_int(); res = C.c_double()
        check(lib().frank_blr_refine_transpose_device(M._h, C.c_void_p(gc.data_ptr()), M.n, C.c_void_p(lam.data_ptr()),
                                                      M.n, gc.shape[0], float(ctx.tol), int(ctx.maxit), C.byref(it),
                                                      C.byref(res), None), "frank_blr_refine_transpose_device")
        out = C.c_double()
        kp = (C.c_double * 2)(ctx.theta, ctx.nugget)
        check(lib().frank_kernel_dtheta_contract(_abi.FRANK_KERNEL_EXP, C.c_void_p(pts.data_ptr()), ctx.dim, ctx.n, kp,
                                                 C.c_void_p(lam.data_ptr()), M.n, C.c_void_p(xc.data_ptr()), M.n,
                                                 gc.shape[0], C.byref(out), None), "frank_kernel_dtheta_contract")
        grad_b = lam.t()
        if ctx.vec:
            grad_b = grad_b[:, 0]
        grad_theta = torch.tensor(-out.value, dtype=torch.float64, device="cuda")
        M.close()
        return grad_b, grad_theta, None, None, None, None, None, None, None, None


def solve_exp(b, theta, points, nb, eps=1e-9, nugget=1e-2, precision="fp64", factor_eps=None, tol=1e-12, maxit=60):
    """x = A(theta)^{-1} b, differentiable in b and theta (a 0-d tensor).
    points: (dim, n) coordinates in the reference's params[d][i] layout."""
    return BLRSolveExp.apply(b, theta, points, nb, eps, nugget, precision,
                             eps if factor_eps is None else factor_eps, tol, maxit)
