"""Adjoint of solve(A(theta), b) for the exponential kernel (the adjoint
workload, scaled down): the hand-written backward (transposed solve with the
same factors + on-the-fly dA/dtheta contraction) against a dense FP64
reference gradient and central finite differences (h = 1e-6)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dense(points, theta, nugget):
    d = np.sqrt(((points[:, :, None] - points[:, None, :]) ** 2).sum(0))
    return np.exp(-d / theta) + nugget * np.eye(points.shape[1]), d


def _dense_loss_grad(points, theta, nugget, b):
    A, d = _dense(points, theta, nugget)
    x = np.linalg.solve(A, b)
    lam = np.linalg.solve(A.T, x)           # dL/db for L = 0.5 ||x||^2
    dA = np.exp(-d / theta) * d / theta ** 2
    return 0.5 * float((x * x).sum()), lam, -float((lam * (dA @ x)).sum())


@pytest.mark.parametrize("precision,factor_eps", [("fp64", 1e-10), ("mixed", 1e-5)])
def test_adjoint_matches_dense_gradient(gpu_lib, precision, factor_eps):
    import torch
    from frank_b200.adjoint import solve_exp
    n, nb, theta, nugget = 1024, 4, 0.2, 1e-2
    rng = np.random.default_rng(6)
    pts = rng.random((2, n))
    b = rng.standard_normal(n)
    bt = torch.tensor(b, device="cuda", requires_grad=True)
    th = torch.tensor(theta, dtype=torch.float64, device="cuda", requires_grad=True)
    x = solve_exp(bt, th, torch.tensor(pts), nb, eps=1e-10, nugget=nugget, precision=precision,
                  factor_eps=factor_eps, tol=1e-13)
    loss = 0.5 * (x * x).sum()
    loss.backward()
    L, lam, gth = _dense_loss_grad(pts, theta, nugget, b)
    assert abs(loss.item() - L) <= 1e-7 * abs(L)
    np.testing.assert_allclose(bt.grad.cpu().numpy(), lam, rtol=0, atol=1e-6 * np.abs(lam).max())
    assert abs(th.grad.item() - gth) <= 1e-6 * abs(gth)


