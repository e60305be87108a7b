"""Adjoint of solve(A(theta), b) for the exponential kernel (the adjoint
workload, scaled down): the hand-written backward (transposed solve with the
same factors + on-the-fly dA/dtheta contraction) against a dense FP64
reference gradient, and against central finite differences of the GPU
forward itself."""
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




def test_adjoint_matches_finite_differences_through_gpu(gpu_lib):
    """d loss / d theta from the GPU backward against central finite
    differences of the GPU forward itself (FP64 plan, A_H at 1e-12, h = 1e-4:
    truncation error O(h^2) ~ 1e-8, rounding ~ 1e-13 / h): agree to 1e-5."""
    import torch
    from frank_b200.adjoint import solve_exp
    n, nb, theta, nugget, h = 1024, 4, 0.2, 1e-2, 1e-4
    rng = np.random.default_rng(8)
    pts = torch.tensor(rng.random((2, n)))
    b = torch.tensor(rng.standard_normal(n), device="cuda")

    def loss_at(t, grad=False):
        th = torch.tensor(t, dtype=torch.float64, device="cuda", requires_grad=grad)
        x = solve_exp(b, th, pts, nb, eps=1e-12, nugget=nugget, precision="fp64", tol=1e-13)
        L = 0.5 * (x * x).sum()
        if grad:
            L.backward()
            return L.item(), th.grad.item()
        return L.item()

    _, g = loss_at(theta, grad=True)
    fd = (loss_at(theta + h) - loss_at(theta - h)) / (2 * h)
    assert abs(g - fd) <= 1e-5 * abs(fd), (g, fd)
