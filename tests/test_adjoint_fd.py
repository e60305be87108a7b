"""CPU check of the adjoint formula used by the GPU adjoint tests: the dense
theta-gradient of L = 0.5 ||A(theta)^{-1} b||^2 against central differences."""
import numpy as np

from tests.test_gpu_adjoint import _dense_loss_grad


def test_adjoint_formula_matches_central_differences():
    """The dense adjoint formula itself against central differences, h = 1e-6
    (CPU only: validates the gradient the GPU path is compared with)."""
    n, theta, nugget, h = 400, 0.2, 1e-2, 1e-6
    rng = np.random.default_rng(7)
    pts = rng.random((2, n))
    b = rng.standard_normal(n)
    _, _, g = _dense_loss_grad(pts, theta, nugget, b)
    Lp = _dense_loss_grad(pts, theta + h, nugget, b)[0]
    Lm = _dense_loss_grad(pts, theta - h, nugget, b)[0]
    assert abs((Lp - Lm) / (2 * h) - g) <= 1e-5 * abs(g)
