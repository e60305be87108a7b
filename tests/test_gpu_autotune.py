"""The launch-parameter autotuner (frank_blr_autotune): its choices are
among the candidates, the tuned plan still factors and refines to 1e-10, a
second call reuses the cached choice, and the band height of the dense update
and the split threshold of the recompression change no result (the
per-element arithmetic order is the same), so the tuned factor is bitwise the
default one when the basis mode is unchanged."""
import numpy as np
import pytest

import oracle.frank_oracle as fo

pytestmark = pytest.mark.gpu


def _plan(x, n, nb):
    from frank_b200 import BLRMatrix
    M = BLRMatrix(n, nb, eps=1e-3, precision="mixed")
    M.build_kernel("laplace", x, 1e-8)
    M.set_lra("rounded_addition_rrqr")
    return M


def test_autotune(gpu_lib):
    import time
    n, nb = 8192, 16
    rng = np.random.default_rng(17)
    x, _ = fo.morton_sort(rng.random((3, n)), 10)
    ref = _plan(x, n, nb)
    ref.getrf()
    M = _plan(x, n, nb)
    t = M.autotune(force=True)
    assert t["band_rows"] in (64, 128, 256)
    assert t["split_rank"] in (0, 16, 32, 48, 64, 96)
    assert t["core_smem_doubles"] in (16384, 6144) or t["core_smem_doubles"] > 16384
    t0 = time.perf_counter()
    assert M.autotune() == t                      # cached for this workload shape
    assert time.perf_counter() - t0 < 1.0
    M.getrf()
    b = rng.standard_normal((n, 2))
    xs, it, res = M.refine(b, tol=1e-10, maxit=30)
    assert res <= 1e-10
    if not t["projected"]:
        for i in range(nb):
            for j in range(nb):
                a, c = ref.block(i, j, 1), M.block(i, j, 1)
                if isinstance(a, tuple):
                    assert ref.rank(i, j, 1) == M.rank(i, j, 1)
                    for u, v in zip(a, c):
                        assert np.array_equal(u, v), (i, j)
                else:
                    assert np.array_equal(a, c), (i, j)
    M.close()
    ref.close()
