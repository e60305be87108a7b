"""Batched uneven systems (the batched workload, scaled down): independent
BLR systems of different orders, 2-D kernel -log(r + 1e-3) + N I, blocks of
256, factored in one captured graph and refined together; each system must
give the same solution as when factored alone, at residual <= 1e-10."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system(n, seed):
    import oracle.frank_oracle as fo
    rng = np.random.default_rng(seed)
    x, _ = fo.morton_sort(rng.random((2, n)), 15)
    return x


def _plan(n, x):
    from frank_b200 import BLRMatrix
    M = BLRMatrix(n, n // 256, eps=1e-4, precision="mixed", max_rank=96)
    M.build_kernel("neglog", x, 1e-6, params=(float(n),))
    return M


def test_batch_matches_individual_solves(gpu_lib):
    import torch
    from frank_b200.batch import BLRBatch
    sizes = [512, 1024, 1536, 768, 1024, 2048]
    nmax = max(sizes)
    pts = [_system(n, 5 + k) for k, n in enumerate(sizes)]
    rng = np.random.default_rng(9)
    B = torch.zeros((len(sizes), 2, nmax), dtype=torch.float64, device="cuda")   # per system: column-major nmax x 2
    for k, n in enumerate(sizes):
        B[k, :, :n] = torch.tensor(rng.standard_normal((2, n)))
    X = torch.zeros_like(B)
    plans = [_plan(n, x) for n, x in zip(sizes, pts)]
    batch = BLRBatch(plans, grid=8)
    batch.getrf()
    its, res = batch.refine_device([B[k].data_ptr() for k in range(len(sizes))],
                                   [X[k].data_ptr() for k in range(len(sizes))], nmax, 2, tol=1e-10)
    assert max(res) <= 1e-10
    for k, n in enumerate(sizes):
        M = _plan(n, pts[k])
        M.getrf()
        b = B[k, :, :n].cpu().numpy().T
        xs, it, r = M.refine(b, tol=1e-10)
        got = X[k, :, :n].cpu().numpy().T
        np.testing.assert_allclose(got, xs, rtol=0, atol=1e-9 * np.abs(xs).max())
        # residual against the FP64 compressed matrix
        rr = b - M.matvec(got)
        assert np.max(np.linalg.norm(rr, axis=0) / np.linalg.norm(b, axis=0)) <= 1e-10
        M.close()
    batch.close()
    for p in plans:
        p.close()


def test_batch_matches_oracle(gpu_lib):
    """The batch against the oracle: each system's refined solution against
    the oracle's own BLR compression of the same kernel matrix
    (build_hierarchical with LowRank(Dense, eps), eps 1e-6, solved densely in
    FP64) -- the two compressions differ by O(eps), so the solutions agree to
    a few eps -- and against the dense kernel matrix itself."""
    import torch
    import oracle.frank_oracle as fo
    from frank_b200.batch import BLRBatch
    sizes = [512, 1024, 768]
    nmax = max(sizes)
    pts = [_system(n, 21 + k) for k, n in enumerate(sizes)]
    rng = np.random.default_rng(23)
    B = torch.zeros((len(sizes), 1, nmax), dtype=torch.float64, device="cuda")
    for k, n in enumerate(sizes):
        B[k, :, :n] = torch.tensor(rng.standard_normal((1, n)))
    X = torch.zeros_like(B)
    plans = [_plan(n, x) for n, x in zip(sizes, pts)]
    batch = BLRBatch(plans, grid=8)
    batch.getrf()
    its, res = batch.refine_device([B[k].data_ptr() for k in range(len(sizes))],
                                   [X[k].data_ptr() for k in range(len(sizes))], nmax, 1, tol=1e-10)
    assert max(res) <= 1e-10
    for k, n in enumerate(sizes):
        kern = fo.make_neglog_shift(float(n))
        H = fo.build_hierarchical(kern, pts[k], n, 256, n // 256, eps=1e-6)
        b = B[k, 0, :n].cpu().numpy()
        x_oracle = np.linalg.solve(fo.to_dense(H), b)
        x_dense = np.linalg.solve(kern(pts[k], 0, n, 0, n), b)
        got = X[k, 0, :n].cpu().numpy()
        assert np.linalg.norm(got - x_oracle) <= 10 * 1e-6 * np.linalg.norm(x_oracle)
        assert np.linalg.norm(got - x_dense) <= 10 * 1e-6 * np.linalg.norm(x_dense)
    batch.close()
    for p in plans:
        p.close()
