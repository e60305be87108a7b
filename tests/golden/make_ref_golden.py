"""Generate the reference fixtures of tests/golden from the reference itself.

Runs oracle/_ref/frank_ref -- FRANK's own sources compiled by
oracle/build_ref.py, driven through FRANK's public API (oracle/ref_driver.cpp)
-- and records its outputs:

* reference_blr.json: per case of the reference's BLR test grids
  (test/blr_fixed_acc_test.cpp:192-198 with FRANK_LRA=rounded_addition;
  test/blr_fixed_rank_test.cpp:58-64 with the default LowRank addition,
  fast_rounded_addition, and with rounded_addition): solve error
  l2_error(x, x_hat) for b = A_H x with the reference's x = random_uniform,
  residual, factorization error ||A_H V - L U V|| / ||A_H V|| on random
  probes, and the per-block ranks of A_H, L and U;
* reference_json_n256.json: write_JSON (util/print.cpp:124-128) of the
  Laplace-1D N=256 matrix in 4 x 4 blocks at eps 1e-8 (block tree and
  per-block singular values);
* reference_vectors.npz: for the fixed-rank Laplace-1D N=2048 workload (8 x 8
  blocks of 256, rank 16; both LowRank additions) and the leading 8 x 8 blocks
  (N=4096) of the headline Laplace-3D point set at eps 1e-8 (4 RHS): the
  solution x_hat, the singular values of every low-rank factor block (basis
  independent) and the diagonal of every U(i, i).

Usage: python tests/golden/make_ref_golden.py [--workdir DIR]
(builds oracle/_ref first if needed; needs the FRANK sources for that).
"""
from __future__ import annotations

import argparse
import itertools
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

EXE = os.path.join(ROOT, "oracle", "_ref", "frank_ref")


def run(args, threads=1):
    out = subprocess.check_output([EXE, *map(str, args), "--threads", str(threads)], text=True)
    return json.loads(out.strip().splitlines()[-1])


def read_factor(path):
    """Blocks of a --dump-factor file: {(i, j, 'L'|'U'): ('dense', A) | ('lr', U, S, V)}.
    The file lists, for each (i, j), L(i, j) when i >= j, then U(i, j) when i <= j."""
    raw = open(path, "rb").read()
    pos, out, seen = 0, {}, set()
    while pos < len(raw):
        i, j, typ, rows, cols, rank = np.frombuffer(raw, dtype=np.int64, count=6, offset=pos)
        pos += 48
        side = "L" if (i > j or (i == j and (i, j) not in seen)) else "U"
        if i == j:
            seen.add((i, j))
        if typ == 0:
            A = np.frombuffer(raw, dtype=np.float64, count=rows * cols, offset=pos).reshape(rows, cols)
            pos += 8 * rows * cols
            out[(int(i), int(j), side)] = ("dense", A.copy())
        elif typ == 1:
            U = np.frombuffer(raw, dtype=np.float64, count=rows * rank, offset=pos).reshape(rows, rank)
            pos += 8 * rows * rank
            S = np.frombuffer(raw, dtype=np.float64, count=rank * rank, offset=pos).reshape(rank, rank)
            pos += 8 * rank * rank
            V = np.frombuffer(raw, dtype=np.float64, count=rank * cols, offset=pos).reshape(rank, cols)
            pos += 8 * rank * cols
            out[(int(i), int(j), side)] = ("lr", U.copy(), S.copy(), V.copy())
        else:
            out[(int(i), int(j), side)] = ("other",)
    return out


def lowrank_singular_values(U, S, V):
    """Singular values of U S V without forming it (QR of both bases)."""
    qu, ru = np.linalg.qr(U)
    qv, rv = np.linalg.qr(V.T)
    return np.linalg.svd(ru @ S @ rv.T, compute_uv=False)


def vectors_case(tag, args, wd, out, threads):
    fx, fd = os.path.join(wd, tag + "_x.bin"), os.path.join(wd, tag + "_f.bin")
    info = run([*args, "--residual", "--factor-error", "--dump-x", fx, "--dump-factor", fd], threads)
    out[tag + "/x"] = np.fromfile(fx, dtype=np.float64)
    blocks = read_factor(fd)
    nb = int(info["nb"])
    for (i, j, side), blk in blocks.items():
        if blk[0] == "lr":
            out["%s/sv/%s/%d/%d" % (tag, side, i, j)] = lowrank_singular_values(*blk[1:])
        elif blk[0] == "dense" and i == j and side == "U":
            out["%s/udiag/%d" % (tag, i)] = np.diag(blk[1]).copy()
    meta = {k: v for k, v in info.items()}
    meta["nb"] = nb
    return meta


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workdir", default=None)
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    a = ap.parse_args()
    if not os.path.exists(EXE):
        from oracle.build_ref import build
        build(os.environ.get("FRANK_REFERENCE", "/root/reference"))
    from bench import make_points, make_rhs

    cases = []
    # test/blr_fixed_acc_test.cpp:192-198 (FRANK_LRA=rounded_addition, SetUp :18)
    for n, eps, admis, at in itertools.product((128, 256), (1e-6, 1e-8, 1e-10), (0.0, 1.0, 4.0),
                                               ("position", "geometry")):
        r = run(["--n", n, "--nb", n // 32, "--eps", eps, "--admis", admis, "--admis-type", at,
                 "--lra", "rounded_addition", "--residual", "--factor-error"])
        cases.append(dict(grid="blr_fixed_acc", lra="rounded_addition", n=n, nleaf=32, eps=eps, admis=admis,
                          admis_type=at, **{k: r[k] for k in ("solve_error", "residual", "factor_error",
                                                              "ranks_h", "ranks_l", "ranks_u")}))
    # test/blr_fixed_rank_test.cpp:58-64 (default LowRank addition) and rounded_addition
    for lra, n, rank, admis, at in itertools.product(("fast", "rounded_addition"), (128, 256), (4, 8),
                                                     (0.0, 0.5, 1.0, 2.0), ("position", "geometry")):
        r = run(["--n", n, "--nb", n // 32, "--rank", rank, "--admis", admis, "--admis-type", at,
                 "--lra", lra, "--residual", "--factor-error"])
        cases.append(dict(grid="blr_fixed_rank", lra=("fast_rounded_addition" if lra == "fast" else lra), n=n,
                          nleaf=32, rank=rank, admis=admis, admis_type=at,
                          **{k: r[k] for k in ("solve_error", "residual", "factor_error", "ranks_h", "ranks_l",
                                               "ranks_u")}))

    vec, meta = {}, {}
    with tempfile.TemporaryDirectory(dir=a.workdir) as wd:
        # fixed-rank Laplace-1D N=2048 (8 x 8 blocks of 256, rank 16)
        for lra in ("fast", "rounded_addition"):
            tag = "cfg1_" + lra
            meta[tag] = vectors_case(tag, ["--n", 2048, "--nb", 8, "--rank", 16, "--lra", lra], wd, vec,
                                     a.threads)
        # leading 8 x 8 blocks of 512 (N=4096) of the headline Laplace-3D point set, eps 1e-8, 4 RHS
        x = make_points(32768, 3, 2, 10)[:, :4096].copy()
        b = make_rhs(4096, 4, 3)
        px, pb = os.path.join(wd, "pts.bin"), os.path.join(wd, "rhs.bin")
        x.tofile(px)
        b.T.copy().tofile(pb)
        tag = "headline4096"
        meta[tag] = vectors_case(tag, ["--n", 4096, "--nb", 8, "--eps", 1e-8, "--lra", "rounded_addition",
                                       "--points", px, "--dim", 3, "--rhs", pb, "--nrhs", 4], wd, vec, a.threads)
        vec[tag + "/points_checksum"] = np.array([x.sum(), (x * x).sum()])
        vec[tag + "/rhs_checksum"] = np.array([b.sum(), (b * b).sum()])
    with tempfile.TemporaryDirectory(dir=a.workdir) as wd:
        pj = os.path.join(wd, "h.json")
        run(["--n", 256, "--nb", 4, "--eps", 1e-8, "--no-solve", "--write-json", pj])
        with open(pj) as f, open(os.path.join(HERE, "reference_json_n256.json"), "w") as g:
            g.write(f.read())
    with open(os.path.join(HERE, "reference_blr.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_ref_golden.py (oracle/_ref/frank_ref)", "cases": cases,
                   "vectors_meta": meta}, f, indent=0)
    np.savez_compressed(os.path.join(HERE, "reference_vectors.npz"), **vec)
    print("cases:", len(cases), "vector entries:", len(vec))


if __name__ == "__main__":
    main()
