"""Regenerate the golden fixtures of tests/golden (run where the FRANK sources
are available; the fixtures are committed so the tests never need them).

Usage: python tests/golden/make_golden.py --reference <FRANK checkout> [--workdir <dir>]

1. libstdcxx_mt19937_seed0.txt: raw std::mt19937(0) outputs and libstdc++
   uniform_real_distribution / normal_distribution draws, printed by
   gen_libstdcxx_mt19937.cpp compiled with the system g++ (the C++ standard
   library the reference's RNG calls resolve to: functions.cpp:36-66,
   util/experiment_setup.cpp:12-23).
2. prototype_dense_lu.npz: the reference's Python prototype (python/FRANK,
   Dense.getrf / Dense.trsm, dense.py:136-170) applied to laplace1d blocks
   (functions.py laplace1d) with the dense_getrf_test diagonal boost
   (test/dense_getrf_test.cpp:25-30), n = 8, 16, 32.
"""
import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def make_rng(workdir):
    exe = os.path.join(workdir, "gen_libstdcxx_mt19937")
    subprocess.check_call(["g++", "-O2", os.path.join(HERE, "gen_libstdcxx_mt19937.cpp"), "-o", exe])
    out = subprocess.check_output([exe]).decode()
    with open(os.path.join(HERE, "libstdcxx_mt19937_seed0.txt"), "w") as f:
        f.write(out)


def make_prototype_lu(reference):
    sys.path.insert(0, os.path.join(reference, "python"))
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from FRANK.dense import Dense            # reference prototype
    from FRANK.functions import laplace1d
    from oracle.frank_oracle import get_sorted_random_vector
    out = {}
    for n in (8, 16, 32):
        x = get_sorted_random_vector(n)
        A = Dense(x, laplace1d, n, n)
        d = n * n
        for i in range(n):
            A.data[i, i] += d
            d -= 1
        out["A%d" % n] = A.data.copy()
        A.getrf()
        out["LU%d" % n] = A.data.copy()
        b = Dense(np.arange(1, n + 1, dtype=float)[:, None].copy())
        b.trsm(A, "l")
        b.trsm(A, "u")
        out["x%d" % n] = b.data.copy()
    np.savez(os.path.join(HERE, "prototype_dense_lu.npz"), **out)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="FRANK source tree (its python/ prototype is imported)")
    ap.add_argument("--workdir", default=None, help="scratch directory for the compiled RNG probe")
    args = ap.parse_args()
    with tempfile.TemporaryDirectory(dir=args.workdir) as wd:
        make_rng(wd)
    make_prototype_lu(args.reference)
    print("ok")
