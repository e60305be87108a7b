"""The reference's BLR / LowRank / dense-op test sequences written against
FRANK's C++ API (tests/cpp/frank_layer_test.cpp) and run through the
engine's C++ layer on the GPU: blr_fixed_acc_test's LU factorization on its
full grid (solve error <= eps, position- and geometry-based admissibility),
blr_fixed_rank_test with the default fast_rounded_addition, lowrank_test's
addition, qr / rq / svd / id / rid, and the dispatch errors of operations
without an overload."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_frank_layer_program(gpu_lib, tmp_path):
    from frank_b200 import build
    lib = build.build_cpp()
    exe = str(tmp_path / "layer")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "frank_b200", "cpp", "include"),
                           os.path.join(ROOT, "tests", "cpp", "frank_layer_test.cpp"), "-o", exe,
                           "-L" + os.path.dirname(lib), "-lfrank_b200_cpp", "-lfrank_b200",
                           "-Wl,-rpath," + os.path.dirname(lib)])
    out = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-4000:] + out.stderr[-2000:]
    assert "0 failures" in out.stdout
    assert out.stdout.count("PASS") >= 36 + 8 + 2 + 5 + 2
