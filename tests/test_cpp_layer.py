"""CPU tests of the C++ layer: the multimethod layer's resolution rules
(tests/cpp/multimethod_test.cpp, no GPU), and the FRANK layer library
building and linking a program written against FRANK's API."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "frank_b200", "cpp", "include")


def test_multimethod_resolution(tmp_path):
    exe = str(tmp_path / "mm")
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I" + INC,
                           os.path.join(ROOT, "tests", "cpp", "multimethod_test.cpp"), "-o", exe])
    out = subprocess.run([exe], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "0 failures" in out.stdout


def test_frank_layer_builds_and_links(tmp_path):
    from frank_b200 import build
    lib = build.build_cpp()
    exe = str(tmp_path / "layer")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-Wall", "-I" + INC,
                           os.path.join(ROOT, "tests", "cpp", "frank_layer_test.cpp"), "-o", exe,
                           "-L" + os.path.dirname(lib), "-lfrank_b200_cpp", "-lfrank_b200",
                           "-Wl,-rpath," + os.path.dirname(lib)])
    assert os.path.exists(exe)
