"""Build the sm_100a shared library `frank_b200/lib/libfrank_b200.so` with nvcc.

The library is built in-tree so it travels with the repository snapshot; no
JIT cache is used.  `python -m frank_b200.build` rebuilds it.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libfrank_b200.so")
SOURCES = ["api.cu", "ops.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps():
    files = []
    for root, _, names in os.walk(CSRC):
        files += [os.path.join(root, n) for n in names if n.endswith((".cu", ".cuh", ".h"))]
    files.append(os.path.join(HERE, "..", "include", "frank_b200.h"))
    return files


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _deps())


CPP_DIR = os.path.join(HERE, "cpp")
CPP_LIB = os.path.join(LIBDIR, "libfrank_b200_cpp.so")


def build_cpp(force: bool = False) -> str:
    """The C++ layer (namespace FRANK over the C ABI) as libfrank_b200_cpp.so,
    linked against libfrank_b200.so next to it."""
    lib = build(force=force)
    srcs = [os.path.join(CPP_DIR, "frank.cpp")]
    deps = srcs + [os.path.join(CPP_DIR, "include", "frank_b200", f) for f in ("FRANK.hpp", "multimethod.hpp")]
    deps.append(os.path.join(HERE, "..", "include", "frank_b200.h"))
    if not force and os.path.exists(CPP_LIB) and all(os.path.getmtime(d) <= os.path.getmtime(CPP_LIB)
                                                      for d in deps + [lib]):
        return CPP_LIB
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall", "-I" + os.path.join(CPP_DIR, "include"), *srcs,
           "-o", CPP_LIB + ".tmp", "-L" + LIBDIR, "-lfrank_b200", "-Wl,-rpath,$ORIGIN"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("g++ failed:\n" + res.stdout + res.stderr)
    os.replace(CPP_LIB + ".tmp", CPP_LIB)
    return CPP_LIB


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    cmd = [_nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "--threads", "2",
           "-diag-suppress", "177", *[os.path.join(CSRC, s) for s in SOURCES], "-o", LIB + ".tmp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    os.replace(LIB + ".tmp", LIB)
    if verbose:
        sys.stdout.write(res.stdout + res.stderr)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
    print(build_cpp())
