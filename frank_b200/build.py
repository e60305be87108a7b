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
SOURCES = ["api.cu", "ops.cu", "hodlr.cu"]
OBJDIR = os.path.join(LIBDIR, "obj")
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


def _includes(path: str, seen=None):
    """The file and every project header it includes (#include "..."), transitively."""
    import re
    seen = set() if seen is None else seen
    path = os.path.normpath(path)
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    with open(path) as f:
        for name in re.findall(r'^\s*#\s*include\s+"([^"]+)"', f.read(), re.M):
            _includes(os.path.join(os.path.dirname(path), name), seen)
    return seen


def _stale_objects(force: bool = False):
    """(source, object) pairs whose object is missing or older than the
    source or a header it includes."""
    out = []
    for src in SOURCES:
        obj = os.path.join(OBJDIR, src.replace(".cu", ".o"))
        newest = max(os.path.getmtime(f) for f in _includes(os.path.join(CSRC, src)))
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < newest:
            out.append((src, obj))
    return out


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    if not all(os.path.getmtime(f) <= t for f in _deps()):
        return False
    # objects present (a fresh checkout carries only the library): the library
    # must also be newer than every object and no object may be stale
    if os.path.isdir(OBJDIR):
        objs = [os.path.join(OBJDIR, s.replace(".cu", ".o")) for s in SOURCES]
        if all(os.path.exists(o) for o in objs):
            return not _stale_objects() and all(os.path.getmtime(o) <= t for o in objs)
    return True


CPP_DIR = os.path.join(HERE, "cpp")
CPP_LIB = os.path.join(LIBDIR, "libfrank_b200_cpp.so")


def build_cpp(force: bool = False) -> str:
    """The C++ layer (namespace FRANK over the C ABI) as libfrank_b200_cpp.so,
    linked against libfrank_b200.so next to it."""
    lib = build()
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


def _compile(src: str, obj: str, verbose: bool) -> None:
    cmd = [_nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-diag-suppress", "177",
           "-c", os.path.join(CSRC, src), "-o", obj + ".tmp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed on %s:\n%s%s" % (src, res.stdout, res.stderr))
    os.replace(obj + ".tmp", obj)
    if verbose:
        sys.stdout.write(res.stdout + res.stderr)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile each translation unit to an object under lib/obj (again only when
    it or a header is newer than its object), in parallel, then link."""
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    jobs = _stale_objects(force)
    if jobs:
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
            for f in [ex.submit(_compile, src, obj, verbose) for src, obj in jobs]:
                f.result()
    objs = [os.path.join(OBJDIR, s.replace(".cu", ".o")) for s in SOURCES]
    cmd = [_nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", *objs, "-o", LIB + ".tmp"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + res.stdout + res.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB
