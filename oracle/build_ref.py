"""TEST INFRASTRUCTURE ONLY.  Build recipe of oracle/_ref: the reference's own
C++ sources (FRANK src/**/*.cpp, unmodified, read where they lie) plus the
driver oracle/ref_driver.cpp, compiled with the system g++ into
oracle/_ref/frank_ref.  No reference build system is run.

What stands in for the reference's external dependencies:
* yomm2 (absent here): oracle/ref_shim/yorel/yomm2/cute.hpp, which maps
  yomm2's macros onto the engine's own multimethod layer
  (frank_b200/cpp/include/frank_b200/multimethod.hpp);
* CBLAS / LAPACKE (absent here): oracle/ref_shim/cblas.h and lapacke.h,
  standard prototypes resolved to the "scipy_"-prefixed exports of the
  OpenBLAS library bundled with scipy (linked with an rpath);
* nlohmann/json (used by util/print.cpp): the copy that ships inside an
  installed pip package, found by searching site-packages.

Usage: python oracle/build_ref.py [--reference DIR] [--jobs N]
(DIR defaults to $FRANK_REFERENCE or /root/reference).  Object files are
cached under oracle/_ref/obj and rebuilt when their source is newer.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")
EXE = os.path.join(OUT, "frank_ref")
SHIM = os.path.join(HERE, "ref_shim")
MM_INCLUDE = os.path.join(ROOT, "frank_b200", "cpp", "include")


def openblas_lib() -> str:
    import scipy
    libs = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    cands = sorted(glob.glob(os.path.join(libs, "libscipy_openblas*.so")))
    if not cands:
        raise RuntimeError("scipy's bundled OpenBLAS not found under " + libs)
    return cands[0]


def json_include() -> str:
    site = sysconfig.get_paths()["purelib"]
    for path in glob.glob(os.path.join(site, "**", "nlohmann", "json.hpp"), recursive=True):
        return os.path.dirname(os.path.dirname(path))
    raise RuntimeError("nlohmann/json.hpp not found under " + site)


def _compile(args):
    src, obj, flags = args
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _shim_mtime()):
        return obj, ""
    res = subprocess.run(["g++", *flags, "-c", src, "-o", obj], capture_output=True, text=True)
    if res.returncode != 0:
        return None, res.stderr
    return obj, ""


def _shim_mtime() -> float:
    files = glob.glob(os.path.join(SHIM, "**", "*"), recursive=True) + [os.path.join(MM_INCLUDE, "frank_b200", "multimethod.hpp")]
    return max(os.path.getmtime(f) for f in files if os.path.isfile(f))


def build(reference: str, jobs: int = 0) -> str:
    os.makedirs(os.path.join(OUT, "obj"), exist_ok=True)
    flags = ["-std=c++17", "-O2", "-I" + os.path.join(reference, "include"), "-I" + SHIM, "-I" + MM_INCLUDE,
             "-I" + json_include()]
    srcs = sorted(glob.glob(os.path.join(reference, "src", "**", "*.cpp"), recursive=True))
    if not srcs:
        raise RuntimeError("no FRANK sources under " + reference)
    srcs.append(os.path.join(HERE, "ref_driver.cpp"))
    work = []
    for s in srcs:
        rel = os.path.relpath(s, reference) if s.startswith(reference) else "driver/" + os.path.basename(s)
        work.append((s, os.path.join(OUT, "obj", rel.replace(os.sep, "_") + ".o"), flags))
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count()) as ex:
        results = list(ex.map(_compile, work))
    errs = [e for o, e in results if o is None]
    if errs:
        raise RuntimeError("g++ failed:\n" + "\n".join(errs)[:4000])
    lib = openblas_lib()
    cmd = ["g++", "-o", EXE, *[o for o, _ in results], lib, "-Wl,-rpath," + os.path.dirname(lib), "-lpthread"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("link failed:\n" + res.stderr[:4000])
    return EXE


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("FRANK_REFERENCE", "/root/reference"))
    ap.add_argument("--jobs", type=int, default=0)
    a = ap.parse_args()
    print(build(a.reference, a.jobs))
