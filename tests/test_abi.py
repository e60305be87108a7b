"""CPU tests of the boundary: the sm_100a library builds, loads without a
GPU, and exports every entry point include/frank_b200.h declares; the ctypes
descriptor matches the C struct; host geometry helpers match the oracle."""
import ctypes as C
import os
import re

import numpy as np

import oracle.frank_oracle as fo

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            names |= set(re.findall(r"^\s*(?:const\s+)?\w[\w\s\*]*?\b(frank_\w+)\s*\(", txt, re.M))
    return names


def test_library_exports_every_declared_symbol():
    from frank_b200 import build
    path = build.build()
    h = C.CDLL(path)
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(h, n)]
    assert not missing, missing
    from frank_b200._abi import SIGNATURES
    assert set(SIGNATURES) == names


def test_library_is_sm100a():
    from frank_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)


def test_desc_layout():
    from frank_b200._abi import BlrDesc
    assert C.sizeof(BlrDesc) == 40
    assert BlrDesc.eps.offset == 24 and BlrDesc.admis.offset == 32


def test_split_offsets_match_index_range():
    from frank_b200.blr import split_offsets
    for n, nb in [(2048, 8), (10, 3), (32768, 64), (1000, 7)]:
        off = split_offsets(n, nb)
        want = [s for s, _ in fo.split_range(0, n, nb)] + [n]
        assert list(off) == want


def test_no_oracle_in_product():
    """The product never imports or links the oracle."""
    for root, _, files in os.walk(os.path.join(ROOT, "frank_b200")):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
                txt = open(os.path.join(root, f)).read()
                assert "oracle" not in txt.replace("oracle is the oracle", ""), f
