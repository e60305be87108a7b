"""frank_b200: a B200-native engine for FRANK's BLR-LU factor-and-solve path.

The compute runs in hand-written sm_100a CUDA kernels behind the C ABI of
include/frank_b200.h (libfrank_b200.so, built in-tree by `frank_b200.build`).
`BLRMatrix` mirrors the reference's getrf / trsm / gemm calls for a
block-low-rank matrix resident on one GPU, `HMatrix` for a multi-level
H-matrix (binary cluster tree, weak admissibility, fixed rank).
"""
from .blr import BLRMatrix, split_offsets, upload_hierarchical  # noqa: F401
from .hodlr import HMatrix, upload_hmatrix  # noqa: F401
from ._abi import FrankError, lib  # noqa: F401

__all__ = ["BLRMatrix", "split_offsets", "upload_hierarchical", "HMatrix", "upload_hmatrix", "FrankError", "lib"]
