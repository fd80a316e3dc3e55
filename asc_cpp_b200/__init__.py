"""B200-native Sparse BLAS hot path (CSR/CSC SpMV and SpMM) for ASCCpp.

The compute lives in ``libasc_sparse_b200.so`` (hand-written sm_100a kernels
behind the C ABI in ``include/asc_sparse_b200.h``).  This package holds the
build recipe, the ctypes binding and a Python mirror of the reference's
``sparse_cuda`` facet.  Importing it does not need a GPU; calling it does.
"""

from . import _abi  # noqa: F401
from ._abi import (Determinism, ElementKind, ErrorCode, FormatKind,  # noqa: F401
                   MemorySpace, SparseBlasLayout, SparseBlasTranspose, Variant)

__all__ = ["Determinism", "ElementKind", "ErrorCode", "FormatKind",
           "MemorySpace", "SparseBlasLayout", "SparseBlasTranspose", "Variant"]
