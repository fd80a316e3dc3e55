"""ctypes declarations of the C ABI in ``include/asc_sparse_b200.h``.

The structs below are field-for-field copies of the header's descriptor
structs; ``load()`` binds every exported entry point with its exact argument
types.  Loading fails loudly when the CUDA library has not been built -- there
is no fallback implementation behind this module.
"""

from __future__ import annotations

import ctypes
import os
from enum import IntEnum

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libasc_sparse_b200.so")


class ErrorCode(IntEnum):
    """asc::ErrorCode (include/asc/core/status.h:35-55)."""
    kOk = 0
    kInvalidArgument = 1
    kShape = 2
    kIndex = 3
    kOverflow = 4
    kInvalidState = 5
    kAllocation = 6
    kMemoryAccess = 7
    kMemoryTransfer = 8
    kUnsupported = 9
    kUnavailable = 10
    kProvider = 11
    kNumerical = 12
    kInternal = 18


class MemorySpace(IntEnum):
    kHost = 0
    kPinnedHost = 1
    kDevice = 2
    kManaged = 3


class ElementKind(IntEnum):
    kFloat = 0
    kDouble = 1
    kComplexFloat = 2
    kComplexDouble = 3


class FormatKind(IntEnum):
    kCoordinate = 0
    kCsr = 1
    kCsc = 2


class SparseBlasTranspose(IntEnum):
    kNone = 0
    kTranspose = 1
    kConjugateTranspose = 2


class SparseBlasLayout(IntEnum):
    kColumnMajor = 0
    kRowMajor = 1


class Determinism(IntEnum):
    kDeterministic = 0
    kBackendDefault = 1


class Variant(IntEnum):
    kAuto = -1
    kRowOrdered = 0
    kVector = 1
    kWarpTiles = 2
    kMergePath = 3
    kRowSplit = 4


PLAN_TRANSPOSE = 1
PLAN_TRIANGULAR = 2
PLAN_ROW_GROUPS = 4
PLAN_HAS_TRANSPOSE = 1
PLAN_HAS_BLOCKS16 = 2
PLAN_HAS_ROW_GROUPS = 4
PLAN_HAS_STAGED_SPMM = 8
SPMM_STAGED = -1  # the TMA-staged SpMM kernel (autotune result, set_spmm choice)
SPMM_AUTO = -2    # asc_sb_plan_set_spmm: the plan's default rules


class SparseDesc(ctypes.Structure):
    _fields_ = [("structure_first", ctypes.c_void_p),
                ("structure_second", ctypes.c_void_p),
                ("values", ctypes.c_void_p),
                ("memory_space", ctypes.c_int32),
                ("element_kind", ctypes.c_int32),
                ("format", ctypes.c_int32),
                ("canonical_structure_trusted", ctypes.c_int32),
                ("rows", ctypes.c_int64),
                ("columns", ctypes.c_int64),
                ("nonzeros", ctypes.c_int64)]


class TensorDesc(ctypes.Structure):
    """asc_sb_tensor: a sparse descriptor of any rank (pointwise evaluation)."""
    _fields_ = [("structure_first", ctypes.c_void_p),
                ("structure_second", ctypes.c_void_p),
                ("values", ctypes.c_void_p),
                ("memory_space", ctypes.c_int32),
                ("element_kind", ctypes.c_int32),
                ("format", ctypes.c_int32),
                ("canonical_structure_trusted", ctypes.c_int32),
                ("rank", ctypes.c_int64),
                ("extents", ctypes.POINTER(ctypes.c_int64)),
                ("nonzeros", ctypes.c_int64)]


class OperandDesc(ctypes.Structure):
    """asc_sb_operand: a view with the destination's structure, or a scalar."""
    _fields_ = [("kind", ctypes.c_int32),
                ("reserved", ctypes.c_int32),
                ("view", TensorDesc),
                ("scalar", ctypes.c_double)]


class VectorDesc(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p),
                ("reachable_data", ctypes.c_void_p),
                ("reachable_size", ctypes.c_size_t),
                ("memory_space", ctypes.c_int32),
                ("element_kind", ctypes.c_int32),
                ("extent", ctypes.c_int64),
                ("stride", ctypes.c_int64),
                ("writable", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class DenseDesc(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p),
                ("reachable_data", ctypes.c_void_p),
                ("reachable_size", ctypes.c_size_t),
                ("memory_space", ctypes.c_int32),
                ("element_kind", ctypes.c_int32),
                ("rows", ctypes.c_int64),
                ("columns", ctypes.c_int64),
                ("leading_dimension", ctypes.c_int64),
                ("layout", ctypes.c_int32),
                ("writable", ctypes.c_int32)]


class IndexedDesc(ctypes.Structure):
    _fields_ = [("indices", ctypes.c_void_p),
                ("values", ctypes.c_void_p),
                ("memory_space", ctypes.c_int32),
                ("element_kind", ctypes.c_int32),
                ("nonzeros", ctypes.c_int64),
                ("dense_extent", ctypes.c_int64),
                ("writable", ctypes.c_int32),
                ("canonical_structure_trusted", ctypes.c_int32)]


class SparseBlasTriangle(IntEnum):
    """asc::SparseBlasTriangle (include/asc/sparse/blas.h:117-120)."""
    kUpper = 0
    kLower = 1


class SparseBlasDiagonal(IntEnum):
    """asc::SparseBlasDiagonal (include/asc/sparse/blas.h:131-134)."""
    kNonUnit = 0
    kUnit = 1


class Level1Op(IntEnum):
    kDot = 0
    kAxpy = 1
    kGather = 2
    kGatherZero = 3
    kScatter = 4


_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_D = ctypes.c_double
_SZ = ctypes.c_size_t
_SP = ctypes.POINTER(SparseDesc)
_VP = ctypes.POINTER(VectorDesc)
_DP = ctypes.POINTER(DenseDesc)

# name -> (restype, argtypes)
SIGNATURES: dict[str, tuple] = {
    "asc_sb_context_create": (ctypes.c_int, [_I32, _P, ctypes.POINTER(_P)]),
    "asc_sb_context_destroy": (ctypes.c_int, [_P]),
    "asc_sb_context_set_determinism": (ctypes.c_int, [_P, _I32]),
    "asc_sb_context_set_variant": (ctypes.c_int, [_P, _I32, _I32]),
    "asc_sb_context_set_wait_limit": (ctypes.c_int, [_P, _I64]),
    "asc_sb_context_set_allocator": (ctypes.c_int, [_P, _P, _P, _P]),
    "asc_sb_context_stream": (_P, [_P]),
    "asc_sb_context_synchronize": (ctypes.c_int, [_P]),
    "asc_sb_context_last_error": (ctypes.c_char_p, [_P]),
    "asc_sb_context_launch_count": (ctypes.c_int64, [_P]),
    "asc_sb_context_device_status": (ctypes.c_int, [_P, ctypes.POINTER(_I32), _I32]),
    "asc_sb_csr_spmv_workspace_size": (ctypes.c_int, [_P, _SP, _VP, _VP, ctypes.POINTER(_SZ)]),
    "asc_sb_csr_spmv": (ctypes.c_int, [_P, _D, _SP, _VP, _D, _VP, _P, _SZ, _I32]),
    "asc_sb_csr_spmv_no_alloc": (ctypes.c_int, [_P, _D, _SP, _VP, _D, _VP]),
    "asc_sb_standard_spmv": (ctypes.c_int, [_P, _I32, _D, _D, _SP, _VP, _VP]),
    "asc_sb_standard_spmm": (ctypes.c_int, [_P, _I32, _D, _D, _SP, _DP, _DP]),
    "asc_sb_plan_workspace_size": (ctypes.c_int, [_P, _SP, _I32, ctypes.POINTER(_SZ)]),
    "asc_sb_plan_create": (ctypes.c_int, [_P, _SP, _I32, _P, _SZ, ctypes.POINTER(_P)]),
    "asc_sb_plan_refresh_values": (ctypes.c_int, [_P, _P]),
    "asc_sb_plan_destroy": (ctypes.c_int, [_P]),
    "asc_sb_plan_csr_spmv": (ctypes.c_int, [_P, _P, _D, _VP, _D, _VP]),
    "asc_sb_plan_standard_spmv": (ctypes.c_int, [_P, _P, _I32, _D, _D, _VP, _VP]),
    "asc_sb_plan_standard_spmm": (ctypes.c_int, [_P, _P, _I32, _D, _D, _DP, _DP]),
    "asc_sb_plan_spmm_autotune": (ctypes.c_int, [_P, _P, _D, _DP, _DP, _I32,
                                                 ctypes.POINTER(ctypes.c_float),
                                                 ctypes.POINTER(_I32)]),
    "asc_sb_plan_set_spmm": (ctypes.c_int, [_P, _P, _I32]),
    "asc_sb_plan_spmm_stage_rows": (ctypes.c_int, [_P, _P, ctypes.c_int64,
                                                   ctypes.POINTER(ctypes.c_int64)]),
    "asc_sb_plan_spmm_tuning": (ctypes.c_int, [_P, _I32, ctypes.POINTER(_I32),
                                               ctypes.POINTER(_I32),
                                               ctypes.POINTER(ctypes.c_float)]),
    "asc_sb_standard_triangular_solve": (ctypes.c_int, [_P, _I32, _D, _D, _SP, _I32, _I32,
                                                        _DP]),
    "asc_sb_plan_triangular_solve": (ctypes.c_int, [_P, _P, _I32, _D, _D, _I32, _I32, _DP]),
    "asc_sb_plan_triangular_analysis": (ctypes.c_int, [_P, _P, _I32, _I32]),
    "asc_sb_clone_csr": (ctypes.c_int, [_P, _SP, _SP]),
    "asc_sb_clone_indexed": (ctypes.c_int, [_P, ctypes.POINTER(IndexedDesc),
                                            ctypes.POINTER(IndexedDesc)]),
    "asc_sb_standard_level1": (ctypes.c_int, [_P, _I32, _I32, _D, _D,
                                              ctypes.POINTER(IndexedDesc), _VP, _VP]),
    "asc_sb_selector_param_count": (ctypes.c_int64, [_I32]),
    "asc_sb_context_set_selector": (ctypes.c_int, [_P, _I32, _P, _P, _P]),
    "asc_sb_plan_properties": (ctypes.c_int, [_P, ctypes.POINTER(_I32)]),
    "asc_sb_plan_variant": (ctypes.c_int, [_P, ctypes.POINTER(_I32), ctypes.POINTER(_I32)]),
    "asc_sb_plan_autotune": (ctypes.c_int, [_P, _P, _VP, _VP, _I32, _P, _P, _I32, _P]),
    "asc_sb_matrix_features": (ctypes.c_int, [_P, _SP, _P, _P]),
    "asc_sb_selector_forward": (ctypes.c_int, [_P, _I32, _P, _P, _I64, _P, _P]),
    "asc_sb_selector_backward": (ctypes.c_int, [_P, _I32, _P, _P, _I64, _P, _P, _P, _P, _P,
                                                _P]),
    "asc_sb_selector_adam": (ctypes.c_int, [_P, _P, _P, _P, _P, _I64, ctypes.c_float,
                                            ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                            _I32]),
    "asc_sb_batch_workspace_size": (ctypes.c_int, [_P, _I64, _SP, ctypes.POINTER(_SZ)]),
    "asc_sb_batch_create": (ctypes.c_int, [_P, _I64, _SP, _VP, _VP, _P, _SZ,
                                           ctypes.POINTER(_P)]),
    "asc_sb_batch_destroy": (ctypes.c_int, [_P]),
    "asc_sb_batch_set_schedule": (ctypes.c_int, [_P, _P, _I32, _I32]),
    "asc_sb_batch_get_schedule": (ctypes.c_int, [_P, ctypes.POINTER(_I32),
                                                 ctypes.POINTER(_I32)]),
    "asc_sb_batch_spmv": (ctypes.c_int, [_P, _P, _D, _D]),
    "asc_sb_batch_spmv_per_matrix": (ctypes.c_int, [_P, _P, _D, _D]),
    "asc_sb_batch_capture": (ctypes.c_int, [_P, _P, _D, _D]),
    "asc_sb_batch_autotune": (ctypes.c_int, [_P, _P, _D, _D, _I32,
                                             ctypes.POINTER(ctypes.c_float)]),
    "asc_sb_convert_workspace_size": (ctypes.c_int, [_P, _I64, _I64, _I64, _I32,
                                                     ctypes.POINTER(_SZ)]),
    "asc_sb_convert_compressed": (ctypes.c_int, [_P, _SP, _SP, _P, _SZ]),
    "asc_sb_convert_coordinates": (ctypes.c_int, [_P, _P, _P, _I32, _I64, _I64, _I64, _SP,
                                                  _P, _SZ]),
    "asc_sb_sparse_storage_bytes": (ctypes.c_int, [_P, _SP, ctypes.POINTER(_SZ),
                                                   ctypes.POINTER(_SZ), ctypes.POINTER(_SZ)]),
    "asc_sb_indexed_storage_bytes": (ctypes.c_int, [_P, ctypes.POINTER(IndexedDesc),
                                                    ctypes.POINTER(_SZ), ctypes.POINTER(_SZ)]),
    "asc_sb_evaluate": (ctypes.c_int, [_P, _I32, ctypes.POINTER(OperandDesc),
                                       ctypes.POINTER(OperandDesc), ctypes.POINTER(TensorDesc)]),
}

_lib: ctypes.CDLL | None = None


def load(path: str | None = None) -> ctypes.CDLL:
    """Load and bind the CUDA library; raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    path = path or os.environ.get("ASC_SB_LIBRARY") or LIB_PATH
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python asc_cpp_b200/build.py` "
            "(there is no non-CUDA implementation of this library)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
