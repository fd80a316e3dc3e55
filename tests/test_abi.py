"""The C-ABI library loads and exports exactly what include/*.h declares
(no compute call: this runs without a GPU)."""

import ctypes
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        names |= set(re.findall(r"ASC_SB_API\s+[\w\s\*]+?\b(asc_sb_\w+)\s*\(", text))
    return names


@pytest.fixture(scope="module")
def lib_path():
    from asc_cpp_b200 import _abi, build
    if not os.path.exists(_abi.LIB_PATH):
        build.build()
    return _abi.LIB_PATH


def test_header_declares_entry_points():
    names = _declared()
    for required in ("asc_sb_context_create", "asc_sb_csr_spmv",
                     "asc_sb_csr_spmv_workspace_size", "asc_sb_standard_spmv",
                     "asc_sb_standard_spmm"):
        assert required in names


def test_library_exports_every_declared_symbol(lib_path):
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    declared = _declared()
    assert declared <= exported, declared - exported
    # nothing beyond the declared C ABI leaks out of the library
    assert {e for e in exported if e.startswith("asc")} == declared


def test_ctypes_binding_covers_header(lib_path):
    from asc_cpp_b200 import _abi
    lib = _abi.load()
    assert set(_abi.SIGNATURES) == _declared()
    for name in _abi.SIGNATURES:
        assert isinstance(getattr(lib, name), ctypes._CFuncPtr)


def test_descriptor_layouts_match_header():
    """Struct sizes/offsets seen by ctypes equal those the C compiler sees."""
    from asc_cpp_b200 import _abi
    src = r'''
#include <stddef.h>
#include <stdio.h>
#include "asc_sparse_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(asc_sb_sparse),
         sizeof(asc_sb_vector), sizeof(asc_sb_dense), offsetof(asc_sb_sparse, rows),
         offsetof(asc_sb_vector, extent), offsetof(asc_sb_dense, leading_dimension),
         offsetof(asc_sb_dense, writable), sizeof(asc_sb_indexed_vector),
         offsetof(asc_sb_indexed_vector, dense_extent), sizeof(asc_sb_tensor),
         offsetof(asc_sb_tensor, extents), sizeof(asc_sb_operand),
         offsetof(asc_sb_operand, scalar));
  return 0;
}
'''
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I" + os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        got = [int(v) for v in subprocess.run([exe], capture_output=True, text=True,
                                              check=True).stdout.split()]
    want = [ctypes.sizeof(_abi.SparseDesc), ctypes.sizeof(_abi.VectorDesc),
            ctypes.sizeof(_abi.DenseDesc), _abi.SparseDesc.rows.offset,
            _abi.VectorDesc.extent.offset, _abi.DenseDesc.leading_dimension.offset,
            _abi.DenseDesc.writable.offset, ctypes.sizeof(_abi.IndexedDesc),
            _abi.IndexedDesc.dense_extent.offset, ctypes.sizeof(_abi.TensorDesc),
            _abi.TensorDesc.extents.offset, ctypes.sizeof(_abi.OperandDesc),
            _abi.OperandDesc.scalar.offset]
    assert got == want


def test_enum_values_match_reference_numbering():
    from asc_cpp_b200 import _abi
    assert _abi.ErrorCode.kMemoryAccess == 7 and _abi.ErrorCode.kProvider == 11
    assert _abi.MemorySpace.kDevice == 2
    assert _abi.SparseBlasTranspose.kConjugateTranspose == 2
    assert _abi.SparseBlasLayout.kRowMajor == 1
    assert _abi.Determinism.kBackendDefault == 1


def test_null_arguments_return_error_codes(lib_path):
    """Every entry point called with a null context and null descriptors
    returns an error code (or, for the destroy calls, succeeds as a no-op)
    instead of dereferencing anything: host logic, no device needed."""
    from asc_cpp_b200 import _abi
    lib = _abi.load()
    no_op = {"asc_sb_context_destroy", "asc_sb_plan_destroy", "asc_sb_batch_destroy"}
    for name, (restype, argtypes) in _abi.SIGNATURES.items():
        args = []
        for t in argtypes:
            if t in (ctypes.c_double, ctypes.c_float):
                args.append(t(0.0))
            elif t in (ctypes.c_int32, ctypes.c_int64, ctypes.c_size_t):
                args.append(t(0))
            else:
                args.append(None)
        r = getattr(lib, name)(*args)
        if name in no_op:
            assert r == _abi.ErrorCode.kOk, name
        elif name == "asc_sb_context_stream":
            assert r is None
        elif name == "asc_sb_context_last_error":
            assert r  # a message, not a crash
        elif name == "asc_sb_context_launch_count":
            assert r == 0
        elif name == "asc_sb_selector_param_count":
            assert r < 0  # zero variants is not a network
        else:
            assert r in (_abi.ErrorCode.kInvalidArgument, _abi.ErrorCode.kInvalidState), (name, r)


def test_context_without_a_device_is_unavailable(lib_path):
    """On a host without a CUDA device the context cannot be created and the
    call says so (ASC_SB_UNAVAILABLE) rather than failing later."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from asc_cpp_b200 import _abi
    lib = _abi.load()
    ctx = ctypes.c_void_p()
    assert lib.asc_sb_context_create(0, None, ctypes.byref(ctx)) == _abi.ErrorCode.kUnavailable
    assert not ctx.value
