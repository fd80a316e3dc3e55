"""The reference's own sparse_cuda acceptance tests, unchanged, run through
the reference-side binding (asc_cpp_b200/binding/sparse_cuda_provider.cc)
over this library:

* tests/sparse_cuda/standard_blas_cuda_test.cc -- standard SpMV/SpMM, Level-1
  and triangular solves through the public templates of
  include/asc/sparse/providers/cuda.h, against the reference's CPU answers;
* tests/sparse_cuda/sparse_cuda_test.cc -- clones (including a memory
  resource that fails on a chosen allocation), strided and unit-stride
  compat SpMV with the workspace rules, workspace overlap, pointwise
  evaluation, independent contexts on concurrent threads, and failure paths
  that must not mutate outputs;
* tests/consumer/sparse_cuda/main.cc -- the packaged consumer check.

The executables are linked by asc_cpp_b200/binding/build_binding.py from the
reference tree; each must exit 0 (77 means the reference's test skipped for
want of a device)."""

import os
import subprocess

import pytest

from asc_cpp_b200.binding import build_binding

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def executables(cuda_lib):
    exes = build_binding.executables()
    if not all(os.path.exists(p) for p in exes.values()):
        if not build_binding.reference_available():
            pytest.fail("binding executables missing and the reference sources are absent")
        exes = build_binding.build()
    return exes


@pytest.mark.parametrize("name", sorted(build_binding.TESTS))
def test_reference_acceptance_test_passes_through_binding(executables, name):
    res = subprocess.run([executables[name]], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, (
        f"{name} exited {res.returncode}\nstdout:\n{res.stdout[-4000:]}\n"
        f"stderr:\n{res.stderr[-4000:]}")
