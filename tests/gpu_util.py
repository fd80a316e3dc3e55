"""Helpers shared by the GPU parity tests (device staging, error bounds)."""

from __future__ import annotations

import numpy as np
import torch

from asc_cpp_b200.sparse_cuda import (CudaCsrArray, CudaStridedVectorView,
                                      SparseCudaContext)
from asc_cpp_b200._abi import Determinism, FormatKind


def context(determinism=Determinism.kDeterministic) -> SparseCudaContext:
    # The legacy default stream orders the library's kernels with torch's
    # uploads and downloads, so the tests need no extra synchronisation.
    return SparseCudaContext.Create(0, stream=torch.cuda.default_stream(0),
                                    determinism=determinism)


def dev(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def csr(rows, cols, ptr, idx, val, fmt=FormatKind.kCsr) -> CudaCsrArray:
    return CudaCsrArray(rows, cols, dev(np.asarray(ptr, np.int64)),
                        dev(np.asarray(idx, np.int64)), dev(np.asarray(val)), fmt)


def vec(t: torch.Tensor, extent=None, stride=1, offset=0, writable=True):
    return CudaStridedVectorView(t, t.numel() if extent is None else extent, stride,
                                 offset, writable)


def host(t: torch.Tensor) -> np.ndarray:
    torch.cuda.synchronize()
    return t.cpu().numpy()


def bits_equal(a, b) -> bool:
    a = np.asarray(a)
    b = np.asarray(b)
    return a.dtype == b.dtype and a.shape == b.shape and a.tobytes() == b.tobytes()


def gamma(n: np.ndarray, dtype) -> np.ndarray:
    u = np.finfo(dtype).eps / 2
    n = np.asarray(n, np.float64)
    return n * u / (1 - n * u)


def assert_within_bound(y, exact, absval, counts, dtype, alpha, beta_term_abs,
                        reference_value):
    """|y - ref| <= gamma_{n+2} * (|alpha| sum|v x| + |beta y0|) (+ one ulp of
    the tiniest normal, to admit exact zeros)."""
    g = gamma(counts + 2, dtype)
    bound = g * (abs(alpha) * np.asarray(absval, np.float64) + beta_term_abs)
    bound = bound + np.finfo(dtype).tiny
    # in long double: the reference is not rounded to the output type first
    err = np.abs(np.asarray(y, np.longdouble) -
                 np.asarray(reference_value, np.longdouble)).astype(np.float64)
    bad = np.nonzero(err > bound)[0]
    assert bad.size == 0, (
        f"{bad.size} outputs outside the bound; first {bad[:5]}: err {err[bad[:5]]} "
        f"bound {bound[bad[:5]]}")
    return float(np.max(err / np.maximum(bound, np.finfo(np.float64).tiny)))
