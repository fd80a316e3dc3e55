import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def restatement():
    from oracle import Restatement, build_oracle
    build_oracle.build_restatement()
    return Restatement()


@pytest.fixture(scope="session")
def reference():
    from oracle import Reference, build_oracle
    build_oracle.build_reference()
    if not Reference.available():
        pytest.skip("reference harness (oracle/_ref) not built here")
    return Reference()


@pytest.fixture(scope="session")
def known_answers():
    return dict(np.load(os.path.join(GOLDEN, "known_answers.npz")))


@pytest.fixture(scope="session")
def trsv_cases():
    return dict(np.load(os.path.join(GOLDEN, "trsv_cases.npz")))


@pytest.fixture(scope="session")
def level1_cases():
    return dict(np.load(os.path.join(GOLDEN, "level1_cases.npz")))


@pytest.fixture(scope="session")
def complex_cases():
    return dict(np.load(os.path.join(GOLDEN, "complex_cases.npz")))


@pytest.fixture(scope="session")
def conversions():
    return dict(np.load(os.path.join(GOLDEN, "conversions.npz")))


@pytest.fixture(scope="session")
def random_cases():
    return dict(np.load(os.path.join(GOLDEN, "random_cases.npz")))


@pytest.fixture(scope="session")
def laplacian_golden():
    return dict(np.load(os.path.join(GOLDEN, "laplacian.npz")))


@pytest.fixture(scope="session")
def cuda_lib():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from asc_cpp_b200 import _abi
    return _abi.load()


@pytest.fixture()
def ctx(cuda_lib):
    from asc_cpp_b200.sparse_cuda import SparseCudaContext
    c = SparseCudaContext.Create(0)
    yield c
    c.synchronize()
    c.close()
