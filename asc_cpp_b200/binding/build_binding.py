"""Build recipe for the reference-side binding and the reference's own
acceptance tests run through it.

``sparse_cuda_provider.cc`` implements the exported surface of the
reference's sparse_cuda provider over ``libasc_sparse_b200.so``.  This script
compiles it against the reference's unchanged public headers and core
internals, together with the reference's own core sources (execution
contexts, memory resources, status) and, for the one test that draws its
inputs from the reference's random module, that module's sparse CUDA
generator -- all straight from the reference tree, the way a maintainer would
build the provider in place.  It then links, unchanged, the reference's

* ``tests/sparse_cuda/standard_blas_cuda_test.cc``,
* ``tests/sparse_cuda/sparse_cuda_test.cc``,
* ``tests/consumer/sparse_cuda/main.cc``

against the binding and this library.  The executables land in
``asc_cpp_b200/binding/_ref/`` (git-ignored; they travel with the working
tree like the other built libraries and find ``libasc_sparse_b200.so``
through an ``$ORIGIN`` run path).  Test infrastructure only: nothing in the
library depends on it.
"""

from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
REFERENCE_ROOT = os.environ.get("ASC_REFERENCE_ROOT", "/root/reference")
OUT = os.path.join(HERE, "_ref")
OBJ = os.path.join(OUT, "obj")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")

TESTS = {
    "standard_blas_cuda_test": "tests/sparse_cuda/standard_blas_cuda_test.cc",
    "sparse_cuda_test": "tests/sparse_cuda/sparse_cuda_test.cc",
    "consumer_sparse_cuda": "tests/consumer/sparse_cuda/main.cc",
}


def executables() -> dict[str, str]:
    return {name: os.path.join(OUT, name) for name in TESTS}


def reference_available() -> bool:
    return all(os.path.isfile(os.path.join(REFERENCE_ROOT, t)) for t in TESTS.values())


def _includes() -> list[str]:
    return ["-I" + os.path.join(REFERENCE_ROOT, "include"),
            "-I" + os.path.join(REFERENCE_ROOT, "src"),
            "-I" + os.path.join(ROOT, "include"),
            "-I" + os.path.join(CUDA, "include")]


def _compile(src: str, tag: str) -> str:
    obj = os.path.join(OBJ, tag + "_" + os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src):
        return obj
    if src.endswith(".cu"):
        cmd = [NVCC, "-std=c++20", "-O2", "-Xcompiler", "-fPIC", "-w",
               "-gencode", "arch=compute_100a,code=sm_100a"] + _includes()
    else:
        cmd = ["g++", "-std=c++20", "-O2", "-fPIC", "-w"] + _includes()
    subprocess.run(cmd + ["-c", src, "-o", obj], check=True)
    return obj


def build(force: bool = False) -> dict[str, str] | None:
    """Builds the three executables; returns their paths, or None where the
    reference sources are absent."""
    if not reference_available():
        return None
    os.makedirs(OBJ, exist_ok=True)
    if force:
        for o in glob.glob(os.path.join(OBJ, "*.o")):
            os.remove(o)
    ref = lambda *p: os.path.join(REFERENCE_ROOT, *p)  # noqa: E731
    core = sorted(glob.glob(ref("src", "core", "*.cc"))) + [ref("src", "core", "cuda",
                                                                "runtime.cc")]
    random = sorted(glob.glob(ref("src", "random", "*.cc"))) + [
        ref("src", "random", "cuda", "sparse.cc"), ref("src", "random", "cuda",
                                                       "sparse_kernels.cu")]
    jobs = ([(s, "core") for s in core] + [(s, "random") for s in random] +
            [(os.path.join(HERE, "sparse_cuda_provider.cc"), "binding")] +
            [(ref(t), "test") for t in TESTS.values()])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = dict(zip([s for s, _ in jobs], ex.map(lambda j: _compile(*j), jobs)))
    common = [objs[os.path.join(HERE, "sparse_cuda_provider.cc")]] + [objs[s] for s in core]
    lib_dir = PKG
    out = {}
    for name, test in TESTS.items():
        exe = os.path.join(OUT, name)
        extra = [objs[s] for s in random] if name == "sparse_cuda_test" else []
        inputs = [objs[ref(test)]] + common + extra + [os.path.join(lib_dir,
                                                                    "libasc_sparse_b200.so")]
        if force or not os.path.exists(exe) or any(
                os.path.getmtime(i) > os.path.getmtime(exe) for i in inputs):
            subprocess.run(["g++", "-o", exe, objs[ref(test)]] + common + extra +
                           ["-L" + lib_dir, "-lasc_sparse_b200",
                            "-Wl,-rpath,$ORIGIN/../..",
                            "-L" + os.path.join(CUDA, "lib64"), "-lcudart_static", "-ldl",
                            "-lrt", "-lpthread"], check=True)
        out[name] = exe
    return out


if __name__ == "__main__":
    built = build(force="--force" in sys.argv)
    print(built if built is not None else "(reference sources absent: nothing built)")
