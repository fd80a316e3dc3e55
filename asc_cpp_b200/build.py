"""Build ``libasc_sparse_b200.so`` in-tree with nvcc for sm_100a.

All CUDA sources (``csrc/*.cu``) and the C++20 host library
(``csrc/host/*.cc``) are compiled by nvcc into one shared library next to this
file.  Only the symbols declared in ``include/asc_sparse_b200.h`` are exported
(``-fvisibility=hidden``).  The CUDA runtime is linked statically, so the
library loads in any process, with or without torch.
"""

from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libasc_sparse_b200.so")
# measurement-only kernels (bench.py's gather-floor workload), a library of their own
PROBE_SRC = os.path.join(CSRC, "probe", "gather_floor.cu")
PROBE_LIB = os.path.join(HERE, "libasc_gather_probe.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++20", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
          "-Xcompiler", "-fvisibility=hidden", "-I" + os.path.join(ROOT, "include")]


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) +
                  glob.glob(os.path.join(CSRC, "host", "*.cc")))


def _headers() -> list[str]:
    return (glob.glob(os.path.join(CSRC, "*.h")) +
            glob.glob(os.path.join(CSRC, "*.cuh")) +
            glob.glob(os.path.join(CSRC, "host", "*.h")) +
            glob.glob(os.path.join(CSRC, "host", "*.inc")) +
            glob.glob(os.path.join(ROOT, "include", "*.h")))


def _object(src: str) -> str:
    rel = os.path.relpath(src, CSRC).replace(os.sep, "_")
    return os.path.join(BUILD, rel + ".o")


def _compile(src: str, newest_header: float, verbose: bool) -> str:
    obj = _object(src)
    if (os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
            and os.path.getmtime(obj) >= newest_header):
        return obj
    cmd = [NVCC] + COMMON + ARCH + ["-c", src, "-o", obj]
    if src.endswith(".cu") and verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr:
        sys.stderr.write(res.stderr)
    return obj


def build(force: bool = False, verbose: bool = False, out: str | None = None,
          defines: list[str] | None = None) -> str:
    """Build the library (default: in-tree).  ``out``/``defines`` build an
    experimental copy elsewhere with extra -D flags (own object directory)."""
    global BUILD, COMMON
    if out is not None:
        saved = (BUILD, COMMON)
        BUILD = os.path.join(os.path.dirname(os.path.abspath(out)), "_objs_" +
                             os.path.basename(out).replace(".", "_"))
        COMMON = COMMON + ["-D" + d for d in (defines or [])]
        try:
            return _build(force, verbose, out)
        finally:
            BUILD, COMMON = saved
    lib = _build(force, verbose, LIB)
    build_probe(force)
    return lib


def build_probe(force: bool = False) -> str:
    """The gather-floor probe library (not part of the Sparse BLAS library)."""
    if (not force and os.path.exists(PROBE_LIB) and
            os.path.getmtime(PROBE_LIB) >= os.path.getmtime(PROBE_SRC)):
        return PROBE_LIB
    cmd = [NVCC] + COMMON + ARCH + ["-shared", PROBE_SRC, "-o", PROBE_LIB]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {PROBE_SRC}:\n{res.stdout}\n{res.stderr}")
    return PROBE_LIB


def _build(force: bool, verbose: bool, lib: str) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    newest_header = max((os.path.getmtime(h) for h in _headers()), default=0.0)
    if force:
        for s in srcs:
            o = _object(s)
            if os.path.exists(o):
                os.remove(o)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, newest_header, verbose), srcs))
    if (force or not os.path.exists(lib) or
            any(os.path.getmtime(o) > os.path.getmtime(lib) for o in objs)):
        cmd = [NVCC] + ARCH + ["-shared", "-o", lib] + objs
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc link failed:\n{res.stdout}\n{res.stderr}")
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
