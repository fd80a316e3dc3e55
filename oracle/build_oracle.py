"""Build recipe for the CPU oracle (test infrastructure, never the product).

Two shared libraries come out of this script:

* ``oracle/liboracle.so`` - the hand-written C restatement in
  ``oracle/sparse_oracle.c``.  Built from this repository alone, so it can be
  rebuilt anywhere gcc exists.
* ``oracle/_ref/libasc_ref.so`` - the reference's own serial Sparse BLAS
  (``src/sparse/reference_blas.cc`` plus the header templates and
  ``src/core/*.cc``) compiled straight from the reference tree, wrapped by
  ``oracle/ref_harness.cc``.  Only built where the reference sources are
  present; the output directory is git-ignored and travels with the
  working tree like any other built library.

Both are compiled with ``-O2`` and no ``-march`` flag, matching the reference's
own x86-64 build, so no fused multiply-add is emitted (``-ffp-contract=off``
makes that explicit for the restatement).
"""

from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REFERENCE_ROOT = os.environ.get("ASC_REFERENCE_ROOT", "/root/reference")
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_SO = os.path.join(REF_DIR, "libasc_ref.so")


def _run(cmd: list[str]) -> None:
    subprocess.run(cmd, check=True)


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_restatement(force: bool = False) -> str:
    src = os.path.join(HERE, "sparse_oracle.c")
    if force or _stale(ORACLE_SO, [src]):
        _run(["gcc", "-std=c11", "-O2", "-ffp-contract=off", "-fPIC", "-shared",
              "-Wall", "-Wextra", "-o", ORACLE_SO, src, "-lm", "-lpthread"])
    return ORACLE_SO


def reference_available() -> bool:
    return os.path.isfile(os.path.join(REFERENCE_ROOT, "src", "sparse",
                                       "reference_blas.cc"))


def build_reference(force: bool = False) -> str | None:
    if not reference_available():
        return REF_SO if os.path.exists(REF_SO) else None
    harness = os.path.join(HERE, "ref_harness.cc")
    sources = [harness, os.path.join(REFERENCE_ROOT, "src", "sparse",
                                     "reference_blas.cc")]
    sources += sorted(glob.glob(os.path.join(REFERENCE_ROOT, "src", "core",
                                             "*.cc")))
    if force or _stale(REF_SO, sources):
        os.makedirs(REF_DIR, exist_ok=True)
        _run(["g++", "-std=c++20", "-O2", "-fPIC", "-shared", "-w",
              "-I" + os.path.join(REFERENCE_ROOT, "include"),
              "-o", REF_SO] + sources + ["-lpthread"])
    return REF_SO


def build(force: bool = False) -> None:
    build_restatement(force)
    build_reference(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print(ORACLE_SO)
    print(REF_SO if os.path.exists(REF_SO) else "(reference harness not built)")
