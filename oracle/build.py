"""Build recipe of the oracle (test infrastructure, never part of the engine).

* ``oracle/_build/liboracle.so``  -- the CPU restatement (oracle.cc), always.
* ``oracle/_ref/libpangu_refcell.so`` -- the reference's own per-cell headers
  (pangu/src/{metric,physics,interpolation,recovery}) compiled with g++ from
  where they lie, through the stand-in headers of ``oracle/refshim``. Only
  when the reference sources are present (this container); the built file
  travels with the repository snapshot like any other built library.
* ``oracle/_ref/libpangu_reftasks_omp.so`` -- the same tasks built for timing
  (the CPU baseline and ``bench.py --impl reference``): the reference's own
  math functions (the C library's pow), -O3 with the compiler's default
  contraction, and the stand-in's par_for/par_reduce spread over the host
  threads with OpenMP, as Kokkos' OpenMP backend would run them.
* ``oracle/_ref/libpangu_reftasks.so`` -- the reference's own stage tasks
  (REF_TASK_SOURCES below, compiled from where they lie) over the host-only
  Parthenon stand-in of ``oracle/refshim/parthenon/package.hpp``, with the
  driver ``ref_tasks.cc``; pow is the correctly rounded one of pgmath.h
  (-DPANGU_REFSHIM_CR_POW). Only when the reference sources are present.

Both are compiled -O2 -ffp-contract=off: no fused multiply-add anywhere, so
the restatement and the reference's host code round identically.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# The reference's solver sources (pangu/src of the PANGU tree): from the
# PANGU_REFERENCE_SRC environment variable, else the read-only checkout this
# repository was built beside.
REFERENCE_SRC = os.environ.get("PANGU_REFERENCE_SRC", "/root/reference/pangu/src")

ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REFCELL_SO = os.path.join(HERE, "_ref", "libpangu_refcell.so")
REFTASKS_SO = os.path.join(HERE, "_ref", "libpangu_reftasks.so")
REFTASKS_OMP_SO = os.path.join(HERE, "_ref", "libpangu_reftasks_omp.so")

# The reference's stage-task sources (paths under pangu/src).
REF_TASK_SOURCES = (
    "fixer/primitive_fixer.cc", "fixer/recovery_fixer.cc",
    "riemann_solver/conservative.cc", "riemann_solver/laxf.cc", "riemann_solver/hll.cc",
    "riemann_solver/riemann_solver.cc", "riemann_solver/source_term.cc",
    "riemann_solver/electron_heating.cc", "constrained_transport/constrained_transport.cc",
    "recovery/invertor.cc", "initialization/timestep_estimation.cc",
)

COMMON = ["-O2", "-ffp-contract=off", "-std=c++17", "-shared", "-fPIC"]


def _newer(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources if os.path.exists(s))


def build_oracle(force: bool = False) -> str:
    src = [os.path.join(HERE, "oracle.cc"), os.path.join(HERE, "oracle_cell.h"),
           os.path.join(ROOT, "include", "pangu_b200.h"),
           os.path.join(ROOT, "pangu_b200", "csrc", "pgmath.h")]
    if not force and _newer(ORACLE_SO, src):
        return ORACLE_SO
    os.makedirs(os.path.dirname(ORACLE_SO), exist_ok=True)
    cmd = ["g++", *COMMON, "-fopenmp", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "pangu_b200", "csrc"), src[0], "-o", ORACLE_SO]
    subprocess.check_call(cmd)
    return ORACLE_SO


def build_refcell(force: bool = False) -> str | None:
    if not os.path.isdir(REFERENCE_SRC):
        return REFCELL_SO if os.path.exists(REFCELL_SO) else None
    src = [os.path.join(HERE, "ref_cell.cc")]
    if not force and _newer(REFCELL_SO, src):
        return REFCELL_SO
    os.makedirs(os.path.dirname(REFCELL_SO), exist_ok=True)
    cmd = ["g++", *COMMON, "-I", os.path.join(HERE, "refshim"),
           "-I", REFERENCE_SRC, src[0], "-o", REFCELL_SO]
    subprocess.check_call(cmd)
    return REFCELL_SO


def build_reftasks(force: bool = False) -> str | None:
    if not os.path.isdir(REFERENCE_SRC):
        return REFTASKS_SO if os.path.exists(REFTASKS_SO) else None
    shim = os.path.join(HERE, "refshim")
    src = [os.path.join(HERE, "ref_tasks.cc"), os.path.join(shim, "parthenon", "package.hpp"),
           os.path.join(shim, "Kokkos_Core.hpp"),
           os.path.join(ROOT, "pangu_b200", "csrc", "pgmath.h")]
    ref = [os.path.join(REFERENCE_SRC, f) for f in REF_TASK_SOURCES]
    if not force and _newer(REFTASKS_SO, src + ref):
        return REFTASKS_SO
    os.makedirs(os.path.dirname(REFTASKS_SO), exist_ok=True)
    cmd = ["g++", *COMMON, "-DPANGU_REFSHIM_CR_POW", "-I", shim,
           "-I", os.path.join(ROOT, "pangu_b200", "csrc"), "-I", os.path.join(ROOT, "include"),
           "-I", REFERENCE_SRC, src[0], *ref, "-o", REFTASKS_SO]
    subprocess.check_call(cmd)
    return REFTASKS_SO


def build_reftasks_omp(force: bool = False) -> str | None:
    if not os.path.isdir(REFERENCE_SRC):
        return REFTASKS_OMP_SO if os.path.exists(REFTASKS_OMP_SO) else None
    shim = os.path.join(HERE, "refshim")
    src = [os.path.join(HERE, "ref_tasks.cc"), os.path.join(shim, "parthenon", "package.hpp"),
           os.path.join(shim, "Kokkos_Core.hpp")]
    ref = [os.path.join(REFERENCE_SRC, f) for f in REF_TASK_SOURCES]
    if not force and _newer(REFTASKS_OMP_SO, src + ref):
        return REFTASKS_OMP_SO
    os.makedirs(os.path.dirname(REFTASKS_OMP_SO), exist_ok=True)
    cmd = ["g++", "-O3", "-std=c++17", "-shared", "-fPIC", "-fopenmp", "-DPANGU_REFSHIM_OMP",
           "-I", shim, "-I", os.path.join(ROOT, "pangu_b200", "csrc"),
           "-I", os.path.join(ROOT, "include"), "-I", REFERENCE_SRC, src[0], *ref,
           "-o", REFTASKS_OMP_SO]
    subprocess.check_call(cmd)
    return REFTASKS_OMP_SO


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build_oracle(force))
    print(build_refcell(force))
    print(build_reftasks(force))
    print(build_reftasks_omp(force))
