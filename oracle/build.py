"""Build recipe of the oracle (test infrastructure, never part of the engine).

* ``oracle/_build/liboracle.so``  -- the CPU restatement (oracle.cc), always.
* ``oracle/_ref/libpangu_refcell.so`` -- the reference's own per-cell headers
  (pangu/src/{metric,physics,interpolation,recovery}) compiled with g++ from
  where they lie, through the stand-in headers of ``oracle/refshim``. Only
  when the reference sources are present (this container); the built file
  travels with the repository snapshot like any other built library.

Both are compiled -O2 -ffp-contract=off: no fused multiply-add anywhere, so
the restatement and the reference's host code round identically.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REFERENCE_SRC = "/root/reference/pangu/src"

ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REFCELL_SO = os.path.join(HERE, "_ref", "libpangu_refcell.so")

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


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build_oracle(force))
    print(build_refcell(force))
