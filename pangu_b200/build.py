"""Builds the engine's shared library in-tree for sm_100a.

    python -m pangu_b200.build [--force] [--verbose]

Produces ``pangu_b200/_lib/libpangu_b200.so`` from ``csrc/engine.cu`` (nvcc,
``-gencode arch=compute_100a,code=sm_100a``) and ``csrc/host_tables.cc``
(g++). Host code that evaluates the coordinate map is compiled with
``-ffp-contract=off`` so its rounding matches a plain C++ build.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libpangu_b200.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "--fmad=false",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-Xcompiler", "-O2"]


def sources():
    out = []
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cu", ".cc", ".cuh", ".h")):
            out.append(os.path.join(CSRC, name))
    out.append(os.path.join(INCLUDE, "pangu_b200.h"))
    return out


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in sources())


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    obj_dir = os.path.join(LIBDIR, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    objs = []
    for name in sorted(os.listdir(CSRC)):
        src = os.path.join(CSRC, name)
        if name.endswith(".cu"):
            obj = os.path.join(obj_dir, name + ".o")
            cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", INCLUDE, "-I", CSRC, "-c", src, "-o", obj]
            if verbose:
                cmd += ["-Xptxas", "-v"]
        elif name.endswith(".cc"):
            obj = os.path.join(obj_dir, name + ".o")
            cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I", INCLUDE,
                   "-I", CSRC, "-c", src, "-o", obj]
        else:
            continue
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
