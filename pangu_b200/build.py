"""Builds the engine's shared library in-tree for sm_100a.

    python -m pangu_b200.build [--force] [--verbose]

Produces ``pangu_b200/_lib/libpangu_b200.so`` from the CUDA sources of
``csrc/`` (nvcc, ``-gencode arch=compute_100a,code=sm_100a``) and
``csrc/host_tables.cc`` (g++). The exact FP64 build (engine.cu) uses
``--fmad=false``; the mixed-precision one (engine_mixed.cu) is built with
``--use_fast_math``, which touches only its FP32 arithmetic. Host code that evaluates the coordinate map is compiled with
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


# Translation units of the mixed-precision form: FMA contraction and the fast
# FP32 division, square root and math functions (2.6 % per cycle on the 2D
# torus, 6.6 % on the 3D one; the errors against FP64 do not change).
MIXED_SOURCES = ("engine_mixed.cu", "engine_mixed_tables.cu")


def sources():
    out = []
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cu", ".cc", ".cuh", ".h")):
            out.append(os.path.join(CSRC, name))
    out.append(os.path.join(INCLUDE, "pangu_b200.h"))
    return out


# Sources without stage kernels: the serving loop (host code over the C ABI)
# and the FP64 peak probe. They do not enter the fingerprint below.
NOT_STAGE = ("serve.cu", "fp64_peak.cu")


def source_hash() -> str:
    """Fingerprint of the sources of the stage kernels and their launchers
    (csrc/ but the files of NOT_STAGE, and the C ABI header): the build that a
    profile summary was captured on carries it, so measurements of other
    kernel sources are never reported against this build."""
    import hashlib
    h = hashlib.sha256()
    for src in sorted(sources()):
        if os.path.basename(src) in NOT_STAGE:
            continue
        with open(src, "rb") as f:
            h.update(os.path.basename(src).encode() + b"\0" + f.read())
    return h.hexdigest()[:16]


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
    objs, jobs = [], []
    for name in sorted(os.listdir(CSRC)):
        src = os.path.join(CSRC, name)
        if name.endswith(".cu"):
            obj = os.path.join(obj_dir, name + ".o")
            flags = NVCC_FLAGS
            if name in MIXED_SOURCES:
                flags = [f if f != "--fmad=false" else "--use_fast_math" for f in flags]
            cmd = [nvcc(), *ARCH, *flags, "-I", INCLUDE, "-I", CSRC, "-c", src, "-o", obj]
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
        jobs.append((subprocess.Popen(cmd), cmd))
        objs.append(obj)
    for proc, cmd in jobs:  # translation units compile in parallel
        if proc.wait() != 0:
            raise subprocess.CalledProcessError(proc.returncode, cmd)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
