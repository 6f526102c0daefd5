"""Build recipe of the Parthenon-shim test library (test infrastructure).

Compiles the product shim pangu_b200/parthenon/b200_tasks.cc and the test
driver driver.cc against the host-only Parthenon stand-in of
oracle/refshim, links them with the engine library, and writes
tests/parthenon_shim/_build/libshim_driver.so.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "_build", "libshim_driver.so")
SOURCES = (os.path.join(ROOT, "pangu_b200", "parthenon", "b200_tasks.cc"),
           os.path.join(HERE, "driver.cc"))
DEPS = SOURCES + (os.path.join(ROOT, "pangu_b200", "parthenon", "b200_tasks.h"),
                  os.path.join(ROOT, "include", "pangu_b200.h"),
                  os.path.join(ROOT, "oracle", "refshim", "parthenon", "package.hpp"))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build(force: bool = False) -> str:
    sys.path.insert(0, ROOT)
    from pangu_b200 import build as engine_build
    lib = engine_build.build()
    deps = DEPS + (lib,)
    if not force and os.path.exists(OUT) and \
            all(os.path.getmtime(s) <= os.path.getmtime(OUT) for s in deps):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    libdir = os.path.dirname(lib)
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-Wall",
           "-I", os.path.join(ROOT, "oracle", "refshim"), "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), *SOURCES,
           "-L", libdir, "-lpangu_b200",
           "-Wl,-rpath,$ORIGIN/" + os.path.relpath(libdir, os.path.dirname(OUT)),
           os.path.join(CUDA, "lib64", "libcudart_static.a"), "-ldl", "-lrt", "-lpthread",
           "-o", OUT + ".tmp"]
    subprocess.check_call(cmd)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
