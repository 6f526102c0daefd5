"""The C-ABI library without a GPU: it loads, exports every function that
include/pangu_b200.h declares, its structs have the header's layout (checked
against a C program compiled with gcc), and argument validation returns the
documented status codes before any device work."""
import ctypes as C
import os
import re
import subprocess

import pytest

from pangu_b200 import abi, engine
from pangu_b200 import params as prm
from pangu_b200 import problems

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pangu_b200.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pangu_\w+)\s*\(", text)))


def test_library_exports_every_header_function():
    L = engine.lib()
    names = header_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def structs():
    out = {"pangu_params": abi.Params, "pangu_mesh": abi.Mesh, "pangu_pack": abi.Pack}
    if hasattr(abi, "ServerStats"):
        out["pangu_server_stats"] = abi.ServerStats
    if hasattr(abi, "Problem"):
        out["pangu_problem"] = abi.Problem
    return out


def test_struct_layout_matches_header(tmp_path):
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "pangu_b200.h"',
           'int main(void) {']
    for cname, cls in structs().items():
        src.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            src.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    src += ['  return 0;', '}']
    c = tmp_path / "layout.c"
    c.write_text("\n".join(src))
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-std=c11", "-I", os.path.dirname(HEADER), str(c), "-o",
                           str(exe)])
    got = {}
    for line in subprocess.check_output([str(exe)], text=True).splitlines():
        s, f, v = line.split()
        got[(s, f)] = int(v)
    for cname, cls in structs().items():
        assert got[(cname, "size")] == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)


def test_num_fields():
    L = engine.lib()
    p = abi.Params()
    for B, H, n in ((0, 0, 6), (1, 0, 9), (0, 1, 7), (1, 1, 10)):
        p.enable_B, p.enable_heating = B, H
        assert L.pangu_num_fields(C.byref(p)) == n == prm.num_components(B, H)
    assert L.pangu_num_fields(None) == abi.PANGU_EINVAL


def _torus_structs():
    pin = problems.fm_torus_input(nx1=64, nx2=32)
    return prm.params_struct(prm.process_packages(pin)), prm.mesh_struct(pin)


def test_create_validates_before_device_work():
    L = engine.lib()
    h = C.c_void_p()
    p, m = _torus_structs()
    assert L.pangu_engine_create(None, C.byref(m), C.byref(h)) == abi.PANGU_EINVAL
    bad = abi.Params.from_buffer_copy(p)
    bad.riemann_solver = 7
    assert L.pangu_engine_create(C.byref(bad), C.byref(m), C.byref(h)) == abi.PANGU_EINVAL
    bad = abi.Params.from_buffer_copy(p)
    bad.precision = 2
    assert L.pangu_engine_create(C.byref(bad), C.byref(m), C.byref(h)) == abi.PANGU_EINVAL
    thin = abi.Mesh.from_buffer_copy(m)
    thin.ng = 2  # PPM4 needs three ghost layers
    assert L.pangu_engine_create(C.byref(p), C.byref(thin), C.byref(h)) == abi.PANGU_ENGHOST
    badbc = abi.Mesh.from_buffer_copy(m)
    badbc.bc[0] = 9
    assert L.pangu_engine_create(C.byref(p), C.byref(badbc), C.byref(h)) == abi.PANGU_EINVAL
    assert h.value is None
    assert L.pangu_pool_create(C.byref(p), C.byref(m), 0, 1, C.byref(h)) == abi.PANGU_EINVAL
    assert L.pangu_stage(None, 1, None, None, 0.5, None, None, None) == abi.PANGU_EINVAL
    assert L.pangu_launches(None) == abi.PANGU_EINVAL


def test_python_layer_fails_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    pin = problems.fm_torus_input(nx1=64, nx2=32)
    with pytest.raises(engine.EngineError):
        engine.Simulation(pin)
