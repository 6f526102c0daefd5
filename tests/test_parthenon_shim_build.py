"""The Parthenon task shim (pangu_b200/parthenon/b200_tasks.cc) compiles
against the Parthenon stand-in, defines the reference's task functions with
their signatures, and -- without a GPU -- fails a task cleanly (TaskStatus::
fail from the engine's error, no crash, no exception through the call)."""
import ctypes as C
import importlib.util
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))

# The reference's task functions (ideal_grmhd.cc:62-110) as g++ mangles
# their declarations in fixer/, riemann_solver/, constrained_transport/,
# recovery/ and initialization/ of pangu/src.
TASKS = {
    "FixPrimitive": "_Z12FixPrimitivePN9parthenon8MeshDataIdEE",
    "CalculateConservative": "_Z21CalculateConservativePN9parthenon8MeshDataIdEE",
    "CalculateFluxes": "_Z15CalculateFluxesPN9parthenon8MeshDataIdEE",
    "ConstraintedTransport": "_Z21ConstraintedTransportPN9parthenon8MeshDataIdEE",
    "AddGeometricSource": "_Z18AddGeometricSourcePN9parthenon8MeshDataIdEEd",
    "Recovery": "_Z8RecoveryPN9parthenon8MeshDataIdEE",
    "ApplyElectronHeating": "_Z20ApplyElectronHeatingPN9parthenon8MeshDataIdEE",
    "FixRecovery": "_Z11FixRecoveryPN9parthenon8MeshDataIdEE",
    "EstimateTimestepMesh": "_Z20EstimateTimestepMeshPN9parthenon8MeshDataIdEE",
}


def _build():
    spec = importlib.util.spec_from_file_location(
        "parthenon_shim_build", os.path.join(HERE, "parthenon_shim", "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build()


def test_shim_defines_the_reference_task_functions():
    path = _build()
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    defined = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for name, sym in TASKS.items():
        assert sym in defined, name


def test_shim_task_without_a_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible: the GPU tests cover the working path")
    from parity_util import Case
    path = _build()
    L = C.CDLL(path)
    L.shim_make.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_int)]
    L.shim_run.argtypes = [C.c_int, C.c_int, C.c_double, C.POINTER(C.c_double)]
    L.shim_num_prim_vars.argtypes = [C.c_void_p]
    case = Case("ot_blocks")
    nb = case.mesh.nbx1 * case.mesh.nbx2 * case.mesh.nbx3
    per = L.shim_num_prim_vars(C.byref(case.params)) + 7
    # dummy non-null addresses: nothing may dereference them on the host
    ptrs = (C.c_uint64 * (nb * per))(*([1 << 40] * (nb * per)))
    h = C.c_int(-1)
    try:
        assert L.shim_make(C.byref(case.params), C.byref(case.mesh), ptrs, C.byref(h)) == 0
        assert L.shim_run(h.value, 0, 0.0, None) == 1  # FixPrimitive: TaskStatus::fail
        out = C.c_double(0.0)
        assert L.shim_run(h.value, 8, 0.0, C.byref(out)) == -1  # EstimateTimestepMesh throws
    finally:
        L.shim_free_all()
