"""ctypes front end of the CPU oracle (test infrastructure only).

Imported by the tests, ``__graft_entry__.smoke()`` and the cpu_baseline leg of
``bench.py`` -- as the checker, never as the thing measured or shipped.
Host containers are numpy arrays in the layout of include/pangu_b200.h.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ROOT = os.path.dirname(_HERE)
if _ROOT not in sys.path:
    sys.path.insert(0, _ROOT)

from pangu_b200 import abi  # noqa: E402  (struct layouts only)

import importlib.util as _ilu  # noqa: E402

_spec = _ilu.spec_from_file_location("pangu_oracle_build", os.path.join(_HERE, "build.py"))
_build = _ilu.module_from_spec(_spec)
_spec.loader.exec_module(_build)

_lib = None
_reflib = None
_P = C.c_void_p
_D = C.POINTER(C.c_double)


def lib():
    global _lib
    if _lib is None:
        path = _build.build_oracle()
        L = C.CDLL(path)
        L.or_create.restype = _P
        L.or_create.argtypes = [C.POINTER(abi.Params), C.POINTER(abi.Mesh)]
        L.or_destroy.argtypes = [_P]
        L.or_num_fields.argtypes = [_P]
        L.or_counters.argtypes = [_P, C.POINTER(C.c_uint64)]
        L.or_reset_counters.argtypes = [_P]
        L.or_set_threads.argtypes = [C.c_int]
        for name in ("or_fix_primitive", "or_calculate_conservative",
                     "or_calculate_fluxes", "or_constrained_transport",
                     "or_exchange_ghosts", "or_recovery",
                     "or_apply_electron_heating", "or_fix_recovery",
                     "or_apply_boundary_conditions"):
            getattr(L, name).argtypes = [_P, C.POINTER(abi.Pack)]
        L.or_flux_divergence_update.argtypes = [_P, C.POINTER(abi.Pack), C.POINTER(abi.Pack),
                                                C.POINTER(abi.Pack), C.c_double]
        L.or_add_geometric_source.argtypes = [_P, C.POINTER(abi.Pack), C.c_double]
        L.or_estimate_dt.restype = C.c_double
        L.or_estimate_dt.argtypes = [_P, C.POINTER(abi.Pack)]
        L.or_stage.argtypes = [_P, C.c_int, C.POINTER(abi.Pack), C.POINTER(abi.Pack),
                               C.c_double, C.c_double, _D]
        _cell_sigs(L, "or_")
        _lib = L
    return _lib


def _cell_sigs(L, pre):
    getattr(L, pre + "cell_metric").argtypes = [C.c_int, _D, C.c_double, C.c_double, _D, _D, _D]
    getattr(L, pre + "cell_christoffel").argtypes = [C.c_int, _D, C.c_double, C.c_double, _D]
    getattr(L, pre + "cell_flux").argtypes = [C.c_double, _D, _D, _D, C.c_double, C.c_int, _D]
    getattr(L, pre + "cell_fast_speed").argtypes = [C.c_double, _D, _D, _D, C.c_int, _D]
    getattr(L, pre + "cell_recon").argtypes = [C.c_int, _D, _D]
    getattr(L, pre + "cell_invert").restype = C.c_int
    getattr(L, pre + "cell_invert").argtypes = [C.c_int, _D, _D, C.c_double, _D, _D]
    getattr(L, pre + "cell_heating").restype = C.c_double
    getattr(L, pre + "cell_heating").argtypes = [_D, C.POINTER(C.c_int), _D]
    getattr(L, pre + "cell_clamp").restype = C.c_double
    getattr(L, pre + "cell_clamp").argtypes = [C.c_double] * 4


def reflib():
    """The reference's own per-cell functions (only where its sources exist)."""
    global _reflib
    if _reflib is None:
        path = _build.build_refcell()
        if path is None or not os.path.exists(path):
            return None
        L = C.CDLL(path)
        _cell_sigs(L, "ref_")
        _reflib = L
    return _reflib


_reftasks = None

# task ids of ref_tasks.cc
REF_TASKS = {"fix_primitive": 0, "calculate_conservative": 1, "calculate_fluxes": 2,
             "constrained_transport": 3, "add_geometric_source": 4, "recovery": 5,
             "apply_electron_heating": 6, "fix_recovery": 7, "estimate_dt": 8}


def reftasks():
    """The reference's own stage tasks over the Parthenon stand-in (only
    where its sources exist, or where the built library travelled)."""
    global _reftasks
    if _reftasks is None:
        path = _build.build_reftasks()
        if path is None or not os.path.exists(path):
            return None
        L = C.CDLL(path)
        L.ref_task.restype = C.c_int
        L.ref_task.argtypes = [C.POINTER(abi.Params), C.POINTER(abi.Mesh), C.POINTER(abi.Pack),
                               C.c_int, C.c_double, _D]
        _reftasks = L
    return _reftasks


_reftasks_omp = None


def reftasks_omp():
    """The timing build of the reference's stage tasks (the C library's pow,
    -O3, par_for over the host threads with OpenMP), or None where it was
    neither built nor travelled with the repository."""
    global _reftasks_omp
    if _reftasks_omp is None:
        path = _build.build_reftasks_omp()
        if path is None or not os.path.exists(path):
            return None
        L = C.CDLL(path)
        L.ref_task.restype = C.c_int
        L.ref_task.argtypes = [C.POINTER(abi.Params), C.POINTER(abi.Mesh), C.POINTER(abi.Pack),
                               C.c_int, C.c_double, _D]
        _reftasks_omp = L
    return _reftasks_omp


class RefTasks:
    """The reference's task functions on host containers (HostContainer);
    timing=True takes the OpenMP timing build."""

    def __init__(self, params: abi.Params, mesh: abi.Mesh, timing: bool = False):
        self.L = reftasks_omp() if timing else reftasks()
        if self.L is None:
            raise RuntimeError("the reference's task library is not built")
        self.params, self.mesh = params, mesh

    def run(self, name, c, dt=0.0):
        p = c.pack()
        out = C.c_double(0.0)
        rc = self.L.ref_task(C.byref(self.params), C.byref(self.mesh), C.byref(p),
                             REF_TASKS[name], dt, C.byref(out))
        if rc != 0:
            raise RuntimeError(f"reference task {name} failed")
        return out.value


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


class CellAPI:
    """Uniform per-cell calls over either library ("or_" or "ref_")."""

    def __init__(self, L, prefix):
        self.L, self.p = L, prefix

    def _f(self, n):
        return getattr(self.L, self.p + n)

    def metric(self, mt, x, a, h):
        x = np.ascontiguousarray(x, dtype=np.float64)
        gcov = np.zeros(16); gcon = np.zeros(16); gdet = np.zeros(1)
        self._f("cell_metric")(mt, dptr(x), a, h, dptr(gcov), dptr(gcon), dptr(gdet))
        return gcov, gcon, gdet[0]

    def christoffel(self, mt, x, a, h):
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.zeros(64)
        self._f("cell_christoffel")(mt, dptr(x), a, h, dptr(out))
        return out

    def flux(self, gam, P, gcov, gcon, gdet, d):
        out = np.zeros(10)
        self._f("cell_flux")(gam, dptr(np.ascontiguousarray(P, dtype=np.float64)),
                             dptr(gcov), dptr(gcon), gdet, d, dptr(out))
        return out

    def fast_speed(self, gam, P, gcov, gcon, d):
        out = np.zeros(2)
        self._f("cell_fast_speed")(gam, dptr(np.ascontiguousarray(P, dtype=np.float64)),
                                   dptr(gcov), dptr(gcon), d, dptr(out))
        return out

    def recon(self, use_mc, q):
        out = np.zeros(2)
        self._f("cell_recon")(use_mc, dptr(np.ascontiguousarray(q, dtype=np.float64)), dptr(out))
        return out

    def invert(self, scheme, U, prim, gam, gcov, gcon):
        pr = np.ascontiguousarray(prim, dtype=np.float64).copy()
        st = self._f("cell_invert")(scheme, dptr(np.ascontiguousarray(U, dtype=np.float64)),
                                    dptr(pr), gam, dptr(gcov), dptr(gcon))
        return st, pr

    def heating(self, hp, flags, cell):
        fl = (C.c_int * 4)(*flags)
        return self._f("cell_heating")(dptr(np.asarray(hp, dtype=np.float64)), fl,
                                       dptr(np.asarray(cell, dtype=np.float64)))

    def clamp(self, rmin, rmax, total, electron):
        return self._f("cell_clamp")(rmin, rmax, total, electron)


class HostContainer:
    """One stage container ("base" or "1") in host memory.

    alfven, efield and flag are shared between the two containers
    (Metadata::OneCopy, package_registration.cc:121-145)."""

    def __init__(self, nb, nf, shape, shared=None):
        n3, n2, n1 = shape
        self.prim = np.zeros((nb, nf, n3, n2, n1))
        self.cons = np.zeros((nb, nf, n3, n2, n1))
        self.flux1 = np.zeros((nb, nf, n3, n2, n1))
        self.flux2 = np.zeros((nb, nf, n3, n2, n1))
        self.flux3 = np.zeros((nb, nf, n3, n2, n1))
        if shared is None:
            self.alfven = np.zeros((nb, 3, n3, n2, n1))
            self.efield = np.zeros((nb, 3, n3, n2, n1))
            self.flag = np.zeros((nb, n3, n2, n1))
        else:
            self.alfven, self.efield, self.flag = shared.alfven, shared.efield, shared.flag

    def pack(self) -> abi.Pack:
        p = abi.Pack()
        for name in ("prim", "cons", "flux1", "flux2", "flux3", "alfven", "efield", "flag"):
            setattr(p, name, getattr(self, name).ctypes.data)
        return p


class Oracle:
    """The CPU oracle for one mesh and parameter set."""

    def __init__(self, params: abi.Params, mesh: abi.Mesh):
        self.L = lib()
        self.params, self.mesh = params, mesh
        self.h = self.L.or_create(C.byref(params), C.byref(mesh))
        self.nf = self.L.or_num_fields(self.h)
        self.nb = mesh.nbx1 * mesh.nbx2 * mesh.nbx3
        act = [mesh.nx1 > 1, mesh.nx2 > 1, mesh.nx3 > 1]
        n = [mesh.nx1, mesh.nx2, mesh.nx3]
        self.shape = tuple(n[d] + 2 * mesh.ng * act[d] for d in (2, 1, 0))

    def __del__(self):
        try:
            self.L.or_destroy(self.h)
        except Exception:
            pass

    def new_containers(self):
        base = HostContainer(self.nb, self.nf, self.shape)
        one = HostContainer(self.nb, self.nf, self.shape, shared=base)
        return base, one

    def counters(self):
        out = (C.c_uint64 * abi.NCOUNTERS)()
        self.L.or_counters(self.h, out)
        return np.array(list(out), dtype=np.uint64)

    def reset_counters(self):
        self.L.or_reset_counters(self.h)

    def _call(self, name, c):
        p = c.pack()
        getattr(self.L, name)(self.h, C.byref(p))

    def fix_primitive(self, c): self._call("or_fix_primitive", c)
    def calculate_conservative(self, c): self._call("or_calculate_conservative", c)
    def calculate_fluxes(self, c): self._call("or_calculate_fluxes", c)
    def constrained_transport(self, c): self._call("or_constrained_transport", c)
    def exchange_ghosts(self, c): self._call("or_exchange_ghosts", c)
    def recovery(self, c): self._call("or_recovery", c)
    def apply_electron_heating(self, c): self._call("or_apply_electron_heating", c)
    def fix_recovery(self, c): self._call("or_fix_recovery", c)
    def apply_boundary_conditions(self, c): self._call("or_apply_boundary_conditions", c)

    def flux_divergence_update(self, mc_init, mc0, mc1, bdt):
        a, b, c = mc_init.pack(), mc0.pack(), mc1.pack()
        self.L.or_flux_divergence_update(self.h, C.byref(a), C.byref(b), C.byref(c), bdt)

    def add_geometric_source(self, c, bdt):
        p = c.pack()
        self.L.or_add_geometric_source(self.h, C.byref(p), bdt)

    def estimate_dt(self, c):
        p = c.pack()
        return self.L.or_estimate_dt(self.h, C.byref(p))

    def stage(self, st, base, one, beta, dt):
        pb, po = base.pack(), one.pack()
        est = C.c_double(0.0)
        self.L.or_stage(self.h, st, C.byref(pb), C.byref(po), beta, dt, C.byref(est))
        return est.value

    def step(self, base, one, dt):
        """One rk2 cycle (two stages, beta = {1.0, 0.5}[stage % 2])."""
        self.stage(1, base, one, 0.5, dt)
        return self.stage(2, base, one, 1.0, dt)


def set_threads(n: int) -> None:
    lib().or_set_threads(int(n))
