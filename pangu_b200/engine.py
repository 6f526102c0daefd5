"""Host side of the engine: library loading, device containers, stage driver.

The compute path is the CUDA library ``_lib/libpangu_b200.so`` reached
through the C ABI of include/pangu_b200.h. There is no CPU fallback: if the
library is missing and cannot be built, or no CUDA device is present, the
calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi
from .params import (ParameterInput, engine_precision, mesh_struct, params_struct,
                     process_packages)

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None

_P = C.c_void_p
_PK = C.POINTER(abi.Pack)
_DP = C.c_void_p  # device double*


class EngineError(RuntimeError):
    pass


_ERRORS = {abi.PANGU_EINVAL: "invalid argument", abi.PANGU_ECUDA: "CUDA error",
           abi.PANGU_ENOMEM: "out of device memory",
           abi.PANGU_ENGHOST: "ghost width too small for the limiter",
           abi.PANGU_ETOOBIG: "size above the supported maximum",
           abi.PANGU_EFULL: "no free pool slot or job id"}


def _check(rc, what):
    if rc != abi.PANGU_OK:
        raise EngineError(f"{what}: {_ERRORS.get(rc, rc)} ({rc})")


def library_path() -> str:
    return os.path.join(_HERE, "_lib", "libpangu_b200.so")


def lib():
    """Loads the engine library (building it in-tree first if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        from . import build
        build.build()
    L = C.CDLL(path)
    L.pangu_num_fields.argtypes = [C.POINTER(abi.Params)]
    L.pangu_engine_create.argtypes = [C.POINTER(abi.Params), C.POINTER(abi.Mesh), C.POINTER(_P)]
    L.pangu_engine_destroy.argtypes = [_P]
    for name in ("pangu_fix_primitive", "pangu_calculate_conservative", "pangu_calculate_fluxes",
                 "pangu_constrained_transport", "pangu_exchange_ghosts", "pangu_recovery",
                 "pangu_apply_electron_heating", "pangu_fix_recovery",
                 "pangu_apply_boundary_conditions"):
        getattr(L, name).argtypes = [_P, _PK, _P]
    L.pangu_flux_divergence_update.argtypes = [_P, _PK, _PK, _PK, C.c_double, _DP, _P]
    L.pangu_add_geometric_source.argtypes = [_P, _PK, C.c_double, _DP, _P]
    L.pangu_estimate_dt.argtypes = [_P, _PK, _DP, _P]
    L.pangu_stage.argtypes = [_P, C.c_int, _PK, _PK, C.c_double, _DP, _DP, _P]
    L.pangu_update_dt.argtypes = [_P, _DP, _DP, C.c_double, _P]
    L.pangu_counters.argtypes = [_P, C.POINTER(C.c_uint64)]
    L.pangu_reset_counters.argtypes = [_P, _P]
    L.pangu_launches.argtypes = [_P]
    L.pangu_launches.restype = C.c_longlong
    L.pangu_device_error.argtypes = [_P, C.POINTER(C.c_int32)]
    L.pangu_pool_create.argtypes = [C.POINTER(abi.Params), C.POINTER(abi.Mesh), C.c_int32,
                                    C.c_int32, C.POINTER(_P)]
    L.pangu_job_attach.argtypes = [_P, C.POINTER(abi.Mesh), C.c_double, C.c_double,
                                   C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    L.pangu_job_start.argtypes = [_P, C.c_int32, _PK, _PK, _P]
    L.pangu_job_detach.argtypes = [_P, C.c_int32]
    L.pangu_job_counters.argtypes = [_P, C.c_int32, C.POINTER(C.c_uint64)]
    L.pangu_active_blocks.argtypes = [_P]
    L.pangu_autotune.argtypes = [_P, _PK, _P]
    L.pangu_generate.argtypes = [_P, C.c_int32, C.POINTER(abi.Problem), _PK, _P]
    L.pangu_server_submit_problem.argtypes = [_P, C.c_int32, C.POINTER(abi.Mesh), C.c_double,
                                              C.c_double, C.c_double, C.c_int64, C.c_double,
                                              C.POINTER(abi.Problem), C.POINTER(C.c_int32)]
    L.pangu_flux_config.argtypes = [_P, C.POINTER(C.c_int32)]
    L.pangu_set_flux_config.argtypes = [_P, C.POINTER(C.c_int32)]
    L.pangu_server_create.argtypes = [C.c_uint64, C.POINTER(_P)]
    L.pangu_server_destroy.argtypes = [_P]
    L.pangu_server_add_class.argtypes = [_P, C.POINTER(abi.Params), C.POINTER(abi.Mesh), C.c_int32,
                                         C.c_int32, C.c_double, C.POINTER(C.c_int32)]
    L.pangu_server_declare_class.argtypes = L.pangu_server_add_class.argtypes
    L.pangu_server_submit.argtypes = [_P, C.c_int32, C.POINTER(abi.Mesh), C.c_double, C.c_double,
                                      C.c_double, C.c_int64, C.c_double, C.c_void_p,
                                      C.POINTER(C.c_int32)]
    L.pangu_server_run.argtypes = [_P]
    L.pangu_server_result.argtypes = [_P, C.c_int32, C.c_void_p, C.c_void_p,
                                      C.POINTER(C.c_uint64)]
    L.pangu_server_get_stats.argtypes = [_P, C.POINTER(abi.ServerStats)]
    L.pangu_server_cancel.argtypes = [_P, C.c_int32, C.c_double]
    L.pangu_server_job_state.argtypes = [_P, C.c_int32]
    _I32P, _I64P = C.POINTER(C.c_int32), C.POINTER(C.c_int64)
    L.pangu_shard_create.argtypes = [C.POINTER(abi.Params), C.POINTER(abi.Mesh), _I32P, C.c_int32,
                                     C.c_int32, C.POINTER(_P)]
    L.pangu_shard_plan.argtypes = [C.POINTER(abi.Params), C.POINTER(abi.Mesh), _I32P, C.c_int32,
                                   C.c_int32, _I64P, _I64P, _I64P, _I64P]
    L.pangu_halo_counts.argtypes = [_P, _I64P, _I64P]
    L.pangu_halo_pack.argtypes = [_P, _PK, _DP, _P]
    L.pangu_halo_unpack.argtypes = [_P, _PK, _DP, _P]
    L.pangu_stage_begin.argtypes = [_P, C.c_int, _PK, _PK, C.c_double, _DP, _DP, _P]
    L.pangu_stage_middle.argtypes = [_P, C.c_int, _PK, _PK, C.c_double, _DP, _P]
    L.pangu_stage_update.argtypes = [_P, C.c_int, _PK, _PK, C.c_double, _DP, _P]
    L.pangu_stage_end.argtypes = [_P, C.c_int, _PK, _PK, _DP, _DP, _P]
    _lib = L
    return L


def _ptr(t):
    """Device pointer of a tensor, or NULL for None or an empty tensor."""
    return t.data_ptr() if t is not None and t.numel() else None


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise EngineError("the engine needs a CUDA device; none is visible")
    return torch


class DeviceContainer:
    """One stage container ("base" or "1") in device memory (torch tensors).

    ``alfven``, ``efield`` and ``flag`` are shared between the two containers
    of a job (Metadata::OneCopy, package_registration.cc:121-145)."""

    FIELDS = ("prim", "cons", "flux1", "flux2", "flux3", "alfven", "efield", "flag")

    def __init__(self, nb, nf, shape, device, shared=None, mixed=False):
        torch = _torch()
        n3, n2, n1 = shape
        z = lambda *s: torch.zeros(s, dtype=torch.float64, device=device)  # noqa: E731
        # the mixed-precision form stores the primitives in FP32
        self.prim = torch.zeros((nb, nf, n3, n2, n1), device=device,
                                dtype=torch.float32 if mixed else torch.float64)
        self.cons = z(nb, nf, n3, n2, n1)
        self.flux1 = z(nb, nf, n3, n2, n1)
        self.flux2 = z(nb, nf, n3, n2, n1)
        self.flux3 = z(nb, nf, n3, n2, n1)
        if shared is None:
            self.alfven = z(nb, 3, n3, n2, n1)
            self.efield = z(nb, 3, n3, n2, n1)
            self.flag = z(nb, n3, n2, n1)
        else:
            self.alfven, self.efield, self.flag = shared.alfven, shared.efield, shared.flag
        self._pack = abi.Pack()
        for f in self.FIELDS:
            setattr(self._pack, f, getattr(self, f).data_ptr())

    @property
    def pack(self):
        return C.byref(self._pack)


class TableContainer:
    """A stage container laid out as Parthenon keeps its variables: one device
    allocation per block and variable, addressed through the pack's
    per-(block, component) pointer tables (pangu_pack.*_vars).

    ``prim_groups`` / ``cons_groups`` split the NF components into variables
    (component counts, e.g. (1, 1, 3, 3, 1) for density, energy,
    weighted_velocity, magnetic_field, entropy; default: one allocation per
    component); the face fluxes follow ``cons_groups``; alfven and efield are
    one 3-component variable, flag one scalar. ``contiguous`` names fields
    kept in the contiguous [NB][NC][N3][N2][N1] layout instead (a pack may mix
    both). ``shared`` takes alfven, efield and flag from another container
    (Metadata::OneCopy)."""

    FIELDS = DeviceContainer.FIELDS

    def __init__(self, nb, nf, shape, device, prim_groups=None, cons_groups=None, shared=None,
                 contiguous=(), mixed=False):
        torch = _torch()
        self.nb, self.nf, self.shape, self.device = nb, nf, tuple(shape), device
        self.ncell = int(np.prod(shape))
        pdt = torch.float32 if mixed else torch.float64
        groups = {"prim": tuple(prim_groups or (1,) * nf), "alfven": (3,), "efield": (3,),
                  "flag": (1,)}
        for f in ("cons", "flux1", "flux2", "flux3"):
            groups[f] = tuple(cons_groups or (1,) * nf)
        # a table must hold NB * NC entries: the kernels index it by (slot, component)
        for f in ("prim", "cons"):
            if sum(groups[f]) != nf or min(groups[f]) < 1:
                raise ValueError(f"{f} variables {groups[f]} do not cover the {nf} components")
        self.arrays, self.tables, self.dense = {}, {}, {}
        self._pack = abi.Pack()
        for f in self.FIELDS:
            if shared is not None and f in ("alfven", "efield", "flag"):
                self.arrays[f] = shared.arrays.get(f)
                self.dense[f] = shared.dense.get(f)
                self.tables[f] = shared.tables.get(f)
            else:
                nc = sum(groups[f])
                dtype = pdt if f == "prim" else torch.float64
                if f in contiguous:
                    shp = (nb, *shape) if f == "flag" else (nb, nc, *shape)
                    self.dense[f] = torch.zeros(shp, dtype=dtype, device=device)
                    self.arrays[f] = None
                    self.tables[f] = None
                else:
                    self.dense[f] = None
                    self.arrays[f] = [[torch.zeros((g, *shape), dtype=dtype, device=device)
                                       for g in groups[f]] for _ in range(nb)]
                    ptrs = []
                    for b in range(nb):
                        for t in self.arrays[f][b]:
                            ptrs += [t.data_ptr() + c * self.ncell * t.element_size()
                                     for c in range(t.shape[0])]
                    self.tables[f] = torch.tensor(ptrs, dtype=torch.int64, device=device)
            if self.dense[f] is not None:
                setattr(self._pack, f, self.dense[f].data_ptr())
            if self.tables[f] is not None:
                setattr(self._pack, f + "_vars", self.tables[f].data_ptr())

    @property
    def pack(self):
        return C.byref(self._pack)

    def gather(self, f):
        """Field f as one [NB][NC][N3][N2][N1] ([NB][N3][N2][N1] for flag) tensor."""
        torch = _torch()
        if self.dense[f] is not None:
            return self.dense[f].clone()
        out = torch.stack([torch.cat(blk, dim=0) for blk in self.arrays[f]])
        return out[:, 0] if f == "flag" else out

    def scatter(self, f, src):
        """Writes field f from a tensor of the gather() shape."""
        if self.dense[f] is not None:
            self.dense[f].copy_(src)
            return
        src = src.reshape(self.nb, -1, *self.shape)
        for b in range(self.nb):
            c = 0
            for t in self.arrays[f][b]:
                t.copy_(src[b, c:c + t.shape[0]])
                c += t.shape[0]

    def load(self, other):
        """Copies every field of a container (DeviceContainer or TableContainer)."""
        for f in self.FIELDS:
            self.scatter(f, other.gather(f) if isinstance(other, TableContainer)
                         else getattr(other, f))


class Engine:
    """An engine handle for one parameter set and mesh."""

    def __init__(self, params: abi.Params, mesh: abi.Mesh, device=0, pool=None, shard=None):
        """pool=None: one mesh (pangu_engine_create). pool=(capacity_blocks,
        max_jobs): an empty block pool of mesh's block shape.
        shard=(block_rank, nranks, rank): rank's blocks of a mesh spread
        over nranks engines (pangu_shard_create)."""
        torch = _torch()
        self.device = torch.device("cuda", device)
        self.L = lib()
        self.params, self.mesh = params, mesh
        h = _P()
        with torch.cuda.device(self.device):
            if shard is not None:
                br = np.ascontiguousarray(shard[0], dtype=np.int32)
                _check(self.L.pangu_shard_create(C.byref(params), C.byref(mesh),
                                                 br.ctypes.data_as(C.POINTER(C.c_int32)),
                                                 int(shard[1]), int(shard[2]), C.byref(h)),
                       "pangu_shard_create")
                pool = (int((br == int(shard[2])).sum()), 1)
            elif pool is None:
                _check(self.L.pangu_engine_create(C.byref(params), C.byref(mesh), C.byref(h)),
                       "pangu_engine_create")
            else:
                _check(self.L.pangu_pool_create(C.byref(params), C.byref(mesh), int(pool[0]),
                                                int(pool[1]), C.byref(h)), "pangu_pool_create")
        self.sharded = shard is not None
        self.h = h
        self.nf = self.L.pangu_num_fields(C.byref(params))
        self.nb = mesh.nbx1 * mesh.nbx2 * mesh.nbx3 if pool is None else int(pool[0])
        act = [mesh.nx1 > 1, mesh.nx2 > 1, mesh.nx3 > 1]
        n = [mesh.nx1, mesh.nx2, mesh.nx3]
        self.shape = tuple(n[d] + 2 * mesh.ng * act[d] for d in (2, 1, 0))

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.pangu_engine_destroy(self.h)
            self.h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stream(self):
        import torch
        return _P(torch.cuda.current_stream(self.device).cuda_stream)

    @property
    def mixed(self) -> bool:
        return self.params.precision == abi.PRECISION["mixed"]

    def new_containers(self):
        base = DeviceContainer(self.nb, self.nf, self.shape, self.device, mixed=self.mixed)
        one = DeviceContainer(self.nb, self.nf, self.shape, self.device, shared=base,
                              mixed=self.mixed)
        return base, one

    # ---- per-task entry points ------------------------------------------
    def _task(self, name, md):
        _check(getattr(self.L, name)(self.h, md.pack, self.stream()), name)

    def fix_primitive(self, md): self._task("pangu_fix_primitive", md)
    def calculate_conservative(self, md): self._task("pangu_calculate_conservative", md)
    def calculate_fluxes(self, md): self._task("pangu_calculate_fluxes", md)
    def constrained_transport(self, md): self._task("pangu_constrained_transport", md)
    def exchange_ghosts(self, md): self._task("pangu_exchange_ghosts", md)
    def recovery(self, md): self._task("pangu_recovery", md)
    def apply_electron_heating(self, md): self._task("pangu_apply_electron_heating", md)
    def fix_recovery(self, md): self._task("pangu_fix_recovery", md)
    def apply_boundary_conditions(self, md): self._task("pangu_apply_boundary_conditions", md)

    def flux_divergence_update(self, mc_init, mc0, mc1, beta, dt_dev):
        _check(self.L.pangu_flux_divergence_update(self.h, mc_init.pack, mc0.pack, mc1.pack,
                                                   beta, dt_dev.data_ptr(), self.stream()),
               "pangu_flux_divergence_update")

    def add_geometric_source(self, md, beta, dt_dev):
        _check(self.L.pangu_add_geometric_source(self.h, md.pack, beta, dt_dev.data_ptr(),
                                                 self.stream()), "pangu_add_geometric_source")

    def estimate_dt(self, md, out_dev):
        _check(self.L.pangu_estimate_dt(self.h, md.pack, out_dev.data_ptr(), self.stream()),
               "pangu_estimate_dt")

    def stage(self, st, base, one, beta, dt_dev, dt_est_dev=None):
        est = dt_est_dev.data_ptr() if dt_est_dev is not None else None
        _check(self.L.pangu_stage(self.h, st, base.pack, one.pack, beta, dt_dev.data_ptr(), est,
                                  self.stream()), "pangu_stage")

    # -- block sharding (pangu_b200.shard drives these) --
    def halo_counts(self, nranks):
        snd, rcv = (C.c_int64 * nranks)(), (C.c_int64 * nranks)()
        _check(self.L.pangu_halo_counts(self.h, snd, rcv), "pangu_halo_counts")
        return list(snd), list(rcv)

    def halo_pack(self, md, send):
        _check(self.L.pangu_halo_pack(self.h, md.pack, _ptr(send), self.stream()),
               "pangu_halo_pack")

    def halo_unpack(self, md, recv):
        _check(self.L.pangu_halo_unpack(self.h, md.pack, _ptr(recv), self.stream()),
               "pangu_halo_unpack")

    def stage_begin(self, st, base, one, beta, dt_dev, send):
        _check(self.L.pangu_stage_begin(self.h, st, base.pack, one.pack, beta, dt_dev.data_ptr(),
                                        _ptr(send), self.stream()), "pangu_stage_begin")

    def stage_update(self, st, base, one, beta, dt_dev):
        _check(self.L.pangu_stage_update(self.h, st, base.pack, one.pack, beta, dt_dev.data_ptr(),
                                         self.stream()), "pangu_stage_update")

    def stage_middle(self, st, base, one, beta, dt_dev):
        _check(self.L.pangu_stage_middle(self.h, st, base.pack, one.pack, beta, dt_dev.data_ptr(),
                                         self.stream()), "pangu_stage_middle")

    def stage_end(self, st, base, one, recv, dt_est_dev=None):
        est = dt_est_dev.data_ptr() if dt_est_dev is not None else None
        _check(self.L.pangu_stage_end(self.h, st, base.pack, one.pack, _ptr(recv), est,
                                      self.stream()), "pangu_stage_end")

    def update_dt(self, dt_dev, dt_est_dev, factor):
        _check(self.L.pangu_update_dt(self.h, dt_dev.data_ptr(), dt_est_dev.data_ptr(), factor,
                                      self.stream()), "pangu_update_dt")

    def counters(self):
        out = (C.c_uint64 * abi.NCOUNTERS)()
        _check(self.L.pangu_counters(self.h, out), "pangu_counters")
        return np.array(list(out), dtype=np.uint64)

    def launches(self) -> int:
        return int(self.L.pangu_launches(self.h))

    def device_error(self) -> bool:
        """True if a kernel of this engine gave up a bounded wait (its results
        are then incomplete)."""
        out = C.c_int32()
        _check(self.L.pangu_device_error(self.h, C.byref(out)), "pangu_device_error")
        return bool(out.value)

    def reset_counters(self):
        _check(self.L.pangu_reset_counters(self.h, self.stream()), "pangu_reset_counters")

    def autotune(self, md):
        """Picks the flux kernels' tile shapes by timing them on md's data."""
        _check(self.L.pangu_autotune(self.h, md.pack, self.stream()), "pangu_autotune")

    def generate(self, job, problem: abi.Problem, base):
        """Initial primitives of a job generated on the device into base."""
        _check(self.L.pangu_generate(self.h, job, C.byref(problem), base.pack, self.stream()),
               "pangu_generate")

    def flux_config(self) -> dict:
        out = (C.c_int32 * 7)()
        _check(self.L.pangu_flux_config(self.h, out), "pangu_flux_config")
        v = list(out)
        return {"x1_march": v[0], "x1_threads": v[1], "x2_march": v[2], "x2_threads": v[3],
                "x3_march": v[4], "x3_threads": v[5], "tuned": bool(v[6])}

    def set_flux_config(self, x1_threads=128, x2_march=2, x2_threads=128, x3_march=2,
                        x3_threads=128, x1_march=1, **_):
        """Sets the flux tile shapes (the keys of flux_config())."""
        cfg = (C.c_int32 * 6)(x1_march, x1_threads, x2_march, x2_threads, x3_march, x3_threads)
        _check(self.L.pangu_set_flux_config(self.h, cfg), "pangu_set_flux_config")

    # ---- block pool --------------------------------------------------------
    def attach(self, mesh: abi.Mesh, a: float, h: float):
        job = C.c_int32()
        nbl = mesh.nbx1 * mesh.nbx2 * mesh.nbx3
        slots = (C.c_int32 * nbl)()
        _check(self.L.pangu_job_attach(self.h, C.byref(mesh), a, h, C.byref(job), slots),
               "pangu_job_attach")
        return job.value, list(slots)

    def job_start(self, job, base, one):
        _check(self.L.pangu_job_start(self.h, job, base.pack, one.pack, self.stream()),
               "pangu_job_start")

    def detach(self, job):
        _check(self.L.pangu_job_detach(self.h, job), "pangu_job_detach")

    def job_counters(self, job):
        out = (C.c_uint64 * abi.NCOUNTERS)()
        _check(self.L.pangu_job_counters(self.h, job, out), "pangu_job_counters")
        return np.array(list(out), dtype=np.uint64)

    def active_blocks(self) -> int:
        return int(self.L.pangu_active_blocks(self.h))


# rk2 of Parthenon's low-storage integrator: beta[stage % 2] with
# beta = {1.0, 0.5} (ideal_grmhd.cc:29).
RK2_BETA = (1.0, 0.5)


class HostState:
    """A job's state in pinned host memory: what one RK2 cycle reads and
    writes (both containers' primitives, the flags and dt)."""

    def __init__(self, sim: "Simulation"):
        _torch()
        import torch
        pin = lambda t: torch.empty(t.shape, dtype=t.dtype).pin_memory()  # noqa: E731
        self.base_prim, self.one_prim = pin(sim.base.prim), pin(sim.one.prim)
        self.flag, self.dt = pin(sim.base.flag), pin(sim.dt)

    @property
    def nbytes(self) -> int:
        return sum(t.numel() * t.element_size()
                   for t in (self.base_prim, self.one_prim, self.flag, self.dt))


class Simulation:
    """A job: packages, mesh, the two stage containers and the dt policy.

    Mirrors Simulator::MakeTaskCollection (ideal_grmhd.cc:23-120) stage by
    stage, with every task on the GPU.
    """

    def __init__(self, pin: ParameterInput, device=0):
        torch = _torch()
        self.pin = pin
        self.packages = process_packages(pin)
        self.params = params_struct(self.packages)
        self.params.precision = engine_precision(pin)
        self.mesh = mesh_struct(pin)
        self.engine = Engine(self.params, self.mesh, device)
        self.base, self.one = self.engine.new_containers()
        dev = self.engine.device
        self.dt_init = pin.get_or_add_real("parthenon/time", "dt_init", 1e-5)
        self.dt_factor = pin.get_or_add_real("parthenon/time", "dt_factor", 2.0)
        self.dt = torch.full((1,), self.dt_init, dtype=torch.float64, device=dev)
        self.dt_est = torch.zeros(1, dtype=torch.float64, device=dev)
        self.cycle = 0
        self._graph = None
        self._copy_streams = None

    def set_primitives(self, prim: np.ndarray):
        """Loads initial primitives (interior values; ghosts are filled here:
        exchange then physical BCs, as Parthenon does after the problem
        generator). Container "1" starts as a copy of "base"."""
        torch = _torch()
        src = torch.as_tensor(prim, device=self.engine.device)
        self.base.prim.copy_(src.to(self.base.prim.dtype))
        self.engine.job_start(0, self.base, self.one)

    def generate(self, name: str):
        """Initial state of the named problem (ot, bw, torus) generated on the
        device from this job's inputfile, then the initial ghost fill."""
        from .problems import problem_struct
        self.base.prim.zero_()
        self.engine.generate(0, problem_struct(name, self.pin), self.base)
        self.engine.job_start(0, self.base, self.one)

    def stage(self, st: int, dt_est=None):
        self.engine.stage(st, self.base, self.one, RK2_BETA[st % 2], self.dt, dt_est)

    def _step_launches(self, fixed_dt: bool):
        self.stage(1)
        self.stage(2, self.dt_est)
        if not fixed_dt:
            self.engine.update_dt(self.dt, self.dt_est, self.dt_factor)

    def autotune(self):
        """Tunes the flux kernels' tile shapes on this job's current state
        (call between cycles). A captured cycle graph holds the old shapes,
        so it is dropped; the next capture() records the tuned launches."""
        self.engine.autotune(self.base)
        self._graph = None

    def capture(self):
        """Captures one RK2 cycle (both stages and the device dt policy) as a
        CUDA graph; later step() calls replay it. Every launch of the cycle is
        stream ordered and reads dt from device memory, so one graph serves
        every step."""
        import torch
        s = torch.cuda.Stream(self.engine.device)
        s.wait_stream(torch.cuda.current_stream(self.engine.device))
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            self._step_launches(False)
        torch.cuda.current_stream(self.engine.device).wait_stream(s)
        self._graph = g

    def step(self, fixed_dt: bool = False):
        """One rk2 cycle; afterwards dt = min(dt_factor * dt, estimate)."""
        if self._graph is not None and not fixed_dt:
            self._graph.replay()
        else:
            self._step_launches(fixed_dt)
        self.cycle += 1

    def pull(self, host: HostState):
        """Copies the job's state to host memory (synchronous)."""
        import torch
        host.base_prim.copy_(self.base.prim)
        host.one_prim.copy_(self.one.prim)
        host.flag.copy_(self.base.flag)
        host.dt.copy_(self.dt)
        torch.cuda.synchronize(self.engine.device)

    def step_host(self, host: HostState, fixed_dt: bool = False):
        """One rk2 cycle of a job whose state lives in pinned host memory: the
        state is copied in, stepped and copied back, with the transfers
        overlapped with the kernels that do not need them and with each
        other (host-to-device and device-to-host run at the same time).
        Container "base" and dt go in first (stage 1 starts from them);
        container "1" and the flags go in on a second stream while stage 1
        runs up to its update (pangu_stage_update: the ghost exchange is their
        first reader). After stage 2's update container "1" is final and goes
        back on a third stream while the rest of stage 2 runs; then the flags
        and dt on that stream and "base" on the main one, which the next
        cycle's inputs of container "1" and the flags overlap. Gives the bits
        of step() on the device-resident state."""
        import torch
        dev = self.engine.device
        s = torch.cuda.current_stream(dev)
        if self._copy_streams is None:
            self._copy_streams = (torch.cuda.Stream(dev), torch.cuda.Stream(dev))
        cin, cout = self._copy_streams
        eng, base, one = self.engine, self.base, self.one
        # the previous cycle's copies back of container "1", the flags and dt
        # (and every kernel that read or wrote them) are complete
        cin.wait_stream(cout)
        s.wait_stream(cout)
        base.prim.copy_(host.base_prim, non_blocking=True)
        self.dt.copy_(host.dt, non_blocking=True)
        with torch.cuda.stream(cin):
            one.prim.copy_(host.one_prim, non_blocking=True)
            base.flag.copy_(host.flag, non_blocking=True)
        eng.stage_update(1, base, one, RK2_BETA[1], self.dt)
        s.wait_stream(cin)
        eng.exchange_ghosts(one)
        eng.stage_middle(1, base, one, RK2_BETA[1], self.dt)
        eng.stage_end(1, base, one, None)
        eng.stage_update(2, base, one, RK2_BETA[0], self.dt)
        cout.wait_stream(s)
        with torch.cuda.stream(cout):
            host.one_prim.copy_(one.prim, non_blocking=True)
        eng.exchange_ghosts(base)
        eng.stage_middle(2, base, one, RK2_BETA[0], self.dt)
        eng.stage_end(2, base, one, None, self.dt_est)
        if not fixed_dt:
            eng.update_dt(self.dt, self.dt_est, self.dt_factor)
        cout.wait_stream(s)
        with torch.cuda.stream(cout):
            host.flag.copy_(base.flag, non_blocking=True)
            host.dt.copy_(self.dt, non_blocking=True)
        host.base_prim.copy_(base.prim, non_blocking=True)
        s.wait_stream(cout)
        self.cycle += 1

    def primitives(self) -> np.ndarray:
        return self.base.prim.double().cpu().numpy()

    def save(self, path: str):
        """Checkpoint of the job between cycles, as one .npz: everything the
        next cycle reads -- both containers' primitives (container "1" holds
        the stale guesses of C2P) and conserved variables (the mixed form
        carries its magnetic field in them), the flags (FixRecovery reads
        ghost flags exchanged in the previous stage), dt and the cycle count --
        with the inputfile text."""
        torch = _torch()
        torch.cuda.synchronize(self.engine.device)
        np.savez(path, base_prim=self.base.prim.cpu().numpy(),
                 one_prim=self.one.prim.cpu().numpy(), base_cons=self.base.cons.cpu().numpy(),
                 one_cons=self.one.cons.cpu().numpy(), flag=self.base.flag.cpu().numpy(),
                 dt=self.dt.cpu().numpy(), cycle=np.int64(self.cycle),
                 inputfile=np.array(self.pin.dump()))

    def write_xdmf(self, prefix: str, time: float = 0.0) -> str:
        """The primitive fields as <prefix>.bin described by <prefix>.xdmf
        (pangu_b200.output)."""
        from .output import write_xdmf
        return write_xdmf(prefix, self.primitives(), self.mesh, bool(self.params.enable_B),
                          bool(self.params.enable_heating), self.cycle, time)

    def write_phdf(self, path: str, time: float = 0.0) -> str:
        """The primitive fields in the Parthenon .phdf layout (needs h5py)."""
        from .output import write_phdf
        return write_phdf(path, self.primitives(), self.mesh, bool(self.params.enable_B),
                          bool(self.params.enable_heating), self.cycle, time)

    @classmethod
    def restart(cls, path: str, device=0) -> "Simulation":
        """A job continued from a checkpoint written by save(): its next
        cycles give the same bits as the uninterrupted run."""
        torch = _torch()
        ck = np.load(path)
        sim = cls(ParameterInput(str(ck["inputfile"])), device=device)
        dev = sim.engine.device
        for name in ("base_prim", "one_prim", "base_cons", "one_cons"):
            cont, field = name.split("_")
            getattr(getattr(sim, cont), field).copy_(torch.as_tensor(ck[name], device=dev))
        sim.base.flag.copy_(torch.as_tensor(ck["flag"], device=dev))
        sim.dt.copy_(torch.as_tensor(ck["dt"], device=dev))
        sim.cycle = int(ck["cycle"])
        return sim


class Pool:
    """Many jobs of one block shape and parameter set (metric spin a and h may
    differ per job) stepped together: every kernel of a stage is one launch
    over the blocks of all attached jobs, through the engine's block table,
    and a whole RK2 cycle of the pool is one CUDA graph replay.

    ``template`` supplies the shared parameters and the block shape
    (<parthenon/meshblock> nx*, nghost). Jobs are attached between cycles.
    """

    # params that may differ between the jobs of a pool
    PER_JOB = ("a", "h")

    def __init__(self, template: ParameterInput, capacity_blocks: int, max_jobs: int, device=0):
        torch = _torch()
        self.params = params_struct(process_packages(template))
        self.params.precision = engine_precision(template)
        block = mesh_struct(template)
        block.nbx1 = block.nbx2 = block.nbx3 = 1
        self.engine = Engine(self.params, block, device, pool=(capacity_blocks, max_jobs))
        self.base, self.one = self.engine.new_containers()
        dev = self.engine.device
        self.dt = torch.zeros(max_jobs, dtype=torch.float64, device=dev)
        self.dt_est = torch.zeros(max_jobs, dtype=torch.float64, device=dev)
        self.dt_factor = template.get_or_add_real("parthenon/time", "dt_factor", 2.0)
        self.capacity, self.max_jobs = capacity_blocks, max_jobs
        self.jobs = {}      # job id -> slots
        self._graph = None

    def free_blocks(self) -> int:
        return self.capacity - sum(len(s) for s in self.jobs.values())

    def _check_compatible(self, p: abi.Params):
        for name, _ in abi.Params._fields_:
            if name in self.PER_JOB:
                continue
            if getattr(p, name) != getattr(self.params, name):
                raise EngineError(f"job parameter {name} differs from the pool's")

    def attach(self, pin: ParameterInput, prim: np.ndarray) -> int:
        """Attaches a job with interior primitives ``prim`` ([block][var][k][j][i],
        numpy or a device tensor), fills its ghosts and sets dt[job] = dt_init."""
        torch = _torch()
        p = params_struct(process_packages(pin))
        p.precision = engine_precision(pin)
        self._check_compatible(p)
        mesh = mesh_struct(pin)
        torch.cuda.synchronize(self.engine.device)  # no pool work in flight
        job, slots = self.engine.attach(mesh, p.a, p.h)
        idx = torch.tensor(slots, dtype=torch.long, device=self.engine.device)
        src = torch.as_tensor(prim, device=self.engine.device).to(self.base.prim.dtype)
        self.base.prim.index_copy_(0, idx, src)
        self.base.cons.index_fill_(0, idx, 0.0)
        self.base.flag.index_fill_(0, idx, 0.0)
        self.dt[job] = pin.get_or_add_real("parthenon/time", "dt_init", 1e-5)
        self.engine.job_start(job, self.base, self.one)
        self.jobs[job] = slots
        self._graph = None
        return job

    def attach_problem(self, pin: ParameterInput, name: str) -> int:
        """Attaches a job whose initial state is generated on the device."""
        from .problems import problem_struct
        torch = _torch()
        p = params_struct(process_packages(pin))
        p.precision = engine_precision(pin)
        self._check_compatible(p)
        torch.cuda.synchronize(self.engine.device)  # no pool work in flight
        job, slots = self.engine.attach(mesh_struct(pin), p.a, p.h)
        idx = torch.tensor(slots, dtype=torch.long, device=self.engine.device)
        for arr in (self.base.prim, self.base.cons):
            arr.index_fill_(0, idx, 0.0)
        self.base.flag.index_fill_(0, idx, 0.0)
        self.dt[job] = pin.get_or_add_real("parthenon/time", "dt_init", 1e-5)
        self.engine.generate(job, problem_struct(name, pin), self.base)
        self.engine.job_start(job, self.base, self.one)
        self.jobs[job] = slots
        self._graph = None
        return job

    def primitives(self, job) -> np.ndarray:
        torch = _torch()
        idx = torch.tensor(self.jobs[job], dtype=torch.long, device=self.engine.device)
        return self.base.prim.index_select(0, idx).double().cpu().numpy()

    def detach(self, job) -> np.ndarray:
        """Detaches a job and returns its primitives."""
        out = self.primitives(job)
        _torch().cuda.synchronize(self.engine.device)  # no pool work in flight
        self.engine.detach(job)
        del self.jobs[job]
        self._graph = None
        return out

    def _cycle(self):
        e = self.engine
        e.stage(1, self.base, self.one, RK2_BETA[1], self.dt)
        e.stage(2, self.base, self.one, RK2_BETA[0], self.dt, self.dt_est)
        e.update_dt(self.dt, self.dt_est, self.dt_factor)

    def autotune(self):
        """Tunes the flux kernels' tile shapes on the attached jobs' state."""
        self.engine.autotune(self.base)
        self._graph = None

    def step(self, graph: bool = True):
        """One RK2 cycle of every attached job."""
        if not self.jobs:
            return
        if not graph:
            self._cycle()
            return
        if self._graph is None:
            import torch
            s = torch.cuda.Stream(self.engine.device)
            s.wait_stream(torch.cuda.current_stream(self.engine.device))
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s):
                self._cycle()
            torch.cuda.current_stream(self.engine.device).wait_stream(s)
            self._graph = g
        self._graph.replay()


class Server:
    """Continuous-batching request loop (pangu_server_*): one block pool per job
    class, jobs admitted at their arrival time as slots free up, every class
    stepped on its own stream, results copied back at completion."""

    def __init__(self, hbm_budget_bytes: int, device=0):
        torch = _torch()
        self.device = torch.device("cuda", device)
        self.L = lib()
        h = _P()
        with torch.cuda.device(self.device):
            _check(self.L.pangu_server_create(int(hbm_budget_bytes), C.byref(h)),
                   "pangu_server_create")
        self.h = h
        self.classes = []   # (params, block mesh, nf, block shape)
        self.tickets = {}   # ticket -> (class, nblocks)

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.pangu_server_destroy(self.h)
            self.h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_class(self, template: ParameterInput, capacity_blocks: int, max_jobs: int,
                  lazy: bool = False) -> int:
        """A job class (the template's parameters and block shape) with a pool
        of `capacity_blocks` block slots for up to `max_jobs` jobs. Its device
        memory is charged against the budget now, or with lazy=True when its
        first job is admitted (and released again while it has nothing to
        run)."""
        params = params_struct(process_packages(template))
        params.precision = engine_precision(template)
        block = mesh_struct(template)
        block.nbx1 = block.nbx2 = block.nbx3 = 1
        factor = template.get_or_add_real("parthenon/time", "dt_factor", 2.0)
        out = C.c_int32()
        fn = "pangu_server_declare_class" if lazy else "pangu_server_add_class"
        _check(getattr(self.L, fn)(self.h, C.byref(params), C.byref(block), int(capacity_blocks),
                                   int(max_jobs), factor, C.byref(out)), fn)
        nf = self.L.pangu_num_fields(C.byref(params))
        act = [block.nx1 > 1, block.nx2 > 1, block.nx3 > 1]
        n = [block.nx1, block.nx2, block.nx3]
        shape = tuple(n[d] + 2 * block.ng * act[d] for d in (2, 1, 0))
        self.classes.append((params, block, nf, shape))
        return out.value

    def submit(self, cls: int, pin: ParameterInput, prim: np.ndarray, cycles: int,
               arrival_s: float) -> int:
        params, _, nf, shape = self.classes[cls]
        p = params_struct(process_packages(pin))
        p.precision = engine_precision(pin)
        for name, _ in abi.Params._fields_:
            if name not in Pool.PER_JOB and getattr(p, name) != getattr(params, name):
                raise EngineError(f"job parameter {name} differs from the class's")
        mesh = mesh_struct(pin)
        arr = np.ascontiguousarray(prim, dtype=np.float64)
        dt_init = pin.get_or_add_real("parthenon/time", "dt_init", 1e-5)
        t = C.c_int32()
        _check(self.L.pangu_server_submit(self.h, cls, C.byref(mesh), p.a, p.h, dt_init,
                                          int(cycles), float(arrival_s),
                                          arr.ctypes.data_as(C.c_void_p), C.byref(t)),
               "pangu_server_submit")
        self.tickets[t.value] = (cls, arr.shape[0])
        return t.value

    def submit_problem(self, cls: int, pin: ParameterInput, name: str, cycles: int,
                       arrival_s: float) -> int:
        """A job whose initial state the server generates on the device at
        admission (no host upload)."""
        from .problems import problem_struct
        params, _, nf, shape = self.classes[cls]
        p = params_struct(process_packages(pin))
        p.precision = engine_precision(pin)
        for name_, _ in abi.Params._fields_:
            if name_ not in Pool.PER_JOB and getattr(p, name_) != getattr(params, name_):
                raise EngineError(f"job parameter {name_} differs from the class's")
        mesh = mesh_struct(pin)
        pb = problem_struct(name, pin)
        dt_init = pin.get_or_add_real("parthenon/time", "dt_init", 1e-5)
        t = C.c_int32()
        _check(self.L.pangu_server_submit_problem(self.h, cls, C.byref(mesh), p.a, p.h, dt_init,
                                                  int(cycles), float(arrival_s), C.byref(pb),
                                                  C.byref(t)), "pangu_server_submit_problem")
        self.tickets[t.value] = (cls, mesh.nbx1 * mesh.nbx2 * mesh.nbx3)
        return t.value

    STATES = ("waiting", "running", "done", "cancelled")

    def cancel(self, ticket: int, at_s: float):
        """Cancels a job at at_s seconds into the run (dropped if still waiting,
        detached at its class's next tick if running; no result)."""
        _check(self.L.pangu_server_cancel(self.h, ticket, float(at_s)), "pangu_server_cancel")

    def state(self, ticket: int) -> str:
        st = self.L.pangu_server_job_state(self.h, ticket)
        _check(min(st, 0), "pangu_server_job_state")
        return self.STATES[st]

    def run(self):
        torch = _torch()
        torch.cuda.synchronize(self.device)
        with torch.cuda.device(self.device):
            _check(self.L.pangu_server_run(self.h), "pangu_server_run")

    def result(self, ticket: int):
        """(primitives [block][var][k][j][i] FP64, (arrival, admission,
        completion) seconds, counters) of a finished job."""
        cls, nb = self.tickets[ticket]
        _, _, nf, shape = self.classes[cls]
        out = np.empty((nb, nf) + shape, dtype=np.float64)
        times = np.empty(3, dtype=np.float64)
        cnt = (C.c_uint64 * abi.NCOUNTERS)()
        _check(self.L.pangu_server_result(self.h, ticket, out.ctypes.data_as(C.c_void_p),
                                          times.ctypes.data_as(C.c_void_p), cnt),
               "pangu_server_result")
        return out, times, np.array(list(cnt), dtype=np.uint64)

    def stats(self) -> dict:
        st = abi.ServerStats()
        _check(self.L.pangu_server_get_stats(self.h, C.byref(st)), "pangu_server_get_stats")
        return {name: getattr(st, name) for name, _ in abi.ServerStats._fields_}
