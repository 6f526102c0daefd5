"""The reference's task functions served by the engine
(pangu_b200/parthenon/b200_tasks.cc) on Parthenon MeshData objects.

The shim is compiled with the test driver tests/parthenon_shim/driver.cc
against the host-only Parthenon stand-in (oracle/refshim), which addresses
each variable of each block through Get(name) as Parthenon does; the test
allocates every (block, variable) as its own device array (Parthenon's
layout, not the engine's contiguous one). Two RK2 cycles run task by task in
ideal_grmhd.cc:62-110 order: the reference's tasks through the shim, the
update, ghost exchange and boundaries (Parthenon's own tasks) through the C
ABI on the same per-variable arrays. After every step each array equals, bit
for bit, the engine's contiguous run of the same step, and every dt estimate
is equal.

Mesh extents are dyadic, so that the per-block extents the shim derives from
each MeshBlock's face coordinates reproduce the block's coordinates exactly.
"""
import ctypes as C
import importlib.util
import os

import numpy as np
import pytest

from parity_util import Case, to_device

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIELDS = ("prim", "cons", "flux1", "flux2", "flux3", "alfven", "efield", "flag")
TASK = {"fix_primitive": 0, "calculate_conservative": 1, "calculate_fluxes": 2,
        "constrained_transport": 3, "add_geometric_source": 4, "recovery": 5,
        "apply_electron_heating": 6, "fix_recovery": 7, "estimate_dt": 8}

# case name -> input settings making every extent and cell width dyadic
DYADIC = {
    "ot_blocks": {},
    "ot_ppm4_hll_heat": {},
    "torus_ppm4_laxf": {("parthenon/mesh", "x1min"): 0.25, ("parthenon/mesh", "x1max"): 6.25,
                        ("parthenon/mesh", "x3min"): -3.0, ("parthenon/mesh", "x3max"): 3.0},
    "torus_robuster": {("parthenon/mesh", "x1min"): 0.25, ("parthenon/mesh", "x1max"): 6.25,
                       ("parthenon/mesh", "x2min"): -0.75, ("parthenon/mesh", "x2max"): 0.75,
                       ("parthenon/mesh", "x3min"): -3.0, ("parthenon/mesh", "x3max"): 3.0},
    "torus_kawazura": {("parthenon/mesh", "x1min"): 0.25, ("parthenon/mesh", "x1max"): 6.25,
                       ("parthenon/mesh", "x2min"): -0.75, ("parthenon/mesh", "x2max"): 0.75,
                       ("parthenon/mesh", "x3min"): -3.0, ("parthenon/mesh", "x3max"): 3.0},
    "torus3d_hll": {("parthenon/mesh", "x1min"): 0.25, ("parthenon/mesh", "x1max"): 6.25,
                    ("parthenon/mesh", "x3min"): -3.0, ("parthenon/mesh", "x3max"): 3.0},
    "cks_excise": {("parthenon/mesh", f"x{d}{e}"): v for d in (1, 2, 3)
                   for e, v in (("min", -4.0), ("max", 4.0))},
}


def _shim():
    spec = importlib.util.spec_from_file_location(
        "parthenon_shim_build", os.path.join(HERE, "parthenon_shim", "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    L = C.CDLL(mod.build())
    L.shim_make.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_int)]
    L.shim_run.argtypes = [C.c_int, C.c_int, C.c_double, C.POINTER(C.c_double)]
    L.shim_num_prim_vars.argtypes = [C.c_void_p]
    return L


def _prim_groups(params):
    g = [1, 1, 3]
    if params.enable_B:
        g.append(3)
    g.append(1)
    if params.enable_heating:
        g.append(1)
    return tuple(g)


def _pointers(L, params, mesh, tab):
    """Per block: each primitive variable, conservative, its three face
    fluxes (0 where inactive), alfven, electric_field, flag (0 without the
    chainer)."""
    active = (True, mesh.nx2 > 1, mesh.nx3 > 1)
    chainer = params.recovery == 0
    out = []
    for b in range(tab.nb):
        out += [t.data_ptr() for t in tab.arrays["prim"][b]]
        out.append(tab.arrays["cons"][b][0].data_ptr())
        for d, f in enumerate(("flux1", "flux2", "flux3")):
            out.append(tab.arrays[f][b][0].data_ptr() if active[d] else 0)
        out.append(tab.arrays["alfven"][b][0].data_ptr())
        out.append(tab.arrays["efield"][b][0].data_ptr())
        out.append(tab.arrays["flag"][b][0].data_ptr() if chainer else 0)
    assert len(out) == tab.nb * (L.shim_num_prim_vars(C.byref(params)) + 7)
    return (C.c_uint64 * len(out))(*out)


def _same(dev, tab, what):
    import torch
    torch.cuda.synchronize()
    for f in FIELDS:
        a = getattr(dev, f).cpu().numpy()
        b = tab.gather(f).cpu().numpy()
        np.testing.assert_array_equal(a.view(np.uint8), b.view(np.uint8), err_msg=f"{what} {f}")


@pytest.mark.parametrize("name", list(DYADIC))
def test_shim_tasks_on_parthenon_layout_equal_engine(name):
    import torch

    import task_golden as tg
    from pangu_b200.engine import Engine, TableContainer
    case = Case(name, DYADIC[name])
    params, mesh = case.params, case.mesh
    L = _shim()
    hb, ho = case.oracle_containers()
    E = Engine(params, mesh, device=0)
    db, do = E.new_containers()
    to_device(hb, db)
    to_device(ho, do)
    groups = (_prim_groups(params), (E.nf,))
    tb = TableContainer(E.nb, E.nf, E.shape, E.device, *groups)
    to = TableContainer(E.nb, E.nf, E.shape, E.device, *groups, shared=tb)
    tb.load(db)
    to.load(do)
    handles = []
    for t in (tb, to):
        h = C.c_int(-1)
        assert L.shim_make(C.byref(params), C.byref(mesh), _pointers(L, params, mesh, t),
                           C.byref(h)) == 0
        handles.append(h.value)
    dt = 1e-3 if mesh.nx2 > 1 else 2e-3
    dt_d = torch.full((1,), dt, dtype=torch.float64, device=E.device)
    est_d = torch.zeros(1, dtype=torch.float64, device=E.device)
    checked = 0
    try:
        for cycle in range(2):
            for st, beta in ((1, 0.5), (2, 1.0)):
                cd = (db, do) if st == 1 else (do, db)
                ct = (tb, to) if st == 1 else (to, tb)
                hs = (handles[0], handles[1]) if st == 1 else (handles[1], handles[0])
                for step, which in tg.stage_steps(params, st):
                    if step == "update":
                        E.flux_divergence_update(db, cd[0], cd[1], beta, dt_d)
                        E.flux_divergence_update(tb, ct[0], ct[1], beta, dt_d)
                        _same(cd[1], ct[1], f"{cycle} {st} update")
                        continue
                    dev, tab, h = cd[which], ct[which], hs[which]
                    if step == "exchange":
                        E.exchange_ghosts(dev)
                        E.exchange_ghosts(tab)
                    elif step == "bcs":
                        E.apply_boundary_conditions(dev)
                        E.apply_boundary_conditions(tab)
                    elif step == "estimate_dt":
                        E.estimate_dt(dev, est_d)
                        got = C.c_double(0.0)
                        assert L.shim_run(h, TASK[step], 0.0, C.byref(got)) == 0
                        assert got.value == est_d.item(), (cycle, st)
                        dt = min(2.0 * dt, got.value)
                        dt_d.fill_(dt)
                    elif step == "add_geometric_source":
                        E.add_geometric_source(dev, beta, dt_d)
                        assert L.shim_run(h, TASK[step], beta * dt, None) == 0
                    else:
                        getattr(E, step)(dev)
                        assert L.shim_run(h, TASK[step], 0.0, None) == 0, step
                    _same(dev, tab, f"{cycle} {st} {step}")
                    checked += 1
    finally:
        L.shim_free_all()
    assert checked >= 20


def test_shim_task_on_a_missing_variable_fails():
    """A MeshData without the flag variable under the chainer recovery: the
    task reports TaskStatus::fail (no launch, no exception through the
    task)."""
    import torch

    from pangu_b200.engine import TableContainer
    case = Case("ot_blocks")
    params, mesh = case.params, case.mesh
    assert params.recovery == 0
    L = _shim()
    nf = int(sum(_prim_groups(params)))
    act = [mesh.nx1 > 1, mesh.nx2 > 1, mesh.nx3 > 1]
    n = [mesh.nx1, mesh.nx2, mesh.nx3]
    shape = tuple(n[d] + 2 * mesh.ng * act[d] for d in (2, 1, 0))
    nb = mesh.nbx1 * mesh.nbx2 * mesh.nbx3
    tab = TableContainer(nb, nf, shape, torch.device("cuda", 0), _prim_groups(params), (nf,))
    ptrs = _pointers(L, params, mesh, tab)
    per = len(ptrs) // nb
    for b in range(nb):
        ptrs[b * per + per - 1] = 0  # no flag arrays: Get("flag") finds nothing
    h = C.c_int(-1)
    try:
        assert L.shim_make(C.byref(params), C.byref(mesh), ptrs, C.byref(h)) == 0
        assert L.shim_run(h.value, TASK["recovery"], 0.0, None) != 0
    finally:
        L.shim_free_all()
