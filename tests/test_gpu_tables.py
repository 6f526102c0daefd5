"""The per-(block, component) pointer tables of pangu_pack: packs whose
arrays are separate device allocations per block and variable (Parthenon's
layout) give bit-identical results to the contiguous layout.

* Whole RK2 cycles through pangu_stage (which runs every task, the update,
  the ghost exchange, the physical boundaries and the dt estimate) on table
  packs with one allocation per (block, component), against the contiguous
  packs, on seven configurations (MKS/Minkowski/CKS, PPM4/MC, LAXF/HLL,
  chainer/robuster, heating, 2D/3D, several blocks).
* Packs mixing both layouts, field by field.
* The mixed-precision form (FP32 primitives behind the table), to rounding.
* A CUDA graph captured on table packs and replayed.
* The TMA-staged flux kernels are replaced by their thread-loaded forms when
  the primitives come through a table; the results do not change.
"""
import numpy as np
import pytest

from parity_util import Case, to_device

pytestmark = pytest.mark.gpu

FIELDS = ("prim", "cons", "flux1", "flux2", "flux3", "alfven", "efield", "flag")


def _worlds(case_name, contiguous=(), precision=None, groups=None):
    import torch

    from pangu_b200 import abi
    from pangu_b200.engine import Engine, TableContainer
    case = Case(case_name)
    params = case.params
    if precision is not None:
        params.precision = abi.PRECISION[precision]
    hb, ho = case.oracle_containers()
    E = Engine(params, case.mesh, device=0)
    db, do = E.new_containers()
    if E.mixed:
        for h, dv in ((hb, db), (ho, do)):
            for f in FIELDS:
                src = torch.from_numpy(np.ascontiguousarray(getattr(h, f)))
                getattr(dv, f).copy_(src.to(getattr(dv, f).dtype))
    else:
        to_device(hb, db)
        to_device(ho, do)
    pg, cg = groups if groups else (None, None)
    tb = TableContainer(E.nb, E.nf, E.shape, E.device, pg, cg, contiguous=contiguous,
                        mixed=E.mixed)
    to = TableContainer(E.nb, E.nf, E.shape, E.device, pg, cg, shared=tb,
                        contiguous=contiguous, mixed=E.mixed)
    tb.load(db)
    to.load(do)
    return case, E, (db, do), (tb, to)


def _same(dev, tab, what):
    import torch
    torch.cuda.synchronize()
    for f in FIELDS:
        a = getattr(dev, f).cpu().numpy()
        b = tab.gather(f).cpu().numpy()
        assert a.shape == b.shape, (what, f)
        np.testing.assert_array_equal(a.view(np.uint8), b.view(np.uint8), err_msg=f"{what} {f}")


def _cycles(E, dev, tab, n, dt0):
    import torch
    dt = torch.full((1,), dt0, dtype=torch.float64, device=E.device)
    est_d = torch.zeros(1, dtype=torch.float64, device=E.device)
    est_t = torch.zeros(1, dtype=torch.float64, device=E.device)
    for c in range(n):
        for st, beta in ((1, 0.5), (2, 1.0)):
            E.stage(st, dev[0], dev[1], beta, dt, est_d if st == 2 else None)
            E.stage(st, tab[0], tab[1], beta, dt, est_t if st == 2 else None)
        _same(dev[0], tab[0], f"cycle {c}")
        torch.cuda.synchronize()
        assert est_d.item() == est_t.item(), c
        dt.copy_(torch.minimum(2.0 * dt, est_d))


@pytest.mark.parametrize("name", ["torus_ppm4_laxf", "ot_blocks", "torus3d_hll", "torus_robuster",
                                  "ot_ppm4_hll_heat", "cks_excise", "torus_kawazura"])
def test_stage_on_per_component_tables_is_bit_identical(name):
    case, E, dev, tab = _worlds(name)
    _cycles(E, dev, tab, 3, 5e-4 if case.mesh.nx2 > 1 else 1e-3)


@pytest.mark.parametrize("contiguous", [("cons", "flux1", "flux2", "flux3"),
                                        ("prim", "alfven", "flag"),
                                        ("efield", "flux2")])
def test_packs_mixing_tables_and_contiguous_arrays(contiguous):
    case, E, dev, tab = _worlds("torus_ppm4_laxf", contiguous=contiguous)
    _cycles(E, dev, tab, 2, 5e-4)


def test_parthenon_variable_groups():
    """Components of a variable contiguous, variables apart (density,
    energy, weighted_velocity[3], magnetic_field[3], entropy,
    electron_entropy, and the conserved variables as one allocation)."""
    case = Case("torus3d_blocks")
    assert case.params.enable_B and case.params.enable_heating
    case, E, dev, tab = _worlds("torus3d_blocks", groups=((1, 1, 3, 3, 1, 1), (10,)))
    _cycles(E, dev, tab, 2, 5e-4)


def test_tables_must_cover_every_component():
    import torch

    from pangu_b200.engine import TableContainer
    with pytest.raises(ValueError):
        TableContainer(2, 10, (1, 8, 8), torch.device("cuda", 0), (1, 1, 3, 3, 1), (10,))


def test_mixed_precision_on_tables():
    """The mixed form is compiled with FMA contraction, and its table
    instantiation is a separate unit whose contraction choices may differ in
    the last bit: the two layouts agree to rounding, not bit for bit."""
    import torch

    from parity_util import rel_l1
    case, E, dev, tab = _worlds("torus_ppm4_laxf", precision="mixed")
    dt = torch.full((1,), 5e-4, dtype=torch.float64, device=E.device)
    for _ in range(2):
        for st, beta in ((1, 0.5), (2, 1.0)):
            E.stage(st, dev[0], dev[1], beta, dt)
            E.stage(st, tab[0], tab[1], beta, dt)
    torch.cuda.synchronize()
    for f in ("prim", "cons"):
        a = getattr(dev[0], f).double().cpu().numpy()
        b = tab[0].gather(f).double().cpu().numpy()
        assert np.all(rel_l1(b, a) <= 1e-9), (f, rel_l1(b, a))


def test_graph_replay_on_tables():
    import torch
    case, E, dev, tab = _worlds("ot_blocks")
    dt = torch.full((1,), 5e-4, dtype=torch.float64, device=E.device)
    est = torch.zeros(1, dtype=torch.float64, device=E.device)
    s = torch.cuda.Stream(E.device)
    s.wait_stream(torch.cuda.current_stream(E.device))
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        E.stage(1, tab[0], tab[1], 0.5, dt)
        E.stage(2, tab[0], tab[1], 1.0, dt, est)
    torch.cuda.current_stream(E.device).wait_stream(s)
    # capture launched nothing: both worlds still hold the same state
    _same(dev[0], tab[0], "after capture")
    for c in range(3):
        E.stage(1, dev[0], dev[1], 0.5, dt)
        E.stage(2, dev[0], dev[1], 1.0, dt)
        g.replay()
        _same(dev[0], tab[0], f"replay {c}")


def test_tma_flux_config_falls_back_on_tables():
    from pangu_b200 import engine as eng
    case, E, dev, tab = _worlds("torus_ppm4_laxf")
    try:
        E.set_flux_config(x1_march=8, x1_threads=128, x2_march=8, x2_threads=128)
    except eng.EngineError:
        pytest.skip("the TMA-staged flux kernels are not available for this shape")
    E.calculate_fluxes(dev[0])
    E.calculate_fluxes(tab[0])
    _same(dev[0], tab[0], "fluxes")
    assert not E.device_error()


def test_table_pack_without_an_array_is_rejected():
    import ctypes as C

    import torch

    from pangu_b200 import abi
    case, E, dev, tab = _worlds("torus_ppm4_laxf")
    bad = abi.Pack.from_buffer_copy(tab[0]._pack)
    bad.cons_vars = None  # and cons is not given contiguously either
    assert E.L.pangu_fix_primitive(E.h, C.byref(bad), None) == abi.PANGU_EINVAL
    torch.cuda.synchronize()
