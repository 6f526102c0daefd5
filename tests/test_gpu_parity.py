"""GPU parity: every task of the stage, and whole RK2 steps, on the engine
(through the C ABI) against the CPU oracle on the same inputs.

Per-task checks resynchronise the engine to the oracle's state before each
task, so each comparison sees identical inputs. The FP64 engine rounds every
operation as the oracle does (no contraction, the oracle's operation order,
the metric tables holding the dense values bit for bit, the shared pow), so
every task is compared bit for bit over the whole index domain, and so are
whole RK2 steps (primitives, conserved variables, flags, dt, counters). The
FP64 accuracy targets (relative L1 <= 1e-12 after one step, <= 1e-9 after
ten) are asserted as well, as a statement of their own.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
from parity_util import CASES, Case, div_b_corner, field, interior, rel_l1, to_device  # noqa: E402

pytestmark = pytest.mark.gpu

TASK_CASES = ["ot_mc_laxf", "ot_ppm4_hll_heat", "ot_blocks", "bw_hll", "torus_ppm4_laxf",
              "torus_mc_hll", "torus_robuster", "torus_kawazura", "torus3d_blocks",
              "torus3d_hll", "torus_bl", "cks_excise"]


def _engine(case):
    from pangu_b200.engine import Engine
    eng = Engine(case.params, case.mesh)
    base, one = eng.new_containers()
    return eng, base, one


def _close(a, b, what=""):
    """Bit for bit; on failure the message gives the count and the largest
    relative difference."""
    same = (a == b) | (np.isnan(a) & np.isnan(b))
    if not same.all():
        d = np.abs(a - b)[~same] / np.maximum(np.abs(b)[~same], 1e-300)
        raise AssertionError(f"{what}: {int((~same).sum())} values differ, max rel {d.max():.3e}")


@pytest.mark.parametrize("name", TASK_CASES)
def test_tasks_match_oracle(name):
    case = Case(name)
    O = case.oracle
    eng, dbase, done = _engine(case)
    hbase, hone = case.oracle_containers()
    # initial ghost fill on the device as well
    dbase.prim.copy_(torch.from_numpy(case.prim0))
    eng.exchange_ghosts(dbase)
    eng.apply_boundary_conditions(dbase)
    np.testing.assert_array_equal(field(dbase, "prim"), hbase.prim)

    p = case.params
    dt = 1e-3 if case.mesh.nx2 > 1 else 5e-4
    dt_dev = torch.full((1,), dt, dtype=torch.float64, device="cuda")
    for stage in (1, 2):
        beta = 0.5 if stage == 1 else 1.0
        h0, h1 = (hbase, hone) if stage == 1 else (hone, hbase)
        d0, d1 = (dbase, done) if stage == 1 else (done, dbase)

        def sync():
            to_device(hbase, dbase)
            to_device(hone, done)

        sync()
        O.fix_primitive(h0)
        eng.fix_primitive(d0)
        _close(field(d0, "prim"), h0.prim, what=f"{name} s{stage} FixPrimitive")
        sync()
        O.calculate_conservative(h0)
        eng.calculate_conservative(d0)
        _close(interior(case.geo, field(d0, "cons")), interior(case.geo, h0.cons),
               what=f"{name} s{stage} CalculateConservative")
        sync()
        O.calculate_fluxes(h0)
        eng.calculate_fluxes(d0)
        for f in ("flux1", "flux2", "flux3"):
            _close(field(d0, f), getattr(h0, f), what=f"{name} s{stage} {f}")
        _close(field(d0, "alfven"), h0.alfven, what=f"{name} s{stage} alfven")
        if p.enable_B:
            sync()
            O.constrained_transport(h0)
            eng.constrained_transport(d0)
            for f in ("flux1", "flux2", "flux3", "efield"):
                np.testing.assert_array_equal(field(d0, f), getattr(h0, f), err_msg=f"CT {f}")
        sync()
        O.flux_divergence_update(hbase, h0, h1, beta * dt)
        eng.flux_divergence_update(dbase, d0, d1, beta, dt_dev)
        np.testing.assert_array_equal(interior(case.geo, field(d1, "cons")),
                                      interior(case.geo, h1.cons), err_msg="update")
        sync()
        O.exchange_ghosts(h1)
        eng.exchange_ghosts(d1)
        np.testing.assert_array_equal(field(d1, "prim"), h1.prim, err_msg="exchange prim")
        np.testing.assert_array_equal(field(d1, "flag"), h1.flag, err_msg="exchange flag")
        sync()
        O.add_geometric_source(h1, beta * dt)
        eng.add_geometric_source(d1, beta, dt_dev)
        _close(interior(case.geo, field(d1, "cons")), interior(case.geo, h1.cons),
               what=f"{name} s{stage} AddGeometricSource")
        sync()
        O.reset_counters()
        eng.reset_counters()
        O.recovery(h1)
        eng.recovery(d1)
        _close(field(d1, "prim"), h1.prim, what=f"{name} s{stage} Recovery")
        if p.recovery == 0:
            np.testing.assert_array_equal(field(d1, "flag"), h1.flag, err_msg="recovery flag")
        np.testing.assert_array_equal(eng.counters(), O.counters(), err_msg="C2P counters")
        if p.enable_heating:
            sync()
            O.apply_electron_heating(h1)
            eng.apply_electron_heating(d1)
            _close(field(d1, "prim"), h1.prim, what=f"{name} s{stage} ApplyElectronHeating")
        if p.recovery == 0:
            sync()
            O.fix_recovery(h1)
            eng.fix_recovery(d1)
            np.testing.assert_array_equal(field(d1, "prim"), h1.prim, err_msg="FixRecovery prim")
            np.testing.assert_array_equal(field(d1, "flag"), h1.flag, err_msg="FixRecovery flag")
        sync()
        O.apply_boundary_conditions(h1)
        eng.apply_boundary_conditions(d1)
        np.testing.assert_array_equal(field(d1, "prim"), h1.prim, err_msg="BCs prim")
        np.testing.assert_array_equal(field(d1, "flag"), h1.flag, err_msg="BCs flag")
    sync()
    est_h = O.estimate_dt(hbase)
    est_d = torch.zeros(1, dtype=torch.float64, device="cuda")
    eng.estimate_dt(dbase, est_d)
    assert est_d.item() == est_h


STEP_CASES = ["ot_mc_laxf", "bw_hll", "torus_ppm4_laxf", "torus_mc_hll", "torus3d_blocks",
              "torus_robuster", "cks_excise"]


def _run_both(case, nsteps, fixed_dt):
    from pangu_b200.engine import Engine
    O = case.oracle
    hbase, hone = case.oracle_containers()
    eng = Engine(case.params, case.mesh)
    dbase, done = eng.new_containers()
    to_device(hbase, dbase)
    to_device(hone, done)
    dt_h = 1e-3 if case.mesh.nx2 > 1 else 5e-4
    dt_d = torch.full((1,), dt_h, dtype=torch.float64, device="cuda")
    est_d = torch.zeros(1, dtype=torch.float64, device="cuda")
    factor = 1.3
    O.reset_counters()
    eng.reset_counters()
    for _ in range(nsteps):
        O.stage(1, hbase, hone, 0.5, dt_h)
        est_h = O.stage(2, hbase, hone, 1.0, dt_h)
        eng.stage(1, dbase, done, 0.5, dt_d)
        eng.stage(2, dbase, done, 1.0, dt_d, est_d)
        if not fixed_dt:
            dt_h = min(factor * dt_h, est_h)
            eng.update_dt(dt_d, est_d, factor)
    torch.cuda.synchronize()
    return O, eng, hbase, dbase, dt_h, dt_d.item()


def _counters_close(c_eng, c_or):
    np.testing.assert_array_equal(c_eng, c_or, err_msg="counters")


@pytest.mark.parametrize("name", STEP_CASES)
def test_one_step(name):
    case = Case(name)
    O, eng, hb, db, dth, dtd = _run_both(case, 1, fixed_dt=True)
    l1 = rel_l1(interior(case.geo, field(db, "cons")), interior(case.geo, hb.cons))
    assert np.all(l1 <= 1e-12), f"{name}: cons rel L1 after 1 step {l1}"
    for f in ("prim", "cons", "flag"):
        _close(field(db, f), getattr(hb, f), what=f"{name} one step {f}")
    _counters_close(eng.counters(), O.counters())


@pytest.mark.parametrize("name", STEP_CASES)
def test_ten_steps(name):
    case = Case(name)
    O, eng, hb, db, dth, dtd = _run_both(case, 10, fixed_dt=False)
    assert dtd == dth
    l1 = rel_l1(interior(case.geo, field(db, "cons")), interior(case.geo, hb.cons))
    assert np.all(l1 <= 1e-9), f"{name}: cons rel L1 after 10 steps {l1}"
    for f in ("prim", "cons", "flag"):
        _close(field(db, f), getattr(hb, f), what=f"{name} ten steps {f}")
    _counters_close(eng.counters(), O.counters())


def test_div_b_kept_at_roundoff():
    """Corner divergence of sqrt(g) B is unchanged by ten steps (flux-CT)."""
    case = Case("ot_mc_laxf")
    from pangu_b200.engine import Simulation
    sim = Simulation(case.pin)
    sim.set_primitives(case.prim0)
    sim.stage(1)
    sim.stage(2, sim.dt_est)
    div0 = div_b_corner(case.geo, field(sim.base, "cons"))
    for _ in range(10):
        sim.step()
    div1 = div_b_corner(case.geo, field(sim.base, "cons"))
    bmax = np.abs(field(sim.base, "cons")[:, 5:7]).max()
    assert np.abs(div1 - div0).max() <= 1e-12 * bmax / min(case.geo.dx[:2])


@pytest.mark.parametrize("name", ["torus_ppm4_laxf", "ot_blocks"])
def test_graph_replay_matches_launches(name):
    """A captured RK2 cycle replayed as a CUDA graph gives bit-identical
    states, counters and dt to the same cycles launched from the host."""
    from pangu_b200.engine import Simulation
    case = Case(name)
    a = Simulation(case.pin)
    b = Simulation(case.pin)
    a.set_primitives(case.prim0)
    b.set_primitives(case.prim0)
    b.capture()
    for _ in range(6):
        a.step()
        b.step()
    torch.cuda.synchronize()
    for f in ("prim", "cons", "flag", "alfven"):
        np.testing.assert_array_equal(field(a.base, f), field(b.base, f), err_msg=f)
        np.testing.assert_array_equal(field(a.one, f), field(b.one, f), err_msg=f)
    assert a.dt.item() == b.dt.item()
    np.testing.assert_array_equal(a.engine.counters(), b.engine.counters())


@pytest.mark.parametrize("name", ["torus_ppm4_laxf", "torus3d_hll"])
def test_autotune_keeps_results(name):
    """The flux tile shapes the autotuner picks change no result: a tuned and
    an untuned engine give bit-identical states after four RK2 cycles."""
    from pangu_b200.engine import Simulation
    case = Case(name)
    a = Simulation(case.pin)
    b = Simulation(case.pin)
    a.set_primitives(case.prim0)
    b.set_primitives(case.prim0)
    b.autotune()
    cfg = b.engine.flux_config()
    assert cfg["tuned"] and cfg["x1_threads"] in (64, 128) and cfg["x2_march"] in (0, 1, 2, 4, 8)
    b.set_primitives(case.prim0)  # the tuning overwrote fluxes only; restart both
    for _ in range(4):
        a.step()
        b.step()
    torch.cuda.synchronize()
    for f in ("prim", "cons", "flag"):
        np.testing.assert_array_equal(field(a.base, f), field(b.base, f), err_msg=f)
