"""Parity at the benchmark sizes: the engine against the CPU oracle on the
full workloads that bench.py measures (512x256 torus, 256^2 Orszag-Tang,
256x128x128 torus in 16 blocks of 64^3), whole RK2 cycles with the dynamic dt
policy. FP64 is bit-identical: primitives, conserved variables and flags
over every cell, dt and every counter. The mixed form at full size stays
within its tolerances (density 1e-5) after the same cycles."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _oracle_run(pin, prim0, cycles):
    import pyoracle as po
    from pangu_b200 import params as prm
    po.set_threads(os.cpu_count() or 1)
    pk = prm.process_packages(pin)
    O = po.Oracle(prm.params_struct(pk), prm.mesh_struct(pin))
    base, one = O.new_containers()
    base.prim[...] = prim0
    O.exchange_ghosts(base)
    O.apply_boundary_conditions(base)
    one.prim[...] = base.prim
    one.cons[...] = base.cons
    dt = pin.get_or_add_real("parthenon/time", "dt_init", 1e-5)
    factor = pin.get_or_add_real("parthenon/time", "dt_factor", 2.0)
    O.reset_counters()
    for _ in range(cycles):
        dt = min(factor * dt, O.step(base, one, dt))
    return O, base, dt


def _engine_run(pin, prim0, cycles):
    import torch
    from pangu_b200.engine import Simulation
    sim = Simulation(pin)
    sim.set_primitives(prim0)
    sim.engine.reset_counters()
    for _ in range(cycles):
        sim.step()
    torch.cuda.synchronize()
    return sim


@pytest.mark.parametrize("workload,cycles", [("torus2d", 3), ("ot", 3), ("torus3d", 1)])
def test_fullsize_fp64_bit_identical(workload, cycles):
    import bench
    pin = bench.job_input(workload, "fp64")
    _, _, _, prim0 = bench.initial_state(pin)
    sim = _engine_run(pin, prim0, cycles)
    O, hbase, dt = _oracle_run(pin, prim0, cycles)
    for name in ("prim", "cons", "flag"):
        np.testing.assert_array_equal(getattr(sim.base, name).cpu().numpy(),
                                      getattr(hbase, name), err_msg=name)
    assert sim.dt.item() == dt
    np.testing.assert_array_equal(sim.engine.counters(), O.counters())


@pytest.mark.parametrize("workload", ["torus2d", "ot"])
def test_fullsize_mixed_within_tolerance(workload):
    import bench
    pin = bench.job_input(workload, "fp64")
    _, _, geo, prim0 = bench.initial_state(pin)
    err = bench.error_vs_fp64(pin, prim0, geo, 10)["rel_l1"]
    assert err["density"] <= 1e-5, err
    assert all(v <= 1e-2 for v in err.values()), err
