"""Checkpoint and restart (Simulation.save / Simulation.restart): a job
stopped after three RK2 cycles, written to disk and continued in a new engine
gives the same bits after three more cycles as the uninterrupted run, in
both precisions."""
import numpy as np
import pytest

from parity_util import Case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,precision", [("torus_ppm4_laxf", "fp64"),
                                            ("torus_ppm4_laxf", "mixed"),
                                            ("ot_blocks", "fp64")])
def test_restart_is_bit_exact(tmp_path, name, precision):
    import torch
    from pangu_b200.engine import Simulation
    case = Case(name)
    case.pin.set("b200", "precision", precision)
    ref = Simulation(case.pin)
    ref.set_primitives(case.prim0)
    for _ in range(6):
        ref.step()
    a = Simulation(case.pin)
    a.set_primitives(case.prim0)
    for _ in range(3):
        a.step()
    path = str(tmp_path / "ck.npz")
    a.save(path)
    del a
    b = Simulation.restart(path)
    assert b.cycle == 3
    for _ in range(3):
        b.step()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(b.primitives(), ref.primitives())
    assert b.dt.item() == ref.dt.item()
