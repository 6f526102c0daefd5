"""A job whose state lives in pinned host memory (HostState, step_host):
the overlapped copies in and out give, cycle after cycle, the same bits as
stepping the device-resident state, in FP64 and in the mixed form, with and
without block-to-block ghost exchange."""
import numpy as np
import pytest

from parity_util import Case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,precision", [("torus_ppm4_laxf", "fp64"),
                                            ("torus_ppm4_laxf", "mixed"),
                                            ("ot_blocks", "fp64"), ("torus3d_blocks", "fp64")])
def test_host_resident_cycles_match_device_cycles(name, precision):
    import torch
    from pangu_b200.engine import HostState, Simulation
    case = Case(name)
    case.pin.set("b200", "precision", precision)
    ref = Simulation(case.pin)
    ref.set_primitives(case.prim0)
    sim = Simulation(case.pin)
    sim.set_primitives(case.prim0)
    host = HostState(sim)
    sim.pull(host)
    for _ in range(4):
        ref.step()
        sim.step_host(host)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(host.base_prim.double().numpy(), ref.primitives())
    np.testing.assert_array_equal(host.one_prim.numpy(), ref.one.prim.cpu().numpy())
    np.testing.assert_array_equal(host.flag.numpy(), ref.base.flag.cpu().numpy())
    assert host.dt.item() == ref.dt.item()
    assert sim.cycle == ref.cycle == 4
    # device-resident cycles may follow host-resident ones
    for _ in range(2):
        ref.step()
        sim.step()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(sim.primitives(), ref.primitives())
