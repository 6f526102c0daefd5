"""A job whose state lives in pinned host memory (HostState, step_host):
the overlapped copies in and out (piece by piece, each piece going back in
as soon as it has come out, with two device copies of container "1" used in
turn) give, cycle after cycle, the same bits as stepping the device-resident
state, in FP64 and in the mixed form, with and without block-to-block ghost
exchange, and device-resident and host-resident cycles may alternate."""
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
    # and host-resident ones again, from the state pulled back to the host
    # (an odd number of cycles, so the two device copies of container "1"
    # have swapped roles)
    sim.pull(host)
    for _ in range(3):
        ref.step()
        sim.step_host(host)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(host.base_prim.double().numpy(), ref.primitives())
    np.testing.assert_array_equal(host.one_prim.numpy(), ref.one.prim.cpu().numpy())
    assert host.dt.item() == ref.dt.item()
    np.testing.assert_array_equal(sim.primitives(), ref.primitives())
    np.testing.assert_array_equal(sim.one.prim.cpu().numpy(), ref.one.prim.cpu().numpy())
