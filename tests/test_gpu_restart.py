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


def test_xdmf_output_of_a_running_job(tmp_path):
    """Simulation.write_xdmf after some cycles: the binary holds the
    interior density of every block as the job has it on the device."""
    import xml.etree.ElementTree as ET
    import torch
    from pangu_b200.engine import Simulation
    case = Case("ot_blocks")
    sim = Simulation(case.pin)
    sim.set_primitives(case.prim0)
    for _ in range(2):
        sim.step()
    torch.cuda.synchronize()
    path = sim.write_xdmf(str(tmp_path / "ot"))
    root = ET.parse(path).getroot()
    coll = root.find("Domain").find("Grid")
    assert coll.find("Information").get("Value") == "2"
    raw = open(str(tmp_path / "ot.bin"), "rb").read()
    prim = sim.primitives()
    s = case.geo.interior()
    for b, g in enumerate(coll.findall("Grid")):
        di = [a for a in g.findall("Attribute") if a.get("Name") == "density"][0].find("DataItem")
        dims = [int(x) for x in di.get("Dimensions").split()]
        got = np.frombuffer(raw, "<f8", int(np.prod(dims)), int(di.get("Seek"))).reshape(dims)
        np.testing.assert_array_equal(got, prim[b, 0, s[0], s[1], s[2]])
