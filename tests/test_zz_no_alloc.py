"""pangu_estimate_dt_noalloc: the dt estimate for callers that may not call
cudaMalloc (device memory owned by a pool or a fixed budget). It must give the
same dt as pangu_estimate_dt, call after call, with its scratch kept in the
library's static device array. Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
from parity_util import Case  # noqa: E402

pytestmark = pytest.mark.gpu


def _noalloc(L):
    f = L.pangu_estimate_dt_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


@pytest.mark.parametrize("name", ["torus_ppm4_laxf", "torus3d_blocks", "ot_blocks"])
def test_noalloc_dt_matches_engine(name):
    from pangu_b200.engine import Simulation, lib
    case = Case(name)
    sim = Simulation(case.pin)
    sim.set_primitives(case.prim0)
    f = _noalloc(lib())
    stream = sim.engine.stream()
    ref = torch.zeros(1, dtype=torch.float64, device="cuda")
    got = torch.zeros(1, dtype=torch.float64, device="cuda")
    for _ in range(2):  # two calls in a row, state advanced in between
        sim.step()
        sim.engine.estimate_dt(sim.base, ref)
        rc = f(C.addressof(sim.params), C.addressof(sim.mesh), sim.base.alfven.data_ptr(),
               got.data_ptr(), stream)
        assert rc == 0
        torch.cuda.synchronize()
        assert np.isfinite(ref.item()) and ref.item() > 0
        assert got.item() == ref.item()


def test_noalloc_rejects_too_many_blocks():
    from pangu_b200.engine import lib
    case = Case("ot_blocks")
    mesh = case.mesh
    mesh.nbx1, mesh.nbx2, mesh.nbx3 = 64, 65, 1  # 4160 blocks > 4096
    f = _noalloc(lib())
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = f(C.addressof(case.params), C.addressof(mesh), dummy.data_ptr(), out.data_ptr(), None)
    assert rc == -5  # PANGU_ETOOBIG
