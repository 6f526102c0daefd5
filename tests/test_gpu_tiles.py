"""The flux kernels' tile shapes (CTA size, march depth, shared-memory
tiles) change how faces are distributed over threads, never what is computed
for a face: every shape
the autotuner may pick gives bit-identical results, in FP64 and in the mixed
form, so a job's result does not depend on the tuning of the engine (or pool,
or server class) that runs it."""
import itertools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(pin, prim0, cfg, cycles=3):
    import torch
    from pangu_b200.engine import Simulation
    sim = Simulation(pin)
    sim.engine.set_flux_config(**cfg)
    sim.set_primitives(prim0)
    for _ in range(cycles):
        sim.step()
    torch.cuda.synchronize()
    return sim.primitives()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("three_d", [False, True])
def test_every_tile_shape_gives_the_same_result(precision, three_d):
    from pangu_b200 import params as prm
    from pangu_b200 import problems
    kw = dict(nx1=32, nx2=16, nx3=8, bx=(16, 8, 8)) if three_d else dict(nx1=64, nx2=32)
    pin, gen = problems.make_problem("torus", seed=2, **kw)
    pin.set("b200", "precision", precision)
    prim0 = gen(problems.Geometry(prm.mesh_struct(pin)), prm.process_packages(pin), pin)
    ref = None
    # (march, CTA size): march 1, 2, 4 faces per thread, or march 0: shared-memory
    # tiles of 32 x (CTA size / 32) faces
    shapes = [(1, 64), (1, 128), (2, 64), (2, 128), (4, 64), (4, 128), (0, 128), (0, 256)]
    for t1, (m2, t2) in itertools.product((64, 128), shapes):
        m3, t3 = (m2, t2) if three_d else (2, 128)
        cfg = dict(x1_threads=t1, x2_march=m2, x2_threads=t2, x3_march=m3, x3_threads=t3)
        got = _run(pin, prim0, cfg)
        if ref is None:
            ref = got
        else:
            np.testing.assert_array_equal(got, ref, err_msg=str(cfg))
