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
    assert not sim.engine.device_error()
    return sim.primitives()


def _tma_rows_ok(pin, precision):
    """TMA-staged flux kernels need rows of whole 16-byte units."""
    from pangu_b200 import params as prm
    m = prm.mesh_struct(pin)
    n1 = m.nx1 + 2 * m.ng
    return (n1 * (8 if precision == "fp64" else 4)) % 16 == 0


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
    x1 = [(1, 64), (1, 128)]
    if _tma_rows_ok(pin, precision):  # primitives staged by TMA
        shapes.append((8, 128))
        x1.append((8, 128))
    for (m1, t1), (m2, t2) in itertools.product(x1, shapes):
        m3, t3 = (m2, t2) if three_d else (2, 128)
        cfg = dict(x1_march=m1, x1_threads=t1, x2_march=m2, x2_threads=t2, x3_march=m3,
                   x3_threads=t3)
        got = _run(pin, prim0, cfg)
        if ref is None:
            ref = got
        else:
            np.testing.assert_array_equal(got, ref, err_msg=str(cfg))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("limiter", ["mc", "ppm4"])
def test_tma_staged_flux_kernels_give_the_same_result(precision, limiter):
    """The TMA-staged x2 tiles and x1 rows (march 8) against the thread-loaded
    tiles and the march kernels, on grids whose rows are whole 16-byte units
    in both precisions (MC: 2 ghost cells, PPM4: 3); the copies start a
    column or two early to align, and for MC the x1 rows start before the
    grid (the copy fills zeros there, which no stencil reads)."""
    from pangu_b200 import params as prm
    from pangu_b200 import problems
    nx1 = 60 if limiter == "mc" else 58  # N1 = 64 either way
    pin, gen = problems.make_problem("torus", seed=3, nx1=nx1, nx2=24, limiter=limiter)
    pin.set("b200", "precision", precision)
    assert _tma_rows_ok(pin, precision)
    prim0 = gen(problems.Geometry(prm.mesh_struct(pin)), prm.process_packages(pin), pin)
    ref = _run(pin, prim0, dict(x1_threads=128, x2_march=2, x2_threads=128))
    for m1, m2, t2 in ((1, 0, 128), (1, 8, 128), (8, 2, 128), (8, 8, 128)):
        got = _run(pin, prim0, dict(x1_march=m1, x1_threads=128, x2_march=m2, x2_threads=t2))
        np.testing.assert_array_equal(got, ref, err_msg=f"x1 march {m1} x2 march {m2}")
