"""Device-side initial conditions (pangu_generate) against the host
generators of pangu_b200/problems.py on the same mesh: the same formulas and
the same counter-based perturbation, so they agree to a few ulps (the device
uses CUDA's transcendental functions, the host numpy's). Jobs generated on
the device run in the serving loop exactly as alone."""
import numpy as np
import pytest

from pangu_b200 import params as prm
from pangu_b200 import problems

pytestmark = pytest.mark.gpu


def _host(pin, name):
    _, gen = problems.make_problem(name)
    return gen(problems.Geometry(prm.mesh_struct(pin)), prm.process_packages(pin), pin)


def _device(pin, name):
    import torch
    from pangu_b200.engine import Simulation
    sim = Simulation(pin)
    sim.base.prim.zero_()
    sim.engine.generate(0, problems.problem_struct(name, pin), sim.base)
    torch.cuda.synchronize()
    return sim.base.prim.double().cpu().numpy()


@pytest.mark.parametrize("name,kw", [("ot", dict(n=32, nblock=16)),
                                     ("bw", dict(n=256, nblock=64)),
                                     ("torus", dict(nx1=64, nx2=32, bx=(32, 16, 1))),
                                     ("torus", dict(nx1=32, nx2=16, nx3=8, bx=(16, 8, 4)))])
def test_device_generator_matches_host(name, kw):
    pin, _ = problems.make_problem(name, **kw)
    host = _host(pin, name)
    dev = _device(pin, name)
    assert host.shape == dev.shape
    # The torus velocities go through the code metric, whose finite-difference
    # Jacobian (delta = 1e-5) amplifies a one-ulp difference of exp between
    # numpy and the C library by 1e5.
    tol = 1e-10 if name == "torus" else 1e-12
    for v in range(host.shape[1]):
        scale = max(np.abs(host[:, v]).max(), 1e-300)
        err = np.abs(dev[:, v] - host[:, v]).max() / scale
        assert err <= tol, (name, v, err)


def test_no_bound_torus_is_an_error():
    from pangu_b200.engine import EngineError
    pin, _ = problems.make_problem("torus", nx1=64, nx2=32, a=0.0)
    pin.set("fm_torus", "rmax", 10.0)  # rin = 6: no bound region at zero spin
    with pytest.raises(EngineError):
        _device(pin, "torus")


def test_server_generated_jobs_match_alone():
    import torch
    from pangu_b200.engine import Server, Simulation
    tb = (32, 16, 1)
    jobs = [("torus", problems.make_problem("torus", nx1=64, nx2=32, bx=tb, seed=3)[0], 4, 0.0),
            ("torus", problems.make_problem("torus", nx1=32, nx2=32, bx=tb, a=0.5, seed=4)[0], 3,
             0.001),
            ("ot", problems.make_problem("ot", n=32, nblock=16)[0], 3, 0.0)]
    srv = Server(4 << 30)
    cls = {"torus": srv.add_class(jobs[0][1], 6, 2), "ot": srv.add_class(jobs[2][1], 4, 1)}
    tickets = [srv.submit_problem(cls[k], pin, k, n, t) for k, pin, n, t in jobs]
    srv.run()
    for tk, (k, pin, n, t) in zip(tickets, jobs):
        got, _, cnt = srv.result(tk)
        sim = Simulation(pin)
        sim.generate(k)
        for _ in range(n):
            sim.step()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(got, sim.primitives(), err_msg=k)
        np.testing.assert_array_equal(cnt, sim.engine.counters(), err_msg=k)
