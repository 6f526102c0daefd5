"""Serving loop: jobs of several classes arriving over time are admitted as
pool slots free up, stepped together, and each result is bit-identical to
the job run alone (states and counters)."""
import numpy as np
import pytest

from pangu_b200 import params as prm
from pangu_b200 import problems

pytestmark = pytest.mark.gpu


def _job(problem, precision="fp64", **kw):
    pin, gen = problems.make_problem(problem, **kw)
    pin.set("b200", "precision", precision)
    geo = problems.Geometry(prm.mesh_struct(pin))
    return pin, gen(geo, prm.process_packages(pin), pin)


def _alone(pin, prim, cycles):
    import torch
    from pangu_b200.engine import Simulation
    sim = Simulation(pin)
    sim.set_primitives(prim)
    for _ in range(cycles):
        sim.step()
    torch.cuda.synchronize()
    return sim.primitives(), sim.engine.counters()


def test_server_results_match_alone():
    from pangu_b200.engine import Server
    tb = (32, 16, 1)
    jobs = [  # (class, (pin, prim), cycles, arrival seconds)
        ("torus", _job("torus", nx1=64, nx2=32, bx=tb, a=0.9375, seed=1), 5, 0.0),
        ("torus", _job("torus", nx1=32, nx2=16, bx=tb, a=0.5, seed=2), 3, 0.0),
        ("torus", _job("torus", nx1=64, nx2=32, bx=tb, a=0.98, seed=3), 4, 0.001),
        ("ot", _job("ot", n=32, nblock=16), 4, 0.0),
        ("ot", _job("ot", n=48, nblock=16), 3, 0.002),
        ("bw", _job("bw", n=256, nblock=64), 6, 0.0),
        ("bw", _job("bw", n=128, nblock=64), 2, 0.003),
        ("mixed", _job("torus", "mixed", nx1=64, nx2=32, bx=tb, a=0.7, seed=4), 3, 0.0),
    ]
    srv = Server(8 << 30)
    templates = {"torus": jobs[0][1][0], "ot": jobs[3][1][0], "bw": jobs[5][1][0],
                 "mixed": jobs[7][1][0]}
    # the torus pool holds 5 blocks: the third torus waits for the second
    caps = {"torus": (5, 2), "ot": (13, 2), "bw": (4, 2), "mixed": (4, 1)}
    cls = {k: srv.add_class(t, *caps[k]) for k, t in templates.items()}
    tickets = [srv.submit(cls[c], pin, prim, n, t) for c, (pin, prim), n, t in jobs]
    srv.run()
    st = srv.stats()
    lat = []
    for tk, (c, (pin, prim), n, t) in zip(tickets, jobs):
        got, times, cnt = srv.result(tk)
        ref, ref_cnt = _alone(pin, prim, n)
        np.testing.assert_array_equal(got, ref, err_msg=c)
        np.testing.assert_array_equal(cnt, ref_cnt, err_msg=c)
        assert times[0] == t and times[1] >= t and times[2] > times[1]
        lat.append(times[2] - times[0])
    assert st["jobs"] == len(jobs)
    assert st["p50_s"] <= st["p99_s"] <= max(lat) + 1e-9
    cells = sum(np.prod([pin.get_or_add_integer("parthenon/mesh", f"nx{d}", 1)
                         for d in (1, 2, 3)]) * n for _, (pin, _p), n, _t in jobs)
    assert st["zone_cycles"] == cells
    # the third torus (4 blocks) could only start after the second finished
    _, t_b, _ = srv.result(tickets[1])
    _, t_c, _ = srv.result(tickets[2])
    assert t_c[1] >= t_b[2]


def test_server_budget_enforced():
    from pangu_b200.engine import EngineError, Server
    pin, _ = _job("torus", nx1=64, nx2=32, bx=(32, 16, 1))
    srv = Server(64 << 20)  # 64 MiB
    with pytest.raises(EngineError):
        srv.add_class(pin, 1000, 4)
    srv.add_class(pin, 4, 2)


def test_server_cancellation():
    """A waiting job cancelled before its slots free up is dropped, a running
    one is detached at a tick boundary; the other jobs finish unaffected."""
    from pangu_b200.engine import EngineError, Server
    tb = (32, 16, 1)
    keep = _job("torus", nx1=64, nx2=32, bx=tb, seed=1)
    long_job = _job("torus", nx1=32, nx2=16, bx=tb, seed=2)
    waiting = _job("torus", nx1=64, nx2=32, bx=tb, seed=3)
    srv = Server(4 << 30)
    c = srv.add_class(keep[0], 5, 3)
    t_keep = srv.submit(c, *keep, 6, 0.0)
    t_long = srv.submit(c, *long_job, 100000, 0.0)  # would run for minutes
    t_wait = srv.submit(c, *waiting, 3, 0.0)         # 4 blocks: no room until keep ends
    srv.cancel(t_long, 0.05)
    srv.cancel(t_wait, 0.0)
    srv.run()
    assert srv.state(t_keep) == "done"
    assert srv.state(t_long) == "cancelled" and srv.state(t_wait) == "cancelled"
    with pytest.raises(EngineError):
        srv.result(t_long)
    ref, ref_cnt = _alone(*keep, 6)
    got, _, cnt = srv.result(t_keep)
    np.testing.assert_array_equal(got, ref)
    np.testing.assert_array_equal(cnt, ref_cnt)
    assert srv.stats()["jobs"] == 1


def test_server_lazy_classes_take_turns_under_budget():
    """Classes declared lazily are charged at their first admission and
    released when idle: with a budget that holds either class's memory but not
    both, the second class's job waits until the first class's job finishes
    and its memory is released; every result equals the job run alone."""
    from pangu_b200.engine import Server
    a_job = _job("torus", nx1=128, nx2=64, bx=(32, 16, 1), seed=5)  # 16 blocks
    b_job = _job("ot", n=128, nblock=32)                             # 16 blocks

    def peak_alone(job):
        srv = Server(8 << 30)
        c = srv.add_class(job[0], 16, 1, lazy=True)
        srv.submit(c, *job, 2, 0.0)
        srv.run()
        st = srv.stats()
        assert st["hbm_bytes"] == 0 and st["memory_waits"] == 0  # released after the run
        return st["hbm_peak_bytes"]

    pa, pb = peak_alone(a_job), peak_alone(b_job)
    # room for either class (the engine's share is measured from the device's
    # free memory, which moves in whole pages), not for both
    budget = max(pa, pb) + max(4 << 20, min(pa, pb) // 3)
    assert budget < pa + pb, (pa, pb)
    srv = Server(budget)
    ca = srv.add_class(a_job[0], 16, 1, lazy=True)
    cb = srv.add_class(b_job[0], 16, 1, lazy=True)
    ta = srv.submit(ca, *a_job, 4, 0.0)
    tb = srv.submit(cb, *b_job, 3, 0.0)
    srv.run()
    st = srv.stats()
    assert st["jobs"] == 2 and st["memory_waits"] == 1
    assert st["hbm_peak_bytes"] <= budget and st["hbm_bytes"] == 0
    (ga, times_a, cnt_a), (gb, times_b, cnt_b) = srv.result(ta), srv.result(tb)
    first, second = (times_a, times_b) if times_a[1] <= times_b[1] else (times_b, times_a)
    assert second[1] >= first[2]  # admitted only after the other class finished
    for got, cnt, (pin, prim), n in ((ga, cnt_a, a_job, 4), (gb, cnt_b, b_job, 3)):
        ref, ref_cnt = _alone(pin, prim, n)
        np.testing.assert_array_equal(got, ref)
        np.testing.assert_array_equal(cnt, ref_cnt)


def test_server_lazy_class_too_big_reports_enomem():
    from pangu_b200.engine import EngineError, Server
    job = _job("torus", nx1=64, nx2=32, bx=(32, 16, 1), seed=6)
    srv = Server(1 << 20)  # 1 MiB: the class never fits
    c = srv.add_class(job[0], 4, 1, lazy=True)
    srv.submit(c, *job, 2, 0.0)
    with pytest.raises(EngineError):
        srv.run()
