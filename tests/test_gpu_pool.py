"""Block pool: jobs stepped together through the block table give results
bit-identical to each job run alone (states, dt and per-job counters), with
jobs attached and detached between cycles and slots reused."""
import numpy as np
import pytest

from pangu_b200 import params as prm
from pangu_b200 import problems

pytestmark = pytest.mark.gpu


def _job(problem, **kw):
    pin, gen = problems.make_problem(problem, **kw)
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
    return sim.primitives(), sim.dt.item(), sim.engine.counters()


def _run_schedule(template, jobs, schedule, capacity, max_jobs, graph=True):
    """jobs: name -> (pin, prim, cycles); schedule: name -> tick of attach.
    Returns name -> (prims, dt, counters) taken when the job finishes."""
    import torch
    from pangu_b200.engine import Pool
    pool = Pool(template, capacity, max_jobs)
    done, live, tick = {}, {}, 0
    while len(done) < len(jobs):
        for name, t0 in schedule.items():
            if t0 == tick:
                pin, prim, _ = jobs[name]
                live[name] = [pool.attach(pin, prim), 0]
        pool.step(graph=graph)
        tick += 1
        for name in list(live):
            live[name][1] += 1
            job, n = live[name]
            if n == jobs[name][2]:
                torch.cuda.synchronize()
                dt = pool.dt[job].item()
                cnt = pool.engine.job_counters(job)
                done[name] = (pool.detach(job), dt, cnt)
                del live[name]
    return done


def _check(done, jobs):
    for name, (pin, prim, cycles) in jobs.items():
        ref_p, ref_dt, ref_c = _alone(pin, prim, cycles)
        got_p, got_dt, got_c = done[name]
        np.testing.assert_array_equal(got_p, ref_p, err_msg=name)
        assert got_dt == ref_dt, name
        np.testing.assert_array_equal(got_c, ref_c, err_msg=name)


def test_pool_tori_match_alone():
    bx = (32, 16, 1)
    jobs = {
        "A": (*_job("torus", nx1=64, nx2=32, bx=bx, a=0.9375, seed=1), 5),
        "B": (*_job("torus", nx1=32, nx2=16, bx=bx, a=0.5, rmax=10.0, seed=2), 3),
        "C": (*_job("torus", nx1=96, nx2=48, bx=bx, a=0.98, beta=30.0, seed=3), 4),
        "D": (*_job("torus", nx1=32, nx2=32, bx=bx, a=0.2, rmax=14.0, seed=4), 3),
    }
    schedule = {"A": 0, "B": 0, "C": 2, "D": 3}  # D reuses B's slot and job id
    template = jobs["A"][0]
    done = _run_schedule(template, jobs, schedule, capacity=4 + 9 + 2, max_jobs=3)
    _check(done, jobs)


def test_pool_orszag_tang_periodic_blocks():
    jobs = {
        "small": (*_job("ot", n=32, nblock=16), 4),
        "large": (*_job("ot", n=48, nblock=16), 3),
    }
    done = _run_schedule(jobs["small"][0], jobs, {"small": 0, "large": 1}, capacity=13,
                         max_jobs=2, graph=False)
    _check(done, jobs)


def test_pool_rejects_mismatched_job():
    from pangu_b200.engine import EngineError, Pool
    pin, prim = _job("torus", nx1=64, nx2=32, bx=(32, 16, 1))
    pool = Pool(pin, 4, 2)
    other, oprim = _job("torus", nx1=64, nx2=32, bx=(16, 16, 1))
    with pytest.raises(EngineError):
        pool.attach(other, oprim)  # block shape differs
    big, bprim = _job("torus", nx1=96, nx2=32, bx=(32, 16, 1))
    pool.attach(pin, prim)
    with pytest.raises(EngineError):
        pool.attach(big, bprim)  # 6 blocks > 0 free slots
