"""The N > 1 path of the benchmark on CPU: two gloo ranks, each stepping its
own independently seeded torus job (the oracle stands in for the GPU), with
the max-over-ranks timing as the only collective. Each rank's result equals
a single-process run of the same seed: nothing crosses ranks on the data
path."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _job(seed, steps=2):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    from pangu_b200 import params as prm
    from pangu_b200 import problems
    pin = problems.fm_torus_input(nx1=32, nx2=16, seed=seed)
    pk = prm.process_packages(pin)
    mesh = prm.mesh_struct(pin)
    prim0 = problems.fm_torus(problems.Geometry(mesh), pk, pin)
    O = po.Oracle(prm.params_struct(pk), mesh)
    base, one = O.new_containers()
    base.prim[...] = prim0
    O.exchange_ghosts(base)
    O.apply_boundary_conditions(base)
    one.prim[...] = base.prim
    one.cons[...] = base.cons
    dt = 1e-5
    for _ in range(steps):
        dt = min(1.3 * dt, O.step(base, one, dt))
    return np.array(base.prim), dt


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    prim, dt = _job(seed=rank)
    fake_ms = 10.0 + 5.0 * rank
    tmax = bench.max_over_ranks(fake_ms, dist, torch.device("cpu"))
    np.save(os.path.join(out, f"rank{rank}.npy"), prim)
    with open(os.path.join(out, f"rank{rank}.txt"), "w") as f:
        f.write(f"{tmax} {dt!r}\n")
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_independent_jobs_max_timing(tmp_path):
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    results = []
    for r in range(2):
        tmax, dt = open(tmp_path / f"rank{r}.txt").read().split()
        assert float(tmax) == 15.0  # max over ranks of 10 and 15 ms
        results.append((np.load(tmp_path / f"rank{r}.npy"), float(dt)))
    assert not np.array_equal(results[0][0], results[1][0])  # seeded per rank
    for r in range(2):
        prim, dt = _job(seed=r)
        np.testing.assert_array_equal(results[r][0], prim)
        assert results[r][1] == dt
