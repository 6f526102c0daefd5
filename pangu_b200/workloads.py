"""The benchmark workloads: their inputs, initial states and job streams.

* ``torus2d``: the 2D Fishbone-Moncrief torus in MKS coordinates, 512 x 256,
  PPM4, LAXF, chainer C2P, electron heating, one meshblock, 200 RK2 cycles.
* ``ot``: the Orszag-Tang vortex, 256^2, Minkowski, MC, LAXF, 100 cycles.
* ``torus3d``: the torus on 256 x 128 x 128 in 16 meshblocks of 64^3, HLL,
  50 cycles.
* ``cks3d``: a magnetised atmosphere around a spinning hole in Cartesian
  Kerr-Schild coordinates with excision, 64^3 in 8 meshblocks of 32^3, MC,
  LAXF, 50 cycles (the metric formed in the kernels, not tabulated).
* ``batch48``: 48 tori of uneven grids in one block pool, 100 cycles each.
* ``serve``: a seeded Poisson stream of Brio-Wu, Orszag-Tang and torus jobs.

Every input is a seeded synthetic initial condition with the shapes, sizes and
parameters of the workload; no dataset is involved.
"""
from __future__ import annotations

import math

import numpy as np

from . import params as prm
from . import problems

# single-mesh workloads: input builder, job length (RK2 cycles), config keys
SINGLE = {
    "torus2d": (lambda seed: problems.fm_torus_input(nx1=512, nx2=256, seed=seed), 200,
                {"grid": "512x256", "meshblocks": 1, "limiter": "ppm4",
                 "riemann_solver": "laxf", "recovery": "chainer", "electron_heating": True,
                 "metric": "mks a=0.9375 h=0.7"}),
    "ot": (lambda seed: problems.orszag_tang_input(n=256), 100,
           {"grid": "256x256", "meshblocks": 1, "limiter": "mc", "riemann_solver": "laxf",
            "recovery": "chainer", "electron_heating": False, "metric": "minkowski"}),
    "torus3d": (lambda seed: problems.fm_torus_input(nx1=256, nx2=128, nx3=128,
                                                     bx=(64, 64, 64), riemann="hll",
                                                     seed=seed), 50,
                {"grid": "256x128x128", "meshblocks": "16 x 64^3", "limiter": "ppm4",
                 "riemann_solver": "hll", "recovery": "chainer", "electron_heating": True,
                 "metric": "mks a=0.9375 h=0.7"}),
    "cks3d": (lambda seed: problems.cks_atmosphere_input(n=64, nblock=32), 50,
              {"grid": "64^3", "meshblocks": "8 x 32^3", "limiter": "mc",
               "riemann_solver": "laxf", "recovery": "chainer", "electron_heating": False,
               "metric": "cks a=0.5, excised inside r = 1.5"}),
}
WORKLOAD_NAMES = {"torus2d": "fm_torus_mks_2d_512x256", "ot": "orszag_tang_2d_256x256",
                  "torus3d": "fm_torus_mks_3d_256x128x128", "cks3d": "cks_atmosphere_3d_64",
                  "batch48": "fm_torus_mks_2d_batch48", "serve": "serving_stream_bw_ot_torus"}

# block shape of the batch and of the served tori
BATCH_BLOCK = (128, 64, 1)


def job_input(workload: str, precision: str = "fp64", seed: int = 0) -> prm.ParameterInput:
    """The inputfile of a single-mesh workload."""
    pin = SINGLE[workload][0](seed)
    pin.set("b200", "precision", precision)
    return pin


def initial_state(pin: prm.ParameterInput):
    """(packages, mesh struct, geometry, interior primitives) of a job's
    inputfile: Orszag-Tang or Brio-Wu on a Minkowski metric (Brio-Wu when
    gamma = 2), the Kerr-Schild atmosphere on a CKS metric, the
    Fishbone-Moncrief torus otherwise."""
    packages = prm.process_packages(pin)
    mesh = prm.mesh_struct(pin)
    geo = problems.Geometry(mesh)
    if packages["metric"].params["metric_type"] == "minkowski":
        gam = packages["core"].params["adiabatic_index"]
        prim = (problems.brio_wu(geo, packages) if gam == 2.0
                else problems.orszag_tang(geo, packages))
    elif packages["metric"].params["metric_type"] == "cks":
        prim = problems.cks_atmosphere(geo, packages)
    else:
        prim = problems.fm_torus(geo, packages, pin)
    return packages, mesh, geo, prim


def interior_cells(pin: prm.ParameterInput) -> int:
    return int(np.prod([pin.get_or_add_integer("parthenon/mesh", f"nx{d}", 1)
                        for d in (1, 2, 3)]))


def batch_jobs(precision: str, n: int = 48, seed: int = 1234, states: bool = False):
    """48 MKS tori: grids drawn from {128x64, 256x128, 384x192, 512x256}, spin
    a ~ U[0, 0.98], beta ~ logU[30, 300], rmax ~ U[10, 14] (seeded). A draw
    with no bound torus (low spin with rmax near 10 for rin = 6) is redrawn.
    Returns the inputs, or (inputs, initial states) with states=True."""
    rng = np.random.default_rng(seed)
    grids = [(128, 64), (256, 128), (384, 192), (512, 256)]
    jobs, prims = [], []
    while len(jobs) < n:
        nx1, nx2 = grids[int(rng.integers(len(grids)))]
        a = float(rng.uniform(0.0, 0.98))
        beta = float(math.exp(rng.uniform(math.log(30.0), math.log(300.0))))
        rmax = float(rng.uniform(10.0, 14.0))
        pin = problems.fm_torus_input(nx1=nx1, nx2=nx2, bx=BATCH_BLOCK, a=a, beta=beta,
                                      rmax=rmax, seed=len(jobs))
        pin.set("b200", "precision", precision)
        try:
            prim = initial_state(pin)[3]
        except ValueError:
            continue
        jobs.append(pin)
        prims.append(prim)
    return (jobs, prims) if states else jobs


def serve_jobs(precision: str, n: int, rate: float, seed: int = 7):
    """Poisson arrivals (rate per second) of Brio-Wu tubes (1024-8192 cells,
    blocks of 1024), Orszag-Tang vortices (128^2-512^2, blocks of 128^2) and
    MKS tori (256x128-512x256, blocks of 128x64) at 200-2000 RK2 cycles.
    Returns [(kind, inputfile, cycles, arrival seconds)]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    for q in range(n):
        t += float(rng.exponential(1.0 / rate))
        kind = ("bw", "ot", "torus")[q % 3]
        if kind == "bw":
            pin = problems.brio_wu_input(n=int(rng.choice([1024, 2048, 4096, 8192])),
                                         nblock=1024)
        elif kind == "ot":
            pin = problems.orszag_tang_input(n=int(rng.choice([128, 256, 384, 512])),
                                             nblock=128)
        else:
            nx1, nx2 = [(256, 128), (384, 192), (512, 256)][int(rng.integers(3))]
            pin = problems.fm_torus_input(nx1=nx1, nx2=nx2, bx=BATCH_BLOCK,
                                          a=float(rng.uniform(0.0, 0.98)), seed=q)
        pin.set("b200", "precision", precision)
        jobs.append((kind, pin, int(rng.integers(200, 2001)), t))
    return jobs
