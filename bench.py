"""Benchmark of the GRMHD stage engine: zone-cycles/s on B200.

Default workload: the 2D Fishbone-Moncrief torus in MKS coordinates,
512 x 256, FP64, PPM4, LAXF, chainer C2P, electron heating (one meshblock).
A step is one RK2 cycle (two stages) of the whole grid; the job length in the
workload definition is 200 steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

N > 1 runs under torchrun, one independent torus job per GPU (weak scaling,
no collective on the data path; the timing is a max over ranks).
``--impl reference`` times the CPU restatement of the reference's stage path
(oracle/) on the host cores for the same workload and metric.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from pangu_b200 import params as prm  # noqa: E402
from pangu_b200 import problems  # noqa: E402

METRIC = "zone-cycles/s"
NX1, NX2 = 512, 256
WORKLOAD = "fm_torus_mks_2d_512x256_fp64"
JOB_STEPS = 200


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def workload_input(seed=0):
    return problems.fm_torus_input(nx1=NX1, nx2=NX2, seed=seed)


def initial_state(pin):
    packages = prm.process_packages(pin)
    mesh = prm.mesh_struct(pin)
    geo = problems.Geometry(mesh)
    prim = problems.fm_torus(geo, packages, pin)
    return packages, mesh, geo, prim


def config(extra=None):
    c = {"workload": WORKLOAD, "nx1": NX1, "nx2": NX2, "meshblocks": 1, "limiter": "ppm4",
         "riemann_solver": "laxf", "recovery": "chainer", "electron_heating": True,
         "metric": "mks a=0.9375 h=0.7", "job_steps": JOB_STEPS,
         "l2": "flushed (256 MiB write) before every timed step",
         "launch": "one CUDA graph replay per RK2 step"}
    if extra:
        c.update(extra)
    return c


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.gpu)], stdout=self.out, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.out.close()

    def summary(self):
        rows = []
        if self.path and os.path.exists(self.path):
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) == 9:
                        rows.append(parts)
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "", 1).isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "", 1).isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows)}


# ---------------------------------------------------------------------------
# algorithmic bytes per launch of each task (FP64, NF fields)
# ---------------------------------------------------------------------------
def task_bytes(nf, n_int, n_ent, ndim):
    w = 8
    return {
        "fix_primitive": 2 * nf * w * n_ent,
        "calculate_conservative": 2 * nf * w * n_int,
        "calculate_fluxes": (nf * w + ndim * (nf * w + w)) * n_int,
        "constrained_transport": (2 * ndim * w + 3 * w + 2 * ndim * w) * n_int,
        "flux_divergence_update": (ndim * nf * w + 2 * nf * w) * n_int,
        "add_geometric_source": (nf * w + 2 * 4 * w) * n_int,
        "recovery": (2 * 9 * w + 8 * w + w) * n_int,
        "apply_electron_heating": (nf * w + 3 * w + w) * n_int,
        "fix_recovery": w * n_int,
        "apply_boundary_conditions": 0,
        "estimate_dt": ndim * w * n_int,
    }


def max_over_ranks(value, dist, device):
    """Max of a per-rank time over all ranks: a multi-GPU run is as fast as
    its slowest rank. The only collective of the benchmark (jobs are
    independent, one per GPU; nothing crosses ranks on the data path)."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.item()


def run_engine(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    from pangu_b200.engine import Simulation

    pin = workload_input(seed=rank)
    packages, mesh, geo, prim0 = initial_state(pin)
    sim = Simulation(pin, device=local)
    sim.set_primitives(prim0)
    n_int = NX1 * NX2
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    for _ in range(args.warmup):
        sim.step()
    torch.cuda.synchronize()
    if not args.no_graph:
        # one RK2 cycle per CUDA graph replay; the capture runs no kernel
        launches_per_step = sim.engine.launches()
        sim.capture()
        launches_per_step = sim.engine.launches() - launches_per_step
        sim.step()  # the first replay is part of the warm-up
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    launches0 = sim.engine.launches()
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        for s in range(args.steps):
            flush.zero_()
            starts[s].record()
            sim.step()
            ends[s].record()
        torch.cuda.synchronize()
    launches = sim.engine.launches() - launches0
    if not args.no_graph:
        launches = launches_per_step * args.steps
    total_ms = sum(a.elapsed_time(b) for a, b in zip(starts, ends))
    if world > 1:
        total_ms = max_over_ranks(total_ms, dist, dev)
        dist.barrier()
    clocks = clk.summary()
    ms_per_step = total_ms / args.steps
    value = world * n_int * args.steps / (total_ms / 1e3)

    # ---- end to end through the public API with host-resident state -------
    e2e = e2e_run(sim, torch, dev, min(args.steps, 100))
    if world > 1:
        e2e["ms"] = max_over_ranks(e2e["ms"], dist, dev)

    # ---- per-task breakdown and the dominant kernel's roofline ---------
    tasks = task_times(sim, torch, flush) if rank == 0 else {}
    line = None
    if rank == 0:
        peak, peak_kind = peaks()
        nf = sim.engine.nf
        n_ent = int(np.prod(sim.engine.shape)) * sim.engine.nb
        tb = task_bytes(nf, n_int, n_ent, 2)
        dom = max(tasks, key=lambda k: tasks[k])
        achieved = tb[dom] / (tasks[dom] / 1e3) / 1e9
        traffic = committed_traffic(dom)
        roof = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 2),
                "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                "frac": round(achieved / peak, 5), "traffic": traffic,
                "algorithmic_bytes_per_launch": tb[dom], "launch_ms": round(tasks[dom], 5),
                "step_achieved_gbs": round(80 * nf * value / world / 1e9, 2),
                "task_ms": {k: round(v, 5) for k, v in tasks.items()}}
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline(pin, prim0, budget_s=args.cpu_budget)
        e2e_value = world * n_int * e2e["steps"] / (e2e["ms"] / 1e3)
        line = {"metric": METRIC, "value": round(value, 1), "unit": METRIC, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 5),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic (seeded torus initial conditions)",
                "config": config({"parallelism": f"{world} independent torus jobs, one per GPU"}),
                "e2e": {"value": round(e2e_value, 1), "unit": METRIC,
                        "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"],
                        "steps": e2e["steps"]},
                "roofline": roof, "cpu_baseline": cpu, "clocks": clocks,
                "gpu_launches": launches}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


def e2e_run(sim, torch, dev, steps):
    """Steps with the job state resident on the HOST: every step copies the
    state in from pinned memory, runs the RK2 cycle and copies it back."""
    base, one = sim.base, sim.one
    h_base = torch.empty(base.prim.shape, dtype=torch.float64).pin_memory()
    h_one = torch.empty(one.prim.shape, dtype=torch.float64).pin_memory()
    h_flag = torch.empty(base.flag.shape, dtype=torch.float64).pin_memory()
    h_dt = torch.empty(1, dtype=torch.float64).pin_memory()
    h_base.copy_(base.prim)
    h_one.copy_(one.prim)
    h_flag.copy_(base.flag)
    h_dt.copy_(sim.dt)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        base.prim.copy_(h_base, non_blocking=True)
        one.prim.copy_(h_one, non_blocking=True)
        base.flag.copy_(h_flag, non_blocking=True)
        sim.dt.copy_(h_dt, non_blocking=True)
        sim.step()
        h_base.copy_(base.prim, non_blocking=True)
        h_one.copy_(one.prim, non_blocking=True)
        h_flag.copy_(base.flag, non_blocking=True)
        h_dt.copy_(sim.dt, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    nbytes = h_base.numel() * 8 + h_one.numel() * 8 + h_flag.numel() * 8 + 8
    return {"ms": e0.elapsed_time(e1), "steps": steps, "h2d": nbytes, "d2h": nbytes}


def task_times(sim, torch, flush, reps=20):
    """Average device time of every task launch (L2 flushed before each)."""
    eng, base, one = sim.engine, sim.base, sim.one
    beta, dt = 0.5, sim.dt
    est = torch.zeros(1, dtype=torch.float64, device=eng.device)
    calls = {
        "fix_primitive": lambda: eng.fix_primitive(base),
        "calculate_conservative": lambda: eng.calculate_conservative(base),
        "calculate_fluxes": lambda: eng.calculate_fluxes(base),
        "constrained_transport": lambda: eng.constrained_transport(base),
        "flux_divergence_update": lambda: eng.flux_divergence_update(base, base, one, beta, dt),
        "add_geometric_source": lambda: eng.add_geometric_source(one, beta, dt),
        "recovery": lambda: eng.recovery(one),
        "apply_electron_heating": lambda: eng.apply_electron_heating(one),
        "fix_recovery": lambda: eng.fix_recovery(one),
        "apply_boundary_conditions": lambda: eng.apply_boundary_conditions(one),
        "estimate_dt": lambda: eng.estimate_dt(one, est),
    }
    out = {}
    for name, fn in calls.items():
        fn()
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(reps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            tot += a.elapsed_time(b)
        out[name] = tot / reps
    return out


def committed_traffic(kernel):
    """DRAM bytes per launch of a task from the committed ncu summary
    (profiles/traffic_fm_torus_512x256.txt: lines 'task bytes'), or None."""
    path = os.path.join(ROOT, "profiles", "traffic_fm_torus_512x256.txt")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 2 and parts[0] == kernel:
                try:
                    return float(parts[1])
                except ValueError:
                    return None
    return None


# ---------------------------------------------------------------------------
# CPU: the oracle (restatement of the reference's stage path), all host cores
# ---------------------------------------------------------------------------
def _oracle_job(pin, prim0, threads):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    po.set_threads(threads)
    packages = prm.process_packages(pin)
    params = prm.params_struct(packages)
    mesh = prm.mesh_struct(pin)
    O = po.Oracle(params, mesh)
    base, one = O.new_containers()
    base.prim[...] = prim0
    O.exchange_ghosts(base)
    O.apply_boundary_conditions(base)
    one.prim[...] = base.prim
    one.cons[...] = base.cons
    return O, base, one


def cpu_baseline(pin, prim0, budget_s=15.0, max_steps=None):
    threads = os.cpu_count() or 1
    O, base, one = _oracle_job(pin, prim0, threads)
    dt = pin.get_or_add_real("parthenon/time", "dt_init", 1e-5)
    factor = pin.get_or_add_real("parthenon/time", "dt_factor", 2.0)
    steps = 0
    t0 = time.perf_counter()
    while True:
        est = O.step(base, one, dt)
        dt = min(factor * dt, est)
        steps += 1
        el = time.perf_counter() - t0
        if el >= budget_s or (max_steps and steps >= max_steps):
            break
    value = NX1 * NX2 * steps / el
    return {"value": round(value, 1), "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"{steps} RK2 steps of the {NX1}x{NX2} torus from its initial state "
                      f"({el:.1f} s, oracle/oracle.cc, OpenMP)"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    pin = workload_input(seed=0)
    packages, mesh, geo, prim0 = initial_state(pin)
    threads = os.cpu_count() or 1
    O, base, one = _oracle_job(pin, prim0, threads)
    dt = pin.get_or_add_real("parthenon/time", "dt_init", 1e-5)
    factor = pin.get_or_add_real("parthenon/time", "dt_factor", 2.0)
    for _ in range(min(args.warmup, 1)):
        dt = min(factor * dt, O.step(base, one, dt))
    budget = args.ref_budget
    steps = 0
    t0 = time.perf_counter()
    while steps < args.steps:
        dt = min(factor * dt, O.step(base, one, dt))
        steps += 1
        if time.perf_counter() - t0 >= budget:
            break
    el = time.perf_counter() - t0
    value = NX1 * NX2 * steps / el
    sample = (f"{steps} of {args.steps} RK2 steps of the {NX1}x{NX2} torus "
              f"({el:.1f} s of CPU time budget {budget:.0f} s)")
    line = {"metric": METRIC, "value": round(value, 1), "unit": METRIC, "n_gpus": 0,
            "steps": steps, "warmup": min(args.warmup, 1), "ms_per_step": round(1e3 * el / steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded torus initial conditions)", "config": config(),
            "impl": "reference",
            "cpu_baseline": {"value": round(value, 1), "unit": METRIC, "cores": threads,
                             "kind": "port", "sample": sample},
            "e2e": {"value": round(value, 1), "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--ref-budget", type=float, default=120.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-graph", action="store_true",
                    help="launch every kernel from the host instead of replaying a CUDA graph")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
