"""Benchmark of the GRMHD stage engine: zone-cycles/s on B200.

Default workload: the 2D Fishbone-Moncrief torus in MKS coordinates,
512 x 256, FP64, PPM4, LAXF, chainer C2P, electron heating (one meshblock).
A step is one RK2 cycle (two stages) of the whole grid; the job length in the
workload definition is 200 steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]
                    [--workload torus2d|ot|torus3d|batch48|serve] [--precision fp64|mixed]

Other workloads: ot (Orszag-Tang 256^2, Minkowski, MC, 100 steps), torus3d
(256 x 128 x 128 torus in 16 meshblocks of 64^3, 50 steps), batch48 (48
tori of uneven grids in one block pool, 100 steps each) and serve (a seeded
Poisson stream of Brio-Wu, Orszag-Tang and torus jobs through the serving
loop; p50/p99 job latency). --precision mixed selects FP32 primitives,
reconstruction, Riemann flux and heating; its lines report the per-field
relative L1 error against an FP64 run of the same job.

N > 1 runs under torchrun, one independent job per GPU (weak scaling, no
collective on the data path; the timing is a max over ranks). With --shard
the GPUs instead share one mesh, its blocks split over the ranks (strong
scaling; halo messages over NCCL point-to-point, dt all-reduced).
``--impl reference`` times the CPU restatement of the reference's stage path
(oracle/) on the host cores for the same workload and metric.
"""
from __future__ import annotations

import argparse
import json
import math
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
# Untimed cycles a job has run when its timed window opens (settling plus the
# W warm-up cycles): the window skips the start-up transient of the initial
# state (up to 7 % of the torus's cells fail Scheme2D in the first cycles,
# 4-60 cells per cycle after cycle 10), as the bulk of a 200-cycle job does.
SETTLED_CYCLES = 40

from pangu_b200.workloads import (BATCH_BLOCK, SINGLE, WORKLOAD_NAMES,  # noqa: E402,F401
                                  batch_jobs, initial_state, interior_cells, job_input,
                                  serve_jobs)


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def workload_input(seed=0):
    return job_input("torus2d", "fp64", seed)


def workload_name(workload, precision):
    return f"{WORKLOAD_NAMES[workload]}_{precision}"


def config(workload="torus2d", precision="fp64", extra=None):
    c = {"workload": workload_name(workload, precision)}
    if workload in SINGLE:
        c.update(SINGLE[workload][2])
        c["job_steps"] = SINGLE[workload][1]
    c.update({"precision": precision,
              "l2": "flushed (256 MiB write) before every timed step",
              "launch": "one CUDA graph replay per RK2 step"})
    if extra:
        c.update(extra)
    return c


def rel_l1(a, b):
    """Per-field relative L1 error, fields along axis 1; vector components
    (velocity 2-4, magnetic field 5-7) normalised by the whole vector."""
    nf = a.shape[1]
    a = np.moveaxis(a, 1, 0).reshape(nf, -1)
    b = np.moveaxis(b, 1, 0).reshape(nf, -1)
    num = np.abs(a - b).sum(axis=1)
    den = np.abs(b).sum(axis=1)
    for lo, hi in ((2, 5), (5, 8)):
        if nf >= hi:
            den[lo:hi] = np.maximum(den[lo:hi], den[lo:hi].sum())
    return num / np.where(den > 0, den, 1)


FIELD_NAMES = ["density", "energy", "u1", "u2", "u3", "b1", "b2", "b3", "entropy",
               "electron_entropy"]


def error_vs_fp64(pin, prim0, geo, cycles):
    """Per-field relative L1 error of the mixed form against FP64 after
    `cycles` RK2 cycles from the same initial state (both on the GPU)."""
    import torch
    from pangu_b200.engine import Simulation
    out = {}
    for prec in ("fp64", "mixed"):
        pin.set("b200", "precision", prec)
        sim = Simulation(pin)
        sim.set_primitives(prim0)
        for _ in range(cycles):
            sim.step()
        torch.cuda.synchronize()
        s = geo.interior()
        out[prec] = sim.primitives()[:, :, s[0], s[1], s[2]]
        del sim
    pin.set("b200", "precision", "mixed")
    err = rel_l1(out["mixed"], out["fp64"])
    names = FIELD_NAMES if len(err) >= 9 else FIELD_NAMES[:5] + FIELD_NAMES[8:]
    return {"cycles": cycles, "rel_l1": {n: float(f"{e:.3e}") for n, e in zip(names, err)}}


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
# The NVML sampling loop of ClockSampler, run as a separate process (a thread
# of this interpreter is starved while the main thread sits in a blocking CUDA
# call that holds the interpreter). Writes "monotonic time, SM MHz, max SM
# MHz, power W, clock-event reason bits" lines until it is terminated.
_NVML_SAMPLER = r"""
import sys, time
import pynvml as nv
nv.nvmlInit()
want = tuple(int(a) for a in sys.argv[1:4])
h = None
for n in range(nv.nvmlDeviceGetCount()):
    c = nv.nvmlDeviceGetHandleByIndex(n)
    pci = nv.nvmlDeviceGetPciInfo(c)
    if (pci.domain, pci.bus, pci.device) == want:
        h = c
if h is None:
    sys.exit(3)
smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
while True:
    t = time.monotonic()
    sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
    pw = nv.nvmlDeviceGetPowerUsage(h) / 1e3
    rb = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
    sys.stdout.write("%.6f,%d,%d,%.1f,%d\n" % (t, sm, smax, pw, rb))
    sys.stdout.flush()
    time.sleep(0.0005)
"""


class ClockSampler:
    """SM clock, power and clock-event reasons of the benchmarked GPU during
    the timed region: a separate process reads NVML about every millisecond
    (NVML's device is the one with the CUDA device's PCI domain, bus and
    device numbers: NVML enumerates every GPU of the machine, CUDA only the
    visible ones), and the samples stamped inside the region are kept.
    Falls back to nvidia-smi (100 ms period) when NVML cannot be opened."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40),
               ("sw_thermal_slowdown", 0x20), ("sw_power_cap", 0x4))

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.nvml = False
        self.t0 = self.t1 = None

    def _start(self, cmd):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.out = open(self.path, "w")
        self.proc = subprocess.Popen(cmd, stdout=self.out, stderr=subprocess.DEVNULL)

    def _stop(self):
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.close()
        self.proc = None

    def __enter__(self):
        import torch
        props = torch.cuda.get_device_properties(self.gpu)
        pci = (props.pci_domain_id, props.pci_bus_id, props.pci_device_id)
        try:
            self._start([sys.executable, "-c", _NVML_SAMPLER, *map(str, pci)])
            # wait for the first sample (or the sampler's exit)
            deadline = time.monotonic() + 20.0
            while time.monotonic() < deadline and self.proc.poll() is None and \
                    os.path.getsize(self.path) == 0:
                time.sleep(0.01)
            self.nvml = os.path.getsize(self.path) > 0
        except OSError:
            self.nvml = False
        if not self.nvml:
            self._stop()
            try:
                self._start(["nvidia-smi", f"--query-gpu={self.FIELDS}",
                             "--format=csv,noheader,nounits", "-lms", "100",
                             "-i", str(self.gpu)])
            except (OSError, FileNotFoundError):
                self.proc = None
        self.t0 = time.monotonic()
        return self

    def __exit__(self, *exc):
        self.t1 = time.monotonic()
        self._stop()

    def summary(self):
        rows = []
        src = "nvml in a separate process, ~1 ms period, samples stamped inside the timed region"
        if self.path and os.path.exists(self.path):
            with open(self.path) as f:
                lines = f.read().splitlines()
            os.unlink(self.path)
            if self.nvml:
                for line in lines:
                    parts = line.split(",")
                    if len(parts) != 5:
                        continue
                    t = float(parts[0])
                    if self.t0 <= t <= self.t1:
                        rows.append((float(parts[1]), float(parts[2]), float(parts[3]),
                                     int(parts[4])))
            else:
                src = "nvidia-smi, 100 ms period, during the timed region"
                bits = [b for _, b in self.REASONS]
                for line in lines:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) == 9 and parts[1].replace(".", "", 1).isdigit():
                        rb = sum(b for b, v in zip(bits, parts[5:9]) if v == "Active")
                        rows.append((float(parts[1]), float(parts[2]), None, rb))
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        reasons = sorted({n for r in rows for n, b in self.REASONS if r[3] & b})
        pw = [r[2] for r in rows if r[2] is not None]
        out = {"sm_mhz": statistics.median(r[0] for r in rows),
               "sm_max_mhz": max(r[1] for r in rows), "reasons": reasons,
               "samples": len(rows), "power_w_max": round(max(pw), 1) if pw else None,
               "source": src}
        if self.t0 is not None and self.t1 is not None:
            out["window_ms"] = round(1e3 * (self.t1 - self.t0), 1)
        return out


def wait_event(ev):
    """Waits for a recorded CUDA event by polling it with short sleeps (the
    host returns as soon as the device is done, and the sampler's window
    closes with the timed region)."""
    while not ev.query():
        time.sleep(0.0002)


# ---------------------------------------------------------------------------
# algorithmic bytes per launch of each task (FP64, NF fields)
# ---------------------------------------------------------------------------
def task_bytes(nf, n_int, n_ent, ndim, pw=8):
    """Compulsory bytes of each task launch; pw = bytes per stored primitive."""
    w = 8
    return {
        "fix_primitive": 2 * nf * pw * n_ent,
        "calculate_conservative": (nf * pw + nf * w) * n_int,
        "calculate_fluxes": (nf * pw + ndim * (nf * w + w)) * n_int,
        "constrained_transport": (2 * ndim * w + 3 * w + 2 * ndim * w) * n_int,
        "flux_divergence_update": (ndim * nf * w + 2 * nf * w) * n_int,
        "add_geometric_source": (nf * pw + 2 * 4 * w) * n_int,
        "recovery": (9 * w + 9 * pw + 8 * pw + w) * n_int,
        "apply_electron_heating": (nf * pw + 3 * w + pw) * n_int,
        "fix_recovery": w * n_int,
        "apply_boundary_conditions": 0,
        "estimate_dt": ndim * w * n_int,
    }


def settle_cycles(args):
    """Untimed cycles run before the W warm-up cycles."""
    return max(0, SETTLED_CYCLES - args.warmup)


def timed_window(args, graph=True):
    """The job cycles the timed steps cover (the graph's first replay is one
    more untimed cycle)."""
    first = settle_cycles(args) + args.warmup + (2 if graph else 1)
    return (f"cycles {first}-{first + args.steps - 1} of the job "
            f"({settle_cycles(args)} settling and {args.warmup} warm-up cycles before, untimed)")


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

    pin = job_input(args.workload, args.precision, seed=rank)
    packages, mesh, geo, prim0 = initial_state(pin)
    sim = Simulation(pin, device=local)
    sim.set_primitives(prim0)
    n_int = interior_cells(pin)
    ndim = 1 + (mesh.nx2 > 1) + (mesh.nx3 > 1)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    for _ in range(settle_cycles(args) + args.warmup):
        sim.step()
    torch.cuda.synchronize()
    sim.autotune()  # flux tile shapes for this grid (results do not depend on them)
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
        wait_event(ends[-1])
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
        pw = sim.base.prim.element_size()
        tb = task_bytes(nf, n_int, n_ent, ndim, pw)
        dom = max(tasks, key=lambda k: tasks[k])
        achieved = tb[dom] / (tasks[dom] / 1e3) / 1e9
        wl = workload_name(args.workload, args.precision)
        traffic_figs, traffic_status = profile_figures("traffic", wl)
        step_bytes = 2 * (2 * nf * pw + 3 * nf * 8) * n_int
        roof = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 2),
                "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                "frac": round(achieved / peak, 5), "traffic": _fig(traffic_figs, dom),
                "traffic_profile": f"profiles/traffic_{wl}.txt ({traffic_status})",
                "algorithmic_bytes_per_launch": tb[dom], "launch_ms": round(tasks[dom], 5),
                "step_algorithmic_bytes": step_bytes,
                "step_achieved_gbs": round(step_bytes * value / n_int / world / 1e9, 2),
                "step_frac": round(step_bytes * value / n_int / world / 1e9 / peak, 5),
                "task_ms": {k: round(v, 5) for k, v in tasks.items()},
                "task_ms_note": "each task launched alone from the host, L2 flushed before "
                                "every launch (cold caches), mean of 20 launches; achieved "
                                "uses the dominant task's time"}
        # FP64 roofline: the kernels are bound by FP64 issue and latency, so
        # the step's FP64 operations against the FP64 FMA peak measured here
        fp_figs, fp_status = profile_figures("fp64_ops", wl)
        fp_peak = fp64_peak_tflops(dev)
        fpz = _fig(fp_figs, "flops_per_zone_cycle")
        roof_fp64 = {"bound": "fp64", "unit": "TFLOP/s",
                     "peak": round(fp_peak, 3) if fp_peak else None,
                     "peak_kind": "measured in this run (pangu_fp64_peak, DFMA)",
                     "flops_per_zone_cycle": fpz,
                     "profile": f"profiles/fp64_ops_{wl}.txt ({fp_status})"}
        if fpz and fp_peak:
            ach = fpz * value / world / 1e12
            roof_fp64.update({"achieved": round(ach, 3), "frac": round(ach / fp_peak, 4)})
            kf = _fig(fp_figs, f"flops_per_launch_{dom}")
            if kf:
                ka = kf / (tasks[dom] / 1e3) / 1e12
                roof_fp64.update({"kernel": dom, "kernel_achieved": round(ka, 3),
                                  "kernel_frac": round(ka / fp_peak, 4)})
            pipe = _fig(fp_figs, "fp64_pipe_active_pct_step")
            if pipe is not None:
                roof_fp64["fp64_pipe_active_pct_step"] = pipe
        tiles = sim.engine.flux_config()
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            pin.set("b200", "precision", "fp64")
            cpu = cpu_baseline(pin, prim0, budget_s=args.cpu_budget)
            pin.set("b200", "precision", args.precision)
        err = None
        if args.precision == "mixed":
            del sim
            err = error_vs_fp64(pin, prim0, geo, min(SINGLE[args.workload][1], 50))
        e2e_value = world * n_int * e2e["steps"] / (e2e["ms"] / 1e3)
        line = {"metric": METRIC, "value": round(value, 1), "unit": METRIC, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 5),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "f32/f64 mixed",
                "data": "synthetic (seeded initial conditions)",
                "config": config(args.workload, args.precision,
                                 {"parallelism": f"{world} independent jobs, one per GPU",
                                  "timed_window": timed_window(args, not args.no_graph)}),
                "e2e": {"value": round(e2e_value, 1), "unit": METRIC,
                        "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"],
                        "steps": e2e["steps"]},
                "roofline": roof, "roofline_fp64": roof_fp64, "cpu_baseline": cpu,
                "clocks": clocks,
                "gpu_launches": launches, "flux_tiles": tiles}
        if err is not None:
            line["error_vs_fp64"] = err
        if world == 1 and args.precision == "fp64" and not args.no_extra_legs:
            # the metric's other halves: the mixed form on the same workload,
            # and a saturated serving stream in both precisions
            del sim
            line["mixed"] = mixed_leg(args, pin, prim0, geo, flush, dev, value)
            line["serving_saturated"] = saturated_serving()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


def mixed_leg(args, pin, prim0, geo, flush, dev, fp64_value):
    """The mixed form on the same job, timed like the FP64 line (warm-up, tile
    tuning, one CUDA graph per RK2 cycle, L2 flushed before each timed step,
    CUDA events), with its per-field relative L1 error against FP64 after 50
    cycles."""
    import torch

    from pangu_b200.engine import Simulation
    pin.set("b200", "precision", "mixed")
    sim = Simulation(pin, device=dev.index or 0)
    sim.set_primitives(prim0)
    for _ in range(settle_cycles(args) + args.warmup):
        sim.step()
    torch.cuda.synchronize()
    sim.autotune()
    sim.capture()
    sim.step()
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with ClockSampler(dev.index or 0) as clk:
        for s in range(args.steps):
            flush.zero_()
            starts[s].record()
            sim.step()
            ends[s].record()
        wait_event(ends[-1])
        torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in zip(starts, ends)) / args.steps
    value = interior_cells(pin) / (ms / 1e3)
    tiles = sim.engine.flux_config()
    del sim
    err = error_vs_fp64(pin, prim0, geo, min(SINGLE[args.workload][1], 50))
    pin.set("b200", "precision", "fp64")
    return {"value": round(value, 1), "unit": METRIC, "ms_per_step": round(ms, 5),
            "over_fp64": round(value / fp64_value, 3), "dtype": "f32/f64 mixed",
            "error_vs_fp64": err, "clocks": clk.summary(), "flux_tiles": tiles}


def run_sharded(args):
    """One mesh over all ranks (block sharding, strong scaling): rank r steps
    its contiguous run of the block lattice, the halo messages move with NCCL
    point-to-point calls while the middle of each stage runs, and dt is
    reduced with an all-reduce(min). value = the mesh's cells x cycles / the
    slowest rank's device time."""
    import datetime

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ.setdefault("MASTER_PORT", "29517")
    os.environ.setdefault("RANK", "0")
    os.environ.setdefault("WORLD_SIZE", "1")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                            device_id=dev)
    from pangu_b200.shard import ShardedSimulation

    pin = job_input(args.workload, args.precision, seed=0)  # the same mesh on every rank
    packages, mesh, geo, prim0 = initial_state(pin)
    sim = ShardedSimulation(pin, device=local)
    sim.set_primitives(prim0)
    n_int = interior_cells(pin)
    for _ in range(args.warmup):
        sim.step()
    torch.cuda.synchronize()
    dist.barrier()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    launches0 = sim.engine.launches()
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        for s in range(args.steps):
            starts[s].record()
            sim.step()
            ends[s].record()
        wait_event(ends[-1])
        torch.cuda.synchronize()
    launches = sim.engine.launches() - launches0
    total_ms = sum(a.elapsed_time(b) for a, b in zip(starts, ends))
    total_ms = max_over_ranks(total_ms, dist, dev)
    halo = 8 * sim.width * (sum(sim.send_counts) + sum(sim.recv_counts))
    halo = max_over_ranks(halo, dist, dev)
    counters = sim.total_counters()
    dist.barrier()
    dist.destroy_process_group()
    if rank != 0:
        return
    value = n_int * args.steps / (total_ms / 1e3)
    line = {"metric": METRIC, "value": round(value, 1), "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(total_ms / args.steps, 5), "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32/f64 mixed",
            "data": "synthetic (seeded initial conditions)",
            "config": config(args.workload, args.precision,
                             {"parallelism": f"one mesh, blocks sharded over {world} GPUs",
                              "halo_bytes_per_stage_max_rank": int(halo),
                              "l2": "not flushed: each rank's state is larger than L2",
                              "launch": "host-launched stage parts, NCCL point-to-point halos"}),
            "e2e": None, "roofline": None, "cpu_baseline": None, "clocks": clk.summary(),
            "gpu_launches": launches,
            "c2p_fail_cells": int(counters[6])}
    print(json.dumps(line), flush=True)


def e2e_run(sim, torch, dev, steps):
    """Steps with the job state resident on the HOST, through the public API
    (Simulation.step_host): every step copies the state in from pinned memory,
    runs the RK2 cycle and copies it back, the copies overlapped with the
    kernels that do not need them."""
    from pangu_b200.engine import HostState
    host = HostState(sim)
    sim.pull(host)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        sim.step_host(host)
    e1.record()
    torch.cuda.synchronize()
    return {"ms": e0.elapsed_time(e1), "steps": steps, "h2d": host.nbytes, "d2h": host.nbytes}


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


def profile_figures(kind, workload):
    """Figures of a committed profile summary, profiles/<kind>_<workload>.txt
    (lines 'name value ...'), with its status: "current" when its 'build' line
    is the fingerprint of the engine sources that this run executes, "stale"
    otherwise (then no figure is returned: a measurement of other sources is
    never reported against this build), "missing" without the file."""
    from pangu_b200 import build as engine_build
    path = os.path.join(ROOT, "profiles", f"{kind}_{workload}.txt")
    if not os.path.exists(path):
        return None, "missing"
    figs = {}
    with open(path) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 2 and not line.startswith("#"):
                figs[parts[0]] = parts[1:]
    if figs.get("build", [None])[0] != engine_build.source_hash():
        return None, "stale"
    return figs, "current"


def _fig(figs, key):
    try:
        return float(figs[key][0]) if figs and key in figs else None
    except ValueError:
        return None


def fp64_peak_tflops(dev, reps=5):
    """FP64 FMA throughput of this GPU (pangu_fp64_peak: eight independent
    DFMA chains per thread, 1184 CTAs of 256 threads), best of `reps` launches
    timed with CUDA events on the launching stream, in TFLOP/s."""
    import ctypes as C

    import torch

    from pangu_b200 import engine
    L = engine.lib()
    L.pangu_fp64_peak.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    L.pangu_fp64_peak_flops.argtypes = [C.c_int, C.c_int]
    L.pangu_fp64_peak_flops.restype = C.c_double
    ctas, iters = 148 * 8, 8192
    sink = torch.zeros(ctas, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    best = None
    for r in range(reps + 1):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rc = L.pangu_fp64_peak(ctas, iters, C.c_void_p(sink.data_ptr()),
                               C.c_void_p(stream.cuda_stream))
        b.record(stream)
        torch.cuda.synchronize(dev)
        if rc != 0:
            return None
        if r:  # the first launch warms up
            ms = a.elapsed_time(b)
            best = ms if best is None else min(best, ms)
    return L.pangu_fp64_peak_flops(ctas, iters) / (best / 1e3) / 1e12


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


class ReferenceJob:
    """One job stepped by the REFERENCE's own stage tasks (pangu/src compiled
    here over the Parthenon stand-in, timing build: OpenMP over par_for, the C
    library's pow, -O3), in the order of ideal_grmhd.cc:62-110, with the
    restatement's versions of the parts Parthenon does (update, ghost
    exchange, boundary conditions). Used where that library exists (it is
    built from the reference's sources and travels with the repository);
    otherwise the restatement alone (oracle.cc) is timed."""

    KIND = "reference"
    WHAT = ("the reference's stage tasks (pangu/src over a Parthenon stand-in, OpenMP) with "
            "the restatement's update, exchange and boundaries")

    def __init__(self, pin, prim0, threads):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle as po
        self.O, self.base, self.one = _oracle_job(pin, prim0, threads)
        packages = prm.process_packages(pin)
        self.params = prm.params_struct(packages)
        self.R = po.RefTasks(self.params, prm.mesh_struct(pin), timing=True)

    def settle(self, n, dt, factor):
        """n untimed cycles by the restatement (the same stage, faster), from
        which the reference's tasks take over; returns the next dt."""
        for _ in range(n):
            dt = min(factor * dt, self.O.step(self.base, self.one, dt))
        return dt

    def step(self, dt):
        O, R, p = self.O, self.R, self.params
        est = None
        for st, beta in ((1, 0.5), (2, 1.0)):
            c0, c1 = (self.base, self.one) if st == 1 else (self.one, self.base)
            R.run("fix_primitive", c0)
            R.run("calculate_conservative", c0)
            R.run("calculate_fluxes", c0)
            if p.enable_B:
                R.run("constrained_transport", c0)
            O.flux_divergence_update(self.base, c0, c1, beta * dt)
            O.exchange_ghosts(c1)
            R.run("add_geometric_source", c1, beta * dt)
            R.run("recovery", c1)
            if p.enable_heating:
                R.run("apply_electron_heating", c1)
            if p.recovery == 0:
                R.run("fix_recovery", c1)
            O.apply_boundary_conditions(c1)
            if st == 2:
                est = R.run("estimate_dt", c1)
        return est


class PortJob:
    """One job stepped by the CPU restatement (oracle.cc, OpenMP)."""

    KIND = "port"
    WHAT = "oracle/oracle.cc, OpenMP"

    def __init__(self, pin, prim0, threads):
        self.O, self.base, self.one = _oracle_job(pin, prim0, threads)

    def settle(self, n, dt, factor):
        for _ in range(n):
            dt = min(factor * dt, self.O.step(self.base, self.one, dt))
        return dt

    def step(self, dt):
        return self.O.step(self.base, self.one, dt)


def cpu_job(pin, prim0, threads):
    """The reference's own tasks where their library exists, else the port."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    if po.reftasks_omp() is not None:
        return ReferenceJob(pin, prim0, threads)
    return PortJob(pin, prim0, threads)


def cpu_baseline(pin, prim0, budget_s=15.0, max_steps=None):
    threads = os.cpu_count() or 1
    job = cpu_job(pin, prim0, threads)
    dt = pin.get_or_add_real("parthenon/time", "dt_init", 1e-5)
    factor = pin.get_or_add_real("parthenon/time", "dt_factor", 2.0)
    dt = job.settle(SETTLED_CYCLES, dt, factor)
    steps = 0
    t0 = time.perf_counter()
    while True:
        est = job.step(dt)
        dt = min(factor * dt, est)
        steps += 1
        el = time.perf_counter() - t0
        if el >= budget_s or (max_steps and steps >= max_steps):
            break
    value = interior_cells(pin) * steps / el
    return {"value": round(value, 1), "unit": METRIC, "cores": threads, "kind": job.KIND,
            "sample": f"{steps} RK2 steps of the same job from cycle {SETTLED_CYCLES + 1} "
                      f"({el:.1f} s, {job.WHAT}, FP64)"}


# ---------------------------------------------------------------------------
# batch of 48 tori in one block pool
# ---------------------------------------------------------------------------
def run_batch(args):
    import torch
    from pangu_b200.engine import Pool
    pins, states = batch_jobs(args.precision, states=True)
    nblocks = [st.shape[0] for st in states]
    pool = Pool(pins[0], sum(nblocks), len(pins))
    for pin, st in zip(pins, states):
        pool.attach(pin, st)
    n_int = sum(interior_cells(pin) for pin in pins)
    for _ in range(args.warmup):
        pool.step(graph=False)
    torch.cuda.synchronize()
    pool.autotune()
    launches0 = pool.engine.launches()
    pool.step()  # captures the cycle graph, then replays it
    torch.cuda.synchronize()
    per_step = pool.engine.launches() - launches0
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        e0.record()
        for _ in range(args.steps):
            pool.step()
        e1.record()
        wait_event(e1)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    value = n_int * args.steps / (ms / 1e3)
    # end to end: every job's state in from pinned host memory and back out
    # around each cycle
    h = torch.empty(pool.base.prim.shape, dtype=pool.base.prim.dtype).pin_memory()
    h.copy_(pool.base.prim)
    torch.cuda.synchronize()
    k = min(args.steps, 20)
    e0.record()
    for _ in range(k):
        pool.base.prim.copy_(h, non_blocking=True)
        pool.step()
        h.copy_(pool.base.prim, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e = n_int * k / (e0.elapsed_time(e1) / 1e3)
    nbytes = h.numel() * h.element_size()
    err = None
    if args.precision == "mixed":
        err, seen = {}, set()
        for pin, st in zip(pins, states):  # one job of each grid
            nx = pin.get_or_add_integer("parthenon/mesh", "nx1", 1)
            ny = pin.get_or_add_integer("parthenon/mesh", "nx2", 1)
            if (nx, ny) in seen:
                continue
            seen.add((nx, ny))
            geo = problems.Geometry(prm.mesh_struct(pin))
            err[f"{nx}x{ny}"] = error_vs_fp64(pin, st, geo, 50)
    line = {"metric": METRIC, "value": round(value, 1), "unit": METRIC, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 5), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32/f64 mixed",
            "data": "synthetic (seeded torus initial conditions)",
            "config": config("batch48", args.precision, {
                "jobs": len(pins), "meshblock": "128x64", "blocks": sum(nblocks),
                "interior_cells": n_int, "job_steps": 100,
                "l2": "not flushed: the state (prim + cons + fluxes) is far larger than L2",
                "launch": "one CUDA graph replay per RK2 step of all 48 jobs"}),
            "e2e": {"value": round(e2e, 1), "unit": METRIC, "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes, "steps": k},
            "clocks": clk.summary(), "gpu_launches": per_step * args.steps,
            "flux_tiles": pool.engine.flux_config()}
    if err is not None:
        line["error_vs_fp64"] = err
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# serving stream
# ---------------------------------------------------------------------------
def serve_stream(precision, n_jobs, rate, capacity_fraction=1.0, lazy=False):
    """Runs a seeded job stream through the serving loop (pangu_server_*).
    Each class's pool holds capacity_fraction of the blocks its jobs need
    together (at least its largest job), so with a fraction below 1 jobs wait
    for slots; lazy classes are charged against the 150 GB budget at their
    first admission and released when idle. Returns (stats, latencies, queue
    times, info)."""
    import torch  # noqa: F401  (initialises the CUDA context)
    from pangu_b200.engine import Server
    jobs = serve_jobs(precision, n_jobs, rate)
    budget = 150 << 30
    srv = Server(budget)
    need, biggest, tmpl, count = {}, {}, {}, {}
    for kind, pin, _, _ in jobs:
        m = prm.mesh_struct(pin)
        nb = m.nbx1 * m.nbx2 * m.nbx3
        need[kind] = need.get(kind, 0) + nb
        biggest[kind] = max(biggest.get(kind, 0), nb)
        count[kind] = count.get(kind, 0) + 1
        tmpl.setdefault(kind, pin)
    cap = {k: max(biggest[k], math.ceil(capacity_fraction * need[k])) for k in tmpl}
    cls = {k: srv.add_class(tmpl[k], cap[k], count[k], lazy=lazy) for k in sorted(tmpl)}
    # initial states are generated on the device at admission (pangu_generate)
    for kind, pin, cycles, t in jobs:
        srv.submit_problem(cls[kind], pin, kind, cycles, t)
    with ClockSampler(0) as clk:
        srv.run()
    st = srv.stats()
    res = [srv.result(tk)[1] for tk in range(len(jobs))]
    lat = sorted(float(r[2] - r[0]) for r in res)
    queued = sorted(float(r[1] - r[0]) for r in res)
    per_job = 0
    for _, pin, _, _ in jobs:
        m = prm.mesh_struct(pin)
        nf = prm.num_components(True, pin.get_or_add_boolean("core", "enable_heating", False))
        cells = 1
        for n in (m.nx1, m.nx2, m.nx3):
            cells *= n + (2 * m.ng if n > 1 else 0)
        per_job += m.nbx1 * m.nbx2 * m.nbx3 * nf * cells * 8
    info = {"jobs": len(jobs), "arrival_rate_per_s": rate, "job_cycles": "U{200..2000}",
            "hbm_budget_bytes": budget, "hbm_peak_bytes": st["hbm_peak_bytes"],
            "memory_waits": st["memory_waits"], "lazy_classes": lazy,
            "classes": {k: {"jobs": count[k], "blocks_needed": need[k],
                            "capacity_blocks": cap[k]} for k in cls},
            "queue_s": {"p50": round(queued[len(queued) // 2], 4), "max": round(queued[-1], 4)},
            "d2h_bytes_per_job": per_job // len(jobs), "clocks": clk.summary()}
    return st, lat, queued, info


def run_serve(args):
    st, lat, queued, info = serve_stream(args.precision, args.serve_jobs, args.serve_rate,
                                         args.serve_capacity, args.serve_lazy)
    clocks = info.pop("clocks")
    per_job = info.pop("d2h_bytes_per_job")
    line = {"metric": METRIC, "value": round(st["zone_cycles_per_s"], 1), "unit": METRIC,
            "n_gpus": 1, "steps": int(st["ticks"]), "warmup": 0, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32/f64 mixed",
            "data": "synthetic (seeded job stream and initial conditions)",
            "config": config("serve", args.precision, dict(info, **{
                "l2": "not flushed (continuous stream)",
                "launch": "one CUDA graph launch per class tick"})),
            "latency_s": {"p50": round(st["p50_s"], 4), "p99": round(st["p99_s"], 4),
                          "max": round(lat[-1], 4)},
            "wall_s": round(st["wall_s"], 3),
            "e2e": {"value": round(st["zone_cycles_per_s"], 1), "unit": METRIC,
                    "h2d_bytes_per_job": 0, "d2h_bytes_per_job": per_job,
                    "note": "host wall clock from the first arrival to the last completion; "
                            "initial states generated on the device at admission, results "
                            "copied to the host at completion"},
            "clocks": clocks}
    print(json.dumps(line), flush=True)


def saturated_serving():
    """The serving stream with every job arriving at once (arrivals faster than
    the GPU serves them), class pools holding a third of the blocks their jobs
    need (so admission gates on free slots), classes charged against the HBM
    budget at their first admission; FP64 and the mixed form."""
    out = {}
    for prec in ("fp64", "mixed"):
        st, lat, queued, info = serve_stream(prec, 36, 1e4, 1.0 / 3.0, lazy=True)
        out[prec] = {"zone_cycles_per_s": round(st["zone_cycles_per_s"], 1),
                     "p50_s": round(st["p50_s"], 4), "p99_s": round(st["p99_s"], 4),
                     "wall_s": round(st["wall_s"], 3), "queue_s": info["queue_s"],
                     "hbm_peak_bytes": info["hbm_peak_bytes"], "clocks": info["clocks"]}
    out["mixed_over_fp64"] = round(out["mixed"]["zone_cycles_per_s"] /
                                   out["fp64"]["zone_cycles_per_s"], 3)
    out["stream"] = ("36 jobs (Brio-Wu 1024-8192 cells, Orszag-Tang 128^2-512^2, MKS tori "
                     "256x128-512x256; 200-2000 RK2 cycles), all arriving at t = 0, pools of a "
                     "third of each class's blocks, 150 GB budget charged at admission")
    return out


# ---------------------------------------------------------------------------
# reference arm: the CPU restatement on the host cores
# ---------------------------------------------------------------------------
def reference_jobs(args):
    if args.workload in SINGLE:
        return [job_input(args.workload, "fp64", 0)]
    if args.workload == "batch48":
        return batch_jobs("fp64")
    return [pin for _, pin, _, _ in serve_jobs("fp64", args.serve_jobs, args.serve_rate)]


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    pins = reference_jobs(args)[:4]
    runs = []
    for pin in pins:
        pin.set("b200", "precision", "fp64")
        prim0 = initial_state(pin)[3]
        job = cpu_job(pin, prim0, threads)
        dt = pin.get_or_add_real("parthenon/time", "dt_init", 1e-5)
        factor = pin.get_or_add_real("parthenon/time", "dt_factor", 2.0)
        # the engine's timed window opens after the start-up transient too
        dt = job.settle(settle_cycles(args), dt, factor)
        runs.append([job, dt, factor, interior_cells(pin)])
    kind, what = runs[0][0].KIND, runs[0][0].WHAT
    budget = args.ref_budget
    # W untimed warm-up steps, round robin over the jobs like the timed ones
    # (bounded by the same time budget)
    warm = 0
    t0 = time.perf_counter()
    while warm < args.warmup and time.perf_counter() - t0 < budget:
        r = runs[warm % len(runs)]
        r[1] = min(r[2] * r[1], r[0].step(r[1]))
        warm += 1
    steps, cells = 0, 0
    t0 = time.perf_counter()
    while steps < args.steps:
        r = runs[steps % len(runs)]
        r[1] = min(r[2] * r[1], r[0].step(r[1]))
        cells += r[3]
        steps += 1
        if time.perf_counter() - t0 >= budget:
            break
    el = time.perf_counter() - t0
    value = cells / el
    sample = (f"{steps} of {args.steps} RK2 steps, round robin over {len(runs)} job(s) of the "
              f"workload after {settle_cycles(args)} settling and {warm} warm-up cycles "
              f"({el:.1f} s of CPU time budget {budget:.0f} s, {what}, FP64)")
    line = {"metric": METRIC, "value": round(value, 1), "unit": METRIC, "n_gpus": 0,
            "steps": steps, "warmup": warm,
            "ms_per_step": round(1e3 * el / steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded initial conditions)",
            "config": config(args.workload, args.precision), "impl": "reference",
            "cpu_baseline": {"value": round(value, 1), "unit": METRIC, "cores": threads,
                             "kind": kind, "sample": sample},
            "e2e": {"value": round(value, 1), "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--workload",
                    choices=["torus2d", "ot", "torus3d", "cks3d", "batch48", "serve"],
                    default="torus2d")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--ref-budget", type=float, default=120.0)
    ap.add_argument("--serve-jobs", type=int, default=36)
    ap.add_argument("--serve-rate", type=float, default=6.0, help="job arrivals per second")
    ap.add_argument("--serve-capacity", type=float, default=1.0,
                    help="pool slots per class as a fraction of the blocks its jobs need")
    ap.add_argument("--serve-lazy", action="store_true",
                    help="charge each class against the HBM budget at its first admission")
    ap.add_argument("--no-extra-legs", action="store_true",
                    help="leave the mixed-form and saturated-serving legs out of the line")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-graph", action="store_true",
                    help="launch every kernel from the host instead of replaying a CUDA graph")
    ap.add_argument("--shard", action="store_true",
                    help="one mesh with its blocks sharded over the GPUs (strong scaling) "
                         "instead of one independent job per GPU")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
    elif args.shard:
        if args.workload not in SINGLE:
            ap.error("--shard takes a single-mesh workload (torus2d, ot, torus3d)")
        run_sharded(args)
    elif args.workload == "batch48":
        run_batch(args)
    elif args.workload == "serve":
        run_serve(args)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
