#!/usr/bin/env python
"""CW-FDTD benchmark: Gcell-updates/s of the B200 solver against its HBM roofline.

Workload (default): the 2x2 MMI-like block, 321 x 161 x 101 cells (5.22 M) at
0.025 um, 20-cell CPML, seeded projected design density, run to steady state at
rtol = 1e-6 in the fp32 storage form.  One bench "step" is one complete CW solve
(ramp, convergence probes every Tn steps, t0/t1 captures, 3-sample extraction).

Reported in one JSON line (rank 0):
  value       cell-updates / device time of the time-stepping (CUDA events on the
              library's stream; materials already resident), summed over ranks
              (each rank solves its own seeded replica: weak scaling)
  e2e         the same metric through the public API ``FDTD.solve_forward`` with
              host buffers: material upload, solve, complex-field download and
              the source-power post-processing, wall clock
  roofline    algorithmic bytes per time step (60 B per cell fp32 / 120 B fp64,
              plus 32 / 64 B per cell and CPML slab) / average step time, against
              the measured HBM copy bandwidth
  fp64        the plain fp64 solve of the same problem and the fp32 error vs it
  cpu_baseline  the reference C++ core (oracle/_ref/FDTD.so, compiled from the
              reference sources) on the host cores, z-slab threads, bounded sample

``--impl reference`` times that reference core alone (rank 0) on the same metric.
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

METRIC = "Gcell-updates/s (CW-FDTD, fp32 storage, MMI block 321x161x101, rtol=1e-6)"
UNIT = "Gcell-updates/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--kernel", default="auto",
                    choices=["auto", "scalar", "fused", "vector", "split"])
    ap.add_argument("--workload", default="mmi",
                    choices=["mmi", "waveguide", "serving", "grad", "grating", "zslab", "modes"])
    ap.add_argument("--slabs", type=int, default=2,
                    help="zslab on one process: z slabs on this GPU (under torchrun: one per rank)")
    ap.add_argument("--copy-halo", action="store_true",
                    help="zslab on one process: exchange halo planes by device copies instead of "
                         "reading the neighbouring slabs' planes in place")
    ap.add_argument("--host-loop", action="store_true",
                    help="zslab on one process: launch every step from the host instead of replaying "
                         "one captured step")
    ap.add_argument("--overlap", action="store_true",
                    help="zslab on one process: halo copies on a side stream, half steps split around "
                         "them (the schedule of the NCCL transport)")
    ap.add_argument("--requests", type=int, default=512, help="serving: requests in the stream")
    ap.add_argument("--rate", type=float, default=20.0, help="serving: mean arrivals per second")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="serving: HBM budget")
    ap.add_argument("--fixed-steps", type=int, default=0,
                    help="run every solve for this many main steps instead of to rtol "
                         "(short runs for profiler captures)")
    ap.add_argument("--request-shape", default="",
                    help="serving: give every request this grid, 'Nz,Ny,Nx' (d = 0.025 um, "
                         "wavelength 1.55 um, 20-cell CPML)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-fp64", action="store_true", help="skip the fp64 comparison solve")
    ap.add_argument("--no-serving", action="store_true",
                    help="default workload: skip the serving-stream sub-object")
    ap.add_argument("--no-grating", action="store_true",
                    help="default workload: skip the grating-slab sub-object")
    return ap.parse_args()


def make_problem(workload: str, seed: int, fixed_steps: int = 0):
    from emopt_b200 import problems as P
    if workload == "mmi":
        return P.mmi_block(seed=seed, fixed_steps=fixed_steps or None)
    return P.waveguide(fixed_steps=fixed_steps or None)


def algorithmic_bytes_per_step(shape, w, word: int) -> int:
    """Bulk: read E, H (6 words) and the 3 E-update coefficients, write E, H (6)
    = 15 words per cell; each CPML slab a cell lies in adds 4 psi reads and 4
    psi writes.  The z-max slab has w-1 active planes (strict comparison)."""
    Nz, Ny, Nx = shape
    n = Nz * Ny * Nx
    slab = (Nz * Ny * (min(w[0], Nx) + min(w[1], Nx)) + Nz * Nx * (min(w[2], Ny) + min(w[3], Ny))
            + Ny * Nx * (min(w[4], Nz) + max(min(w[5], Nz) - 1, 0)))
    return word * (15 * n + 8 * slab)


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        try:
            rows = [l.split(",") for l in open(self.path).read().strip().splitlines() if l.strip()]
            os.unlink(self.path)
        except Exception:
            return out
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except ValueError:
                continue
            for name, val in zip(names, r[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if sm:
            out.update(sm_mhz=statistics.median(sm), sm_max_mhz=max(mx), samples=len(sm),
                       reasons=sorted(reasons))
        return out


def dist_setup(n_gpus: int):
    """One process per GPU (torchrun env): NCCL when the GPUs are visible,
    gloo on a CPU-only host (the multi-process tests).  Ranks solve their
    own seeded replica: no collective on the data path, only the timing
    reductions below."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def _reduce(values: list[float], world: int, op):
    if world == 1:
        return values
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor(values, dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op))
    return t.tolist()


def barrier_max(values: list[float], world: int):
    """Max over ranks of each value (device-timed seconds)."""
    return _reduce(values, world, "MAX")


def barrier_sum(values: list[float], world: int):
    """Sum over ranks of each value (cell updates)."""
    return _reduce(values, world, "SUM")


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_baseline(p, budget_s: float = 12.0):
    """Reference core on the host cores (z-slab threads), bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import oracle_for
    from oracle import driver
    kind = "reference" if driver.available("ref") else "port"
    lib = "ref" if kind == "reference" else "oracle"
    try:
        cores = len(os.sched_getaffinity(0))
    except Exception:
        cores = os.cpu_count() or 1
    o = oracle_for(p, lib)
    t_cal = o.run_fixed_slabs(0, cores, time_only_steps=2)
    steps = max(2, int(budget_s / max(t_cal / 2, 1e-6)))
    steps = min(steps, 400)
    o = oracle_for(p, lib)
    t = o.run_fixed_slabs(0, cores, time_only_steps=steps)
    gcells = p.ncells * steps / t / 1e9
    return {"value": gcells, "unit": UNIT, "cores": cores, "kind": kind,
            "sample": f"{steps} time steps of {p.name} (fp64, reference arithmetic), "
                      f"{cores} z-slab threads, {t:.1f} s"}


def run_reference(args):
    world, rank, local = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return
    p = make_problem(args.workload, 0, fixed_steps=args.fixed_steps)
    for _ in range(args.warmup):
        cpu_baseline(p, budget_s=2.0)
    vals = [cpu_baseline(p, budget_s=12.0) for _ in range(args.steps)]
    v = statistics.median([x["value"] for x in vals])
    base = dict(vals[0])
    base["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": p.name, "cells": p.ncells, "precision": "fp64 (reference)",
                       "sample": base["sample"]},
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    world, rank, local = dist_setup(args.gpus)
    from emopt_b200 import problems as P
    p = make_problem(args.workload, seed=rank, fixed_steps=args.fixed_steps)
    sim = P.make_solver(p, precision=args.precision, kernel=args.kernel, device=local)
    t0 = [sim._Ex_fwd_t0, sim._Ey_fwd_t0, sim._Ez_fwd_t0, sim._Hx_fwd_t0, sim._Hy_fwd_t0,
          sim._Hz_fwd_t0]
    t1 = [sim._Ex_fwd_t1, sim._Ey_fwd_t1, sim._Ez_fwd_t1, sim._Hx_fwd_t1, sim._Hy_fwd_t1,
          sim._Hz_fwd_t1]
    for _ in range(max(args.warmup, 1)):
        sim._solve(t0, t1, sim._sources)
    barrier(world)
    # ---- device-timed region: K complete solves, inputs resident
    infos = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            infos.append(sim._solve(t0, t1, sim._sources))
    barrier(world)
    dev_s = sum(i["device_ms"] for i in infos) / 1e3
    steps_total = sum(i["steps"] for i in infos)
    launches = sum(i.get("launches", 0) for i in infos)
    cell_updates = float(p.ncells) * steps_total
    (dev_s_max,) = barrier_max([dev_s], world)
    (cell_updates_all,) = barrier_sum([cell_updates], world)
    value = cell_updates_all / dev_s_max / 1e9
    fields32 = np.stack([sim._raw(c, False).copy() for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")])

    # ---- e2e: public API with host buffers (materials re-uploaded each call);
    # one untimed call first pays the path's one-time costs (module imports,
    # first launches of the source-power kernel)
    sim._materials_dirty = True
    sim.solve_forward()
    barrier(world)
    wall = []
    for _ in range(args.steps):
        sim._materials_dirty = True
        t_a = time.perf_counter()
        sim.solve_forward()
        wall.append(time.perf_counter() - t_a)
    (wall_max,) = barrier_max([sum(wall)], world)
    e2e_steps = sim.last_solve["steps"] * args.steps
    (e2e_updates,) = barrier_sum([float(p.ncells) * e2e_steps], world)
    src_bytes = sum(6 * a[0].size * 16 for a, *_ in p.sources)
    h2d = 6 * p.ncells * 16 + src_bytes
    d2h = 6 * p.ncells * 16

    # ---- roofline of the step kernel
    word = 4 if args.precision == "fp32" else 8
    alg = algorithmic_bytes_per_step(p.shape, p.w_pml, word)
    step_s = dev_s / steps_total
    peak, peak_kind = measured_peak()
    achieved = alg / step_s / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", f"traffic_{args.kernel}_{args.precision}_{p.name}.json")
    if os.path.exists(prof):
        with open(prof) as f:
            traffic = json.load(f).get("dram_bytes_per_launch")

    result = None
    if rank == 0:
        line = {
            "metric": METRIC if (args.workload == "mmi" and args.precision == "fp32") else
            f"Gcell-updates/s ({args.workload}, {args.precision})",
            "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * dev_s_max / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "fp32" else "f64", "data": "synthetic",
            "config": {"workload": p.name, "cells": p.ncells, "time_steps_per_solve":
                       infos[-1]["steps"], "rtol": p.rtol, "kernel": args.kernel,
                       "precision": args.precision, "parallelism": f"replicas{world}",
                       "l2": "working set %.0f MB > 126 MB L2; no flush needed" %
                             ((2 * 6 + 3) * word * p.ncells / 1e6)},
            "e2e": {"value": round(e2e_updates / wall_max / 1e9, 3), "unit": UNIT,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                         "peak_source": peak_kind,
                         "alg_bytes_per_step": alg, "step_us": round(step_s * 1e6, 2)},
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        result = line
    # ---- fp64 comparison solve (not in the timed region)
    if rank == 0 and not args.no_fp64 and args.precision == "fp32":
        sim64 = P.make_solver(p, precision="fp64", kernel=args.kernel, device=local)
        info64 = sim64._solve([sim64._Ex_fwd_t0, sim64._Ey_fwd_t0, sim64._Ez_fwd_t0,
                               sim64._Hx_fwd_t0, sim64._Hy_fwd_t0, sim64._Hz_fwd_t0],
                              [sim64._Ex_fwd_t1, sim64._Ey_fwd_t1, sim64._Ez_fwd_t1,
                               sim64._Hx_fwd_t1, sim64._Hy_fwd_t1, sim64._Hz_fwd_t1],
                              sim64._sources)
        f64 = np.stack([sim64._raw(c, False) for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")])
        err = float(np.linalg.norm(fields32 - f64) / np.linalg.norm(f64))
        # the fp64 solve end to end through the public API (host buffers)
        sim64._materials_dirty = True
        t_a = time.perf_counter()
        sim64.solve_forward()
        e2e64 = p.ncells * sim64.last_solve["steps"] / (time.perf_counter() - t_a) / 1e9
        alg64 = algorithmic_bytes_per_step(p.shape, p.w_pml, 8)
        step64 = info64["device_ms"] / 1e3 / info64["steps"]
        result["fp64"] = {"value": round(p.ncells * info64["steps"] / (info64["device_ms"] / 1e3) / 1e9, 3),
                          "steps": info64["steps"], "fp32_steps": infos[-1]["steps"],
                          "fp32_rel_l2_vs_fp64": err,
                          "e2e": {"value": round(e2e64, 3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                                  "d2h_bytes_per_step": d2h},
                          "roofline_frac": round(alg64 / step64 / 1e9 / peak, 4),
                          "speedup_fp32_over_fp64": round(value / (p.ncells * info64["steps"] /
                                                                   (info64["device_ms"] / 1e3) / 1e9), 3)}
        del sim64
    # ---- the other forms of the path, on the same GPU, after the timed region
    if rank == 0 and world == 1 and args.workload == "mmi" and args.precision == "fp32":
        del sim
        import torch
        torch.cuda.empty_cache()
        if not args.no_serving:
            r = serving_result(local, 512, 20.0, 150.0, 4, first=128)
            result["serving"] = {"workload": "first 128 requests (by arrival) of the 512-request "
                                             "Poisson stream at 20/s, seed 3, fp32, rtol 1e-6",
                                 **{k: v for k, v in r.items() if k != "clocks"},
                                 "clocks": r["clocks"]}
            torch.cuda.empty_cache()
        if not args.no_grating:
            result["grating"] = {"workload": "grating slab 1201x601x301 (217 M cells), rtol 1e-6",
                                 **grating_result(local)}
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            result["cpu_baseline"] = cpu_baseline(p)
        except Exception as e:  # the baseline is reported, never required
            result["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "port",
                                      "sample": f"unavailable: {e}"}
    if rank == 0:
        print(json.dumps(result), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def serving_result(local: int, requests: int, rate: float, budget_gb: float, warmup: int,
                   first: int = 0, request_shape: str = "", fixed_steps: int = 0, world: int = 1,
                   rank: int = 0):
    """Serve a Poisson stream of CW solves (config: 512 requests at 20/s,
    seed 3) through the continuous-batching engine; ``first`` > 0 serves only
    the first that many requests (by arrival) of the stream.  Returns the
    result dict (aggregate Gcell-updates/s, latency and service-time
    percentiles, roofline fraction of the aggregate)."""
    from emopt_b200 import serving as S
    kw = {}
    if request_shape:
        kw = dict(shape=tuple(int(v) for v in request_shape.split(",")), d=0.025,
                  wavelength=1.55, w_pml=20)
    specs = S.poisson_stream(requests, rate, seed=3 + rank, **kw)
    if first:
        specs = sorted(specs, key=lambda sp: sp.arrival)[:first]
    for sp in specs:
        sp.fixed_steps = fixed_steps
    # warm-up: small requests through a throw-away engine (graph, kernels, allocator)
    if warmup > 0:
        warm = S.ServeEngine(local, 8e9, 8, 32)
        S.run_stream(S.poisson_stream(min(warmup, 4), 1e9, seed=99, shape=(40, 40, 48), w_pml=8),
                     warm, realtime=False)
        warm.close()
    eng = S.ServeEngine(local, budget_gb * 1e9, 128, 32)
    barrier(world)
    with ClockSampler(local) as clk:
        out = S.run_stream(specs, eng, realtime=True)
    barrier(world)
    eng.close()
    (makespan,) = barrier_max([out["makespan"]], world)
    (cu,) = barrier_sum([out["cell_updates"]], world)
    value = cu / makespan / 1e9
    steps = [r["steps"] for r in out["results"].values()]
    # algorithmic bytes of every request's time steps (fp32), over the makespan
    alg = sum(algorithmic_bytes_per_step(sp.shape, [sp.w_pml] * 6, 4) * out["results"][sp.rid]["steps"]
              for sp in specs)
    peak, peak_kind = measured_peak()
    return {
        "value": value, "unit": UNIT, "requests": len(specs), "makespan_s": makespan,
        "latency_s": {"p50": out["p50"], "p99": out["p99"], "max": float(out["latency"].max()),
                      "mean": float(out["latency"].mean())},
        "service_s": {"p50": out["service_p50"], "p99": out["service_p99"],
                      "max": float(out["service"].max())},
        "roofline": {"bound": "hbm", "achieved": alg / makespan / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / makespan / 1e9 / peak, "peak_source": peak_kind,
                     "note": "aggregate over the makespan (arrival gaps and set-up included)"},
        "time_steps": {"total": int(sum(steps)), "median": float(np.median(steps)),
                       "max": int(max(steps))},
        "nmax_hits": int(sum(1 for r in out["results"].values() if r["status"] != 0)),
        "clocks": clk.summary(),
    }


def run_serving(args):
    """Serving form: a Poisson stream of CW solves of mixed grids and
    wavelengths through the continuous-batching engine (FDTD_serve_*)."""
    world, rank, local = dist_setup(args.gpus)
    r = serving_result(local, args.requests, args.rate, args.budget_gb, args.warmup,
                       request_shape=args.request_shape, fixed_steps=args.fixed_steps, world=world,
                       rank=rank)
    result = {
        "metric": "serving: aggregate Gcell-updates/s with p50/p99 latency (CW-FDTD requests, "
                  "Poisson arrivals, mixed grids 64^3..384x256x128, fp32, rtol=1e-6)",
        "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": r["requests"],
        "warmup": min(args.warmup, 4), "ms_per_step": 1e3 * r["makespan_s"] / max(r["requests"], 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "serving_stream", "requests": args.requests, "rate_per_s": args.rate,
                   "budget_gb": args.budget_gb, "steps_per_replay": 32, "seed": 3,
                   "parallelism": f"replicas{world}"},
    }
    result.update({k: v for k, v in r.items() if k not in ("value", "unit")})
    if rank == 0:
        print(json.dumps(result), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_grad(args):
    """Differentiation form on the full MMI design problem (80 x 80 density):
    forward + adjoint solve + fused gradient kernel, fp32 and fp64."""
    world, rank, local = dist_setup(args.gpus)
    import torch
    from emopt_b200 import adjoint as A
    from emopt_b200 import problems as P
    p = P.mmi_gradient(seed=1, nd=(80, 80))
    res = {}
    for prec in ("fp32", "fp64"):
        obj, params = A.mmi_objective(p, prec, device=local)
        times = []
        for k in range(args.warmup + args.steps):
            x = params.clone().requires_grad_(True)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            F = obj(x)
            F.backward()
            torch.cuda.synchronize()
            if k >= args.warmup:
                times.append(time.perf_counter() - t0)
        res[prec] = {"F": F.item(), "grad": x.grad.detach().cpu().numpy(), "s": statistics.median(times),
                     "fwd_steps": obj.solver.last["forward"]["steps"],
                     "adj_steps": obj.solver.last["adjoint"]["steps"],
                     "fwd_ms": obj.solver.last["forward"]["device_ms"],
                     "adj_ms": obj.solver.last["adjoint"]["device_ms"]}
    g32, g64 = res["fp32"]["grad"], res["fp64"]["grad"]
    cells = p.ncells * (res["fp32"]["fwd_steps"] + res["fp32"]["adj_steps"])
    result = {
        "metric": "gradient evaluations/s (forward + adjoint CW solve + overlap, MMI 321x161x101, "
                  "80x80 density, fp32)",
        "value": 1.0 / res["fp32"]["s"], "unit": "gradients/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * res["fp32"]["s"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "mmi_grad_321x161x101", "density": [80, 80], "rtol": 1e-6},
        "gcell_updates_per_s": cells / res["fp32"]["s"] / 1e9,
        "fp32": {k: v for k, v in res["fp32"].items() if k != "grad"},
        "fp64": {k: v for k, v in res["fp64"].items() if k != "grad"},
        "fp32_vs_fp64": {"objective_rel": abs(res["fp32"]["F"] - res["fp64"]["F"]) / abs(res["fp64"]["F"]),
                         "gradient_rel_l2": float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64))},
    }
    if rank == 0:
        print(json.dumps(result), flush=True)


def grating_result(local: int, fixed_steps: int = 0):
    """Large single solve: the 1201 x 601 x 301 grating slab (217 M cells),
    float32 and float64 on one GPU, through FDTD_solve_cw with device-built
    materials and device phasors; both rates, their roofline fractions and
    the fp32 field error against the fp64 solve."""
    import ctypes
    import torch
    from emopt_b200 import fdtd_ctypes as ct
    from emopt_b200 import serving as S
    spec0 = S.grating_spec()
    dev = torch.device("cuda", local)
    mu_ones = torch.ones(spec0.ncells, dtype=torch.complex128, device=dev)
    out, fields = {}, {}
    peak, src = measured_peak()
    for prec in (32, 64):
        spec = S.grating_spec(precision=prec)
        spec.fixed_steps = fixed_steps
        req = S.Request(spec, local, mu_ones)
        req.set_outputs()
        res = ct.SolveResult()
        st = ct.libFDTD.FDTD_solve_cw(req.h, ctypes.byref(req.opt), ctypes.byref(res))
        if st not in (ct.FDTD_OK, ct.FDTD_NMAX):
            raise RuntimeError(ct.last_error(req.h))
        req.release_inputs()
        w = spec.w_pml
        alg = algorithmic_bytes_per_step(spec.shape, [w] * 6, prec // 8)
        step_us = 1e3 * res.device_ms / res.steps
        out[prec] = {"gcell_updates_per_s": spec.ncells * res.steps / res.device_ms / 1e6,
                     "steps": res.steps, "n_main": res.n_main, "status": st,
                     "device_s": res.device_ms / 1e3, "total_s": res.total_ms / 1e3,
                     "step_us": step_us, "roofline_frac": alg / (step_us * 1e-6) / 1e9 / peak}
        fields[prec] = req.out
        req.out = None
        req.close()
        torch.cuda.empty_cache()
    num = sum(float(torch.sum(torch.abs(a - b) ** 2)) for a, b in zip(fields[32], fields[64]))
    den = sum(float(torch.sum(torch.abs(b) ** 2)) for b in fields[64])
    del fields, mu_ones
    torch.cuda.empty_cache()
    return {"value": out[32]["gcell_updates_per_s"], "unit": UNIT, "cells": spec0.ncells,
            "fp32": out[32], "fp64": out[64], "fp32_rel_l2_vs_fp64": (num / den) ** 0.5,
            "speedup_fp32_over_fp64": out[32]["gcell_updates_per_s"] / out[64]["gcell_updates_per_s"],
            "peak_gbs": peak, "peak_source": src}


def run_grating(args):
    world, rank, local = dist_setup(args.gpus)
    r = grating_result(local, args.fixed_steps)
    result = {
        "metric": "Gcell-updates/s (CW-FDTD, fp32 storage, grating slab 1201x601x301, rtol=1e-6)",
        "value": r["value"], "unit": UNIT, "n_gpus": 1, "steps": 1, "warmup": 0,
        "ms_per_step": 1e3 * r["fp32"]["device_s"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "grating_1201x601x301", "cells": r["cells"], "rtol": 1e-6,
                   "fixed_steps": args.fixed_steps},
    }
    result.update({k: v for k, v in r.items() if k not in ("value", "unit", "cells")})
    if rank == 0:
        print(json.dumps(result), flush=True)


def run_zslab(args):
    """One MMI-block solve split into z slabs (emopt_b200/zslab.py): under
    torchrun one slab per rank with the halo planes sent over NCCL, otherwise
    --slabs slabs on this GPU linked by device copies.  Strong scaling: the
    grid is fixed, the ranks share it."""
    world, rank, local = dist_setup(args.gpus)
    import torch
    from emopt_b200 import problems as P
    from emopt_b200 import zslab
    p = P.mmi_block(fixed_steps=args.fixed_steps or None)
    nslab = world if world > 1 else max(1, args.slabs)
    ranges = zslab.ownership(p.shape[0], nslab)
    torch.cuda.set_device(local)
    ss = zslab.SlabSet(p, ranges, precision=args.precision, devices=[local],
                       rank=rank if world > 1 else None, overlap=args.overlap,
                       direct=False if args.copy_halo else None,
                       graphs=False if args.host_loop else None)
    times, res = [], None
    with ClockSampler(local) as clk:
        for it in range(args.warmup + args.steps):
            ss.begin()
            barrier(world)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            res = ss.run()
            e1.record()
            torch.cuda.synchronize()
            barrier(world)
            if it >= args.warmup:
                times.append(e0.elapsed_time(e1) / 1e3)
    ss.finish()
    ss.close()
    (t,) = barrier_max([statistics.median(times)], world)
    value = p.ncells * res.steps / t / 1e9
    result = {
        "metric": "Gcell-updates/s (CW-FDTD, %s storage, MMI block 321x161x101 split in z slabs, rtol=1e-6)"
                  % args.precision,
        "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32" if args.precision == "fp32" else "f64", "data": "synthetic",
        "config": {"workload": "mmi_321x161x101_zslab", "slabs": nslab, "ranges": ranges,
                   "time_steps_per_solve": res.steps, "n_main": res.n_main,
                   "transport": "nccl" if world > 1 else
                   ("neighbour planes read in place (one GPU)" if ss.direct else "device copies (one GPU)"),
                   "schedule": "overlapped" if world > 1 or args.overlap else "plain",
                   "step_graph": ss.graphs},
        "step_us": 1e6 * t / res.steps,
        "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(result), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_modes(args):
    """Mode-source generation: ModeFullVector.build + solve (4 modes nearest
    n0 = 3.45) + get_source on the cross-section of the MMI block's input
    waveguide (0.5 x 0.22 um silicon strip in oxide, 161 x 101 plane at
    0.025 um: 97,566 unknowns), as the reference's mode-source set-up does it.
    The oracle (the reference's matrices, SuperLU + ARPACK shift-and-invert)
    is timed beside it on the host."""
    import torch
    from emopt_b200 import grid
    from emopt_b200.misc import DomainCoordinates
    from emopt_b200.modes import ModeFullVector
    d, wl = 0.025, 1.55
    Xs, Ys, Zs = 8.0, 4.0, 2.5
    core = grid.Rectangle(Xs / 2, Ys / 2, 2 * Xs, 0.5)
    core.layer, core.material_value = 1, 12.25
    clad = grid.Rectangle(Xs / 2, Ys / 2, 2 * Xs, 2 * Ys)
    clad.layer, clad.material_value = 2, 2.085
    eps = grid.StructuredMaterial3D(Xs, Ys, Zs, d, d, d)
    eps.add_primitive(clad, -Zs, Zs)
    eps.add_primitive(core, Zs / 2 - 0.11, Zs / 2 + 0.11)
    mu = grid.ConstantMaterial3D(1.0)
    plane = DomainCoordinates.from_indices(100, 101, 0, 161, 0, 101, d, d, d)
    times, applies = [], []
    for k in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        m = ModeFullVector(wl, eps, mu, plane, n0=3.45, neigs=4, device=0)
        m.build()
        m.solve()
        src = m.get_source(0, d, d, d)
        torch.cuda.synchronize()
        if k >= args.warmup:
            times.append(time.perf_counter() - t0)
    # one operator application (B v, forward + backward sweep: the captured
    # graph), device-timed
    m._vin.copy_(torch.randn(m._NL * m._nb, dtype=torch.complex128, device="cuda"))
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(3):
        m._graph.replay()
    reps = 20
    e0.record(st)
    for _ in range(reps):
        m._graph.replay()
    e1.record(st)
    torch.cuda.synchronize()
    apply_ms = e0.elapsed_time(e1) / reps
    nb, NL, nq = m._nb, m._NL, int(m._QpQn32.numel())
    # every inverted block read once by the back-substitution, its coupling
    # rows once more by the reduction (all lines but the top one)
    w_bytes = ((NL - 1) * nq + NL * nb) * nb * 16
    peak = None
    try:
        peak = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                           "MEASURED_PEAKS.json")))["hbm_gbs"]
        peak_kind = "measured"
    except Exception:
        peak, peak_kind = 6650.0, "fallback"
    achieved = w_bytes / (apply_ms * 1e-3) / 1e9
    med = statistics.median(times)
    # the timed step is the public API end to end (material objects in, the
    # six source planes out as host arrays; the Krylov start vector goes up)
    # this library's kernels per mode source: 9 material-plane samplings, the
    # assembly, one application outside the graph (before capture), every
    # replayed application, the source kernel
    per_apply = 2 + sum(1 + (lev["e1_32"].numel() > 0) + (lev["e2_32"].numel() > 0) + 2
                        + (lev["odd_n32"].numel() > 0) for lev in m._levels)
    launches = 9 + 1 + per_apply * (1 + m.stats["applications"]) + 1
    result = {
        "metric": "mode solves/s (full-vector, 161x101 plane, 4 modes near n0=3.45, with get_source)",
        "value": 1.0 / med, "unit": "solves/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * med, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c128", "data": "synthetic",
        "config": {"workload": "mode_161x101_strip", "unknowns": 6 * 161 * 101, "lines": NL, "block": nb},
        "e2e": {"value": 1.0 / med, "unit": "solves/s", "h2d_bytes_per_step": m._NL * m._nb * 16,
                "d2h_bytes_per_step": 6 * 161 * 101 * 16},
        "gpu_launches": launches,
        "neff": [complex(x).real for x in m.neff], "stats": m.stats,
        "roofline": {"kernel": "k_lines_gemv (one apply: %d reduction levels)" % m.stats_levels, "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "apply_ms": apply_ms, "bytes_per_apply": w_bytes},
    }
    if not args.no_cpu:
        sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
        from oracle import modes as O
        ef = lambda k, j, i: np.where((np.abs(j * d - Ys / 2) < 0.25) & (np.abs(i * d - Zs / 2) < 0.11),
                                      12.25, 2.085) + 0j
        mf = lambda k, j, i: np.ones(np.shape(k)) + 0j
        t0 = time.perf_counter()
        planes = O.material_planes(ef, mf, "x", 101, 161, 100, 0, 0)
        A, B = O.build_system(planes, 101, 161, d, d, wl)
        neff, V = O.solve(A, B, 3.45, 4)
        tc = time.perf_counter() - t0
        result["cpu_baseline"] = {"value": 1.0 / tc, "unit": "solves/s", "cores": 1, "kind": "port",
                                  "sample": "one solve of the same plane (SuperLU + ARPACK, 4 modes)",
                                  "neff": [complex(x).real for x in neff]}
    print(json.dumps(result), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "serving":
        run_serving(args)
    elif args.workload == "grad":
        run_grad(args)
    elif args.workload == "grating":
        run_grating(args)
    elif args.workload == "zslab":
        run_zslab(args)
    elif args.workload == "modes":
        run_modes(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
