"""Benchmark: pressure solves/s at 256^3, variable coefficient (density ratio 1000),
to relative residual 1e-10 -- the B200 bbmg solver.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one pressure solve of the fixed operator: right-hand side and zero
initial guess in, solution out, iterated to max|r|/max|r0| <= 1e-10 (the
reference's criterion, bbmg_class.f90:627,694-699).  Operator setup (Galerkin
hierarchy) is timed separately.  Workload: 256^3 cells on the unit cube,
periodic in x and z, walls (Neumann) in y, 48 seeded spherical drops of radius
6-20 cells with density 1000 inside and 1 outside, tanh-smeared over 1.5 cells;
RHS = -vol div(u) of a seeded curl field plus N(0, 0.01) noise.  Synthetic, seeded.

`value` is the mixed-precision solver (FP32 V-cycle preconditioning FP64 CG),
device-resident inputs; `e2e` is the same through the C ABI with pinned host
arrays (host->device copy of rhs and initial guess, device->host copy of the
solution inside every step).  The FP64 GPU solver (the reference's arithmetic)
is reported beside it.  With N GPUs every rank solves its own replica (no
exchange: a pressure solve does not shard across GPUs here) and `value` is the
aggregate.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solves/s at 256³ var-coeff to 1e-10 rel. residual: FP64 MG vs mixed+learned"
WORKLOAD = ("256^3 variable-coefficient pressure Poisson: rho=1000 in 48 seeded drops (radii 6-20 cells), "
            "rho=1 outside, tanh width 1.5 cells; periodic x/z, Neumann walls y; RHS=-vol*div(curl field + "
            "N(0,0.01) noise)")
NCU_CAP = 3


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-n", type=int, default=128, help="grid of the bounded CPU sample")
    ap.add_argument("--profile", action="store_true", help="short run for ncu (no CPU leg, 1 step)")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_rank{index}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            self.f.close()

    def summary(self):
        if self.p is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------- reference arm
def _cpu_worker(args):
    """Solve the bounded CPU sample with the oracle's release build (the reference's
    algorithm with its GNU release flags, 1 rank on 1 core)."""
    n, seed, nsolve, q = args
    from nga2_b200 import problems as P
    from oracle.oracle import PCG_BBOX, OracleBBMG
    # the same physical drops as the 256^3 workload (radii scale with the grid)
    pb = P.drops_poisson(n, seed=seed, rmin=6.0 * n / 256, rmax=20.0 * n / 256)
    o = OracleBBMG(n, n, n, True, False, True, method=PCG_BBOX, rcvg=1e-10, release=True)
    t0 = time.perf_counter()
    o.setup(pb.stc, pb.opr)
    t_setup = time.perf_counter() - t0
    times, its = [], []
    for _ in range(nsolve):
        t0 = time.perf_counter()
        _, it, rerr = o.solve(pb.rhs)
        times.append(time.perf_counter() - t0)
        its.append(it)
    return {"setup_s": t_setup, "solve_s": times, "it": its}


def cpu_sample(n, seed, nsolve, procs):
    """Run `procs` independent single-core oracle instances (spawned processes)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        return pool.map(_cpu_worker, [(n, seed, nsolve, i) for i in range(procs)])


def run_reference(a):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    import psutil
    cores = os.cpu_count() or 1
    mem = psutil.virtual_memory().available
    n = a.cpu_n
    per_inst = 100.0 * (n + 2) ** 3 * 8  # ~ reference-layout doubles per cell
    procs = max(1, min(cores, int(mem * 0.6 // per_inst)))
    nsolve = max(1, min(a.steps, 3))
    res = cpu_sample(n, a.seed, nsolve, procs)
    per = [np.mean(r["solve_s"]) for r in res]
    scale = (a.n / n) ** 3
    sps = sum(1.0 / (t * scale) for t in per)
    line = {
        "impl": "reference", "metric": METRIC, "value": sps, "unit": "solves/s", "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 / sps * procs if sps else None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "method": "pcg_bbox V(2,2), direct coarsest", "inputs": "host"},
        "cpu_baseline": {"value": sps, "unit": "solves/s", "cores": procs, "kind": "port",
                         "sample": f"{nsolve} full pcg_bbox solve(s) of the same generator at {n}^3 per "
                                   f"process, {procs} independent 1-core processes (the reference is MPI-only, "
                                   f"1 rank per core); 256^3 time = {n}^3 time x (256/{n})^3; oracle release "
                                   f"build (-O3 -fno-tree-vectorize -ffast-math -funroll-loops)",
                         "iterations": [r["it"] for r in res], "setup_s": float(np.mean([r["setup_s"] for r in res]))},
        "e2e": {"value": sps, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ----------------------------------------------------------------------------- our arm
def true_rerr(pb, x):
    """FP64 max|b - A x| / max|b| with numpy (independent of the solver)."""
    o = pb.opr
    Ax = o[..., 0] * x
    Ax += o[..., 1] * np.roll(x, -1, 2) + o[..., 2] * np.roll(x, 1, 2)
    Ax += o[..., 3] * np.roll(x, -1, 1) + o[..., 4] * np.roll(x, 1, 1)
    Ax += o[..., 5] * np.roll(x, -1, 0) + o[..., 6] * np.roll(x, 1, 0)
    return float(np.abs(pb.rhs - Ax).max() / np.abs(pb.rhs).max())


def time_solves(torch, g, rhs, sol, steps, warmup, stream, reset):
    """W warm-up solves, then K solves between CUDA events on the solver's stream."""
    for _ in range(warmup):
        reset()
        g.solve(rhs, sol)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    its, launches = [], 0
    e0.record(stream)
    for _ in range(steps):
        reset()
        _, it, rerr, st = g.solve(rhs, sol)
        its.append(it)
        launches += g.info["launches"]
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), its, rerr, launches


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
        return
    ws, rank, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from nga2_b200 import problems as P
    from nga2_b200.bbmg import BBMG, FP64, MIXED, PCG_BBOX

    n = a.n
    t0 = time.perf_counter()
    pb = P.drops_poisson(n, seed=a.seed, rmin=6.0 * n / 256, rmax=20.0 * n / 256)
    t_gen = time.perf_counter() - t0
    per = (pb.xper, pb.yper, pb.zper)
    stream = torch.cuda.Stream()

    def make(precision):
        g = BBMG(n, n, n, *per, method=PCG_BBOX, precision=precision, rcvg=1e-10, maxit=100, device=local)
        g.set_stream(stream.cuda_stream)
        g.setup(pb.stc, pb.opr)
        return g

    gm = make(MIXED)
    g64 = None if a.profile else make(FP64)
    setup_ms = {"mixed": gm.info["setup_ms"], "fp64": g64.info["setup_ms"] if g64 else None}

    # device-resident inputs (value) -------------------------------------------------
    with torch.cuda.stream(stream):
        drhs = torch.from_numpy(pb.rhs).to(f"cuda:{local}")
        dsol = torch.zeros_like(drhs)
    torch.cuda.synchronize()

    def reset_dev():
        with torch.cuda.stream(stream):
            dsol.zero_()

    barrier = (lambda: __import__("torch.distributed").distributed.barrier()) if ws > 1 else (lambda: None)
    steps, warmup = (1, 1) if a.profile else (a.steps, max(a.warmup, 3))

    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ms_mixed, its_mixed, rerr_mixed, launches_mixed = time_solves(torch, gm, drhs, dsol, steps, warmup, stream,
                                                                       reset_dev)
    torch.cuda.synchronize()
    barrier()
    if a.profile:
        print(json.dumps({"profile_run": True, "n": n, "ms": ms_mixed, "it": its_mixed, "rerr": rerr_mixed}))
        return
    x_mixed = dsol.cpu().numpy()
    ms_fp64, its_fp64, rerr_fp64, _ = time_solves(torch, g64, drhs, dsol, steps, 1 if a.profile else 3, stream,
                                                  reset_dev)
    x_fp64 = dsol.cpu().numpy()
    if ws > 1:
        import torch.distributed as dist
        t = torch.tensor([ms_mixed, ms_fp64], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_mixed, ms_fp64 = t.tolist()

    # end to end through the C ABI with pinned host arrays ----------------------------
    hrhs = torch.from_numpy(pb.rhs).pin_memory().numpy()
    hsol_t = torch.zeros(pb.rhs.shape, dtype=torch.float64).pin_memory()
    hsol = hsol_t.numpy()

    def reset_host():
        hsol[...] = 0.0

    ms_e2e, its_e2e, _, _ = time_solves(torch, gm, hrhs, hsol, steps, 1, stream, reset_host)
    if ws > 1:
        t = torch.tensor([ms_e2e], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = t.item()
    if rank != 0:
        if ws > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    sps = ws * steps / (ms_mixed / 1e3)
    sps64 = ws * steps / (ms_fp64 / 1e3)
    sps_e2e = ws * steps / (ms_e2e / 1e3)
    err_vs_fp64 = float(np.abs(P.remove_mean(x_mixed) - P.remove_mean(x_fp64)).max()
                        / np.abs(P.remove_mean(x_fp64)).max())
    tr_mixed = true_rerr(pb, x_mixed)
    tr_fp64 = true_rerr(pb, x_fp64)

    # roofline of the dominant kernel: one colour of the level-1 FP32 Gauss-Seidel
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    reps = 20
    ms_sweep = gm.profile("relax", 1, 1, prec=1, reps=reps)  # one forward sweep as the V-cycle runs it
    lvl1 = gm.info["level1_stencil"]
    ncell = n ** 3
    c1, sv = 4, 4  # symmetric 7-point: 4 coefficients per cell; FP32 vectors
    bytes_sweep = ncell * (c1 * 4 + 3 * sv)
    nlaunch = 4 if lvl1 in (4, 7) else 8  # colour phases by Hamming weight on 7-point levels
    t_launch = ms_sweep / nlaunch / 1e3
    achieved = bytes_sweep / (ms_sweep / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "relax_fp32_traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get("bytes_per_launch_256")
        except Exception:
            traffic = None
    roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
            "traffic": traffic,
            "kernel": f"k_relax_phase7<float,{lvl1}> (level-1 Gauss-Seidel, one sweep = {nlaunch} launches)",
            "bytes_per_launch": bytes_sweep / nlaunch, "ms_per_launch": t_launch * 1e3, "ms_per_sweep": ms_sweep,
            "peak_source": peak_src}
    # other kernels, for the record
    kern = {}
    for name, lvl, prec in (("relax", 1, 0), ("residual", 1, 1), ("residual", 1, 0), ("restrict", 1, 1),
                            ("prolong", 1, 1), ("relax", 2, 1), ("relax", 3, 1), ("relax", 4, 1)):
        try:
            kern[f"{name}_L{lvl}_{'fp32' if prec else 'fp64'}_ms"] = gm.profile(name, lvl, 1, prec, 10)
        except Exception as e:  # noqa: BLE001
            kern[f"{name}_L{lvl}"] = str(e)

    cpu = None
    if not a.no_cpu_baseline and not a.profile and ws == 1:
        try:
            t0 = time.perf_counter()
            r = cpu_sample(a.cpu_n, a.seed, 1, 1)[0]
            t_cpu = r["solve_s"][0] * (n / a.cpu_n) ** 3
            cpu = {"value": 1.0 / t_cpu, "unit": "solves/s", "cores": 1, "kind": "port",
                   "sample": f"one pcg_bbox solve of the same generator at {a.cpu_n}^3 ({r['it'][0]} it, "
                             f"{r['solve_s'][0]:.1f} s), scaled by (256/{a.cpu_n})^3; oracle release build, "
                             f"1 rank on 1 core", "setup_s_sample": r["setup_s"],
                   "wall_s": time.perf_counter() - t0}
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": "solves/s", "cores": 1, "kind": "port", "sample": f"failed: {e}"}

    h2d = 2 * pb.rhs.nbytes
    d2h = pb.rhs.nbytes
    line = {
        "metric": METRIC, "value": sps, "unit": "solves/s", "n_gpus": ws, "steps": steps, "warmup": warmup,
        "ms_per_step": ms_mixed / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 V-cycle / f64 outer", "data": "synthetic",
        "config": {"workload": WORKLOAD, "seed": a.seed, "n": n, "method": "pcg_bbox V(2,2), direct coarsest",
                   "precision": "FP32 V-cycle preconditioning FP64 CG", "parallelism": f"replicas x{ws}",
                   "l2": "inputs larger than L2 (operator 0.94 GB, vectors 134 MB each)",
                   "setup_ms": setup_ms, "generator_s": t_gen},
        "fp64": {"value": sps64, "unit": "solves/s", "ms_per_step": ms_fp64 / steps, "it": its_fp64,
                 "rerr": rerr_fp64, "true_rerr": tr_fp64},
        "mixed": {"it": its_mixed, "rerr": rerr_mixed, "true_rerr": tr_mixed, "err_vs_fp64": err_vs_fp64},
        "speedup_mixed_over_fp64": sps / sps64,
        "e2e": {"value": sps_e2e, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "it": its_e2e},
        "roofline": roof,
        "kernels": kern,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "gpu_launches": int(launches_mixed),
    }
    print(json.dumps(line))
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
