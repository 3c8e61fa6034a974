"""Benchmark: sTDA solves/s on one B200 (N GPUs run independent replicas).

Workload (single large sTDA, mixed precision): a synthetic graphene flake
C384H48 with a minimal valence basis (1584 AOs, 780 occupied MOs, seeded
MOs/energies), ax = 0.5, E_thr = 7 eV, PT threshold 1e-4, lowest 50 roots.
One step = one full solve through the engine (orbital window -> S^1/2 ->
charges -> screen -> PT selection -> blocked Davidson -> properties with the
velocity correction).

* ``value``: solves/s with inputs already resident on the device, timed with
  CUDA events on the engine's stream (max over ranks).
* ``e2e``: the same through the C ABI with host buffers: every step copies the
  wavefunction and AO integrals host->device (std2g_load) and reads the
  results back.
* ``fp64_form``: the plain FP64 GPU form of the same solve (the denominator
  of the mixed-vs-FP64 comparison) and the mixed form's deviation from it.
* ``roofline``: the tensor-core contraction of the PT selection, algorithmic
  FLOPs (2 M N K with K = atoms) over its device time, against the measured
  bf16 peak.
* ``cpu_baseline``: the FP64 CPU restatement of the reference algorithm
  (numpy, all host threads) on a bounded sample of the same solve.

``--impl reference`` times that CPU restatement alone (the reference std2 is
Fortran and cannot be built on this image).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

KW = dict(ax=0.5, e_thr_ev=7.0, thrp=1e-4, nroots=50)
WORKLOAD = ("graphene flake C384H48, valence minimal basis (1584 AOs), ax=0.5, E_thr=7 eV, "
            "thrp=1e-4, lowest 50 roots")


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, dev):
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_{os.getpid()}.csv")
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={dev}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in open(self.path):
            t = [x.strip() for x in ln.split(",")]
            if len(t) < 9:
                continue
            try:
                sm.append(float(t[1]))
                mx = float(t[2])
            except ValueError:
                continue
            for nm, v in zip(names, t[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_workload(n=8):
    """Flake C_{6n^2}H_{6n}; n = 8 is the benchmark workload (C384H48)."""
    from stda_b200 import synth
    from stda_b200.engine import boundary_inputs
    mol, ints = synth.graphene_flake(n, with_ints=True)
    return mol, ints, boundary_inputs(mol, ints)


def cpu_sample(mol, ints, budget_s=15.0):
    """FP64 CPU restatement timed on a bounded sample of the same solve."""
    from oracle.stda_fp64 import Params, stda_timed
    S, L, V, M = ints
    p = Params(**{k: v for k, v in KW.items() if k != "nroots"})
    return stda_timed(mol.xyz4(), mol.C, mol.eps, mol.occ, mol.iaoat(), S, L, V, M, p,
                      budget_s=budget_s)


def run_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    mol, ints, _ = build_workload(args.flake)
    times, info = [], None
    for step in range(args.warmup + args.steps):
        info = cpu_sample(mol, ints, budget_s=args.cpu_budget)
        if step >= args.warmup:
            times.append(info["est_total_s"])
    per = statistics.median(times)
    v = 1.0 / per
    print(json.dumps({
        "impl": "reference", "metric": "sTDA solves/s", "value": v, "unit": "solves/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD},
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": info["threads"], "kind": "port",
                         "sample": info["sample"]},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64-form comparison")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--flake", type=int, default=8,
                    help="flake size n of C_{6n^2}H_{6n}; 8 = the benchmark workload, smaller "
                         "values are profiling cases")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        return run_reference(args)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist_
        torch.cuda.set_device(local)
        dist_.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = dist_

    from stda_b200.engine import Engine, Keywords
    mol, ints, b = build_workload(args.flake)
    prec = 1 if args.precision == "mixed" else 0
    kw = Keywords(**KW)
    eng = Engine(local, prec)
    eng.load(b)
    for _ in range(args.warmup):
        sol = eng.solve(kw)

    def barrier():
        if dist is not None:
            import torch
            t = torch.zeros(1, device=f"cuda:{local}")
            dist.all_reduce(t)
            torch.cuda.synchronize(local)

    # ---- device-resident throughput: CUDA-event time of each solve ----
    barrier()
    clk = Clocks(local)
    l0 = eng.kernel_launches()
    lat = []
    tc_ms, tc_launch, tc_flop = 0.0, 0, 0.0
    for _ in range(args.steps):
        sol = eng.solve(kw)
        lat.append(sol.ms)
        st = eng.kernel_stats()
        tc_ms += st["tc_ms"]
        tc_launch += st["tc_launches"]
        tc_flop += st["tc_flop"]
    launches = eng.kernel_launches() - l0
    clocks = clk.stop()
    barrier()
    total_ms = float(sum(lat))
    if dist is not None:
        import torch
        t = torch.tensor([total_ms], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * args.steps / (total_ms / 1e3)
    phases = eng.phase_times()
    solver = eng.solver_stats()

    # ---- end to end through the C ABI with host buffers ----
    h2d = sum(a.nbytes for a in (b.xyz4, b.C, b.eps, b.occ, b.iaoat1, b.S, b.muL, b.muV, b.muM))
    e2e_lat = []
    for _ in range(max(2, args.steps // 2)):
        t0 = time.perf_counter()
        eng.load(b)
        s2 = eng.solve(kw)
        e2e_lat.append(time.perf_counter() - t0)
    d2h = 8 * 5 * len(s2.omega) + 8 * 6
    e2e = {"value": world / statistics.median(e2e_lat), "unit": "solves/s",
           "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
           "note": "std2g_load (H2D of MOs + AO integrals) + std2g_solve + result D2H, wall clock"}

    out = {"metric": "sTDA solves/s", "value": value, "unit": "solves/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "bf16x3->f32 contractions, f64 screen/RR" if prec else "f64",
           "data": "synthetic",
           "config": {"workload": WORKLOAD if args.flake == 8 else f"flake n={args.flake} (profiling case)",
                      "nci": sol.nci, "nex": sol.nex, "nexpt": sol.nexpt,
                      "new_pt": sol.new, "no": sol.no, "nv": sol.nv, "nroots": len(sol.omega),
                      "parallelism": f"replicas x{world}",
                      "l2": "inputs > L2: per-solve charge/PT buffers are GBs"},
           "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
           "phases_ms": {k: round(v, 3) for k, v in phases.items()}, "solver": solver,
           "gpu_launches": int(launches), "clocks": clocks, "e2e": e2e}

    if tc_launch > 0:
        pk, src = peaks()
        ach = tc_flop / (tc_ms / 1e3) / 1e12
        out["roofline"] = {"bound": "tensor", "achieved": ach, "peak": pk["bf16_tflops"],
                           "unit": "TFLOP/s", "frac": ach / pk["bf16_tflops"], "traffic": None,
                           "kernel": "k_tc_gemm_bf16x3 (PT-selection contractions)",
                           "flop_count": "algorithmic 2*M*N*N_atoms; the bf16 hi/lo split "
                                         "executes 3x as many tensor-core FLOPs",
                           "peak_source": src, "avg_launch_ms": tc_ms / tc_launch}

    if rank == 0 and not args.no_fp64 and prec == 1:
        e64 = Engine(local, 0)
        e64.load(b)
        s64 = e64.solve(kw)
        l64 = [e64.solve(kw).ms for _ in range(2)]
        iconf_m, _ = eng.csf()
        iconf_d, _ = e64.csf()
        n = min(len(s64.omega), len(sol.omega))
        big = s64.fL[:n] > 1e-3
        out["fp64_form"] = {
            "solves_per_s": 1e3 / statistics.median(l64), "ms": statistics.median(l64),
            "speedup_mixed_vs_fp64": statistics.median(l64) / (total_ms / args.steps),
            "max_root_err_ev": float(np.abs(sol.omega[:n] - s64.omega[:n]).max() * 27.21139),
            "max_fL_rel_err_fL_gt_1e-3": float(np.max(np.abs(sol.fL[:n][big] - s64.fL[:n][big]) /
                                                      s64.fL[:n][big])) if big.any() else None,
            "max_fL_abs_err": float(np.abs(sol.fL[:n] - s64.fL[:n]).max()),
            "csf_identical": bool(np.array_equal(iconf_m, iconf_d)),
            "phases_ms": {k: round(v, 3) for k, v in e64.phase_times().items()}}
        e64.close()

    if rank == 0 and world == 1 and not args.no_cpu:
        info = cpu_sample(mol, ints, budget_s=args.cpu_budget)
        out["cpu_baseline"] = {"value": 1.0 / info["est_total_s"], "unit": "solves/s",
                               "cores": info["threads"], "kind": "port", "sample": info["sample"]}
    if rank == 0:
        print(json.dumps(out))
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
