#!/usr/bin/env python
"""Throughput of the generalized-harmonic RK4 step on B200: point-updates per second.

One "step" is one classical RK4 step (four right-hand sides with Kreiss-Oliger dissipation,
the ghost fill before each, the stage arithmetic) over the whole mesh of the workload. A
point is an owned point counted N^3 per block, as the reference counts it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload kerr_schild_static|fourier]
    python bench.py --impl reference ...   # the CPU restatement of the reference's path

Workloads (seeded synthetic inputs, fully specified by their parameters):
  kerr_schild_static  static Kerr-Schild hole M=1, a=7/10 on [-8,8]^3, 64 blocks of 32^3
                      (h = 1/8), Dirichlet faces, :damped interior r_0=0.8 r_1=1.3 rho_max=4/M,
                      sampled gauge source, Gaussian damping, eps_KO = 1/2, q = 4, dt = h/(4 lambda)
  fourier             Minkowski + 8 Fourier modes (amplitude 1e-4) per component on the periodic
                      [-1,1]^3, 8 blocks of 32^3, q = 4, eps_KO = 1/2, gamma0 = 1, dt = h/4
"""
import argparse
import ctypes
import importlib.util
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
PKG = ROOT / "treegeneralizedharmonic.jl_b200"

# Algorithmic FP64 operations of one right-hand-side point at q = 4 (adds + multiplies +
# divides + square roots; an FMA is two), fixed by running the oracle's point right-hand side
# with an op-counting scalar (orc_count_flops): no gauge source / sampled gauge source.
FLOP_PER_POINT_RHS = {"none": 7909, "sampled": 7975}
# RK4 stage arithmetic per point-update: 20 variables x (4 + 4 + 4 + 2) flops
FLOP_PER_POINT_STAGES = 280


def load_package():
    spec = importlib.util.spec_from_file_location("tgh_b200", PKG / "__init__.py",
                                                  submodule_search_locations=[str(PKG)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["tgh_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def workload(tgh, name):
    if name == "kerr_schild_static":
        case = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=8.0, r0=0.8, r1=1.3, rho_max=4.0, variant="damped",
                                    gauge="sampled", eps_ko=0.5)
        forest = tgh.gh_forest(case, 32, 4)
        sample = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=4.0, r0=0.8, r1=1.3, rho_max=4.0,
                                      variant="damped", gauge="sampled", eps_ko=0.5)
        sample_forest = tgh.gh_forest(sample, 32, 2)
        cfg = {"workload": "kerr_schild_static", "M": 1.0, "a": 0.7, "domain": "[-8,8]^3", "blocks": 64,
               "block": "32^3", "h": 0.125, "q": 4, "boundary": "dirichlet", "interior": "damped r0=0.8 r1=1.3",
               "gauge_source": "sampled", "eps_ko": 0.5, "cfl": 0.25}
        return case, forest, sample, sample_forest, cfg, "sampled", False
    if name == "fourier":
        case = tgh.perturbed_minkowski_case()
        forest = tgh.gh_forest(case, 32, 2)
        cfg = {"workload": "fourier_minkowski", "domain": "[-1,1]^3 periodic", "blocks": 8, "block": "32^3",
               "h": 1 / 32, "q": 4, "modes": 8, "amplitude": 1e-4, "eps_ko": 0.5, "gamma0": 1.0, "cfl": 0.25}
        return case, forest, case, forest, cfg, "none", True
    raise SystemExit(f"unknown workload {name}")


def initial(tgh, P, forest, perturbed):
    import torch
    u = P.initial_state(P.statevector(), 0.0)
    if perturbed:
        u += torch.from_numpy(tgh.perturbation(forest, amplitude=1e-4)).cuda()
    return u


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9]
        mx = [float(r[2]) for r in rows if len(r) >= 9]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i - 5] for r in rows if len(r) >= 9 for i in range(5, 9) if r[i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sm)}


def cpu_baseline(tgh, sample_case, sample_forest, perturbed, steps=1):
    """The oracle's RK4 step (the C++ restatement of the reference's CPU path) on a bounded
    sample of the workload, with every host thread."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_binding  # noqa: E402  (test infrastructure, loaded for the baseline only)
    orc = oracle_binding.Oracle.load()
    orc.lib.orc_set_threads(os.cpu_count() or 1)
    O = orc.problem(sample_case, sample_forest, 4)
    u = O.initial_state(O.statevector(), 0.0)
    if perturbed:
        u = u + tgh.perturbation(sample_forest, amplitude=1e-4)
    st, lam = O.max_speed(u, 0.0)
    dt = 0.25 * sample_forest.h0 / lam
    O.rk4_step(u, 0.0, dt)  # warm
    t0 = time.perf_counter()
    for n in range(steps):
        O.rk4_step(u, (n + 1) * dt, dt)
    el = time.perf_counter() - t0
    pts = sample_forest.points() * steps
    return {"value": pts / el, "unit": "point-updates/s", "cores": int(orc.lib.orc_get_threads()), "kind": "port",
            "sample": f"{sample_forest.nblocks} blocks of {sample_forest.N}^3 of the same configuration, "
                      f"{steps} RK4 step(s), {el:.2f} s"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    tgh = load_package()
    case, forest, scase, sforest, cfg, gauge, perturbed = workload(tgh, args.workload)
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_binding  # noqa: E402
    orc = oracle_binding.Oracle.load()
    orc.lib.orc_set_threads(os.cpu_count() or 1)
    O = orc.problem(scase, sforest, 4)
    u = O.initial_state(O.statevector(), 0.0)
    if perturbed:
        u = u + tgh.perturbation(sforest, amplitude=1e-4)
    _, lam = O.max_speed(u, 0.0)
    dt = 0.25 * sforest.h0 / lam
    for n in range(args.warmup):
        O.rk4_step(u, n * dt, dt)
    t0 = time.perf_counter()
    for n in range(args.steps):
        O.rk4_step(u, (args.warmup + n) * dt, dt)
    el = time.perf_counter() - t0
    val = sforest.points() * args.steps / el
    cores = int(orc.lib.orc_get_threads())
    out = {"metric": "RK4 point-updates/s", "value": val, "unit": "point-updates/s", "impl": "reference",
           "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": cfg,
           "cpu_baseline": {"value": val, "unit": "point-updates/s", "cores": cores, "kind": "port",
                            "sample": f"each step: one RK4 step of {sforest.nblocks} blocks of {sforest.N}^3 of the "
                                      "same configuration (the reference is Julia and cannot run here; this is "
                                      "the C++ restatement of its CPU path)"},
           "e2e": {"value": val, "unit": "point-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="kerr_schild_static", choices=["kerr_schild_static", "fourier"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--rhs-only", action="store_true",
                    help="time only the right-hand side (head + Pi kernels, stage epilogue) on the workload: "
                         "the command the kernel profiles are taken with")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    tgh = load_package()
    case, forest, scase, sforest, cfg, gauge, perturbed = workload(tgh, args.workload)
    stream = torch.cuda.current_stream()
    P = tgh.GHProblem(case, forest, 4, margin_check=False)
    u0 = initial(tgh, P, forest, perturbed)
    if args.rhs_only:
        ms = P.time_rhs(u0, 0.0, mode=1, nlaunch=2)
        print(json.dumps({"workload": cfg["workload"], "rhs_ms_per_launch": ms,
                          "points_per_launch": (forest.N + 1) ** 3 * forest.nblocks}))
        P.close()
        return 0
    lam = P.max_speed(u0, 0.0)
    dt = 0.25 * forest.h0 / lam
    K, W = args.steps, max(3, args.warmup)

    # warm-up: W untimed K-step runs on copies (the first captures the graph)
    for _ in range(W):
        w = u0.clone()
        P.step_batched(w, 0.0, dt, K)
    torch.cuda.synchronize()

    u = u0.clone()
    clocks = Clocks(local)
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    P.step_batched(u, 0.0, dt, K)
    e1.record(stream)
    torch.cuda.synchronize()
    launches = P.last_launch_count()
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    ck = clocks.stop()
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    if not bool(torch.isfinite(u).all()):
        raise SystemExit("the evolved state is not finite")
    pts = forest.points()
    value = world * pts * K / (ms * 1e-3)

    # the dominant kernel alone: the right-hand side with the fused RK4 epilogue
    rhs_ms = P.time_rhs(u0, 0.0, mode=1, nlaunch=max(4, K))
    n1pts = (forest.N + 1) ** 3 * forest.nblocks
    flops = FLOP_PER_POINT_RHS[gauge] * n1pts
    achieved = flops / (rhs_ms * 1e-3) / 1e12
    peak = tgh.fp64_peak_tflops()
    traffic = None
    tf = ROOT / "profiles" / "traffic.txt"
    if tf.exists():
        for line in tf.read_text().splitlines():
            parts = line.split()
            if len(parts) >= 3 and parts[0] == cfg["workload"] and parts[1] == "rhs_stage":
                traffic = float(parts[2])

    # end to end through the public API with host buffers: per step the state is copied in
    # from pinned host memory and the result copied back
    uh = u0.cpu().pin_memory()
    res_h = torch.empty_like(uh).pin_memory()
    P.step_batched(u0.clone(), 0.0, dt, 1)  # graph for one step
    torch.cuda.synchronize()
    ud = torch.empty_like(u0)
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(K):
        ud.copy_(uh, non_blocking=True)
        P.step_batched(ud, 0.0, dt, 1)
        res_h.copy_(ud, non_blocking=True)
    e3.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e2.elapsed_time(e3)
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    nbytes = uh.numel() * 8

    out = {"metric": "RK4 point-updates/s", "value": value, "unit": "point-updates/s", "n_gpus": world,
           "steps": K, "warmup": W, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {**cfg, "form": "batched (fused RK4 epilogue, CUDA graph)", "points": pts,
                      "l2_flush": "inputs larger than L2 (working arrays %.0f MB)" % (P.work_length * 8 / 1e6),
                      "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
           "roofline": {"bound": "fp64", "kernel": "rhs_head_kernel + rhs_pi_kernel (one RHS, RK4 stage epilogue)",
                        "achieved": achieved, "peak": peak,
                        "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
                        "flop_per_point": FLOP_PER_POINT_RHS[gauge], "points_per_launch": n1pts,
                        "ms_per_launch": rhs_ms,
                        "peak_source": "measured FP64 FMA probe on this GPU (MEASURED_PEAKS.json has no FP64)"},
           "e2e": {"value": world * pts * K / (e2e_ms * 1e-3), "unit": "point-updates/s",
                   "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes},
           "gpu_launches": launches, "clocks": ck}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(tgh, scase, sforest, perturbed)
    if rank == 0:
        print(json.dumps(out))
    P.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
