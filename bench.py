#!/usr/bin/env python
"""Throughput of the generalized-harmonic RK4 step on B200: point-updates per second.

One "step" is one classical RK4 step (four right-hand sides with Kreiss-Oliger dissipation,
the ghost fill before each, the stage arithmetic) over the whole mesh of the workload. A
point is an owned point counted N^3 per block, as the reference counts it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload hierarchy|kerr_schild_static|fourier|g5]
    python bench.py --impl reference ...   # the CPU restatement of the reference's path

One GPU: the batched form (the whole K-step run one CUDA graph). N GPUs (torchrun, one rank
per GPU): the workload's mesh sharded over the ranks, per-level Morton partition, one NCCL
all-to-all of halo points before each fill phase; the mesh is the same for every N (strong
scaling). --shard runs that sharded path on one GPU. On one GPU the default (hierarchy) line
also carries `g5_chart`: the reference's G5 chart (the g5 workload) stepped the same way, with
its device time per M of evolution.

Workloads (seeded synthetic inputs, fully specified by their parameters):
  hierarchy           (the default) the hole of kerr_schild_static boosted to v = 0.1 along x,
                      on [-40,40]^3 refined around its path in 5 levels to 2472 blocks of 32^3
                      (finest h = 5/256), algebraic Kerr-Schild gauge source, moving :damped
                      core; ~117 GB on the device in the batched form. The plain forms are
                      timed after the batched problem is released, on a problem of their own
  kerr_schild_static  static Kerr-Schild hole M=1, a=7/10 on [-8,8]^3, 64 blocks of 32^3
                      (h = 1/8), Dirichlet faces, :damped interior r_0=0.8 r_1=1.3 rho_max=4/M,
                      sampled gauge source, Gaussian damping, eps_KO = 1/2, q = 4, dt = h/(4 lambda)
  fourier             Minkowski + 8 Fourier modes (amplitude 1e-4) per component on the periodic
                      [-1,1]^3, 8 blocks of 32^3, q = 4, eps_KO = 1/2, gamma0 = 1, dt = h/4
  hierarchy_small     the same hole on [-6,6]^3 refined in 2 levels (radii 3.0, 1.6) to 120
                      blocks of 32^3: one coarse-fine interface, a few GB, for ncu captures
  g5                  the reference's G5 chart: Kerr M=1, a=7/10 in harmonic coordinates (no gauge
                      source) on [-5/4,5/4]^3, one root of 8^3 refined with radii 10, 8/5, 13/10, 1
                      to 2472 blocks of 8^3 (1,265,664 points, h = 5/256), :fitted interior
                      r_0 = 0.8, r_1 = 1 relaxing toward the analytic cache; the CPU baseline runs
                      on this same mesh
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
# with an op-counting scalar (orc_count_flops) at the centre of the first block of each
# workload: no gauge source (fourier), sampled (kerr_schild_static), algebraic (hierarchy).
FLOP_PER_POINT_RHS = {"none": 7909, "sampled": 7957, "algebraic": 8283}
# RK4 stage arithmetic per point-update: 20 variables x (4 + 4 + 4 + 2) flops
FLOP_PER_POINT_STAGES = 280
# The constraint monitors' algorithmic FP64 operations per point at q = 4, counted the same way
# (orc_count_monitor_flops) at the same points: the gauge constraint and the ADM constraints
# (the Ricci tensor contracted in the kernel's order; the reference's assembly counts 2,557 more).
FLOP_PER_POINT_MONITORS = {"gauge": {"none": 2169, "sampled": 2159, "algebraic": 2490},
                           "adm": {"none": 13830, "sampled": 13890, "algebraic": 14226}}


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
    if name in ("hierarchy", "hierarchy_small"):
        small = name == "hierarchy_small"
        radii = [3.0, 1.6] if small else [30.0, 16.0, 8.0, 4.5, 2.6]
        case = tgh.kerr_schild_case(M=1.0, a=0.7, v=0.1, halfwidth=6.0 if small else 40.0, r0=0.8, r1=1.3,
                                    rho_max=4.0, variant="damped", gauge="algebraic", eps_ko=0.5)
        # the shells follow the centre over the 200-step run (t_end ~ 0.6, so 0.07 along x)
        forest = tgh.hole_forest(case, 32, 2 if small else 4, radii, path=((0.0, 0.0, 0.0), (0.07, 0.0, 0.0)))
        sample = tgh.kerr_schild_case(M=1.0, a=0.7, v=0.1, halfwidth=4.0, r0=0.8, r1=1.3, rho_max=4.0,
                                      variant="damped", gauge="algebraic", eps_ko=0.5)
        sample_forest = tgh.gh_forest(sample, 32, 2)
        counts = [int(c) for c in __import__("numpy").bincount(forest.level)]
        cfg = {"workload": "kerr_schild_hierarchy" + ("_small" if small else ""), "M": 1.0, "a": 0.7,
               "velocity": [0.1, 0.0, 0.0], "domain": "[-6,6]^3" if small else "[-40,40]^3",
               "blocks": forest.nblocks, "blocks_per_level": counts, "block": "32^3",
               "h_min": forest.h0 / 2 ** int(forest.level.max()), "refinement_radii": radii, "q": 4,
               "boundary": "dirichlet", "interior": "damped moving core r0=0.8 r1=1.3",
               "gauge_source": "algebraic", "eps_ko": 0.5, "cfl": 0.25}
        return case, forest, sample, sample_forest, cfg, "algebraic", False
    if name == "g5":
        case = tgh.harmonic_kerr_case(M=1.0, a=0.7, halfwidth=1.25, r0=0.8, r1=1.0, rho_max=4.0,
                                      variant="fitted", eps_ko=0.5)
        radii = [10.0, 1.6, 1.3, 1.0]
        forest = tgh.hole_forest(case, 8, 1, radii)
        counts = [int(c) for c in __import__("numpy").bincount(forest.level)]
        cfg = {"workload": "g5_harmonic_kerr", "M": 1.0, "a": 0.7, "chart": "harmonic", "domain": "[-1.25,1.25]^3",
               "blocks": forest.nblocks, "blocks_per_level": counts, "block": "8^3",
               "h_min": forest.h0 / 2 ** int(forest.level.max()), "refinement_radii": radii, "q": 4,
               "boundary": "dirichlet", "interior": "fitted r0=0.8 r1=1.0, analytic cache",
               "gauge_source": "none", "eps_ko": 0.5, "cfl": 0.25}
        return case, forest, case, forest, cfg, "none", False
    raise SystemExit(f"unknown workload {name}")


def ready(case, P, forest):
    """A :fitted problem relaxes toward its target cache: fill it from the analytic state (the
    stand-in for the fit) before the first step."""
    if case.interior and case.interior.get("variant") == "fitted":
        if not hasattr(P, "fill_target_analytic"):
            raise SystemExit("the sharded path takes no :fitted interior")
        P.fill_target_analytic(0.0, case.interior["r1"] + h_min(forest), 0.0)
    return P


def h_min(forest):
    """The finest spacing of a forest: the time step is set by it (one dt for every level)."""
    return forest.h0 / 2 ** int(forest.level.max())


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


def rhs_kernels(P, cfg):
    """The kernels one timed right-hand side launches, as the roofline's label."""
    v = P.variant() if hasattr(P, "variant") else {"pi": "l1"}
    pi = "rhs_pi_tma_kernel" if v.get("pi") == "tma" else "rhs_pi_kernel"
    names = ["rhs_head_kernel", pi]
    if "interior" in cfg and "none" not in str(cfg["interior"]):
        names.insert(0, "interior_kernel")
    return " + ".join(names) + " (one RHS, RK4 stage epilogue)"


def cpu_model():
    """The host CPU's model name (for the CPU baseline's record)."""
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def simd_oracle(case, forest):
    """The oracle build with the host's widest SIMD lanes (AVX-512: 8 doubles, else AVX2: 4), every
    host thread, and a problem on it whose right-hand side runs on those lanes, as the reference's
    CPU kernel does (src/lanes.jl)."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_binding  # noqa: E402  (test infrastructure, loaded for the baseline only)
    orc = oracle_binding.Oracle.load_widest()
    orc.lib.orc_set_threads(os.cpu_count() or 1)
    O = ready(case, orc.problem(case, forest, 4), forest)
    O.set_simd_width(orc.lanes())
    return orc, O


def simd_label(orc):
    n = orc.lanes()
    return f"{n} FP64 lanes along x ({'AVX-512' if n == 8 else 'AVX2'}), groups straddling the interior point by point"


def cpu_baseline(tgh, sample_case, sample_forest, perturbed, seconds=10.0, max_steps=40):
    """The oracle's RK4 step (the C++ restatement of the reference's CPU path) on a bounded
    sample of the workload, with every host thread: steps until about `seconds` of work."""
    orc, O = simd_oracle(sample_case, sample_forest)
    u = O.initial_state(O.statevector(), 0.0)
    if perturbed:
        u = u + tgh.perturbation(sample_forest, amplitude=1e-4)
    st, lam = O.max_speed(u, 0.0)
    dt = 0.25 * h_min(sample_forest) / lam
    O.rk4_step(u, 0.0, dt)  # warm
    t0 = time.perf_counter()
    steps = 0
    while steps < max_steps and (steps == 0 or time.perf_counter() - t0 < seconds):
        O.rk4_step(u, (steps + 1) * dt, dt)
        steps += 1
    el = time.perf_counter() - t0
    pts = sample_forest.points() * steps
    # the constraint monitors on the sample's state, once each (prepare included, as on the GPU)
    d = O.diag()
    t1 = time.perf_counter()
    O.gh_constraint(d, u, 0.0)
    t2 = time.perf_counter()
    O.adm_constraint(d, u, 0.0)
    t3 = time.perf_counter()
    npts = (sample_forest.N + 1) ** 3 * sample_forest.nblocks
    monitors = {"gh_constraint_ms": (t2 - t1) * 1e3, "adm_constraint_ms": (t3 - t2) * 1e3,
                "points": npts, "unit": "ms per call on the sample"}
    return {"value": pts / el, "unit": "point-updates/s", "cores": int(orc.lib.orc_get_threads()), "kind": "port",
            "cpu_model": cpu_model(), "simd": simd_label(orc),
            "sample": f"{sample_forest.nblocks} blocks of {sample_forest.N}^3 of the same configuration, "
                      f"{steps} RK4 step(s), {el:.2f} s",
            "monitors": monitors}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    tgh = load_package()
    case, forest, scase, sforest, cfg, gauge, perturbed = workload(tgh, args.workload)
    orc, O = simd_oracle(scase, sforest)
    u = O.initial_state(O.statevector(), 0.0)
    if perturbed:
        u = u + tgh.perturbation(sforest, amplitude=1e-4)
    _, lam = O.max_speed(u, 0.0)
    dt = 0.25 * h_min(sforest) / lam
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
                            "cpu_model": cpu_model(), "simd": simd_label(orc),
                            "sample": f"each step: one RK4 step of {sforest.nblocks} blocks of {sforest.N}^3 of the "
                                      "same configuration (the reference is Julia and cannot run here; this is "
                                      "the C++ restatement of its CPU path)"},
           "e2e": {"value": val, "unit": "point-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def run_sharded(args, tgh, world, rank, local, case, forest, cfg, gauge, perturbed):
    """--gpus N > 1: the workload's mesh sharded over the N ranks (per-level Morton partition),
    each fill phase preceded by one NCCL all-to-all of the halo points; the mesh is the same
    for every N (strong scaling). Device time, max over ranks."""
    import torch
    import torch.distributed as dist
    stream = torch.cuda.current_stream()
    owner = tgh.partition(forest, world)
    S = ready(case, tgh.ShardedGHProblem(case, forest, 4, rank, world, owner=owner, margin_check=False), forest)
    u0 = S.initial_state(S.statevector(), 0.0)
    if perturbed:
        u0 += S.local(torch.from_numpy(tgh.perturbation(forest, amplitude=1e-4)).cuda())

    def gmax(x):
        t = torch.tensor([float(x)], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    dt = 0.25 * h_min(forest) / gmax(S.max_speed(u0, 0.0))
    K, W = args.steps, max(3, args.warmup)
    u = u0.clone()
    for _ in range(-(-W // K)):
        u.copy_(u0)
        S.step(u, 0.0, dt, K)
    torch.cuda.synchronize()
    u.copy_(u0)
    clocks = Clocks(local)
    time.sleep(0.3)
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    S.step(u, 0.0, dt, K)
    e1.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    ms = gmax(e0.elapsed_time(e1))
    ck = clocks.stop()
    launches = S.last_launch_count()
    if gmax(0.0 if bool(torch.isfinite(u).all()) else 1.0) > 0.0:
        raise SystemExit("the evolved state is not finite")
    pts = forest.points()
    value = pts * K / (ms * 1e-3)
    rhs_ms = gmax(S.time_rhs(u, 0.0, nlaunch=max(2, K // 10)))
    n1pts = (forest.N + 1) ** 3 * forest.nblocks
    achieved = FLOP_PER_POINT_RHS[gauge] * n1pts / (rhs_ms * 1e-3) / 1e12
    peak = tgh.fp64_peak_tflops() * world
    # end to end: per step this rank's state in from pinned host memory and back
    uh = u0.cpu().pin_memory()
    res_h = torch.empty_like(uh).pin_memory()
    ud = torch.empty_like(u0)
    dist.barrier()
    torch.cuda.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(K):
        ud.copy_(uh, non_blocking=True)
        S.step(ud, 0.0, dt, 1)
        res_h.copy_(ud, non_blocking=True)
    e3.record(stream)
    torch.cuda.synchronize()
    e2e_ms = gmax(e2.elapsed_time(e3))
    nbytes = uh.numel() * 8
    out = {"metric": "RK4 point-updates/s", "value": value, "unit": "point-updates/s", "n_gpus": world,
           "steps": K, "warmup": W, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "strong",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {**cfg, "form": "batched, sharded (host-driven stages, no graph)", "points": pts,
                      "l2_flush": "inputs larger than L2 on every rank" if S.state_length * 8 > 126e6
                      else "per-rank working set below L2 size",
                      "parallelism": f"sharded x{world}: per-level Morton partition, NCCL all-to-all per fill phase",
                      "blocks_per_rank": int(len(S.leaves))},
           "roofline": {"bound": "fp64", "kernel": rhs_kernels(S, cfg),
                        "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                        "traffic": None, "flop_per_point": FLOP_PER_POINT_RHS[gauge], "points_per_launch": n1pts,
                        "ms_per_launch": rhs_ms,
                        "peak_source": f"measured FP64 FMA probe x {world} GPUs"},
           "e2e": {"value": pts * K / (e2e_ms * 1e-3), "unit": "point-updates/s",
                   "h2d_bytes_per_step": nbytes * world, "d2h_bytes_per_step": nbytes * world},
           "plain_form": {"skipped": "the plain form runs on one GPU"},
           "gpu_launches": launches, "clocks": ck}
    if rank == 0:
        print(json.dumps(out))
    S.close()
    dist.destroy_process_group()
    return 0


def time_monitors(P, u, stream, gauge, n1pts, peak, reps=5):
    """The gauge and ADM constraint monitors and the norms' fold on the workload's state: CUDA
    events around `reps` calls each. Each monitor call includes its prepare (the scatter and
    ghost fill at t, as the reference's gh_constraint! and adm_constraint! do); the kernels are
    also timed alone (CUDA events around back-to-back launches after one prepare), which is the
    time the rooflines use."""
    import torch
    out = {}
    for name, fn in (("prepare", lambda: P.prepare(u, 0.0)),
                     ("gh_constraint", lambda: P.gh_constraint(u, 0.0)),
                     ("adm_constraint", lambda: P.adm_constraint(u, 0.0))):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        out[name + "_ms"] = e0.elapsed_time(e1) / reps
    for name in ("gauge", "adm"):
        kms = P.time_monitor(u, 0.0, name, nlaunch=reps)
        flops = FLOP_PER_POINT_MONITORS[name][gauge]
        out[name + "_kernel_ms"] = kms
        out[name + "_flop_per_point"] = flops
        out[name + "_tflops"] = flops * n1pts / (kms * 1e-3) / 1e12
        out[name + "_frac"] = out[name + "_tflops"] / peak
    t0 = time.perf_counter()
    n = P.constraint_norms()
    out["norms_ms_host"] = (time.perf_counter() - t0) * 1e3
    # the refinement indicator (prepare, masked amplitudes, tau, tau_max) and the two firing sweeps,
    # each a host call that returns its numbers
    P.tau(u, 0.0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = P.tau(u, 0.0)
    t1 = time.perf_counter()
    P.firing([0.4, 0.1])
    t2 = time.perf_counter()
    out["indicator_ms_host"] = (t1 - t0) * 1e3
    out["firing_ms_host"] = (t2 - t1) * 1e3
    out["tau_max"] = r["tau_max"]
    out["gauge_l2"] = n["gauge_l2"]
    out["ham_l2"] = n["ham_l2"]
    out["mom_l2"] = n["mom_l2"]
    return out


def g5_chart(tgh, K, stream, with_cpu=True):
    """The reference's G5 chart beside the headline (harmonic Kerr a = 7/10 on its 2472-block mesh
    of 8^3, the `g5` workload): the batched step timed the same way, K steps after one warm-up
    run, and the device time per M of evolution at dt = h/(4 lambda)."""
    import torch
    case, forest, *_ = workload(tgh, "g5")
    P = ready(case, tgh.GHProblem(case, forest, 4, margin_check=False), forest)
    u0 = P.initial_state(P.statevector(), 0.0)
    dt = 0.25 * h_min(forest) / P.max_speed(u0, 0.0)
    u = u0.clone()
    P.step_batched(u, 0.0, dt, K)
    u.copy_(u0)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    P.step_batched(u, 0.0, dt, K)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / K
    finite = bool(torch.isfinite(u).all())
    P.close()
    out = {"workload": "g5_harmonic_kerr", "blocks": forest.nblocks, "points": forest.points(), "steps": K,
           "ms_per_step": ms, "value": forest.points() / (ms * 1e-3), "unit": "point-updates/s",
           "steps_per_M": 1.0 / dt, "device_seconds_per_M": ms * 1e-3 / dt, "finite": finite}
    if with_cpu:
        # the oracle on SIMD lanes on this same mesh: the CPU baseline with the same configuration
        cb = cpu_baseline(tgh, case, forest, False, seconds=8.0, max_steps=4)
        cb.pop("monitors", None)
        out["cpu_baseline_same_mesh"] = cb
    return {**out,
            "reference": "630 s of a 64-core node per M for the reference's G5 runs, horizon finder and fits "
                         "included (SINGULARITY_HANDLING.md:1272)"}


def e2e_buffers(nbytes):
    """Three device buffers (and three pinned host result buffers) where both memories hold them
    with room to spare, else two."""
    import torch
    import psutil
    free_dev, _ = torch.cuda.mem_get_info()
    host = psutil.virtual_memory().available
    return 3 if free_dev > 3 * nbytes + (4 << 30) and host > 4 * nbytes + (16 << 30) else 2


def end_to_end(P, uh, dt, K, world, pts, stream, dist, NB=3):
    """The metric through the public API with host buffers: per step the state is copied in
    from pinned host memory (uh), stepped, and copied back, all inside the timed region. The
    steps are independent requests, pipelined over NB device buffers: step n+1's upload (one
    copy stream) and step n-1's download (another) run while step n computes; with NB = 3 no
    upload waits for the download of the buffer it refills (step n-2's, long finished), so the two
    directions run at once; with NB = 2 (where memory holds no third buffer) the upload of step
    n+1 waits for step n-1's download."""
    import torch
    res_h = [torch.empty(uh.numel(), dtype=uh.dtype, pin_memory=True) for _ in range(NB)]
    ud = [torch.empty(uh.numel(), dtype=uh.dtype, device="cuda") for _ in range(NB)]
    ud[0].copy_(uh)
    P.step_batched(ud[0], 0.0, dt, 1)  # graph for one step
    torch.cuda.synchronize()
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(NB)]
    ev_done = [torch.cuda.Event() for _ in range(NB)]
    ev_out = [torch.cuda.Event() for _ in range(NB)]
    for e in ev_out:
        e.record(stream)
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    s_in.wait_event(e2)
    s_out.wait_event(e2)
    for n in range(K):
        i = n % NB
        s_in.wait_event(ev_out[i])  # buffer i's previous result has been read back
        with torch.cuda.stream(s_in):
            ud[i].copy_(uh, non_blocking=True)
        ev_in[i].record(s_in)
        stream.wait_event(ev_in[i])
        P.step_batched(ud[i], 0.0, dt, 1)
        ev_done[i].record(stream)
        s_out.wait_event(ev_done[i])
        with torch.cuda.stream(s_out):
            res_h[i].copy_(ud[i], non_blocking=True)
        ev_out[i].record(s_out)
    for e in ev_out:
        stream.wait_event(e)
    e3.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e2.elapsed_time(e3)
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    nbytes = uh.numel() * 8
    ok = all(bool(torch.isfinite(r).all()) for r in res_h[:min(NB, K)])
    return {"value": world * pts * K / (e2e_ms * 1e-3), "unit": "point-updates/s", "ms_per_step": e2e_ms / K,
            "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes, "results_finite": ok,
            "pipelining": f"step n+1's upload and step n-1's download overlap step n ({NB} device buffers, "
                          "two copy streams, one cudaMemcpyAsync each way per step)"}


def plain_forms(P, u0, dt, K, pts, stream):
    """The plain per-stage form (per stage: fill of u, RHS into du over all blocks, stage update;
    host-issued) and the plain per-block form (the same, with one RHS launch and one stage update
    per block), each timed with CUDA events over a few steps from the workload's state."""
    import torch
    out = {}
    for name, fn, steps in (("per_stage", P.rk4_step, max(3, K // 3)), ("per_block", P.rk4_step_blocks, 3)):
        up = u0.clone()
        fn(up, 0.0, dt)
        torch.cuda.synchronize()
        e4, e5 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e4.record(stream)
        for n in range(steps):
            fn(up, n * dt, dt)
        e5.record(stream)
        torch.cuda.synchronize()
        ms = e4.elapsed_time(e5) / steps
        out[name] = {"value": pts / (ms * 1e-3), "unit": "point-updates/s", "ms_per_step": ms, "steps": steps}
        if name == "per_block":
            out[name]["gpu_launches_per_step"] = P.last_launch_count()
        del up
    out["per_stage"]["form"] = "per stage: fill of u, one RHS launch pair over all blocks into du, stage update"
    out["per_block"]["form"] = ("per stage: fill of u, then per block one RHS launch pair and one stage update "
                                "(the reference's block map), host-issued")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="hierarchy", choices=["hierarchy", "kerr_schild_static", "fourier",
                                                                       "hierarchy_small", "g5"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="mixed: FP32 stencil sums and algebra on the FP64 state (one GPU)")
    ap.add_argument("--shard", action="store_true",
                    help="run the sharded step (the --gpus N > 1 path) even on one GPU")
    ap.add_argument("--monitors-only", action="store_true",
                    help="time only the constraint monitors (each with its prepare) on the workload's state: "
                         "the command the monitor profiles are taken with")
    ap.add_argument("--pi", default="auto", choices=["auto", "l1", "tma"],
                    help="the Pi kernel: the autotuner's recorded choice (auto), the L1 one-point kernel, or "
                         "the TMA-staged pair kernel")
    ap.add_argument("--step-only", action="store_true",
                    help="time only the batched step (the graph of K steps) on the workload: the command the "
                         "launch lists are taken with")
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
    if world > 1 or args.shard:
        import datetime
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29533")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), rank=rank, world_size=world,
                                device_id=torch.device("cuda", local))
    tgh = load_package()
    case, forest, scase, sforest, cfg, gauge, perturbed = workload(tgh, args.workload)
    if world > 1 or args.shard:
        return run_sharded(args, tgh, world, rank, local, case, forest, cfg, gauge, perturbed)
    stream = torch.cuda.current_stream()
    P = ready(case, tgh.GHProblem(case, forest, 4, margin_check=False, precision=args.precision), forest)
    if args.pi != "auto":
        P.set_variant(pi=args.pi)
    u0 = initial(tgh, P, forest, perturbed)
    if args.rhs_only:
        ms = P.time_rhs(u0, 0.0, mode=1, nlaunch=2)
        print(json.dumps({"workload": cfg["workload"], "rhs_ms_per_launch": ms, "variant": P.variant(),
                          "points_per_launch": (forest.N + 1) ** 3 * forest.nblocks}))
        P.close()
        return 0
    if args.monitors_only:
        n1 = (forest.N + 1) ** 3 * forest.nblocks
        print(json.dumps({"workload": cfg["workload"], "points": n1,
                          **time_monitors(P, u0, stream, gauge, n1, tgh.fp64_peak_tflops(), reps=1)}))
        P.close()
        return 0
    lam = P.max_speed(u0, 0.0)
    dt = 0.25 * h_min(forest) / lam
    K, W = args.steps, max(3, args.warmup)

    big = args.workload == "hierarchy"
    # warm-up: at least W untimed steps, as K-step runs of the graph the timed run replays
    # (the first run captures it), on one copy of the initial state
    u = u0.clone()
    for _ in range(-(-W // K)):
        u.copy_(u0)
        P.step_batched(u, 0.0, dt, K)
    torch.cuda.synchronize()
    u.copy_(u0)
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
    if args.step_only:
        print(json.dumps({"workload": cfg["workload"], "value": value, "unit": "point-updates/s", "ms_per_step": ms / K,
                          "steps": K, "variant": P.variant(), "gpu_launches": launches, "clocks": ck}))
        P.close()
        return 0

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

    # the constraint monitors on the same state (their per-chunk cadence: not part of a step)
    monitors = time_monitors(P, u0, stream, gauge, n1pts, peak)

    # end to end through the public API with host buffers: per step the state is copied in
    # from pinned host memory and the result copied back
    uh = torch.empty(u0.numel(), dtype=u0.dtype, pin_memory=True)
    uh.copy_(u0)
    del u
    if big:
        del u0  # the hierarchy's state is 14 GB: its device buffers sit beside the batched problem's
        torch.cuda.empty_cache()
    e2e = end_to_end(P, uh, dt, K, world, pts, stream, dist, NB=e2e_buffers(uh.numel() * 8))
    if big:
        # the plain forms' own buffers (k, acc, y) do not fit beside the batched form's: a problem
        # of their own once the batched one is released
        P.close()
        torch.cuda.empty_cache()
        P = ready(case, tgh.GHProblem(case, forest, 4, margin_check=False, precision=args.precision), forest)
        if args.pi != "auto":
            P.set_variant(pi=args.pi)
        u0 = uh.cuda()
    plain = plain_forms(P, u0, dt, K, pts, stream)

    out = {"metric": "RK4 point-updates/s", "value": value, "unit": "point-updates/s", "n_gpus": world,
           "steps": K, "warmup": W, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32 arithmetic, f64 state",
           "data": "synthetic",
           "config": {**cfg, "form": "batched (fused RK4 epilogue, CUDA graph)", "points": pts,
                      "kernel_variant": P.variant(),
                      "precision": args.precision,
                      "l2_flush": "inputs larger than L2 (working arrays %.0f MB)" % (P.work_length * 8 / 1e6),
                      "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
           "roofline": {"bound": "fp64", "kernel": rhs_kernels(P, cfg),
                        "achieved": achieved, "peak": peak,
                        "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
                        "flop_per_point": FLOP_PER_POINT_RHS[gauge], "points_per_launch": n1pts,
                        "ms_per_launch": rhs_ms,
                        "peak_source": "measured FP64 FMA probe on this GPU (MEASURED_PEAKS.json has no FP64)"},
           "e2e": e2e,
           "plain_form": plain["per_stage"],
           "plain_per_block": plain["per_block"],
           "speedup_vs_plain_per_block": plain["per_block"]["ms_per_step"] / (ms / K),
           "speedup_vs_plain_per_stage": plain["per_stage"]["ms_per_step"] / (ms / K),
           "monitors": monitors,
           "gpu_launches": launches, "clocks": ck}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(tgh, scase, sforest, perturbed)
    P.close()
    if big and world == 1:
        torch.cuda.empty_cache()
        out["g5_chart"] = g5_chart(tgh, K, stream, with_cpu=not args.no_cpu_baseline)
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
