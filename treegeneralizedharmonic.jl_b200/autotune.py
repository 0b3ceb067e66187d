"""The autotuner of the right-hand side's kernels.

The reference compiles its kernels per problem through KernelAbstractions and picks no launch
shape itself. Here the choices are made by measurement on the GPU the problem runs on: for a
problem (its mesh, order, precision and case), every candidate variant - the Pi half through L1
at 3, 4 or 5 resident CTAs per SM or from TMA-staged tiles, the head and one-point Pi kernels at
64 or 128 threads a CTA - is timed over whole right-hand sides of the batched form (head + Pi,
RK4 stage epilogue, CUDA events on the problem's stream), and the fastest is recorded in
tuning/<gpu>.json under the configuration's key. GHProblem applies the recorded choice at
construction (tuned=True); every variant computes the same bits, so the choice changes speed
only.
"""
import json
import os
from pathlib import Path

import torch

TUNING_DIR = Path(__file__).resolve().parent / "tuning"


def gpu_key():
    name = torch.cuda.get_device_name() if torch.cuda.is_available() else "none"
    return "".join(c if c.isalnum() else "_" for c in name).strip("_").lower()


def config_key(problem):
    """The configuration a record holds for: order, block size, arithmetic, interior or not."""
    c = problem.case
    return f"q{problem.q}_n{problem.forest.N}_{problem.precision}_{'interior' if c.interior else 'nointerior'}"


def candidates(problem):
    out = []
    for threads in (128, 64):
        for mb in (4, 3, 5):
            out.append({"pi": "l1", "threads": threads, "pi_mb": mb})
    if problem.q == 4 and problem.forest.N == 32 and problem.precision == "fp64":
        for threads in (128, 64):
            out.append({"pi": "tma", "threads": threads, "pi_mb": 4})
    return out


def tune(problem, u, t=0.0, nlaunch=6, repeats=3, record=True, path=None):
    """Time every candidate on `problem` (state u at t) and, with record, store the fastest.
    Returns {"key", "gpu", "choice", "sweep": [{variant, ms}...]}."""
    sweep = []
    for v in candidates(problem):
        problem.set_variant(**v)
        problem.time_rhs(u, t, nlaunch=2)  # warm (and the TMA maps made)
        ms = min(problem.time_rhs(u, t, nlaunch=nlaunch) for _ in range(repeats))
        problem.device_status()
        sweep.append({**v, "ms_per_rhs": ms})
    best = min(sweep, key=lambda r: r["ms_per_rhs"])
    choice = {k: best[k] for k in ("pi", "threads", "pi_mb")}
    problem.set_variant(**choice)
    res = {"key": config_key(problem), "gpu": gpu_key(), "choice": choice, "sweep": sweep,
           "points_per_rhs": (problem.forest.N + 1) ** 3 * problem.forest.nblocks}
    if record:
        save_record(res, path)
    return res


def _file(path=None):
    return Path(path) if path else TUNING_DIR / f"{gpu_key()}.json"


def save_record(res, path=None):
    f = _file(path)
    f.parent.mkdir(parents=True, exist_ok=True)
    data = json.loads(f.read_text()) if f.exists() else {}
    data[res["key"]] = {"choice": res["choice"], "sweep": res["sweep"], "points_per_rhs": res["points_per_rhs"]}
    tmp = f.with_suffix(".partial")
    tmp.write_text(json.dumps(data, indent=1, sort_keys=True) + "\n")
    os.replace(tmp, f)


def recorded_choice(problem, path=None):
    """The recorded fastest variant for the problem's configuration on this GPU, or None."""
    f = _file(path)
    if not f.exists():
        return None
    rec = json.loads(f.read_text()).get(config_key(problem))
    if not rec:
        return None
    choice = rec["choice"]
    if choice["pi"] == "tma" and not (problem.q == 4 and problem.forest.N == 32 and problem.precision == "fp64"):
        return None
    return dict(choice)
