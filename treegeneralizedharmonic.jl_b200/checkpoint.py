"""Checkpoint and restart of the stepping path's state (src/checkpoint.jl).

The reference writes its checkpoints through TreeIOHDF5 (HDF5), which is not installed here:
the container is numpy's `.npz` instead, with the reference's naming, rotation and refusals
(src/checkpoint.jl:40-140): the file after `iteration` steps is `<prefix>.it<10 digits>.npz`;
a write goes to `<file>.partial` and is renamed into place once it is complete and synced, so
a failed write never leaves a file the listing would take for a checkpoint; after a write all
but the newest `num_keep` files are removed, the one just written always kept; a restart whose
recipe (the case and the order, every parameter that decides a number) differs from the
file's is refused by name. Each file holds the forest, the recipe, the time, the iteration
and the state vector bit for bit (the run state of the reference's driver, its horizon track
and fits, belongs to the driver and is not on this path; `extra` carries what a caller adds).
"""
import json
import os
import re

import numpy as np

SUFFIX = ".npz"


def checkpoint_filename(prefix, iteration):
    return f"{prefix}.it{int(iteration):010d}{SUFFIX}"


def checkpoint_files(prefix):
    """(iteration, path) of `prefix`'s checkpoints, sorted: the files in its directory named
    exactly `<basename>.it<digits>.npz` (not a `.partial`, not another prefix)."""
    d, base = os.path.split(prefix)
    if not base:
        return []
    listed = d or "."
    if not os.path.isdir(listed):
        return []
    pat = re.compile("^" + re.escape(base) + r"\.it(\d+)" + re.escape(SUFFIX) + "$")
    found = []
    for name in os.listdir(listed):
        m = pat.match(name)
        if m:
            path = os.path.join(d, name) if d else name
            if os.path.isfile(path):
                found.append((int(m.group(1)), path))
    return sorted(found)


def latest_checkpoint(prefix):
    """The checkpoint of `prefix` with the highest iteration, or None."""
    files = checkpoint_files(prefix)
    return files[-1][1] if files else None


def rotate_checkpoints(prefix, num_keep, keep):
    """Remove all of `prefix`'s checkpoints but `keep` (recognised by its name) and the newest
    num_keep - 1 others; returns the paths removed."""
    others = [p for _, p in checkpoint_files(prefix) if os.path.basename(p) != os.path.basename(keep)]
    removed = others[:max(0, len(others) - (num_keep - 1))]
    for p in removed:
        os.remove(p)
    return removed


def recipe(case, q, precision="fp64"):
    """Every parameter of a run that decides a number: the case and the order."""
    return {"background": case.background, "box": [list(b) for b in case.box], "periodic": list(case.periodic),
            "eps_ko": case.eps_ko, "gamma0": case.gamma0, "gamma2": case.gamma2, "interior": case.interior,
            "gauge": case.gauge, "ks_source": case.ks_source, "M": case.M, "q": int(q), "precision": precision}


def _canon(x):
    return json.loads(json.dumps(x, sort_keys=True, default=list))


def save_checkpoint(prefix, iteration, P, u, t, num_keep=2, extra=None):
    """Write the state u of problem P at time t after `iteration` steps; returns the path."""
    import torch
    path = checkpoint_filename(prefix, iteration)
    f = P.forest
    if isinstance(u, torch.Tensor) and u.is_cuda:
        torch.cuda.synchronize()  # the problem's stream may not be the current one
    host = u.detach().to("cpu").numpy() if isinstance(u, torch.Tensor) else np.asarray(u)
    fields = {
        "application": np.array("TreeGeneralizedHarmonic.jl (B200 stepping path)"), "version": np.array(1),
        "recipe": np.array(json.dumps(_canon(recipe(P.case, P.q, P.precision)), sort_keys=True)),
        "extra": np.array(json.dumps(_canon(extra or {}), sort_keys=True)),
        "t": np.array(float(t), dtype=np.float64), "iteration": np.array(int(iteration), dtype=np.int64),
        "N": np.array(f.N), "lo": np.array(f.lo, dtype=np.float64), "h0": np.array(f.h0, dtype=np.float64),
        "cells0": np.array(f.cells0), "periodic": np.array(f.periodic), "level": np.asarray(f.level, dtype=np.int32),
        "corner": np.asarray(f.corner, dtype=np.int32), "state": host,
    }
    tmp = path + ".partial"
    with open(tmp, "wb") as fh:
        np.savez(fh, **fields)
        fh.flush()
        os.fsync(fh.fileno())
    os.replace(tmp, path)
    rotate_checkpoints(prefix, num_keep, keep=path)
    return path


def load_checkpoint(path, case=None, q=None, precision="fp64"):
    """The forest, state (host array), t, iteration and extra of a checkpoint; with case and q,
    a recipe that differs from the file's is refused, naming the first parameter that differs."""
    from .forest import Forest
    with np.load(path, allow_pickle=False) as z:
        rec = json.loads(str(z["recipe"]))
        if case is not None:
            mine = _canon(recipe(case, q, precision))
            for k in sorted(set(rec) | set(mine)):
                if rec.get(k) != mine.get(k):
                    raise ValueError(f"the checkpoint {path} was written with {k} = {rec.get(k)!r}, and this run has "
                                     f"{k} = {mine.get(k)!r}: a restart continues the same run")
        f = Forest(int(z["N"]), tuple(float(x) for x in z["lo"]), float(z["h0"]), tuple(int(x) for x in z["cells0"]),
                   tuple(bool(x) for x in z["periodic"]), np.array(z["level"]), np.array(z["corner"]))
        return {"forest": f, "state": np.array(z["state"]), "t": float(z["t"]), "iteration": int(z["iteration"]),
                "recipe": rec, "extra": json.loads(str(z["extra"]))}
