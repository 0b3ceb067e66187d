"""Checkpoint and restart (src/checkpoint.jl): names, rotation, atomic writes, the state bit for
bit, and the refusal of a restart with another recipe. CPU: a problem stand-in carries what a
checkpoint reads (forest, case, order); GPU: a run restarted from its checkpoint is the run."""
import os
from types import SimpleNamespace

import numpy as np
import pytest


def _stand_in(tgh, q=4):
    case = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=2.0, r0=0.8, r1=1.3, gauge="sampled")
    forest = tgh.gh_forest(case, 8, 2)
    return SimpleNamespace(case=case, forest=forest, q=q, precision="fp64")


def test_names_rotation_and_the_latest(tgh, tmp_path):
    C = tgh.checkpoint
    P = _stand_in(tgh)
    prefix = str(tmp_path / "run")
    u = np.random.default_rng(1).standard_normal(P.forest.nblocks * 20 * 9 ** 3)
    assert tgh.latest_checkpoint(prefix) is None
    for it in (8, 16, 24):
        path = tgh.save_checkpoint(prefix, it, P, u + it, 0.125 * it, num_keep=2)
        assert os.path.basename(path) == f"run.it{it:010d}.npz"
    assert [i for i, _ in C.checkpoint_files(prefix)] == [16, 24]
    assert tgh.latest_checkpoint(prefix).endswith("run.it0000000024.npz")
    # a partial write and another prefix are not checkpoints
    (tmp_path / "run.it0000000032.npz.partial").write_bytes(b"x")
    (tmp_path / "run2.it0000000040.npz").write_bytes(b"x")
    assert [i for i, _ in C.checkpoint_files(prefix)] == [16, 24]
    # a restart from an older checkpoint keeps the file it writes, even when it is not the newest
    path = tgh.save_checkpoint(prefix, 20, P, u, 2.5, num_keep=1)
    assert [i for i, _ in C.checkpoint_files(prefix)] == [20]


def test_the_state_reads_back_bit_for_bit_and_a_changed_recipe_is_refused(tgh, tmp_path):
    P = _stand_in(tgh)
    prefix = str(tmp_path / "hole")
    u = np.random.default_rng(2).standard_normal(P.forest.nblocks * 20 * 9 ** 3)
    path = tgh.save_checkpoint(prefix, 3, P, u, 0.375, extra={"growth": 1.5})
    r = tgh.load_checkpoint(path, case=P.case, q=P.q)
    assert np.array_equal(r["state"], u) and r["t"] == 0.375 and r["iteration"] == 3
    assert r["extra"] == {"growth": 1.5}
    assert np.array_equal(r["forest"].corner, P.forest.corner) and r["forest"].h0 == P.forest.h0
    with pytest.raises(ValueError, match="q"):
        tgh.load_checkpoint(path, case=P.case, q=2)
    other = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=2.0, r0=0.8, r1=1.3, gauge="sampled", eps_ko=0.25)
    with pytest.raises(ValueError, match="eps_ko"):
        tgh.load_checkpoint(path, case=other, q=P.q)


@pytest.mark.gpu
def test_a_restarted_run_is_the_run(tgh, tmp_path):
    import torch
    case = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=2.0, r0=0.8, r1=1.3, gauge="sampled")
    forest = tgh.gh_forest(case, 8, 2)
    P = tgh.GHProblem(case, forest, 4, margin_check=False)
    u = P.initial_state(P.statevector(), 0.0)
    dt = P.gh_dt(u, cfl=0.25)
    P.step_batched(u, 0.0, dt, 3)
    path = tgh.save_checkpoint(str(tmp_path / "ks"), 3, P, u, 3 * dt)
    P.step_batched(u, 3 * dt, dt, 2)
    r = tgh.load_checkpoint(path, case=case, q=4)
    P2 = tgh.GHProblem(case, r["forest"], 4, margin_check=False)
    u2 = torch.from_numpy(r["state"]).cuda()
    P2.step_batched(u2, r["t"], dt, 2)
    torch.cuda.synchronize()
    assert torch.equal(u, u2)
