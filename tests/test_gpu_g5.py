"""The reference's G5 chart (test/hole_runs.jl:2416-2435, SINGULARITY_HANDLING.md:1066, 1272): Kerr
M = 1, a = 7/10 in harmonic coordinates on [-5/4, 5/4]^3, one root block of 8^3 refined by
hole_forest with radii 10, 8/5, 13/10, 1. The mesh is the reference's to the leaf: 2472 blocks
of 8^3, 1,265,664 points, finest h = 5/256 (the numbers the reference states for it). The
interior here is the :fitted branch over a sphere (r_0 = 0.8, r_1 = 1), relaxing toward the
analytic cache (the reference's fitted target needs its horizon track). The whole mesh is small
enough for the oracle: the right-hand side of every block at 1e-12 of rhs_scale, and one RK4 step,
plain and batched."""
import numpy as np
import pytest
import torch

from helpers import rhs_error, rhs_scale

pytestmark = pytest.mark.gpu


def _g5(tgh):
    case = tgh.harmonic_kerr_case(M=1.0, a=0.7, halfwidth=1.25, r0=0.8, r1=1.0, rho_max=4.0, variant="fitted",
                                  eps_ko=0.5)
    return case, tgh.hole_forest(case, 8, 1, [10.0, 1.6, 1.3, 1.0])


def test_g5_rhs_and_step_match_the_oracle_on_the_whole_mesh(tgh, oracle):
    case, f = _g5(tgh)
    P = tgh.GHProblem(case, f, 4)  # the radius checks on (margin_check)
    O = oracle.problem(case, f, 4, margin_check=True)
    r_fill = 1.0 + f.h0 / 16
    P.fill_target_analytic(0.0, r_fill)
    O.fill_target_analytic(0.0, r_fill, 0.0)
    u = O.initial_state(O.statevector(), 0.0) + tgh.perturbation(f, amplitude=1e-6, seed=8)
    du_ref = np.zeros(O.L)
    O.gh_rhs(du_ref, u, 0.0)
    ug = torch.from_numpy(u).cuda()
    dug = torch.full_like(ug, float("nan"))
    P.gh_rhs(dug, ug, 0.0)
    du = dug.cpu().numpy()
    assert np.all(np.isfinite(du))
    assert rhs_error(du, du_ref, rhs_scale(O.work(), f, 4), f) < 1e-12
    _, lam = O.max_speed(u, 0.0)
    dt = 0.25 * (f.h0 / 16) / lam
    uo = u.copy()
    O.rk4_step(uo, 0.0, dt)
    scale = max(1.0, float(np.abs(uo).max()))
    up = torch.from_numpy(u).cuda()
    P.rk4_step(up, 0.0, dt)
    assert float(np.max(np.abs(up.cpu().numpy() - uo))) < 1e-12 * scale
    ub = torch.from_numpy(u).cuda()
    P.step_batched(ub, 0.0, dt, 1)
    P.settle(ub, dt)
    us = torch.from_numpy(uo).cuda()
    P.settle(us, dt)
    assert torch.max(torch.abs(ub - us)).item() < 1e-12 * scale
    P.close()
