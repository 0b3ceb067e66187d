"""The CUDA path against the CPU oracle on identical inputs (the parity gate).

Tolerances (the reference's own, test/evolution_tests.jl:141-179): the right-hand side
within 1e-12 of rhs_scale per point, on every row, the moving hole's included; the ghost
fill bit for bit: copies, prolongation and the Dirichlet ghosts (the analytic state is
evaluated on the device in the oracle's order with every operation rounded on its own); one
RK4 step within 1e-12 absolute on states of order one.
"""
import math

import numpy as np
import pytest
import torch

from helpers import N_ROWS, cases, rhs_error, rhs_scale, two_level_forest

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-12


def _to_gpu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _initial(tgh, P, O, case, forest, name, t):
    u = O.initial_state(O.statevector(), t)
    if name.startswith("perturbed"):
        u = u + tgh.perturbation(forest, amplitude=1e-4)
    elif name.startswith("kerr") or name.startswith("gauge") or name.startswith("harmonic"):
        u = u + tgh.perturbation(forest, amplitude=1e-6, seed=11)
    if name.endswith("pasted"):
        O.stage_limit(u, t)
    return u


@pytest.mark.parametrize("row", range(N_ROWS))
def test_rhs_matches_oracle(tgh, oracle, row):
    name, case, forest, q, t = cases(tgh)[row]
    P = tgh.GHProblem(case, forest, q, margin_check=False)
    O = oracle.problem(case, forest, q)
    u = _initial(tgh, P, O, case, forest, name, t)
    du_ref = np.zeros(O.L)
    O.gh_rhs(du_ref, u, t)
    ug = _to_gpu(u)
    dug = torch.full_like(ug, float("nan"))
    P.gh_rhs(dug, ug, t)
    torch.cuda.synchronize()
    assert torch.equal(ug, _to_gpu(u)), "u was written"
    du = dug.cpu().numpy()
    assert np.all(np.isfinite(du))
    err = rhs_error(du, du_ref, rhs_scale(O.work(), forest, q), forest)
    # A moving hole's layer and core read the target's rate as the centered difference
    # (Pi(t + d) - Pi(t - d)) / 2d with d = eps^(1/3) r_0 (src/initialdata.jl:1721-1729): an ulp
    # of difference between two evaluations of the analytic Pi would move it by ~1e-11 |Pi|.
    # The device evaluates that state bit for bit as the oracle does, so the bound holds there
    # as everywhere else.
    assert err < RHS_TOL, f"{name}: {err}"


@pytest.mark.parametrize("n32", [False, True])
def test_second_differences_are_the_references_sums_at_fine_spacing(tgh, oracle, n32):
    """A Kerr-Schild hole's exterior at h = 1/2048 (r ~ 1.6): a second difference's rounding,
    eps |u| sum|w| / h^2, is ~6e-10 of rhs_scale there, so a summation order or rounding other
    than the reference's (axis_stencil, mixed_stencil, src/evolution.jl:192-219) would miss the
    1e-12 bound by orders of magnitude. Blocks of 8^3 (the general kernels) and of 32^3 (the
    N = 32 kernels: the one-point Pi kernel and the TMA-staged one)."""
    c = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=4.0, r0=0.8, r1=1.3, gauge="algebraic")
    N = 32 if n32 else 8
    leaves = sorted((0, (x, y, z)) for z in (0, N) for y in (0, N) for x in (0, N))
    f = tgh.Forest(N, (1.5, 0.3, 0.2), 1.0 / 2048, (2 * N, 2 * N, 2 * N), (False, False, False),
                   np.array([l for l, _ in leaves], dtype=np.int32),
                   np.array([c_ for _, c_ in leaves], dtype=np.int32))
    P = tgh.GHProblem(c, f, 4, margin_check=False)
    O = oracle.problem(c, f, 4)
    u = O.initial_state(O.statevector(), 0.0) + tgh.perturbation(f, amplitude=1e-9, seed=3)
    du_ref = np.zeros(O.L)
    O.gh_rhs(du_ref, u, 0.0)
    scale = rhs_scale(O.work(), f, 4)
    ug = _to_gpu(u)
    for pi in ("l1", "tma") if n32 else ("l1",):
        P.set_variant(pi=pi)
        dug = torch.full_like(ug, float("nan"))
        P.gh_rhs(dug, ug, 0.0)
        torch.cuda.synchronize()
        err = rhs_error(dug.cpu().numpy(), du_ref, scale, f)
        assert err < RHS_TOL, (pi, err)
    P.close()


def test_matter_source_matches_oracle(tgh, oracle):
    c = tgh.gauge_wave_case(eps_ko=0.5, gamma0=1.0, gamma2=-0.5)
    f = tgh.gh_forest(c, 8, 2)
    P = tgh.GHProblem(c, f, 4)
    O = oracle.problem(c, f, 4)
    u = O.initial_state(O.statevector(), 0.1)
    rng = np.random.default_rng(3)
    m = 1e-3 * rng.standard_normal(10 * (f.N + 1) ** 3 * f.nblocks)
    du_ref = np.zeros(O.L)
    O.gh_rhs(du_ref, u, 0.1, m)
    du = torch.zeros(O.L, dtype=torch.float64, device="cuda")
    P.gh_rhs(du, _to_gpu(u), 0.1, _to_gpu(m))
    assert rhs_error(du.cpu().numpy(), du_ref, rhs_scale(O.work(), f, 4), f) < RHS_TOL
    # and the matter term is live
    du0 = torch.zeros_like(du)
    P.gh_rhs(du0, _to_gpu(u), 0.1)
    assert torch.max(torch.abs(du - du0)).item() > 1e-6


@pytest.mark.parametrize("which", ["periodic", "dirichlet", "two_level"])
def test_fill_matches_oracle(tgh, oracle, which):
    if which == "periodic":
        c = tgh.perturbed_minkowski_case()
        f = tgh.gh_forest(c, 8, 2)
    elif which == "dirichlet":
        c = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=2.0, r0=0.8, r1=1.3, gauge="algebraic")
        f = tgh.gh_forest(c, 8, 2)
    else:
        c = tgh.gauge_wave_case(eps_ko=0.5, gamma0=1.0)
        f = two_level_forest(tgh, c)
    P = tgh.GHProblem(c, f, 4, margin_check=False)
    O = oracle.problem(c, f, 4)
    u = O.initial_state(O.statevector(), 0.2) + tgh.perturbation(f, amplitude=1e-5, seed=5)
    O.prepare(u, 0.2)
    P.prepare(_to_gpu(u), 0.2)
    wg = P.copy_work().cpu().numpy()
    wo = O.work()
    assert np.array_equal(wg, wo)


@pytest.mark.parametrize("row", [0, 2, 6, 7, 9, 11, 14, 17, 18, 19, 20, 21])
def test_rk4_step_matches_oracle(tgh, oracle, row):
    name, case, forest, q, t = cases(tgh)[row]
    P = tgh.GHProblem(case, forest, q, margin_check=False)
    O = oracle.problem(case, forest, q)
    u = _initial(tgh, P, O, case, forest, name, t)
    dt = 0.25 * (forest.h0 / 2 ** int(forest.level.max())) / 2.0
    ug = _to_gpu(u)
    P.rk4_step(ug, t, dt)
    uo = u.copy()
    O.rk4_step(uo, t, dt)
    tol = 1e-12
    assert np.max(np.abs(ug.cpu().numpy() - uo)) < tol
    if not name.endswith("pasted"):
        ub = _to_gpu(u)
        P.step_batched(ub, t, dt, 1)
        # compare settled states (the batched form keeps each copy at its primary's value)
        P.settle(ub, t + dt)
        us = _to_gpu(uo)
        P.settle(us, t + dt)
        assert torch.max(torch.abs(ub - us)).item() < tol


def test_two_level_rk4_step_matches_oracle(tgh, oracle):
    c = tgh.gauge_wave_case(eps_ko=0.5, gamma0=1.0, gamma2=-0.5)
    f = two_level_forest(tgh, c)
    P = tgh.GHProblem(c, f, 4)
    O = oracle.problem(c, f, 4)
    u = O.initial_state(O.statevector(), 0.0)
    dt = 0.25 * f.h0 / 2 / 2.0
    ug = _to_gpu(u)
    P.rk4_step(ug, 0.0, dt)
    uo = u.copy()
    O.rk4_step(uo, 0.0, dt)
    assert np.max(np.abs(ug.cpu().numpy() - uo)) < 1e-12


def test_max_speed_and_error_norm_match_oracle(tgh, oracle):
    c = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=2.0, r0=0.8, r1=1.3, gauge="algebraic")
    f = tgh.gh_forest(c, 8, 2)
    P = tgh.GHProblem(c, f, 4, margin_check=False)
    O = oracle.problem(c, f, 4)
    u = O.initial_state(O.statevector(), 0.0)
    ug = P.initial_state(P.statevector(), 0.0)
    assert np.max(np.abs(ug.cpu().numpy() - u)) < 1e-13 * max(1.0, np.max(np.abs(u)))
    st, lam_o = O.max_speed(u, 0.0)
    assert st == 0
    assert P.max_speed(ug, 0.0) == pytest.approx(lam_o, rel=1e-14)
    pert = tgh.perturbation(f, amplitude=1e-6, seed=9)
    l2o, lio = O.error_norm(u + pert, 0.0)
    l2g, lig = P.error_norm(_to_gpu(u + pert), 0.0)
    assert l2g == pytest.approx(l2o, rel=1e-10) and lig == pytest.approx(lio, rel=1e-10)
    assert l2o > 0


def test_flat_speed_is_sqrt3_and_nonfinite_refused(tgh):
    c = tgh.minkowski_case(L=1.0)
    f = tgh.gh_forest(c, 8, 2)
    P = tgh.GHProblem(c, f, 4)
    u = P.initial_state(P.statevector(), 0.0)
    assert P.max_speed(u, 0.0) == pytest.approx(math.sqrt(3.0), rel=1e-15)
    u[1234] = float("nan")
    with pytest.raises(tgh._abi.TGHError) as e:
        P.max_speed(u, 0.0)
    assert e.value.code == tgh._abi.TGH_ERR_NONFINITE
    u.zero_()
    u[:] = float("nan")
    with pytest.raises(tgh._abi.TGHError):
        P.max_speed(u, 0.0)


def test_hole_interior_is_masked_for_speed(tgh):
    # a NaN inside r_1 is not a reason to refuse (src/evolution.jl:1531-1537)
    c = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=2.0, r0=0.8, r1=1.3, gauge="algebraic")
    f = tgh.gh_forest(c, 8, 2)
    P = tgh.GHProblem(c, f, 4, margin_check=False)
    u = P.initial_state(P.statevector(), 0.0)
    N1 = f.N + 1
    # block 0 is [-2,0]^3; its corner point (N, N, N) is the origin
    u[0 * 20 * N1 ** 3 + f.N + N1 * (f.N + N1 * f.N)] = float("nan")
    assert math.isfinite(P.max_speed(u, 0.0))


def test_analytic_state_is_the_oracles_bit_for_bit(tgh, oracle):
    """The device's analytic state (Dirichlet ghosts, layer and core targets) at points around a
    resting and a moving (boosted) spinning hole, in Kerr-Schild and in harmonic coordinates, and
    near the chart's singular set: every h, Pi bit for bit the oracle's. The moving hole's target rates are centred differences of this state
    over 1.2e-5 r_0 in t, which would turn one ulp into ~1e-11. Both charts take only
    +, -, *, / and square roots, correctly rounded on both sides; shifted Minkowski's tanh (and
    the gauge wave's sin) come from CUDA's and the C library's own functions, which may differ
    in the last bit, and psi = A (1 - tanh^2) carries that on: there, within 1e-15 of max(1, |u|)."""
    rng = np.random.default_rng(7)
    for case in (tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=2.0, r0=0.8, r1=1.3, gauge="algebraic"),
                 tgh.kerr_schild_case(M=1.0, a=0.7, v=0.1, halfwidth=2.0, r0=0.8, r1=1.3, gauge="algebraic"),
                 tgh.harmonic_kerr_case(M=1.0, a=0.7, halfwidth=2.0, r0=0.9, r1=1.4),
                 tgh.harmonic_kerr_case(M=1.0, a=0.7, v=0.1, halfwidth=2.0, r0=0.9, r1=1.4),
                 tgh.shifted_minkowski_case(eps_ko=0.5, gamma0=1.0, gamma2=-0.5)):
        f = tgh.gh_forest(case, 8, 2)
        P = tgh.GHProblem(case, f, 4, margin_check=False)
        bg = oracle.background(case)
        pts = np.concatenate([rng.uniform(-2.0, 2.0, (40, 3)), rng.uniform(-0.9, 0.9, (20, 3))])
        for k, x in enumerate(pts):
            t = 0.3 + 1e-5 * k
            got = np.array(P.point_physics(t, x)[:20])
            it = case.interior
            if it and np.linalg.norm(x - (np.array(it["c0"]) + t * np.array(it["v"]))) < it["r0"]:
                continue  # the core rule moves the point; the background is compared off the core
            h, Pi, _, _ = oracle.background_state(bg, t, x)
            ref = np.concatenate([h, Pi])
            if case.background["kind"] in ("kerr_schild", "harmonic_kerr"):
                assert np.array_equal(got, ref), (k, x, got - ref)
            else:
                assert np.all(np.abs(got - ref) <= 1e-15 * np.maximum(np.abs(ref), 1.0)), (k, x, got - ref)
        P.close()


@pytest.mark.parametrize("row", [7, 19])
def test_per_block_form_is_the_plain_form(tgh, oracle, row):
    """The plain per-block form (one right-hand-side launch and one stage update per block, the
    reference's block map) is the plain per-stage form's step bit for bit."""
    name, case, forest, q, t = cases(tgh)[row]
    P = tgh.GHProblem(case, forest, q, margin_check=False)
    O = oracle.problem(case, forest, q)
    u = _to_gpu(_initial(tgh, P, O, case, forest, name, t))
    dt = 0.25 * (forest.h0 / 2 ** int(forest.level.max())) / 2.0
    a, b = u.clone(), u.clone()
    for n in range(2):
        P.rk4_step(a, t + n * dt, dt)
        P.rk4_step_blocks(b, t + n * dt, dt)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    assert P.last_launch_count() >= 4 * 3 * forest.nblocks
    P.close()
