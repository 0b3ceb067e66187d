"""Size-independent properties of the CUDA path: exact zeros on flat space, purity and
repeatability, the dissipation switch, convergence at order q (the reference's convergence
oracle, test/convergence_tests.jl:37-136), and the full-size Fourier-mode workload."""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _gh_errors(tgh, case, N, roots, q, t_end, cfl=0.25, batched=False):
    f = tgh.gh_forest(case, N, roots)
    P = tgh.GHProblem(case, f, q)
    u = P.initial_state(P.statevector(), 0.0)
    dt = P.gh_dt(u, cfl, 0.0)
    n = max(1, math.ceil(t_end / dt))
    P.gh_solve(u, (0.0, t_end), t_end / n, batched=batched)
    l2, li = P.error_norm(u, t_end)
    return f.h0, l2, li, n


def _rate(hs, es):
    x, y = np.log(hs), np.log(es)
    return float(np.sum((x - x.mean()) * (y - y.mean())) / np.sum((x - x.mean()) ** 2))


@pytest.mark.parametrize("q", [2, 4, 6])
def test_minkowski_is_exactly_stationary(tgh, q):
    N = 10 if q == 6 else 8
    c = tgh.minkowski_case(L=1.0, eps_ko=0.5, gamma0=1.0, gamma2=-0.5)
    P = tgh.GHProblem(c, tgh.gh_forest(c, N, 2), q)
    u = P.initial_state(P.statevector(), 0.0)
    assert torch.count_nonzero(u).item() == 0
    du = torch.full_like(u, float("nan"))
    P.gh_rhs(du, u, 3 / 7)
    assert torch.count_nonzero(du).item() == 0
    for _ in range(3):
        P.rk4_step(u, 0.0, 0.01)
    P.step_batched(u, 0.03, 0.01, 3)
    assert torch.count_nonzero(u).item() == 0


def test_rhs_is_pure_and_repeatable(tgh):
    c = tgh.shifted_minkowski_case(eps_ko=0.5, gamma0=1.0, gamma2=-0.5)
    P = tgh.GHProblem(c, tgh.gh_forest(c, 8, 1), 4)
    u = P.initial_state(P.statevector(), 0.0)
    u0 = u.clone()
    d1, d2 = torch.empty_like(u), torch.empty_like(u)
    P.gh_rhs(d1, u, 1 / 8)
    P.gh_rhs(d2, u, 1 / 8)
    assert torch.equal(u, u0) and torch.equal(d1, d2)
    assert torch.count_nonzero(d1).item() > 0 and bool(torch.isfinite(d1).all())


def test_dissipation_switch(tgh):
    out = []
    for eps in (0.0, 1e-300):
        c = tgh.gauge_wave_case(eps_ko=eps, gamma0=1.0, gamma2=0.0)
        P = tgh.GHProblem(c, tgh.gh_forest(c, 8, 1), 4)
        u = P.initial_state(P.statevector(), 0.0)
        du = torch.empty_like(u)
        P.gh_rhs(du, u, 0.0)
        out.append(du)
    a, b = out
    assert bool((torch.abs(a - b) <= 64 * 2.2e-16 * torch.abs(a) + 1e-290).all())


@pytest.mark.parametrize("q", [2, 4, 6])
def test_gauge_wave_converges_at_order_q(tgh, q):
    N = 10 if q == 6 else 8
    c = tgh.gauge_wave_case(A=1 / 20, d=1.0, eps_ko=0.0, gamma0=1.0, gamma2=0.0)
    res = [_gh_errors(tgh, c, N, r, q, 1 / 8) for r in (1, 2, 3)]
    hs = [r[0] for r in res]
    l2 = [r[1] for r in res]
    li = [r[2] for r in res]
    assert _rate(hs, l2) >= q - 0.25 and _rate(hs, li) >= q - 0.25
    assert l2 == sorted(l2, reverse=True) and l2[-1] > 1e-12


def test_dissipation_keeps_the_order(tgh):
    c = tgh.gauge_wave_case(A=1 / 20, d=1.0, eps_ko=0.5, gamma0=1.0, gamma2=-0.5)
    res = [_gh_errors(tgh, c, 8, r, 4, 1 / 8, batched=True) for r in (1, 2, 3)]
    assert _rate([r[0] for r in res], [r[1] for r in res]) >= 3.75


def test_shifted_minkowski_converges_through_a_dirichlet_face(tgh):
    c = tgh.shifted_minkowski_case(A=0.5, w=2.0, halfwidth=2.0, eps_ko=0.0, gamma0=1.0, gamma2=0.0)
    res = [_gh_errors(tgh, c, 8, r, 4, 1 / 4) for r in (2, 3, 4)]
    assert _rate([r[0] for r in res], [r[1] for r in res]) >= 3.75


def test_fourier_workload_full_size(tgh):
    """8 blocks of 32^3 on [-1,1]^3: batched = plain after settle; Minkowski speed bound."""
    c = tgh.perturbed_minkowski_case()
    f = tgh.gh_forest(c, 32, 2)
    P = tgh.GHProblem(c, f, 4)
    u0 = P.initial_state(P.statevector(), 0.0)
    u0 += torch.from_numpy(tgh.perturbation(f, amplitude=1e-4)).cuda()
    dt = 0.25 * f.h0
    a, b = u0.clone(), u0.clone()
    for n in range(2):
        P.rk4_step(a, n * dt, dt)
    P.step_batched(b, 0.0, dt, 2)
    P.settle(a, 2 * dt)
    P.settle(b, 2 * dt)
    assert torch.max(torch.abs(a - b)).item() < 1e-15
    assert torch.max(torch.abs(a - u0)).item() > 1e-8
    lam = P.max_speed(a, 2 * dt)
    assert abs(lam - math.sqrt(3.0)) < 1e-2
