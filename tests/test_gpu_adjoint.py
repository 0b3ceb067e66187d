"""The reverse-mode adjoint of the plain form against the tangent-linear form and against finite
differences.

An adjoint is checked by the transpose identity <lam, J v> = <J^T lam, v> on random lam and v,
with J v from the tangent-linear form (itself checked against central differences in
test_gpu_gradient.py): for the right-hand side (one level, and two levels, where the fill's
prolongation is transposed too), for one RK4 step, and for the parameters' directions. The
checkpointed sweep of the C5 study (8 blocks of 32^3, 40 steps, a checkpoint every 8) then gives
the masked error's gradient, compared with the 12 tangent-linear runs and with central
differences; and the gradient with respect to the whole initial state, through the
torch.autograd.Function, with a directional difference."""
import numpy as np
import pytest
import torch

from helpers import two_level_forest

pytestmark = pytest.mark.gpu

PARAMS = ("rho_max", "ramp", "damp_near")


def _hole(tgh, N=16):
    case = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=4.0, r0=0.8, r1=1.3, gauge="sampled")
    return case, tgh.gh_forest(case, N, 2)


def _rand(u, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    return torch.randn(u.shape, dtype=torch.float64, device="cuda", generator=g)


def _dot(a, b):
    return float(torch.dot(a, b))


@pytest.mark.parametrize("mesh", ["hole", "two_level"])
def test_adjoint_rhs_is_the_transpose_of_the_tangent(tgh, mesh):
    if mesh == "hole":
        case, f = _hole(tgh)
    else:
        case = tgh.gauge_wave_case(eps_ko=0.5, gamma0=1.0, gamma2=-0.5)
        f = two_level_forest(tgh, case, N=8)
    P = tgh.GHProblem(case, f, 4, margin_check=False)
    u = P.initial_state(P.statevector(), 0.1) + 1e-6 * _rand(P.statevector(), 1)
    v, lam = _rand(u, 2), _rand(u, 3)
    du, dut = torch.zeros_like(u), torch.zeros_like(u)
    P.tangent_rhs(du, dut, u, v, 0.1, "state")
    lam_u, th = P.adjoint_rhs(u, 0.1, lam)
    a, b = _dot(lam, dut), _dot(lam_u, v)
    assert abs(a - b) <= 1e-11 * max(abs(a), abs(b)), (a, b)
    if mesh == "hole":
        for k, name in enumerate(PARAMS):
            P.tangent_rhs(du, dut, u, torch.zeros_like(u), 0.1, name)
            a = _dot(lam, dut)
            assert abs(a - th[k]) <= 1e-11 * max(abs(a), 1e-300), (name, a, th[k])
    P.close()


def test_adjoint_rk4_step_is_the_transpose_of_the_tangent_step(tgh):
    case, f = _hole(tgh)
    P = tgh.GHProblem(case, f, 4, margin_check=False)
    u0 = P.initial_state(P.statevector(), 0.0) + 1e-6 * _rand(P.statevector(), 4)
    v, lam = _rand(u0, 5), _rand(u0, 6)
    dt = 0.25 * f.h0 / 2
    u, ut = u0.clone(), v.clone()
    P.tangent_rk4_step(u, ut, 0.0, dt, "state")
    lam0 = lam.clone()
    th = [0.0, 0.0, 0.0]
    P.adjoint_rk4_step(u0, 0.0, dt, lam0, th)
    a, b = _dot(lam, ut), _dot(lam0, v)
    assert abs(a - b) <= 1e-11 * max(abs(a), abs(b)), (a, b)
    for k, name in enumerate(PARAMS):
        u, ut = u0.clone(), torch.zeros_like(u0)
        P.tangent_rk4_step(u, ut, 0.0, dt, name)
        a = _dot(lam, ut)
        assert abs(a - th[k]) <= 1e-11 * max(abs(a), 1e-300), (name, a, th[k])
    P.close()


def _study(tgh, N=32, nsteps=40):
    from tgh_b200.gradient import MaskedErrorStudy
    case = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=4.0, r0=0.8, r1=1.3, gauge="sampled")
    return MaskedErrorStudy(tgh.gh_forest(case, N, 2), q=4, nsteps=nsteps)


def test_adjoint_gradient_matches_tangents_and_differences(tgh):
    """C5: 40 steps, a checkpoint every 8; the adjoint's 12 derivatives equal the tangent-linear
    runs' to 1e-9 and central differences to 1e-6; a checkpoint every 3 steps changes nothing."""
    from tgh_b200.gradient import NAMES, NOMINAL
    st = _study(tgh)
    loss_a, ga, lam = st.gradient_adjoint(NOMINAL, every=8)
    loss_t, gt = st.gradient(NOMINAL)
    assert loss_a == pytest.approx(loss_t, rel=1e-13)
    for name, a, b in zip(NAMES, ga, gt):
        if name == "trail_ramp":
            assert a == 0.0 and b == 0.0
            continue
        assert abs(a - b) <= 1e-9 * abs(b), (name, a, b)
    for k in (0, 2, 7):  # rho_max, damp_near, a3: Richardson-extrapolated central differences
        f1 = st.finite_differences(NOMINAL, rel=1e-3, i=k)[k]
        f2 = st.finite_differences(NOMINAL, rel=5e-4, i=k)[k]
        fd = (4.0 * f2 - f1) / 3.0
        assert abs(ga[k] - fd) <= 1e-6 * abs(ga[k]), (NAMES[k], ga[k], fd)
    _, g3, lam3 = st.gradient_adjoint(NOMINAL, every=3)
    assert float((lam3 - lam).abs().max()) <= 1e-12 * float(lam.abs().max())
    assert np.allclose(g3, ga, rtol=1e-12, atol=0.0)


def test_state_gradient_through_autograd(tgh):
    """The gradient with respect to every value of the initial state, from the autograd Function,
    along a random direction against a central difference of the loss."""
    from tgh_b200.adjoint import MaskedErrorOfState
    case, f = _hole(tgh)
    P = tgh.GHProblem(case, f, 4, margin_check=False)
    u0 = P.initial_state(P.statevector(), 0.0) + 1e-5 * _rand(P.statevector(), 7)
    dt, n = 0.25 * f.h0 / 2, 6
    x = u0.clone().requires_grad_(True)
    loss = MaskedErrorOfState.apply(x, P, 0.0, dt, n, 2)
    loss.backward()
    d = _rand(u0, 8)
    d = d / float(d.norm())

    def L(y):
        y = y.clone()
        for k in range(n):
            P.rk4_step(y, k * dt, dt)
        return P.error_norm(y, n * dt)[0]

    eps = 1e-6 * float(u0.norm()) / np.sqrt(u0.numel())
    fd = (L(u0 + eps * d) - L(u0 - eps * d)) / (2 * eps)
    g = _dot(x.grad, d)
    assert abs(g - fd) <= 1e-6 * abs(g), (g, fd)
    P.close()
