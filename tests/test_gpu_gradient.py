"""Gradients of the masked error against the analytic Kerr solution, by forward-mode tangents,
against central finite differences.

The study is the static spinning hole M = 1, a = 7/10 on 8 blocks of 32^3 ([-4,4]^3, 64^3
vertices), 40 plain-form FP64 RK4 steps from the analytic data plus 8 seeded perturbation modes
of amplitude 1e-5, and the loss is the masked L2 error at the end. Its gradient with respect to
rho_max, the ramp width, the damping strength, trail_ramp and the 8 amplitudes is compared with
Richardson-extrapolated central differences (steps 1e-3 and 5e-4 of each parameter): measured
agreement 2e-11 for the layer and damping parameters and 1e-9..5e-9 for the amplitudes (where
the differences' roundoff dominates); the bound asserted is 1e-6.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _study(tgh, N=32, nsteps=40):
    from tgh_b200.gradient import MaskedErrorStudy
    case = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=4.0, r0=0.8, r1=1.3, gauge="sampled")
    return MaskedErrorStudy(tgh.gh_forest(case, N, 2), q=4, nsteps=nsteps)


def test_tangent_rhs_values_and_directional_derivative(tgh):
    case = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=4.0, r0=0.8, r1=1.3, gauge="sampled")
    f = tgh.gh_forest(case, 16, 2)
    P = tgh.GHProblem(case, f, 4, margin_check=False)
    u = P.initial_state(P.statevector(), 0.0) + torch.from_numpy(tgh.perturbation(f, 1e-6, seed=3)).cuda()
    ut = torch.from_numpy(tgh.perturbation(f, 1.0, seed=7)).cuda()
    du = torch.zeros_like(u)
    P.gh_rhs(du, u, 0.0)
    du2, dut = torch.zeros_like(u), torch.zeros_like(u)
    P.tangent_rhs(du2, dut, u, ut, 0.0, "state")
    torch.cuda.synchronize()
    assert float((du - du2).abs().max()) <= 1e-13 * float(du.abs().max())
    # the tangent is the derivative: central differences converge onto it quadratically
    errs = []
    for eps in (1e-4, 1e-5):
        dp, dm = torch.zeros_like(u), torch.zeros_like(u)
        P.gh_rhs(dp, u + eps * ut, 0.0)
        P.gh_rhs(dm, u - eps * ut, 0.0)
        errs.append(float(((dp - dm) / (2 * eps) - dut).abs().max() / dut.abs().max()))
    assert errs[1] < 1e-7 and errs[1] < errs[0] / 50


def test_masked_error_gradient_matches_central_differences(tgh):
    from tgh_b200.gradient import NAMES, NOMINAL
    st = _study(tgh)
    loss, g = st.gradient(NOMINAL)
    assert np.isfinite(loss) and loss > 0.0
    assert st.loss(NOMINAL) == pytest.approx(loss, rel=1e-12)
    f1 = st.finite_differences(NOMINAL, rel=1e-3)
    f2 = st.finite_differences(NOMINAL, rel=5e-4)
    fd = (4.0 * f2 - f1) / 3.0
    for name, a, b in zip(NAMES, g, fd):
        if name == "trail_ramp":
            assert a == 0.0 and b == 0.0  # no :fitted interior: the loss does not depend on it
            continue
        assert abs(a - b) <= 1e-6 * abs(a), (name, a, b)


def test_autograd_function_returns_the_tangents(tgh):
    from tgh_b200.gradient import MaskedError, NOMINAL
    st = _study(tgh, N=16, nsteps=8)
    loss, g = st.gradient(NOMINAL)
    p = torch.tensor(NOMINAL, dtype=torch.float64, requires_grad=True)
    out = MaskedError.apply(p, st)
    (2.0 * out).backward()
    assert float(out.detach()) == loss
    assert np.array_equal(p.grad.numpy(), 2.0 * g)


def test_tangent_form_refuses_what_it_does_not_differentiate(tgh):
    c = tgh.kerr_schild_case(M=1.0, a=0.7, v=0.1, halfwidth=4.0, r0=0.8, r1=1.3, gauge="algebraic")
    f = tgh.gh_forest(c, 8, 2)
    P = tgh.GHProblem(c, f, 4, margin_check=False)
    u = P.initial_state(P.statevector(), 0.0)
    with pytest.raises(tgh._abi.TGHError, match="interior"):
        P.tangent_rk4_step(u, torch.zeros_like(u), 0.0, 0.01, "rho_max")
