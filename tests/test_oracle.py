"""The CPU oracle pinned against the reference's golden vectors and known answers.

Mirrors test/stencils_tests.jl, test/evolution_tests.jl (host_rhs_at, Minkowski, the
epsilon switch, the Dirichlet hook, the CFL speed), test/pointwise_identity_tests.jl and
test/gauge_source_tests.jl of the reference, run on the oracle (no GPU).
"""
import json
import math
from fractions import Fraction
from pathlib import Path

import numpy as np
import pytest

PINS = json.loads((Path(__file__).parent / "golden" / "reference_pins.json").read_text())


@pytest.mark.parametrize("q", [2, 4, 6, 8])
def test_derivative_weights_are_the_textbook_tables(oracle, q):
    assert oracle.weights(q, 1) == [tuple(x) for x in PINS["FD1_TABLE"][str(q)]]
    assert oracle.weights(q, 2) == [tuple(x) for x in PINS["FD2_TABLE"][str(q)]]


@pytest.mark.parametrize("r", [2, 3, 4, 5])
def test_dissipation_weights_are_the_textbook_tables(oracle, r):
    assert oracle.weights(r, 0) == [tuple(x) for x in PINS["KO_TABLE"][str(r)]]


@pytest.mark.parametrize("r", [2, 3, 4, 5])
def test_dissipation_damps_the_nyquist_mode_at_exactly_one(oracle, r):
    # src/stencils.jl:254-265: on u_j = (-1)^j the contraction is -sin^{2r}(pi/2) u = -u
    w = [Fraction(n, d) for n, d in oracle.weights(r, 0)]
    s = sum(wj * (-1) ** abs(j - r) for j, wj in enumerate(w))  # the mode is 1 at the center
    assert s == -1
    assert w[r] < 0
    assert sum(w) == 0


@pytest.mark.parametrize("q", [2, 4, 6, 8])
def test_derivative_orders(oracle, q):
    # exact on polynomials of degree <= q (first) and <= q+1 (second), not beyond
    r = q // 2
    for m, exact_deg in ((1, q), (2, q + 1)):
        w = [Fraction(n, d) for n, d in oracle.weights(q, m)]
        for deg in range(exact_deg + 2):
            approx = sum(wj * Fraction(j - r) ** deg for j, wj in enumerate(w))
            true = Fraction(math.factorial(deg), math.factorial(deg - m)) * 0 ** (deg - m) if deg >= m else 0
            if deg <= exact_deg:
                assert approx == true
            elif deg == exact_deg + 1:
                assert approx != true


def test_weights_round_once(oracle):
    for q in (2, 4, 6, 8):
        for m in (1, 2):
            exact = [n / d for n, d in oracle.weights(q, m)]
            assert list(oracle.weights_double(q, m)) == exact


def test_kerr_schild_coefficients_at_one_and_a_half_M(oracle, tgh):
    pin = PINS["kerr_schild_a0_r1.5"]
    bg = tgh.kerr_schild_case(M=1.0, a=0.0).config(4).bg
    h, _, _, _ = oracle.background_state(bg, 0.0, [pin["r"], 0.0, 0.0])
    mq = oracle.metric_quantities(h)
    b = mq["beta"][0]
    a = mq["alpha"] * math.sqrt(mq["gamu"][0, 0])
    assert round(b, 3) == pin["b"] and round(a, 3) == pin["a"]
    assert abs(b - 4 / 7) < 1e-15 and abs(a - 3 / 7) < 1e-15


def test_box_corner_speed_of_the_static_hole(oracle, tgh):
    pin = PINS["box_corner_speed"]
    bg = tgh.kerr_schild_case(M=1.0, a=0.0).config(4).bg
    hw = pin["halfwidth"]
    h, _, _, _ = oracle.background_state(bg, 0.0, [hw, hw, hw])
    mq = oracle.metric_quantities(h)
    lam = mq["alpha"] * math.sqrt(np.trace(mq["gamu"])) + np.linalg.norm(mq["beta"])
    assert round(lam, pin["digits"]) == pin["lambda"]


def test_flat_speed_is_sqrt3(oracle, tgh):
    case = tgh.minkowski_case(L=1.0)
    f = tgh.gh_forest(case, 8, 2)
    P = oracle.problem(case, f, 4)
    u = P.initial_state(P.statevector(), 0.0)
    st, lam = P.max_speed(u, 0.0)
    assert st == 0 and lam == pytest.approx(math.sqrt(3.0), rel=1e-15)


@pytest.mark.parametrize("v", [0.0, 0.1])
def test_algebraic_gauge_source_is_the_background_source(oracle, tgh, v):
    # check_gauge_source (src/gauge.jl:381): the closed form reproduces H_a = -Gamma_a, 1e-9
    case = tgh.kerr_schild_case(M=1.0, a=0.7, v=v, gauge="algebraic")
    bg = case.config(4).bg
    for x in ([2.3, 1.7, -3.1], [-1.9, 2.7, 1.3], [3.7, -2.1, 0.9]):
        t = 0.37
        Hs, dHs = oracle.gauge_source_grad(bg, [t] + x)
        h, Pi, dh, dtg = oracle.background_state(bg, t, x)
        Ha, dHa = oracle.algebraic_gauge_source(1.0, [0, 0, 0.7], [v, 0, 0], h, dtg, dh)
        assert np.max(abs(Hs - Ha)) < 1e-9 and np.max(abs(dHs - dHa)) < 1e-9


def test_source_spellings_agree_to_roundoff(oracle):
    # test/pointwise_identity_tests.jl: the lean kernel spelling equals the reference spelling
    rng = np.random.default_rng(7)
    for _ in range(20):
        h = 0.2 * rng.standard_normal(10)
        dth, dh = rng.standard_normal(10), rng.standard_normal(30)
        Hl, dHl = rng.standard_normal(4), rng.standard_normal(16)
        a = oracle.source(0, h, dth, dh, Hl, dHl, 0.7, -0.3)
        b = oracle.source(1, h, dth, dh, Hl, dHl, 0.7, -0.3)
        assert np.max(abs(a - b)) <= 1e-13 * max(1.0, np.max(abs(b)))
        d0 = oracle.divergences(0, h, dh)
        d1 = oracle.divergences(1, h, dh)
        assert np.max(abs(d0 - d1)) <= 1e-13 * max(1.0, np.max(abs(d1)))


@pytest.mark.parametrize("q", [2, 4, 6])
@pytest.mark.parametrize("eps", [0.0, 0.5])
def test_minkowski_rhs_is_exactly_zero(oracle, tgh, q, eps):
    N = 10 if q == 6 else 8
    case = tgh.minkowski_case(L=1.0, eps_ko=eps, gamma0=1.0, gamma2=-0.5)
    P = oracle.problem(case, tgh.gh_forest(case, N, 2), q)
    u = P.initial_state(P.statevector(), 0.0)
    assert np.all(u == 0)
    du = np.full(P.L, np.nan)
    P.gh_rhs(du, u, 3 / 7)
    assert np.all(du == 0)


def _stream_vs_expanded(oracle, tgh, case, q, N, roots, t=0.25):
    f = tgh.gh_forest(case, N, roots)
    P = oracle.problem(case, f, q)
    u = P.initial_state(P.statevector(), t)
    du = np.zeros(P.L)
    P.gh_rhs(du, u, t)
    N1, S = N + 1, (N + 1) ** 3
    worst = 0.0
    for b in range(f.nblocks):
        for (i, j, k) in ((0, 0, 0), (1, N // 2 - 1, N - 1), (N - 1, N - 1, N - 1), (N // 2 - 1, 2, N - 2), (N, N, N)):
            ref = P.host_rhs_at(b, i, j, k, t)
            got = du[b * 20 * S + i + N1 * (j + N1 * k) + S * np.arange(20)]
            worst = max(worst, np.max(abs(got - ref)) / P.rhs_scale(b, i, j, k))
    return worst


@pytest.mark.parametrize("q,eps,which", [(2, 0.5, "gw"), (4, 0.0, "gw"), (4, 0.5, "gw"), (6, 0.5, "gw"),
                                         (4, 0.0, "shifted"), (4, 0.5, "shifted"), (4, 0.0, "ks"), (4, 0.5, "ks")])
def test_streaming_rhs_is_the_expanded_equation(oracle, tgh, q, eps, which):
    # test/evolution_tests.jl:141-179: kernel = host_rhs_at to < 1e-12 of rhs_scale
    N = 10 if q == 6 else 8
    if which == "gw":
        case, roots = tgh.gauge_wave_case(eps_ko=eps, gamma0=1.0, gamma2=-0.5), 2
    elif which == "shifted":
        case, roots = tgh.shifted_minkowski_case(eps_ko=eps, gamma0=1.0, gamma2=-0.5), 1
    else:
        case = tgh.kerr_schild_case(M=1.0, a=0.9, variant=None, gauge="sampled", eps_ko=eps, gamma0=1.0,
                                    gamma2=-0.5)
        case.box, roots = ((2.0, 4.0),) * 3, 1
    assert _stream_vs_expanded(oracle, tgh, case, q, N, roots) < 1e-12


def test_dissipation_switch_is_exactly_zero(oracle, tgh):
    # test/evolution_tests.jl:322-360
    out = []
    for eps in (0.0, 1e-300):
        case = tgh.gauge_wave_case(eps_ko=eps, gamma0=1.0, gamma2=0.0)
        P = oracle.problem(case, tgh.gh_forest(case, 8, 1), 4)
        u = P.initial_state(P.statevector(), 0.0)
        du = np.zeros(P.L)
        P.gh_rhs(du, u, 0.0)
        out.append(du)
    assert np.all(abs(out[0] - out[1]) <= 64 * np.finfo(float).eps * abs(out[0]) + 1e-290)


def test_dirichlet_ghosts_are_the_analytic_state(oracle, tgh):
    # test/evolution_tests.jl:239-288: a moving background, the hook built at t
    case = tgh.gauge_wave_case(A=1 / 20, d=2.0)
    case.periodic = (False, False, False)
    f = tgh.gh_forest(case, 8, 1)
    P = oracle.problem(case, f, 4)
    t = 1 / 3
    u = P.initial_state(P.statevector(), t)
    P.prepare(u, t)
    G, W = 3, 8 + 2 * 3 + 1
    w = P.work().reshape(20, W, W, W)
    worst = 0.0
    for (i, j, k) in ((0, 4, 4), (1, 4, 4), (G - 1, 4, 4), (4, 0, 4), (4, 4, 1), (8 + G, 4, 4), (4, 8 + 2 * G, 4)):
        x = [f.lo[d] + (idx - G) * f.h0 for d, idx in enumerate((i, j, k))]
        h, Pi, _, _ = oracle.background_state(case.config(4).bg, t, x)
        worst = max(worst, np.max(abs(w[:, k, j, i] - np.concatenate([h, Pi]))))
    assert worst == 0.0
    h0, _, _, _ = oracle.background_state(case.config(4).bg, 0.0, [f.lo[0] - G * f.h0, 0.25, 0.25])
    h1, _, _, _ = oracle.background_state(case.config(4).bg, t, [f.lo[0] - G * f.h0, 0.25, 0.25])
    assert np.max(abs(h1 - h0)) > 1e-2


def test_rk4_step_of_minkowski_stays_zero(oracle, tgh):
    case = tgh.minkowski_case(L=1.0, eps_ko=0.5, gamma0=1.0)
    P = oracle.problem(case, tgh.gh_forest(case, 8, 2), 4)
    u = P.initial_state(P.statevector(), 0.0)
    P.rk4_step(u, 0.0, 0.01)
    assert np.all(u == 0)


def test_nonfinite_state_is_refused(oracle, tgh):
    case = tgh.minkowski_case(L=1.0)
    P = oracle.problem(case, tgh.gh_forest(case, 8, 1), 4)
    u = P.initial_state(P.statevector(), 0.0)
    u[123] = np.nan
    st, _ = P.max_speed(u, 0.0)
    assert st == 2  # TGH_ERR_NONFINITE
