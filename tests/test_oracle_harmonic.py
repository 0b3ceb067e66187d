"""Kerr in harmonic coordinates (harmonic_kerr_case, src/initialdata.jl:1300-1326), as the oracle
restates it.

SpacetimeMetrics (which defines Harmonic(M, a)) is not vendored and the reference holds no golden
value of the metric, so parity with the reference's chart rests on the properties its own tests
state: the chart is harmonic, H_a = -g^{bc} Gamma_{a,bc} = 0 to roundoff
(test/harmonic_holes_tests.jl:117-119: check_gauge_source(Harmonic(1), ...) < 1e-12), for a boost
too (a boost of a harmonic chart is harmonic, src/initialdata.jl:1313-1316); its radial coordinate
is the Kerr-Schild spheroid's with the same a, the horizon at r_H = sqrt(M^2 - a^2)
(test/tracking_tests.jl:113-130, src/initialdata.jl:1309-1312); it is a vacuum solution; and at
a = 0 it is the textbook horizon-penetrating harmonic Schwarzschild metric.
"""
import math

import numpy as np
import pytest

from test_oracle_monitors import _offset

EPS = np.finfo(float).eps
POINTS = ([2.3, 1.7, -3.1], [-1.9, 2.7, 1.3], [1.2, -0.4, 0.9], [0.3, 0.2, 1.1], [-0.9, 1.4, -0.2])


def _bg(tgh, a, v=0.0, x0=0.0):
    return tgh.harmonic_kerr_case(M=1.0, a=a, v=v, x0=x0, variant=None).config(4).bg


@pytest.mark.parametrize("a", [0.0, 0.5, 0.7, 0.9])
@pytest.mark.parametrize("v", [0.0, 0.3])
def test_the_chart_is_harmonic(oracle, tgh, a, v):
    bg = _bg(tgh, a, v, x0=0.25)
    for x in POINTS:
        g, dg = oracle.dmetric(bg, [0.37] + x)
        Hl, dHl = oracle.gauge_source_grad(bg, [0.37] + x)
        scale = max(1.0, np.abs(dg).max())
        assert np.abs(Hl).max() < 64 * EPS * scale, (a, v, x, Hl)
        assert np.abs(dHl).max() < 1e-11 * scale ** 2, (a, v, x, dHl)


def test_kerr_schild_is_not_harmonic(oracle, tgh):
    # the control: the same check fails on the Kerr-Schild chart (test/harmonic_holes_tests.jl:120)
    bg = tgh.kerr_schild_case(M=1.0, a=0.7, variant=None).config(4).bg
    Hl, _ = oracle.gauge_source_grad(bg, [0.0, 1.2, -0.4, 0.9])
    assert np.abs(Hl).max() > 0.1


def test_schwarzschild_limit_is_the_closed_form(oracle, tgh):
    """a = 0: ds^2 = -(r-M)/(r+M) dt^2 + 2 (4M^2/(r+M)^2) dt dr
    + ((r+M)^2 + 4M^2)(r+3M)/(r+M)^3 dr^2 + (r+M)^2 dOmega^2 (harmonic r = areal radius - M)."""
    M = 1.0
    bg = _bg(tgh, 0.0)
    for x in POINTS:
        p = np.array(x)
        r = float(np.linalg.norm(p))
        n = p / r
        R = r + M
        ref = np.zeros((4, 4))
        ref[0, 0] = -(r - M) / (r + M)
        ref[0, 1:] = ref[1:, 0] = 4 * M * M / R ** 2 * n
        grr = (R * R + 4 * M * M) * (R + 2 * M) / R ** 3
        ref[1:, 1:] = (R * R / (r * r)) * (np.eye(3) - np.outer(n, n)) + grr * np.outer(n, n)
        g, _ = oracle.dmetric(bg, [0.0] + x)
        assert np.abs(g - ref).max() < 16 * EPS * max(1.0, np.abs(ref).max()), (x, g - ref)


@pytest.mark.parametrize("a", [0.0, 0.7])
def test_the_chart_is_a_vacuum_solution(oracle, tgh, a):
    bg = _bg(tgh, a, 0.2)
    for x in POINTS:
        g, dg, ddg = oracle.ddmetric(bg, np.array([0.3, *x]))
        out = oracle.adm_at_node(_offset(g), dg, ddg)
        scale = max(1.0, np.abs(ddg).max(), np.abs(dg).max() ** 2)
        assert np.abs(out).max() < 64 * EPS * scale, (a, x, out)


@pytest.mark.parametrize("a", [0.0, 0.5, 0.9])
def test_the_horizon_is_on_the_spheroid_r_H_equal_sqrt_M2_minus_a2(oracle, tgh, a):
    """The future horizon is the null surface r_H = sqrt(M^2 - a^2): there g^{ab} d_a r_H d_b r_H
    = 0 (the surface's normal is null), outside it is positive."""
    bg = _bg(tgh, a)
    rng = np.random.default_rng(11)
    for _ in range(6):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        for rH, sign in ((math.sqrt(1.0 - a * a), 0), (1.5, 1)):
            # the point of the spheroid r_H along direction d: x^2 + y^2 = (rH^2 + a^2) s^2, z = rH c
            s2 = d[0] ** 2 + d[1] ** 2
            lam = 1.0 / math.sqrt(s2 / (rH * rH + a * a) + d[2] ** 2 / (rH * rH))
            x = lam * d
            g, _ = oracle.dmetric(bg, [0.0, *x])
            gi = np.linalg.inv(g)
            # d r_H / d x^i = r_H (x_i r_H^2 + a^2 z delta_iz) / (r_H^4 + a^2 z^2)
            q = rH ** 4 + a * a * x[2] ** 2
            dr = np.array([0.0, rH * x[0] * rH * rH / q, rH * x[1] * rH * rH / q,
                           rH * (x[2] * rH * rH + a * a * x[2]) / q])
            nn = dr @ gi @ dr
            if sign == 0:
                assert abs(nn) < 1e-12, (a, x, nn)
            else:
                assert nn > 0.1


def test_the_case_refuses_extremal_spin_and_defaults_to_no_gauge_source(tgh):
    with pytest.raises(ValueError):
        tgh.harmonic_kerr_case(M=1.0, a=1.0)
    c = tgh.harmonic_kerr_case(M=1.0, a=0.7, v=0.1)
    assert c.gauge == "none" and c.background["kind"] == "harmonic_kerr"
    assert tgh.horizon_min_radius(1.0, 0.6, chart="harmonic") == pytest.approx(0.8)
