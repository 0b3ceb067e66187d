"""The range projection's host side (no GPU): StateBounds refuses what cannot be a range, and the
gate helpers (test/bounds_tests.jl:154-166, 285-300)."""
import math

import pytest

GOOD = dict(alpha_min=1 / 50, alpha_max=50.0, lambda_min=1 / 100, lambda_max=1000.0, beta_max=10.0, K_max=100.0,
            r_gate=1.0)


def test_state_bounds_refuses_what_cannot_be_a_range(tgh):
    assert tgh.StateBounds(**GOOD).K_max == 100.0
    for bad in (dict(alpha_min=2.0), dict(alpha_max=0.5), dict(alpha_min=0.0), dict(lambda_min=1.5),
                dict(lambda_max=0.5), dict(beta_max=0.0), dict(K_max=0.0), dict(r_gate=0.0),
                dict(lambda_max=math.inf), dict(alpha_min=math.nan)):
        with pytest.raises(ValueError):
            tgh.StateBounds(**{**GOOD, **bad})
    assert tgh.default_bounds(M=2, r_gate=1).K_max == 50.0


def test_the_gate_sits_below_every_evolved_stencil_or_is_refused(tgh):
    case = tgh.kerr_schild_case(M=1.0, a=0.0, halfwidth=2.0, r0=0.4, r1=1.15, gauge="sampled")
    forest = tgh.gh_forest(case, 8, 2)
    q, G = 2, 2
    h, n = tgh.layer_spacing(case, forest)
    assert n > 0 and h == forest.h0
    assert tgh.default_gate(case, forest, q) == pytest.approx(1.15 - 2 * G * h)
    b = tgh.default_bounds(M=1, r_gate=tgh.default_gate(case, forest, q))
    assert tgh.check_bounds_gate(case, forest, b, q)[2] == pytest.approx(1.15 - G * h)
    with pytest.raises(ValueError, match="too shallow"):
        tgh.check_bounds_gate(case, forest, tgh.default_bounds(M=1, r_gate=1.15 - h), q)
    with pytest.raises(ValueError, match="no interior"):
        tgh.default_gate(tgh.gauge_wave_case(), tgh.gh_forest(tgh.gauge_wave_case(), 8, 2), q)
