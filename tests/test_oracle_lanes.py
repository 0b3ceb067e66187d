"""The oracle's right-hand side on SIMD lanes (the restatement of the reference's CPU kernel on
SIMD.jl's Vec{W,T}, src/lanes.jl, gh_rhs_lanes! src/evolution.jl:698-790) against the point-by-point
evaluation. With no contraction into fused multiply-adds each lane does its point's scalar
operations, so the two agree bit for bit (the reference states bit for bit on the gauge wave and
an eps of the terms on a hole, where its compiler fuses products differently in the two
contexts): without a hole, with a hole whose layer a group straddles (those groups fall back to
point by point), with the sampled and the algebraic gauge source, and on the harmonic chart. Both
builds run where the host has them: AVX2 (4 lanes) and AVX-512 (8 lanes)."""
import numpy as np
import pytest

from oracle_binding import Oracle, host_has_avx512


def _builds():
    out = [("avx2", Oracle.load)]
    if host_has_avx512():
        out.append(("avx512", Oracle.load_widest))
    return out


def _cases(tgh):
    c = tgh.gauge_wave_case(eps_ko=0.5, gamma0=1.0, gamma2=-0.5)
    yield "gauge_wave", c, tgh.gh_forest(c, 16, 2), 0.25
    c = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=2.0, r0=0.8, r1=1.3, gauge="sampled")
    yield "kerr_schild_sampled", c, tgh.gh_forest(c, 8, 2), 0.0
    c = tgh.kerr_schild_case(M=1.0, a=0.7, v=0.1, halfwidth=2.0, r0=0.8, r1=1.3, gauge="algebraic",
                             eps_ko={"eps_out": 0.5, "eps_in": 2.0, "r_1": 1.3, "r_h": 1.7, "c0": (0, 0, 0)})
    yield "kerr_schild_moving_horizon_dissipation", c, tgh.gh_forest(c, 8, 2), 0.3
    c = tgh.harmonic_kerr_case(M=1.0, a=0.7, halfwidth=2.0, r0=0.9, r1=1.4)
    yield "harmonic_kerr", c, tgh.gh_forest(c, 16, 2), 0.0


@pytest.mark.parametrize("build", [b for b, _ in _builds()])
def test_lanes_are_the_scalar_rhs_bit_for_bit(tgh, build):
    O = dict(_builds())[build]()
    for name, case, forest, t in _cases(tgh):
        P = O.problem(case, forest, 4)
        u = P.initial_state(P.statevector(), t) + tgh.perturbation(forest, amplitude=1e-6, seed=3)
        ref = np.zeros(P.L)
        assert P.set_simd_width(1) == 1
        P.gh_rhs(ref, u, t)
        got = np.full(P.L, np.nan)
        assert P.set_simd_width(O.lanes()) == O.lanes()
        P.gh_rhs(got, u, t)
        assert np.array_equal(got, ref), (build, name, np.nanmax(np.abs(got - ref)))


def test_the_lane_counts_are_the_builds(oracle):
    assert oracle.lanes() == 4
    if host_has_avx512():
        assert Oracle.load_widest().lanes() == 8
