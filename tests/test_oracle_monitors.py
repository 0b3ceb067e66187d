"""The oracle's constraint monitors pinned against the reference's known answers (no GPU).

Restates test/constraints_tests.jl: the Ricci assembly is roundoff on a vacuum solution's
analytic derivatives and O(1) off it (:63-108); the one-direction chain rule is the
three-direction one (:130-159); both monitors are exactly zero on flat space (:161-181); on a
uniform gauge wave they sit at roundoff and across a coarse-fine face they converge at order q
(:233-266); on a curved background they converge at order q (:268-293); a mask writes exact
zeros and the norms divide by the evolved volume (:295-).
"""
import math

import numpy as np
import pytest

from helpers import two_level_forest

EPS = np.finfo(float).eps
PACK = [(0, 0), (1, 0), (2, 0), (3, 0), (1, 1), (2, 1), (3, 1), (2, 2), (3, 2), (3, 3)]
ETA = np.diag([-1.0, 1.0, 1.0, 1.0])
POINTS = [(2.1, -1.3, 0.7), (3.0, 0.5, -2.2), (-1.7, 2.4, 1.1)]


def _offset(g):
    return np.array([g[a, b] - ETA[a, b] for a, b in PACK])


def _rate(hs, vals):
    return [math.log(vals[i] / vals[i + 1]) / math.log(hs[i] / hs[i + 1]) for i in range(len(vals) - 1)]


def _backgrounds(tgh):
    return [("kerr_schild", tgh.kerr_schild_case(M=1.0, a=0.7, variant=None).config(4).bg),
            ("kerr_schild_boosted", tgh.kerr_schild_case(M=1.0, a=0.7, v=0.1, variant=None,
                                                         gauge="algebraic").config(4).bg),
            ("gauge_wave", tgh.gauge_wave_case(A=0.05).config(4).bg)]


def test_adm_constraints_vanish_on_exact_vacuum_solutions(tgh, oracle):
    for name, bg in _backgrounds(tgh):
        for x in POINTS:
            g, dg, ddg = oracle.ddmetric(bg, np.array([0.3, *x]))
            out = oracle.adm_at_node(_offset(g), dg, ddg)
            scale = max(1.0, np.abs(ddg).max(), np.abs(dg).max() ** 2)
            assert np.abs(out).max() < 16 * EPS * scale, (name, x, out)


def test_the_kernels_ricci_contraction_is_the_references(tgh, oracle):
    # the GPU monitor contracts the Ricci tensor in another order (first-derivative terms, then
    # one metric component's second derivatives at a time): the same numbers to roundoff, on the
    # vacuum solutions and on arbitrary (non-solution) derivatives alike
    for name, bg in _backgrounds(tgh):
        for x in POINTS:
            g, dg, ddg = oracle.ddmetric(bg, np.array([0.3, *x]))
            scale = max(1.0, np.abs(ddg).max(), np.abs(dg).max() ** 2)
            a = oracle.adm_at_node(_offset(g), dg, ddg)
            b = oracle.adm_at_node(_offset(g), dg, ddg, streamed=True)
            assert np.abs(a - b).max() < 64 * EPS * scale, (name, x, a, b)
    rng = np.random.default_rng(7)
    for _ in range(20):
        m = rng.normal(size=(4, 4))
        g = ETA + 0.05 * (m + m.T)  # Lorentzian: g^tt < 0, spatial part positive definite
        assert np.linalg.inv(g)[0, 0] < 0 and np.linalg.eigvalsh(g[1:, 1:]).min() > 0
        dg = rng.normal(size=(4, 4, 4))
        dg = 0.5 * (dg + dg.transpose(0, 2, 1))
        ddg = rng.normal(size=(4, 4, 4, 4))
        ddg = 0.25 * (ddg + ddg.transpose(1, 0, 2, 3) + ddg.transpose(0, 1, 3, 2) + ddg.transpose(1, 0, 3, 2))
        a = oracle.adm_at_node(_offset(g), dg, ddg)
        b = oracle.adm_at_node(_offset(g), dg, ddg, streamed=True)
        assert np.abs(a - b).max() < 1e-12 * max(1.0, np.abs(a).max()), (a, b)


def test_adm_constraints_are_not_vacuous_off_the_solution(tgh, oracle):
    bg = _backgrounds(tgh)[0][1]
    g, dg, ddg = oracle.ddmetric(bg, np.array([0.3, *POINTS[0]]))
    bumped = ddg.copy()
    bumped[1, 1, 2, 2] += 0.1
    out = oracle.adm_at_node(_offset(g), dg, bumped)
    assert abs(out[0]) > 1e-3
    assert np.abs(out[1:]).max() > 1e-3


def test_one_direction_chain_rule_is_the_three_direction_one(tgh, oracle):
    for name, bg in _backgrounds(tgh):
        for x in POINTS:
            h, _, dh, _ = oracle.background_state(bg, 0.3, np.array(x))
            md = oracle.metric_derivatives(h, dh)
            mq = oracle.metric_quantities(h)
            scale = max(1.0, np.abs(dh).max())
            for i in range(3):
                al = oracle.metric_derivatives_along(h, dh[i])
                assert abs(al["dal"] - md["dal"][i]) < 64 * EPS * scale
                assert np.abs(al["dbeta"] - md["dbeta"][i]).max() < 64 * EPS * scale
                # d sqrt(gamma) and d gamma^{jk} reassemble d(alpha sqrt(gamma) gamma^{jk})
                re = (al["dal"] * mq["sqrtg"] * mq["gamu"] + mq["alpha"] * al["dsq"] * mq["gamu"]
                      + mq["alpha"] * mq["sqrtg"] * al["dgamu"])
                assert np.abs(re - md["dA"][i]).max() < 256 * EPS * scale


@pytest.mark.parametrize("q", [2, 4])
def test_both_monitors_are_exactly_zero_on_flat_space(tgh, oracle, q):
    case = tgh.minkowski_case(L=1.0, eps_ko=0.5, gamma0=1.0, gamma2=-0.5)
    O = oracle.problem(case, tgh.gh_forest(case, 8, 2), q)
    u = O.initial_state(O.statevector(), 0.0)
    d = O.diag()
    O.gh_constraint(d, u, 0.0)
    O.adm_constraint(d, u, 0.0)
    assert np.all(O.constraint_norms(d) == 0.0)


def _run(O, t):
    u = O.initial_state(O.statevector(), t)
    d = O.diag()
    O.gh_constraint(d, u, t)
    O.adm_constraint(d, u, t)
    n = O.constraint_norms(d)
    return {"gauge_l2": float(np.sqrt((n[0:4] ** 2).sum())), "ham_l2": n[8],
            "mom_l2": float(np.sqrt((n[10:13] ** 2).sum()))}


def test_uniform_gauge_wave_has_no_constraint_violation(tgh, oracle):
    # it depends on x - t alone, so the temporal and spatial truncation errors cancel
    case = tgh.gauge_wave_case(A=1 / 20, d=1.0, eps_ko=0.0, gamma0=1.0, gamma2=0.0)
    r = _run(oracle.problem(case, tgh.gh_forest(case, 16, 1), 4), 1 / 8)
    assert r["gauge_l2"] < 1e-14
    assert r["ham_l2"] < 1e-12
    assert r["mom_l2"] < 1e-14


def test_both_monitors_converge_at_order_q_across_a_coarse_fine_face(tgh, oracle):
    q = 4
    case = tgh.gauge_wave_case(A=1 / 20, d=1.0, eps_ko=0.0, gamma0=1.0, gamma2=0.0)
    rows, hs = [], []
    for N in (8, 12, 16):
        f = two_level_forest(tgh, case, N)
        assert len(f.level) == 15
        rows.append(_run(oracle.problem(case, f, q), 1 / 8))
        hs.append(1.0 / (2 * N))
    for key in ("gauge_l2", "ham_l2", "mom_l2"):
        vals = [r[key] for r in rows]
        assert min(_rate(hs, vals)) >= q - 0.25, (key, vals)
        assert vals == sorted(vals, reverse=True)
        assert vals[0] > 1e-9


def test_both_monitors_converge_at_order_q_on_a_curved_background(tgh, oracle):
    # Kerr-Schild a = 0.7 in a box off the hole (the reference's row is harmonic Kerr there)
    q = 4
    rows, hs = [], []
    for N in (8, 12, 16):
        case = tgh.cases.Case({"kind": "kerr_schild", "M": 1.0, "a": 0.7}, ((2.0, 4.0),) * 3, (False, False, False),
                              0.0, 1.0, 0.0, None, "sampled", None, 1.0)
        rows.append(_run(oracle.problem(case, tgh.gh_forest(case, N, 1), q), 0.0))
        hs.append(2.0 / N)
    for key in ("gauge_l2", "ham_l2", "mom_l2"):
        vals = [r[key] for r in rows]
        assert min(_rate(hs, vals)) >= q - 0.25, (key, vals)
        assert vals == sorted(vals, reverse=True)


def _bench_constants():
    import importlib.util
    from pathlib import Path
    spec = importlib.util.spec_from_file_location("bench_constants", Path(__file__).resolve().parent.parent / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _first_block(tgh, case, level, h):
    """A one-block problem whose block is the workload's first: same point, same spacing."""
    lo = tuple(case.box[d][0] for d in range(3))
    box = tuple((lo[d], lo[d] + 32 * h) for d in range(3))
    c = tgh.cases.Case(case.background, box, (False,) * 3, case.eps_ko, case.gamma0, case.gamma2, case.interior,
                       case.gauge, case.ks_source, case.M)
    return c, tgh.gh_forest(c, 32, 1)


def test_flop_constants_are_the_oracle_counts(tgh, oracle):
    # the numerators of the bench's rooflines, counted by the oracle at the centre of each
    # workload's first block (the static hole, the Fourier modes, the hierarchy's level-1 corner)
    bench = _bench_constants()
    ks = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=8.0, r0=0.8, r1=1.3, rho_max=4.0, variant="damped",
                              gauge="sampled", eps_ko=0.5)
    c, f = _first_block(tgh, ks, 0, 0.125)
    O = oracle.problem(c, f, 4)
    O.prepare(O.initial_state(O.statevector(), 0.0), 0.0)
    assert O.count_flops(0.0) == bench.FLOP_PER_POINT_RHS["sampled"]
    assert O.count_flops(0.0, "gauge") == bench.FLOP_PER_POINT_MONITORS["gauge"]["sampled"]
    assert O.count_flops(0.0, "adm") == bench.FLOP_PER_POINT_MONITORS["adm"]["sampled"]
    fm = tgh.perturbed_minkowski_case()
    f = tgh.gh_forest(fm, 32, 2)
    O = oracle.problem(fm, f, 4)
    O.prepare(O.initial_state(O.statevector(), 0.0) + tgh.perturbation(f, amplitude=1e-4), 0.0)
    assert O.count_flops(0.0) == bench.FLOP_PER_POINT_RHS["none"]
    assert O.count_flops(0.0, "gauge") == bench.FLOP_PER_POINT_MONITORS["gauge"]["none"]
    assert O.count_flops(0.0, "adm") == bench.FLOP_PER_POINT_MONITORS["adm"]["none"]
    hk = tgh.kerr_schild_case(M=1.0, a=0.7, v=0.1, halfwidth=40.0, r0=0.8, r1=1.3, rho_max=4.0, variant="damped",
                              gauge="algebraic", eps_ko=0.5)
    c, f = _first_block(tgh, hk, 1, 80.0 / 128 / 2)
    O = oracle.problem(c, f, 4)
    O.prepare(O.initial_state(O.statevector(), 0.0), 0.0)
    assert O.count_flops(0.0, "gauge") == bench.FLOP_PER_POINT_MONITORS["gauge"]["algebraic"]
    assert O.count_flops(0.0, "adm") == bench.FLOP_PER_POINT_MONITORS["adm"]["algebraic"]


@pytest.mark.parametrize("periodic", [True, False])
def test_the_norms_count_each_lattice_point_once(tgh, oracle, periodic):
    # A block holds both face planes; the fold reads every point at its primary copy, the
    # lower face's, and on a periodic axis the top block's upper face is the bottom block's
    # lower face. An indicator of every block's upper x face therefore has L2 = 0 on a
    # periodic mesh, and not on a Dirichlet one, whose top blocks own their upper faces.
    if periodic:
        case = tgh.gauge_wave_case()
    else:
        case = tgh.cases.Case({"kind": "minkowski"}, ((0.0, 1.0),) * 3, (False, False, False), 0.0, 0.0, 0.0)
    f = tgh.gh_forest(case, 8, 2)
    O = oracle.problem(case, f, 4)
    d = O.diag().reshape(len(f.level), 10, 9, 9, 9)
    d[:, 8] = 1.0
    d[:, 0, :, :, 8] = 1.0
    n = O.constraint_norms(d.ravel(), weighting="points")
    if periodic:
        assert n[0] == 0.0 and n[4] == 0.0
    else:
        # the domain's upper x plane, 17 x 17 points once each (the four top blocks share
        # their edges there), among 17^3 points
        assert abs(n[0] - math.sqrt(17 ** 2 / 17 ** 3)) < 1e-15 and n[4] == 1.0


def test_the_mask_writes_exact_zeros_and_the_norms_divide_by_the_evolved_volume(tgh, oracle):
    case = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=2.0, r0=0.8, r1=1.3, gauge="sampled")
    f = tgh.gh_forest(case, 8, 2)
    O = oracle.problem(case, f, 4)
    u = O.initial_state(O.statevector(), 0.0)
    d = O.diag()
    O.gh_constraint(d, u, 0.0)
    O.adm_constraint(d, u, 0.0)
    S = 9 ** 3
    dd = d.reshape(len(f.level), 10, S)[:, :9]
    h = f.h0
    idx = np.arange(S)
    i, j, k = idx % 9, (idx // 9) % 9, idx // 81
    masked = 0
    for b in range(len(f.level)):
        c = f.corner[b]
        x = np.stack([f.lo[0] + (c[0] + i) * h, f.lo[1] + (c[1] + j) * h, f.lo[2] + (c[2] + k) * h])
        inside = np.sqrt((x ** 2).sum(0)) < 1.3
        assert np.all(dd[b, :, inside] == 0.0)
        assert np.all(dd[b, 8, ~inside] == 1.0)
        masked += int(inside.sum())
    assert masked > 0
    n_int = O.constraint_norms(d)
    # every point evolved: the interior's values enter and the volume grows
    d_all = O.diag()
    O.gh_constraint(d_all, u, 0.0, allpoints=True)
    O.adm_constraint(d_all, u, 0.0, allpoints=True)
    n_all = O.constraint_norms(d_all)
    assert np.all(np.isfinite(n_all))
    assert n_all[9] > n_int[9]  # the layer and core's Hamiltonian constraint is larger
    # points weighting: the same sums over a count instead of a volume (one level, so the
    # two differ by h^3 in the volume and cancel in the ratio)
    n_pts = O.constraint_norms(d, weighting="points")
    assert np.allclose(n_pts, n_int, rtol=1e-13, atol=0.0)
