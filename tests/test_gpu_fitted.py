"""The :fitted interior and its target cache (src/evolution.jl:517-548, 600-653; src/fit.jl:1030-1285)
against the oracle, over the sphere interior.

The layer and the core relax toward A + (t - t_f) S read from a 40-field cache, with the cache's
slope fed forward under target_rate. Checked: the right-hand side with an arbitrary cache (the
analytic state plus seeded noise, a random slope, t away from t_f) within 1e-12 of rhs_scale, with
and without the rate, on Kerr-Schild and harmonic Kerr; the fills (snapshot, analytic with its
centred-difference slope) and the fitted initial data bit for bit; the analytic cache of a resting
hole turning the :fitted layer into the :damped one bit for bit; one RK4 step, plain and batched;
and the refusal of a step before the cache is filled.
"""
import numpy as np
import pytest
import torch

from helpers import rhs_error, rhs_scale

pytestmark = pytest.mark.gpu


def _to_gpu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _case(tgh, chart, rate, v=0.0):
    mk = tgh.harmonic_kerr_case if chart == "harmonic" else tgh.kerr_schild_case
    kw = {} if chart == "harmonic" else {"gauge": "algebraic"}
    r0, r1 = (0.9, 1.4) if chart == "harmonic" else (0.8, 1.3)
    return mk(M=1.0, a=0.7, v=v, halfwidth=2.0, r0=r0, r1=r1, variant="fitted", target_rate=rate, **kw)


def _cache(tgh, P, O, forest, seed):
    """The analytic fill at t_f = 0.2 plus noise in A and a random slope, set on both sides."""
    O.fill_target_analytic(0.2, P.default_fill_radius(), 0.0)
    tw = O.target().reshape(forest.nblocks, 40, -1)
    rng = np.random.default_rng(seed)
    inside = np.any(tw[:, :20] != 0.0, axis=1, keepdims=True)
    tw[:, :20] += 1e-3 * rng.standard_normal(tw[:, :20].shape) * inside
    tw[:, 20:] = 0.05 * rng.standard_normal(tw[:, 20:].shape) * inside
    tw = tw.reshape(-1)
    O.set_target(tw, 0.2)
    P.set_target(_to_gpu(tw), 0.2)
    return tw


@pytest.mark.parametrize("chart", ["kerr_schild", "harmonic"])
@pytest.mark.parametrize("rate", [False, True])
def test_fitted_rhs_matches_oracle(tgh, oracle, chart, rate):
    case = _case(tgh, chart, rate)
    f = tgh.gh_forest(case, 8, 2)
    P = tgh.GHProblem(case, f, 4, margin_check=False)
    O = oracle.problem(case, f, 4)
    _cache(tgh, P, O, f, seed=3)
    t = 0.35
    u = O.initial_state(O.statevector(), t) + tgh.perturbation(f, amplitude=1e-6, seed=11)
    du_ref = np.zeros(O.L)
    O.gh_rhs(du_ref, u, t)
    dug = torch.full((O.L,), float("nan"), dtype=torch.float64, device="cuda")
    P.gh_rhs(dug, _to_gpu(u), t)
    du = dug.cpu().numpy()
    assert np.all(np.isfinite(du))
    err = rhs_error(du, du_ref, rhs_scale(O.work(), f, 4), f)
    assert err < 1e-12, (chart, rate, err)
    # the core and the layer do read the cache: the rate changes them
    P.close()


@pytest.mark.parametrize("dt", [0.0, 1e-3])
def test_target_fills_and_fitted_initial_state_are_the_oracles_bit_for_bit(tgh, oracle, dt):
    case = _case(tgh, "kerr_schild", True, v=0.1)
    f = tgh.gh_forest(case, 8, 2)
    P = tgh.GHProblem(case, f, 4, margin_check=False)
    O = oracle.problem(case, f, 4)
    r_fill = P.default_fill_radius()
    P.fill_target_analytic(0.3, r_fill, dt)
    O.fill_target_analytic(0.3, r_fill, dt)
    assert np.array_equal(P.target().cpu().numpy(), O.target())
    for d_init in (0.0, 0.2):
        u = P.fitted_initial_state(P.statevector(), 0.31, d_init)
        uo = O.fitted_initial_state(O.statevector(), 0.31, d_init)
        assert np.array_equal(u.cpu().numpy(), uo), d_init
    us = O.initial_state(O.statevector(), 0.3) + tgh.perturbation(f, amplitude=1e-6, seed=2)
    P.fill_target_snapshot(_to_gpu(us), 0.3, r_fill)
    O.fill_target_snapshot(us, 0.3, r_fill)
    got = P.target().cpu().numpy()
    assert np.array_equal(got, O.target())
    tw = got.reshape(f.nblocks, 40, -1)
    assert np.all(tw[:, 20:] == 0.0)
    assert np.count_nonzero(tw[:, :20]) > 0
    P.close()


def test_analytic_cache_makes_the_fitted_layer_the_damped_one(tgh):
    """A resting hole, the cache filled from the analytic state with no slope: the :fitted layer
    relaxes toward exactly the :damped layer's target, so the evolved region and the layer agree
    bit for bit; in the core :damped is frozen (du = 0) and :fitted relaxes at rho_max."""
    kw = dict(M=1.0, a=0.7, halfwidth=2.0, r0=0.8, r1=1.3, gauge="algebraic")
    cf, cd = tgh.kerr_schild_case(variant="fitted", **kw), tgh.kerr_schild_case(variant="damped", **kw)
    f = tgh.gh_forest(cf, 8, 2)
    Pf = tgh.GHProblem(cf, f, 4, margin_check=False)
    Pd = tgh.GHProblem(cd, f, 4, margin_check=False)
    Pf.fill_target_analytic(0.0)
    u = Pd.initial_state(Pd.statevector(), 0.0)
    u += torch.from_numpy(tgh.perturbation(f, amplitude=1e-6, seed=4)).cuda()
    duf, dud = torch.zeros_like(u), torch.zeros_like(u)
    Pf.gh_rhs(duf, u, 0.0)
    Pd.gh_rhs(dud, u, 0.0)
    N1 = f.N + 1
    x = np.stack(np.meshgrid(*[np.arange(N1)] * 3, indexing="ij"), -1)[..., ::-1].reshape(-1, 3)
    r = np.zeros((f.nblocks, N1 ** 3))
    for b in range(f.nblocks):
        h = f.h0 / 2 ** int(f.level[b])
        pos = np.array(f.lo) + (np.array(f.corner[b]) + x) * h
        r[b] = np.linalg.norm(pos, axis=1)
    a = duf.cpu().numpy().reshape(f.nblocks, 20, -1)
    d = dud.cpu().numpy().reshape(f.nblocks, 20, -1)
    outside_core = np.broadcast_to((r >= 0.8 + 1e-9)[:, None, :], a.shape)
    assert np.array_equal(a[outside_core], d[outside_core])
    core = np.broadcast_to((r < 0.8 - 1e-9)[:, None, :], a.shape)
    assert np.all(d[core] == 0.0) and np.count_nonzero(a[core]) > 0
    Pf.close()
    Pd.close()


@pytest.mark.parametrize("rate", [False, True])
def test_fitted_rk4_step_plain_and_batched_match_oracle(tgh, oracle, rate):
    case = _case(tgh, "harmonic", rate, v=0.1)
    f = tgh.gh_forest(case, 8, 2)
    P = tgh.GHProblem(case, f, 4, margin_check=False)
    O = oracle.problem(case, f, 4)
    _cache(tgh, P, O, f, seed=9)
    t = 0.3
    u = O.fitted_initial_state(O.statevector(), t)
    u = u + tgh.perturbation(f, amplitude=1e-6, seed=5)
    dt = 0.25 * f.h0 / 2.0
    ug = _to_gpu(u)
    P.rk4_step(ug, t, dt)
    uo = u.copy()
    O.rk4_step(uo, t, dt)
    scale = max(1.0, float(np.abs(uo).max()))
    assert np.max(np.abs(ug.cpu().numpy() - uo)) < 1e-12 * scale
    ub = _to_gpu(u)
    P.step_batched(ub, t, dt, 1)
    P.settle(ub, t + dt)
    us = _to_gpu(uo)
    P.settle(us, t + dt)
    assert torch.max(torch.abs(ub - us)).item() < 1e-12 * scale
    P.close()


def test_fitted_steps_are_refused_until_the_cache_is_filled(tgh):
    case = _case(tgh, "kerr_schild", False)
    f = tgh.gh_forest(case, 8, 2)
    P = tgh.GHProblem(case, f, 4, margin_check=False)
    u = P.initial_state(P.statevector(), 0.0)
    with pytest.raises(tgh._abi.TGHError, match="target cache"):
        P.rk4_step(u, 0.0, 0.01)
    with pytest.raises(tgh._abi.TGHError, match="target cache"):
        P.step_batched(u, 0.0, 0.01, 1)
    P.fill_target_analytic(0.0)
    P.rk4_step(u, 0.0, 0.01)
    assert torch.isfinite(u).all()
    Pd = tgh.GHProblem(tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=2.0, gauge="algebraic"), f, 4,
                       margin_check=False)
    with pytest.raises(tgh._abi.TGHError, match="not :fitted"):
        Pd.fill_target_analytic(0.0, 1.0)
    P.close()
    Pd.close()
