"""The constraint monitors on the GPU against the oracle on identical inputs.

Tolerance: the reference's own for the gauge monitor's kernel against a host assembly
(test/constraints_tests.jl:183-231, 1e-12 of the derivative scale), applied per point with
the right-hand side's scale (max(1, |D2 u| / h^2, |u|)) to every slot; the mask slot and the
masked points exactly. The norms (one fold over the primaries) within 1e-12 relative.
"""
import numpy as np
import pytest
import torch

from helpers import cases, rhs_scale, two_level_forest
from test_gpu_parity import _initial, _to_gpu

pytestmark = pytest.mark.gpu

TOL = 1e-12
ROWS = [0, 1, 2, 3, 4, 6, 7, 8, 10, 11, 12, 17, 19]
ND = 10  # diag slots per block: C_a, H, M_i, mask, tau


def _monitor_rows(tgh):
    rows = cases(tgh)
    out = [rows[i] for i in ROWS]
    c = tgh.gauge_wave_case(A=1 / 20, d=1.0, eps_ko=0.0, gamma0=1.0, gamma2=0.0)
    out.append(("gauge_wave_two_level", c, two_level_forest(tgh, c, 8), 4, 0.125))
    return out


def _compare(tgh, oracle, name, case, forest, q, t, mask):
    P = tgh.GHProblem(case, forest, q, margin_check=False)
    O = oracle.problem(case, forest, q)
    u = _initial(tgh, P, O, case, forest, name, t)
    allp = mask == "all"
    d_ref = O.diag()
    O.gh_constraint(d_ref, u, t, allpoints=allp)
    O.adm_constraint(d_ref, u, t, allpoints=allp)
    ug = _to_gpu(u)
    P.gh_constraint(ug, t, mask=mask)
    P.adm_constraint(ug, t, mask=mask)
    d = P.diag()
    torch.cuda.synchronize()
    assert torch.equal(ug, _to_gpu(u)), "u was written"
    d = d.cpu().numpy()
    N1 = forest.N + 1
    a = d.reshape(forest.nblocks, ND, N1, N1, N1)[:, :9]
    b = d_ref.reshape(forest.nblocks, ND, N1, N1, N1)[:, :9]
    assert np.array_equal(a[:, 8], b[:, 8]), f"{name}: mask"
    off = b[:, 8] == 0.0
    assert np.all(a[:, :8][np.broadcast_to(off[:, None], a[:, :8].shape)] == 0.0), f"{name}: masked points"
    assert np.all(np.isfinite(a))
    scale = rhs_scale(O.work(), forest, q)
    err = float(np.max(np.max(np.abs(a[:, :8] - b[:, :8]), axis=1) / scale))
    assert err < TOL, f"{name}: {err}"
    # the norms of what the monitors wrote
    for weighting in ("volume", "points"):
        n = P.constraint_norms(weighting=weighting)
        nr = O.constraint_norms(d_ref, weighting=weighting)
        got = np.array(n["gauge_l2"] + n["gauge_linf"] + [n["ham_l2"], n["ham_linf"]] + n["mom_l2"] + n["mom_linf"])
        floor = 1e-12 * max(1.0, float(np.max(np.abs(nr))))
        assert np.allclose(got, nr, rtol=1e-10, atol=floor), (name, weighting, got, nr)
    return P, O, u


@pytest.mark.parametrize("row", range(len(ROWS) + 1))
def test_monitors_match_oracle(tgh, oracle, row):
    name, case, forest, q, t = _monitor_rows(tgh)[row]
    _compare(tgh, oracle, name, case, forest, q, t, "interior")


@pytest.mark.parametrize("row", [6, 7, 8])
def test_monitors_match_oracle_on_every_point(tgh, oracle, row):
    # the damped, frozen and algebraic-source holes with their layers and cores evaluated too
    name, case, forest, q, t = _monitor_rows(tgh)[row]
    _compare(tgh, oracle, name, case, forest, q, t, "all")


@pytest.mark.parametrize("q", [2, 4])
def test_monitors_are_exactly_zero_on_flat_space(tgh, q):
    case = tgh.minkowski_case(L=1.0, eps_ko=0.5, gamma0=1.0, gamma2=-0.5)
    P = tgh.GHProblem(case, tgh.gh_forest(case, 8, 2), q)
    u = P.initial_state(P.statevector(), 0.0)
    P.gh_constraint(u, 0.0).adm_constraint(u, 0.0)
    n = P.constraint_norms()
    assert all(v == 0.0 for v in n["gauge_l2"] + n["gauge_linf"] + n["mom_l2"] + n["mom_linf"])
    assert n["ham_l2"] == 0.0 and n["ham_linf"] == 0.0


def test_adm_monitor_with_matter_matches_oracle(tgh, oracle):
    case = tgh.gauge_wave_case(A=1 / 20, d=1.0, eps_ko=0.5, gamma0=1.0, gamma2=-0.5)
    forest = tgh.gh_forest(case, 8, 2)
    P = tgh.GHProblem(case, forest, 4)
    O = oracle.problem(case, forest, 4)
    u = O.initial_state(O.statevector(), 0.25)
    rng = np.random.default_rng(5)
    matter = rng.uniform(-1e-3, 1e-3, size=forest.nblocks * 10 * (forest.N + 1) ** 3)
    d_ref = O.diag()
    O.adm_constraint(d_ref, u, 0.25, matter=matter)
    P.adm_constraint(_to_gpu(u), 0.25, matter=_to_gpu(matter))
    d = P.diag().cpu().numpy()
    N1 = forest.N + 1
    a = d.reshape(forest.nblocks, ND, N1, N1, N1)[:, 4:9]
    b = d_ref.reshape(forest.nblocks, ND, N1, N1, N1)[:, 4:9]
    scale = rhs_scale(O.work(), forest, 4)
    assert float(np.max(np.max(np.abs(a - b), axis=1) / scale)) < TOL
    # the matter moved the constraints by its 16 pi rho and 8 pi S_i (and its source)
    d0 = O.diag()
    O.adm_constraint(d0, u, 0.25)
    assert np.abs(d0.reshape(forest.nblocks, ND, -1)[:, 4] - d_ref.reshape(forest.nblocks, ND, -1)[:, 4]).max() > 1e-3


def test_norms_per_level_match_oracle(tgh, oracle):
    case = tgh.gauge_wave_case(A=1 / 20, d=1.0, eps_ko=0.0, gamma0=1.0, gamma2=0.0)
    forest = two_level_forest(tgh, case, 8)
    P = tgh.GHProblem(case, forest, 4)
    O = oracle.problem(case, forest, 4)
    u = O.initial_state(O.statevector(), 0.125)
    d_ref = O.diag()
    O.gh_constraint(d_ref, u, 0.125)
    O.adm_constraint(d_ref, u, 0.125)
    ug = _to_gpu(u)
    P.gh_constraint(ug, 0.125).adm_constraint(ug, 0.125)
    for lev in (0, 1):
        n = P.constraint_norms(weighting="points", at_level=lev)
        nr = O.constraint_norms(d_ref, weighting="points", at_level=lev)
        got = np.array(n["gauge_l2"] + n["gauge_linf"] + [n["ham_l2"], n["ham_linf"]] + n["mom_l2"] + n["mom_linf"])
        assert np.allclose(got, nr, rtol=1e-10, atol=1e-12 * max(1.0, float(np.max(np.abs(nr))))), (lev, got, nr)
        assert got[9] > 0.0
    # a level with no block: nothing evolved, the L2 is 0 by definition
    n = P.constraint_norms(at_level=5)
    assert n["ham_l2"] == 0.0 and n["ham_linf"] == 0.0


def test_monitor_arguments_are_checked(tgh):
    import ctypes
    case = tgh.gauge_wave_case()
    P = tgh.GHProblem(case, tgh.gh_forest(case, 8, 1), 4)
    u = P.initial_state(P.statevector(), 0.0)
    with pytest.raises(tgh._abi.TGHError):
        P._check(P.lib.tgh_gh_constraint(P._h, ctypes.c_void_p(u.data_ptr()), 0.0, 7))
    with pytest.raises(tgh._abi.TGHError):
        P._check(P.lib.tgh_constraint_norms(P._h, 3, -1, (ctypes.c_double * 16)()))
    with pytest.raises(ValueError):
        P.constraint_norms(weighting="cells")
