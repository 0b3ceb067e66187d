"""The refinement indicator on the GPU against the oracle on identical inputs: tau bit for bit at
every owned point (each operation rounded on its own in both), the masked amplitudes and tau_max
exactly, the firing counts and boxes exactly, and so the marks identical."""
import numpy as np
import pytest
import torch

from helpers import cases, two_level_forest
from test_gpu_parity import _initial, _to_gpu
from test_refinement import _hole, _ref

pytestmark = pytest.mark.gpu

ND = 10


def _rows(tgh):
    rows = cases(tgh)
    out = [("hole_fixture", _hole(tgh), tgh.gh_forest(_hole(tgh), 8, 4), 2, 0.0)]
    out += [rows[i] for i in (1, 2, 6, 7, 10, 11, 17, 19)]
    c = tgh.gauge_wave_case(A=1 / 20, d=1.0, eps_ko=0.0, gamma0=1.0, gamma2=0.0)
    out.append(("gauge_wave_two_level", c, two_level_forest(tgh, c, 8), 4, 0.125))
    return out


@pytest.mark.parametrize("row", range(10))
@pytest.mark.parametrize("mask", ["interior", "all"])
def test_tau_and_firing_match_oracle_bit_for_bit(tgh, oracle, row, mask):
    name, case, forest, q, t = _rows(tgh)[row]
    P = tgh.GHProblem(case, forest, q, margin_check=False)
    O = oracle.problem(case, forest, q)
    u = _initial(tgh, P, O, case, forest, name, t)
    allp = mask == "all"
    d_ref = O.diag()
    r_ref = O.tau(d_ref, u, t, allpoints=allp)
    r = P.tau(_to_gpu(u), t, mask=mask)
    d = P.diag().cpu().numpy()
    N1 = forest.N + 1
    a = d.reshape(forest.nblocks, ND, N1, N1, N1)[:, 9]
    b = d_ref.reshape(forest.nblocks, ND, N1, N1, N1)[:, 9]
    if case.interior is None:
        # copies and prolongation only: the working arrays are equal bit for bit, and so is tau
        assert np.array_equal(a, b, equal_nan=True), f"{name}: tau differs at {np.argwhere(a != b)[:5]}"
        assert r["tau_max"] == r_ref["tau_max"]
    else:
        # the Dirichlet ghosts are two evaluations of the analytic metric, equal to ~1e-13
        # relative; tau moves by at most 4 delta / (4 eps scale) with it, well inside 1e-10
        assert float(np.max(np.abs(a - b))) < 1e-10, name
        assert abs(r["tau_max"] - r_ref["tau_max"]) < 1e-10
    # the masked amplitudes read owned points only: exact
    assert r["scales"] == r_ref["scales"] and r["scale"] == r_ref["scale"]
    # the firing sweeps on the GPU's own tau are the oracle's, exactly
    tols = [0.4, 0.1, 0.01, 1e-4]
    c, bx = P.firing(tols)
    cr, bxr = O.firing(d, tols)
    assert np.array_equal(c, cr) and np.array_equal(bx, bxr), name


def test_indicator_flags_match_the_oracle_pipeline(tgh, oracle):
    case = _hole(tgh)
    forest = tgh.gh_forest(case, 8, 4)
    ref = _ref(tgh)
    P = tgh.GHProblem(case, forest, 2, margin_check=False)
    O = oracle.problem(case, forest, 2)
    u = O.initial_state(O.statevector(), 0.0)
    out = tgh.indicator_flags(P, case, _to_gpu(u), 0.0, ref, buffer=1)
    d = O.diag()
    r = O.tau(d, u, 0.0)
    c, bx = O.firing(d, [ref.refine_tol, ref.coarsen_tol])
    R = tgh.refinement
    lb = R.level_bounds(case, forest, 0.0, 2, ref)
    assert out["flags"] == R.refine_flags(forest, lb, ref, c, bx, buffer=1)
    assert abs(out["tau_max"] - r["tau_max"]) < 1e-10  # Dirichlet ghosts: see above
    assert out["nfiring"] == int(c[:, 1].sum())
    cen = R.refinement_centroid(forest, c, bx)
    assert (out["centroid"] is None and cen is None) or np.array_equal(out["centroid"], cen)
    # around a static hole at the origin the refined region is centred near it
    assert out["centroid"] is not None and np.linalg.norm(out["centroid"]) < 3 * R.spacing(forest, 0)
    assert any(m == R.REFINE for m in out["flags"])


def _regrid_rows(tgh):
    """(name, case, forest, q, t, marks): a hole refined where its indicator asks, a two-level
    gauge wave coarsened back, and the moving-hole hierarchy with its finest level coarsened and
    root blocks refined (rebalanced)."""
    R = tgh.refinement
    rows = []
    hole = _hole(tgh)
    f = tgh.gh_forest(hole, 8, 4)
    rows.append(("hole_fixture_indicator", hole, f, 2, 0.0, None))
    c = tgh.gauge_wave_case(A=1 / 20, d=1.0, eps_ko=0.0, gamma0=1.0, gamma2=0.0)
    f = two_level_forest(tgh, c, 8)
    rows.append(("gauge_wave_coarsened", c, f, 4, 0.125, [R.COARSEN if lv == 1 else R.KEEP for lv in f.level]))
    name, c, f, q, t = cases(tgh)[19]
    top = int(f.level.max())
    marks = [R.COARSEN if lv == top else (R.REFINE if lv == 0 and i % 5 == 0 else R.KEEP)
             for i, lv in enumerate(f.level)]
    rows.append((name, c, f, q, t, marks))
    return rows


@pytest.mark.parametrize("row", range(3))
def test_regrid_transfer_matches_oracle_bit_for_bit(tgh, oracle, row):
    name, case, forest, q, t, marks = _regrid_rows(tgh)[row]
    R = tgh.refinement
    P = tgh.GHProblem(case, forest, q, margin_check=False)
    O = oracle.problem(case, forest, q)
    u = _initial(tgh, P, O, case, forest, name, t)
    if marks is None:
        marks = tgh.indicator_flags(P, case, _to_gpu(u), t, _ref(tgh), buffer=1)["flags"]
    f2 = R.regrid_forest(forest, marks)
    assert f2.nblocks != forest.nblocks or not np.array_equal(f2.corner, forest.corner)
    P2, u2 = R.regrid(P, _to_gpu(u), t, marks)
    O2 = oracle.problem(case, f2, q)
    ref = O2.transfer_from(O, u, t)
    O2.stage_limit(ref, t)
    got = u2.cpu().numpy()
    assert np.array_equal(got, ref), f"{name}: {np.abs(got - ref).max()}"
    # the new problem steps on the transferred state
    lam = P2.max_speed(u2, t)
    assert np.isfinite(lam) and lam > 0
