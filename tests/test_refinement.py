"""The refinement criterion on the CPU: the oracle's indicator and the host-side marks, restating
the reference's test/refinement_tests.jl (the algebra :50-102, the masked amplitude :104-141,
the four marks :143-215, the level floor :217-291, the mask :293-337, the margin :400-414)."""
import math

import numpy as np
import pytest

ND = 10  # diag slots per block (tau is slot 9)


def _hole(tgh):
    # adaptive_hole_fixture (test/evolution_cases.jl:327-340): M = 1, a = 0, box [-5, 5]^3,
    # r_0 = 3/10, r_1 = 5/4, margin 4, q = 2
    return tgh.kerr_schild_case(M=1.0, a=0.0, halfwidth=5.0, r0=0.3, r1=1.25, margin=4, variant="damped",
                                gauge="sampled")


def _ref(tgh, **kw):
    args = dict(refine_tol=2 / 5, coarsen_tol=1 / 10, maxlevel_cap=1, floor_margin=0.0, ceiling_cells=1)
    args.update(kw)
    return tgh.Refinement(**args)


def _refined_forest(tgh, case, N=8, roots=4):
    """roots^3 level-0 blocks with the root block at the origin's lower corner refined once."""
    f = tgh.gh_forest(case, N, roots)
    leaves = [(0, tuple(int(v) for v in c)) for c in f.corner if tuple(c) != (0, 0, 0)]
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                leaves.append((1, (dx * N, dy * N, dz * N)))
    leaves.sort()
    return tgh.Forest(N, f.lo, f.h0, f.cells0, f.periodic, np.array([l for l, _ in leaves], dtype=np.int32),
                      np.array([c for _, c in leaves], dtype=np.int32))


def _plain_bounds(tgh, forest, cap):
    r = tgh.refinement
    return r.LevelBounds(forest, (0.0, 0.0, 0.0), 0.0, -1.0, 0, ((-5.0, 5.0),) * 3, (False,) * 3, 0.0, cap, cap)


def test_lohner_algebra(tgh):
    lohner = tgh.refinement.lohner
    assert lohner(1.0, 1.0, 1.0, 1.0) == 0
    assert lohner(0.0, 1.0, 2.0, 1.0) == 0
    for um, u0, up in ((0.0, 1.0, 0.0), (-1.0, 2.0, 5.0), (3.0, -1.0, 3.0)):
        assert 0 <= lohner(um, u0, up, 1.0) <= 1
    f = lambda r: 2 / r  # noqa: E731
    tau_of = lambda h: lohner(f(1.2 - h), f(1.2), f(1.2 + h), 2.0)  # noqa: E731
    assert tau_of(0.1) > tau_of(0.05) > tau_of(0.025)
    for h in (0.1, 0.05):
        assert 0.25 <= tau_of(h / 2) / tau_of(h) <= 0.5
    s = 1e3
    assert math.isclose(lohner(s * f(1.1), s * f(1.2), s * f(1.3), s * 2.0), lohner(f(1.1), f(1.2), f(1.3), 2.0),
                        rel_tol=1e-12)
    # the noise floor is global, or the dust refines everything
    um, u0, up = 3.9e-16, 3.6e-17, 3.6e-17
    assert lohner(um, u0, up, abs(u0)) > 0.9
    assert lohner(um, u0, up, 0.0) > 0.9
    assert lohner(um, u0, up, 1.0) < 1e-13
    assert lohner(0.0, 1.0, 0.0, 1.0) > 0.1


def test_refinement_parameters_are_checked(tgh):
    with pytest.raises(ValueError):
        _ref(tgh, refine_tol=0.1, coarsen_tol=0.1)
    with pytest.raises(ValueError):
        _ref(tgh, refine_tol=2.0)
    with pytest.raises(ValueError):
        _ref(tgh, eps=0.0)
    with pytest.raises(ValueError):
        _ref(tgh, ceiling_level=3)


def test_the_reference_amplitude_is_masked_and_shared_by_the_ten(tgh, oracle):
    case = _hole(tgh)
    f = tgh.gh_forest(case, 8, 2)
    O = oracle.problem(case, f, 2)
    u = O.initial_state(O.statevector(), 0.0)
    d = O.diag()
    masked = O.tau(d, u, 0.0)["scales"]
    unmasked = O.tau(d, u, 0.0, allpoints=True)["scales"]
    assert max(masked) < max(unmasked)
    assert math.isclose(max(masked), 2 / 1.25, rel_tol=0.25)
    assert math.isclose(max(unmasked), 2 / 0.3, rel_tol=0.25)
    gw = tgh.gauge_wave_case(eps_ko=0.5, gamma0=1.0, gamma2=0.0)
    fg = tgh.gh_forest(gw, 8, 1)
    Og = oracle.problem(gw, fg, 2)
    ug = Og.initial_state(Og.statevector(), 0.0)
    r = Og.tau(Og.diag(), ug, 0.0)
    assert sum(1 for x in r["scales"] if x == 0.0) >= 6
    assert r["scale"] > 0


def test_the_four_marks_with_the_box_keyed_on_coarsen_tol(tgh, oracle):
    case = _hole(tgh)
    forest = _refined_forest(tgh, case)
    O = oracle.problem(case, forest, 2)
    ref = _ref(tgh, maxlevel_cap=2)
    lb = _plain_bounds(tgh, forest, 2)
    R = tgh.refinement
    nb = len(forest.level)
    levels = [int(x) for x in forest.level]
    b0 = levels.index(0)
    d = O.diag().reshape(nb, ND, 9, 9, 9)

    def marks(rf, bounds):
        counts, boxes = O.firing(d.ravel(), [rf.refine_tol, rf.coarsen_tol])
        return R.refine_flags(forest, bounds, rf, counts, boxes)

    # everything quiet: a bare Coarsen above level 0, a bare Keep at it
    m = marks(ref, lb)
    assert all(m[b] == (R.COARSEN if levels[b] > 0 else R.KEEP) for b in range(nb))
    # one block under-resolved below the cap: (Refine, box), the box the coarsen_tol sweep's,
    # in cells max(1, lo - 1):min(N, hi) of the firing nodes (2:6, 4, 5), 1-based
    d[b0, 9, 4, 3, 2] = 0.9
    d[b0, 9, 4, 3, 1] = d[b0, 9, 4, 3, 5] = 0.2
    m = marks(ref, lb)
    assert m[b0] == (R.REFINE, ((1, 6), (3, 4), (4, 5)))
    # the same block at the cap: (Keep, box), the equal-level margin
    capped = _ref(tgh, maxlevel_cap=0)
    m = marks(capped, _plain_bounds(tgh, forest, 0))
    assert m[b0] == (R.KEEP, ((1, 6), (3, 4), (4, 5)))
    # between the thresholds, below the cap: held with its box
    d[b0, 9] = 0.0
    d[b0, 9, 4, 3, 2] = 0.2
    m = marks(ref, lb)
    assert m[b0] == (R.KEEP, ((2, 3), (3, 4), (4, 5)))


def test_the_level_floor_is_the_level_the_interior_radii_need(tgh):
    case = _hole(tgh)
    forest = tgh.gh_forest(case, 8, 4)
    G = 2
    R = tgh.refinement
    lev = R.horizon_floor_level(forest, case, G)
    assert lev == 1
    r_h = R.horizon_radii(case)[0]
    it = case.interior
    for h, holds in ((R.spacing(forest, lev), True), (R.spacing(forest, lev - 1), False)):
        ok = it["r1"] <= r_h - it["margin"] * h and it["r1"] - it["r0"] >= 2 * (G + 1) * h
        assert ok == holds
    with pytest.raises(ValueError):
        R.level_bounds(case, forest, 0.0, G, _ref(tgh, maxlevel_cap=0))


def _tau_pass(tgh, oracle, case, forest, q=2, allpoints=False, scale=None):
    O = oracle.problem(case, forest, q)
    u = O.initial_state(O.statevector(), 0.0)
    d = O.diag()
    r = O.tau(d, u, 0.0, allpoints=allpoints, scale=scale)
    return O, d, r


def test_the_floor_binds_only_when_loose(tgh, oracle):
    case = _hole(tgh)
    forest = tgh.gh_forest(case, 8, 4)
    R = tgh.refinement
    ref = _ref(tgh)
    O, d, _ = _tau_pass(tgh, oracle, case, forest)
    lb = R.level_bounds(case, forest, 0.0, 2, ref)
    assert lb.floor_level == 1
    nofloor = R.LevelBounds(forest, lb.center, lb.floor_lo, lb.floor_hi, 0, lb.box, lb.periodic, lb.ceiling_margin,
                            lb.ceiling_level, lb.maxlevel_cap)
    c, bx = O.firing(d, [ref.refine_tol, ref.coarsen_tol])
    assert R.refine_flags(forest, lb, ref, c, bx) == R.refine_flags(forest, nofloor, ref, c, bx)
    loose = _ref(tgh, refine_tol=0.99, coarsen_tol=0.9, maxlevel_cap=1)
    c, bx = O.firing(d, [loose.refine_tol, loose.coarsen_tol])
    floored = R.refine_flags(forest, lb, loose, c, bx)
    flat = R.refine_flags(forest, nofloor, loose, c, bx)
    assert floored != flat
    assert all(m == R.KEEP for m in flat)
    nref = sum(1 for m in floored if m == R.REFINE or (isinstance(m, tuple) and m[0] == R.REFINE))
    assert nref > 0
    assert nref == sum(1 for b in range(len(forest.level)) if R.block_level_bounds(lb, b)[0] > 0)


def test_the_indicator_is_zero_inside_r1_and_the_core_cannot_fire(tgh, oracle):
    case = _hole(tgh)
    forest = tgh.gh_forest(case, 8, 4)
    O, d, r = _tau_pass(tgh, oracle, case, forest)
    nb, N1 = len(forest.level), 9
    tau = d.reshape(nb, ND, N1, N1, N1)[:, 9]
    idx = np.arange(N1)
    inside, worst = 0, 0.0
    for b in range(nb):
        h = forest.h0
        o = [forest.lo[k] + forest.corner[b][k] * h for k in range(3)]
        z, y, x = np.meshgrid(o[2] + idx * h, o[1] + idx * h, o[0] + idx * h, indexing="ij")
        r2 = np.sqrt(x * x + y * y + z * z)
        m = r2 < 1.25
        inside += int(m.sum())
        assert np.all(tau[b][m] == 0.0)
        if (~m).any():
            worst = max(worst, float(tau[b][~m].max()))
    assert inside > 0 and worst > 0
    assert r["tau_max"] == worst
    _, _, ru = _tau_pass(tgh, oracle, case, forest, allpoints=True, scale=r["scale"])
    assert ru["tau_max"] > r["tau_max"]


def test_the_travelling_margin_is_derived_and_refuses_a_long_chunk(tgh):
    case = _hole(tgh)
    forest = tgh.gh_forest(case, 8, 4)
    R = tgh.refinement
    assert R.refinement_buffer(forest, 1, 0.0) == 1
    h = R.spacing(forest, 1)
    assert R.refinement_buffer(forest, 1, 3 * h) == 4
    with pytest.raises(ValueError):
        R.refinement_buffer(forest, 1, 9 * h)


def test_the_margin_promotes_the_neighbours_of_a_box(tgh, oracle):
    # a Refine with its box at a block's face recruits the face neighbour; a quiet Keep recruits nothing
    case = _hole(tgh)
    forest = tgh.gh_forest(case, 8, 4)
    O = oracle.problem(case, forest, 2)
    R = tgh.refinement
    ref = _ref(tgh, maxlevel_cap=2)
    lb = _plain_bounds(tgh, forest, 2)
    nb = len(forest.level)
    d = O.diag().reshape(nb, ND, 9, 9, 9)
    corners = [tuple(int(v) for v in c) for c in forest.corner]
    b = corners.index((8, 8, 8))
    nbr = corners.index((16, 8, 8))
    d[b, 9, 4, 4, 8] = 0.9  # on the block's upper x face
    c, bx = O.firing(d.ravel(), [ref.refine_tol, ref.coarsen_tol])
    plain = R.refine_flags(forest, lb, ref, c, bx)
    assert plain[b][0] == R.REFINE and plain[nbr] == R.KEEP
    buffered = R.refine_flags(forest, lb, ref, c, bx, buffer=1)
    assert buffered[b] == R.REFINE and buffered[nbr] == R.REFINE
    assert sum(1 for m in buffered if m == R.REFINE) < nb


# ---- the regrid: the new forest and the state transfer (TreeAMR's regrid!, src/driver.jl:1660-1695) ----
def _marks_for(forest, R, refine=(), coarsen_level=None):
    out = []
    for b in range(len(forest.level)):
        c = tuple(int(x) for x in forest.corner[b])
        lev = int(forest.level[b])
        if (lev, c) in refine:
            out.append(R.REFINE)
        elif coarsen_level is not None and lev == coarsen_level:
            out.append(R.COARSEN)
        else:
            out.append(R.KEEP)
    return out


def test_regrid_forest_refines_coarsens_and_balances(tgh):
    R = tgh.refinement
    case = tgh.gauge_wave_case()
    f = tgh.gh_forest(case, 8, 2)
    f1 = R.regrid_forest(f, _marks_for(f, R, refine={(0, (0, 0, 0))}))
    assert len(f1.level) == 15 and sorted(set(int(x) for x in f1.level)) == [0, 1]
    # the eight children all marked Coarsen become their parent again
    f0 = R.regrid_forest(f1, _marks_for(f1, R, coarsen_level=1))
    assert len(f0.level) == 8 and np.array_equal(np.sort(f0.corner, axis=0), np.sort(f.corner, axis=0))
    # seven of eight siblings marked Coarsen: nothing coarsens
    m = _marks_for(f1, R, coarsen_level=1)
    m[[i for i, lv in enumerate(f1.level) if lv == 1][0]] = R.KEEP
    assert len(R.regrid_forest(f1, m).level) == 15
    # refining a level-1 leaf in the corner block's far corner forces its level-0 neighbours to refine
    corner = max(tuple(int(x) for x in c) for c, lv in zip(f1.corner, f1.level) if lv == 1)
    f2 = R.regrid_forest(f1, _marks_for(f1, R, refine={(1, corner)}))
    levels = [int(x) for x in f2.level]
    assert max(levels) == 2 and levels.count(0) < 7


def test_transfer_is_exact_where_points_coincide(tgh, oracle):
    # onto the same forest, and refined then coarsened back: the identity, bit for bit
    R = tgh.refinement
    case = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=2.0, r0=0.8, r1=1.3, gauge="sampled")
    f = tgh.gh_forest(case, 8, 2)
    O = oracle.problem(case, f, 4)
    u = O.initial_state(O.statevector(), 0.0)
    Os = oracle.problem(case, f, 4)
    assert np.array_equal(Os.transfer_from(O, u, 0.0), u)
    f1 = R.regrid_forest(f, _marks_for(f, R, refine={(0, (0, 0, 0))}))
    O1 = oracle.problem(case, f1, 4)
    u1 = O1.transfer_from(O, u, 0.0)
    O0 = oracle.problem(case, R.regrid_forest(f1, _marks_for(f1, R, coarsen_level=1)), 4)
    assert np.array_equal(O0.transfer_from(O1, u1, 0.0), u)


def test_transfer_prolongs_at_the_operator_order(tgh, oracle):
    # smooth periodic data onto a refined mesh: the new points' error against the exact state
    # falls at the prolongation's order as the mesh is refined
    R = tgh.refinement
    case = tgh.gauge_wave_case(A=0.05)
    errs = []
    for N in (8, 16):
        f = tgh.gh_forest(case, N, 2)
        O = oracle.problem(case, f, 4)
        u = O.initial_state(O.statevector(), 0.0)
        f1 = R.regrid_forest(f, _marks_for(f, R, refine={(0, (0, 0, 0))}))
        O1 = oracle.problem(case, f1, 4)
        errs.append(float(np.abs(O1.transfer_from(O, u, 0.0) - O1.initial_state(O1.statevector(), 0.0)).max()))
    assert errs[0] > 0 and errs[0] / errs[1] > 2 ** 5.5  # order q + 2 = 6 prolongation
