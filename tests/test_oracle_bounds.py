"""The oracle's range projection pinned to the reference's claims (no GPU).

Restates test/bounds_tests.jl:26-300: nine states, each of which must be repaired by moving the
ADM blocks that are wrong and no others, bit for bit (:79-141, :163-200); every repaired state
inside its ranges (:65-77); the projection idempotent on the state and on its flag (:191-197);
a raised lapse keeps (alpha/sqrt(gamma)) Pi and a cap keeps Pi's direction (:201-212); and the
identity, bit for bit, on healthy Kerr-Schild data down to the core (:217-238). The mesh pass
writes back only where it fired and counts each lattice point once (:300-).
"""
import math

import numpy as np
import pytest

# default_bounds(M = 1, r_gate = 1) (src/bounds.jl:158-175): alpha, lambda, beta, K, r_gate
BD = (1 / 50, 50.0, 1 / 100, 1000.0, 10.0, 100.0, 1.0)
PACK = [(0, 0), (1, 0), (2, 0), (3, 0), (1, 1), (2, 1), (3, 1), (2, 2), (3, 2), (3, 3)]


def _pack(m):
    return np.array([m[a, b] for a, b in PACK])


def _sym(h):
    m = np.zeros((4, 4))
    for n, (a, b) in enumerate(PACK):
        m[a, b] = m[b, a] = h[n]
    return m


def synthetic_state(lam, htt, beta, Pi=None):
    """A state from its ADM parts: gamma's spectrum in a fixed generic rotation (no eigenvector
    along an axis), the lowered shift beta_i = h_ti, h_tt and Pi."""
    a, b, c = 1 / 3, 2 / 5, 3 / 7
    Rz = np.array([[math.cos(a), -math.sin(a), 0], [math.sin(a), math.cos(a), 0], [0, 0, 1]])
    Ry = np.array([[math.cos(b), 0, math.sin(b)], [0, 1, 0], [-math.sin(b), 0, math.cos(b)]])
    Rx = np.array([[1, 0, 0], [0, math.cos(c), -math.sin(c)], [0, math.sin(c), math.cos(c)]])
    R = Rz @ Ry @ Rx
    g = R @ np.diag(lam) @ R.T
    g = (g + g.T) / 2
    hm = np.zeros((4, 4))
    hm[0, 0] = htt
    hm[0, 1:] = hm[1:, 0] = beta
    hm[1:, 1:] = g - np.eye(3)
    P = np.array([(v - 5) / 20 for v in range(1, 11)]) if Pi is None else np.asarray(Pi, dtype=float)
    return _pack(hm), P


def _split(h):
    hm = _sym(h)
    g = hm[1:, 1:] + np.eye(3)
    beta = hm[0, 1:]
    bb = beta @ np.linalg.solve(g, beta)
    return g, (1 - hm[0, 0]) + bb, bb, np.linalg.det(g)


def moved(h, h2, P, P2):
    m = []
    if h[0].tobytes() != h2[0].tobytes():
        m.append("tt")
    if h[1:4].tobytes() != h2[1:4].tobytes():
        m.append("beta")
    if h[4:].tobytes() != h2[4:].tobytes():
        m.append("gamma")
    if P.tobytes() != P2.tobytes():
        m.append("Pi")
    return sorted(m)


def in_ranges(h, P, bd, rtol):
    a0, a1, l0, l1, bmax, kmax, _ = bd
    g, a2, bb, detg = _split(h)
    lam = np.linalg.eigvalsh(g)
    if not (a2 > 0 and detg > 0):
        return False
    alpha = math.sqrt(a2)
    a = alpha / math.sqrt(detg)
    return (a0 * (1 - rtol) <= alpha <= a1 * (1 + rtol) and l0 * (1 - rtol) <= lam.min()
            and lam.max() <= l1 * (1 + rtol) and math.sqrt(bb) <= bmax * (1 + rtol)
            and np.max(np.abs(a * P)) <= kmax * (1 + rtol))


def _ks(tgh):
    return tgh.kerr_schild_case(M=1.0, a=0.0, variant=None).config(4).bg


def bounds_states(tgh, oracle):
    bg = _ks(tgh)
    hb, Pb, _, _ = oracle.background_state(bg, 0.0, np.array([2.0, 1.0, -1.0]))
    hnan = hb.copy()
    hnan[5] = np.nan  # gamma_xy
    Pinf = Pb.copy()
    Pinf[1] = np.inf  # Pi_tx
    x0 = 0.4 * np.ones(3) / math.sqrt(3.0)
    h0, P0, _, _ = oracle.background_state(bg, 0.0, x0)
    big = [500.0 if v == 6 else (v - 5) / 20 for v in range(1, 11)]
    return [
        ("one negative eigenvalue of gamma",
         synthetic_state((-0.3, 1.2, 2.0), 0.2, (0.1, -0.2, 0.05)), ["gamma"]),
        ("two negative eigenvalues of gamma, det gamma > 0",
         synthetic_state((-0.4, -0.7, 1.5), 0.2, (0.05, 0.05, -0.05)), ["gamma"]),
        ("-g^tt < 0 with gamma healthy", synthetic_state((0.8, 1.0, 1.2), 1.5, (0.1, 0.0, 0.0)), ["tt"]),
        ("a NaN in one component of h", (hnan, Pb), ["gamma"]),
        ("an Inf in one component of Pi", (hb, Pinf), ["Pi"]),
        ("healthy Kerr-Schild at the core's edge", (h0, P0), []),
        ("|beta| above beta_max", synthetic_state((1.0, 1.0, 1.0), -1.0, (12.0, 0.0, 0.0)), ["beta"]),
        ("a positive lapse below alpha_min", synthetic_state((1.0, 1.0, 1.0), 1.0 - 1e-6, (0.0, 0.0, 0.0)),
         ["Pi", "tt"]),
        ("(alpha/sqrt(gamma)) Pi above K_max", synthetic_state((1.0, 1.0, 1.0), 0.0, (0.0, 0.0, 0.0), big), ["Pi"]),
    ]


def test_each_state_is_repaired_and_only_what_is_wrong_moves(tgh, oracle):
    for name, (h, P), moves in bounds_states(tgh, oracle):
        h2, P2, hit, nonfinite = oracle.bounds_project(h, P, BD)
        assert hit == bool(moves), name
        assert nonfinite == (not (np.all(np.isfinite(h)) and np.all(np.isfinite(P)))), name
        assert moved(h, h2, P, P2) == sorted(moves), (name, moved(h, h2, P, P2))
        assert in_ranges(h2, P2, BD, 1e-9), name
        # bitwise idempotent, and the flag with it
        h3, P3, hit2, nf2 = oracle.bounds_project(h2, P2, BD)
        assert h3.tobytes() == h2.tobytes() and P3.tobytes() == P2.tobytes(), name
        assert not hit2 and not nf2, name


def test_the_states_are_what_their_names_say(tgh, oracle):
    rows = bounds_states(tgh, oracle)
    g, _, _, detg = _split(rows[1][1][0])
    assert detg > 0 and np.sum(np.linalg.eigvalsh(g) < 0) == 2
    assert _split(rows[2][1][0])[1] < 0
    # the non-finite rows go to Minkowski in the offending component, every other bit kept
    h, P = rows[3][1]
    h2, P2, _, _ = oracle.bounds_project(h, P, BD)
    want = np.where(np.isfinite(h), h, 0.0)
    assert h2.tobytes() == want.tobytes() and P2.tobytes() == P.tobytes()
    h, P = rows[4][1]
    h2, P2, _, _ = oracle.bounds_project(h, P, BD)
    want = np.where(np.isfinite(P), P, 0.0)
    assert h2.tobytes() == h.tobytes() and P2.tobytes() == want.tobytes()


def test_a_raised_lapse_keeps_the_momentum_term_and_a_cap_keeps_its_direction(tgh, oracle):
    rows = bounds_states(tgh, oracle)
    h, P = rows[7][1]
    h2, P2, _, _ = oracle.bounds_project(h, P, BD)
    a0, a1 = math.sqrt(_split(h)[1]), math.sqrt(_split(h2)[1])
    assert a1 == pytest.approx(BD[0], rel=1e-12)
    assert np.allclose(a1 * P2, a0 * P, rtol=1e-12, atol=0)
    h, P = rows[8][1]
    _, P2, _, _ = oracle.bounds_project(h, P, BD)
    assert np.max(np.abs(P2)) == pytest.approx(BD[5], rel=1e-14)
    assert np.allclose(P2, P * (BD[5] / np.max(np.abs(P))), rtol=1e-14, atol=0)


def test_the_identity_on_healthy_data(tgh, oracle):
    bgs = [_ks(tgh), tgh.kerr_schild_case(M=1.0, a=0.7, variant=None).config(4).bg,
           tgh.gauge_wave_case(A=0.05).config(4).bg]
    pts = [(2.1, -1.3, 0.7), (3.0, 0.5, -2.2), (-1.7, 2.4, 1.1)]
    for bg in bgs:
        for x in pts:
            h, P, _, _ = oracle.background_state(bg, 0.3, np.array(x))
            h2, P2, hit, _ = oracle.bounds_project(h, P, BD)
            assert not hit and h2.tobytes() == h.tobytes() and P2.tobytes() == P.tobytes()
    # inside the layer and core, down to r_0 = 2/5, where the data are steepest
    for r in (0.4, 0.5, 1.15):
        for n in ((0, 0, 1), (1, 1, 1), (-2, 1, 3)):
            x = r * np.array(n, dtype=float) / np.linalg.norm(n)
            h, P, _, _ = oracle.background_state(_ks(tgh), 0.0, x)
            h2, P2, hit, _ = oracle.bounds_project(h, P, BD)
            assert not hit and h2.tobytes() == h.tobytes() and P2.tobytes() == P.tobytes()


def test_random_states_land_in_range_and_are_fixed_points(oracle):
    # |h| <= 5, |Pi| <= 100 (the range of the reference's measurement of the re-test passes)
    rng = np.random.default_rng(3)
    fired = 0
    for _ in range(2000):
        h = rng.uniform(-5, 5, 10) * rng.uniform(0, 1) ** 2
        P = rng.uniform(-100, 100, 10) * rng.uniform(0, 1) ** 2
        h2, P2, hit, _ = oracle.bounds_project(h, P, BD)
        fired += hit
        if hit:
            assert in_ranges(h2, P2, BD, 1e-9)
        h3, P3, hit2, _ = oracle.bounds_project(h2, P2, BD)
        assert not hit2 and h3.tobytes() == h2.tobytes() and P3.tobytes() == P2.tobytes()
    assert fired > 500


def _hole(tgh):
    case = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=2.0, r0=0.8, r1=1.3, gauge="sampled")
    return case, tgh.gh_forest(case, 8, 2)


def test_the_mesh_pass_repairs_inside_the_gate_only_and_counts_primaries(tgh, oracle):
    case, forest = _hole(tgh)
    O = oracle.problem(case, forest, 4)
    u = O.initial_state(O.statevector(), 0.0)
    N1 = forest.N + 1
    S = N1 ** 3
    bd = BD[:6] + (1.0,)
    bad_h, bad_P = synthetic_state((-0.3, 1.2, 2.0), 0.2, (0.1, -0.2, 0.05))
    # the healthy hole, its core filled from the sphere r_0: nothing fires, nothing moves
    clean = u.copy()
    assert O.apply_bounds(u, 0.0, bd)["fired"] == 0
    assert u.tobytes() == clean.tobytes()
    # plant the bad state at every owned point of block 0 and of the last block
    for b in (0, forest.nblocks - 1):
        for v in range(10):
            u[(b * 20 + v) * S:(b * 20 + v + 1) * S] = bad_h[v]
            u[(b * 20 + 10 + v) * S:(b * 20 + 10 + v + 1) * S] = bad_P[v]
    before = u.copy()
    r = O.apply_bounds(u, 0.0, bd)
    # the domain [-2,2]^3 in 8 blocks: the hole sits at a corner of every block, so each of the
    # two planted blocks has points inside r_gate = 1 and points outside it
    changed = np.any((u != before).reshape(forest.nblocks, 20, S), axis=1)
    assert changed[1:-1].sum() == 0  # healthy blocks keep their bits (gate or not)
    assert 0 < changed[0].sum() < S and 0 < changed[-1].sum() < S
    assert r["fired"] > 0 and 0.0 < r["r_max"] < 1.0 and r["nonfinite"] == 0
    # a second pass fires nowhere
    again = O.apply_bounds(u, 0.0, bd)
    assert again["fired"] == 0
