"""The range projection on the GPU against the oracle (src/bounds.jl, test/bounds_tests.jl).

The projection is integer-like in its decisions (which blocks of a state move) and a fixed
sequence of correctly rounded operations where it moves one, so the bar is bit for bit: the
projected state vector and the counts equal the oracle's exactly. Then the claims the reference
makes of the mesh pass (:300-): written back only where it fired, idempotent, and, as the plain
RK4 step's stage limiter, a run on which it never fires is bit for bit the run without it.
"""
import numpy as np
import pytest
import torch

from test_oracle_bounds import BD, bounds_states

pytestmark = pytest.mark.gpu


def _hole(tgh, q=4, a=0.7):
    case = tgh.kerr_schild_case(M=1.0, a=a, halfwidth=2.0, r0=0.8, r1=1.3, gauge="sampled")
    return case, tgh.gh_forest(case, 8, 2)


def _random_states(tgh, oracle, forest, seed):
    """Every owned point a random state (|h| <= 5, |Pi| <= 100, most out of some range), the
    nine named states of the reference's tests among them, and a few non-finite components."""
    rng = np.random.default_rng(seed)
    N1 = forest.N + 1
    S = N1 ** 3
    u = np.empty(forest.nblocks * 20 * S)
    v = u.reshape(forest.nblocks, 20, S)
    v[:, :10] = rng.uniform(-5, 5, (forest.nblocks, 10, S)) * rng.uniform(0, 1, (forest.nblocks, 1, S)) ** 2
    v[:, 10:] = rng.uniform(-100, 100, (forest.nblocks, 10, S)) * rng.uniform(0, 1, (forest.nblocks, 1, S)) ** 2
    for n, (_, (h, P), _) in enumerate(bounds_states(tgh, oracle)):
        v[0, :10, 7 * n] = h
        v[0, 10:, 7 * n] = P
    v[1, 3, 11] = np.nan
    v[1, 15, 12] = -np.inf
    return u


@pytest.mark.parametrize("seed", [1, 2])
def test_projection_matches_oracle_bit_for_bit(tgh, oracle, seed):
    case, forest = _hole(tgh)
    P = tgh.GHProblem(case, forest, 4, margin_check=False)
    O = oracle.problem(case, forest, 4)
    u = _random_states(tgh, oracle, forest, seed)
    bounds = tgh.StateBounds(*BD[:6], 100.0)  # a gate beyond the domain: every point
    ref = u.copy()
    cr = O.apply_bounds(ref, 0.0, bounds.as_tuple())
    ug = torch.from_numpy(u).cuda()
    cg = P.apply_bounds(ug, 0.0, bounds)
    got = ug.cpu().numpy()
    assert cr["fired"] > 1000
    assert got.tobytes() == ref.tobytes(), int(np.sum(got.view(np.int64) != ref.view(np.int64)))
    assert cg == cr
    # idempotent on the state and on its flag
    again = P.apply_bounds(ug, 0.0, bounds)
    assert again["fired"] == 0 and ug.cpu().numpy().tobytes() == got.tobytes()
    P.close()


def test_the_gate_and_the_primaries(tgh, oracle):
    case, forest = _hole(tgh)
    P = tgh.GHProblem(case, forest, 4, margin_check=False)
    O = oracle.problem(case, forest, 4)
    u0 = O.initial_state(O.statevector(), 0.0)
    u = _random_states(tgh, oracle, forest, 5)
    # random states everywhere, projected only inside a gate of 1.2
    bounds = tgh.StateBounds(*BD[:6], 1.2)
    ref = u.copy()
    cr = O.apply_bounds(ref, 0.0, bounds.as_tuple())
    ug = torch.from_numpy(u).cuda()
    cg = P.apply_bounds(ug, 0.0, bounds)
    assert ug.cpu().numpy().tobytes() == ref.tobytes()
    assert cg == cr and 0 < cr["r_max"] < 1.2
    # the healthy hole's own data: nothing fires, nothing moves
    ug = torch.from_numpy(u0).cuda()
    assert P.apply_bounds(ug, 0.0, tgh.StateBounds(*BD[:6], 1.2))["fired"] == 0
    assert ug.cpu().numpy().tobytes() == u0.tobytes()
    P.close()


def test_as_the_stage_limiter_a_run_it_never_fires_on_is_the_run_without(tgh):
    # h = 1/8, so that the default gate r_1 - 2 G h = 0.55 lies inside the core
    case = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=2.0, r0=0.8, r1=1.3, gauge="sampled")
    forest = tgh.gh_forest(case, 8, 4)
    P = tgh.GHProblem(case, forest, 4, margin_check=False)
    u0 = P.initial_state(P.statevector(), 0.0)
    dt = 0.25 * forest.h0 / 2
    a, b = u0.clone(), u0.clone()
    for n in range(3):
        P.rk4_step(a, n * dt, dt)
    P.set_bounds(tgh.default_bounds(M=1.0, r_gate=tgh.default_gate(case, forest, 4)))
    for n in range(3):
        P.rk4_step(b, n * dt, dt)
    acc = P.bounds_accounting()
    assert torch.equal(a, b)
    assert acc["calls"] == 12 and acc["hits"] == 0 and np.isnan(acc["first_t"])
    with pytest.raises(tgh._abi.TGHError, match="range projection"):
        P.step_batched(b.clone(), 0.0, dt, 1)
    # a planted failure inside the gate is repaired by the next stage, and counted
    c = u0.clone()
    N1 = forest.N + 1
    S = N1 ** 3
    r = tgh.default_gate(case, forest, 4)
    x = np.stack(np.meshgrid(*[np.arange(N1)] * 3, indexing="ij"), -1).reshape(-1, 3)[:, ::-1]
    # every copy of the lattice points near the centre (the counts take each at its primary)
    planted = 0
    for blk in range(forest.nblocks):
        h = forest.h0 / 2 ** int(forest.level[blk])
        pos = forest.lo + (forest.corner[blk] + x) * h
        for i in np.nonzero(np.linalg.norm(pos, axis=1) < 0.5 * r)[0]:
            c[(blk * 20 + 4) * S + int(i)] = -3.0  # h_xx: gamma_xx = -2
            planted += 1
    assert planted > 0
    P.set_bounds(tgh.default_bounds(M=1.0, r_gate=r))
    P.rk4_step(c, 0.0, dt)
    acc = P.bounds_accounting()
    assert acc["hits"] >= 1 and acc["first_t"] == pytest.approx(0.5 * dt) and 0 < acc["r_max"] < r
    assert torch.isfinite(c).all()
    P.set_bounds(None)
    P.step_batched(b.clone(), 0.0, dt, 1)
    P.close()
