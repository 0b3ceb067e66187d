"""The contract between prepare and rhs (src/evolution.jl:1376-1384): rhs! reads the working
array as the last prepare! left it. The C ABI keeps a generation counter, so that tgh_rhs
refuses with TGH_ERR_STALE once another verb has written the working array, instead of
silently computing the right-hand side of whatever that verb left there."""
import pytest
import torch

pytestmark = pytest.mark.gpu


def _stale(tgh, P, du, t):
    with pytest.raises(tgh._abi.TGHError) as e:
        P.rhs(du, t)
    assert e.value.code == tgh._abi.TGH_ERR_STALE
    return str(e.value)


def test_rhs_refuses_a_working_array_another_verb_wrote(tgh):
    c = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=2.0, r0=0.8, r1=1.3, gauge="algebraic")
    f = tgh.gh_forest(c, 8, 2)
    P = tgh.GHProblem(c, f, 4, margin_check=False)
    u = P.initial_state(P.statevector(), 0.0)
    du = torch.zeros_like(u)
    assert "no tgh_prepare yet" in _stale(tgh, P, du, 0.0)
    P.prepare(u, 0.0)
    P.rhs(du, 0.0)
    ref = du.clone()
    assert P.prepare_generation() == (1, True)
    # verbs that do not touch the working array leave it current
    P.max_speed(u, 0.0)
    P.rhs(du, 0.0)
    assert torch.equal(du, ref)
    # a monitor prepares for itself: rhs must be prepared again
    P.gh_constraint(u, 0.0)
    assert "constraint monitor" in _stale(tgh, P, du, 0.0)
    assert P.prepare_generation() == (1, False)
    P.prepare(u, 0.0)
    P.error_norm(u, 0.0)
    assert "tgh_error_norm" in _stale(tgh, P, du, 0.0)
    P.prepare(u, 0.0)
    v = u.clone()
    P.rk4_step(v, 0.0, 0.01)
    assert "tgh_rk4_step" in _stale(tgh, P, du, 0.0)
    P.prepare(u, 0.0)
    P.step_batched(v, 0.0, 0.01, 1)
    assert "tgh_step_batched" in _stale(tgh, P, du, 0.0)
    # settle is a prepare of its state; gh_rhs prepares itself
    P.settle(u, 0.0)
    P.rhs(du, 0.0)
    assert torch.equal(du, ref)
    P.gh_constraint(u, 0.0)
    P.gh_rhs(du, u, 0.0)
    assert torch.equal(du, ref)
    # six fills by tgh_prepare and settle and gh_rhs, four more by the RK4 step's stages
    assert P.prepare_generation() == (10, True)
    P.close()
