"""The right-hand side's kernel variants: the Pi half from TMA-staged shared-memory tiles against
the one-point L1 kernel, the launch shapes, the bounded device waits and the autotuner.

Every variant computes the same arithmetic in the same order, so the state after a batched
step (and the plain form's du) must agree bit for bit across variants."""
import numpy as np
import pytest
import torch

from helpers import cases

pytestmark = pytest.mark.gpu

N32_ROWS = ("gauge_wave_q4_n32", "kerr_schild_damped_n32", "kerr_schild_algebraic_n32")
VARIANTS = [{"pi": "l1", "threads": 128, "pi_mb": 4}, {"pi": "tma", "threads": 128, "pi_mb": 4},
            {"pi": "l1", "threads": 64, "pi_mb": 3}, {"pi": "l1", "threads": 128, "pi_mb": 5},
            {"pi": "tma", "threads": 64, "pi_mb": 4}]


def _row(tgh, name):
    return next(r for r in cases(tgh) if r[0] == name)


def _state(tgh, P, forest, t):
    u = P.initial_state(P.statevector(), t)
    g = torch.Generator(device="cuda").manual_seed(3)
    return u + 1e-6 * torch.randn(u.shape, dtype=torch.float64, device="cuda", generator=g)


@pytest.mark.parametrize("name", N32_ROWS)
def test_variants_give_the_same_bits(tgh, name):
    _, case, forest, q, t = _row(tgh, name)
    P = tgh.GHProblem(case, forest, q, margin_check=False, tuned=False)
    u0 = _state(tgh, P, forest, t)
    dt = 0.25 * forest.h0 / 4
    outs, dus = [], []
    for v in VARIANTS:
        P.set_variant(**v)
        assert P.variant() == v
        u = u0.clone()
        P.step_batched(u, t, dt, 2)
        du = torch.full_like(u0, float("nan"))
        P.gh_rhs(du, u0, t)
        P.device_status()
        outs.append(u)
        dus.append(du)
    for u, du in zip(outs[1:], dus[1:]):
        assert torch.equal(u, outs[0])
        assert torch.equal(du, dus[0])
    assert torch.isfinite(outs[0]).all()
    P.close()


def test_tma_kernel_on_a_moving_hole_hierarchy(tgh, bench_module):
    case, forest = bench_module.workload(tgh, "hierarchy_small")[:2]
    P = tgh.GHProblem(case, forest, 4, margin_check=False, tuned=False)
    u0 = _state(tgh, P, forest, 0.3)
    dt = 0.25 * forest.h0 / 2 ** int(forest.level.max()) / 2
    res = []
    for pi in ("l1", "tma"):
        P.set_variant(pi=pi)
        u = u0.clone()
        P.step_batched(u, 0.3, dt, 2)
        P.device_status()
        res.append(u)
    assert torch.equal(res[0], res[1])
    P.close()


def test_tma_variant_is_refused_where_it_does_not_apply(tgh):
    for name in ("gauge_wave_q2_n32", "kerr_schild_damped"):
        _, case, forest, q, t = _row(tgh, name)
        P = tgh.GHProblem(case, forest, q, margin_check=False, tuned=False)
        with pytest.raises(tgh._abi.TGHError) as e:
            P.set_variant(pi="tma")
        assert e.value.code == tgh._abi.TGH_ERR_ARG
        with pytest.raises(tgh._abi.TGHError):
            P.set_variant(pi="l1", threads=96)
        P.close()


def test_a_device_wait_that_runs_out_is_reported(tgh):
    """A wait limit that runs out at once: every CTA of the TMA kernel gives up on its first
    copy, records TGH_ERR_TIMEOUT, lets its copies land and leaves; the host reads the status.
    With the limit restored the same call gives the L1 kernel's bits again."""
    _, case, forest, q, t = _row(tgh, "kerr_schild_damped_n32")
    P = tgh.GHProblem(case, forest, q, margin_check=False, tuned=False)
    u0 = _state(tgh, P, forest, t)
    ref = torch.zeros_like(u0)
    P.gh_rhs(ref, u0, t)
    P.set_variant(pi="tma")
    P.set_wait_limit(-1)
    du = torch.zeros_like(u0)
    P.gh_rhs(du, u0, t)
    with pytest.raises(tgh._abi.TGHError) as e:
        P.device_status()
    assert e.value.code == tgh._abi.TGH_ERR_TIMEOUT
    P.device_status()  # the status was cleared
    P.set_wait_limit(1 << 26)
    P.gh_rhs(du, u0, t)
    P.device_status()
    assert torch.equal(du, ref)
    P.close()


def test_autotuner_records_and_applies_its_choice(tgh, tmp_path):
    from importlib import import_module
    at = import_module(tgh.__name__ + ".autotune")
    _, case, forest, q, t = _row(tgh, "kerr_schild_damped_n32")
    P = tgh.GHProblem(case, forest, q, margin_check=False, tuned=False)
    u = _state(tgh, P, forest, t)
    f = tmp_path / "tuning.json"
    res = at.tune(P, u, t, nlaunch=2, repeats=1, path=f)
    assert len(res["sweep"]) == len(at.candidates(P)) == 8
    assert all(r["ms_per_rhs"] > 0 for r in res["sweep"])
    assert res["choice"] == {k: min(res["sweep"], key=lambda r: r["ms_per_rhs"])[k] for k in ("pi", "threads", "pi_mb")}
    assert at.recorded_choice(P, path=f) == res["choice"]
    assert P.variant() == res["choice"]
    P.close()
