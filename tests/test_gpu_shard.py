"""The sharded batched step on the GPU against the unsharded one, bit for bit.

Several ranks are emulated in one process on one GPU: each is its own ShardedGHProblem (its
own leaves and halo, its own buffers), and the exchange between them is a device-to-device
copy of the peer-major send and receive segments, the layout the all-to-all of a multi-GPU
run moves. No kernel waits on another rank: the ranks are driven in lock step from the host.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

NV = 20


def _exchange(ranks, ph):
    R = len(ranks)
    soff = [np.concatenate([[0], np.cumsum(r.send_count[ph])]) for r in ranks]
    roff = [np.concatenate([[0], np.cumsum(r.recv_count[ph])]) for r in ranks]
    for r in range(R):
        for o in range(R):
            n = int(ranks[r].recv_count[ph][o])
            assert n == int(ranks[o].send_count[ph][r])
            if n:
                ranks[r].recv_buf[ph][roff[r][o] * NV:(roff[r][o] + n) * NV].copy_(
                    ranks[o].send_buf[ph][soff[o][r] * NV:(soff[o][r] + n) * NV])


def _sharded_steps(ranks, us, t, dt, nsteps):
    for s, x in zip(ranks, us):
        s.begin(x)
    for n in range(nsteps):
        tn = t + n * dt
        for st in range(4):
            for ph in range(ranks[0].phases):
                for s in ranks:
                    s.pack(st, ph)
                _exchange(ranks, ph)
                for s in ranks:
                    s.unpack(st, ph)
                    s.fill(st, ph, tn, dt)
            for s in ranks:
                s.rhs(st, tn, dt)
    for s, x in zip(ranks, us):
        s.end(x)


def _cases(tgh):
    c = tgh.kerr_schild_case(M=1.0, a=0.7, v=0.1, halfwidth=4.0, r0=0.8, r1=1.3, gauge="algebraic")
    hier = tgh.hole_forest(c, 8, 2, [3.0, 1.8, 1.4], path=((0.0, 0.0, 0.0), (0.05, 0.0, 0.0)))
    g = tgh.gauge_wave_case(eps_ko=0.5, gamma0=1.0, gamma2=-0.5)
    s = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=4.0, r0=0.8, r1=1.3, gauge="sampled")
    return {"moving_hole_hierarchy": (c, hier, 0.3), "gauge_wave_periodic": (g, tgh.gh_forest(g, 8, 3), 0.25),
            "static_hole_sampled": (s, tgh.gh_forest(s, 8, 3), 0.0)}


@pytest.mark.parametrize("name,nranks", [("moving_hole_hierarchy", 2), ("moving_hole_hierarchy", 3),
                                         ("gauge_wave_periodic", 2), ("static_hole_sampled", 4)])
def test_sharded_step_equals_unsharded(tgh, name, nranks):
    case, forest, t = _cases(tgh)[name]
    P = tgh.GHProblem(case, forest, 4, margin_check=False)
    u = P.initial_state(P.statevector(), t)
    u += torch.from_numpy(tgh.perturbation(forest, amplitude=1e-6, seed=5)).cuda()
    dt = 0.25 * (forest.h0 / 2 ** int(forest.level.max())) / 2.0
    ref = u.clone()
    P.step_batched(ref, t, dt, 2)
    owner = tgh.partition(forest, nranks)
    ranks = [tgh.ShardedGHProblem(case, forest, 4, r, nranks, owner=owner, margin_check=False)
             for r in range(nranks)]
    if nranks > 1:
        assert sum(int(r.recv_count[0].sum()) for r in ranks) > 0
    us = [r.local(u).clone() for r in ranks]
    _sharded_steps(ranks, us, t, dt, 2)
    torch.cuda.synchronize()
    for r, x in zip(ranks, us):
        assert torch.isfinite(x).all()
        assert torch.equal(x, r.local(ref)), f"{name}: rank {r.rank} of {nranks} differs"


def test_one_rank_shard_is_the_batched_step(tgh):
    case, forest, t = _cases(tgh)["moving_hole_hierarchy"]
    P = tgh.GHProblem(case, forest, 4, margin_check=False)
    u = P.initial_state(P.statevector(), t)
    dt = 0.25 * (forest.h0 / 2 ** int(forest.level.max())) / 2.0
    ref = u.clone()
    P.step_batched(ref, t, dt, 1)
    S = tgh.ShardedGHProblem(case, forest, 4, 0, 1, margin_check=False)
    x = u.clone()
    S.step(x, t, dt, 1)
    torch.cuda.synchronize()
    assert torch.equal(x, ref)


def test_plain_verbs_refuse_a_sharded_problem(tgh):
    case, forest, t = _cases(tgh)["gauge_wave_periodic"]
    S = tgh.ShardedGHProblem(case, forest, 4, 0, 2, margin_check=False)
    u = S.statevector()
    with pytest.raises(tgh._abi.TGHError, match="sharded"):
        S._check(S.lib.tgh_prepare(S._h, ctypes.c_void_p(u.data_ptr()), 0.0))
