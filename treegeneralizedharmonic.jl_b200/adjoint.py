"""Reverse-mode gradients of the masked error, with checkpointed recomputation.

The loss is the reference's masked, volume-weighted L2 error against the analytic solution
(src/constraints.jl:311-396) after n plain-form FP64 RK4 steps (src/stepping.jl:208-225). Its
gradient with respect to the whole initial state - every value of every point, not a handful of
directions - comes from one backward sweep of the adjoint step (tgh_adjoint_rk4_step), with the
gradient with respect to the interior layer's rho_max and ramp width and the damping strength
accumulated on the way.

The backward sweep needs the state at the start of every step, last step first. The forward
run keeps a checkpoint every `every` steps; the backward sweep recomputes one segment at a time
from its checkpoint (every - 1 extra steps per segment, so about one extra forward run in all)
and holds at most `every` states at once.
"""
import torch


def masked_error_adjoint(P, u0, t0, dt, nsteps, every=8):
    """(loss, d loss / d u0 as a state vector, d loss / d (rho_max, ramp, damping strength))
    for the masked error after nsteps RK4 steps of dt from u0 at t0 on problem P."""
    nsteps, every = int(nsteps), max(1, int(every))
    ckpt = {0: u0.clone()}
    u = u0.clone()
    for n in range(nsteps):
        P.rk4_step(u, t0 + n * dt, dt)
        if (n + 1) % every == 0 and n + 1 < nsteps:
            ckpt[n + 1] = u.clone()
    loss, lam = P.adjoint_error_norm(u, t0 + nsteps * dt)
    del u
    th = [0.0, 0.0, 0.0]
    for start in sorted(ckpt, reverse=True):
        stop = min(start + every, nsteps)
        states = [ckpt.pop(start)]
        for n in range(start, stop - 1):
            v = states[-1].clone()
            P.rk4_step(v, t0 + n * dt, dt)
            states.append(v)
        for n in range(stop - 1, start - 1, -1):
            P.adjoint_rk4_step(states[n - start], t0 + n * dt, dt, lam, th)
        del states
    return loss, lam, th


class MaskedErrorOfState(torch.autograd.Function):
    """loss = MaskedErrorOfState.apply(u0, P, t0, dt, nsteps): the masked error after nsteps
    steps as a function of the initial state vector u0, differentiable by the adjoint sweep
    (the counterpart of a ChainRulesCore rrule around the stepping)."""

    @staticmethod
    def forward(ctx, u0, P, t0, dt, nsteps, every=8):
        loss, lam, _ = masked_error_adjoint(P, u0.detach(), t0, dt, nsteps, every)
        ctx.save_for_backward(lam)
        return torch.as_tensor(loss, dtype=u0.dtype, device=u0.device)

    @staticmethod
    def backward(ctx, g):
        (lam,) = ctx.saved_tensors
        return g * lam, None, None, None, None, None


__all__ = ["masked_error_adjoint", "MaskedErrorOfState"]
