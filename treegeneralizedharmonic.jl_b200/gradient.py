"""Gradients of the masked error against the analytic Kerr solution.

The loss is the reference's masked, volume-weighted L2 error of the state against the analytic
solution over the evolved points (r >= r_1; src/constraints.jl:311-396), after n RK4 steps of
the plain FP64 form from the analytic data plus seeded perturbation modes. Its parameters:

    rho_max, ramp    the interior layer's relaxation rate and ramp width (w_ramp = rho_ramp)
    damp_near        the damping strength (GaussianDamping's value at the hole)
    trail_ramp       the trailing ramp of the reference's :fitted interior; this static sphere
                     has none, so the loss does not depend on it and its derivative is 0
    a0 .. a7         the amplitudes of the 8 seeded perturbation modes

Two ways to the same derivatives (exact to roundoff):
  gradient          forward-mode tangents, one tangent-linear run of the step per parameter
                    (tgh_tangent_rk4_step); no checkpoints, the tangent travels with the state
  gradient_adjoint  one reverse sweep of the adjoint step (tgh_adjoint_rk4_step, adjoint.py)
                    with checkpointed recomputation: the gradient with respect to the whole
                    initial state at once, the modes' amplitudes read off it, the layer's and
                    damping's parameters accumulated along the sweep
`MaskedError` wraps the loss and its gradient as a torch.autograd.Function (method "tangent" or
"adjoint"); adjoint.MaskedErrorOfState differentiates with respect to the initial state itself.
"""
import numpy as np
import torch

from .cases import kerr_schild_case
from .initialdata import perturbation
from .problem import GHProblem

NAMES = ("rho_max", "ramp", "damp_near", "trail_ramp") + tuple(f"a{m}" for m in range(8))
NOMINAL = (4.0, 0.5, 1.0, 0.5) + (1e-5,) * 8


class MaskedErrorStudy:
    """The static spinning hole M = 1, a = 7/10 on a forest, evolved nsteps steps of dt from the
    analytic data plus sum_m a_m phi_m, and its masked error at the end."""

    def __init__(self, forest, q=4, nsteps=40, dt=None, M=1.0, a=0.7, r0=0.8, r1=1.3, eps_ko=0.5):
        self.forest, self.q, self.nsteps = forest, int(q), int(nsteps)
        self.M, self.a, self.r0, self.r1, self.eps_ko = M, a, r0, r1, eps_ko
        self.modes = []
        for m in range(8):
            scale = np.zeros((20, 8))
            scale[:, m] = 1.0
            self.modes.append(torch.from_numpy(perturbation(forest, 1.0, scale=scale)).cuda())
        self.halfwidth = -float(forest.lo[0])
        P = self.problem(NOMINAL)
        u = P.initial_state(P.statevector(), 0.0)
        hmin = forest.h0 / 2 ** int(forest.level.max())
        self.dt = 0.25 * hmin / P.max_speed(u, 0.0) if dt is None else float(dt)
        self.t_end = self.nsteps * self.dt

    def case(self, params):
        rho_max, ramp, near = float(params[0]), float(params[1]), float(params[2])
        gamma0 = {"near": near, "far": 1.0 / (10.0 * self.M), "width": 3.0 * self.M, "c0": (0.0, 0.0, 0.0),
                  "v": (0.0, 0.0, 0.0)}
        return kerr_schild_case(M=self.M, a=self.a, halfwidth=self.halfwidth, r0=self.r0, r1=self.r1,
                                rho_max=rho_max, w_ramp=ramp, rho_ramp=ramp, gamma0=gamma0, gauge="sampled",
                                eps_ko=self.eps_ko)

    def problem(self, params):
        return GHProblem(self.case(params), self.forest, self.q, margin_check=False)

    def initial(self, P, params):
        u = P.initial_state(P.statevector(), 0.0)
        for m in range(8):
            u += float(params[4 + m]) * self.modes[m]
        return u

    def loss(self, params):
        """The masked L2 error after nsteps plain-form FP64 RK4 steps."""
        P = self.problem(params)
        u = self.initial(P, params)
        for n in range(self.nsteps):
            P.rk4_step(u, n * self.dt, self.dt)
        return P.error_norm(u, self.t_end)[0]

    def gradient(self, params):
        """(loss, d loss / d params) with one tangent-linear run per parameter."""
        P = self.problem(params)
        grad = np.zeros(len(NAMES))
        loss = None
        for i, name in enumerate(NAMES):
            if name == "trail_ramp":
                continue  # no :fitted interior: the loss does not depend on it
            u = self.initial(P, params)
            ut = self.modes[i - 4].clone() if name.startswith("a") else torch.zeros_like(u)
            direction = "state" if name.startswith("a") else name
            for n in range(self.nsteps):
                P.tangent_rk4_step(u, ut, n * self.dt, self.dt, direction)
            l2, dl2 = P.tangent_error_norm(u, ut, self.t_end)
            loss = l2 if loss is None else loss
            grad[i] = dl2
        return loss, grad

    def gradient_adjoint(self, params, every=8):
        """(loss, d loss / d params, d loss / d u0) from one reverse sweep (adjoint.py) with a
        checkpoint every `every` steps: the parameters' part accumulated along the sweep, the
        amplitudes' as the state gradient against each mode."""
        from .adjoint import masked_error_adjoint
        P = self.problem(params)
        u0 = self.initial(P, params)
        loss, lam, th = masked_error_adjoint(P, u0, 0.0, self.dt, self.nsteps, every)
        grad = np.zeros(len(NAMES))
        grad[0:3] = th
        for m in range(8):
            grad[4 + m] = float(torch.dot(lam, self.modes[m]))
        return loss, grad, lam

    def finite_differences(self, params, rel=1e-3, i=None):
        """Central differences of the loss, step rel * |p| (rel for a zero parameter)."""
        idx = range(len(NAMES)) if i is None else [i]
        out = np.zeros(len(NAMES))
        for k in idx:
            p = np.array(params, dtype=float)
            h = rel * (abs(p[k]) if p[k] != 0.0 else 1.0)
            p[k] += h
            lp = self.loss(p)
            p[k] -= 2.0 * h
            lm = self.loss(p)
            out[k] = (lp - lm) / (2.0 * h)
        return out


class MaskedError(torch.autograd.Function):
    """loss = MaskedError.apply(params, study): the masked error as a function of the 12
    parameters (NAMES order), differentiable through the forward-mode tangents."""

    @staticmethod
    def forward(ctx, params, study, method="tangent"):
        p = params.detach().cpu().numpy()
        if method == "adjoint":
            loss, grad, _ = study.gradient_adjoint(p)
        else:
            loss, grad = study.gradient(p)
        ctx.save_for_backward(torch.as_tensor(grad, dtype=params.dtype, device=params.device))
        return torch.as_tensor(loss, dtype=params.dtype, device=params.device)

    @staticmethod
    def backward(ctx, g):
        (grad,) = ctx.saved_tensors
        return g * grad, None, None


def nominal_params(dtype=torch.float64):
    return torch.tensor(NOMINAL, dtype=dtype)


__all__ = ["NAMES", "NOMINAL", "MaskedErrorStudy", "MaskedError", "nominal_params"]
