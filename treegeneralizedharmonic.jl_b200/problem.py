"""GHProblem and the verbs of the reference's stepping path, on one GPU.

Host-side mirror of src/evolution.jl:995-1560 and src/stepping.jl:91-239. Every verb is one
call into libtgh_b200.so (include/tgh.h); the state vectors are torch float64 CUDA tensors
owned by the caller. There is no CPU path: a missing library or a missing GPU raises.
"""
import ctypes

import torch

from . import _abi


def _ptr(t):
    if t is None:
        return None
    if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
        raise TypeError("state vectors are contiguous float64 CUDA tensors")
    return ctypes.c_void_p(t.data_ptr())


class GHProblem:
    """Everything one right-hand-side evaluation needs (GHProblem, src/evolution.jl:995-1149):
    the forest's fill plan, the ghosted working array, the sampled gauge source and the case's
    constants, on the current CUDA device and stream."""

    def __init__(self, case, forest, q, margin_check=True, precision="fp64", stream=None, tuned=True):
        if not torch.cuda.is_available():
            raise RuntimeError("GHProblem runs on a CUDA device; none is available")
        self.lib = _abi.load_library()
        self.case, self.forest, self.q = case, forest, int(q)
        self.margin_check, self.precision = margin_check, precision
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        self._cfg = case.config(q, precision)
        self._mesh = forest.mesh()
        h = ctypes.c_void_p()
        st = self.lib.tgh_problem_create(ctypes.byref(self._cfg), ctypes.byref(self._mesh),
                                         ctypes.c_void_p(self.stream.cuda_stream), 1 if margin_check else 0,
                                         ctypes.byref(h))
        self._h = h
        if st != _abi.TGH_OK:
            msg = self.lib.tgh_last_error(h).decode() if h.value else "allocation failed"
            self.close()
            raise _abi.TGHError(st, msg)
        self.state_length = int(self.lib.tgh_state_length(h))
        self.work_length = int(self.lib.tgh_work_length(h))
        if tuned:
            # the kernel variant the autotuner recorded as fastest for this configuration
            from .autotune import recorded_choice
            choice = recorded_choice(self)
            if choice is not None:
                self.set_variant(**choice)

    # ---- lifetime ----
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.tgh_problem_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != _abi.TGH_OK:
            raise _abi.TGHError(st, self.lib.tgh_last_error(self._h).decode())

    # ---- state vectors ----
    def statevector(self):
        return torch.zeros(self.state_length, dtype=torch.float64, device="cuda")

    def evolved_sets(self):
        """The field sets this package evolves, in segment order (src/stepping.jl:125)."""
        return (self,)

    # ---- the verbs ----
    def prepare(self, u, t):
        """prepare!(p, u, t): scatter u and fill the ghosts with the hook at t."""
        self._check(self.lib.tgh_prepare(self._h, _ptr(u), float(t)))
        return self

    def rhs(self, du, t, matter=None):
        """rhs!(du, p, t; matter): the right-hand side of the state prepare left. Raises
        TGHError(TGH_ERR_STALE) when another verb has written the working array since."""
        self._check(self.lib.tgh_rhs(self._h, _ptr(du), float(t), _ptr(matter)))

    # ---- the right-hand side's kernel variants (tgh_set_variant) ----
    PI_VARIANTS = {"l1": _abi.TGH_PI_L1, "tma": _abi.TGH_PI_TMA}

    def set_variant(self, pi="l1", threads=128, pi_mb=4):
        """The kernels the right-hand side launches: the Pi half through L1 ("l1") or from tiles
        staged by the Tensor Memory Accelerator ("tma", q = 4 and N = 32 only), the CTA size of
        the head and one-point Pi kernels, the one-point Pi kernel's resident CTAs per SM."""
        self._check(self.lib.tgh_set_variant(self._h, self.PI_VARIANTS[pi], int(threads), int(pi_mb)))

    def variant(self):
        v, t, m = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.tgh_get_variant(self._h, ctypes.byref(v), ctypes.byref(t), ctypes.byref(m)))
        name = {k: n for n, k in self.PI_VARIANTS.items()}[v.value]
        return {"pi": name, "threads": t.value, "pi_mb": m.value}

    def set_wait_limit(self, polls):
        """Polls a device-side wait may make before it gives up (negative: at once)."""
        self._check(self.lib.tgh_set_wait_limit(self._h, int(polls)))

    def device_status(self):
        """Synchronize and raise TGHError(TGH_ERR_TIMEOUT) if a device wait gave up since the
        last call."""
        self._check(self.lib.tgh_device_status(self._h))

    def prepare_generation(self):
        """(number of prepare calls, whether the working array still holds the last one)."""
        g, c = ctypes.c_long(), ctypes.c_int()
        self._check(self.lib.tgh_prepare_generation(self._h, ctypes.byref(g), ctypes.byref(c)))
        return g.value, bool(c.value)

    def gh_rhs(self, du, u, t, matter=None):
        """gh_rhs!(du, u, p, t; matter) = prepare! then rhs!."""
        self._check(self.lib.tgh_gh_rhs(self._h, _ptr(du), _ptr(u), float(t), _ptr(matter)))

    def settle(self, u, t):
        """settle!(p, u, t): u as the mesh sees it (fill, then gather)."""
        self._check(self.lib.tgh_settle(self._h, _ptr(u), float(t)))
        return u

    def stage_limit(self, u, t):
        self._check(self.lib.tgh_stage_limit(self._h, _ptr(u), float(t)))

    def step_limit(self, u, t):
        self._check(self.lib.tgh_step_limit(self._h, _ptr(u), float(t)))

    def max_speed(self, u, t):
        """max_speed(p, u, t): the checked maximum characteristic speed over evolved points."""
        lam = ctypes.c_double()
        self._check(self.lib.tgh_max_speed(self._h, _ptr(u), float(t), ctypes.byref(lam)))
        return lam.value

    def initial_state(self, u, t):
        """initial_state!(u, p, t): the case's exact state, limited."""
        self._check(self.lib.tgh_initial_state(self._h, _ptr(u), float(t)))
        return u

    def fill_counts(self):
        """The fill plan's sizes: copied points, Dirichlet ghosts, prolonged points, prolongation tiles."""
        c = (ctypes.c_longlong * 4)()
        self._check(self.lib.tgh_fill_counts(self._h, c))
        return {"copies": c[0], "hooks": c[1], "prolonged": c[2], "tiles": c[3]}

    # ---- the :fitted target cache (src/fit.jl:1030-1285) ----

    def target_length(self):
        """Doubles in the target cache: 40 fields of (N+1)^3 owned points per block."""
        return 2 * self.state_length

    def default_fill_radius(self):
        """r_fill of fill_target! for the sphere interior: r_1 plus the finest spacing (the layer's
        outer radius plus one cell, src/fit.jl:1147)."""
        it = self.case.interior
        return it["r1"] + self.forest.h0 / 2 ** int(self.forest.level.max())

    def set_target(self, tw, t_f):
        """The cache from a device array of target_length() doubles (A then S per block)."""
        self._check(self.lib.tgh_set_target(self._h, _ptr(tw), float(t_f)))

    def fill_target_snapshot(self, u, t_f, r_fill=None):
        """fill_snapshot!: A = u, S = 0 inside r_fill at t_f, zero elsewhere."""
        r = self.default_fill_radius() if r_fill is None else float(r_fill)
        self._check(self.lib.tgh_fill_target_snapshot(self._h, _ptr(u), float(t_f), r))

    def fill_target_analytic(self, t_f, r_fill=None, dt=0.0):
        """The case's analytic state at t_f in place of a fit, S its centred difference over dt."""
        r = self.default_fill_radius() if r_fill is None else float(r_fill)
        self._check(self.lib.tgh_fill_target_analytic(self._h, float(t_f), r, float(dt)))

    def fitted_initial_state(self, u, t, d_init=0.0):
        """fitted_state_kernel! without the blend: the background outside r_1 - d_init, the cached
        target inside."""
        self._check(self.lib.tgh_fitted_initial_state(self._h, _ptr(u), float(t), float(d_init)))
        return u

    def target(self):
        """A copy of the target cache (a device tensor of target_length() doubles)."""
        out = torch.empty(self.target_length(), dtype=torch.float64, device="cuda")
        self._check(self.lib.tgh_copy_target(self._h, _ptr(out)))
        return out

    def gh_dt(self, u, cfl=0.25, t=0.0):
        """cfl * h_min / lambda_max (src/evolution.jl:1509-1519)."""
        hmin = self.forest.h0 / 2 ** (self.forest.nlevels - 1)
        return cfl * hmin / self.max_speed(u, t)

    def error_norm(self, u, t):
        """Masked volume-weighted (L2, Linf) of |u - u_exact| over evolved primaries."""
        l2, li = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.tgh_error_norm(self._h, _ptr(u), float(t), ctypes.byref(l2), ctypes.byref(li)))
        return l2.value, li.value

    # ---- the constraint monitors (src/constraints.jl:559-609, 848-865) ----
    MASKS = {"interior": _abi.MASK_INTERIOR, "all": _abi.MASK_ALL}

    def gh_constraint(self, u, t, mask="interior"):
        """The gauge constraint C_a of u at t into the diag field set (gh_constraint!)."""
        self._check(self.lib.tgh_gh_constraint(self._h, _ptr(u), float(t), self.MASKS[mask]))
        return self

    def adm_constraint(self, u, t, mask="interior", matter=None):
        """The ADM Hamiltonian and momentum constraints of u at t into the diag field set
        (adm_constraint!); matter as for rhs."""
        self._check(self.lib.tgh_adm_constraint(self._h, _ptr(u), float(t), self.MASKS[mask], _ptr(matter)))
        return self

    def constraint_norms(self, weighting="volume", at_level=None):
        """constraint_norms(p; weighting, at_level): masked L2 and Linf of what the monitors last
        wrote, over the primaries (each lattice point once)."""
        if weighting not in ("volume", "points"):
            raise ValueError("weighting is 'volume' or 'points'")
        out = (ctypes.c_double * 16)()
        self._check(self.lib.tgh_constraint_norms(self._h, 0 if weighting == "volume" else 1,
                                                  -1 if at_level is None else int(at_level), out))
        o = list(out)
        return {"gauge_l2": o[0:4], "gauge_linf": o[4:8], "ham_l2": o[8], "ham_linf": o[9],
                "mom_l2": o[10:13], "mom_linf": o[13:16]}

    # ---- the refinement indicator (src/refinement.jl:280-400, include/tgh.h) ----
    def tau(self, u, t, eps=1 / 100, scale=None, mask="interior"):
        """The masked Loehner indicator of u at t into the diag field set (slot 9): returns the ten
        masked maxima of |h_v| (field_scales), the scale used and tau_max."""
        out = (ctypes.c_double * 12)()
        self._check(self.lib.tgh_tau(self._h, _ptr(u), float(t), self.MASKS[mask], float(eps),
                                     -1.0 if scale is None else float(scale), out))
        o = list(out)
        return {"scales": o[:10], "scale": o[10], "tau_max": o[11]}

    def firing(self, tols):
        """The firing sweeps over the indicator the last tau wrote: per block and threshold the
        count of points above it and the bounding box (0-based nodes, low then high)."""
        tols = [float(x) for x in tols]
        n = len(tols)
        nb = self.forest.nblocks
        counts = (ctypes.c_int * (nb * n))()
        boxes = (ctypes.c_int * (6 * nb * n))()
        self._check(self.lib.tgh_firing(self._h, n, (ctypes.c_double * n)(*tols), counts, boxes))
        import numpy as np
        return np.array(counts).reshape(nb, n), np.array(boxes).reshape(nb, n, 6)

    def transfer_from(self, src, u_src, t, u):
        """The state u_src of problem `src` at t onto this problem's forest, into u (the regrid's
        transfer: copies where the old forest holds the point at its level or finer, else the
        order q + 2 prolongation from the old leaf one level coarser)."""
        self._check(self.lib.tgh_transfer(self._h, src._h, _ptr(u_src), float(t), _ptr(u)))
        return u

    def diag(self):
        """A copy of the diag field set: per block 10 slots of (N+1)^3 points (C_a, H, M_i, mask, tau)."""
        d = torch.empty(int(self.lib.tgh_diag_length(self._h)), dtype=torch.float64, device="cuda")
        self._check(self.lib.tgh_copy_diag(self._h, _ptr(d)))
        return d

    # ---- the range projection (src/bounds.jl:458-825) ----
    def apply_bounds(self, u, t, bounds):
        """apply_bounds!: bounds_project at every owned point of u with r < r_gate, written back
        only where it fired. Returns the counts over the primary copies: fired, nonfinite, r_max."""
        fired, nonfin, rmax = ctypes.c_long(), ctypes.c_long(), ctypes.c_double()
        self._check(self.lib.tgh_apply_bounds(self._h, _ptr(u), float(t), ctypes.byref(bounds.to_c()),
                                              ctypes.byref(fired), ctypes.byref(nonfin), ctypes.byref(rmax)))
        return {"fired": fired.value, "nonfinite": nonfin.value, "r_max": rmax.value}

    def set_bounds(self, bounds):
        """The bounds the stage and step limiters apply (None: none); resets the accounting. The
        batched form refuses a problem with bounds."""
        self._check(self.lib.tgh_set_bounds(self._h, ctypes.byref(bounds.to_c()) if bounds is not None else None))
        return self

    def bounds_accounting(self):
        """BoundsAccounting's totals since set_bounds: calls, hits, nonfinite, r_max, first_t, first_r."""
        n, v = (ctypes.c_long * 3)(), (ctypes.c_double * 3)()
        self._check(self.lib.tgh_bounds_accounting(self._h, n, v))
        return {"calls": n[0], "hits": n[1], "nonfinite": n[2], "r_max": v[0], "first_t": v[1], "first_r": v[2]}

    # ---- derivatives: the tangent-linear plain form (include/tgh.h) ----
    TANGENTS = {"state": 0, "rho_max": 1, "ramp": 2, "damp_near": 3}

    def tangent_rhs(self, du, dut, u, ut, t, direction="state"):
        """du = gh_rhs!(u, t) and dut its derivative along (ut, direction)."""
        self._check(self.lib.tgh_tangent_rhs(self._h, _ptr(du), _ptr(dut), _ptr(u), _ptr(ut), float(t),
                                             self.TANGENTS[direction]))

    def tangent_rk4_step(self, u, ut, t, dt, direction="state"):
        """One plain-form RK4 step of u and of its tangent ut, in place."""
        self._check(self.lib.tgh_tangent_rk4_step(self._h, _ptr(u), _ptr(ut), float(t), float(dt),
                                                  self.TANGENTS[direction]))

    def tangent_error_norm(self, u, ut, t):
        """The masked L2 error of u and its derivative along ut."""
        l2, dl2 = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.tgh_tangent_error_norm(self._h, _ptr(u), _ptr(ut), float(t), ctypes.byref(l2),
                                                    ctypes.byref(dl2)))
        return l2.value, dl2.value

    # ---- reverse mode (tgh_adjoint_*) ----
    def adjoint_error_norm(self, u, t):
        """(the masked L2 error of u at t, its gradient with respect to u as a state vector)."""
        lam = torch.zeros_like(u)
        l2 = ctypes.c_double()
        self._check(self.lib.tgh_adjoint_error_norm(self._h, _ptr(u), float(t), ctypes.byref(l2), _ptr(lam)))
        return l2.value, lam

    def adjoint_rhs(self, u, t, lam_du):
        """((d du/d u)^T lam_du, lam_du . d du/d(rho_max, ramp, damping strength)) for du = gh_rhs!(u, t)."""
        lam_u = torch.empty_like(u)
        th = (ctypes.c_double * 3)()
        self._check(self.lib.tgh_adjoint_rhs(self._h, _ptr(u), float(t), _ptr(lam_du), _ptr(lam_u), th))
        return lam_u, list(th)

    def adjoint_rk4_step(self, u, t, dt, lam, th=None):
        """lam (in place): the cotangent of the state after one plain RK4 step of dt from u at t
        becomes the cotangent of u; th (a list of 3, accumulated) the parameters' cotangents."""
        acc = (ctypes.c_double * 3)(*(th if th is not None else [0.0, 0.0, 0.0]))
        self._check(self.lib.tgh_adjoint_rk4_step(self._h, _ptr(u), float(t), float(dt), _ptr(lam), acc))
        if th is not None:
            th[:] = list(acc)
        return lam

    def point_physics(self, t, x):
        """Diagnostics: the case's analytic state (h, Pi: the Dirichlet data through the core rule)
        and sampled gauge tuple (H_b, d_a H_b) at one point x, evaluated on the device: 40 values."""
        xs = (ctypes.c_double * 3)(*[float(v) for v in x])
        out = (ctypes.c_double * 40)()
        self._check(self.lib.tgh_point_physics(self._h, float(t), xs, out))
        return list(out)

    def copy_work_blocks(self, b0, nblocks):
        """Blocks b0 .. b0 + nblocks - 1 of the working array, (N+2G+1)^3 x 20 doubles each."""
        W = self.forest.N + 2 * (self.q // 2 + 1) + 1
        w = torch.empty(nblocks * 20 * W ** 3, dtype=torch.float64, device="cuda")
        self._check(self.lib.tgh_copy_work_blocks(self._h, int(b0), int(nblocks), _ptr(w)))
        return w

    def copy_work(self):
        w = torch.empty(self.work_length, dtype=torch.float64, device="cuda")
        self._check(self.lib.tgh_copy_work(self._h, _ptr(w)))
        return w

    # ---- time integration ----
    def rk4_step(self, u, t, dt):
        """One classical RK4 step, plain form (per stage: fill, RHS, stage update)."""
        self._check(self.lib.tgh_rk4_step(self._h, _ptr(u), float(t), float(dt)))

    def rk4_step_blocks(self, u, t, dt):
        """The same RK4 step in the plain per-block form: per stage one fill, then one
        right-hand-side launch and one stage update per block (the reference's block map)."""
        self._check(self.lib.tgh_rk4_step_blocks(self._h, _ptr(u), float(t), float(dt)))

    def step_batched(self, u, t, dt, nsteps):
        """nsteps RK4 steps, batched form: fused stage epilogue, one CUDA graph."""
        self._check(self.lib.tgh_step_batched(self._h, _ptr(u), float(t), float(dt), int(nsteps)))

    def time_rhs(self, u, t, mode=1, nlaunch=10):
        """Average duration (ms) of the right-hand-side kernel alone, CUDA events on this
        problem's stream; mode 1 is the batched form's kernel, 0 the plain form's."""
        ms = ctypes.c_double()
        self._check(self.lib.tgh_time_rhs(self._h, _ptr(u), float(t), int(mode), int(nlaunch), ctypes.byref(ms)))
        return ms.value

    def time_monitor(self, u, t, which="adm", nlaunch=5):
        """Average duration (ms) of a constraint monitor's kernel alone ("gauge" or "adm", the
        interior mask), CUDA events on this problem's stream after one prepare of u at t."""
        ms = ctypes.c_double()
        w = {"gauge": 0, "adm": 1}[which]
        self._check(self.lib.tgh_time_monitor(self._h, _ptr(u), float(t), w, int(nlaunch), ctypes.byref(ms)))
        return ms.value

    def last_launch_count(self):
        """Kernels the last step_batched call launched: the fill of u, the captured graph's
        kernel nodes and the gather."""
        n = ctypes.c_long()
        self._check(self.lib.tgh_last_launch_count(self._h, ctypes.byref(n)))
        return n.value

    def gh_solve(self, u, tspan, dt, batched=False):
        """Integrate u from tspan[0] to tspan[1] with RK4 steps of at most dt, the last one
        shortened to land on tspan[1] (gh_solve, src/stepping.jl:235-239)."""
        t0, t1 = float(tspan[0]), float(tspan[1])
        n = max(1, int(-(-(t1 - t0) // dt)))
        dtu = (t1 - t0) / n
        if batched:
            self.step_batched(u, t0, dtu, n)
        else:
            for i in range(n):
                self.rk4_step(u, t0 + i * dtu, dtu)
        return u


def fp64_peak_tflops(iters=4000):
    """Sustained FP64 FMA throughput of the current GPU in TFLOP/s (2 flop per FMA)."""
    lib = _abi.load_library()
    return lib.tgh_fp64_probe(ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), int(iters))
