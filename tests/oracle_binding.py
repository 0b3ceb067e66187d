"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so): test infrastructure only."""
import ctypes
import subprocess
from pathlib import Path

import numpy as np

from conftest import load_package

ROOT = Path(__file__).resolve().parent.parent
LIB = ROOT / "oracle" / "_build" / "liboracle.so"
LIB_V4 = ROOT / "oracle" / "_build" / "liboracle_v4.so"  # AVX-512 build, 8 SIMD lanes


def host_has_avx512():
    try:
        return " avx512f" in Path("/proc/cpuinfo").read_text()
    except OSError:
        return False

_D = ctypes.c_double
_VP = ctypes.c_void_p
_DP = ctypes.POINTER(ctypes.c_double)


def _dp(a):
    return a.ctypes.data_as(_DP)


class Oracle:
    _inst = None

    def __init__(self, lib):
        self.lib = lib
        abi = load_package()._abi
        self.abi = abi
        sig = {
            "orc_create": (_VP, [ctypes.POINTER(abi.Config), ctypes.POINTER(abi.Mesh), ctypes.c_int, ctypes.c_char_p,
                                 ctypes.c_int]),
            "orc_destroy": (None, [_VP]),
            "orc_last_error": (ctypes.c_char_p, [_VP]),
            "orc_state_length": (ctypes.c_size_t, [_VP]),
            "orc_work_length": (ctypes.c_size_t, [_VP]),
            "orc_set_threads": (None, [ctypes.c_int]),
            "orc_set_simd_width": (ctypes.c_int, [_VP, ctypes.c_int]),
            "orc_simd_lanes": (ctypes.c_int, []),
            "orc_get_threads": (ctypes.c_int, []),
            "orc_prepare": (ctypes.c_int, [_VP, _DP, _D]),
            "orc_rhs": (ctypes.c_int, [_VP, _DP, _D, _DP]),
            "orc_gh_rhs": (ctypes.c_int, [_VP, _DP, _DP, _D, _DP]),
            "orc_copy_work": (ctypes.c_int, [_VP, _DP]),
            "orc_copy_hsrc": (ctypes.c_int, [_VP, _DP]),
            "orc_set_work": (ctypes.c_int, [_VP, _DP]),
            "orc_initial_state": (ctypes.c_int, [_VP, _DP, _D]),
            "orc_stage_limit": (ctypes.c_int, [_VP, _DP, _D]),
            "orc_set_target": (ctypes.c_int, [_VP, _DP, _D]),
            "orc_fill_target_snapshot": (ctypes.c_int, [_VP, _DP, _D, _D]),
            "orc_fill_target_analytic": (ctypes.c_int, [_VP, _D, _D, _D]),
            "orc_fitted_initial_state": (ctypes.c_int, [_VP, _DP, _D, _D]),
            "orc_copy_target": (ctypes.c_int, [_VP, _DP]),
            "orc_max_speed": (ctypes.c_int, [_VP, _DP, _D, _DP]),
            "orc_rk4_step": (ctypes.c_int, [_VP, _DP, _D, _D]),
            "orc_error_norm": (ctypes.c_int, [_VP, _DP, _D, _DP, _DP]),
            "orc_host_rhs_at": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D, _DP]),
            "orc_rhs_scale": (_D, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
            "orc_weights": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int64),
                                           ctypes.POINTER(ctypes.c_int64)]),
            "orc_weights_double": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _DP]),
            "orc_axis_stencil": (_D, [ctypes.c_int, ctypes.c_int, _DP, ctypes.c_long, ctypes.c_long]),
            "orc_mixed_stencil": (_D, [ctypes.c_int, _DP, ctypes.c_long, ctypes.c_long, ctypes.c_long]),
            "orc_metric_quantities": (None, [_DP, _DP]),
            "orc_source": (None, [ctypes.c_int, _DP, _DP, _DP, _DP, _DP, _D, _D, _DP]),
            "orc_divergences": (None, [ctypes.c_int, _DP, _DP, _DP]),
            "orc_dmetric": (None, [ctypes.POINTER(abi.Background), _DP, _DP, _DP]),
            "orc_background_state": (None, [ctypes.POINTER(abi.Background), _D, _DP, _DP, _DP, _DP, _DP]),
            "orc_gauge_source_grad": (None, [ctypes.POINTER(abi.Background), _DP, _DP, _DP]),
            "orc_algebraic_gauge_source": (None, [_D, _DP, _DP, _DP, _DP, _DP, _DP, _DP]),
            "orc_smoothstep": (_D, [_D]),
            "orc_diag_length": (ctypes.c_size_t, [_VP]),
            "orc_gh_constraint": (ctypes.c_int, [_VP, _DP, _D, ctypes.c_int, _DP]),
            "orc_adm_constraint": (ctypes.c_int, [_VP, _DP, _D, ctypes.c_int, _DP, _DP]),
            "orc_constraint_norms": (ctypes.c_int, [_VP, _DP, ctypes.c_int, ctypes.c_int, _DP]),
            "orc_ddmetric": (None, [ctypes.POINTER(abi.Background), _DP, _DP, _DP, _DP]),
            "orc_adm_at_node": (None, [_DP, _DP, _DP, _DP]),
            "orc_adm_at_node_streamed": (None, [_DP, _DP, _DP, _DP]),
            "orc_metric_derivatives_along": (None, [_DP, _DP, _DP]),
            "orc_metric_derivatives": (None, [_DP, _DP, _DP]),
            "orc_count_flops": (ctypes.c_int, [_VP, _D, ctypes.POINTER(ctypes.c_long)]),
            "orc_tau": (ctypes.c_int, [_VP, _DP, _D, ctypes.c_int, _D, _D, _DP, _DP]),
            "orc_transfer": (ctypes.c_int, [_VP, _VP, _DP, _D, _DP]),
            "orc_firing": (ctypes.c_int, [_VP, _DP, ctypes.c_int, _DP, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int)]),
            "orc_count_monitor_flops": (ctypes.c_int, [_VP, _D, ctypes.c_int, ctypes.POINTER(ctypes.c_long)]),
            "orc_bounds_project": (None, [_DP, _DP, _DP, _DP, _DP, ctypes.POINTER(ctypes.c_int)]),
            "orc_apply_bounds": (ctypes.c_int, [_VP, _DP, _D, _DP, ctypes.POINTER(ctypes.c_long),
                                                ctypes.POINTER(ctypes.c_long), ctypes.POINTER(_D)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args

    @classmethod
    def load(cls):
        if cls._inst is None:
            if not LIB.exists():
                subprocess.run(["make", "-C", str(ROOT / "oracle")], check=True, capture_output=True)
            cls._inst = cls(ctypes.CDLL(str(LIB)))
        return cls._inst

    _inst_v4 = None

    @classmethod
    def load_widest(cls):
        """The build with the host's widest SIMD lanes: the AVX-512 one (8 lanes) where the CPU
        has AVX-512, else the AVX2 one (4 lanes)."""
        if not host_has_avx512():
            return cls.load()
        if cls._inst_v4 is None:
            if not LIB_V4.exists():
                subprocess.run(["make", "-C", str(ROOT / "oracle")], check=True, capture_output=True)
            cls._inst_v4 = cls(ctypes.CDLL(str(LIB_V4)))
        return cls._inst_v4

    def lanes(self):
        return int(self.lib.orc_simd_lanes())

    def problem(self, case, forest, q, margin_check=False):
        return OracleProblem(self, case, forest, q, margin_check)

    # pointwise helpers
    def weights(self, q, m):
        num = (ctypes.c_int64 * 16)()
        den = (ctypes.c_int64 * 16)()
        n = self.lib.orc_weights(q, m, num, den)
        return [(num[i], den[i]) for i in range(n)]

    def weights_double(self, q, m):
        out = np.zeros(16)
        n = self.lib.orc_weights_double(q, m, _dp(out))
        return out[:n]

    def axis_stencil(self, q, which, data, base, stride):
        """The oracle's stencil sum (which: 1 first, 2 second derivative, 0 dissipation)."""
        return float(self.lib.orc_axis_stencil(q, which, _dp(data), int(base), int(stride)))

    def mixed_stencil(self, q, data, base, s1, s2):
        return float(self.lib.orc_mixed_stencil(q, _dp(data), int(base), int(s1), int(s2)))

    def metric_quantities(self, h):
        out = np.zeros(46)
        self.lib.orc_metric_quantities(_dp(np.ascontiguousarray(h, dtype=float)), _dp(out))
        return dict(g4=out[:16].reshape(4, 4), gu4=out[16:32].reshape(4, 4), alpha=out[32], beta=out[33:36],
                    gamu=out[36:45].reshape(3, 3), sqrtg=out[45])

    def source(self, which, h, dth, dh, Hl, dHl, g0, g2):
        out = np.zeros(10)
        args = [np.ascontiguousarray(a, dtype=float) for a in (h, dth, dh, Hl, dHl)]
        self.lib.orc_source(which, *[_dp(a) for a in args], g0, g2, _dp(out))
        return out

    def divergences(self, which, h, dh):
        out = np.zeros(4)
        a = [np.ascontiguousarray(x, dtype=float) for x in (h, dh)]
        self.lib.orc_divergences(which, _dp(a[0]), _dp(a[1]), _dp(out))
        return out

    def background(self, case):
        return case.config(4).bg

    def dmetric(self, bg, p):
        g = np.zeros(16)
        dg = np.zeros(64)
        self.lib.orc_dmetric(ctypes.byref(bg), _dp(np.ascontiguousarray(p, dtype=float)), _dp(g), _dp(dg))
        return g.reshape(4, 4), dg.reshape(4, 4, 4)

    def background_state(self, bg, t, x):
        h, Pi, dh, dtg = np.zeros(10), np.zeros(10), np.zeros(30), np.zeros(10)
        self.lib.orc_background_state(ctypes.byref(bg), t, _dp(np.ascontiguousarray(x, dtype=float)), _dp(h),
                                      _dp(Pi), _dp(dh), _dp(dtg))
        return h, Pi, dh.reshape(3, 10), dtg

    def bounds_project(self, h, Pi, bounds):
        """bounds_project(h, Pi, bounds) at one point: (h', Pi', hit, nonfinite); bounds is the
        7-tuple (alpha_min, alpha_max, lambda_min, lambda_max, beta_max, K_max, r_gate)."""
        ho, Po, fl = np.zeros(10), np.zeros(10), (ctypes.c_int * 2)()
        a = [np.ascontiguousarray(x, dtype=float) for x in (h, Pi, bounds)]
        self.lib.orc_bounds_project(*[_dp(x) for x in a], _dp(ho), _dp(Po), fl)
        return ho, Po, bool(fl[0]), bool(fl[1])

    def gauge_source_grad(self, bg, p):
        Hl, dHl = np.zeros(4), np.zeros(16)
        self.lib.orc_gauge_source_grad(ctypes.byref(bg), _dp(np.ascontiguousarray(p, dtype=float)), _dp(Hl),
                                       _dp(dHl))
        return Hl, dHl.reshape(4, 4)

    def algebraic_gauge_source(self, M, spin, vel, h, dth, dh):
        Hl, dHl = np.zeros(4), np.zeros(16)
        a = [np.ascontiguousarray(x, dtype=float) for x in (spin, vel, h, dth, dh)]
        self.lib.orc_algebraic_gauge_source(M, *[_dp(x) for x in a], _dp(Hl), _dp(dHl))
        return Hl, dHl.reshape(4, 4)

    def ddmetric(self, bg, p):
        """g, dg[a,b,c] = d_a g_bc and ddg[a,b,c,d] = d_a d_b g_cd of a background, analytic."""
        g, dg, ddg = np.zeros(16), np.zeros(64), np.zeros(256)
        self.lib.orc_ddmetric(ctypes.byref(bg), _dp(np.ascontiguousarray(p, dtype=float)), _dp(g), _dp(dg),
                              _dp(ddg))
        return g.reshape(4, 4), dg.reshape(4, 4, 4), ddg.reshape(4, 4, 4, 4)

    def adm_at_node(self, h, dg, ddg, streamed=False):
        """(H, M_x, M_y, M_z) of the Ricci assembly at one point of offset h (streamed: the
        contraction in the GPU monitor kernel's order)."""
        out = np.zeros(4)
        a = [np.ascontiguousarray(x, dtype=float).ravel() for x in (h, dg, ddg)]
        fn = self.lib.orc_adm_at_node_streamed if streamed else self.lib.orc_adm_at_node
        fn(*[_dp(x) for x in a], _dp(out))
        return out

    def metric_derivatives_along(self, h, dg10):
        out = np.zeros(14)
        a = [np.ascontiguousarray(x, dtype=float) for x in (h, dg10)]
        self.lib.orc_metric_derivatives_along(_dp(a[0]), _dp(a[1]), _dp(out))
        return dict(dal=out[0], dbeta=out[1:4], dsq=out[4], dgamu=out[5:14].reshape(3, 3))

    def metric_derivatives(self, h, dh):
        out = np.zeros(39)
        a = [np.ascontiguousarray(x, dtype=float).ravel() for x in (h, dh)]
        self.lib.orc_metric_derivatives(_dp(a[0]), _dp(a[1]), _dp(out))
        return dict(dal=out[:3], dbeta=out[3:12].reshape(3, 3), dA=out[12:39].reshape(3, 3, 3))


class OracleProblem:
    def __init__(self, orc, case, forest, q, margin_check=False):
        self.orc, self.lib = orc, orc.lib
        self.case, self.forest, self.q = case, forest, q
        self._cfg = case.config(q)
        self._mesh = forest.mesh()
        err = ctypes.create_string_buffer(512)
        self.h = self.lib.orc_create(ctypes.byref(self._cfg), ctypes.byref(self._mesh), int(margin_check), err, 512)
        if not self.h:
            raise RuntimeError(err.value.decode())
        self.L = int(self.lib.orc_state_length(self.h))
        self.LW = int(self.lib.orc_work_length(self.h))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def statevector(self):
        return np.zeros(self.L)

    def set_simd_width(self, w):
        """1 (point by point) or the build's lane count; returns the width set."""
        return int(self.lib.orc_set_simd_width(self.h, int(w)))

    def initial_state(self, u, t):
        self.lib.orc_initial_state(self.h, _dp(u), t)
        return u

    def prepare(self, u, t):
        st = self.lib.orc_prepare(self.h, _dp(u), t)
        assert st == 0, self.lib.orc_last_error(self.h)

    def rhs(self, du, t, matter=None):
        st = self.lib.orc_rhs(self.h, _dp(du), t, _dp(matter) if matter is not None else None)
        assert st == 0, self.lib.orc_last_error(self.h)

    # the :fitted target cache (40 fields of the owned points per block)
    def set_target(self, tw, t_f):
        tw = np.ascontiguousarray(tw, dtype=float)
        assert tw.size == 2 * self.L
        self.lib.orc_set_target(self.h, _dp(tw), t_f)

    def fill_target_snapshot(self, u, t_f, r_fill):
        self.lib.orc_fill_target_snapshot(self.h, _dp(np.ascontiguousarray(u, dtype=float)), t_f, r_fill)

    def fill_target_analytic(self, t_f, r_fill, dt=0.0):
        self.lib.orc_fill_target_analytic(self.h, t_f, r_fill, dt)

    def fitted_initial_state(self, u, t, d_init=0.0):
        self.lib.orc_fitted_initial_state(self.h, _dp(u), t, d_init)
        return u

    def target(self):
        out = np.zeros(2 * self.L)
        self.lib.orc_copy_target(self.h, _dp(out))
        return out

    def gh_rhs(self, du, u, t, matter=None):
        self.prepare(u, t)
        self.rhs(du, t, matter)

    def work(self):
        w = np.zeros(self.LW)
        self.lib.orc_copy_work(self.h, _dp(w))
        return w

    def set_work(self, w):
        w = np.ascontiguousarray(w, dtype=float)
        assert w.size == self.LW
        self.lib.orc_set_work(self.h, _dp(w))

    def hsrc(self):
        w = np.zeros(self.L)
        self.lib.orc_copy_hsrc(self.h, _dp(w))
        return w

    def rk4_step(self, u, t, dt):
        st = self.lib.orc_rk4_step(self.h, _dp(u), t, dt)
        assert st == 0, self.lib.orc_last_error(self.h)

    def max_speed(self, u, t):
        lam = ctypes.c_double()
        st = self.lib.orc_max_speed(self.h, _dp(u), t, ctypes.byref(lam))
        return st, lam.value

    def error_norm(self, u, t):
        a, b = ctypes.c_double(), ctypes.c_double()
        self.lib.orc_error_norm(self.h, _dp(u), t, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def host_rhs_at(self, b, i, j, k, t):
        out = np.zeros(20)
        self.lib.orc_host_rhs_at(self.h, b, i, j, k, t, _dp(out))
        return out

    # the constraint monitors: a diag field set of 9 slots per block (C_a, H, M_i, mask)
    def diag(self):
        return np.zeros(int(self.lib.orc_diag_length(self.h)))

    def gh_constraint(self, diag, u, t, allpoints=False):
        self.lib.orc_gh_constraint(self.h, _dp(u), t, int(allpoints), _dp(diag))
        return diag

    def adm_constraint(self, diag, u, t, allpoints=False, matter=None):
        self.lib.orc_adm_constraint(self.h, _dp(u), t, int(allpoints), _dp(matter) if matter is not None else None,
                                    _dp(diag))
        return diag

    def transfer_from(self, src, u_src, t):
        """The regrid's transfer of src's state at t onto this problem's forest."""
        u = self.statevector()
        st = self.lib.orc_transfer(self.h, src.h, _dp(np.ascontiguousarray(u_src)), t, _dp(u))
        assert st == 0, self.lib.orc_last_error(self.h)
        return u

    def tau(self, diag, u, t, eps=1 / 100, scale=None, allpoints=False):
        """The masked Loehner indicator into diag slot 9; returns (the ten maxima, scale, tau_max)."""
        out = np.zeros(12)
        self.lib.orc_tau(self.h, _dp(u), t, int(allpoints), eps, -1.0 if scale is None else scale, _dp(diag),
                         _dp(out))
        return {"scales": list(out[:10]), "scale": out[10], "tau_max": out[11]}

    def firing(self, diag, tols):
        n = len(tols)
        nb = len(self.forest.level)
        counts = np.zeros(nb * n, dtype=np.int32)
        boxes = np.zeros(6 * nb * n, dtype=np.int32)
        t = np.ascontiguousarray(tols, dtype=float)
        self.lib.orc_firing(self.h, _dp(diag), n, _dp(t), counts.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                            boxes.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        return counts.reshape(nb, n), boxes.reshape(nb, n, 6)

    def count_flops(self, t, monitor=None):
        """Algorithmic FP64 operations at the centre of block 0 of the prepared problem: the
        right-hand side, or monitor "gauge" / "adm" (the Ricci tensor contracted in the GPU
        kernel's order) / "adm_reference" (the reference's assembly); adds + multiplies +
        divides + roots."""
        out = (ctypes.c_long * 4)()
        if monitor is None:
            st = self.lib.orc_count_flops(self.h, t, out)
        else:
            st = self.lib.orc_count_monitor_flops(self.h, t, {"gauge": 0, "adm_reference": 1, "adm": 2}[monitor], out)
        assert st == 0
        return sum(out)

    def apply_bounds(self, u, t, bounds):
        """gh_bounds_kernel! over the state vector u in place; counts over the primaries."""
        fired, nonfin, rmax = ctypes.c_long(), ctypes.c_long(), ctypes.c_double()
        b = np.ascontiguousarray(bounds, dtype=float)
        assert self.lib.orc_apply_bounds(self.h, _dp(u), t, _dp(b), ctypes.byref(fired), ctypes.byref(nonfin),
                                         ctypes.byref(rmax)) == 0
        return {"fired": fired.value, "nonfinite": nonfin.value, "r_max": rmax.value}

    def constraint_norms(self, diag, weighting="volume", at_level=None):
        out = np.zeros(16)
        self.lib.orc_constraint_norms(self.h, _dp(diag), 0 if weighting == "volume" else 1,
                                      -1 if at_level is None else int(at_level), _dp(out))
        return out

    def rhs_scale(self, b, i, j, k):
        return self.lib.orc_rhs_scale(self.h, b, i, j, k)

    def stage_limit(self, u, t):
        self.lib.orc_stage_limit(self.h, _dp(u), t)
