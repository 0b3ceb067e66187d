"""Cases: a background, a box, its boundaries and the parameters the right-hand side reads.

Mirrors the reference's GHCase builders (src/initialdata.jl:158-311, 860-1326):
minkowski_case, gauge_wave_case, shifted_minkowski_case and the hole cases
(kerr_schild_case / hole_case). A Case turns into the POD `tgh_config` of include/tgh.h.
"""
from dataclasses import dataclass, field
import math

from . import _abi


@dataclass
class Case:
    background: dict                      # kind + parameters of the metric
    box: tuple                            # ((lo_x, hi_x), (lo_y, hi_y), (lo_z, hi_z))
    periodic: tuple = (True, True, True)
    eps_ko: float = 0.0                   # a number, or a dict for HorizonDissipation
    gamma0: object = 0.0                  # a number (ConstantDamping) or a dict (GaussianDamping)
    gamma2: float = 0.0
    interior: dict = None                 # sphere Interior: variant, c0, v, r0, r1, rho_max, w_ramp, rho_ramp
    gauge: str = "none"                   # "none" | "sampled" | "algebraic"
    ks_source: dict = None                # KerrSchildSource(M, spin, velocity)
    M: float = 1.0

    def config(self, q, precision="fp64"):
        c = _abi.Config()
        c.q = int(q)
        bg = self.background
        kinds = {"minkowski": _abi.BG_MINKOWSKI, "gauge_wave": _abi.BG_GAUGE_WAVE,
                 "shifted_minkowski": _abi.BG_SHIFTED_MINKOWSKI, "kerr_schild": _abi.BG_KERR_SCHILD,
                 "harmonic_kerr": _abi.BG_HARMONIC_KERR}
        c.bg.kind = kinds[bg["kind"]]
        c.bg.A = bg.get("A", 0.0)
        c.bg.d = bg.get("d", 1.0)
        c.bg.M = bg.get("M", 0.0)
        c.bg.a = bg.get("a", 0.0)
        for i, v in enumerate(bg.get("boost", (0.0, 0.0, 0.0))):
            c.bg.boost[i] = v
        for i, v in enumerate(bg.get("translate", (0.0, 0.0, 0.0, 0.0))):
            c.bg.translate[i] = v
        c.gauge = {"none": _abi.GAUGE_NONE, "sampled": _abi.GAUGE_SAMPLED,
                   "algebraic": _abi.GAUGE_KERR_SCHILD}[self.gauge]
        if self.ks_source:
            c.ks_M = self.ks_source["M"]
            for i in range(3):
                c.ks_spin[i] = self.ks_source["spin"][i]
                c.ks_velocity[i] = self.ks_source["velocity"][i]
        if isinstance(self.gamma0, dict):
            g = self.gamma0
            c.damping = _abi.DAMP_GAUSSIAN
            c.damp_near, c.damp_far, c.damp_width = g["near"], g["far"], g["width"]
            for i in range(3):
                c.damp_c0[i] = g["c0"][i]
                c.damp_v[i] = g.get("v", (0, 0, 0))[i]
        else:
            c.damping = _abi.DAMP_CONSTANT
            c.gamma0 = float(self.gamma0)
        c.gamma2 = float(self.gamma2)
        if isinstance(self.eps_ko, dict):
            e = self.eps_ko
            c.dissipation = _abi.DISS_HORIZON
            c.eps_out, c.eps_in, c.eps_r1, c.eps_rh = e["eps_out"], e["eps_in"], e["r_1"], e["r_h"]
            for i in range(3):
                c.eps_c0[i] = e["c0"][i]
                c.eps_v[i] = e.get("v", (0, 0, 0))[i]
        else:
            c.dissipation = _abi.DISS_CONSTANT
            c.eps_ko = float(self.eps_ko)
        if self.interior:
            it = self.interior
            c.interior = {"damped": _abi.INT_DAMPED, "frozen": _abi.INT_FROZEN, "pasted": _abi.INT_PASTED,
                          "fitted": _abi.INT_FITTED}[it.get("variant", "damped")]
            c.target_rate = 1 if it.get("target_rate", False) else 0
            for i in range(3):
                c.int_c0[i] = it["c0"][i]
                c.int_v[i] = it.get("v", (0, 0, 0))[i]
            c.r0, c.r1 = it["r0"], it["r1"]
            c.rho_max = it.get("rho_max", 4.0 / self.M)
            c.w_ramp = it.get("w_ramp", 0.5)
            c.rho_ramp = it.get("rho_ramp", 0.5)
        else:
            c.interior = _abi.INT_NONE
        c.precision = {"fp64": _abi.PREC_FP64, "mixed": _abi.PREC_MIXED}[precision]
        return c


def minkowski_case(L=1.0, eps_ko=0.0, gamma0=0.0, gamma2=0.0):
    """Flat space on a periodic box of side L (src/initialdata.jl:868-870)."""
    return Case({"kind": "minkowski"}, ((0.0, L),) * 3, (True, True, True), eps_ko, gamma0, gamma2)


def gauge_wave_case(A=1 / 20, d=1.0, eps_ko=0.0, gamma0=0.0, gamma2=0.0):
    """The Apples-with-Apples gauge wave on one periodic wavelength cubed (src/initialdata.jl:908-911)."""
    return Case({"kind": "gauge_wave", "A": A, "d": d}, ((0.0, d),) * 3, (True, True, True), eps_ko, gamma0,
                gamma2)


def shifted_minkowski_case(A=0.5, w=2.0, halfwidth=2.0, eps_ko=0.0, gamma0=0.0, gamma2=0.0):
    """Flat space in t^ = t + A w tanh(x/w): Dirichlet in x, periodic in y, z, sampled gauge
    source (src/initialdata.jl:944-947)."""
    return Case({"kind": "shifted_minkowski", "A": A, "d": w}, ((-halfwidth, halfwidth),) * 3,
                (False, True, True), eps_ko, gamma0, gamma2, gauge="sampled")


def perturbed_minkowski_case(halfwidth=1.0, eps_ko=0.5, gamma0=1.0, gamma2=0.0):
    """Minkowski on the periodic box [-1, 1]^3, the background of the Fourier-mode workload."""
    return Case({"kind": "minkowski"}, ((-halfwidth, halfwidth),) * 3, (True, True, True), eps_ko, gamma0, gamma2)


def kerr_schild_case(M=1.0, a=0.0, v=0.0, x0=0.0, halfwidth=8.0, r0=0.8, r1=1.3, rho_max=None,
                     variant="damped", gauge="sampled", eps_ko=0.5, gamma0=None, gamma2=0.0, w_ramp=0.5,
                     rho_ramp=0.5, margin=8, target_rate=False):
    """A Kerr-Schild hole in a Dirichlet box with the damping layer (hole_case /
    kerr_schild_case, src/initialdata.jl:1044-1300). The hole sits at (x0 + v t, 0, 0): the
    background is translate(boost(KerrSchild(M, a), (-v, 0, 0)), (0, x0, 0, 0)). A moving hole
    needs the algebraic gauge source. The default damping is GHSO2's Gaussian: 1/M at the hole,
    1/(10 M) far away, width 3 M. variant "fitted" relaxes the layer and core toward the problem's
    target cache (GHProblem.fill_target_*, set_target), with target_rate feeding its rate forward."""
    if v != 0.0 and gauge == "sampled":
        raise ValueError("a moving hole's gauge source depends on time: pass gauge='algebraic'")
    bg = {"kind": "kerr_schild", "M": M, "a": a, "boost": (-v, 0.0, 0.0), "translate": (0.0, x0, 0.0, 0.0)}
    centre = (x0, 0.0, 0.0)
    vel = (v, 0.0, 0.0)
    if gamma0 is None:
        gamma0 = {"near": 1.0 / M, "far": 1.0 / (10.0 * M), "width": 3.0 * M, "c0": centre, "v": vel}
    interior = None
    if variant is not None:
        interior = {"variant": variant, "c0": centre, "v": vel, "r0": r0, "r1": r1,
                    "rho_max": 4.0 / M if rho_max is None else rho_max, "w_ramp": w_ramp, "rho_ramp": rho_ramp,
                    "margin": margin, "target_rate": bool(target_rate)}
    ks = {"M": M, "spin": (0.0, 0.0, a), "velocity": vel}
    return Case(bg, ((-halfwidth, halfwidth),) * 3, (False, False, False), eps_ko, gamma0, gamma2, interior,
                gauge, ks, M)


def harmonic_kerr_case(M=1.0, a=0.0, v=0.0, x0=0.0, halfwidth=8.0, r0=0.8, r1=1.3, rho_max=None,
                       variant="damped", gauge="none", eps_ko=0.5, gamma0=None, gamma2=0.0, w_ramp=0.5,
                       rho_ramp=0.5, margin=8, target_rate=False):
    """A hole in fully harmonic Cartesian coordinates (harmonic_kerr_case,
    src/initialdata.jl:1300-1326): the background is translate(boost(Harmonic(M, a), (-v, 0, 0)),
    (0, x0, 0, 0)), horizon penetrating and harmonic, so H = 0 exactly and no gauge source is
    needed, moving or not (a boost of a harmonic chart is harmonic). Every other keyword is
    kerr_schild_case's. The chart's singular set is the disk x^2 + y^2 <= a^2, z = 0, which the
    frozen core must contain (r0 > |a|)."""
    if not abs(a) < M:
        raise ValueError("the harmonic chart needs |a| < M")
    c = kerr_schild_case(M=M, a=a, v=v, x0=x0, halfwidth=halfwidth, r0=r0, r1=r1, rho_max=rho_max,
                         variant=variant, gauge="algebraic" if gauge == "algebraic" else "none", eps_ko=eps_ko,
                         gamma0=gamma0, gamma2=gamma2, w_ramp=w_ramp, rho_ramp=rho_ramp, margin=margin,
                         target_rate=target_rate)
    c.background = dict(c.background, kind="harmonic_kerr")
    c.gauge = gauge
    if gauge != "algebraic":
        c.ks_source = None
    return c


def horizon_min_radius(M, a, v=0.0, chart="kerr_schild"):
    """The smallest coordinate radius of the horizon, Lorentz-contracted along the motion: the
    spheroidal radius r_+ = M + sqrt(M^2 - a^2) in Kerr-Schild coordinates, r_+ - M =
    sqrt(M^2 - a^2) in the harmonic chart (on the spin axis)."""
    r = math.sqrt(M * M - a * a) + (M if chart == "kerr_schild" else 0.0)
    return r * math.sqrt(1.0 - v * v)
