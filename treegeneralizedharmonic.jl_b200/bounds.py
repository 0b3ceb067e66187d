"""The range projection's ranges and gate (src/bounds.jl:81-247).

StateBounds holds the ranges bounds_project keeps the state inside: the lapse, every eigenvalue
of the spatial metric, the shift's norm and the momentum's scale (alpha/sqrt(gamma)) Pi, at the
points r < r_gate from the interior's centre. The projection itself runs on the GPU
(GHProblem.apply_bounds, or set_bounds for the stage limiter of the plain RK4 step).
"""
import ctypes
import math
from dataclasses import dataclass

from . import _abi


@dataclass(frozen=True)
class StateBounds:
    """StateBounds(alpha_min, alpha_max, lambda_min, lambda_max, beta_max, K_max, r_gate): no
    defaults, as in the reference; the constructor refuses what cannot be a range (the checks of
    src/bounds.jl:106-147, made by the library) with ValueError."""
    alpha_min: float
    alpha_max: float
    lambda_min: float
    lambda_max: float
    beta_max: float
    K_max: float
    r_gate: float

    def __post_init__(self):
        buf = ctypes.create_string_buffer(512)
        if _abi.load_library().tgh_bounds_check(ctypes.byref(self.to_c()), buf, 512) != 0:
            raise ValueError(buf.value.decode())

    def to_c(self):
        return _abi.BoundsC(*(float(getattr(self, n)) for n in
                              ("alpha_min", "alpha_max", "lambda_min", "lambda_max", "beta_max", "K_max", "r_gate")))

    def as_tuple(self):
        return (self.alpha_min, self.alpha_max, self.lambda_min, self.lambda_max, self.beta_max, self.K_max,
                self.r_gate)


def default_bounds(M, r_gate):
    """The reference's proposed ranges (src/bounds.jl:150-175): alpha in [1/50, 50], lambda in
    [1/100, 1000], |beta| <= 10, K_max = 100/M; r_gate has no default."""
    return StateBounds(1 / 50, 50.0, 1 / 100, 1000.0, 10.0, 100.0 / M, float(r_gate))


def _interior(case):
    it = case.interior
    if not it or it.get("variant") in (None, "none"):
        raise ValueError("the range projection's gate is a radius from the interior's centre; this case has no "
                         "interior")
    return it


def layer_spacing(case, forest, t=0.0):
    """layer_spacing (src/interior.jl:1065-1075): the largest spacing of the leaves whose box meets
    the sphere r = r_1 about the interior's centre at t, and their number."""
    it = _interior(case)
    c = [it["c0"][d] + t * it["v"][d] for d in range(3)]
    h, n = 0.0, 0
    for b in range(forest.nblocks):
        hb = forest.h0 / 2 ** int(forest.level[b])
        lo = [forest.lo[d] + forest.corner[b, d] * hb for d in range(3)]
        hi = [lo[d] + forest.N * hb for d in range(3)]
        near = math.sqrt(sum(max(lo[d] - c[d], 0.0, c[d] - hi[d]) ** 2 for d in range(3)))
        far = math.sqrt(sum(max(abs(lo[d] - c[d]), abs(hi[d] - c[d])) ** 2 for d in range(3)))
        if near <= it["r1"] <= far:
            h, n = max(h, hb), n + 1
    return h, n


def default_gate(case, forest, q, t=0.0):
    """default_gate (src/bounds.jl:177-184): r_1 - 2 G h, G = q/2 + 1, h the spacing of the blocks
    containing r_1."""
    h, _ = layer_spacing(case, forest, t)
    return _interior(case)["r1"] - 2 * (q // 2 + 1) * h


def check_bounds_gate(case, forest, bounds, q, t=0.0):
    """check_bounds_gate (src/bounds.jl:196-232): the gate must lie deeper than every point an
    evolved stencil reads, r_1 - R h with R = max(q/2 + 1, sqrt(2) q/2); ValueError otherwise.
    Returns (h, R, allowed)."""
    h, _ = layer_spacing(case, forest, t)
    R = max(float(q // 2 + 1), math.sqrt(2.0) * (q // 2))
    allowed = _interior(case)["r1"] - R * h
    if not bounds.r_gate <= allowed:
        raise ValueError(f"the range projection's gate is too shallow: r_gate = {bounds.r_gate} but the layer's "
                         f"outer radius is r_1 = {_interior(case)['r1']} at a spacing h = {h}, and the stencils "
                         f"reach {R} spacings, so an evolved point reads points down to r = {allowed}; move "
                         f"r_gate inward (default_gate proposes r_1 - 2 G h) or refine around r_1")
    return h, R, allowed
