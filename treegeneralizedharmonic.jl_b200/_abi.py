"""ctypes mirror of include/tgh.h and the loader of the native library.

The structs below must match include/tgh.h field for field; tests check their sizes and
offsets against the C compiler's.
"""
import ctypes
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "lib" / "libtgh_b200.so"

(TGH_OK, TGH_ERR_ARG, TGH_ERR_NONFINITE, TGH_ERR_SPEED, TGH_ERR_RADII, TGH_ERR_TIMEOUT, TGH_ERR_CUDA, TGH_ERR_NOMEM,
 TGH_ERR_STALE) = range(9)
BG_MINKOWSKI, BG_GAUGE_WAVE, BG_SHIFTED_MINKOWSKI, BG_KERR_SCHILD, BG_HARMONIC_KERR = range(5)
GAUGE_NONE, GAUGE_SAMPLED, GAUGE_KERR_SCHILD = range(3)
DAMP_CONSTANT, DAMP_GAUSSIAN = range(2)
DISS_CONSTANT, DISS_HORIZON = range(2)
INT_NONE, INT_DAMPED, INT_FROZEN, INT_PASTED, INT_FITTED = range(5)
PREC_FP64, PREC_MIXED = range(2)
MASK_INTERIOR, MASK_ALL = range(2)
TGH_PI_L1, TGH_PI_TMA = range(2)
NDIAG = 10  # diag slots per block: C_a (0..3), H (4), M_i (5..7), mask (8), tau (9)

D3 = ctypes.c_double * 3
D4 = ctypes.c_double * 4
I3 = ctypes.c_int * 3


class Background(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("A", ctypes.c_double), ("d", ctypes.c_double),
                ("M", ctypes.c_double), ("a", ctypes.c_double), ("boost", D3), ("translate", D4)]


class Config(ctypes.Structure):
    _fields_ = [("q", ctypes.c_int), ("bg", Background), ("gauge", ctypes.c_int),
                ("ks_M", ctypes.c_double), ("ks_spin", D3), ("ks_velocity", D3),
                ("damping", ctypes.c_int), ("gamma0", ctypes.c_double),
                ("damp_near", ctypes.c_double), ("damp_far", ctypes.c_double),
                ("damp_width", ctypes.c_double), ("damp_c0", D3), ("damp_v", D3),
                ("gamma2", ctypes.c_double), ("dissipation", ctypes.c_int),
                ("eps_ko", ctypes.c_double), ("eps_out", ctypes.c_double), ("eps_in", ctypes.c_double),
                ("eps_r1", ctypes.c_double), ("eps_rh", ctypes.c_double), ("eps_c0", D3), ("eps_v", D3),
                ("interior", ctypes.c_int), ("int_c0", D3), ("int_v", D3), ("r0", ctypes.c_double),
                ("r1", ctypes.c_double), ("rho_max", ctypes.c_double), ("w_ramp", ctypes.c_double),
                ("rho_ramp", ctypes.c_double), ("precision", ctypes.c_int), ("target_rate", ctypes.c_int)]


class Mesh(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int), ("nblocks", ctypes.c_int), ("lo", D3), ("h0", ctypes.c_double),
                ("cells0", I3), ("periodic", I3), ("level", ctypes.POINTER(ctypes.c_int32)),
                ("corner", ctypes.POINTER(ctypes.c_int32))]


# every entry point include/tgh.h declares, with its ctypes signature
_VP = ctypes.c_void_p
_D = ctypes.c_double
class BoundsC(ctypes.Structure):
    """tgh_bounds: StateBounds (src/bounds.jl:81-147)."""
    _fields_ = [(n, ctypes.c_double) for n in ("alpha_min", "alpha_max", "lambda_min", "lambda_max", "beta_max",
                                               "K_max", "r_gate")]


SIGNATURES = {
    "tgh_problem_create": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(Mesh), _VP, ctypes.c_int,
                                          ctypes.POINTER(_VP)]),
    "tgh_problem_destroy": (None, [_VP]),
    "tgh_last_error": (ctypes.c_char_p, [_VP]),
    "tgh_state_length": (ctypes.c_size_t, [_VP]),
    "tgh_work_length": (ctypes.c_size_t, [_VP]),
    "tgh_copy_work": (ctypes.c_int, [_VP, _VP]),
    "tgh_copy_work_blocks": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _VP]),
    "tgh_prepare": (ctypes.c_int, [_VP, _VP, _D]),
    "tgh_prepare_generation": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_int)]),
    "tgh_rhs": (ctypes.c_int, [_VP, _VP, _D, _VP]),
    "tgh_gh_rhs": (ctypes.c_int, [_VP, _VP, _VP, _D, _VP]),
    "tgh_settle": (ctypes.c_int, [_VP, _VP, _D]),
    "tgh_stage_limit": (ctypes.c_int, [_VP, _VP, _D]),
    "tgh_step_limit": (ctypes.c_int, [_VP, _VP, _D]),
    "tgh_max_speed": (ctypes.c_int, [_VP, _VP, _D, ctypes.POINTER(_D)]),
    "tgh_initial_state": (ctypes.c_int, [_VP, _VP, _D]),
    "tgh_fill_counts": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_longlong)]),
    "tgh_set_target": (ctypes.c_int, [_VP, _VP, _D]),
    "tgh_fill_target_snapshot": (ctypes.c_int, [_VP, _VP, _D, _D]),
    "tgh_fill_target_analytic": (ctypes.c_int, [_VP, _D, _D, _D]),
    "tgh_fitted_initial_state": (ctypes.c_int, [_VP, _VP, _D, _D]),
    "tgh_copy_target": (ctypes.c_int, [_VP, _VP]),
    "tgh_rk4_step": (ctypes.c_int, [_VP, _VP, _D, _D]),
    "tgh_rk4_step_blocks": (ctypes.c_int, [_VP, _VP, _D, _D]),
    "tgh_set_variant": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "tgh_adjoint_error_norm": (ctypes.c_int, [_VP, _VP, _D, ctypes.POINTER(_D), _VP]),
    "tgh_adjoint_rhs": (ctypes.c_int, [_VP, _VP, _D, _VP, _VP, ctypes.POINTER(_D)]),
    "tgh_adjoint_rk4_step": (ctypes.c_int, [_VP, _VP, _D, _D, _VP, ctypes.POINTER(_D)]),
    "tgh_get_variant": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int)]),
    "tgh_set_wait_limit": (ctypes.c_int, [_VP, ctypes.c_longlong]),
    "tgh_device_status": (ctypes.c_int, [_VP]),
    "tgh_step_batched": (ctypes.c_int, [_VP, _VP, _D, _D, ctypes.c_int]),
    "tgh_error_norm": (ctypes.c_int, [_VP, _VP, _D, ctypes.POINTER(_D), ctypes.POINTER(_D)]),
    "tgh_gh_constraint": (ctypes.c_int, [_VP, _VP, _D, ctypes.c_int]),
    "tgh_adm_constraint": (ctypes.c_int, [_VP, _VP, _D, ctypes.c_int, _VP]),
    "tgh_constraint_norms": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_D)]),
    "tgh_tau": (ctypes.c_int, [_VP, _VP, _D, ctypes.c_int, _D, _D, ctypes.POINTER(_D)]),
    "tgh_firing": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.POINTER(_D), ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_int)]),
    "tgh_transfer": (ctypes.c_int, [_VP, _VP, _VP, _D, _VP]),
    "tgh_diag_length": (ctypes.c_size_t, [_VP]),
    "tgh_copy_diag": (ctypes.c_int, [_VP, _VP]),
    "tgh_bounds_check": (ctypes.c_int, [ctypes.POINTER(BoundsC), ctypes.c_char_p, ctypes.c_int]),
    "tgh_apply_bounds": (ctypes.c_int, [_VP, _VP, _D, ctypes.POINTER(BoundsC), ctypes.POINTER(ctypes.c_long),
                                        ctypes.POINTER(ctypes.c_long), ctypes.POINTER(_D)]),
    "tgh_set_bounds": (ctypes.c_int, [_VP, ctypes.POINTER(BoundsC)]),
    "tgh_bounds_accounting": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(_D)]),
    "tgh_max_speed_noalloc": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(Mesh), _VP, _D, _VP,
                                             ctypes.POINTER(_D), ctypes.c_char_p, ctypes.c_int]),
    "tgh_tangent_rhs": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP, _D, ctypes.c_int]),
    "tgh_tangent_rk4_step": (ctypes.c_int, [_VP, _VP, _VP, _D, _D, ctypes.c_int]),
    "tgh_tangent_error_norm": (ctypes.c_int, [_VP, _VP, _VP, _D, ctypes.POINTER(_D), ctypes.POINTER(_D)]),
    "tgh_partition": (ctypes.c_int, [ctypes.POINTER(Mesh), ctypes.c_int, _VP]),
    "tgh_shard_plan": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(Mesh), _VP, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, _VP, _VP, _VP, _VP, ctypes.c_char_p, ctypes.c_int]),
    "tgh_problem_create_shard": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(Mesh), _VP, ctypes.c_int,
                                                ctypes.c_int, _VP, ctypes.c_int, ctypes.POINTER(_VP)]),
    "tgh_shard_phases": (ctypes.c_int, [_VP]),
    "tgh_shard_counts": (ctypes.c_int, [_VP, ctypes.c_int, _VP, _VP]),
    "tgh_shard_begin": (ctypes.c_int, [_VP, _VP]),
    "tgh_shard_pack": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _VP]),
    "tgh_shard_unpack": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _VP]),
    "tgh_shard_fill": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _D, _D]),
    "tgh_shard_rhs": (ctypes.c_int, [_VP, ctypes.c_int, _D, _D]),
    "tgh_shard_end": (ctypes.c_int, [_VP, _VP]),
}
EXTRA_SIGNATURES = {
    "tgh_fp64_probe": (ctypes.c_double, [_VP, ctypes.c_int]),
    "tgh_time_rhs": (ctypes.c_int, [_VP, _VP, _D, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_D)]),
    "tgh_time_monitor": (ctypes.c_int, [_VP, _VP, _D, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_D)]),
    "tgh_copy_hsrc": (ctypes.c_int, [_VP, _VP]),
    "tgh_point_physics": (ctypes.c_int, [_VP, _D, ctypes.POINTER(_D), ctypes.POINTER(_D)]),
    "tgh_last_launch_count": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_long)]),
}

_lib = None


def load_library(path=None):
    """Load libtgh_b200.so (built in-tree by `make` in this package directory)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"the native library {p} is missing: build it with __graft_entry__.build() "
                           f"or `make -C {_HERE}`; there is no fallback path")
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in {**SIGNATURES, **EXTRA_SIGNATURES}.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class TGHError(RuntimeError):
    """A non-zero status from the native library, with its message."""

    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code
