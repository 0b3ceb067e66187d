"""B200-native generalized-harmonic time stepping (the hot path of TreeGeneralizedHarmonic.jl).

The package loads as `tgh_b200` (its directory name is not a Python identifier):

    import importlib.util, sys
    spec = importlib.util.spec_from_file_location(
        "tgh_b200", "<repo>/treegeneralizedharmonic.jl_b200/__init__.py",
        submodule_search_locations=["<repo>/treegeneralizedharmonic.jl_b200"])

Public surface, named after the reference's:
  cases      minkowski_case, gauge_wave_case, shifted_minkowski_case, kerr_schild_case,
             harmonic_kerr_case, ...
  forests    gh_forest, hole_forest
  problem    GHProblem with prepare, rhs, gh_rhs, settle, stage_limit, step_limit, max_speed,
             initial_state, gh_dt, rk4_step, step_batched, gh_solve, error_norm,
             gh_constraint, adm_constraint, constraint_norms, tau, firing
  refinement Refinement, level_bounds, refine_flags, indicator_flags: the masked Loehner verdict
  shard      partition, exchange_plan, ShardedGHProblem (one rank per GPU)
  gradient   MaskedErrorStudy, MaskedError: the masked error's gradient by forward-mode tangents
             or by the reverse sweep
  adjoint    masked_error_adjoint, MaskedErrorOfState: the reverse sweep with checkpoints
  autotune   tune, recorded_choice: the right-hand side's kernel variants, timed and recorded
"""
from . import _abi
from . import bounds, checkpoint, refinement
from .bounds import StateBounds, check_bounds_gate, default_bounds, default_gate, layer_spacing
from .checkpoint import latest_checkpoint, load_checkpoint, save_checkpoint
from .refinement import Refinement, indicator_flags, level_bounds, refine_flags
from .cases import (Case, gauge_wave_case, harmonic_kerr_case, horizon_min_radius, kerr_schild_case,
                    minkowski_case, perturbed_minkowski_case, shifted_minkowski_case)
from .forest import Forest, gh_forest, hole_forest
from .initialdata import fourier_modes, perturbation
from .problem import GHProblem, fp64_peak_tflops
from .shard import ShardedGHProblem, exchange_plan, partition
from .gradient import MaskedError, MaskedErrorStudy
from .adjoint import MaskedErrorOfState, masked_error_adjoint
from . import autotune

__all__ = ["StateBounds", "check_bounds_gate", "default_bounds", "default_gate", "layer_spacing", "Case", "Forest", "GHProblem", "gauge_wave_case", "gh_forest", "hole_forest", "kerr_schild_case", "harmonic_kerr_case",
           "minkowski_case", "perturbed_minkowski_case", "shifted_minkowski_case", "horizon_min_radius",
           "fourier_modes", "perturbation", "fp64_peak_tflops", "load_library", "ShardedGHProblem",
           "exchange_plan", "partition", "MaskedError", "MaskedErrorStudy", "Refinement", "indicator_flags",
           "level_bounds", "refine_flags", "refinement", "checkpoint", "latest_checkpoint", "load_checkpoint",
           "save_checkpoint", "MaskedErrorOfState", "masked_error_adjoint", "autotune"]

load_library = _abi.load_library
