/*
 * tgh.h -- the C ABI of the B200-native generalized-harmonic time-stepping path.
 *
 * One shared library (libtgh_b200.so, built from treegeneralizedharmonic.jl_b200/csrc)
 * implements the verbs of TreeGeneralizedHarmonic.jl's stepping path on one GPU:
 *
 *   reference verb (TreeGeneralizedHarmonic.jl)          this ABI
 *   ---------------------------------------------------   -----------------------------
 *   GHProblem(U, schedule, case; q, t, interior)           tgh_problem_create
 *     src/evolution.jl:1034-1149
 *   prepare!(p, u, t)          src/evolution.jl:1349       tgh_prepare
 *   rhs!(du, p, t; matter)     src/evolution.jl:1386       tgh_rhs
 *   gh_rhs!(du, u, p, t)       src/evolution.jl:1327       tgh_gh_rhs
 *   settle!(p, u, t)           src/evolution.jl:1370       tgh_settle
 *   stage_limit!(u, p, t)      src/stepping.jl:91          tgh_stage_limit
 *   step_limit!(u, p, t)       src/stepping.jl:97          tgh_step_limit
 *   max_speed(p, u, t)         src/evolution.jl:1539       tgh_max_speed
 *   initial_state!(u, p, t)    src/stepping.jl:110         tgh_initial_state
 *   IRK.step!(gh_integrator(...)) src/stepping.jl:208-225  tgh_rk4_step (plain per-block form)
 *                                                          tgh_step_batched (fused, graph-captured form)
 *   error_norms / gh_error_kernel! src/constraints.jl:311-396, 716-792
 *                                                          tgh_error_norm
 *   apply_bounds! / gh_stage_limiter!, StateBounds         tgh_apply_bounds, tgh_set_bounds,
 *     src/bounds.jl:81-175, 458-663, 686-825              tgh_bounds_check, tgh_bounds_accounting
 *   gh_constraint!, adm_constraint!, constraint_norms     tgh_gh_constraint,
 *     src/constraints.jl:211-271, 432-532, 559-609, 848    tgh_adm_constraint,
 *                                                          tgh_constraint_norms
 *
 * Conventions (all as in the reference):
 *  - The state vector holds, per block, (N+1)^3 owned points (closed blocks: both face
 *    planes are owned) for 20 variables: h_ab in 0..9 and Pi_ab in 10..19, packed
 *    (tt,tx,ty,tz,xx,xy,xz,yy,yz,zz); x fastest, then y, z, variable, block
 *    (src/evolution.jl:170-178, src/pointwise.jl:22-26).
 *  - u / du pointers passed to the verbs are DEVICE pointers owned by the caller
 *    (a CuArray, a torch tensor, ...), holding tgh_state_length() doubles.
 *  - The problem owns its ghosted working array, the sampled gauge source and all
 *    scratch; no verb allocates device memory after tgh_problem_create.
 *  - rhs reads the working array as the last prepare left it (src/evolution.jl:1376-1384).
 *    Here every other verb that writes the working array (error_norm, the monitors, tau,
 *    transfer, the RK4 forms, the tangent-linear form, the sharded step) marks it
 *    overwritten, and tgh_rhs then refuses with TGH_ERR_STALE until the next tgh_prepare;
 *    settle is a prepare and keeps it current; max_speed and initial_state do not touch it.
 *  - Every entry point returns a status code and never aborts; tgh_last_error gives
 *    the message of the last failure on that problem.
 *  - A problem is bound to one CUDA stream (given at create) and is not thread-safe.
 */
#ifndef TGH_H
#define TGH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TGH_NVARS 20
#define TGH_NC 10

/* status codes (the reference throws ArgumentError with a message instead) */
enum {
  TGH_OK = 0,
  TGH_ERR_ARG = 1,        /* construction checks, src/evolution.jl:1039-1136 */
  TGH_ERR_NONFINITE = 2,  /* non-finite evolved data, src/evolution.jl:1540-1548 */
  TGH_ERR_SPEED = 3,      /* speed not finite and positive, src/evolution.jl:1551-1558 */
  TGH_ERR_RADII = 4,      /* interior radius checks, src/interior.jl:1104-1153 */
  TGH_ERR_TIMEOUT = 5,    /* a bounded device-side wait gave up */
  TGH_ERR_CUDA = 6,       /* a CUDA runtime call failed */
  TGH_ERR_NOMEM = 7,
  TGH_ERR_STALE = 8       /* tgh_rhs after another verb overwrote what tgh_prepare filled */
};

/* backgrounds (SpacetimeMetrics metrics named by the reference's cases) */
enum {
  TGH_BG_MINKOWSKI = 0,          /* h = 0 */
  TGH_BG_GAUGE_WAVE = 1,         /* ds^2 = -H dt^2 + H dx^2 + dy^2 + dz^2, H = 1 - A sin(2pi(x-t)/d) */
  TGH_BG_SHIFTED_MINKOWSKI = 2,  /* flat space in t^ = t + A w tanh(x/w) */
  TGH_BG_KERR_SCHILD = 3,        /* Kerr-Schild (M, a), spin about +z */
  TGH_BG_HARMONIC_KERR = 4       /* Kerr (M, a) in horizon-penetrating harmonic coordinates (Harmonic(M, a),
                                    src/initialdata.jl:1300-1326): the Kerr-Schild metric pulled back along
                                    x + i y = (r_H + i a) e^{i phi} sin(theta), z = r_H cos(theta) with
                                    r = r_H + M and t = T_KS - 2 M ln(r - r_-); H_a = 0 exactly */
};

/* gauge source kinds: GHProblem's HASH switch (src/evolution.jl:1099) */
enum { TGH_GAUGE_NONE = 0, TGH_GAUGE_SAMPLED = 1, TGH_GAUGE_KERR_SCHILD = 2 };
/* constraint-damping profile (src/gauge.jl:1094-1147) */
enum { TGH_DAMP_CONSTANT = 0, TGH_DAMP_GAUSSIAN = 1 };
/* Kreiss-Oliger amplitude (src/gauge.jl:1180-1266) */
enum { TGH_DISS_CONSTANT = 0, TGH_DISS_HORIZON = 1 };
/* interior variant (src/interior.jl:178-238): :none, :damped, :frozen, :pasted, and :fitted, whose
 * layer and core relax toward a target read from the problem's target cache (src/evolution.jl:
 * 517-548, 600-653; the cache src/fit.jl:1030-1055), here over the sphere interior */
enum { TGH_INT_NONE = 0, TGH_INT_DAMPED = 1, TGH_INT_FROZEN = 2, TGH_INT_PASTED = 3, TGH_INT_FITTED = 4 };
/* arithmetic of the right-hand side */
enum { TGH_PREC_FP64 = 0, TGH_PREC_MIXED = 1 };

typedef struct {
  int kind;              /* TGH_BG_* */
  double A, d;           /* gauge wave (A, wavelength d); shifted Minkowski (A, w) */
  double M, a;           /* Kerr mass and spin parameter (Kerr-Schild and harmonic charts) */
  double boost[3];       /* boost(metric, u): evaluated at Lambda(u) x, the hole moves at -u */
  double translate[4];   /* translate(metric, (t, x, y, z)), applied after the boost */
} tgh_background;

/* Everything a GHCase + GHProblem carry that the kernels read
 * (src/initialdata.jl:158-311, src/evolution.jl:995-1149). */
typedef struct {
  int q;                       /* even order 2..8; ghost width G = q/2 + 1 */
  tgh_background bg;
  int gauge;                   /* TGH_GAUGE_* */
  double ks_M;                 /* KerrSchildSource(M, spin, velocity), src/gauge.jl:257-290 */
  double ks_spin[3];
  double ks_velocity[3];
  int damping;                 /* TGH_DAMP_* */
  double gamma0;               /* ConstantDamping */
  double damp_near, damp_far, damp_width, damp_c0[3], damp_v[3]; /* GaussianDamping */
  double gamma2;
  int dissipation;             /* TGH_DISS_* */
  double eps_ko;               /* constant epsilon */
  double eps_out, eps_in, eps_r1, eps_rh, eps_c0[3], eps_v[3];   /* HorizonDissipation */
  int interior;                /* TGH_INT_* */
  double int_c0[3], int_v[3];  /* HoleCenter(c0, v) */
  double r0, r1, rho_max, w_ramp, rho_ramp;
  int precision;               /* TGH_PREC_*: FP64, or FP32 offset-metric stencils + algebra */
  int target_rate;             /* :fitted: feed the target's rate forward (GHProblem's target_rate,
                                  src/evolution.jl:1015-1018): (1 - w) d_t u_fit in the layer, d_t u_fit
                                  in the core */
} tgh_config;

/* A forest's leaves: closed vertex-centered blocks of N cells per edge (N+1 points).
 * Level l has spacing h0 / 2^l; a block's points sit at lo + (corner + i) * h_l,
 * i = 0..N, corner in the level's cell index space (a multiple of N).
 * The leaves tile the domain [lo, lo + cells0 * h0]. */
typedef struct {
  int N;
  int nblocks;
  double lo[3];
  double h0;
  int cells0[3];               /* level-0 domain extent in cells per axis */
  int periodic[3];
  const int32_t* level;        /* [nblocks] */
  const int32_t* corner;       /* [3 * nblocks] */
} tgh_mesh;

typedef struct tgh_problem tgh_problem;

/* --- construction (GHProblem, src/evolution.jl:1034-1149) --- */
int tgh_problem_create(const tgh_config* cfg, const tgh_mesh* mesh, void* cuda_stream,
                       int margin_check, tgh_problem** out);
void tgh_problem_destroy(tgh_problem* p);
const char* tgh_last_error(const tgh_problem* p);
/* doubles in one state vector: (N+1)^3 * 20 * nblocks */
size_t tgh_state_length(const tgh_problem* p);
/* doubles in the ghosted working array: (N+2G+1)^3 * 20 * blocks held (a rank of a sharded
 * problem holds its own leaves and its halo) */
size_t tgh_work_length(const tgh_problem* p);
/* the fill plan's sizes (points per fill of the batched form): counts[0] copied points (ghosts
 * from their primary, owned copies that are not primary), [1] Dirichlet ghosts, [2] prolonged
 * points of all levels, [3] prolongation tiles (0 where a level runs point by point) */
int tgh_fill_counts(const tgh_problem* p, long long counts[4]);
/* copy the working array (device to device) for inspection */
int tgh_copy_work(tgh_problem* p, double* dst);
/* the same for the blocks b0 .. b0 + nblocks - 1 of the working array (each (N+2G+1)^3 * 20
 * doubles, blocks in forest order on a problem of one rank) */
int tgh_copy_work_blocks(tgh_problem* p, int b0, int nblocks, double* dst);

/* --- the verbs (src/evolution.jl:1327-1390, src/stepping.jl:91-125) --- */
int tgh_prepare(tgh_problem* p, const double* u, double t);
/* the prepare/rhs contract as a generation counter: the number of tgh_prepare calls so far,
 * and whether the working array still holds the last one's fill (1) or another verb has
 * written it since (0, when tgh_rhs answers TGH_ERR_STALE) */
int tgh_prepare_generation(const tgh_problem* p, long* generation, int* current);
/* matter: nullable device pointer, 10 values per owned point in state layout
 * (rho, S_x, S_y, S_z, S_xx, S_xy, S_xz, S_yy, S_yz, S_zz); the GH-3 adapter
 * of src/evolution.jl:1288-1316 sampled at the owned points. */
int tgh_rhs(tgh_problem* p, double* du, double t, const double* matter);
int tgh_gh_rhs(tgh_problem* p, double* du, const double* u, double t, const double* matter);
int tgh_settle(tgh_problem* p, double* u, double t);
int tgh_stage_limit(tgh_problem* p, double* u, double t);
int tgh_step_limit(tgh_problem* p, double* u, double t);
int tgh_max_speed(tgh_problem* p, const double* u, double t, double* lambda);
int tgh_initial_state(tgh_problem* p, double* u, double t);

/* --- the :fitted target cache (src/fit.jl:1030-1285; GHProblem's target, t_target and
 * target_rate, src/evolution.jl:1009-1018) ---
 * A :fitted interior's layer and core relax toward A + (t - t_f) S read at the point, where the
 * cache holds per block 40 fields of the owned points, state layout (N+1)^3 per field: the target
 * A (the packed h, Pi; fields 0-19) at the fill time t_f and its slope S (fields 20-39). The
 * right-hand side and the steps refuse a :fitted problem (TGH_ERR_ARG) until one of the first
 * three verbs has filled the cache; every one of them needs interior = TGH_INT_FITTED.
 *   tgh_set_target            the cache from a device array of 40 (N+1)^3 nb doubles (a caller's own
 *                             fit: fill_target! with fit_target_kernel!, src/fit.jl:1134-1156)
 *   tgh_fill_target_snapshot  fill_snapshot! (src/fit.jl:1189-1222): A = u, S = 0 where the
 *                             interior radius at t_f is below r_fill, zero elsewhere
 *   tgh_fill_target_analytic  the case's analytic state at t_f (core rule included) in place of a
 *                             fit, with S its centred difference over t_f +- dt (dt = 0: S = 0), in
 *                             the same region
 *   tgh_fitted_initial_state  fitted_state_kernel! (src/fit.jl:1247-1285) without the blend: the
 *                             background's state where r >= r_1 - d_init, the cached target at t below
 *   tgh_copy_target           the cache into a device array of the same shape */
int tgh_set_target(tgh_problem* p, const double* tw, double t_f);
int tgh_fill_target_snapshot(tgh_problem* p, const double* u, double t_f, double r_fill);
int tgh_fill_target_analytic(tgh_problem* p, double t_f, double r_fill, double dt);
int tgh_fitted_initial_state(tgh_problem* p, double* u, double t, double d_init);
int tgh_copy_target(tgh_problem* p, double* out);

/* --- one classical RK4 step (IMEXRungeKutta RK4 via gh_integrator, src/stepping.jl:208-225) ---
 * plain form: per stage one ghost fill, one right-hand-side launch, one stage update */
int tgh_rk4_step(tgh_problem* p, double* u, double t, double dt);
/* plain per-block form: the same step with the reference's block-wise map (map_blocks!,
 * src/evolution.jl:1387): per stage one fill, then one right-hand-side launch and one stage
 * update per block, issued from the host. Bit for bit tgh_rk4_step's result. */
int tgh_rk4_step_blocks(tgh_problem* p, double* u, double t, double dt);
/* batched form: the state stays ghosted on the device; each stage is one fill launch and
 * one right-hand-side launch with the RK4 epilogue fused in; nsteps steps are captured
 * once as a CUDA graph and replayed. u is read before the first step and written after
 * the last. */
int tgh_step_batched(tgh_problem* p, double* u, double t, double dt, int nsteps);

/* --- the right-hand side's kernel variants (no counterpart in the reference, whose kernels
 * are compiled per problem by KernelAbstractions) ---
 * tgh_set_variant picks the kernels the right-hand side launches; the autotuner (autotune.py)
 * times them on the problem's own mesh and records the fastest per configuration:
 *   pi_variant  TGH_PI_L1:  the Pi half as one point per thread, its stencils read through L1;
 *               TGH_PI_TMA: two points per thread from tiles of the working array staged into
 *               shared memory by the Tensor Memory Accelerator (q = 4, N = 32, FP64 only);
 *   threads     CTA size of the head and one-point Pi kernels, 64 or 128;
 *   pi_mb       the one-point Pi kernel's resident CTAs per SM (its launch bound), 3, 4 or 5.
 * All variants give the same bits. A change drops the batched form's captured graph.
 * tgh_set_wait_limit bounds the polls of every device-side wait (the TMA kernel's waits for its
 * copies); a wait that runs out records TGH_ERR_TIMEOUT and its CTA writes nothing. A negative
 * limit gives up at once (for tests). tgh_device_status synchronizes the problem's stream and
 * returns (and clears) TGH_ERR_TIMEOUT if a wait gave up since the last call. */
enum { TGH_PI_L1 = 0, TGH_PI_TMA = 1 };
int tgh_set_variant(tgh_problem* p, int pi_variant, int threads, int pi_mb);
int tgh_get_variant(const tgh_problem* p, int* pi_variant, int* threads, int* pi_mb);
int tgh_set_wait_limit(tgh_problem* p, long long polls);
int tgh_device_status(tgh_problem* p);

/* --- analysis (src/constraints.jl:311-396, 716-792) ---
 * masked, volume-weighted L2 and max of |u - u_exact| over the evolved primaries */
int tgh_error_norm(tgh_problem* p, const double* u, double t, double* l2, double* linf);

/* --- constraint monitors (src/constraints.jl:211-271, 432-532, 716-865) ---
 * The monitors write the problem's diag field set: per block TGH_NDIAG slots of (N+1)^3
 * points, slot-major like the state vector. Slots 0..3 hold the gauge constraint C_a
 * (the reference's DIAG_CGH), 4 the ADM Hamiltonian constraint (DIAG_HAM), 5..7 the
 * momentum constraint M_i (DIAG_MOM), 8 the mask indicator (DIAG_MASK), 9 the refinement
 * indicator tau (DIAG_TAU, written by tgh_tau below). Each monitor
 * first runs prepare at t (scatter and fill, as _prepare_monitor! does), so the working
 * array is overwritten, and writes only its own slots and the mask.
 *   mask: TGH_MASK_INTERIOR (the interior's r >= r_1; every point without an interior) or
 *         TGH_MASK_ALL (AllPoints). A masked point holds zeros.
 *   tgh_gh_constraint    gh_constraint!(p, u, t; mask)            src/constraints.jl:559
 *   tgh_adm_constraint   adm_constraint!(p, u, t; mask, matter)   src/constraints.jl:584
 *                        matter: null, or (N+1)^3 x 10 per block (rho, S_i, S_ij packed
 *                        xx,xy,xz,yy,yz,zz), as for tgh_rhs; the constraints are then
 *                        H - 16 pi rho and M_i - 8 pi S_i
 *   tgh_constraint_norms constraint_norms(p; weighting, at_level) src/constraints.jl:848
 *                        one fold over the primaries of what the monitors last wrote;
 *                        weighting 0 = volume (h^3), 1 = points; at_level < 0: all levels.
 *                        out[16] = gauge_l2[4], gauge_linf[4], ham_l2, ham_linf, mom_l2[3],
 *                        mom_linf[3]; L2 = sqrt(sum u^2 w / evolved volume), 0 when nothing
 *                        is evolved; L-infinity keeps NaN.
 * Problems of one rank only (TGH_ERR_ARG for a shard). */
#define TGH_NDIAG 10
enum { TGH_MASK_INTERIOR = 0, TGH_MASK_ALL = 1 };
int tgh_gh_constraint(tgh_problem* p, const double* u, double t, int mask);
int tgh_adm_constraint(tgh_problem* p, const double* u, double t, int mask, const double* matter);
int tgh_constraint_norms(tgh_problem* p, int weighting, int at_level, double* out);

/* --- the refinement indicator (src/refinement.jl:170-400, 738-796) ---
 * tgh_tau: prepare at t, then field_scales (the largest |h_v| over the evolved owned points,
 *   one per component), then the masked Loehner indicator at every owned point into diag
 *   slot 9: the worst over the ten components of h and the three axes of
 *     |u+ - 2 u0 + u-| / (|u+ - u0| + |u0 - u-| + 4 eps scale)   (0 where the denominator is),
 *   zero where the mask leaves the point out; and its maximum over the mesh (tau_max).
 *   scale > 0 is the reference amplitude to use, else the largest of the ten maxima.
 *   out[12] = the ten maxima, the scale used, tau_max.
 * tgh_firing: the firing sweeps of refine_flags over slot 9, ntol (1..4) thresholds at once:
 *   per block b and threshold n the number of owned points with tau > tol[n] in
 *   counts[b * ntol + n] and the bounding box of their node indices (0-based, i j k low then
 *   i j k high; low N+1 and high -1 where none fired) in boxes[6 (b * ntol + n) + 0..5].
 *   counts and boxes are host arrays. */
int tgh_tau(tgh_problem* p, const double* u, double t, int mask, double eps, double scale, double* out);
int tgh_firing(tgh_problem* p, int ntol, const double* tol, int* counts, int* boxes);

/* --- the regrid's state transfer (TreeAMR's regrid!, driver src/driver.jl:1660-1695) ---
 * The state u_src of problem src at t onto the forest of problem dst (same case, order, block
 * size and root grid; the caller builds dst on the regridded forest): src is prepared at t
 * (its ghosts filled with this t's hook), then every owned point of every dst leaf takes its
 * lattice point's value there, copied from the finest src leaf holding it at its level or
 * finer, else prolonged (order q + 2) from the src leaf one level coarser covering it. u_dst is
 * a device state vector of dst. The transfer plans on the host and allocates (and frees) its
 * point lists on the device: it runs once per regrid. Problems of one rank only. */
int tgh_transfer(tgh_problem* dst, tgh_problem* src, const double* u_src, double t, double* u_dst);
/* the diag field set: its length in doubles, and a copy of it into a device buffer */
size_t tgh_diag_length(const tgh_problem* p);
int tgh_copy_diag(tgh_problem* p, double* out);

/* --- the range projection of the stage limiter (src/bounds.jl:81-175, 458-663, 686-825) ---
 * tgh_bounds is StateBounds: alpha_min <= alpha <= alpha_max (the lapse, alpha^2 =
 *   beta_i beta^i - g_tt), lambda_min <= every eigenvalue of gamma_ij <= lambda_max,
 *   |beta| = sqrt(beta_i gamma^ij beta_j) <= beta_max, max_ab |(alpha/sqrt(gamma)) Pi_ab| <= K_max,
 *   held at the points r < r_gate from the interior's centre.
 * tgh_bounds_check: StateBounds' own checks (every bound finite, 0 < alpha_min < 1 < alpha_max,
 *   0 < lambda_min < 1 < lambda_max, beta_max, K_max and r_gate positive). Host only; errbuf
 *   (nullable) receives the reason.
 * tgh_apply_bounds: apply_bounds!: bounds_project at every owned point of the device state
 *   vector u with r < r_gate, written back only where it fired (a point it leaves alone keeps
 *   its bits), and over the primary copies the number of points it fired at, of those with a
 *   non-finite component, and the largest r it fired at (0 when none). Needs an interior.
 * tgh_set_bounds: the problem's bounds (NULL: none). The stage and step limiters (and so
 *   tgh_rk4_step and tgh_initial_state) then apply the projection before the :pasted paste and
 *   add its counts to the problem's accounting, reset here; the batched form refuses a
 *   problem with bounds.
 * tgh_bounds_accounting: BoundsAccounting's totals: counts3 = calls, hits, non-finite hits;
 *   vals3 = the largest r fired at, the t and r of the first call that fired (NaN before). */
typedef struct {
  double alpha_min, alpha_max, lambda_min, lambda_max, beta_max, K_max, r_gate;
} tgh_bounds;
int tgh_bounds_check(const tgh_bounds* b, char* errbuf, int errlen);
int tgh_apply_bounds(tgh_problem* p, double* u, double t, const tgh_bounds* b, long* fired, long* nonfinite,
                     double* r_max);
int tgh_set_bounds(tgh_problem* p, const tgh_bounds* b);
int tgh_bounds_accounting(const tgh_problem* p, long* counts3, double* vals3);

/* --- allocation-free speed (no counterpart in the reference) ---
 * tgh_max_speed without a problem handle, for callers that cannot allocate device memory
 * (their device memory belongs to another allocator or pool, or allocation is forbidden in
 * the loop that asks for the time step). It allocates nothing: its scratch is one fixed
 * device array in the library, which holds the block table of at most
 * TGH_NOALLOC_MAX_BLOCKS blocks; larger meshes are refused with TGH_ERR_ARG. u is a device
 * state vector of mesh's layout; the result and the checks are those of tgh_max_speed. The
 * first call on a device looks up the array's address (make it before any stream capture);
 * every call shares the array, so calls that overlap on the GPU race. errbuf (nullable)
 * receives the message of a failure. */
#define TGH_NOALLOC_MAX_BLOCKS 8192
int tgh_max_speed_noalloc(const tgh_config* cfg, const tgh_mesh* mesh, const double* u, double t,
                          void* cuda_stream, double* lambda, char* errbuf, int errlen);

/* --- derivatives (the tangent-linear plain form; forward mode along one direction) ---
 * The reference's gradients of the masked error (the error of src/constraints.jl:311-396 against
 * the analytic solution) with respect to the interior layer's parameters, the damping strength
 * and the initial data, taken one direction at a time: ut is the tangent of the state u (the
 * derivative of u along the direction), and `direction` adds one parameter's own dependence:
 *   TGH_TAN_STATE      none (the initial data's amplitudes enter through ut alone)
 *   TGH_TAN_RHO_MAX    the layer's rho_max
 *   TGH_TAN_RAMP       the layer's ramp width (w_ramp and rho_ramp together)
 *   TGH_TAN_DAMP_NEAR  the damping strength (ConstantDamping's gamma0, GaussianDamping's near)
 * tgh_tangent_rhs: du = gh_rhs!(u, t) and dut its derivative (du agrees with tgh_gh_rhs's to
 * roundoff).
 * tgh_tangent_rk4_step: one plain-form RK4 step of (u, ut) together.
 * tgh_tangent_error_norm: the masked volume-weighted L2 error of u and its derivative.
 * FP64, one rank, no matter term, an interior that does not move and is not :pasted. */
enum { TGH_TAN_STATE = 0, TGH_TAN_RHO_MAX = 1, TGH_TAN_RAMP = 2, TGH_TAN_DAMP_NEAR = 3 };
int tgh_tangent_rhs(tgh_problem* p, double* du, double* dut, const double* u, const double* ut, double t,
                    int direction);
int tgh_tangent_rk4_step(tgh_problem* p, double* u, double* ut, double t, double dt, int direction);
int tgh_tangent_error_norm(tgh_problem* p, const double* u, const double* ut, double t, double* l2, double* dl2);

/* --- derivatives in reverse mode (the adjoint of the plain form; no counterpart in the reference,
 * which differentiates nothing) ---
 * The masked error's gradient with respect to the whole initial state in one backward sweep,
 * and with respect to the interior layer's rho_max and ramp width and the damping strength
 * (the directions of the tangent-linear form above):
 *   tgh_adjoint_error_norm  the masked volume-weighted L2 error of u at t (src/constraints.jl:
 *                           311-396) and lam = its gradient (device, state layout; zero away from
 *                           the evolved primary entries)
 *   tgh_adjoint_rhs         lam_u = (d du / d u)^T lam_du for du = gh_rhs!(u, t); th3 (host,
 *                           nullable) = lam_du . d du / d(rho_max, ramp, damping strength)
 *   tgh_adjoint_rk4_step    lam: in, the cotangent of the state after one plain RK4 step of dt
 *                           from u at t; out, the cotangent of u. The step's stage values are
 *                           recomputed from u; th3 (host, nullable) is accumulated
 * A caller checkpoints the states of the forward run and sweeps back (adjoint.py). FP64, one
 * rank, no matter term, an interior that does not move and is not :pasted, no range projection.
 * The first adjoint call allocates the adjoint's buffers (20 x 8 doubles of feature cotangents
 * per working-array point, and six state vectors). */
int tgh_adjoint_error_norm(tgh_problem* p, const double* u, double t, double* l2, double* lam);
int tgh_adjoint_rhs(tgh_problem* p, const double* u, double t, const double* lam_du, double* lam_u, double* th3);
int tgh_adjoint_rk4_step(tgh_problem* p, const double* u, double t, double dt, double* lam, double* th3);

/* --- one rank per GPU (TreeAMR's distribution of a forest's blocks over the ranks of a
 * communicator, src/distributed.jl:1-22; the forest itself is on every rank) ---
 * tgh_partition: the owner rank of every leaf: per refinement level, the level's leaves in
 * Morton order of their block coordinates cut into nranks runs of nearly equal length. Host
 * only.
 * tgh_problem_create_shard: the problem of `rank`'s leaves (owner[b] == rank) over the whole
 * forest `mesh`; its state vectors hold its own leaves in forest order. Its working arrays
 * also hold halo blocks: the other ranks' leaves its ghost fill reads.
 * The batched step is then driven by the caller, which owns the transport between ranks:
 *   tgh_shard_begin(u)
 *   per step, per stage s = 0..3:
 *     per phase f = 0 .. tgh_shard_phases() - 1:        (0: copies and Dirichlet ghosts;
 *       tgh_shard_pack(s, f, send)                        f >= 1: level f's prolongation)
 *       exchange: send holds, peer after peer, send_count[r] points of 20 doubles for rank r;
 *                 recv receives recv_count[r] points from rank r likewise (tgh_shard_counts)
 *       tgh_shard_unpack(s, f, recv); tgh_shard_fill(s, f, t, dt)
 *     tgh_shard_rhs(s, t, dt)
 *   tgh_shard_end(u)
 * Every call is ordered on the problem's stream; send and recv are device buffers. With one
 * rank the sequence is the batched step without its graph. The plain form's verbs refuse a
 * problem of more than one rank. */
int tgh_partition(const tgh_mesh* mesh, int nranks, int* owner);
/* host-only view of rank's exchange in one fill phase: per peer the point counts and, when the
 * arrays are given (2 ints per point), the (forest leaf, work index) pairs sent and received,
 * peer-major; the lists tgh_problem_create_shard builds. errbuf (nullable) receives a failure. */
int tgh_shard_plan(const tgh_config* cfg, const tgh_mesh* mesh, const int* owner, int rank, int nranks, int phase,
                   long* send_count, long* recv_count, int* send_pts, int* recv_pts, char* errbuf, int errlen);
int tgh_problem_create_shard(const tgh_config* cfg, const tgh_mesh* mesh, const int* owner, int rank, int nranks,
                             void* cuda_stream, int margin_check, tgh_problem** out);
int tgh_shard_phases(const tgh_problem* p);
int tgh_shard_counts(tgh_problem* p, int phase, long* send_count, long* recv_count);
int tgh_shard_begin(tgh_problem* p, const double* u);
int tgh_shard_pack(tgh_problem* p, int stage, int phase, double* send);
int tgh_shard_unpack(tgh_problem* p, int stage, int phase, const double* recv);
int tgh_shard_fill(tgh_problem* p, int stage, int phase, double t, double dt);
int tgh_shard_rhs(tgh_problem* p, int stage, double t, double dt);
int tgh_shard_end(tgh_problem* p, double* u);

#ifdef __cplusplus
}
#endif
#endif
