// TEST INFRASTRUCTURE: the CPU oracle of the generalized-harmonic stepping path.
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load
// liboracle.so (through ctypes); the product library never links or calls it.
//
// A plain FP64 restatement of the reference's algorithm:
//   gh_rhs_kernel! / gh_rhs_point! / gh_rhs_head / _dth / gh_rhs_pi   src/evolution.jl:258-695
//   axis_stencil, mixed_stencil (summation order)                     src/evolution.jl:192-219
//   host_rhs_at (the expanded reference spelling)                     test/evolution_tests.jl:37-89
//   rhs_scale                                                         test/evolution_tests.jl:97-108
//   gh_speed_kernel!, max_speed(p,u,t)                                src/evolution.jl:932-949, 1539-1560
//   gh_error_kernel!, masked volume-weighted L2                       src/constraints.jl:311-396, 716-792
//   sample_gauge_source!, gauge_at                                    src/gauge.jl:156-212
//   initial_state!, stage_limit!, gh_paste_kernel!                    src/stepping.jl:91-115, src/evolution.jl:888-905
//   bounds_project, gh_bounds_kernel! (bounds.hpp)                    src/bounds.jl:256-663
// and of the un-vendored packages under it (no exact pin; compat bounds only):
//   TreeAMR 0.3: closed vertex-centered blocks, scatter!, fill_ghosts! (same-level copies
//     from the primary copy, restriction by injection, the Dirichlet CellBoundary hook,
//     tensor-product Lagrange prolongation of order p = q + 2, coarsest level first),
//     semantics from CODE.md:406-466, 713-777 of the reference. The fill is written here as
//     a recursive definition of the value at any lattice point of any level.
//   IMEXRungeKutta 1.2: classical RK4 with the limiter on the three stage values and the
//     step's result (CODE.md:3415-3434); the accumulation order is this oracle's choice.
#include <omp.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <type_traits>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "adm_streamed.hpp"
#include "bounds.hpp"
#include "lanes.hpp"
#include "physics.hpp"
#include "pointwise.hpp"
#include "spacetime.hpp"
#include "stencils.hpp"

namespace orc {

static const int NV = 20;

struct Problem {
  tgh_config cfg;
  int q, G, N, N1, W, nb, maxlevel = 0;
  double lo[3], h0;
  int cells0[3], periodic[3];
  std::vector<int> level, corner;                     // per leaf
  std::vector<std::unordered_map<int64_t, int>> lut;  // per level: block coordinate -> leaf
  Stencils st;
  std::vector<double> wP;  // prolongation weights at the half-way point (p = q + 2 points)
  Interior in;
  Profiles pr;
  KSSource ks;
  bool diss = false;
  std::vector<double> work, Hsrc;
  int simd = 1;  // points the right-hand side evaluates at once along x: 1 or ORC_SIMD_W
  std::vector<double> ustate;  // the state the last prepare scattered
  double t_prep = 0.0;
  // the :fitted target cache (src/fit.jl:1030-1055): per block 40 fields of the owned points, the
  // target A (h, Pi) at the fill time t_f and its slope S
  std::vector<double> tw;
  double t_f = 0.0;
  bool target_set = false;
  std::string err;

  explicit Problem(int q_) : st(q_) {}
  size_t npt_state() const { return (size_t)N1 * N1 * N1; }
  size_t npt_work() const { return (size_t)W * W * W; }
  double spacing(int l) const { return std::ldexp(h0, -l); }
  int64_t key(int bx, int by, int bz) const {
    return ((int64_t)bx * 1048576 + by) * 1048576 + bz;
  }
  void position(int l, const int64_t n[3], double x[3]) const {
    double h = spacing(l);
    for (int d = 0; d < 3; ++d) x[d] = lo[d] + (double)n[d] * h;
  }
};

// ---- the primary owner of a lattice point: the coarsest leaf holding it, and within a level
// the one holding it on its lower face. A point of level l's lattice lies on level k < l's when
// its index is a multiple of 2^(l - k). ----
static bool find_owner(const Problem& P, int l, const int64_t nin[3], int& leaf, int loc[3]) {
  for (int k = 0; k <= P.maxlevel; ++k) {
    int64_t m[3], per[3];
    bool on = true;
    for (int d = 0; d < 3; ++d) {
      if (k >= l) {
        m[d] = nin[d] << (k - l);
      } else {
        const int64_t s = (int64_t)1 << (l - k);
        if (((nin[d] % s) + s) % s) on = false;
        m[d] = nin[d] >= 0 ? nin[d] / s : -((-nin[d]) / s);
      }
      per[d] = (int64_t)P.cells0[d] << k;
    }
    if (!on) continue;
    int64_t cand[3][2];
    int nc[3];
    for (int d = 0; d < 3; ++d) {
      int64_t c = m[d] >= 0 ? m[d] / P.N : -((-m[d] + P.N - 1) / P.N);
      nc[d] = 0;
      cand[d][nc[d]++] = c;
      if (m[d] % P.N == 0) cand[d][nc[d]++] = c - 1;
      (void)per;
    }
    for (int iz = 0; iz < nc[2]; ++iz)
      for (int iy = 0; iy < nc[1]; ++iy)
        for (int ix = 0; ix < nc[0]; ++ix) {
          auto it = P.lut[k].find(P.key((int)cand[0][ix], (int)cand[1][iy], (int)cand[2][iz]));
          if (it == P.lut[k].end()) continue;
          leaf = it->second;
          for (int d = 0; d < 3; ++d) loc[d] = (int)(m[d] - P.corner[3 * leaf + d]);
          return true;
        }
  }
  return false;
}

// whether block b holds the primary copy of its owned point (i, j, k): the lattice point,
// wrapped on a periodic axis (the upper periodic face is the lower one), has b as its owner
static bool is_primary(const Problem& P, int b, int i, int j, int k) {
  const int l = P.level[b];
  int64_t n[3] = {(int64_t)P.corner[3 * b] + i, (int64_t)P.corner[3 * b + 1] + j, (int64_t)P.corner[3 * b + 2] + k};
  for (int d = 0; d < 3; ++d)
    if (P.periodic[d]) {
      const int64_t per = (int64_t)P.cells0[d] << l;
      n[d] %= per;
      if (n[d] < 0) n[d] += per;
    }
  int leaf, loc[3];
  return find_owner(P, l, n, leaf, loc) && leaf == b;
}

static void hook_value(const Problem& P, double t, const double x[3], double out[NV]) {
  double xc[3], dh[3][NC], dg[NC];
  P.in.core_position(t, x, xc);
  background_state(P.cfg.bg, t, xc, out, out + NC, dh, dg);
}

// The value of all 20 variables at lattice point n of level l, as a filled working
// array holds it: the hook outside the domain, the primary copy where a leaf of this or a
// finer level owns the point (injection from the finer one), and otherwise the
// tensor-product Lagrange prolongation of the next coarser level (x summed innermost).
static void value20(const Problem& P, const std::vector<double>& u, double t, int l,
                    const int64_t nin[3], double out[NV]) {
  int64_t n[3];
  for (int d = 0; d < 3; ++d) {
    n[d] = nin[d];
    int64_t per = (int64_t)P.cells0[d] << l;
    if (P.periodic[d]) {
      n[d] %= per;
      if (n[d] < 0) n[d] += per;
    }
  }
  for (int d = 0; d < 3; ++d) {
    int64_t per = (int64_t)P.cells0[d] << l;
    if (!P.periodic[d] && (n[d] < 0 || n[d] > per)) {
      double x[3];
      P.position(l, n, x);
      hook_value(P, t, x, out);
      return;
    }
  }
  int leaf, loc[3];
  if (find_owner(P, l, n, leaf, loc)) {
    size_t base = (size_t)leaf * NV * P.npt_state() + loc[0] + P.N1 * (loc[1] + (size_t)P.N1 * loc[2]);
    for (int v = 0; v < NV; ++v) out[v] = u[base + v * P.npt_state()];
    return;
  }
  if (l == 0) throw std::runtime_error("lattice point not covered by the forest");
  // prolongation from level l-1
  int64_t idx[3][16];
  double w[3][16];
  int cnt[3];
  const int p = (int)P.wP.size();
  for (int d = 0; d < 3; ++d) {
    if (n[d] % 2 == 0) {
      cnt[d] = 1;
      idx[d][0] = n[d] / 2;
      w[d][0] = 1.0;
    } else {
      int64_t base = (n[d] - 1) / 2 - (p / 2 - 1);
      cnt[d] = p;
      for (int k = 0; k < p; ++k) {
        idx[d][k] = base + k;
        w[d][k] = P.wP[k];
      }
    }
  }
  double sz[NV];
  for (int v = 0; v < NV; ++v) sz[v] = 0.0;
  for (int kz = 0; kz < cnt[2]; ++kz) {
    double sy[NV];
    for (int v = 0; v < NV; ++v) sy[v] = 0.0;
    for (int ky = 0; ky < cnt[1]; ++ky) {
      double sx[NV];
      for (int v = 0; v < NV; ++v) sx[v] = 0.0;
      for (int kx = 0; kx < cnt[0]; ++kx) {
        int64_t m[3] = {idx[0][kx], idx[1][ky], idx[2][kz]};
        double c[NV];
        value20(P, u, t, l - 1, m, c);
        for (int v = 0; v < NV; ++v) sx[v] = kx == 0 ? w[0][kx] * c[v] : sx[v] + w[0][kx] * c[v];
      }
      for (int v = 0; v < NV; ++v) sy[v] = ky == 0 ? w[1][ky] * sx[v] : sy[v] + w[1][ky] * sx[v];
    }
    for (int v = 0; v < NV; ++v) sz[v] = kz == 0 ? w[2][kz] * sy[v] : sz[v] + w[2][kz] * sy[v];
  }
  for (int v = 0; v < NV; ++v) out[v] = sz[v];
}

// prepare!: scatter + fill_ghosts! with the hook at t (src/evolution.jl:1349-1357)
static void prepare(Problem& P, const double* u, double t) {
  size_t L = P.npt_state() * NV * P.nb;
  P.ustate.assign(u, u + L);
  P.t_prep = t;
  P.work.assign(P.npt_work() * NV * P.nb, 0.0);
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < P.nb; ++b) {
    const int l = P.level[b];
    double vals[NV];
    for (int k = 0; k < P.W; ++k)
      for (int j = 0; j < P.W; ++j)
        for (int i = 0; i < P.W; ++i) {
          int64_t n[3] = {(int64_t)P.corner[3 * b] + i - P.G, (int64_t)P.corner[3 * b + 1] + j - P.G,
                          (int64_t)P.corner[3 * b + 2] + k - P.G};
          value20(P, P.ustate, t, l, n, vals);
          size_t base = (size_t)b * NV * P.npt_work() + i + P.W * (j + (size_t)P.W * k);
          for (int v = 0; v < NV; ++v) P.work[base + v * P.npt_work()] = vals[v];
        }
  }
}

// ---- the right-hand side at one owned point (src/evolution.jl:258-388, 448-695) ----
struct PointCtx {
  const double* wk;  // this block's working array
  size_t sv;         // per-variable stride
  int st[3];         // per-axis strides
  size_t var;        // the point's linear index
};

template <class T = double>
static inline T axis_stencil(const std::vector<double>& w, const double* wk, size_t base, long stride) {
  const int n = (int)w.size(), r = (n - 1) / 2;
  T s = T(w[0]) * ldw<T>(wk + base + (long)(-r) * stride);
  for (int k = 1; k < n; ++k) s = s + T(w[k]) * ldw<T>(wk + base + (long)(k - r) * stride);
  return s;
}
template <class T = double>
static inline T mixed_stencil(const std::vector<double>& w, const double* wk, size_t base, long s1, long s2) {
  const int n = (int)w.size(), r = (n - 1) / 2;
  T outer = T(0.0);
  for (int a = 0; a < n; ++a) {
    T inner = T(w[0]) * ldw<T>(wk + base + (long)(a - r) * s1 + (long)(-r) * s2);
    for (int e = 1; e < n; ++e) inner = inner + T(w[e]) * ldw<T>(wk + base + (long)(a - r) * s1 + (long)(e - r) * s2);
    outer = a == 0 ? T(w[0]) * inner : outer + T(w[a]) * inner;
  }
  return outer;
}

template <class T>
static void gauge_at_point(const Problem& P, int b, const int I[3], const T* h, const T* dth,
                           const T* const dh[3], T Hl[4], T dHl[4][4]) {
  if (P.cfg.gauge == TGH_GAUGE_NONE) {
    for (int a = 0; a < 4; ++a) {
      Hl[a] = T(0.0);
      for (int c = 0; c < 4; ++c) dHl[a][c] = T(0.0);
    }
  } else if (P.cfg.gauge == TGH_GAUGE_SAMPLED) {
    size_t o = (size_t)b * NV * P.npt_state() + I[0] + P.N1 * (I[1] + (size_t)P.N1 * I[2]);
    for (int a = 0; a < 4; ++a) Hl[a] = ldw<T>(P.Hsrc.data() + o + a * P.npt_state());
    for (int k = 0; k < 16; ++k) dHl[k % 4][k / 4] = ldw<T>(P.Hsrc.data() + o + (4 + k) * P.npt_state());
  } else {
    algebraic_gauge_source<T>(P.ks, h, dth, dh, Hl, dHl);
  }
}

// F(u) at one owned point as two vectors (gh_rhs_at_point, src/evolution.jl:423-435)
template <class T>
static void rhs_at_point(const Problem& P, const PointCtx& c, int b, const int I[3], const double x[3],
                         double t, const double* matter, T dth_out[NC], T dtPi_out[NC]) {
  const double h = P.spacing(P.level[b]);
  const T inv_h = T(1.0) / T(h);
  const T inv_h2 = inv_h * inv_h;
  // the profiles at each point of the group (one point, or a group's lanes along x)
  auto lane_x = [&](int l, double xl[3]) {
    int64_t n[3] = {(int64_t)P.corner[3 * b] + I[0] + l, (int64_t)P.corner[3 * b + 1] + I[1],
                    (int64_t)P.corner[3 * b + 2] + I[2]};
    P.position(P.level[b], n, xl);
  };
  const T g0 = PerLane<T>::make([&](int l) {
    double xl[3];
    if (l == 0) return P.pr.damping_rate(t, x);
    lane_x(l, xl);
    return P.pr.damping_rate(t, xl);
  });
  const T eh = PerLane<T>::make([&](int l) {
    double xl[3];
    if (l == 0) return P.pr.dissipation_rate(t, x);
    lane_x(l, xl);
    return P.pr.dissipation_rate(t, xl);
  }) * inv_h;
  const double* wk = c.wk;
  T hv[NC], Pv[NC], dhs[3][NC];
  for (int v = 0; v < NC; ++v) {
    hv[v] = ldw<T>(wk + c.var + v * c.sv);
    Pv[v] = ldw<T>(wk + c.var + (NC + v) * c.sv);
  }
  for (int d = 0; d < 3; ++d)
    for (int v = 0; v < NC; ++v) dhs[d][v] = inv_h * axis_stencil<T>(P.st.w1, wk, c.var + v * c.sv, c.st[d]);
  const T* dh[3] = {dhs[0], dhs[1], dhs[2]};
  Coef<T> C;
  metric_quantities(hv, C);
  const T a_div = C.alpha / C.sqrtg;
  T dth[NC];
  for (int v = 0; v < NC; ++v) {
    T s = C.beta[0] * dh[0][v] + C.beta[1] * dh[1][v] + C.beta[2] * dh[2][v] + a_div * Pv[v];
    if (P.diss) {
      size_t bh = c.var + v * c.sv;
      s = s + eh * (axis_stencil<T>(P.st.wD, wk, bh, c.st[0]) + axis_stencil<T>(P.st.wD, wk, bh, c.st[1]) +
                    axis_stencil<T>(P.st.wD, wk, bh, c.st[2]));
    }
    dth[v] = s;
  }
  T Hl[4], dHl[4][4];
  gauge_at_point<T>(P, b, I, hv, dth, dh, Hl, dHl);
  T msrc[NC];
  gh_node_source_lean(C, dth, dh, Hl, dHl, g0, T(P.cfg.gamma2), msrc);
  if constexpr (std::is_same<T, double>::value) if (matter) {
    size_t o = (size_t)b * 10 * P.npt_state() + I[0] + P.N1 * (I[1] + (size_t)P.N1 * I[2]);
    double m[10];
    for (int k = 0; k < 10; ++k) m[k] = matter[o + k * P.npt_state()];
    double S3[3] = {m[1], m[2], m[3]};
    double Sij[3][3] = {{m[4], m[5], m[6]}, {m[5], m[7], m[8]}, {m[6], m[8], m[9]}};
    double ms[NC];
    matter_source(C, m[0], S3, Sij, ms);
    for (int v = 0; v < NC; ++v) msrc[v] = msrc[v] + ms[v];
  }
  T am = C.alpha * C.sqrtg;
  T A[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) A[i][j] = am * C.gamu[i][j];
  T divb, divA[3];
  metric_divergences(C, dh, divb, divA);
  for (int v = 0; v < NC; ++v) dth_out[v] = dth[v];
  // gh_rhs_pi, one component at a time (src/evolution.jl:324-354)
  for (int v = 0; v < NC; ++v) {
    size_t bh = c.var + v * c.sv, bP = bh + NC * c.sv;
    T Pi_v = ldw<T>(wk + bP);
    T d1 = inv_h * axis_stencil<T>(P.st.w1, wk, bh, c.st[0]);
    T d2 = inv_h * axis_stencil<T>(P.st.w1, wk, bh, c.st[1]);
    T d3 = inv_h * axis_stencil<T>(P.st.w1, wk, bh, c.st[2]);
    T p1 = inv_h * axis_stencil<T>(P.st.w1, wk, bP, c.st[0]);
    T p2 = inv_h * axis_stencil<T>(P.st.w1, wk, bP, c.st[1]);
    T p3 = inv_h * axis_stencil<T>(P.st.w1, wk, bP, c.st[2]);
    T s = C.beta[0] * p1 + C.beta[1] * p2 + C.beta[2] * p3 + divb * Pi_v + divA[0] * d1 +
               divA[1] * d2 + divA[2] * d3;
    s = s + (A[0][0] * (inv_h2 * axis_stencil<T>(P.st.w2, wk, bh, c.st[0])) +
             A[1][1] * (inv_h2 * axis_stencil<T>(P.st.w2, wk, bh, c.st[1])) +
             A[2][2] * (inv_h2 * axis_stencil<T>(P.st.w2, wk, bh, c.st[2])));
    T dxy = inv_h2 * mixed_stencil<T>(P.st.w1, wk, bh, c.st[0], c.st[1]);
    T dxz = inv_h2 * mixed_stencil<T>(P.st.w1, wk, bh, c.st[0], c.st[2]);
    T dyz = inv_h2 * mixed_stencil<T>(P.st.w1, wk, bh, c.st[1], c.st[2]);
    s = s + T(2.0) * (A[0][1] * dxy + A[0][2] * dxz + A[1][2] * dyz);
    if (P.diss)
      s = s + eh * (axis_stencil<T>(P.st.wD, wk, bP, c.st[0]) + axis_stencil<T>(P.st.wD, wk, bP, c.st[1]) +
                    axis_stencil<T>(P.st.wD, wk, bP, c.st[2]));
    dtPi_out[v] = s + msrc[v];
  }
}

// gh_rhs_point! (src/evolution.jl:448-695), the sphere interior's branches
static void rhs_point(const Problem& P, int b, const int I[3], double t, const double* matter, double out[NV]) {
  PointCtx c;
  c.wk = P.work.data() + (size_t)b * NV * P.npt_work();
  c.sv = P.npt_work();
  c.st[0] = 1;
  c.st[1] = P.W;
  c.st[2] = P.W * P.W;
  c.var = (size_t)(I[0] + P.G) + P.W * ((size_t)(I[1] + P.G) + (size_t)P.W * (I[2] + P.G));
  int64_t n[3] = {(int64_t)P.corner[3 * b] + I[0], (int64_t)P.corner[3 * b + 1] + I[1],
                  (int64_t)P.corner[3 * b + 2] + I[2]};
  double x[3];
  P.position(P.level[b], n, x);
  if (P.in.variant == TGH_INT_NONE) {
    rhs_at_point(P, c, b, I, x, t, matter, out, out + NC);
    return;
  }
  const Interior& ia = P.in;
  double r = ia.radius(t, x);
  if (ia.variant == TGH_INT_FITTED) {
    // the :fitted branches (src/evolution.jl:528-548, 619-653) with the cache's target
    // A + (t - t_f) S (_cached_target, src/fit.jl:1050) and rate S (_cached_rate, :1055)
    const size_t S = P.npt_state();
    const double* tw = P.tw.data() + (size_t)b * 2 * NV * S + (I[0] + P.N1 * ((size_t)I[1] + (size_t)P.N1 * I[2]));
    auto target = [&](int v) { return tw[v * S] + (t - P.t_f) * tw[(NV + v) * S]; };
    auto rate = [&](int v) { return tw[(NV + v) * S]; };
    const bool rt = P.cfg.target_rate != 0;
    if (ia.is_frozen(r)) {
      const double rc = ia.rho_max;
      for (int v = 0; v < NV; ++v)
        out[v] = rt ? rate(v) - rc * (c.wk[c.var + v * c.sv] - target(v)) : -rc * (c.wk[c.var + v * c.sv] - target(v));
      return;
    }
    double F[NV];
    rhs_at_point(P, c, b, I, x, t, matter, F, F + NC);
    if (ia.is_outside(r)) {
      for (int v = 0; v < NV; ++v) out[v] = F[v];
      return;
    }
    double w, rho;
    ia.profiles(r, w, rho);
    const double of = 1.0 - w;
    for (int v = 0; v < NV; ++v)
      out[v] = rt ? w * F[v] + of * rate(v) - rho * (c.wk[c.var + v * c.sv] - target(v))
                  : w * F[v] - rho * (c.wk[c.var + v * c.sv] - target(v));
    return;
  }
  if (ia.is_frozen(r)) {
    if (ia.core_follows()) {
      double rho = ia.core_rate(), dl = ia.layer_rate_step();
      double xc[3], hd[NC], Pd[NC], dhd[3][NC], dgd[NC], dthd[NC], dtPd[NC], hu[NC], dhr[NC];
      ia.core_position(t, x, xc);
      background_state(P.cfg.bg, t, xc, hd, Pd, dhd, dgd);
      core_target_rate(ia, P.cfg.bg, t, x, dl, dthd, dtPd);
      for (int v = 0; v < NC; ++v) hu[v] = c.wk[c.var + v * c.sv];
      core_relaxation_rate(hu, hd, rho, dthd, dhr);
      for (int v = 0; v < NC; ++v) {
        out[v] = dhr[v];
        out[NC + v] = dtPd[v] - rho * (c.wk[c.var + (NC + v) * c.sv] - Pd[v]);
      }
    } else {
      for (int v = 0; v < NV; ++v) out[v] = 0.0;
    }
    return;
  }
  double F[NV];
  rhs_at_point(P, c, b, I, x, t, matter, F, F + NC);
  if (ia.is_outside(r)) {
    for (int v = 0; v < NV; ++v) out[v] = F[v];
    return;
  }
  double w, rho;
  ia.profiles(r, w, rho);
  if (ia.core_follows()) {
    double hm[NC], Pm[NC], dthm[NC], dtPm[NC];
    background_state_rate(P.cfg.bg, t, x, ia.layer_rate_step(), hm, Pm, dthm, dtPm);
    double om = 1.0 - w;
    for (int v = 0; v < NC; ++v) {
      out[v] = w * F[v] + om * dthm[v] - rho * (c.wk[c.var + v * c.sv] - hm[v]);
      out[NC + v] = w * F[NC + v] + om * dtPm[v] - rho * (c.wk[c.var + (NC + v) * c.sv] - Pm[v]);
    }
  } else {
    double he[NC], Pe[NC], dh[3][NC], dg[NC];
    background_state(P.cfg.bg, t, x, he, Pe, dh, dg);
    for (int v = 0; v < NC; ++v) {
      out[v] = w * F[v] - rho * (c.wk[c.var + v * c.sv] - he[v]);
      out[NC + v] = w * F[NC + v] - rho * (c.wk[c.var + (NC + v) * c.sv] - Pe[v]);
    }
  }
}

// A group of W points along x on SIMD lanes (gh_rhs_lanes!, src/evolution.jl:698-790): F on the
// lanes where the interior does not act at any of them (no hole, or every point at r >= r_1)
// and there is no matter term; otherwise point by point through rhs_point, branch for branch.
static void rhs_group(const Problem& P, int b, int i0, int j, int k, double t, const double* matter, double* du) {
  constexpr int W = ORC_SIMD_W;
  typedef Lane<W> V;
  const size_t S = P.npt_state();
  bool lanes = matter == nullptr;
  double x[W][3];
  for (int l = 0; l < W; ++l) {
    int64_t n[3] = {(int64_t)P.corner[3 * b] + i0 + l, (int64_t)P.corner[3 * b + 1] + j,
                    (int64_t)P.corner[3 * b + 2] + k};
    P.position(P.level[b], n, x[l]);
    if (P.in.variant != TGH_INT_NONE && !P.in.is_outside(P.in.radius(t, x[l]))) lanes = false;
  }
  const size_t o = (size_t)b * NV * S + i0 + P.N1 * (j + (size_t)P.N1 * k);
  if (!lanes) {
    double out[NV];
    for (int l = 0; l < W; ++l) {
      int I[3] = {i0 + l, j, k};
      rhs_point(P, b, I, t, matter, out);
      for (int v = 0; v < NV; ++v) du[o + l + v * S] = out[v];
    }
    return;
  }
  PointCtx c;
  c.wk = P.work.data() + (size_t)b * NV * P.npt_work();
  c.sv = P.npt_work();
  c.st[0] = 1;
  c.st[1] = P.W;
  c.st[2] = P.W * P.W;
  c.var = (size_t)(i0 + P.G) + P.W * ((size_t)(j + P.G) + (size_t)P.W * (k + P.G));
  int I[3] = {i0, j, k};
  V F[NV];
  rhs_at_point<V>(P, c, b, I, x[0], t, nullptr, F, F + NC);
  for (int v = 0; v < NV; ++v)
    for (int l = 0; l < W; ++l) du[o + l + v * S] = F[v].v[l];
}

static void rhs(Problem& P, double* du, double t, const double* matter) {
  const size_t S = P.npt_state();
  if (P.simd > 1 && P.N1 >= ORC_SIMD_W) {
    // the groups of a row: every W-th point from the first as far as a whole group fits, and
    // the group ending at the row's last point (is_lane_leader, src/lanes.jl:108-117)
    const int last = P.N1 - ORC_SIMD_W;
#pragma omp parallel for schedule(dynamic) collapse(2)
    for (int b = 0; b < P.nb; ++b)
      for (int k = 0; k < P.N1; ++k)
        for (int j = 0; j < P.N1; ++j) {
          int i0 = 0;
          for (; i0 <= last; i0 += ORC_SIMD_W) rhs_group(P, b, i0, j, k, t, matter, du);
          if (i0 - ORC_SIMD_W != last) rhs_group(P, b, last, j, k, t, matter, du);
        }
    return;
  }
#pragma omp parallel for schedule(dynamic) collapse(2)
  for (int b = 0; b < P.nb; ++b)
    for (int k = 0; k < P.N1; ++k) {
      double out[NV];
      for (int j = 0; j < P.N1; ++j)
        for (int i = 0; i < P.N1; ++i) {
          int I[3] = {i, j, k};
          rhs_point(P, b, I, t, matter, out);
          size_t o = (size_t)b * NV * S + i + P.N1 * (j + (size_t)P.N1 * k);
          for (int v = 0; v < NV; ++v) du[o + v * S] = out[v];
        }
    }
}

// The state the case puts at x: case_state_tuple (src/initialdata.jl:1816-1830)
static void exact_state(const Problem& P, double t, const double x[3], double out[NV]) { hook_value(P, t, x, out); }

// gh_paste_kernel! (src/evolution.jl:888-905), the :pasted variant's limiter
static void stage_limit(Problem& P, double* u, double t) {
  if (P.in.variant != TGH_INT_PASTED) return;
  const size_t S = P.npt_state();
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < P.nb; ++b)
    for (int k = 0; k < P.N1; ++k)
      for (int j = 0; j < P.N1; ++j)
        for (int i = 0; i < P.N1; ++i) {
          int64_t n[3] = {(int64_t)P.corner[3 * b] + i, (int64_t)P.corner[3 * b + 1] + j,
                          (int64_t)P.corner[3 * b + 2] + k};
          double x[3];
          P.position(P.level[b], n, x);
          if (P.in.is_outside(P.in.radius(t, x))) continue;
          double vals[NV];
          exact_state(P, t, x, vals);
          size_t o = (size_t)b * NV * S + i + P.N1 * (j + (size_t)P.N1 * k);
          for (int v = 0; v < NV; ++v) u[o + v * S] = vals[v];
        }
}

static void initial_state(Problem& P, double* u, double t) {
  const size_t S = P.npt_state();
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < P.nb; ++b)
    for (int k = 0; k < P.N1; ++k)
      for (int j = 0; j < P.N1; ++j)
        for (int i = 0; i < P.N1; ++i) {
          int64_t n[3] = {(int64_t)P.corner[3 * b] + i, (int64_t)P.corner[3 * b + 1] + j,
                          (int64_t)P.corner[3 * b + 2] + k};
          double x[3], vals[NV];
          P.position(P.level[b], n, x);
          exact_state(P, t, x, vals);
          size_t o = (size_t)b * NV * S + i + P.N1 * (j + (size_t)P.N1 * k);
          for (int v = 0; v < NV; ++v) u[o + v * S] = vals[v];
        }
  stage_limit(P, u, t);
}

// The :fitted target cache's fills. snapshot_target_kernel! (src/fit.jl:1189-1212): the state itself
// inside r_fill about the interior's centre at t_f, slope 0, zero elsewhere. The analytic fill is
// fit_target_kernel! (src/fit.jl:1070-1116) with the exact solution standing in for the fit: the
// case's state (core rule included) at t_f and, with dt > 0, its rate as the centred difference
// (A(t_f + dt) - A(t_f - dt)) / (2 dt).
static void fill_target(Problem& P, const double* u, double t_f, double r_fill, double dt) {
  const size_t S = P.npt_state();
  P.tw.assign((size_t)P.nb * 2 * NV * S, 0.0);
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < P.nb; ++b)
    for (size_t ip = 0; ip < S; ++ip) {
      const int i = (int)(ip % P.N1), j = (int)((ip / P.N1) % P.N1), k = (int)(ip / ((size_t)P.N1 * P.N1));
      int64_t n[3] = {(int64_t)P.corner[3 * b] + i, (int64_t)P.corner[3 * b + 1] + j, (int64_t)P.corner[3 * b + 2] + k};
      double x[3];
      P.position(P.level[b], n, x);
      if (!(P.in.radius(t_f, x) < r_fill)) continue;
      double* o = P.tw.data() + (size_t)b * 2 * NV * S + ip;
      if (u) {
        for (int v = 0; v < NV; ++v) o[v * S] = u[(size_t)b * NV * S + v * S + ip];
        continue;
      }
      double a[NV];
      exact_state(P, t_f, x, a);
      for (int v = 0; v < NV; ++v) o[v * S] = a[v];
      if (dt > 0.0) {
        double ap[NV], am[NV];
        exact_state(P, t_f + dt, x, ap);
        exact_state(P, t_f - dt, x, am);
        const double id = 1.0 / (2.0 * dt);
        for (int v = 0; v < NV; ++v) o[(NV + v) * S] = id * (ap[v] - am[v]);
      }
    }
  P.t_f = t_f;
  P.target_set = true;
}

// fitted_state_kernel! (src/fit.jl:1247-1285) without the blend: the background's state where
// r >= r_1 - d_init, the cached target at t below
static void fitted_initial_state(Problem& P, double* u, double t, double d_init) {
  const size_t S = P.npt_state();
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < P.nb; ++b)
    for (size_t ip = 0; ip < S; ++ip) {
      const int i = (int)(ip % P.N1), j = (int)((ip / P.N1) % P.N1), k = (int)(ip / ((size_t)P.N1 * P.N1));
      int64_t n[3] = {(int64_t)P.corner[3 * b] + i, (int64_t)P.corner[3 * b + 1] + j, (int64_t)P.corner[3 * b + 2] + k};
      double x[3];
      P.position(P.level[b], n, x);
      double* o = u + (size_t)b * NV * S + ip;
      if (P.in.radius(t, x) >= P.in.r1 - d_init) {
        double dh[3][NC], dg[NC], vals[NV];
        background_state(P.cfg.bg, t, x, vals, vals + NC, dh, dg);
        for (int v = 0; v < NV; ++v) o[v * S] = vals[v];
      } else {
        const double* tw = P.tw.data() + (size_t)b * 2 * NV * S + ip;
        for (int v = 0; v < NV; ++v) o[v * S] = tw[v * S] + (t - P.t_f) * tw[(NV + v) * S];
      }
    }
}

static bool is_evolved(const Problem& P, double t, const double x[3]) {
  return P.in.variant == TGH_INT_NONE ? true : P.in.radius(t, x) >= P.in.r1;
}

// max_speed(p, u, t) (src/evolution.jl:1539-1560 with gh_speed_kernel! :932-949)
static int max_speed(Problem& P, const double* u, double t, double* lam) {
  const size_t S = P.npt_state();
  long nbad = 0;
  double best = 0.0;
  bool nan = false;
  for (int b = 0; b < P.nb; ++b)
    for (int k = 0; k < P.N1; ++k)
      for (int j = 0; j < P.N1; ++j)
        for (int i = 0; i < P.N1; ++i) {
          int64_t n[3] = {(int64_t)P.corner[3 * b] + i, (int64_t)P.corner[3 * b + 1] + j,
                          (int64_t)P.corner[3 * b + 2] + k};
          double x[3];
          P.position(P.level[b], n, x);
          if (!is_evolved(P, t, x)) continue;
          size_t o = (size_t)b * NV * S + i + P.N1 * (j + (size_t)P.N1 * k);
          double hv[NC];
          for (int v = 0; v < NV; ++v)
            if (!std::isfinite(u[o + v * S])) ++nbad;
          for (int v = 0; v < NC; ++v) hv[v] = u[o + v * S];
          Coef<double> C;
          metric_quantities(hv, C);
          double l = C.alpha * std::sqrt(C.gamu[0][0] + C.gamu[1][1] + C.gamu[2][2]) +
                     std::sqrt(C.beta[0] * C.beta[0] + C.beta[1] * C.beta[1] + C.beta[2] * C.beta[2]);
          if (std::isnan(l)) nan = true;
          if (l > best) best = l;
        }
  if (nbad > 0) {
    P.err = "the state is not finite where it is evolved: " + std::to_string(nbad) + " values";
    return TGH_ERR_NONFINITE;
  }
  *lam = nan ? NAN : best;
  if (!(std::isfinite(*lam) && *lam > 0)) {
    P.err = "the maximum characteristic speed is not finite and positive";
    return TGH_ERR_SPEED;
  }
  return TGH_OK;
}

// RK4 with the accumulation order this oracle and the product share:
//   acc = u + (dt/6) k1;  y2 = u + (dt/2) k1
//   acc = acc + (dt/3) k2;  y3 = u + (dt/2) k2
//   acc = acc + (dt/3) k3;  y4 = u + dt k3
//   u_new = acc + (dt/6) k4          each update one fused multiply-add
static void rk4_step(Problem& P, double* u, double t, double dt) {
  if (P.in.variant == TGH_INT_FITTED && !P.target_set)
    throw std::runtime_error("a :fitted interior relaxes toward the target cache: fill or set it first");
  const size_t L = P.npt_state() * NV * P.nb;
  std::vector<double> k(L), acc(L), y(L), u0(u, u + L);
  const double b16 = dt / 6.0, b13 = dt / 3.0, a12 = 0.5 * dt;
  const double tm = t + 0.5 * dt, te = t + dt;
  prepare(P, u0.data(), t);
  rhs(P, k.data(), t, nullptr);
  for (size_t i = 0; i < L; ++i) {
    acc[i] = std::fma(b16, k[i], u0[i]);
    y[i] = std::fma(a12, k[i], u0[i]);
  }
  stage_limit(P, y.data(), tm);
  prepare(P, y.data(), tm);
  rhs(P, k.data(), tm, nullptr);
  for (size_t i = 0; i < L; ++i) {
    acc[i] = std::fma(b13, k[i], acc[i]);
    y[i] = std::fma(a12, k[i], u0[i]);
  }
  stage_limit(P, y.data(), tm);
  prepare(P, y.data(), tm);
  rhs(P, k.data(), tm, nullptr);
  for (size_t i = 0; i < L; ++i) {
    acc[i] = std::fma(b13, k[i], acc[i]);
    y[i] = std::fma(dt, k[i], u0[i]);
  }
  stage_limit(P, y.data(), te);
  prepare(P, y.data(), te);
  rhs(P, k.data(), te, nullptr);
  for (size_t i = 0; i < L; ++i) u[i] = std::fma(b16, k[i], acc[i]);
  stage_limit(P, u, te);
}

// the masked, volume-weighted L2 and max of |u - u_exact| over evolved primaries, read
// from the settled working array (src/constraints.jl:311-396, 716-792)
static void error_norm(Problem& P, const double* u, double t, double* l2, double* linf) {
  prepare(P, u, t);
  double s2 = 0.0, vol = 0.0, mx = 0.0;
  for (int b = 0; b < P.nb; ++b) {
    double h = P.spacing(P.level[b]);
    double w = h * h * h;
    for (int k = 0; k < P.N1; ++k)
      for (int j = 0; j < P.N1; ++j)
        for (int i = 0; i < P.N1; ++i) {
          int64_t n[3] = {(int64_t)P.corner[3 * b] + i, (int64_t)P.corner[3 * b + 1] + j,
                          (int64_t)P.corner[3 * b + 2] + k};
          if (!is_primary(P, b, i, j, k)) continue;
          double x[3];
          P.position(P.level[b], n, x);
          if (!is_evolved(P, t, x)) continue;
          double ex[NV];
          exact_state(P, t, x, ex);
          size_t o = (size_t)b * NV * P.npt_work() + (i + P.G) + P.W * ((j + P.G) + (size_t)P.W * (k + P.G));
          double e2 = 0.0;
          for (int v = 0; v < NV; ++v) {
            double d = P.work[o + v * P.npt_work()] - ex[v];
            e2 = v == 0 ? d * d : e2 + d * d;
          }
          double e = std::sqrt(e2);
          s2 += e * e * w;
          vol += w;
          if (e > mx) mx = e;
        }
  }
  *l2 = vol == 0.0 ? 0.0 : std::sqrt(s2 / vol);
  *linf = mx;
}

// ---- the constraint monitors (src/constraints.jl:211-271, 432-532) into a diag field set:
// per block NDIAG slots of (N+1)^3 points, C_a (4), H, M_i (3), the mask indicator ----
static const int NDIAG = 10;
enum { DG_CGH = 0, DG_HAM = 4, DG_MOM = 5, DG_MASK = 8, DG_TAU = 9 };

static PointCtx point_ctx(const Problem& P, int b, const int I[3], double x[3]) {
  PointCtx c;
  c.wk = P.work.data() + (size_t)b * NV * P.npt_work();
  c.sv = P.npt_work();
  c.st[0] = 1;
  c.st[1] = P.W;
  c.st[2] = P.W * P.W;
  c.var = (size_t)(I[0] + P.G) + P.W * ((size_t)(I[1] + P.G) + (size_t)P.W * (I[2] + P.G));
  int64_t n[3] = {(int64_t)P.corner[3 * b] + I[0], (int64_t)P.corner[3 * b + 1] + I[1],
                  (int64_t)P.corner[3 * b + 2] + I[2]};
  P.position(P.level[b], n, x);
  return c;
}

// gh_constraint_kernel! at one owned point: C_a = g_ab (Gamma^b + H^b), d_t g from the first
// evolution equation without the dissipation
template <class T>
static void gh_constraint_point(const Problem& P, const PointCtx& c, int b, const int I[3], T out[4]) {
  const T inv_h = T(1.0) / T(P.spacing(P.level[b]));
  T hv[NC], Pv[NC], dhs[3][NC], dth[NC];
  for (int v = 0; v < NC; ++v) {
    hv[v] = T(c.wk[c.var + v * c.sv]);
    Pv[v] = T(c.wk[c.var + (NC + v) * c.sv]);
  }
  for (int d = 0; d < 3; ++d)
    for (int v = 0; v < NC; ++v) dhs[d][v] = inv_h * axis_stencil<T>(P.st.w1, c.wk, c.var + v * c.sv, c.st[d]);
  const T* dh[3] = {dhs[0], dhs[1], dhs[2]};
  Coef<T> C;
  metric_quantities(hv, C);
  const T a_div = C.alpha / C.sqrtg;
  for (int v = 0; v < NC; ++v)
    dth[v] = C.beta[0] * dh[0][v] + C.beta[1] * dh[1][v] + C.beta[2] * dh[2][v] + a_div * Pv[v];
  T Hl[4], dHl[4][4];
  gauge_at_point<T>(P, b, I, hv, dth, dh, Hl, dHl);
  T dgl[4][4][4], Hup[4], Cup[4];
  for (int a = 0; a < 4; ++a)
    for (int e = 0; e < 4; ++e)
      for (int cc = 0; cc < 4; ++cc) dgl[a][e][cc] = cc == 0 ? dth[pairindex(a, e)] : dh[cc - 1][pairindex(a, e)];
  for (int a = 0; a < 4; ++a) {
    T s = C.gu4[a][0] * Hl[0];
    for (int e = 1; e < 4; ++e) s = s + C.gu4[a][e] * Hl[e];
    Hup[a] = s;
  }
  gauge_constraint_at_node(C.g4, dgl, Hup, Cup);
  for (int a = 0; a < 4; ++a) {
    T s = C.g4[a][0] * Cup[0];
    for (int e = 1; e < 4; ++e) s = s + C.g4[a][e] * Cup[e];
    out[a] = s;
  }
}

// adm_constraint_kernel! at one owned point: every second derivative of g, the d_t d_i and
// d_t d_t blocks from the evolution equations (d_t Pi from gh_node_rhs_expanded, source and
// damping included, no dissipation), then the Ricci assembly; with matter, H - 16 pi rho and
// M_i - 8 pi S_i. out: H, M_x, M_y, M_z
// STREAMED: the Ricci contraction in the GPU kernel's order (adm_streamed.hpp), for its flop
// count; the monitors' values use the reference's assembly.
template <class T, bool STREAMED = false>
static void adm_constraint_point(const Problem& P, const PointCtx& c, int b, const int I[3], const double x[3],
                                 double t, const double* matter, T out[4]) {
  static const int P3[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
  static const int D1[6] = {0, 0, 0, 1, 1, 2}, D2[6] = {0, 1, 2, 1, 2, 2};
  const T inv_h = T(1.0) / T(P.spacing(P.level[b]));
  const T inv_h2 = inv_h * inv_h;
  T hv[NC], Pv[NC], dhs[3][NC], dPs[3][NC], dds[6][NC];
  for (int v = 0; v < NC; ++v) {
    hv[v] = T(c.wk[c.var + v * c.sv]);
    Pv[v] = T(c.wk[c.var + (NC + v) * c.sv]);
  }
  for (int d = 0; d < 3; ++d)
    for (int v = 0; v < NC; ++v) {
      dhs[d][v] = inv_h * axis_stencil<T>(P.st.w1, c.wk, c.var + v * c.sv, c.st[d]);
      dPs[d][v] = inv_h * axis_stencil<T>(P.st.w1, c.wk, c.var + (NC + v) * c.sv, c.st[d]);
    }
  for (int n = 0; n < 6; ++n)
    for (int v = 0; v < NC; ++v) {
      size_t bh = c.var + v * c.sv;
      dds[n][v] = inv_h2 * (D1[n] == D2[n] ? axis_stencil<T>(P.st.w2, c.wk, bh, c.st[D1[n]])
                                           : mixed_stencil<T>(P.st.w1, c.wk, bh, c.st[D1[n]], c.st[D2[n]]));
    }
  const T* dh[3] = {dhs[0], dhs[1], dhs[2]};
  const T* dP[3] = {dPs[0], dPs[1], dPs[2]};
  const T* ddh[6] = {dds[0], dds[1], dds[2], dds[3], dds[4], dds[5]};
  Coef<T> C;
  metric_quantities(hv, C);
  const T a_div = C.alpha / C.sqrtg;
  T dth0[NC];
  for (int v = 0; v < NC; ++v)
    dth0[v] = C.beta[0] * dh[0][v] + C.beta[1] * dh[1][v] + C.beta[2] * dh[2][v] + a_div * Pv[v];
  T Hl[4], dHl[4][4];
  gauge_at_point<T>(P, b, I, hv, dth0, dh, Hl, dHl);
  const T g0 = T(P.pr.damping_rate(t, x));
  T dth[NC], dtPi[NC];
  gh_node_rhs_expanded(hv, Pv, dh, dP, ddh, Hl, dHl, g0, T(P.cfg.gamma2), dth, dtPi);
  double rho = 0.0, S3[3] = {0.0, 0.0, 0.0};
  if constexpr (std::is_same<T, double>::value) if (matter) {
    const size_t S = P.npt_state();
    size_t om = (size_t)b * 10 * S + I[0] + P.N1 * (I[1] + (size_t)P.N1 * I[2]);
    double m[10];
    for (int q = 0; q < 10; ++q) m[q] = matter[om + q * S];
    rho = m[0];
    S3[0] = m[1];
    S3[1] = m[2];
    S3[2] = m[3];
    double Sij[3][3] = {{m[4], m[5], m[6]}, {m[5], m[7], m[8]}, {m[6], m[8], m[9]}};
    double ms[NC];
    matter_source(C, rho, S3, Sij, ms);
    for (int v = 0; v < NC; ++v) dtPi[v] = dtPi[v] + ms[v];
  }
  const T phi = C.alpha / C.sqrtg;
  T dtd[3][NC];
  for (int d = 0; d < 3; ++d) {
    T dal, dbeta[3], dsq, dgamu[3][3];
    metric_derivatives_along(C, dh[d], dal, dbeta, dsq, dgamu);
    const T dphi = (dal - phi * dsq) / C.sqrtg;
    for (int v = 0; v < NC; ++v) {
      T acc = dphi * Pv[v] + phi * dP[d][v];
      dtd[d][v] = acc + (dbeta[0] * dh[0][v] + dbeta[1] * dh[1][v] + dbeta[2] * dh[2][v]) +
                  (C.beta[0] * ddh[P3[d][0]][v] + C.beta[1] * ddh[P3[d][1]][v] + C.beta[2] * ddh[P3[d][2]][v]);
    }
  }
  T dalt, dbt[3], dsqt, dgut[3][3], dtt[NC];
  metric_derivatives_along(C, dth, dalt, dbt, dsqt, dgut);
  const T dphit = (dalt - phi * dsqt) / C.sqrtg;
  for (int v = 0; v < NC; ++v)
    dtt[v] = dphit * Pv[v] + phi * dtPi[v] + (dbt[0] * dh[0][v] + dbt[1] * dh[1][v] + dbt[2] * dh[2][v]) +
             (C.beta[0] * dtd[0][v] + C.beta[1] * dtd[1][v] + C.beta[2] * dtd[2][v]);
  const T* dd[NC] = {dtt, dtd[0], dtd[1], dtd[2], ddh[0], ddh[1], ddh[2], ddh[3], ddh[4], ddh[5]};
  T dg[4][4][4], ddg[4][4][4][4];
  dg4(dth, dh, dg);
  for (int m = 0; m < 4; ++m)
    for (int n = 0; n < 4; ++n)
      for (int a = 0; a < 4; ++a)
        for (int e = 0; e < 4; ++e) ddg[m][n][a][e] = dd[pairindex(m, n)][pairindex(a, e)];
  T ham, mom[3];
  if constexpr (STREAMED) adm_constraints_streamed(C.g4, C.gu4, C.alpha, C.beta, dg, ddg, ham, mom);
  else adm_constraints_at_node(C.g4, C.gu4, C.alpha, C.beta, dg, ddg, ham, mom);
  if constexpr (std::is_same<T, double>::value) if (matter) {
    const double c8 = 8.0 * M_PI;
    ham = ham - 2.0 * (c8 * rho);
    for (int a = 0; a < 3; ++a) mom[a] = mom[a] - c8 * S3[a];
  }
  out[0] = ham;
  for (int a = 0; a < 3; ++a) out[1 + a] = mom[a];
}

// the monitors over every owned point; a masked point writes zeros and reads nothing
static void gh_constraint(Problem& P, const double* u, double t, bool all, double* diag) {
  prepare(P, u, t);
  const size_t S = P.npt_state();
#pragma omp parallel for schedule(dynamic) collapse(2)
  for (int b = 0; b < P.nb; ++b)
    for (int k = 0; k < P.N1; ++k)
      for (int j = 0; j < P.N1; ++j)
        for (int i = 0; i < P.N1; ++i) {
          int I[3] = {i, j, k};
          double x[3], out[4] = {0.0, 0.0, 0.0, 0.0};
          PointCtx c = point_ctx(P, b, I, x);
          size_t o = (size_t)b * NDIAG * S + i + P.N1 * (j + (size_t)P.N1 * k);
          const bool keep = all || is_evolved(P, t, x);
          if (keep) gh_constraint_point<double>(P, c, b, I, out);
          for (int a = 0; a < 4; ++a) diag[o + (DG_CGH + a) * S] = out[a];
          diag[o + DG_MASK * S] = keep ? 1.0 : 0.0;
        }
}

static void adm_constraint(Problem& P, const double* u, double t, bool all, const double* matter, double* diag) {
  prepare(P, u, t);
  const size_t S = P.npt_state();
#pragma omp parallel for schedule(dynamic) collapse(2)
  for (int b = 0; b < P.nb; ++b)
    for (int k = 0; k < P.N1; ++k)
      for (int j = 0; j < P.N1; ++j)
        for (int i = 0; i < P.N1; ++i) {
          int I[3] = {i, j, k};
          double x[3], out[4] = {0.0, 0.0, 0.0, 0.0};
          PointCtx c = point_ctx(P, b, I, x);
          size_t o = (size_t)b * NDIAG * S + i + P.N1 * (j + (size_t)P.N1 * k);
          const bool keep = all || is_evolved(P, t, x);
          if (keep) adm_constraint_point<double>(P, c, b, I, x, t, matter, out);
          diag[o + DG_HAM * S] = out[0];
          for (int a = 0; a < 3; ++a) diag[o + (DG_MOM + a) * S] = out[1 + a];
          diag[o + DG_MASK * S] = keep ? 1.0 : 0.0;
        }
}

static inline double nanmax(double a, double b) { return (a != a || b != b) ? NAN : (a > b ? a : b); }

// ---- the masked Loehner indicator (src/refinement.jl:170-218, 280-330, 390-391) ----
// lohner: the second difference over the two first differences and the noise floor
static inline double lohner(double um, double u0, double up, double scale, double eps) {
  const double num = std::fabs(up - 2.0 * u0 + um);
  const double den = std::fabs(up - u0) + std::fabs(u0 - um) + 4.0 * eps * std::fabs(scale);
  return den == 0.0 ? 0.0 : num / den;
}

// field_scales (the largest |h_v| over the evolved owned points), then tau at every owned point
// (cell_tau: the worst over the ten components of h and the three axes; zero where the mask
// leaves the point out) into the diag slot DG_TAU, then tau_max over the mesh.
// out: the ten maxima, the scale used (scale_in if positive, else their largest), tau_max
static void tau(Problem& P, const double* u, double t, bool all, double eps, double scale_in, double* diag,
                double out[12]) {
  prepare(P, u, t);
  const size_t S = P.npt_state();
  double sc[NC];
  for (int v = 0; v < NC; ++v) sc[v] = 0.0;
  for (int b = 0; b < P.nb; ++b)
    for (int k = 0; k < P.N1; ++k)
      for (int j = 0; j < P.N1; ++j)
        for (int i = 0; i < P.N1; ++i) {
          int I[3] = {i, j, k};
          double x[3];
          PointCtx c = point_ctx(P, b, I, x);
          if (!all && !is_evolved(P, t, x)) continue;
          for (int v = 0; v < NC; ++v) sc[v] = nanmax(sc[v], std::fabs(c.wk[c.var + v * c.sv]));
        }
  double scale = 0.0;
  for (int v = 0; v < NC; ++v) {
    out[v] = sc[v];
    scale = nanmax(scale, sc[v]);
  }
  if (scale_in > 0.0) scale = scale_in;
  double tmax = 0.0;
  for (int b = 0; b < P.nb; ++b)
    for (int k = 0; k < P.N1; ++k)
      for (int j = 0; j < P.N1; ++j)
        for (int i = 0; i < P.N1; ++i) {
          int I[3] = {i, j, k};
          double x[3];
          PointCtx c = point_ctx(P, b, I, x);
          double tv = 0.0;
          if (all || is_evolved(P, t, x))
            for (int v = 0; v < NC; ++v) {
              const size_t q = c.var + v * c.sv;
              for (int d = 0; d < 3; ++d)
                tv = nanmax(tv, lohner(c.wk[q - c.st[d]], c.wk[q], c.wk[q + c.st[d]], scale, eps));
            }
          diag[(size_t)b * NDIAG * S + DG_TAU * S + i + P.N1 * (j + (size_t)P.N1 * k)] = tv;
          tmax = nanmax(tmax, tv);
        }
  out[10] = scale;
  out[11] = tmax;
}

// firing_boxes over the diag slot DG_TAU: per block and threshold the number of owned points
// with tau > tol and the bounding box of their node indices (low N+1 and high -1 where none)
static void firing(const Problem& P, const double* diag, int ntol, const double* tol, int* counts, int* boxes) {
  const size_t S = P.npt_state();
  for (int b = 0; b < P.nb; ++b)
    for (int n = 0; n < ntol; ++n) {
      const size_t o = (size_t)b * ntol + n;
      counts[o] = 0;
      for (int d = 0; d < 3; ++d) {
        boxes[6 * o + d] = P.N1;
        boxes[6 * o + 3 + d] = -1;
      }
      for (int k = 0; k < P.N1; ++k)
        for (int j = 0; j < P.N1; ++j)
          for (int i = 0; i < P.N1; ++i) {
            const double tv = diag[(size_t)b * NDIAG * S + DG_TAU * S + i + P.N1 * (j + (size_t)P.N1 * k)];
            if (!(tv > tol[n])) continue;
            const int I[3] = {i, j, k};
            ++counts[o];
            for (int d = 0; d < 3; ++d) {
              boxes[6 * o + d] = std::min(boxes[6 * o + d], I[d]);
              boxes[6 * o + 3 + d] = std::max(boxes[6 * o + 3 + d], I[d]);
            }
          }
    }
}

// diag_norms over the slots C_a .. mask (src/constraints.jl:716-778, 825-865): each lattice point
// once, at its primary copy; weight h^3 (volume) or 1 (points), blocks of level at_level only
// when at_level >= 0; L2 = sqrt(sum u^2 w / evolved volume), Linf the largest |u| (NaN kept).
// out: gauge_l2[4], gauge_linf[4], ham_l2, ham_linf, mom_l2[3], mom_linf[3]
static void constraint_norms(const Problem& P, const double* diag, bool volume, int at_level, double out[16]) {
  const size_t S = P.npt_state();
  double vol = 0.0, s2[8] = {0}, mx[8] = {0};
  for (int b = 0; b < P.nb; ++b) {
    if (at_level >= 0 && P.level[b] != at_level) continue;
    const double h = P.spacing(P.level[b]);
    const double w = volume ? h * h * h : 1.0;
    for (int k = 0; k < P.N1; ++k)
      for (int j = 0; j < P.N1; ++j)
        for (int i = 0; i < P.N1; ++i) {
          if (!is_primary(P, b, i, j, k)) continue;
          size_t o = (size_t)b * NDIAG * S + i + P.N1 * (j + (size_t)P.N1 * k);
          vol += diag[o + DG_MASK * S] * w;
          for (int s = 0; s < 8; ++s) {
            double uu = diag[o + s * S];
            s2[s] += uu * uu * w;
            mx[s] = nanmax(mx[s], std::fabs(uu));
          }
        }
  }
  double l2[8];
  for (int s = 0; s < 8; ++s) l2[s] = vol == 0.0 ? 0.0 : std::sqrt(s2[s] / vol);
  for (int a = 0; a < 4; ++a) {
    out[a] = l2[DG_CGH + a];
    out[4 + a] = mx[DG_CGH + a];
  }
  out[8] = l2[DG_HAM];
  out[9] = mx[DG_HAM];
  for (int a = 0; a < 3; ++a) {
    out[10 + a] = l2[DG_MOM + a];
    out[13 + a] = mx[DG_MOM + a];
  }
}

}  // namespace orc

using namespace orc;

extern "C" {

void* orc_create(const tgh_config* cfg, const tgh_mesh* m, int margin_check, char* errbuf, int errlen) {
  (void)margin_check;
  try {
    if (cfg->q < 2 || cfg->q % 2 != 0 || cfg->q > 8) throw std::invalid_argument("q must be even in 2..8");
    Problem* P = new Problem(cfg->q);
    P->cfg = *cfg;
    P->q = cfg->q;
    P->G = cfg->q / 2 + 1;
    P->N = m->N;
    P->N1 = m->N + 1;
    P->W = m->N + 2 * P->G + 1;
    P->nb = m->nblocks;
    P->h0 = m->h0;
    for (int d = 0; d < 3; ++d) {
      P->lo[d] = m->lo[d];
      P->cells0[d] = m->cells0[d];
      P->periodic[d] = m->periodic[d];
    }
    P->level.assign(m->level, m->level + m->nblocks);
    P->corner.assign(m->corner, m->corner + 3 * m->nblocks);
    for (int b = 0; b < P->nb; ++b) P->maxlevel = std::max(P->maxlevel, P->level[b]);
    P->lut.resize(P->maxlevel + 1);
    for (int b = 0; b < P->nb; ++b)
      P->lut[P->level[b]][P->key(P->corner[3 * b] / P->N, P->corner[3 * b + 1] / P->N, P->corner[3 * b + 2] / P->N)] = b;
    // prolongation weights: Lagrange on p = q + 2 nodes, at the midpoint of the middle pair
    {
      const int p = cfg->q + 2;
      std::vector<Rat> ns;
      for (int k = 0; k < p; ++k) ns.push_back(Rat(2 * (k - (p / 2 - 1)) - 1, 2));
      P->wP = to_double(lagrange_derivative_weights(ns, 0));
    }
    P->in.variant = cfg->interior;
    for (int i = 0; i < 3; ++i) {
      P->in.c0[i] = cfg->int_c0[i];
      P->in.v[i] = cfg->int_v[i];
    }
    P->in.r0 = cfg->r0;
    P->in.r1 = cfg->r1;
    P->in.rho_max = cfg->rho_max;
    P->in.w_ramp = cfg->w_ramp;
    P->in.rho_ramp = cfg->rho_ramp;
    P->pr.damping = cfg->damping;
    P->pr.gamma0 = cfg->gamma0;
    P->pr.dn = cfg->damp_near;
    P->pr.df = cfg->damp_far;
    P->pr.dw = cfg->damp_width;
    P->pr.dissipation = cfg->dissipation;
    P->pr.eps = cfg->eps_ko;
    P->pr.eo = cfg->eps_out;
    P->pr.ei = cfg->eps_in;
    P->pr.er1 = cfg->eps_r1;
    P->pr.erh = cfg->eps_rh;
    for (int i = 0; i < 3; ++i) {
      P->pr.dc0[i] = cfg->damp_c0[i];
      P->pr.dv[i] = cfg->damp_v[i];
      P->pr.ec0[i] = cfg->eps_c0[i];
      P->pr.ev[i] = cfg->eps_v[i];
    }
    P->diss = P->pr.has_dissipation();
    P->ks = make_ks_source(cfg->ks_M, cfg->ks_spin, cfg->ks_velocity);
    if (cfg->gauge == TGH_GAUGE_SAMPLED) {
      // sample_gauge_source! at t = 0 with the core rule (src/gauge.jl:156-170)
      const size_t S = P->npt_state();
      P->Hsrc.assign(S * NV * P->nb, 0.0);
#pragma omp parallel for schedule(dynamic)
      for (int b = 0; b < P->nb; ++b)
        for (int k = 0; k < P->N1; ++k)
          for (int j = 0; j < P->N1; ++j)
            for (int i = 0; i < P->N1; ++i) {
              int64_t n[3] = {(int64_t)P->corner[3 * b] + i, (int64_t)P->corner[3 * b + 1] + j,
                              (int64_t)P->corner[3 * b + 2] + k};
              double x[3], xc[3];
              P->position(P->level[b], n, x);
              P->in.core_position(0.0, x, xc);
              double p4[4] = {0.0, xc[0], xc[1], xc[2]}, Hl[4], dHl[4][4];
              gauge_source_grad(cfg->bg, p4, Hl, dHl);
              size_t o = (size_t)b * NV * S + i + P->N1 * (j + (size_t)P->N1 * k);
              for (int a = 0; a < 4; ++a) P->Hsrc[o + a * S] = Hl[a];
              for (int kk = 0; kk < 16; ++kk) P->Hsrc[o + (4 + kk) * S] = dHl[kk % 4][kk / 4];
            }
    }
    return P;
  } catch (const std::exception& e) {
    if (errbuf && errlen > 0) {
      std::strncpy(errbuf, e.what(), errlen - 1);
      errbuf[errlen - 1] = 0;
    }
    return nullptr;
  }
}

void orc_destroy(void* p) { delete (Problem*)p; }
const char* orc_last_error(void* p) { return ((Problem*)p)->err.c_str(); }
size_t orc_state_length(void* p) { Problem* P = (Problem*)p; return P->npt_state() * NV * P->nb; }
size_t orc_work_length(void* p) { Problem* P = (Problem*)p; return P->npt_work() * NV * P->nb; }
void orc_set_threads(int n) { omp_set_num_threads(n); }
// The right-hand side's SIMD width: 1 (point by point) or the build's ORC_SIMD_W; returns the width set.
int orc_set_simd_width(void* p, int w) {
  ((Problem*)p)->simd = w == ORC_SIMD_W ? ORC_SIMD_W : 1;
  return ((Problem*)p)->simd;
}
int orc_simd_lanes(void) { return ORC_SIMD_W; }
int orc_get_threads(void) { return omp_get_max_threads(); }

int orc_prepare(void* p, const double* u, double t) {
  try { prepare(*(Problem*)p, u, t); } catch (const std::exception& e) { ((Problem*)p)->err = e.what(); return TGH_ERR_ARG; }
  return TGH_OK;
}
int orc_rhs(void* p, double* du, double t, const double* matter) {
  Problem& P = *(Problem*)p;
  if (P.in.variant == TGH_INT_FITTED && !P.target_set) {
    P.err = "a :fitted interior relaxes toward the target cache: fill or set it first";
    return TGH_ERR_ARG;
  }
  rhs(P, du, t, matter);
  return TGH_OK;
}
int orc_gh_rhs(void* p, double* du, const double* u, double t, const double* matter) {
  int s = orc_prepare(p, u, t);
  if (s) return s;
  return orc_rhs(p, du, t, matter);
}
int orc_copy_work(void* p, double* dst) {
  Problem* P = (Problem*)p;
  std::memcpy(dst, P->work.data(), P->work.size() * sizeof(double));
  return TGH_OK;
}
// the working array set from outside (a filled array of the product's layout): the right-hand
// side of blocks cut out of a larger mesh, whose ghosts another fill has already written
int orc_set_work(void* p, const double* src) {
  Problem* P = (Problem*)p;
  P->work.assign(src, src + P->npt_work() * NV * P->nb);
  return TGH_OK;
}
int orc_copy_hsrc(void* p, double* dst) {
  Problem* P = (Problem*)p;
  std::memcpy(dst, P->Hsrc.data(), P->Hsrc.size() * sizeof(double));
  return TGH_OK;
}
int orc_initial_state(void* p, double* u, double t) { initial_state(*(Problem*)p, u, t); return TGH_OK; }
int orc_stage_limit(void* p, double* u, double t) { stage_limit(*(Problem*)p, u, t); return TGH_OK; }
int orc_set_target(void* p, const double* tw, double t_f) {
  Problem& P = *(Problem*)p;
  const size_t L = (size_t)P.nb * 2 * NV * P.npt_state();
  P.tw.assign(tw, tw + L);
  P.t_f = t_f;
  P.target_set = true;
  return TGH_OK;
}
int orc_fill_target_snapshot(void* p, const double* u, double t_f, double r_fill) {
  fill_target(*(Problem*)p, u, t_f, r_fill, 0.0);
  return TGH_OK;
}
int orc_fill_target_analytic(void* p, double t_f, double r_fill, double dt) {
  fill_target(*(Problem*)p, nullptr, t_f, r_fill, dt);
  return TGH_OK;
}
int orc_fitted_initial_state(void* p, double* u, double t, double d_init) {
  fitted_initial_state(*(Problem*)p, u, t, d_init);
  return TGH_OK;
}
int orc_copy_target(void* p, double* out) {
  const Problem& P = *(Problem*)p;
  std::copy(P.tw.begin(), P.tw.end(), out);
  return TGH_OK;
}
int orc_max_speed(void* p, const double* u, double t, double* lam) { return max_speed(*(Problem*)p, u, t, lam); }
int orc_rk4_step(void* p, double* u, double t, double dt) {
  try { rk4_step(*(Problem*)p, u, t, dt); } catch (const std::exception& e) { ((Problem*)p)->err = e.what(); return TGH_ERR_ARG; }
  return TGH_OK;
}
int orc_error_norm(void* p, const double* u, double t, double* l2, double* linf) {
  error_norm(*(Problem*)p, u, t, l2, linf);
  return TGH_OK;
}
size_t orc_diag_length(void* p) { Problem* P = (Problem*)p; return P->npt_state() * NDIAG * P->nb; }
int orc_gh_constraint(void* p, const double* u, double t, int allpoints, double* diag) {
  gh_constraint(*(Problem*)p, u, t, allpoints != 0, diag);
  return TGH_OK;
}
int orc_adm_constraint(void* p, const double* u, double t, int allpoints, const double* matter, double* diag) {
  adm_constraint(*(Problem*)p, u, t, allpoints != 0, matter, diag);
  return TGH_OK;
}
int orc_constraint_norms(void* p, const double* diag, int weighting, int at_level, double* out16) {
  constraint_norms(*(Problem*)p, diag, weighting == 0, at_level, out16);
  return TGH_OK;
}
// the regrid's transfer: every owned point of every leaf of `pd` takes the value its lattice
// point has in `ps`'s state at t (value20: the primary copy, injection from a finer leaf, else the
// prolongation of the next coarser level; the hook outside the domain)
int orc_transfer(void* pd, void* ps, const double* u_src, double t, double* u_dst) {
  Problem& D = *(Problem*)pd;
  const Problem& Sr = *(Problem*)ps;
  const std::vector<double> u(u_src, u_src + Sr.npt_state() * NV * Sr.nb);
  const size_t S = D.npt_state();
  try {
    for (int b = 0; b < D.nb; ++b)
      for (int k = 0; k < D.N1; ++k)
        for (int j = 0; j < D.N1; ++j)
          for (int i = 0; i < D.N1; ++i) {
            int64_t n[3] = {(int64_t)D.corner[3 * b] + i, (int64_t)D.corner[3 * b + 1] + j,
                            (int64_t)D.corner[3 * b + 2] + k};
            double out[NV];
            value20(Sr, u, t, D.level[b], n, out);
            for (int v = 0; v < NV; ++v) u_dst[(size_t)b * NV * S + v * S + i + D.N1 * (j + (size_t)D.N1 * k)] = out[v];
          }
  } catch (const std::exception& e) {
    D.err = e.what();
    return TGH_ERR_ARG;
  }
  return TGH_OK;
}
int orc_tau(void* p, const double* u, double t, int allpoints, double eps, double scale, double* diag, double* out12) {
  tau(*(Problem*)p, u, t, allpoints != 0, eps, scale, diag, out12);
  return TGH_OK;
}
int orc_firing(void* p, const double* diag, int ntol, const double* tol, int* counts, int* boxes) {
  firing(*(Problem*)p, diag, ntol, tol, counts, boxes);
  return TGH_OK;
}
// the pointwise pieces alone, for the pins of test/constraints_tests.jl:63-158
void orc_ddmetric(const tgh_background* bg, const double* p4, double* g16, double* dg64, double* ddg256) {
  double g[4][4], dg[4][4][4], ddg[4][4][4][4];
  ddmetric(*bg, p4, g, dg, ddg);
  std::memcpy(g16, g, sizeof(g));
  std::memcpy(dg64, dg, sizeof(dg));
  std::memcpy(ddg256, ddg, sizeof(ddg));
}
void orc_adm_at_node(const double* h10, const double* dg64, const double* ddg256, double* out4) {
  Coef<double> C;
  metric_quantities(h10, C);
  double dg[4][4][4], ddg[4][4][4][4], ham, mom[3];
  std::memcpy(dg, dg64, sizeof(dg));
  std::memcpy(ddg, ddg256, sizeof(ddg));
  adm_constraints_at_node(C.g4, C.gu4, C.alpha, C.beta, dg, ddg, ham, mom);
  out4[0] = ham;
  for (int a = 0; a < 3; ++a) out4[1 + a] = mom[a];
}
// the same with the Ricci tensor contracted in the GPU kernel's order
void orc_adm_at_node_streamed(const double* h10, const double* dg64, const double* ddg256, double* out4) {
  Coef<double> C;
  metric_quantities(h10, C);
  double dg[4][4][4], ddg[4][4][4][4], ham, mom[3];
  std::memcpy(dg, dg64, sizeof(dg));
  std::memcpy(ddg, ddg256, sizeof(ddg));
  adm_constraints_streamed(C.g4, C.gu4, C.alpha, C.beta, dg, ddg, ham, mom);
  out4[0] = ham;
  for (int a = 0; a < 3; ++a) out4[1 + a] = mom[a];
}
// out: d alpha, d beta (3), d sqrt(gamma), d gamma^{jk} (9) along the direction of dg10
void orc_metric_derivatives_along(const double* h10, const double* dg10, double* out14) {
  Coef<double> C;
  metric_quantities(h10, C);
  double dal, dbeta[3], dsq, dgamu[3][3];
  metric_derivatives_along(C, dg10, dal, dbeta, dsq, dgamu);
  out14[0] = dal;
  for (int j = 0; j < 3; ++j) out14[1 + j] = dbeta[j];
  out14[4] = dsq;
  for (int j = 0; j < 3; ++j)
    for (int k = 0; k < 3; ++k) out14[5 + 3 * j + k] = dgamu[j][k];
}
// metric_derivatives at a point (three directions): d alpha (3), d beta [i][j] (9), dA [i][j][k] (27)
void orc_metric_derivatives(const double* h10, const double* dh30, double* out39) {
  Coef<double> C;
  metric_quantities(h10, C);
  const double* dh[3] = {dh30, dh30 + NC, dh30 + 2 * NC};
  double dal[3], dbeta[3][3], dA[3][3][3];
  metric_derivatives(C, dh, dal, dbeta, dA);
  for (int i = 0; i < 3; ++i) out39[i] = dal[i];
  std::memcpy(out39 + 3, dbeta, sizeof(dbeta));
  std::memcpy(out39 + 12, dA, sizeof(dA));
}

// test/evolution_tests.jl:37-89: the expanded reference spelling at one owned point of
// the current working array, with the dissipation correction of the source.
int orc_host_rhs_at(void* p, int b, int i, int j, int k, double t, double out[20]) {
  Problem& P = *(Problem*)p;
  const double h = P.spacing(P.level[b]);
  const double* wk = P.work.data() + (size_t)b * NV * P.npt_work();
  const size_t sv = P.npt_work();
  const long st[3] = {1, P.W, (long)P.W * P.W};
  const size_t var = (size_t)(i + P.G) + P.W * ((size_t)(j + P.G) + (size_t)P.W * (k + P.G));
  int64_t n[3] = {(int64_t)P.corner[3 * b] + i, (int64_t)P.corner[3 * b + 1] + j, (int64_t)P.corner[3 * b + 2] + k};
  double x[3];
  P.position(P.level[b], n, x);
  double g0 = P.pr.damping_rate(t, x);
  double hv[NC], Pv[NC], dhs[3][NC], dPs[3][NC], dds[6][NC];
  for (int v = 0; v < NC; ++v) {
    hv[v] = wk[var + v * sv];
    Pv[v] = wk[var + (NC + v) * sv];
    for (int d = 0; d < 3; ++d) {
      dhs[d][v] = axis_stencil(P.st.w1, wk, var + v * sv, st[d]) / h;
      dPs[d][v] = axis_stencil(P.st.w1, wk, var + (NC + v) * sv, st[d]) / h;
    }
    const int pairs[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
    for (int m = 0; m < 6; ++m) {
      int d1 = pairs[m][0], d2 = pairs[m][1];
      dds[m][v] = d1 == d2 ? axis_stencil(P.st.w2, wk, var + v * sv, st[d1]) / (h * h)
                           : mixed_stencil(P.st.w1, wk, var + v * sv, st[d1], st[d2]) / (h * h);
    }
  }
  const double* dh[3] = {dhs[0], dhs[1], dhs[2]};
  const double* dP[3] = {dPs[0], dPs[1], dPs[2]};
  const double* dd[6] = {dds[0], dds[1], dds[2], dds[3], dds[4], dds[5]};
  double Hl[4], dHl[4][4];
  int I[3] = {i, j, k};
  double dth0[NC];
  {
    // gauge source: the sampled field, or the closed form from the undissipated d_t h
    Coef<double> C;
    metric_quantities(hv, C);
    double a_div = C.alpha / C.sqrtg;
    for (int v = 0; v < NC; ++v)
      dth0[v] = C.beta[0] * dh[0][v] + C.beta[1] * dh[1][v] + C.beta[2] * dh[2][v] + a_div * Pv[v];
  }
  double eps = P.pr.dissipation_rate(t, x);
  double Qh[NC], QP[NC];
  for (int v = 0; v < NC; ++v) {
    Qh[v] = (eps / h) * ((axis_stencil(P.st.wD, wk, var + v * sv, st[0]) + axis_stencil(P.st.wD, wk, var + v * sv, st[1])) +
                         axis_stencil(P.st.wD, wk, var + v * sv, st[2]));
    QP[v] = (eps / h) * ((axis_stencil(P.st.wD, wk, var + (NC + v) * sv, st[0]) +
                          axis_stencil(P.st.wD, wk, var + (NC + v) * sv, st[1])) +
                         axis_stencil(P.st.wD, wk, var + (NC + v) * sv, st[2]));
  }
  double dthq[NC];
  for (int v = 0; v < NC; ++v) dthq[v] = P.diss ? dth0[v] + Qh[v] : dth0[v];
  gauge_at_point(P, b, I, hv, dthq, dh, Hl, dHl);
  double dth[NC], dtP[NC];
  gh_node_rhs_expanded(hv, Pv, dh, dP, dd, Hl, dHl, g0, P.cfg.gamma2, dth, dtP);
  if (P.diss) {
    Coef<double> C;
    metric_quantities(hv, C);
    double dg1[4][4][4], dg2[4][4][4], s1[NC], s2[NC], dtq[NC];
    for (int v = 0; v < NC; ++v) dtq[v] = dth[v] + Qh[v];
    dg4(dtq, dh, dg1);
    dg4(dth, dh, dg2);
    gh_node_source(C, dg1, Hl, dHl, g0, P.cfg.gamma2, s1);
    gh_node_source(C, dg2, Hl, dHl, g0, P.cfg.gamma2, s2);
    for (int v = 0; v < NC; ++v) {
      dth[v] = dth[v] + Qh[v];
      dtP[v] = dtP[v] + QP[v] + (s1[v] - s2[v]);
    }
  }
  for (int v = 0; v < NC; ++v) {
    out[v] = dth[v];
    out[NC + v] = dtP[v];
  }
  return TGH_OK;
}

// test/evolution_tests.jl:97-108
double orc_rhs_scale(void* p, int b, int i, int j, int k) {
  Problem& P = *(Problem*)p;
  const double h = P.spacing(P.level[b]);
  const double* wk = P.work.data() + (size_t)b * NV * P.npt_work();
  const size_t sv = P.npt_work();
  const long st[3] = {1, P.W, (long)P.W * P.W};
  const size_t var = (size_t)(i + P.G) + P.W * ((size_t)(j + P.G) + (size_t)P.W * (k + P.G));
  double s = 0.0;
  for (int v = 0; v < NV; ++v)
    for (int d = 0; d < 3; ++d) {
      double a = std::fabs(axis_stencil(P.st.w2, wk, var + v * sv, st[d])) / (h * h);
      double c = std::fabs(wk[var + v * sv]);
      s = std::max(s, std::max(a, c));
    }
  return std::max(s, 1.0);
}

// ---- pointwise entry points for the unit tests ----
int orc_weights(int q, int m, int64_t* num, int64_t* den) {
  std::vector<Rat> w = m == 0 ? rational_dissipation_weights(q) : rational_derivative_weights(q, m);
  for (size_t i = 0; i < w.size(); ++i) {
    num[i] = (int64_t)w[i].n;
    den[i] = (int64_t)w[i].d;
  }
  return (int)w.size();
}
int orc_weights_double(int q, int m, double* out) {
  std::vector<Rat> w = m == 0 ? rational_dissipation_weights(q) : rational_derivative_weights(q, m);
  std::vector<double> d = to_double(w);
  for (size_t i = 0; i < d.size(); ++i) out[i] = d[i];
  return (int)d.size();
}
// The right-hand side's stencil sums on a caller's array, for the tests that pin their order:
// which 1 = first derivative, 2 = second derivative, 0 = dissipation (axis_stencil at `base`
// along `stride`); orc_mixed_stencil is the first-derivative tensor product, outer along s1.
double orc_axis_stencil(int q, int which, const double* data, long base, long stride) {
  const Stencils st(q);
  const std::vector<double>& w = which == 1 ? st.w1 : which == 2 ? st.w2 : st.wD;
  return axis_stencil<double>(w, data, (size_t)base, stride);
}
double orc_mixed_stencil(int q, const double* data, long base, long s1, long s2) {
  const Stencils st(q);
  return mixed_stencil<double>(st.w1, data, (size_t)base, s1, s2);
}
// out: g4[16], gu4[16], alpha, beta[3], gamu[9], sqrtg
void orc_metric_quantities(const double* h, double* out) {
  Coef<double> C;
  metric_quantities(h, C);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      out[a * 4 + b] = C.g4[a][b];
      out[16 + a * 4 + b] = C.gu4[a][b];
    }
  out[32] = C.alpha;
  for (int i = 0; i < 3; ++i) out[33 + i] = C.beta[i];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) out[36 + 3 * i + j] = C.gamu[i][j];
  out[45] = C.sqrtg;
}
// dh: [3][10]; dHl: [4][4] row-major dHl[a][b] = d_a H_b; which: 0 lean, 1 reference spelling
void orc_source(int which, const double* h, const double* dth, const double* dh, const double* Hl,
                const double* dHl, double g0, double g2, double* msrc) {
  Coef<double> C;
  metric_quantities(h, C);
  const double* d3[3] = {dh, dh + 10, dh + 20};
  double H[4][4];
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) H[a][b] = dHl[a * 4 + b];
  if (which == 0) {
    gh_node_source_lean(C, dth, d3, Hl, H, g0, g2, msrc);
  } else {
    double dg[4][4][4];
    dg4(dth, d3, dg);
    gh_node_source(C, dg, Hl, H, g0, g2, msrc);
  }
}
// divergences: which 0 lean (metric_divergences), 1 contraction of metric_derivatives
void orc_divergences(int which, const double* h, const double* dh, double* out4) {
  Coef<double> C;
  metric_quantities(h, C);
  const double* d3[3] = {dh, dh + 10, dh + 20};
  if (which == 0) {
    metric_divergences(C, d3, out4[0], out4 + 1);
  } else {
    double dal[3], db[3][3], dA[3][3][3];
    metric_derivatives(C, d3, dal, db, dA);
    out4[0] = (db[0][0] + db[1][1]) + db[2][2];
    for (int j = 0; j < 3; ++j) out4[1 + j] = (dA[0][0][j] + dA[1][1][j]) + dA[2][2][j];
  }
}
void orc_dmetric(const tgh_background* bg, const double* p4, double* g16, double* dg64) {
  double g[4][4], dg[4][4][4];
  dmetric(*bg, p4, g, dg);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      g16[a * 4 + b] = g[a][b];
      for (int c = 0; c < 4; ++c) dg64[(a * 4 + b) * 4 + c] = dg[a][b][c];
    }
}
void orc_background_state(const tgh_background* bg, double t, const double* x3, double* h, double* Pi, double* dh30,
                          double* dtg) {
  double dh[3][NC];
  background_state(*bg, t, x3, h, Pi, dh, dtg);
  for (int d = 0; d < 3; ++d)
    for (int v = 0; v < NC; ++v) dh30[d * NC + v] = dh[d][v];
}
void orc_gauge_source_grad(const tgh_background* bg, const double* p4, double* Hl, double* dHl16) {
  double dH[4][4];
  gauge_source_grad(*bg, p4, Hl, dH);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) dHl16[a * 4 + b] = dH[a][b];
}
void orc_algebraic_gauge_source(double M, const double* spin, const double* vel, const double* h, const double* dth,
                                const double* dh30, double* Hl, double* dHl16) {
  KSSource k = make_ks_source(M, spin, vel);
  const double* d3[3] = {dh30, dh30 + 10, dh30 + 20};
  double dH[4][4];
  algebraic_gauge_source(k, h, dth, d3, Hl, dH);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) dHl16[a * 4 + b] = dH[a][b];
}
double orc_smoothstep(double s) { return smoothstep(s); }

}  // extern "C"

// ---- an op-counting scalar: the algorithmic FP64 work of one right-hand-side point ----
namespace orc {
struct Cnt {
  double v;
  static long nadd, nmul, ndiv, nsqrt;
  Cnt() : v(0) {}
  Cnt(double x) : v(x) {}
};
long Cnt::nadd = 0, Cnt::nmul = 0, Cnt::ndiv = 0, Cnt::nsqrt = 0;
static inline Cnt operator+(Cnt a, Cnt b) { ++Cnt::nadd; return Cnt(a.v + b.v); }
static inline Cnt operator-(Cnt a, Cnt b) { ++Cnt::nadd; return Cnt(a.v - b.v); }
static inline Cnt operator-(Cnt a) { return Cnt(-a.v); }
static inline Cnt operator*(Cnt a, Cnt b) {
  // products by an exact zero weight (the first derivative's center tap) are not work
  if (a.v != 0.0 && b.v != 0.0) ++Cnt::nmul;
  return Cnt(a.v * b.v);
}
static inline Cnt operator/(Cnt a, Cnt b) { ++Cnt::ndiv; return Cnt(a.v / b.v); }
static inline bool operator!=(Cnt a, Cnt b) { return a.v != b.v; }
static inline Cnt sqrt(Cnt a) { ++Cnt::nsqrt; return Cnt(std::sqrt(a.v)); }
static inline double dval(Cnt a) { return a.v; }
static inline Cnt select_pos(Cnt c, Cnt a, Cnt b) { return c.v > 0 ? a : b; }
}  // namespace orc

extern "C" {
// Counts the floating-point operations of F(u) at one interior owned point of block 0 of a
// prepared problem (no interior branches). out: adds, multiplies, divides, square roots.
// A multiply feeding an add is counted as two operations (an FMA is 2 flops).
int orc_count_flops(void* p, double t, long* out) {
  Problem& P = *(Problem*)p;
  PointCtx c;
  c.wk = P.work.data();
  c.sv = P.npt_work();
  c.st[0] = 1;
  c.st[1] = P.W;
  c.st[2] = P.W * P.W;
  const int I[3] = {P.N / 2, P.N / 2, P.N / 2};
  c.var = (size_t)(I[0] + P.G) + P.W * ((size_t)(I[1] + P.G) + (size_t)P.W * (I[2] + P.G));
  int64_t n[3] = {(int64_t)P.corner[0] + I[0], (int64_t)P.corner[1] + I[1], (int64_t)P.corner[2] + I[2]};
  double x[3];
  P.position(P.level[0], n, x);
  Cnt::nadd = Cnt::nmul = Cnt::ndiv = Cnt::nsqrt = 0;
  Cnt a[NC], b[NC];
  try {
    rhs_at_point<Cnt>(P, c, 0, I, x, t, nullptr, a, b);
  } catch (const std::exception& e) {
    P.err = e.what();
    return TGH_ERR_ARG;
  }
  out[0] = Cnt::nadd;
  out[1] = Cnt::nmul;
  out[2] = Cnt::ndiv;
  out[3] = Cnt::nsqrt;
  return TGH_OK;
}

// bounds_project (src/bounds.jl:458-527) at one point: h10, P10 in; the projected state out,
// flags2 = (hit, nonfinite). bd7: alpha_min, alpha_max, lambda_min, lambda_max, beta_max, K_max,
// r_gate.
void orc_bounds_project(const double* h10, const double* P10, const double* bd7, double* hout, double* Pout,
                        int* flags2) {
  Bounds bd{bd7[0], bd7[1], bd7[2], bd7[3], bd7[4], bd7[5], bd7[6]};
  for (int v = 0; v < 10; ++v) {
    hout[v] = h10[v];
    Pout[v] = P10[v];
  }
  bool nf = false;
  flags2[0] = bounds_project(hout, Pout, bd, nf) ? 1 : 0;
  flags2[1] = nf ? 1 : 0;
}

// gh_bounds_kernel! (src/bounds.jl:635-663) over a state vector u in place: every owned point
// at interior radius r < r_gate is projected and written back only where it fired. Counted
// over the primary copies (each lattice point once): fired, non-finite, and the largest r at
// which it fired (0 when none).
int orc_apply_bounds(void* p, double* u, double t, const double* bd7, long* fired, long* nonfinite, double* rmax) {
  Problem& P = *(Problem*)p;
  Bounds bd{bd7[0], bd7[1], bd7[2], bd7[3], bd7[4], bd7[5], bd7[6]};
  const size_t S = P.npt_state();
  long nf = 0, nn = 0;
  double rm = 0.0;
  for (int b = 0; b < P.nb; ++b)
    for (int k = 0; k < P.N1; ++k)
      for (int j = 0; j < P.N1; ++j)
        for (int i = 0; i < P.N1; ++i) {
          double x[3];
          int64_t n[3] = {(int64_t)P.corner[3 * b] + i, (int64_t)P.corner[3 * b + 1] + j,
                          (int64_t)P.corner[3 * b + 2] + k};
          P.position(P.level[b], n, x);
          const double r = P.in.radius(t, x);
          if (!(r < bd.r_gate)) continue;
          const size_t o = (size_t)b * NV * S + i + P.N1 * (j + (size_t)P.N1 * k);
          double h[10], Pi[10];
          for (int v = 0; v < 10; ++v) {
            h[v] = u[o + v * S];
            Pi[v] = u[o + (10 + v) * S];
          }
          bool nfin = false;
          const bool hit = bounds_project(h, Pi, bd, nfin);
          if (hit)
            for (int v = 0; v < 10; ++v) {
              u[o + v * S] = h[v];
              u[o + (10 + v) * S] = Pi[v];
            }
          if (is_primary(P, b, i, j, k)) {
            if (hit) {
              ++nf;
              rm = std::fmax(rm, r);
            }
            if (nfin) ++nn;
          }
        }
  *fired = nf;
  *nonfinite = nn;
  *rmax = rm;
  return TGH_OK;
}

// The same count for a constraint monitor at that point (which = 0: the gauge constraint,
// 1: the ADM constraints, vacuum, the reference's Ricci assembly; 2: the same with the Ricci
// tensor contracted in the GPU kernel's order), on a prepared problem.
int orc_count_monitor_flops(void* p, double t, int which, long* out) {
  Problem& P = *(Problem*)p;
  const int I[3] = {P.N / 2, P.N / 2, P.N / 2};
  double x[3];
  PointCtx c = point_ctx(P, 0, I, x);
  Cnt::nadd = Cnt::nmul = Cnt::ndiv = Cnt::nsqrt = 0;
  Cnt r[4];
  if (which == 0) gh_constraint_point<Cnt>(P, c, 0, I, r);
  else if (which == 1) adm_constraint_point<Cnt>(P, c, 0, I, x, t, nullptr, r);
  else adm_constraint_point<Cnt, true>(P, c, 0, I, x, t, nullptr, r);
  out[0] = Cnt::nadd;
  out[1] = Cnt::nmul;
  out[2] = Cnt::ndiv;
  out[3] = Cnt::nsqrt;
  return TGH_OK;
}
}
