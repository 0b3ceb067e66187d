// The fused right-hand side of the generalized-harmonic system at one owned point per
// thread, in the reference's streaming order (src/evolution.jl:258-388):
//   1. h, Pi at the point; the 30 first derivatives d_i h; the coefficient set;
//   2. d_t h = beta^i d_i h + (alpha/sqrt(gamma)) Pi + (eps/h) sum_d KO_d(h), stored at once;
//   3. the gauge source, the reduced source with damping (+ matter);
//   4. per component v (run-time loop): beta^i d_i Pi + (d_i beta^i) Pi + d_i A^{ij} d_j h
//      + A^{ij} d_i d_j h + (eps/h) sum_d KO_d(Pi) + msrc_v, stored as it is finished.
// The interior branches of gh_rhs_point! (src/evolution.jl:489-695) wrap it: the frozen
// core is asked before any stencil is read.
//
// Two epilogues share the body:
//   MODE_DU     write du in state layout (the plain form, rhs!)
//   MODE_STAGE  the RK4 stage update in place of du: acc and the next stage's ghosted
//               working array are written, u_n read (the batched form)
#pragma once
#include <type_traits>

#include "algebra.cuh"
#include "tangent.cuh"

namespace tgh {

enum { MODE_DU = 0, MODE_STAGE = 1 };

// finite-difference weights on unit spacing (exact rationals, correctly rounded once)
template <int Q> struct W;
template <> struct W<2> {
  static constexpr int R = 1, RD = 2;
  __device__ static constexpr double d1(int k) { return k == 1 ? 1.0 / 2.0 : 0.0; }  // antisymmetric, k > 0
  __device__ static constexpr double d2(int k) { return k == 0 ? -2.0 : 1.0; }
  __device__ static constexpr double ko(int k) { return k == 0 ? -6.0 / 16.0 : k == 1 ? 4.0 / 16.0 : -1.0 / 16.0; }
};
template <> struct W<4> {
  static constexpr int R = 2, RD = 3;
  __device__ static constexpr double d1(int k) { return k == 1 ? 2.0 / 3.0 : -1.0 / 12.0; }
  __device__ static constexpr double d2(int k) { return k == 0 ? -5.0 / 2.0 : k == 1 ? 4.0 / 3.0 : -1.0 / 12.0; }
  __device__ static constexpr double ko(int k) {
    return k == 0 ? -20.0 / 64.0 : k == 1 ? 15.0 / 64.0 : k == 2 ? -6.0 / 64.0 : 1.0 / 64.0;
  }
};
template <> struct W<6> {
  static constexpr int R = 3, RD = 4;
  __device__ static constexpr double d1(int k) { return k == 1 ? 3.0 / 4.0 : k == 2 ? -3.0 / 20.0 : 1.0 / 60.0; }
  __device__ static constexpr double d2(int k) {
    return k == 0 ? -49.0 / 18.0 : k == 1 ? 3.0 / 2.0 : k == 2 ? -3.0 / 20.0 : 1.0 / 90.0;
  }
  __device__ static constexpr double ko(int k) {
    return k == 0 ? -70.0 / 256.0 : k == 1 ? 56.0 / 256.0 : k == 2 ? -28.0 / 256.0 : k == 3 ? 8.0 / 256.0 : -1.0 / 256.0;
  }
};
template <> struct W<8> {
  static constexpr int R = 4, RD = 5;
  __device__ static constexpr double d1(int k) {
    return k == 1 ? 4.0 / 5.0 : k == 2 ? -1.0 / 5.0 : k == 3 ? 4.0 / 105.0 : -1.0 / 280.0;
  }
  __device__ static constexpr double d2(int k) {
    return k == 0 ? -205.0 / 72.0 : k == 1 ? 8.0 / 5.0 : k == 2 ? -1.0 / 5.0 : k == 3 ? 8.0 / 315.0 : -1.0 / 560.0;
  }
  __device__ static constexpr double ko(int k) {
    return k == 0 ? -252.0 / 1024.0
                  : k == 1 ? 210.0 / 1024.0
                           : k == 2 ? -120.0 / 1024.0 : k == 3 ? 45.0 / 1024.0 : k == 4 ? -10.0 / 1024.0 : 1.0 / 1024.0;
  }
};

template <class T> __device__ __forceinline__ T ld(const double* p) { return T(__ldg(p)); }
// in the tangent-linear kernel a working-array value comes with its tangent
template <> __device__ __forceinline__ Tan ld<Tan>(const double* p) { return Tan(__ldg(p), __ldg(p + c_tan_off)); }
// a value that carries no tangent (the sampled gauge source, the matter term)
template <class T> __device__ __forceinline__ T ldk(const double* p) { return T(__ldg(p)); }

// The stencils. With T = double the second differences are the reference's sums, term by
// term (below); the first differences and the dissipation pair the taps at +-k. With
// T = float (the mixed form) every difference of state values is formed in FP64, where it
// cancels, and rounded once; the weighted sum then runs in FP32. The symmetric stencils use
// that their weights sum to zero: w_0 c + sum_k w_k (u_k + u_-k) = sum_k w_k ((u_k - c) + (u_-k - c)).
template <class T> __host__ __device__ constexpr bool is_fp32() { return sizeof(T) == sizeof(float); }

// sum_k w_k u[k s] on the antisymmetric first-derivative stencil (center weight zero)
template <int Q, class T> __device__ __forceinline__ T st_d1(const double* p, long s) {
  T acc = T(0.0);
#pragma unroll
  for (int k = 1; k <= W<Q>::R; ++k) {
    if constexpr (!is_fp32<T>()) acc = fma(T(W<Q>::d1(k)), ld<T>(p + k * s) - ld<T>(p - k * s), acc);
    else acc = fma(T(W<Q>::d1(k)), T(ld<double>(p + k * s) - ld<double>(p - k * s)), acc);
  }
  return acc;
}
// The first-derivative weight at a signed offset (the table holds k > 0; d1(-k) = -d1(k) exactly).
template <int Q> __device__ __forceinline__ constexpr double d1s(int k) { return k > 0 ? W<Q>::d1(k) : -W<Q>::d1(-k); }

// The second differences in FP64 are the reference's sums term by term (axis_stencil and
// mixed_stencil, src/evolution.jl:192-219): from the lowest offset to the highest, each
// product and each sum rounded on its own (no fused multiply-add), so that they are the
// reference's bits. Their terms are O(|u|) and their value O(h^2 |u''|), so any other order
// or rounding differs by eps |u| / h^2, which at fine spacing is above 1e-12 of the right-hand
// side's scale. Terms of zero weight (the centre of a first-derivative table) are exact zeros
// there and are left out. The first differences and the dissipation, whose rounding is scaled
// by 1/h only, keep the paired form with fused multiply-adds.
template <int Q> __device__ __forceinline__ double st_d2_ref(const double* p, long s, double c) {
  constexpr int R = W<Q>::R;
  double acc = __dmul_rn(W<Q>::d2(R), __ldg(p - R * s));
#pragma unroll
  for (int k = -R + 1; k <= R; ++k) {
    const double u = k == 0 ? c : __ldg(p + k * s);
    acc = __dadd_rn(acc, __dmul_rn(W<Q>::d2(k < 0 ? -k : k), u));
  }
  return acc;
}
// outer sum along s1, inner along s2
template <int Q> __device__ __forceinline__ double st_mixed_ref(const double* p, long s1, long s2) {
  constexpr int R = W<Q>::R;
  double outer = 0.0;
#pragma unroll
  for (int a = -R; a <= R; ++a) {
    if (a == 0) continue;
    const double* pa = p + a * s1;
    double in = __dmul_rn(d1s<Q>(-R), __ldg(pa - R * s2));
#pragma unroll
    for (int e = -R + 1; e <= R; ++e) {
      if (e == 0) continue;
      in = __dadd_rn(in, __dmul_rn(d1s<Q>(e), __ldg(pa + e * s2)));
    }
    outer = a == -R ? __dmul_rn(d1s<Q>(a), in) : __dadd_rn(outer, __dmul_rn(d1s<Q>(a), in));
  }
  return outer;
}

template <int Q, class T> __device__ __forceinline__ T st_d2(const double* p, long s, T c) {
  if constexpr (std::is_same<T, double>::value) {
    return st_d2_ref<Q>(p, s, c);
  } else if constexpr (!is_fp32<T>()) {
    T acc = T(W<Q>::d2(0)) * c;
#pragma unroll
    for (int k = 1; k <= W<Q>::R; ++k) acc = fma(T(W<Q>::d2(k)), ld<T>(p + k * s) + ld<T>(p - k * s), acc);
    return acc;
  } else {
    const double c0 = ld<double>(p);
    T acc = T(0.0);
#pragma unroll
    for (int k = 1; k <= W<Q>::R; ++k)
      acc = fma(T(W<Q>::d2(k)), T((ld<double>(p + k * s) - c0) + (ld<double>(p - k * s) - c0)), acc);
    return acc;
  }
}
template <int Q, class T> __device__ __forceinline__ T st_ko(const double* p, long s, T c) {
  if constexpr (!is_fp32<T>()) {
    T acc = T(W<Q>::ko(0)) * c;
#pragma unroll
    for (int k = 1; k <= W<Q>::RD; ++k) acc = fma(T(W<Q>::ko(k)), ld<T>(p + k * s) + ld<T>(p - k * s), acc);
    return acc;
  } else {
    const double c0 = ld<double>(p);
    T acc = T(0.0);
#pragma unroll
    for (int k = 1; k <= W<Q>::RD; ++k)
      acc = fma(T(W<Q>::ko(k)), T((ld<double>(p + k * s) - c0) + (ld<double>(p - k * s) - c0)), acc);
    return acc;
  }
}
// d_1 d_2 as the tensor product of two first-derivative stencils
template <int Q, class T> __device__ __forceinline__ T st_mixed(const double* p, long s1, long s2) {
  if constexpr (std::is_same<T, double>::value) return st_mixed_ref<Q>(p, s1, s2);
  T acc = T(0.0);
#pragma unroll
  for (int a = 1; a <= W<Q>::R; ++a) {
    T in = T(0.0);
#pragma unroll
    for (int e = 1; e <= W<Q>::R; ++e) {
      const double* pp = p + a * s1;
      const double* pm = p - a * s1;
      T d;
      if constexpr (!is_fp32<T>())
        d = (ld<T>(pp + e * s2) - ld<T>(pp - e * s2)) - (ld<T>(pm + e * s2) - ld<T>(pm - e * s2));
      else
        d = T((ld<double>(pp + e * s2) - ld<double>(pp - e * s2)) - (ld<double>(pm + e * s2) - ld<double>(pm - e * s2)));
      in = fma(T(W<Q>::d1(e)), d, in);
    }
    acc = fma(T(W<Q>::d1(a)), in, acc);
  }
  return acc;
}

// Per-point coefficients the head kernel leaves for the Pi kernel (struct of arrays,
// slot c of point p at coef[c * npts + p]).
enum {
  CF_B0 = 0, CF_B1, CF_B2,            // beta^i
  CF_DIVB,                            // d_i beta^i
  CF_DA0, CF_DA1, CF_DA2,             // d_i (alpha sqrt(gamma) gamma^{ij})
  CF_AXX, CF_AXY, CF_AXZ, CF_AYY, CF_AYZ, CF_AZZ,  // alpha sqrt(gamma) gamma^{ij}, off-diagonals doubled
  CF_EH,                              // eps_KO / h
  CF_W,                               // the layer's w (1 outside; negative: the point is finished)
  CF_M0,                              // 10 additive terms: msrc (+ the layer's relaxation)
  CF_DTH0 = CF_M0 + NC,               // batched form: the 10 d_t h values, updated by the Pi kernel
  NCOEF = CF_DTH0 + NC
};

// one launch's geometry and buffers
struct RhsArgs {
  const double* work;     // ghosted working array, (W^3 x 20) per block
  const double* Hsrc;     // sampled gauge source, (N1^3 x 20) per block, or null
  const double* matter;   // (N1^3 x 10) per block, or null
  const double* blk;      // per block: domain lo (3), h, integer corner (3), pad
  double* coef;           // NCOEF x npts scratch between the two kernels
  double* du;             // MODE_DU: state layout
  // MODE_STAGE
  const double* u0;       // state at the start of the step (ghosted layout)
  double* acc;            // accumulator (state layout)
  double* next;           // the next stage's ghosted working array (owned points written)
  double ca, cb;          // next = u0 + ca k ; acc = (stage 1 ? u0 : acc) + cb k ; final: next = acc + cb k
  int stage;              // 1..4
  int N1, Wd, G, Wx;      // block edge + 1, ghosted cube edge, ghost width, row pitch
  long npts;              // N1^3 * nblocks
  long p0, p1;            // the points [p0, p1) this launch covers (whole blocks)
  double t;
  int threads;            // CTA size of the launch (64 or 128)
  int pi_mb;              // the one-point Pi kernel's resident CTAs per SM (3, 4 or 5)
};

// Where a finished component goes: straight to du (plain form) or into the RK4 stage
// update (batched form).
struct EmitDu {
  double* d;
  long S;
  __device__ __forceinline__ void put(int v, double val) { d[v * S] = val; }
};
struct EmitStage {
  double* ac;
  double* nx;
  const double* u0;
  long S, sv;
  double ca, cb;
  int stage;
  __device__ __forceinline__ void put(int v, double kv) {
    if (stage == 4) {
      nx[v * sv] = fma(cb, kv, ac[v * S]);
    } else {
      const double un = u0[v * sv];
      ac[v * S] = fma(cb, kv, stage == 1 ? un : ac[v * S]);
      nx[v * sv] = fma(ca, kv, un);
    }
  }
  // the same update in two halves, so that its loads can be issued before k is known
  __device__ __forceinline__ double pre_u(int v) const { return stage == 4 ? 0.0 : u0[v * sv]; }
  __device__ __forceinline__ double pre_a(int v) const { return stage == 1 ? 0.0 : ac[v * S]; }
  __device__ __forceinline__ void fin(int v, double kv, double un, double a) {
    if (stage == 4) {
      nx[v * sv] = fma(cb, kv, a);
    } else {
      ac[v * S] = fma(cb, kv, stage == 1 ? un : a);
      nx[v * sv] = fma(ca, kv, un);
    }
  }
};

// the owned point p of a launch: block, index within the block, position, work offset
struct PointIdx {
  int b, i, j, k;
  long ip, wo;
  double x[3], h;
};
__device__ __forceinline__ PointIdx point_index(const RhsArgs& A, long p) {
  PointIdx q;
  const int N1 = A.N1;
  const long S = (long)N1 * N1 * N1;
  q.b = (int)(p / S);
  q.ip = p - (long)q.b * S;
  q.k = (int)(q.ip / ((long)N1 * N1));
  q.j = (int)((q.ip / N1) % N1);
  q.i = (int)(q.ip % N1);
  const double* bl = A.blk + 8 * q.b;
  q.h = bl[3];
  q.x[0] = __dadd_rn(bl[0], __dmul_rn(bl[4] + (double)q.i, q.h));
  q.x[1] = __dadd_rn(bl[1], __dmul_rn(bl[5] + (double)q.j, q.h));
  q.x[2] = __dadd_rn(bl[2], __dmul_rn(bl[6] + (double)q.k, q.h));
  const long sv = (long)A.Wx * A.Wd * A.Wd;
  q.wo = (long)q.b * NV * sv + (q.i + A.G) + (long)A.Wx * ((q.j + A.G) + (long)A.Wd * (q.k + A.G));
  return q;
}

// The launch's geometry with the block size fixed at compile time when N1S > 0 (the usual
// N = 32 blocks): every stencil offset is then an immediate of its load instruction.
template <int Q, int N1S> __device__ __forceinline__ RhsArgs fixed_geometry(const RhsArgs& A) {
  RhsArgs B = A;
  if (N1S > 0) {
    B.N1 = N1S;
    B.G = Q / 2 + 1;
    B.Wd = N1S + 2 * (Q / 2 + 1);
    B.Wx = B.Wd + (B.Wd & 1);
  }
  return B;
}

// The arithmetic of the state and the coefficient set (inverse metric, lapse, sqrt(gamma)):
// FP64 in the FP64 and the mixed form, and with its tangent in the tangent-linear kernel.
template <class T> struct StateT {
  using type = double;
};
template <> struct StateT<Tan> {
  using type = Tan;
};

// Steps 1-2 of the streaming order at one point (src/evolution.jl:258-285): the state, the
// 30 first derivatives of h, the coefficient set and d_t h (with the dissipation). The state
// and the coefficient set are in StateT<T>; the derivatives and d_t h in T (FP32 in the
// mixed form).
template <int Q, bool DISS, class T>
__device__ __forceinline__ void rhs_dt(const Case& cs, const RhsArgs& A, const double* wk, long sv,
                                       const double* x, double inv_h, typename StateT<T>::type hv[NC], T dh0[NC],
                                       T dh1[NC], T dh2[NC], Coef<typename StateT<T>::type>& C, T dth[NC], T& eh) {
  using H = typename StateT<T>::type;
  const long s1 = 1, s2 = A.Wx, s3 = (long)A.Wx * A.Wd;
  const T ih = T(inv_h);
  eh = T(DISS ? dissipation_rate(cs, A.t, x) * inv_h : 0.0);
#pragma unroll
  for (int v = 0; v < NC; ++v) {
    const double* p = wk + v * sv;
    hv[v] = ld<H>(p);
    dh0[v] = ih * st_d1<Q, T>(p, s1);
    dh1[v] = ih * st_d1<Q, T>(p, s2);
    dh2[v] = ih * st_d1<Q, T>(p, s3);
    // the dissipation stencils read the same rows: sum them here, scale them below
    if (DISS) dth[v] = st_ko<Q, T>(p, s1, T(hv[v])) + st_ko<Q, T>(p, s2, T(hv[v])) + st_ko<Q, T>(p, s3, T(hv[v]));
  }
  metric_quantities(hv, C);
  const T a_div = T(C.alpha / C.sqrtg);
#pragma unroll
  for (int v = 0; v < NC; ++v) {
    const double* p = wk + v * sv;
    T s = T(C.beta[0]) * dh0[v] + T(C.beta[1]) * dh1[v] + T(C.beta[2]) * dh2[v] + a_div * ld<T>(p + NC * sv);
    if (DISS) s = fma(eh, dth[v], s);
    dth[v] = s;
  }
}

// the coefficient set in the right-hand side's arithmetic
template <class T> __device__ __forceinline__ Coef<T> coef_in(const Coef<typename StateT<T>::type>& C) {
  if constexpr (!is_fp32<T>()) {
    return C;
  } else {
    Coef<T> c;
#pragma unroll
    for (int n = 0; n < NC; ++n) {
      c.g[n] = T(C.g[n]);
      c.gu[n] = T(C.gu[n]);
    }
    c.alpha = T(C.alpha);
    c.sqrtg = T(C.sqrtg);
#pragma unroll
    for (int i = 0; i < 3; ++i) c.beta[i] = T(C.beta[i]);
#pragma unroll
    for (int i = 0; i < 6; ++i) c.gamu[i] = T(C.gamu[i]);
    return c;
  }
}

// The coefficients the Pi components read (src/pointwise.jl:754-778), stored at once so
// that the shift, the spatial inverse metric and the divergences are dead before the source.
template <class T>
__device__ __forceinline__ void store_pi_coefficients(const Coef<T>& C, const T* const dh[3], T eh, double* cfo,
                                                      long npts) {
  T divb, divA[3];
  metric_divergences(C, dh, divb, divA);
  const T am = C.alpha * C.sqrtg;
  cfo[CF_B0 * npts] = C.beta[0];
  cfo[CF_B1 * npts] = C.beta[1];
  cfo[CF_B2 * npts] = C.beta[2];
  cfo[CF_DIVB * npts] = divb;
  cfo[CF_DA0 * npts] = divA[0];
  cfo[CF_DA1 * npts] = divA[1];
  cfo[CF_DA2 * npts] = divA[2];
  cfo[CF_AXX * npts] = am * C.gamu[0];
  cfo[CF_AXY * npts] = T(2.0) * am * C.gamu[1];
  cfo[CF_AXZ * npts] = T(2.0) * am * C.gamu[2];
  cfo[CF_AYY * npts] = am * C.gamu[3];
  cfo[CF_AYZ * npts] = T(2.0) * am * C.gamu[4];
  cfo[CF_AZZ * npts] = am * C.gamu[5];
  cfo[CF_EH * npts] = eh;
}

// The matter term (src/pointwise.jl:667-698) of the point, parked in the additive slots of
// the Pi coefficients until the source is added to it.
template <class T>
__device__ __forceinline__ void store_matter(const Coef<T>& C, const RhsArgs& A, int b, long ip, double* cfo) {
  const long S = (long)A.N1 * A.N1 * A.N1;
  const double* q = A.matter + (long)b * 10 * S + ip;
  T m[10], ms[NC];
#pragma unroll
  for (int k = 0; k < 10; ++k) m[k] = ldk<T>(q + k * S);
  matter_source(C, m, ms);
#pragma unroll
  for (int v = 0; v < NC; ++v) cfo[(CF_M0 + v) * A.npts] = value(ms[v]);
}

// Step 3 (src/evolution.jl:286-297): the gauge source (sampled, closed-form Kerr-Schild or
// none) and the reduced source with damping, from D[c] = d_c h (c = t, x, y, z).
template <class T>
__device__ __forceinline__ void rhs_source(const Case& cs, const RhsArgs& A, int b, long ip, T g0, const T hv[NC],
                                           const Coef<T>& C, const T* const D[4], T msrc[NC]) {
  if (cs.gauge == TGH_GAUGE_NONE) {
    gh_source<T, false>(C, D, nullptr, nullptr, g0, T(cs.g2), msrc);
    return;
  }
  T Hl[4], dHs[NC];
  if (cs.gauge == TGH_GAUGE_SAMPLED) {
    // rows: H_a (4), then d_c H_a at 4 + c + 4 a
    const long S = (long)A.N1 * A.N1 * A.N1;
    const double* q = A.Hsrc + (long)b * NV * S + ip;
#pragma unroll
    for (int a = 0; a < 4; ++a) Hl[a] = ldk<T>(q + a * S);
#pragma unroll
    for (int n = 0; n < NC; ++n) {
      const int a = prow(n), c = pcol(n);
      dHs[n] = ldk<T>(q + (4 + a + 4 * c) * S) + ldk<T>(q + (4 + c + 4 * a) * S);
    }
  } else {
    T dHl[4][4];
    ks_gauge_source<T>(cs, hv, D, Hl, dHl);
#pragma unroll
    for (int n = 0; n < NC; ++n) dHs[n] = dHl[prow(n)][pcol(n)] + dHl[pcol(n)][prow(n)];
  }
  gh_source<T, true>(C, D, Hl, dHs, g0, T(cs.g2), msrc);
}

// The interior layer's parts that do not depend on the stencils (src/evolution.jl:600-695): for
// the d_t h half D_v = (1 - w) d_t h_target - rho (h - h_target), for the Pi half
// T_v = (1 - w) d_t Pi_target - rho (Pi - Pi_target); the point's right-hand side is then
// w F + D (resp. w F_Pi + T). A resting interior's target is the analytic state at the point;
// a moving core's (core_follows) adds its rate: d_t g from the dual pass and d_t Pi as the
// centred difference over t +- cbrt(eps) r_0 (src/initialdata.jl:1721-1729). Evaluated by
// interior_kernel ahead of the head kernel and parked in the point's own output slots until the
// stencil part is known.
static __device__ __noinline__ void layer_targets(const Case& cs, double t, const double* x, const double* wk, long sv,
                                           double w, double rho, double* dD, long sD, double* dT, long sT) {
  const double om = 1.0 - w;
  double he[NC], Pe[NC];
  if (core_follows(cs)) {
    double dthe[NC], hx[NC], Pp[NC], Pq[NC];
    rn_background_state(cs, t, x, he, Pe, dthe);
    const double dl = layer_rate_step(cs), tp = t + dl, tm = t - dl;
    rn_background_state(cs, tp, x, hx, Pp);
    rn_background_state(cs, tm, x, hx, Pq);
    for (int v = 0; v < NC; ++v) {
      dD[v * sD] = om * dthe[v] - rho * (wk[v * sv] - he[v]);
      const double dtP = (Pp[v] - Pq[v]) / (tp - tm);
      dT[v * sT] = om * dtP - rho * (wk[(NC + v) * sv] - Pe[v]);
    }
  } else {
    rn_background_state(cs, t, x, he, Pe);
    for (int v = 0; v < NC; ++v) {
      dD[v * sD] = -(rho * (wk[v * sv] - he[v]));
      dT[v * sT] = -(rho * (wk[(NC + v) * sv] - Pe[v]));
    }
  }
}

// The interior's points, ahead of the head kernel (gh_rhs_point!'s branches,
// src/evolution.jl:489-695), over the blocks that can hold a point with r < r_1: a frozen core
// point's whole right-hand side - zero, or with a moving :damped core (core_follows) the
// relaxation of the ADM variables towards the core target and its rate (src/interior.jl:420-459,
// src/initialdata.jl:1784-1796) - and a layer point's target parts D, T (layer_targets), parked
// where the head and Pi kernels will add the stencil part. Kept out of the head kernel so that
// its registers serve the main path alone.
template <int MODE>
__global__ void __launch_bounds__(128) interior_kernel(const Case cs, const RhsArgs A, const int* __restrict__ blocks) {
  const long S = (long)A.N1 * A.N1 * A.N1;
  const long per = (S + blockDim.x - 1) / blockDim.x;
  const int b = blocks[blockIdx.x / per];
  const long ip = (blockIdx.x % per) * blockDim.x + threadIdx.x;
  if (ip >= S) return;
  const long p = (long)b * S + ip;
  if (p < A.p0 || p >= A.p1) return;
  const PointIdx q = point_index(A, p);
  const double r = interior_radius(cs, A.t, q.x);
  if (r >= cs.r1) return;
  const long sv = (long)A.Wx * A.Wd * A.Wd;
  const double* wk = A.work + q.wo;
  double* cfo = A.coef + p;
  EmitDu ed{A.du + (long)q.b * NV * S + q.ip, S};
  EmitStage es{A.acc + (long)q.b * NV * S + q.ip, A.next + q.wo, A.u0 + q.wo, S, sv, A.ca, A.cb, A.stage};
  auto put = [&](int v, double val) {
    if (MODE == MODE_DU) ed.put(v, val);
    else es.put(v, val);
  };
  const bool frozen = cs.interior == TGH_INT_PASTED ? r < cs.r1 : r < cs.r0;
  if (cs.interior == TGH_INT_FITTED) {
    // the :fitted branches (src/evolution.jl:528-548, 619-653): the target A + (t - t_f) S read
    // from the cache at the point (two loads a variable), its rate S fed forward with
    // target_rate; the core relaxes at rho_max, the layer's parts are parked as above
    const double* tw = cs.tw + (long)q.b * (2 * NV) * S + q.ip;
    const double dt = A.t - *cs.tf;
    if (frozen) {
      const double rc = cs.rho_max;
      for (int v = 0; v < NV; ++v) {
        const double sl = tw[(NV + v) * S];
        const double tg = tw[v * S] + dt * sl;
        put(v, cs.trate ? sl - rc * (wk[v * sv] - tg) : -(rc * (wk[v * sv] - tg)));
      }
      return;
    }
    double w, rho;
    layer_profiles(cs, r, w, rho);
    const double om = 1.0 - w;
    double* dD = MODE == MODE_DU ? ed.d : cfo + CF_DTH0 * A.npts;
    double* dT = MODE == MODE_DU ? ed.d + NC * S : es.nx + NC * sv;
    const long sD = MODE == MODE_DU ? S : A.npts, sT = MODE == MODE_DU ? S : sv;
    for (int v = 0; v < NV; ++v) {
      const double sl = tw[(NV + v) * S];
      const double tg = tw[v * S] + dt * sl;
      const double val = cs.trate ? om * sl - rho * (wk[v * sv] - tg) : -(rho * (wk[v * sv] - tg));
      if (v < NC)
        dD[v * sD] = val;
      else
        dT[(v - NC) * sT] = val;
    }
    return;
  }
  if (!frozen) {
    double w, rho;
    layer_profiles(cs, r, w, rho);
    if (MODE == MODE_DU)
      layer_targets(cs, A.t, q.x, wk, sv, w, rho, ed.d, S, ed.d + NC * S, S);
    else
      layer_targets(cs, A.t, q.x, wk, sv, w, rho, cfo + CF_DTH0 * A.npts, A.npts, es.nx + NC * sv, sv);
    return;
  }
  if (!core_follows(cs)) {
    for (int v = 0; v < NV; ++v) put(v, 0.0);
    return;
  }
  const double rc = core_rate(cs), dl = layer_rate_step(cs);
  double xc[3], hd[NC], Pd[NC];
  core_position(cs, A.t, q.x, xc);
  rn_background_state(cs, A.t, xc, hd, Pd);
  double dthd[NC], dtPd[NC];
  const double sw = core_rate_weight(cs, r);
  if (sw == 0.0) {
    for (int n = 0; n < NC; ++n) dthd[n] = dtPd[n] = 0.0;
  } else {
    const double tp = A.t + dl, tm = A.t - dl;
    double xp[3], xm[3], hp[NC], Pp[NC], hm[NC], Pm[NC];
    core_position(cs, tp, q.x, xp);
    core_position(cs, tm, q.x, xm);
    rn_background_state(cs, tp, xp, hp, Pp);
    rn_background_state(cs, tm, xm, hm, Pm);
    const double f = sw / (tp - tm);
    for (int n = 0; n < NC; ++n) {
      dthd[n] = f * (hp[n] - hm[n]);
      dtPd[n] = f * (Pp[n] - Pm[n]);
    }
  }
  double hu[NC], rr[NC];
  for (int v = 0; v < NC; ++v) hu[v] = wk[v * sv];
  core_relaxation_rate(hu, hd, rc, dthd, rr);
  for (int v = 0; v < NC; ++v) {
    put(v, rr[v]);
    put(NC + v, dtPd[v] - rc * (wk[(NC + v) * sv] - Pd[v]));
  }
}

// The head kernel: d_t h at every owned point (emitted in the plain form; in the batched
// form left in the coefficients for the Pi kernel's stage update), the coefficients and
// additive source of the Pi components (stored for the Pi kernel), and - with an interior - the
// branches of gh_rhs_point! (src/evolution.jl:489-695): a frozen core is finished here and
// never reaches a stencil (interior_kernel has written its right-hand side); a layer point
// combines w F - rho (u - u_exact) (+ the moving target's rate), the Pi half as
// w * (stencil part) + coef[CF_M0 + v]. The layer's target parts are parked by interior_kernel,
// until they are added, where the point's own results go later: D in du (plain form) or the
// d_t h coefficient slots (batched form), T in du's Pi half or the next stage's Pi values at the
// point, both written only by the Pi kernel afterwards.
template <int Q, bool DISS, int MODE, bool INT, int N1S, class T>
__global__ void __launch_bounds__(128, is_fp32<T>() ? 3 : 1) rhs_head_kernel(const Case cs, const RhsArgs A0) {
  const RhsArgs A = fixed_geometry<Q, N1S>(A0);
  const long p = A.p0 + (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= A.p1) return;
  const PointIdx q = point_index(A, p);
  const long S = (long)A.N1 * A.N1 * A.N1;
  const long sv = (long)A.Wx * A.Wd * A.Wd;
  const double* wk = A.work + q.wo;
  const double inv_h = 1.0 / q.h;
  double* cfo = A.coef + p;
  EmitDu ed{A.du + (long)q.b * NV * S + q.ip, S};
  EmitStage es{A.acc + (long)q.b * NV * S + q.ip, A.next + q.wo, A.u0 + q.wo, S, sv, A.ca, A.cb, A.stage};
  // d_t h of an evolved point: stored at once in the plain form; in the batched form parked in
  // the coefficients, and the Pi kernel (more warps to cover the loads) does its stage update
  auto put_dth = [&](int v, double val) {
    if (MODE == MODE_DU) ed.put(v, val);
    else cfo[(CF_DTH0 + v) * A.npts] = val;
  };
  double w = 1.0, rho = 0.0, r = 0.0;
  if (INT) {
    // the interior's points were visited first by interior_kernel: a frozen point is finished,
    // a layer point has its target parts parked
    r = interior_radius(cs, A.t, q.x);
    const bool frozen = cs.interior == TGH_INT_PASTED ? r < cs.r1 : r < cs.r0;
    if (frozen) {
      cfo[CF_W * A.npts] = -1.0;
      return;
    }
    if (r < cs.r1) layer_profiles(cs, r, w, rho);
  }
  // d_t h first, emitted at once (in the layer r_0 <= r < r_1 combined with the target)
  double hv[NC];
  T dh0[NC], dh1[NC], dh2[NC], dth[NC], eh;
  Coef<double> C;
  static_assert(sizeof(typename StateT<T>::type) == sizeof(double), "the head kernel's state is FP64");
  rhs_dt<Q, DISS, T>(cs, A, wk, sv, q.x, inv_h, hv, dh0, dh1, dh2, C, dth, eh);
  const bool layer = INT && r < cs.r1;
  if (!layer) {
#pragma unroll
    for (int v = 0; v < NC; ++v) put_dth(v, (double)dth[v]);
  } else {
    // w d_t h + D, D parked at the layer's entry in the slot this value replaces
    const double* dD = MODE == MODE_DU ? ed.d : cfo + CF_DTH0 * A.npts;
    const long sD = MODE == MODE_DU ? S : A.npts;
#pragma unroll
    for (int v = 0; v < NC; ++v) put_dth(v, fma(w, (double)dth[v], dD[v * sD]));
  }
  // the Pi coefficients (and the matter term), then the source, in the form's arithmetic
  const T* dh[3] = {dh0, dh1, dh2};
  const Coef<T> Ct = coef_in<T>(C);
  store_pi_coefficients(Ct, dh, eh, cfo, A.npts);
  if (A.matter) store_matter(Ct, A, q.b, q.ip, cfo);
  T msrc[NC], ht[NC];
#pragma unroll
  for (int v = 0; v < NC; ++v) ht[v] = T(hv[v]);
  const T* D[4] = {dth, dh0, dh1, dh2};
  rhs_source(cs, A, q.b, q.ip, T(damping_rate(cs, A.t, q.x)), ht, Ct, D, msrc);
  if (A.matter) {
#pragma unroll
    for (int v = 0; v < NC; ++v) msrc[v] += T(cfo[(CF_M0 + v) * A.npts]);
  }
  if (!layer) {
#pragma unroll
    for (int v = 0; v < NC; ++v) cfo[(CF_M0 + v) * A.npts] = msrc[v];
    cfo[CF_W * A.npts] = 1.0;
    return;
  }
  // the layer's Pi half: w msrc + T, T = (1 - w) d_t Pi_target - rho (Pi - Pi_target) parked at
  // the layer's entry
  {
    const double* dT = MODE == MODE_DU ? ed.d + NC * S : es.nx + NC * sv;
    const long sT = MODE == MODE_DU ? S : sv;
#pragma unroll
    for (int v = 0; v < NC; ++v) cfo[(CF_M0 + v) * A.npts] = fma(w, (double)msrc[v], dT[v * sT]);
  }
  cfo[CF_W * A.npts] = w;
}

// Step 4 (src/evolution.jl:324-354): per component v the stencils of h_v and Pi_v
// contracted with the head's coefficients, formed, consumed and dropped:
//   beta^i d_i Pi + (d_i beta^i) Pi + d_i A^{ij} d_j h + A^{ij} d_i d_j h + (eps/h) KO(Pi)
// then w * that + coef[CF_M0 + v]. Few registers, so many warps hide the load latency.
template <int Q, bool DISS, int MODE, class T, int N1S, int MB = 4>
__global__ void __launch_bounds__(128, MB) rhs_pi_kernel(const Case cs, const RhsArgs A0) {
  const RhsArgs A = fixed_geometry<Q, N1S>(A0);
  const long p = A.p0 + (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= A.p1) return;
  const double* cfi = A.coef + p;
  const double w = cfi[CF_W * A.npts];
  if (w < 0.0) return;
  const PointIdx q = point_index(A, p);
  const long S = (long)A.N1 * A.N1 * A.N1;
  const long sv = (long)A.Wx * A.Wd * A.Wd;
  const long s1 = 1, s2 = A.Wx, s3 = (long)A.Wx * A.Wd;
  const double* wk = A.work + q.wo;
  const double inv_h = 1.0 / q.h;
  const T ih = T(inv_h), ih2 = T(inv_h * inv_h);
  const T b0 = T(cfi[CF_B0 * A.npts]), b1 = T(cfi[CF_B1 * A.npts]), b2 = T(cfi[CF_B2 * A.npts]);
  const T divb = T(cfi[CF_DIVB * A.npts]);
  const T da0 = T(cfi[CF_DA0 * A.npts]), da1 = T(cfi[CF_DA1 * A.npts]), da2 = T(cfi[CF_DA2 * A.npts]);
  const T Axx = T(cfi[CF_AXX * A.npts]), Axy = T(cfi[CF_AXY * A.npts]), Axz = T(cfi[CF_AXZ * A.npts]);
  const T Ayy = T(cfi[CF_AYY * A.npts]), Ayz = T(cfi[CF_AYZ * A.npts]), Azz = T(cfi[CF_AZZ * A.npts]);
  const T eh = T(cfi[CF_EH * A.npts]);
  EmitDu ed{A.du + (long)q.b * NV * S + q.ip, S};
  EmitStage es{A.acc + (long)q.b * NV * S + q.ip, A.next + q.wo, A.u0 + q.wo, S, sv, A.ca, A.cb, A.stage};
#pragma unroll 1
  for (int v = 0; v < NC; ++v) {
    // the epilogue's loads first: they are in flight while the stencils are formed
    const double m = cfi[(CF_M0 + v) * A.npts];
    double kh = 0.0, uh = 0.0, up = 0.0, ah = 0.0, ap = 0.0;
    if (MODE == MODE_STAGE) {
      kh = cfi[(CF_DTH0 + v) * A.npts];
      uh = es.pre_u(v);
      up = es.pre_u(NC + v);
      ah = es.pre_a(v);
      ap = es.pre_a(NC + v);
    }
    const double* ph = wk + v * sv;
    const double* pp = ph + NC * sv;
    const T hc = ld<T>(ph), pc = ld<T>(pp);
    T s = b0 * (ih * st_d1<Q, T>(pp, s1));
    s = fma(b1, ih * st_d1<Q, T>(pp, s2), s);
    s = fma(b2, ih * st_d1<Q, T>(pp, s3), s);
    s = fma(divb, pc, s);
    s = fma(da0, ih * st_d1<Q, T>(ph, s1), s);
    s = fma(da1, ih * st_d1<Q, T>(ph, s2), s);
    s = fma(da2, ih * st_d1<Q, T>(ph, s3), s);
    T p2 = Axx * st_d2<Q, T>(ph, s1, hc);
    p2 = fma(Ayy, st_d2<Q, T>(ph, s2, hc), p2);
    p2 = fma(Azz, st_d2<Q, T>(ph, s3, hc), p2);
    p2 = fma(Axy, st_mixed<Q, T>(ph, s1, s2), p2);
    p2 = fma(Axz, st_mixed<Q, T>(ph, s1, s3), p2);
    p2 = fma(Ayz, st_mixed<Q, T>(ph, s2, s3), p2);
    s = fma(ih2, p2, s);
    if (DISS) s = fma(eh, st_ko<Q, T>(pp, s1, pc) + st_ko<Q, T>(pp, s2, pc) + st_ko<Q, T>(pp, s3, pc), s);
    const double val = w == 1.0 ? (double)s + m : fma(w, (double)s, m);
    if (MODE == MODE_DU) {
      ed.put(NC + v, val);
    } else {
      es.fin(v, kh, uh, ah);
      es.fin(NC + v, val, up, ap);
    }
  }
}

}  // namespace tgh
