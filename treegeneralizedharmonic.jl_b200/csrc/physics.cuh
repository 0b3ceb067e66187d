// Device-side physics of the generalized-harmonic path: the analytic backgrounds with
// forward-mode derivatives, the Kerr-Schild gauge source, the damping / dissipation
// profiles and the sphere interior. Everything here is evaluated per point inside the
// kernels (Dirichlet ghosts, the layer target, the sampled gauge source at set-up).
//
// Reference behaviour followed (the analytic state itself, background_state, which the
// centred-difference rates of src/initialdata.jl:1721-1796 are built on, is in analytic.cuh):
//   KerrSchildSource            src/gauge.jl:257-336
//   gauge_tuple / gauge_at      src/gauge.jl:156-212  (H_b, then d_a H_b column-major)
//   Constant/GaussianDamping    src/gauge.jl:1094-1147
//   HorizonDissipation          src/gauge.jl:1180-1266
//   Interior, smoothstep, ...   src/interior.jl:117-625
// The metrics themselves come from SpacetimeMetrics in the reference (not vendored);
// their closed forms are listed in include/tgh.h.
#pragma once
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/tgh.h"

#define TGH_HD __host__ __device__ __forceinline__

// one rounded operation each, never contracted into a fused multiply-add (the interior's
// placement and profiles and the analytic state are evaluated this way, in the reference's
// order, so that they agree with a CPU evaluation bit for bit)
#ifdef __CUDA_ARCH__
#define TGH_RADD(a, b) __dadd_rn(a, b)
#define TGH_RSUB(a, b) __dsub_rn(a, b)
#define TGH_RMUL(a, b) __dmul_rn(a, b)
#define TGH_RDIV(a, b) __ddiv_rn(a, b)
#define TGH_RSQRT(a) __dsqrt_rn(a)
#else
#define TGH_RADD(a, b) ((a) + (b))
#define TGH_RSUB(a, b) ((a) - (b))
#define TGH_RMUL(a, b) ((a) * (b))
#define TGH_RDIV(a, b) ((a) / (b))
#define TGH_RSQRT(a) std::sqrt(a)
#endif

namespace tgh {

constexpr int NC = 10;
constexpr int NV = 20;

// packed slot of the symmetric pair (a, b), 0-based, column-major lower triangle
TGH_HD constexpr int pidx(int a, int b) {
  return (a > b ? b : a) * 4 - ((a > b ? b : a) * ((a > b ? b : a) - 1)) / 2 + ((a > b ? a : b) - (a > b ? b : a));
}
TGH_HD constexpr int prow(int n) { return n < 4 ? n : n < 7 ? n - 3 : n < 9 ? n - 5 : 3; }
TGH_HD constexpr int pcol(int n) { return n < 4 ? 0 : n < 7 ? 1 : n < 9 ? 2 : 3; }
TGH_HD constexpr double etad(int a) { return a == 0 ? -1.0 : 1.0; }

// ---------------------------------------------------------------------------------
// Forward-mode numbers with four partials (t, x, y, z). Nested once (Dn<Dn<double>>)
// they give the second derivatives the sampled gauge source needs.
template <class T> struct Dn {
  T v, d[4];
  TGH_HD Dn() {}
  TGH_HD Dn(double c) : v(c) {
#pragma unroll
    for (int i = 0; i < 4; ++i) d[i] = T(0.0);
  }
};
template <class T> TGH_HD Dn<T> dconst(const T& c) {
  Dn<T> r;
  r.v = c;
  r.d[0] = r.d[1] = r.d[2] = r.d[3] = T(0.0);
  return r;
}
template <class T> TGH_HD Dn<T> operator+(const Dn<T>& a, const Dn<T>& b) {
  Dn<T> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
template <class T> TGH_HD Dn<T> operator-(const Dn<T>& a, const Dn<T>& b) {
  Dn<T> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
template <class T> TGH_HD Dn<T> operator-(const Dn<T>& a) {
  Dn<T> r;
  r.v = -a.v;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = -a.d[i];
  return r;
}
template <class T> TGH_HD Dn<T> operator*(const Dn<T>& a, const Dn<T>& b) {
  Dn<T> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
template <class T> TGH_HD Dn<T> operator*(double s, const Dn<T>& a) {
  Dn<T> r;
  r.v = s * a.v;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = s * a.d[i];
  return r;
}
template <class T> TGH_HD Dn<T> operator/(const Dn<T>& a, const Dn<T>& b) {
  Dn<T> r;
  T ib = T(1.0) / b.v;
  r.v = a.v * ib;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
  return r;
}
template <class T> TGH_HD Dn<T> fchain(const Dn<T>& a, const T& f, const T& df) {
  Dn<T> r;
  r.v = f;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = df * a.d[i];
  return r;
}
TGH_HD double dsqrt(double a) { return sqrt(a); }
TGH_HD double dsin(double a) { return sin(a); }
TGH_HD double dcos(double a) { return cos(a); }
TGH_HD double dtanh(double a) { return tanh(a); }
template <class T> TGH_HD Dn<T> dsqrt(const Dn<T>& a) {
  T s = dsqrt(a.v);
  return fchain(a, s, T(0.5) / s);
}
template <class T> TGH_HD Dn<T> dsin(const Dn<T>& a) { return fchain(a, dsin(a.v), dcos(a.v)); }
template <class T> TGH_HD Dn<T> dcos(const Dn<T>& a) { return fchain(a, dcos(a.v), -dsin(a.v)); }
template <class T> TGH_HD Dn<T> dtanh(const Dn<T>& a) {
  T th = dtanh(a.v);
  return fchain(a, th, T(1.0) - th * th);
}
template <class T> TGH_HD T cst(double c) { return T(c); }
template <> TGH_HD Dn<double> cst<Dn<double>>(double c) { return dconst(c); }
template <> TGH_HD Dn<Dn<double>> cst<Dn<Dn<double>>>(double c) { return dconst(dconst(c)); }

// ---------------------------------------------------------------------------------
// The run's constants, passed by value to every kernel that evaluates physics.
struct Case {
  tgh_background bg;
  double L[4][4];       // boost matrix (identity when there is none)
  int boosted;
  int gauge;
  double ksM, ksS[4], ksU[4];
  int damping;
  double g0, dnear, dfar, dwidth, dc0[3], dv[3];
  double g2;
  int dissipation;
  double eps, eout, ein, er1, erh, ec0[3], ev[3];
  int interior;
  double ic0[3], iv[3], r0, r1, rho_max, w_ramp, rho_ramp;
  // :fitted: the target cache (per block 40 fields of the owned points: the target A, the packed
  // (h, Pi), then its slope S), the fill time t_f (one double in device memory, so that a captured
  // step graph reads the current one) and whether the target's rate is fed forward
  const double* tw;
  const double* tf;
  int trate;
};

// g_ab at a spacetime point x = (t, x, y, z), in any scalar type S
template <class S> TGH_HD void kerr_schild_rest(double M, double a, const S* x, S g[4][4]) {
  S X = x[1], Y = x[2], Z = x[3];
  S a2 = cst<S>(a * a);
  S half = 0.5 * (X * X + Y * Y + Z * Z - a2);
  S r2 = half + dsqrt(half * half + a2 * Z * Z);
  S r = dsqrt(r2);
  S H = cst<S>(M) * r * r2 / (r2 * r2 + a2 * Z * Z);
  S den = r2 + a2;
  S l[4];
  l[0] = cst<S>(1.0);
  l[1] = (r * X + cst<S>(a) * Y) / den;
  l[2] = (r * Y - cst<S>(a) * X) / den;
  l[3] = Z / r;
  S H2 = 2.0 * H;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    S hl = H2 * l[i];
#pragma unroll
    for (int j = 0; j < 4; ++j) g[i][j] = cst<S>(i == j ? etad(i) : 0.0) + hl * l[j];
  }
}

template <class S> TGH_HD void ks_rest(double M, double a, const S* x, S g[4][4]) { kerr_schild_rest(M, a, x, g); }

// Kerr (M, a) in horizon-penetrating harmonic coordinates in its rest frame (t = x[0]; the
// metric does not depend on t): the Kerr-Schild metric pulled back, g = J^T g_KS J, along
//   X + i Y = w (x + i y),  Z = (r / r_H) z,  T = t + 2 M ln(r_H + sqrt(M^2 - a^2)),
//   w = (r + i a) / (r_H + i a),  r = r_H + M,
// r_H the spheroidal radius of (x, y, z) with parameter a (the Kerr-Schild quartic). Both charts
// share the Kerr-Schild angle; the harmonic radius is the Boyer-Lindquist radius minus M, and the
// harmonic time t_BL + 2 M r_+ int dr / Delta is regular on the future horizon. J comes in closed
// form from d r_H / d x^i = r_H (x_i r_H^2 + a^2 z delta_iz) / (r_H^4 + a^2 z^2), so the metric's
// derivatives come from S's own (forward-mode numbers). Every coordinate function is harmonic
// (H_a = 0); at a = 0 this is the harmonic Schwarzschild metric g_tt = -(r - M)/(r + M),
// g_tr = 4 M^2 / (r + M)^2. The operations are the oracle's, one by one (with a rounded S the
// result is the oracle's bit for bit).
template <class S> TGH_HD void harmonic_kerr_rest(double M, double a, const S* x, S g[4][4]) {
  const S X = x[1], Y = x[2], Z = x[3];
  const S rho2 = X * X + Y * Y + Z * Z;
  const S a2 = cst<S>(TGH_RMUL(a, a));
  const S half = cst<S>(0.5) * (rho2 - a2);
  const S r2 = half + dsqrt(half * half + a2 * Z * Z);
  const S rh = dsqrt(r2);
  const S q = r2 * r2 + a2 * Z * Z;
  const S dr[3] = {rh * (X * r2) / q, rh * (Y * r2) / q, rh * (Z * r2 + a2 * Z) / q};
  const S r = rh + cst<S>(M);
  const S D = r2 + a2;
  const S wr = (r * rh + a2) / D;
  const S wi = cst<S>(-TGH_RMUL(a, M)) / D;
  const S D2 = D * D;
  const S dwr = cst<S>(-M) * (r2 - a2) / D2;
  const S dwi = cst<S>(TGH_RMUL(TGH_RMUL(2.0, M), a)) * rh / D2;
  const S px = X * dwr - Y * dwi;
  const S py = X * dwi + Y * dwr;
  const S zr = r / rh;
  const S zd = cst<S>(-M) * Z / r2;
  const S tr = cst<S>(TGH_RMUL(2.0, M)) / (rh + cst<S>(TGH_RSQRT(TGH_RSUB(TGH_RMUL(M, M), TGH_RMUL(a, a)))));
  const S xk[4] = {x[0], wr * X - wi * Y, wr * Y + wi * X, zr * Z};
  S J[4][4];
  J[0][0] = cst<S>(1.0);
  J[1][0] = J[2][0] = J[3][0] = cst<S>(0.0);
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    J[0][j + 1] = tr * dr[j];
    J[1][j + 1] = px * dr[j];
    J[2][j + 1] = py * dr[j];
    J[3][j + 1] = zd * dr[j];
  }
  J[1][1] = wr + J[1][1];
  J[1][2] = J[1][2] - wi;
  J[2][1] = wi + J[2][1];
  J[2][2] = wr + J[2][2];
  J[3][3] = zr + J[3][3];
  S gk[4][4];
  ks_rest(M, a, xk, gk);
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      S acc = cst<S>(0.0);
#pragma unroll
      for (int A = 0; A < 4; ++A) {
        S t = J[0][s] * gk[A][0];
#pragma unroll
        for (int B = 1; B < 4; ++B) t = t + J[B][s] * gk[A][B];
        acc = acc + J[A][p] * t;
      }
      g[p][s] = acc;
    }
}

template <class S> TGH_HD void hole_rest(const Case& c, const S* x, S g[4][4]) {
  if (c.bg.kind == TGH_BG_HARMONIC_KERR)
    harmonic_kerr_rest(c.bg.M, c.bg.a, x, g);
  else
    kerr_schild_rest(c.bg.M, c.bg.a, x, g);
}

template <class S> TGH_HD void metric(const Case& c, const S* xin, S g[4][4]) {
  S x[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) x[i] = xin[i] - cst<S>(c.bg.translate[i]);
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) g[i][j] = cst<S>(i == j ? etad(i) : 0.0);
  if (c.bg.kind == TGH_BG_GAUGE_WAVE) {
    S H = cst<S>(1.0) - cst<S>(c.bg.A) * dsin(cst<S>(2.0 * M_PI / c.bg.d) * (x[1] - x[0]));
    g[0][0] = -H;
    g[1][1] = H;
  } else if (c.bg.kind == TGH_BG_SHIFTED_MINKOWSKI) {
    S th = dtanh(x[1] / cst<S>(c.bg.d));
    S psi = cst<S>(c.bg.A) * (cst<S>(1.0) - th * th);
    g[0][1] = -psi;
    g[1][0] = -psi;
    g[1][1] = cst<S>(1.0) - psi * psi;
  } else if (c.bg.kind == TGH_BG_KERR_SCHILD || c.bg.kind == TGH_BG_HARMONIC_KERR) {
    if (!c.boosted) {
      hole_rest(c, x, g);
    } else {
      S xr[4], gr[4][4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
        xr[i] = cst<S>(c.L[i][0]) * x[0] + cst<S>(c.L[i][1]) * x[1] + cst<S>(c.L[i][2]) * x[2] +
                cst<S>(c.L[i][3]) * x[3];
      hole_rest(c, xr, gr);
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          S s = cst<S>(0.0);
#pragma unroll
          for (int p = 0; p < 4; ++p) {
            S t = c.L[0][b] * gr[p][0] + c.L[1][b] * gr[p][1];
            t = t + c.L[2][b] * gr[p][2] + c.L[3][b] * gr[p][3];
            s = s + c.L[p][a] * t;
          }
          g[a][b] = s;
        }
    }
  }
}

// ---- metric_quantities (restated for the device; src/pointwise.jl:145-184) ----
template <class T> struct Coef {
  T g[NC], gu[NC];  // packed g_ab and g^ab
  T alpha, beta[3], gamu[6], sqrtg;  // gamu packed (xx, xy, xz, yy, yz, zz)
};
TGH_HD constexpr int sidx3(int i, int j) {
  return (i > j ? j : i) * 3 - ((i > j ? j : i) * ((i > j ? j : i) - 1)) / 2 + ((i > j ? i : j) - (i > j ? j : i));
}

template <class T> TGH_HD T det3v(T a, T b, T c, T d, T e, T f, T g, T h, T i) {
  return a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
}

// inverse of the symmetric 4x4 g = eta + h and the offset identities for alpha, sqrt(gamma)
template <class T> TGH_HD void metric_quantities(const T* h, Coef<T>& C) {
  T m[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) m[a][b] = h[pidx(a, b)] + T(a == b ? etad(a) : 0.0);
#pragma unroll
  for (int n = 0; n < NC; ++n) C.g[n] = m[prow(n)][pcol(n)];
  // cofactors of the symmetric matrix (10 unique)
  T cof[NC];
#pragma unroll
  for (int n = 0; n < NC; ++n) {
    const int i = prow(n), j = pcol(n);
    int r[3], c[3], kr = 0, kc = 0;
#pragma unroll
    for (int ii = 0; ii < 4; ++ii)
      if (ii != i) r[kr++] = ii;
#pragma unroll
    for (int jj = 0; jj < 4; ++jj)
      if (jj != j) c[kc++] = jj;
    T mi = det3v(m[r[0]][c[0]], m[r[0]][c[1]], m[r[0]][c[2]], m[r[1]][c[0]], m[r[1]][c[1]], m[r[1]][c[2]],
                 m[r[2]][c[0]], m[r[2]][c[1]], m[r[2]][c[2]]);
    cof[n] = ((i + j) % 2 == 0) ? mi : -mi;
  }
  T det = m[0][0] * cof[0] + m[0][1] * cof[1] + m[0][2] * cof[2] + m[0][3] * cof[3];
  T idet = T(1.0) / det;
  T gi[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) gi[a][b] = cof[pidx(a, b)] * idet;
  // g^ab - eta^ab = -(g^-1 h) eta : full relative precision of the offset
  T guo00 = T(0.0);
#pragma unroll
  for (int n = 0; n < NC; ++n) {
    const int a = prow(n), b = pcol(n);
    T s = gi[a][0] * h[pidx(0, b)];
#pragma unroll
    for (int k = 1; k < 4; ++k) s = s + gi[a][k] * h[pidx(k, b)];
    T o = b == 0 ? s : -s;
    if (n == 0) guo00 = o;
    C.gu[n] = o + T(a == b ? etad(a) : 0.0);
  }
  const T gutt = C.gu[0];
  C.alpha = T(1.0) / dsqrt(T(1.0) - guo00);
  const T igutt = T(1.0) / gutt;
#pragma unroll
  for (int i = 0; i < 3; ++i) C.beta[i] = -C.gu[pidx(0, i + 1)] * igutt;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = i; j < 3; ++j)
      C.gamu[sidx3(i, j)] = C.gu[pidx(i + 1, j + 1)] - C.gu[pidx(0, i + 1)] * C.gu[pidx(0, j + 1)] * igutt;
  // det(g) + 1 from the elementary symmetric polynomials of B = eta h
  T B[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) B[a][b] = a == 0 ? -h[pidx(a, b)] : h[pidx(a, b)];
  T trB = B[0][0] + B[1][1] + B[2][2] + B[3][3];
  T trB2 = T(0.0), trB3 = T(0.0);
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      trB2 = trB2 + B[a][b] * B[b][a];
      T s = B[b][0] * B[0][a] + B[b][1] * B[1][a] + B[b][2] * B[2][a] + B[b][3] * B[3][a];
      trB3 = trB3 + B[a][b] * s;
    }
  // det(B) by 2x2 minors
  T s0 = B[0][0] * B[1][1] - B[1][0] * B[0][1];
  T s1 = B[0][0] * B[1][2] - B[1][0] * B[0][2];
  T s2 = B[0][0] * B[1][3] - B[1][0] * B[0][3];
  T s3 = B[0][1] * B[1][2] - B[1][1] * B[0][2];
  T s4 = B[0][1] * B[1][3] - B[1][1] * B[0][3];
  T s5 = B[0][2] * B[1][3] - B[1][2] * B[0][3];
  T c5 = B[2][2] * B[3][3] - B[3][2] * B[2][3];
  T c4 = B[2][1] * B[3][3] - B[3][1] * B[2][3];
  T c3 = B[2][1] * B[3][2] - B[3][1] * B[2][2];
  T c2 = B[2][0] * B[3][3] - B[3][0] * B[2][3];
  T c1 = B[2][0] * B[3][2] - B[3][0] * B[2][2];
  T c0 = B[2][0] * B[3][1] - B[3][0] * B[2][1];
  T e4 = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
  T e2 = (trB * trB - trB2) * T(0.5);
  T e3 = (trB * trB * trB - T(3.0) * trB * trB2 + T(2.0) * trB3) * T(1.0 / 6.0);
  T d1 = -(trB + e2 + e3 + e4);
  T detgm1 = -d1 - guo00 + d1 * guo00;
  C.sqrtg = dsqrt(T(1.0) + detgm1);
}

// H_b = -g^{cd} Gamma_{b,cd} of the background and d_a H_b, by nested forward-mode numbers;
// out[0..3] = H_b, out[4 + a + 4 b] = d_a H_b (the sampled field's 20 values)
TGH_HD void gauge_tuple(const Case& c, double t, const double* x, double* out) {
  typedef Dn<double> D1;
  typedef Dn<D1> D2;
  D2 p[4];
  const double pv[4] = {t, x[0], x[1], x[2]};
  for (int i = 0; i < 4; ++i) {
    p[i] = cst<D2>(pv[i]);
    p[i].v.d[i] = 1.0;
    p[i].d[i] = dconst(1.0);
  }
  D2 g2[4][4];
  metric(c, p, g2);
  // the inverse metric with its first derivatives: cofactors of the symmetric matrix, each
  // index a compile-time constant (fully unrolled)
  D1 cof[NC];
#pragma unroll
  for (int n = 0; n < NC; ++n) {
    const int i = prow(n), j = pcol(n);
    const int r0 = i == 0 ? 1 : 0, r1 = i <= 1 ? 2 : 1, r2 = i <= 2 ? 3 : 2;
    const int c0 = j == 0 ? 1 : 0, c1 = j <= 1 ? 2 : 1, c2 = j <= 2 ? 3 : 2;
    D1 mi = det3v(g2[r0][c0].v, g2[r0][c1].v, g2[r0][c2].v, g2[r1][c0].v, g2[r1][c1].v, g2[r1][c2].v,
                  g2[r2][c0].v, g2[r2][c1].v, g2[r2][c2].v);
    cof[n] = ((i + j) % 2 == 0) ? mi : -mi;
  }
  const D1 det = g2[0][0].v * cof[pidx(0, 0)] + g2[0][1].v * cof[pidx(0, 1)] + g2[0][2].v * cof[pidx(0, 2)] +
                 g2[0][3].v * cof[pidx(0, 3)];
  const D1 idet = D1(1.0) / det;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    D1 s = dconst(0.0);
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int d = 0; d < 4; ++d) {
        // Gamma_{a,kd} = (d_k g_ad + d_d g_ak - d_a g_kd) / 2, with d_k g_ab = g2[a][b].d[k]
        const D1 low = 0.5 * (g2[a][d].d[k] + g2[a][k].d[d] - g2[k][d].d[a]);
        s = s + (cof[pidx(d, k)] * idet) * low;
      }
    out[a] = -s.v;
#pragma unroll
    for (int k = 0; k < 4; ++k) out[4 + k + 4 * a] = -s.d[k];
  }
}

// the closed-form Kerr-Schild gauge source: Hl[a], dHl[c][a] = d_c H_a
// (src/gauge.jl:302-336); D[c] are the packed d_c h (c = t, x, y, z)
template <class T>
TGH_HD void ks_gauge_source(const Case& c, const T* h, const T* const D[4], T Hl[4], T dHl[4][4]) {
  T w[4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
    w[a] = h[pidx(a, 0)] * T(c.ksU[0]) + h[pidx(a, 1)] * T(c.ksU[1]) + h[pidx(a, 2)] * T(c.ksU[2]) +
           h[pidx(a, 3)] * T(c.ksU[3]);
  T K = T(c.ksU[0]) * w[0] + T(c.ksU[1]) * w[1] + T(c.ksU[2]) * w[2] + T(c.ksU[3]) * w[3];
  T sw = T(c.ksS[0]) * w[0] + T(c.ksS[1]) * w[1] + T(c.ksS[2]) * w[2] + T(c.ksS[3]) * w[3];
  T rad = T(c.ksM * c.ksM) - sw * sw;
  T root = rad > T(0.0) ? sqrt(rad) : T(0.0);
  T Dd = T(c.ksM) + root;
  T iD = T(1.0) / Dd;
#pragma unroll
  for (int a = 0; a < 4; ++a) Hl[a] = -K * iD * w[a];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    T dw[4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
      dw[a] = D[k][pidx(a, 0)] * T(c.ksU[0]) + D[k][pidx(a, 1)] * T(c.ksU[1]) + D[k][pidx(a, 2)] * T(c.ksU[2]) +
              D[k][pidx(a, 3)] * T(c.ksU[3]);
    T dK = T(c.ksU[0]) * dw[0] + T(c.ksU[1]) * dw[1] + T(c.ksU[2]) * dw[2] + T(c.ksU[3]) * dw[3];
    T Sdw = T(c.ksS[0]) * dw[0] + T(c.ksS[1]) * dw[1] + T(c.ksS[2]) * dw[2] + T(c.ksS[3]) * dw[3];
    T dD = root > T(0.0) ? -sw * Sdw / root : T(0.0);
#pragma unroll
    for (int a = 0; a < 4; ++a) dHl[k][a] = -(dK * w[a] + K * dw[a]) * iD + K * w[a] * dD * iD * iD;
  }
}

// ---- profiles (each operation rounded on its own, in the reference's order) ----
// src/interior.jl:117-120
TGH_HD double smoothstep(double s) {
  const double u = s < 0.0 ? 0.0 : (s > 1.0 ? 1.0 : s);
  const double uuu = TGH_RMUL(TGH_RMUL(u, u), u);
  const double p = TGH_RMUL(uuu, TGH_RADD(10.0, TGH_RMUL(u, TGH_RSUB(TGH_RMUL(6.0, u), 15.0))));
  return p < 0.0 ? 0.0 : (p > 1.0 ? 1.0 : p);
}
// |x - (c0 + t v)|
TGH_HD double moving_distance(const double c0[3], const double v[3], double t, const double* x) {
  double d[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) d[i] = TGH_RSUB(x[i], TGH_RADD(c0[i], TGH_RMUL(t, v[i])));
  return TGH_RSQRT(TGH_RADD(TGH_RADD(TGH_RMUL(d[0], d[0]), TGH_RMUL(d[1], d[1])), TGH_RMUL(d[2], d[2])));
}
TGH_HD double damping_rate(const Case& c, double t, const double* x) {
  if (c.damping == TGH_DAMP_CONSTANT) return c.g0;
  double d[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) d[i] = TGH_RSUB(x[i], TGH_RADD(c.dc0[i], TGH_RMUL(t, c.dv[i])));
  const double r2 = TGH_RADD(TGH_RADD(TGH_RMUL(d[0], d[0]), TGH_RMUL(d[1], d[1])), TGH_RMUL(d[2], d[2]));
  const double e = exp(TGH_RDIV(-r2, TGH_RMUL(TGH_RMUL(2.0, c.dwidth), c.dwidth)));
  return TGH_RADD(c.dfar, TGH_RMUL(TGH_RSUB(c.dnear, c.dfar), e));
}
TGH_HD double dissipation_rate(const Case& c, double t, const double* x) {
  if (c.dissipation == TGH_DISS_CONSTANT) return c.eps;
  const double r = moving_distance(c.ec0, c.ev, t, x);
  if (r >= c.erh) return c.eout;
  if (r <= c.er1) return c.ein;
  const double s = TGH_RDIV(TGH_RSUB(c.erh, r), TGH_RSUB(c.erh, c.er1));
  return TGH_RADD(c.eout, TGH_RMUL(TGH_RSUB(c.ein, c.eout), smoothstep(s)));
}
// the distance from the interior's centre c0 + t v (HoleCenter, src/interior.jl:75-93)
TGH_HD double interior_radius(const Case& c, double t, const double* x) {
  return moving_distance(c.ic0, c.iv, t, x);
}
// is_evolved(mask, x) of the interior's mask: r >= r_1 (src/constraints.jl:74-75)
TGH_HD bool evolved(const Case& cs, double t, const double* x) {
  return cs.interior == TGH_INT_NONE ? true : interior_radius(cs, t, x) >= cs.r1;
}
TGH_HD bool core_follows(const Case& c) {
  return c.interior == TGH_INT_DAMPED && !(c.iv[0] == 0.0 && c.iv[1] == 0.0 && c.iv[2] == 0.0);
}
// core_position (src/interior.jl:615-625): a point of the core is placed on the sphere r_0
// along its direction from the centre (straight up at the centre itself)
TGH_HD void core_position(const Case& c, double t, const double* x, double* out) {
  if (c.interior == TGH_INT_NONE) {
    out[0] = x[0]; out[1] = x[1]; out[2] = x[2];
    return;
  }
  double cc[3], d[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    cc[i] = TGH_RADD(c.ic0[i], TGH_RMUL(t, c.iv[i]));
    d[i] = TGH_RSUB(x[i], cc[i]);
  }
  const double r = TGH_RSQRT(TGH_RADD(TGH_RADD(TGH_RMUL(d[0], d[0]), TGH_RMUL(d[1], d[1])), TGH_RMUL(d[2], d[2])));
  if (r >= c.r0) {
    out[0] = x[0]; out[1] = x[1]; out[2] = x[2];
    return;
  }
  double n[3] = {0.0, 0.0, 1.0};
  if (r != 0.0) {
#pragma unroll
    for (int i = 0; i < 3; ++i) n[i] = TGH_RDIV(d[i], r);
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) out[i] = TGH_RADD(cc[i], TGH_RMUL(c.r0, n[i]));
}
// _layer_profiles (src/interior.jl:567-590): the switch-on w and the relaxation rate rho
TGH_HD void layer_profiles(const Case& c, double r, double& w, double& rho) {
  const double s = TGH_RDIV(TGH_RSUB(r, c.r0), TGH_RSUB(c.r1, c.r0));
  w = smoothstep(TGH_RDIV(s, c.w_ramp));
  rho = c.interior == TGH_INT_FROZEN ? 0.0 : TGH_RMUL(c.rho_max, smoothstep(TGH_RDIV(TGH_RSUB(1.0, s), c.rho_ramp)));
}
TGH_HD double core_rate(const Case& c) {
  const double s = TGH_RSQRT(TGH_RADD(TGH_RADD(TGH_RMUL(c.iv[0], c.iv[0]), TGH_RMUL(c.iv[1], c.iv[1])),
                                      TGH_RMUL(c.iv[2], c.iv[2])));
  const double k = TGH_RDIV(TGH_RMUL(12.0, s), c.r0);
  return c.rho_max > k ? c.rho_max : k;
}
// core_rate_weight (src/interior.jl:560-565): smoothstep(4 r / r_0 - 1)
TGH_HD double core_rate_weight(const Case& c, double r) {
  return smoothstep(TGH_RSUB(TGH_RDIV(TGH_RMUL(4.0, r), c.r0), 1.0));
}
// cbrt(eps) r_0 with eps the double epsilon (src/interior.jl:545)
TGH_HD double layer_rate_step(const Case& c) { return 6.0554544523933395e-06 * c.r0; }

TGH_HD void inv3sym(const double g[3][3], double o[3][3]) {
  double c00 = g[1][1] * g[2][2] - g[1][2] * g[2][1];
  double c01 = g[1][2] * g[2][0] - g[1][0] * g[2][2];
  double c02 = g[1][0] * g[2][1] - g[1][1] * g[2][0];
  double det = g[0][0] * c00 + g[0][1] * c01 + g[0][2] * c02;
  double id = 1.0 / det;
  o[0][0] = c00 * id; o[1][0] = c01 * id; o[2][0] = c02 * id;
  o[0][1] = (g[0][2] * g[2][1] - g[0][1] * g[2][2]) * id;
  o[1][1] = (g[0][0] * g[2][2] - g[0][2] * g[2][0]) * id;
  o[2][1] = (g[0][1] * g[2][0] - g[0][0] * g[2][1]) * id;
  o[0][2] = (g[0][1] * g[1][2] - g[0][2] * g[1][1]) * id;
  o[1][2] = (g[0][2] * g[1][0] - g[0][0] * g[1][2]) * id;
  o[2][2] = (g[0][0] * g[1][1] - g[0][1] * g[1][0]) * id;
}
TGH_HD void adm_split(const double* h, double& A, double bu[3], double bl[3], double g[3][3]) {
  g[0][0] = 1.0 + h[4]; g[0][1] = h[5]; g[0][2] = h[6];
  g[1][0] = h[5]; g[1][1] = 1.0 + h[7]; g[1][2] = h[8];
  g[2][0] = h[6]; g[2][1] = h[8]; g[2][2] = 1.0 + h[9];
  bl[0] = h[1]; bl[1] = h[2]; bl[2] = h[3];
  double gi[3][3];
  inv3sym(g, gi);
  for (int i = 0; i < 3; ++i) bu[i] = gi[i][0] * bl[0] + gi[i][1] * bl[1] + gi[i][2] * bl[2];
  A = (1.0 - h[0]) + (bu[0] * bl[0] + bu[1] * bl[1] + bu[2] * bl[2]);
}
// the moving core's rate in the ADM variables (src/interior.jl:420-459)
TGH_HD void core_relaxation_rate(const double* h, const double* ht, double rho, const double* dtht, double* out) {
  double A, bu[3], bl[3], g[3][3], At, but[3], blt[3], gt[3][3];
  adm_split(h, A, bu, bl, g);
  adm_split(ht, At, but, blt, gt);
  double dgt[3][3] = {{dtht[4], dtht[5], dtht[6]}, {dtht[5], dtht[7], dtht[8]}, {dtht[6], dtht[8], dtht[9]}};
  double gti[3][3];
  inv3sym(gt, gti);
  double dgtb[3], rhs3[3], dbt[3];
  for (int i = 0; i < 3; ++i) dgtb[i] = dgt[i][0] * but[0] + dgt[i][1] * but[1] + dgt[i][2] * but[2];
  for (int i = 0; i < 3; ++i) rhs3[i] = dtht[1 + i] - dgtb[i];
  for (int i = 0; i < 3; ++i) dbt[i] = gti[i][0] * rhs3[0] + gti[i][1] * rhs3[1] + gti[i][2] * rhs3[2];
  double dAt = -dtht[0] + (but[0] * dgtb[0] + but[1] * dgtb[1] + but[2] * dgtb[2]) +
               2.0 * (blt[0] * dbt[0] + blt[1] * dbt[1] + blt[2] * dbt[2]);
  double dA = dAt - rho * (A - At);
  double db[3];
  for (int i = 0; i < 3; ++i) db[i] = dbt[i] - rho * (bu[i] - but[i]);
  double e[6] = {h[4] - ht[4], h[5] - ht[5], h[6] - ht[6], h[7] - ht[7], h[8] - ht[8], h[9] - ht[9]};
  double dg[3][3] = {{dgt[0][0] - rho * e[0], dgt[0][1] - rho * e[1], dgt[0][2] - rho * e[2]},
                     {dgt[1][0] - rho * e[1], dgt[1][1] - rho * e[3], dgt[1][2] - rho * e[4]},
                     {dgt[2][0] - rho * e[2], dgt[2][1] - rho * e[4], dgt[2][2] - rho * e[5]}};
  double dgb[3], gdb[3];
  for (int i = 0; i < 3; ++i) {
    dgb[i] = dg[i][0] * bu[0] + dg[i][1] * bu[1] + dg[i][2] * bu[2];
    gdb[i] = g[i][0] * db[0] + g[i][1] * db[1] + g[i][2] * db[2];
  }
  out[0] = -dA + (bu[0] * dgb[0] + bu[1] * dgb[1] + bu[2] * dgb[2]) + 2.0 * (bl[0] * db[0] + bl[1] * db[1] + bl[2] * db[2]);
  for (int i = 0; i < 3; ++i) out[1 + i] = dgb[i] + gdb[i];
  out[4] = dg[0][0]; out[5] = dg[1][0]; out[6] = dg[2][0];
  out[7] = dg[1][1]; out[8] = dg[2][1]; out[9] = dg[2][2];
}

}  // namespace tgh
