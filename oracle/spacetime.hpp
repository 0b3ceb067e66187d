// TEST INFRASTRUCTURE -- part of the CPU oracle (see stencils.hpp).
//
// Analytic backgrounds and their derivatives by forward-mode duals. The reference takes
// these from the un-vendored SpacetimeMetrics package (compat 1.6, git main, no manifest:
// no exact pin); its call sites are src/initialdata.jl:1682-1694 (dmetric),
// src/gauge.jl:114,182 (dmetric, gauge_source_grad) and src/initialdata.jl:1295-1296
// (boost, translate). Restated here from the published closed forms:
//   Minkowski          g = eta
//   GaugeWave(A, d)    ds^2 = -H dt^2 + H dx^2 + dy^2 + dz^2, H = 1 - A sin(2 pi (x - t)/d)
//                      (src/initialdata.jl:895-911)
//   ShiftedMinkowski   flat space in t^ = t + A w tanh(x/w) (src/initialdata.jl:914-947)
//   KerrSchild(M, a)   g = eta + 2 H l l,  H = M r^3 / (r^4 + a^2 z^2),
//                      l = (1, (r x + a y)/(r^2+a^2), (r y - a x)/(r^2+a^2), z/r)
//   Harmonic(M, a)     Kerr in horizon-penetrating harmonic coordinates: the Kerr-Schild metric
//                      pulled back, g = J^T g_KS J, along the map from the harmonic chart
//                      X + i Y = w (x + i y), Z = (r / r_H) z, T = t + 2 M ln(r_H + sqrt(M^2 - a^2)),
//                      w = (r + i a) / (r_H + i a), r = r_H + M, r_H the spheroidal radius of
//                      (x, y, z) with parameter a (the Kerr-Schild quartic): both charts share the
//                      Kerr-Schild angle phi, the harmonic radius is r - M, and the harmonic time
//                      t_BL + 2 M r_+ int dr / Delta is regular on the future horizon. J is formed
//                      in closed form from d r_H / d x^i = r_H (x_i r_H^2 + a^2 z delta_iz) /
//                      (r_H^4 + a^2 z^2); the chart is harmonic (H_a = 0) and at a = 0 it is the
//                      harmonic Schwarzschild metric g_tt = -(r-M)/(r+M), g_tr = 4M^2/(r+M)^2
//   boost(m, u)        m evaluated at Lambda(u) x and pulled back, the hole moves at -u
//                      (src/interior.jl:67-73)
//   translate(m, D)    m evaluated at x - D
// and the gauge source H_a = -g^{cd} Gamma_{a,cd} with its gradient by nested duals
// (src/gauge.jl:156-212: H_b then d_a H_b, column-major).
#pragma once
#include <cmath>

#include "../include/tgh.h"
#include "pointwise.hpp"

namespace orc {

// ---- forward-mode dual with four directions (t, x, y, z) ----
template <class T> struct D4 {
  T v;
  T d[4];
  D4() : v(0) { d[0] = d[1] = d[2] = d[3] = T(0); }
  D4(double c) : v(c) { d[0] = d[1] = d[2] = d[3] = T(0); }
  D4(const T& c, int) : v(c) { d[0] = d[1] = d[2] = d[3] = T(0); }
};
template <class T> static inline D4<T> mkc(const T& c) { return D4<T>(c, 0); }
template <class T> static inline D4<T> operator+(const D4<T>& a, const D4<T>& b) {
  D4<T> r;
  r.v = a.v + b.v;
  for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
template <class T> static inline D4<T> operator-(const D4<T>& a, const D4<T>& b) {
  D4<T> r;
  r.v = a.v - b.v;
  for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
template <class T> static inline D4<T> operator-(const D4<T>& a) {
  D4<T> r;
  r.v = -a.v;
  for (int i = 0; i < 4; ++i) r.d[i] = -a.d[i];
  return r;
}
template <class T> static inline D4<T> operator*(const D4<T>& a, const D4<T>& b) {
  D4<T> r;
  r.v = a.v * b.v;
  for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
template <class T> static inline D4<T> operator/(const D4<T>& a, const D4<T>& b) {
  D4<T> r;
  r.v = a.v / b.v;
  for (int i = 0; i < 4; ++i) r.d[i] = (a.d[i] * b.v - a.v * b.d[i]) / (b.v * b.v);
  return r;
}
template <class T> static inline bool operator!=(const D4<T>& a, const D4<T>& b) { return a.v != b.v; }
template <class T> static inline D4<T> chain(const D4<T>& a, const T& f, const T& df) {
  D4<T> r;
  r.v = f;
  for (int i = 0; i < 4; ++i) r.d[i] = df * a.d[i];
  return r;
}
template <class T> static inline D4<T> sqrt(const D4<T>& a) {
  using std::sqrt;
  T s = sqrt(a.v);
  return chain(a, s, T(1) / (T(2) * s));
}
template <class T> static inline D4<T> sin(const D4<T>& a) {
  using std::cos;
  using std::sin;
  return chain(a, sin(a.v), cos(a.v));
}
template <class T> static inline D4<T> cos(const D4<T>& a) {
  using std::cos;
  using std::sin;
  return chain(a, cos(a.v), -sin(a.v));
}
template <class T> static inline D4<T> tanh(const D4<T>& a) {
  using std::tanh;
  T th = tanh(a.v);
  return chain(a, th, T(1) - th * th);
}
template <class T> static inline D4<T> exp(const D4<T>& a) {
  using std::exp;
  T e = exp(a.v);
  return chain(a, e, e);
}

typedef D4<double> Dd;
typedef D4<Dd> Ddd;

template <class S> static inline S sq(const S& a) { return a * a; }

// Kerr-Schild in its rest frame (t = x[0])
template <class S> static inline void kerr_schild(double M, double a, const S x[4], S g[4][4]) {
  S X = x[1], Y = x[2], Z = x[3];
  S rho2 = X * X + Y * Y + Z * Z;
  S a2 = S(a * a);
  S half = S(0.5) * (rho2 - a2);
  S r2 = half + sqrt(half * half + a2 * Z * Z);
  S r = sqrt(r2);
  S H = S(M) * r * r2 / (r2 * r2 + a2 * Z * Z);
  S den = r2 + a2;
  S l[4] = {S(1.0), (r * X + S(a) * Y) / den, (r * Y - S(a) * X) / den, Z / r};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) g[i][j] = S(i == j ? eta(i) : 0.0) + S(2.0) * H * l[i] * l[j];
}

// Kerr in harmonic coordinates in its rest frame (t = x[0]; the metric does not depend on t)
template <class S> static inline void harmonic_kerr(double M, double a, const S x[4], S g[4][4]) {
  S X = x[1], Y = x[2], Z = x[3];
  S rho2 = X * X + Y * Y + Z * Z;
  S a2 = S(a * a);
  S half = S(0.5) * (rho2 - a2);
  S r2 = half + sqrt(half * half + a2 * Z * Z);  // r_H^2
  S rh = sqrt(r2);
  S q = r2 * r2 + a2 * Z * Z;
  // d r_H / d x^i
  S dr[3] = {rh * (X * r2) / q, rh * (Y * r2) / q, rh * (Z * r2 + a2 * Z) / q};
  S r = rh + S(M);
  S D = r2 + a2;
  S wr = (r * rh + a2) / D;  // w = (r + i a) / (r_H + i a)
  S wi = S(-a * M) / D;
  S D2 = D * D;
  S dwr = S(-M) * (r2 - a2) / D2;  // d w / d r_H = -M / (r_H + i a)^2
  S dwi = S(2.0 * M * a) * rh / D2;
  S px = X * dwr - Y * dwi;  // Re, Im of (x + i y) d w / d r_H
  S py = X * dwi + Y * dwr;
  S zr = r / rh;
  S zd = S(-M) * Z / r2;
  S tr = S(2.0 * M) / (rh + S(std::sqrt(M * M - a * a)));
  // the Kerr-Schild point and J[A][b] = d X^A / d x^b
  S xk[4] = {x[0], wr * X - wi * Y, wr * Y + wi * X, zr * Z};
  S J[4][4];
  J[0][0] = S(1.0);
  J[1][0] = J[2][0] = J[3][0] = S(0.0);
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
  kerr_schild(M, a, xk, gk);
  for (int p = 0; p < 4; ++p)
    for (int s = 0; s < 4; ++s) {
      S acc = S(0.0);
      for (int A = 0; A < 4; ++A) {
        S t = J[0][s] * gk[A][0];
        for (int B = 1; B < 4; ++B) t = t + J[B][s] * gk[A][B];
        acc = acc + J[A][p] * t;
      }
      g[p][s] = acc;
    }
}

// the boost matrix Lambda(u): x_rest = Lambda x_lab
static inline void boost_matrix(const double u[3], double L[4][4]) {
  double u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  double gam = 1.0 / std::sqrt(1.0 - u2);
  L[0][0] = gam;
  for (int i = 0; i < 3; ++i) {
    L[0][i + 1] = gam * u[i];
    L[i + 1][0] = gam * u[i];
    for (int j = 0; j < 3; ++j)
      L[i + 1][j + 1] = (i == j ? 1.0 : 0.0) + (u2 > 0 ? (gam - 1.0) * u[i] * u[j] / u2 : 0.0);
  }
}

template <class S> static inline void metric_eval(const tgh_background& bg, const S xin[4], S g[4][4]) {
  S x[4];
  for (int i = 0; i < 4; ++i) x[i] = xin[i] - S(bg.translate[i]);
  switch (bg.kind) {
    case TGH_BG_MINKOWSKI:
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) g[i][j] = S(i == j ? eta(i) : 0.0);
      return;
    case TGH_BG_GAUGE_WAVE: {
      S H = S(1.0) - S(bg.A) * sin(S(2.0 * M_PI) * (x[1] - x[0]) / S(bg.d));
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) g[i][j] = S(i == j ? eta(i) : 0.0);
      g[0][0] = -H;
      g[1][1] = H;
      return;
    }
    case TGH_BG_SHIFTED_MINKOWSKI: {
      S c = tanh(x[1] / S(bg.d));
      S psi = S(bg.A) * (S(1.0) - c * c);  // A sech^2(x/w)
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) g[i][j] = S(i == j ? eta(i) : 0.0);
      g[0][1] = -psi;
      g[1][0] = -psi;
      g[1][1] = S(1.0) - psi * psi;
      return;
    }
    case TGH_BG_KERR_SCHILD:
    case TGH_BG_HARMONIC_KERR: {
      auto rest = [&](const S* y, S (*gy)[4]) {
        if (bg.kind == TGH_BG_KERR_SCHILD)
          kerr_schild(bg.M, bg.a, y, gy);
        else
          harmonic_kerr(bg.M, bg.a, y, gy);
      };
      bool boosted = bg.boost[0] != 0.0 || bg.boost[1] != 0.0 || bg.boost[2] != 0.0;
      if (!boosted) {
        rest(x, g);
        return;
      }
      double L[4][4];
      boost_matrix(bg.boost, L);
      S xr[4];
      for (int i = 0; i < 4; ++i) {
        S s = S(L[i][0]) * x[0];
        for (int j = 1; j < 4; ++j) s = s + S(L[i][j]) * x[j];
        xr[i] = s;
      }
      S gr[4][4];
      rest(xr, gr);
      for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) {
          S s = S(0.0);
          for (int c = 0; c < 4; ++c)
            for (int d = 0; d < 4; ++d) s = s + S(L[c][a] * L[d][b]) * gr[c][d];
          g[a][b] = s;
        }
      return;
    }
  }
}

// dmetric: g and dg[a][b][c] = d_c g_ab (SpacetimeMetrics' order, derivative axis last)
static inline void dmetric(const tgh_background& bg, const double p[4], double g[4][4],
                           double dg[4][4][4]) {
  Dd x[4];
  for (int i = 0; i < 4; ++i) {
    x[i] = Dd(p[i]);
    x[i].d[i] = 1.0;
  }
  Dd gd[4][4];
  metric_eval(bg, x, gd);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      g[a][b] = gd[a][b].v;
      for (int c = 0; c < 4; ++c) dg[a][b][c] = gd[a][b].d[c];
    }
}

// ddmetric: g, dg[a][b][c] = d_a g_bc and ddg[a][b][c][d] = d_a d_b g_cd (derivative axes
// first) by nested duals: what the ADM pin of test/constraints_tests.jl:63-108 feeds the
// Ricci assembly
static inline void ddmetric(const tgh_background& bg, const double p[4], double g[4][4], double dg[4][4][4],
                            double ddg[4][4][4][4]) {
  Ddd x[4];
  for (int i = 0; i < 4; ++i) {
    x[i] = Ddd(p[i]);
    x[i].v.d[i] = 1.0;
    x[i].d[i] = Dd(1.0);
  }
  Ddd gg[4][4];
  metric_eval(bg, x, gg);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      g[a][b] = gg[a][b].v.v;
      for (int c = 0; c < 4; ++c) {
        dg[c][a][b] = gg[a][b].v.d[c];
        for (int e = 0; e < 4; ++e) ddg[e][c][a][b] = gg[a][b].d[e].d[c];
      }
    }
}

// src/initialdata.jl:1681-1694: h, Pi, dh from one dual pass (and d_t g)
static inline void background_state(const tgh_background& bg, double t, const double x[3],
                                    double h[NC], double Pi[NC], double dh[3][NC],
                                    double dtg[NC]) {
  double p[4] = {t, x[0], x[1], x[2]};
  double g[4][4], dg[4][4][4];
  dmetric(bg, p, g, dg);
  for (int n = 0; n < NC; ++n) {
    int a, b;
    unpair(n, a, b);
    h[n] = g[a][b] - (a == b ? eta(a) : 0.0);
    dtg[n] = dg[a][b][0];
    for (int i = 0; i < 3; ++i) dh[i][n] = dg[a][b][i + 1];
  }
  Coef<double> C;
  metric_quantities(h, C);
  double f = C.sqrtg / C.alpha;
  for (int n = 0; n < NC; ++n)
    Pi[n] = f * (dtg[n] - C.beta[0] * dh[0][n] - C.beta[1] * dh[1][n] - C.beta[2] * dh[2][n]);
}

// gauge_source_grad: Hl[b] = -g^{cd} Gamma_{b,cd} of the background, dHl[a][b] = d_a H_b
static inline void gauge_source_grad(const tgh_background& bg, const double p[4], double Hl[4],
                                     double dHl[4][4]) {
  Ddd x[4];
  for (int i = 0; i < 4; ++i) {
    x[i] = Ddd(p[i]);
    x[i].v.d[i] = 1.0;     // inner direction
    x[i].d[i] = Dd(1.0);   // outer direction
  }
  Ddd gg[4][4];
  metric_eval(bg, x, gg);
  Dd g[4][4], dg[4][4][4];  // dg[c][a][b] = d_c g_ab (with inner derivatives)
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      g[a][b] = gg[a][b].v;
      for (int c = 0; c < 4; ++c) dg[c][a][b] = gg[a][b].d[c];
    }
  Dd gu[4][4];
  inv4(g, gu);
  for (int a = 0; a < 4; ++a) {
    Dd s(0.0);
    for (int c = 0; c < 4; ++c)
      for (int d = 0; d < 4; ++d) {
        Dd G = Dd(0.5) * (dg[c][a][d] + dg[d][a][c] - dg[a][c][d]);
        s = s + gu[c][d] * G;
      }
    Dd H = -s;
    Hl[a] = H.v;
    for (int c = 0; c < 4; ++c) dHl[c][a] = H.d[c];
  }
}

// The closed-form Kerr-Schild gauge source (src/gauge.jl:257-326)
struct KSSource {
  double M, S[4], u[4];
};
static inline KSSource make_ks_source(double M, const double spin[3], const double vel[3]) {
  KSSource k;
  double v2 = vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2];
  double gam = 1.0 / std::sqrt(1.0 - v2);
  double va = vel[0] * spin[0] + vel[1] * spin[1] + vel[2] * spin[2];
  k.M = M;
  k.S[0] = gam * va;
  for (int i = 0; i < 3; ++i) k.S[i + 1] = v2 == 0.0 ? spin[i] : spin[i] + ((gam - 1.0) * va / v2) * vel[i];
  k.u[0] = gam;
  for (int i = 0; i < 3; ++i) k.u[i + 1] = gam * vel[i];
  return k;
}
// the value of a scalar for the branch conditions (an op-counting scalar overloads it)
static inline double dval(double x) { return x; }
// a where c > 0, else b (both formed; per lane for SIMD lanes)
static inline double select_pos(double c, double a, double b) { return c > 0 ? a : b; }

// src/gauge.jl:302-326 (+ _algebraic_dH :330-336); dHl[c][a] = d_c H_a. Templated on the
// scalar so the op-counting instantiation sees its arithmetic.
template <class T>
static inline void algebraic_gauge_source(const KSSource& src, const T* h, const T* dth, const T* const dh[3],
                                          T Hl[4], T dHl[4][4]) {
  using std::sqrt;
  T hm[4][4];
  sym4(h, hm);
  T w[4];
  for (int a = 0; a < 4; ++a) {
    T s = hm[a][0] * T(src.u[0]);
    for (int b = 1; b < 4; ++b) s = s + hm[a][b] * T(src.u[b]);
    w[a] = s;
  }
  T K = T(src.u[0]) * w[0];
  for (int a = 1; a < 4; ++a) K = K + T(src.u[a]) * w[a];
  T sw = T(src.S[0]) * w[0];
  for (int a = 1; a < 4; ++a) sw = sw + T(src.S[a]) * w[a];
  T rad = T(src.M) * T(src.M) - sw * sw;
  T root = select_pos(rad, sqrt(rad), T(0.0));
  T D = T(src.M) + root;
  for (int a = 0; a < 4; ++a) Hl[a] = (-K / D) * w[a];
  const T* Dp[4] = {dth, dh[0], dh[1], dh[2]};
  T dw[4][4];
  for (int c = 0; c < 4; ++c) {
    T dm[4][4];
    sym4(Dp[c], dm);
    for (int a = 0; a < 4; ++a) {
      T s = dm[a][0] * T(src.u[0]);
      for (int b = 1; b < 4; ++b) s = s + dm[a][b] * T(src.u[b]);
      dw[c][a] = s;
    }
  }
  for (int c = 0; c < 4; ++c) {
    T dK = T(src.u[0]) * dw[c][0];
    for (int a = 1; a < 4; ++a) dK = dK + T(src.u[a]) * dw[c][a];
    T Sdw = T(src.S[0]) * dw[c][0];
    for (int a = 1; a < 4; ++a) Sdw = Sdw + T(src.S[a]) * dw[c][a];
    T dD = select_pos(root, -sw * Sdw / root, T(0.0));
    for (int a = 0; a < 4; ++a) dHl[c][a] = -(dK * w[a] + K * dw[c][a]) / D + K * w[a] * dD / (D * D);
  }
}

}  // namespace orc
