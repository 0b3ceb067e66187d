// The analytic state of a case, evaluated with every operation rounded on its own.
//
// The moving hole's target rates are centred differences of the analytic state at t +- dl with
// dl = cbrt(eps) r_0 (src/initialdata.jl:1721-1729, 1784-1796): a one-ulp change in either
// evaluation moves the rate by ulp / (2 dl), about 1e-11 of the state. So that the kernels'
// rates are the oracle's to roundoff of the rate itself, the state they difference is
// evaluated here in the reference's own spelling, with no product fused into a sum
// (__dadd_rn / __dmul_rn / __ddiv_rn / __dsqrt_rn on the device): the closed forms in the order
// SpacetimeMetrics' restatement evaluates them, forward-mode duals with the quotient and root
// rules of ForwardDiff (value and partials, src/initialdata.jl:1681-1694), metric_quantities in
// the spelling of src/pointwise.jl:145-184 (the 4x4 inverse by cofactors, the elementary
// symmetric polynomials of eta h for sqrt(gamma)), and the sphere interior's placement
// (src/interior.jl:615-625, in physics.cuh). Division and square root are IEEE correctly
// rounded on both sides, so the same sequence of rounded operations gives the same bits.
//
// These evaluations serve the Dirichlet ghosts, the initial state, the :pasted overwrite, the
// error norm's exact solution and the interior layer's and core's targets; the right-hand side's
// own algebra (physics.cuh metric_quantities, algebra.cuh) stays contracted.
#pragma once
#include "physics.cuh"

#ifdef __CUDACC__
#define TGH_NOINLINE __noinline__
#else
#define TGH_NOINLINE __attribute__((noinline))
#endif

namespace tgh {

// double arithmetic rounded per operation (never contracted into a fused multiply-add)
struct RN {
  double v;
  TGH_HD RN() {}
  TGH_HD RN(double x) : v(x) {}
};
TGH_HD RN operator+(RN a, RN b) { return RN(TGH_RADD(a.v, b.v)); }
TGH_HD RN operator-(RN a, RN b) { return RN(TGH_RSUB(a.v, b.v)); }
TGH_HD RN operator*(RN a, RN b) { return RN(TGH_RMUL(a.v, b.v)); }
TGH_HD RN operator/(RN a, RN b) { return RN(TGH_RDIV(a.v, b.v)); }
TGH_HD RN operator-(RN a) { return RN(-a.v); }
TGH_HD RN rsqrt_n(RN a) { return RN(TGH_RSQRT(a.v)); }
TGH_HD RN rsin_n(RN a) { return RN(sin(a.v)); }
TGH_HD RN rcos_n(RN a) { return RN(cos(a.v)); }
TGH_HD RN rtanh_n(RN a) { return RN(tanh(a.v)); }

// forward-mode dual over (t, x, y, z) with ForwardDiff's rules, each step rounded
struct RD {
  RN v, d[4];
  TGH_HD RD() {}
  TGH_HD RD(double c) : v(c) { d[0] = d[1] = d[2] = d[3] = RN(0.0); }
};
TGH_HD RD operator+(const RD& a, const RD& b) {
  RD r;
  r.v = a.v + b.v;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
TGH_HD RD operator-(const RD& a, const RD& b) {
  RD r;
  r.v = a.v - b.v;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
TGH_HD RD operator-(const RD& a) {
  RD r;
  r.v = -a.v;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = -a.d[i];
  return r;
}
TGH_HD RD operator*(const RD& a, const RD& b) {
  RD r;
  r.v = a.v * b.v;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
TGH_HD RD operator/(const RD& a, const RD& b) {
  RD r;
  r.v = a.v / b.v;
  const RN bb = b.v * b.v;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = (a.d[i] * b.v - a.v * b.d[i]) / bb;
  return r;
}
TGH_HD RD rd_chain(const RD& a, RN f, RN df) {
  RD r;
  r.v = f;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = df * a.d[i];
  return r;
}
TGH_HD RD rsqrt_n(const RD& a) {
  const RN s = rsqrt_n(a.v);
  return rd_chain(a, s, RN(1.0) / (RN(2.0) * s));
}
TGH_HD RD rsin_n(const RD& a) { return rd_chain(a, rsin_n(a.v), rcos_n(a.v)); }
TGH_HD RD rtanh_n(const RD& a) {
  const RN th = rtanh_n(a.v);
  return rd_chain(a, th, RN(1.0) - th * th);
}

// Kerr-Schild in its rest frame at (t, x, y, z): g = eta + 2 H l l
TGH_HD void rn_kerr_schild(double M, double a, const RD x[4], RD g[4][4]) {
  const RD X = x[1], Y = x[2], Z = x[3];
  const RD rho2 = X * X + Y * Y + Z * Z;
  const RD a2 = RD(a * a);
  const RD half = RD(0.5) * (rho2 - a2);
  const RD r2 = half + rsqrt_n(half * half + a2 * Z * Z);
  const RD r = rsqrt_n(r2);
  const RD H = RD(M) * r * r2 / (r2 * r2 + a2 * Z * Z);
  const RD den = r2 + a2;
  const RD l[4] = {RD(1.0), (r * X + RD(a) * Y) / den, (r * Y - RD(a) * X) / den, Z / r};
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) g[i][j] = RD(i == j ? etad(i) : 0.0) + RD(2.0) * H * l[i] * l[j];
}

// the rounded duals for the templated closed forms of physics.cuh (found by argument lookup)
TGH_HD RD dsqrt(const RD& a) { return rsqrt_n(a); }
TGH_HD void ks_rest(double M, double a, const RD* x, RD g[4][4]) { rn_kerr_schild(M, a, x, g); }

// a hole's metric in its rest frame: Kerr-Schild, or Kerr in harmonic coordinates
TGH_HD void rn_hole_rest(const Case& c, const RD x[4], RD g[4][4]) {
  if (c.bg.kind == TGH_BG_HARMONIC_KERR)
    harmonic_kerr_rest<RD>(c.bg.M, c.bg.a, x, g);
  else
    rn_kerr_schild(c.bg.M, c.bg.a, x, g);
}

// the case's metric g_ab with its first derivatives at xin = (t, x, y, z)
TGH_HD void rn_metric(const Case& c, const RD xin[4], RD g[4][4]) {
  RD x[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) x[i] = xin[i] - RD(c.bg.translate[i]);
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) g[i][j] = RD(i == j ? etad(i) : 0.0);
  if (c.bg.kind == TGH_BG_GAUGE_WAVE) {
    const RD H = RD(1.0) - RD(c.bg.A) * rsin_n(RD(2.0 * M_PI) * (x[1] - x[0]) / RD(c.bg.d));
    g[0][0] = -H;
    g[1][1] = H;
  } else if (c.bg.kind == TGH_BG_SHIFTED_MINKOWSKI) {
    const RD th = rtanh_n(x[1] / RD(c.bg.d));
    const RD psi = RD(c.bg.A) * (RD(1.0) - th * th);
    g[0][1] = -psi;
    g[1][0] = -psi;
    g[1][1] = RD(1.0) - psi * psi;
  } else if (c.bg.kind == TGH_BG_KERR_SCHILD || c.bg.kind == TGH_BG_HARMONIC_KERR) {
    if (!c.boosted) {
      rn_hole_rest(c, x, g);
      return;
    }
    RD xr[4], gr[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      RD s = RD(c.L[i][0]) * x[0];
#pragma unroll
      for (int j = 1; j < 4; ++j) s = s + RD(c.L[i][j]) * x[j];
      xr[i] = s;
    }
    rn_hole_rest(c, xr, gr);
    // g_ab = sum_cd (L_ca L_db) g_rest_cd, c outer, d inner
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        RD s = RD(0.0);
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) s = s + RD(TGH_RMUL(c.L[p][a], c.L[q][b])) * gr[p][q];
        g[a][b] = s;
      }
  }
}

TGH_HD RN rn_det3(RN a, RN b, RN c, RN d, RN e, RN f, RN g, RN h, RN i) {
  return a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
}
TGH_HD RN rn_minor(const RN m[4][4], int i, int j) {
  int r[3], c[3], kr = 0, kc = 0;
#pragma unroll
  for (int ii = 0; ii < 4; ++ii)
    if (ii != i) r[kr++] = ii;
#pragma unroll
  for (int jj = 0; jj < 4; ++jj)
    if (jj != j) c[kc++] = jj;
  return rn_det3(m[r[0]][c[0]], m[r[0]][c[1]], m[r[0]][c[2]], m[r[1]][c[0]], m[r[1]][c[1]], m[r[1]][c[2]],
                 m[r[2]][c[0]], m[r[2]][c[1]], m[r[2]][c[2]]);
}

// metric_quantities (src/pointwise.jl:145-184) in its own spelling: the lapse, the shift and
// sqrt(gamma) the analytic Pi needs
TGH_HD void rn_metric_quantities(const RN h[NC], RN& alpha, RN beta[3], RN& sqrtg) {
  RN hm[4][4], g4[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      hm[a][b] = h[pidx(a, b)];
      g4[a][b] = RN(a == b ? etad(a) : 0.0) + hm[a][b];
    }
  RN cof[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const RN mi = rn_minor(g4, i, j);
      cof[i][j] = ((i + j) % 2 == 0) ? mi : -mi;
    }
  const RN det = g4[0][0] * cof[0][0] + g4[0][1] * cof[0][1] + g4[0][2] * cof[0][2] + g4[0][3] * cof[0][3];
  RN gi[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) gi[i][j] = cof[j][i] / det;
  RN gu4[4][4], q1 = RN(0.0);
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      RN s = gi[a][0] * hm[0][b];
#pragma unroll
      for (int k = 1; k < 4; ++k) s = s + gi[a][k] * hm[k][b];
      const RN guo = -(s * RN(etad(b)));
      if (a == 0 && b == 0) q1 = guo;
      gu4[a][b] = RN(a == b ? etad(a) : 0.0) + guo;
    }
  const RN gutt = gu4[0][0];
  alpha = RN(1.0) / rsqrt_n(RN(1.0) - q1);
#pragma unroll
  for (int i = 0; i < 3; ++i) beta[i] = -gu4[0][i + 1] / gutt;
  RN B[4][4], B2[4][4], B3[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) B[a][b] = RN(etad(a)) * hm[a][b];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      RN s = B[a][0] * B[0][b];
#pragma unroll
      for (int k = 1; k < 4; ++k) s = s + B[a][k] * B[k][b];
      B2[a][b] = s;
    }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      RN s = B2[a][0] * B[0][b];
#pragma unroll
      for (int k = 1; k < 4; ++k) s = s + B2[a][k] * B[k][b];
      B3[a][b] = s;
    }
  const RN trB = ((B[0][0] + B[1][1]) + B[2][2]) + B[3][3];
  const RN trB2 = ((B2[0][0] + B2[1][1]) + B2[2][2]) + B2[3][3];
  const RN trB3 = ((B3[0][0] + B3[1][1]) + B3[2][2]) + B3[3][3];
  const RN e2 = (trB * trB - trB2) / RN(2.0);
  const RN e3 = (trB * trB * trB - RN(3.0) * trB * trB2 + RN(2.0) * trB3) / RN(6.0);
  // det(B) by cofactors along the first row
  RN e4 = RN(0.0);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    int c[3], k = 0;
#pragma unroll
    for (int jj = 0; jj < 4; ++jj)
      if (jj != j) c[k++] = jj;
    const RN mi = rn_det3(B[1][c[0]], B[1][c[1]], B[1][c[2]], B[2][c[0]], B[2][c[1]], B[2][c[2]], B[3][c[0]],
                          B[3][c[1]], B[3][c[2]]);
    e4 = (j % 2 == 0) ? e4 + B[0][j] * mi : e4 - B[0][j] * mi;
  }
  const RN d1 = -(((trB + e2) + e3) + e4);
  const RN detgm1 = -d1 - q1 + d1 * q1;
  sqrtg = rsqrt_n(RN(1.0) + detgm1);
}

// background_state (src/initialdata.jl:1681-1694): h, Pi and (optionally) d_t g of the
// background at (t, x), from one dual pass. Called, not inlined: the kernels reach it only at
// Dirichlet ghosts and interior points, and its dual arithmetic would otherwise crowd the
// registers of their main path.
static __host__ __device__ TGH_NOINLINE void rn_background_state(const Case& c, double t, const double* x,
                                                                 double* h, double* Pi, double* dtg_out = nullptr) {
  RD p[4];
  const double pv[4] = {t, x[0], x[1], x[2]};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    p[i] = RD(pv[i]);
    p[i].d[i] = RN(1.0);
  }
  RD g[4][4];
  rn_metric(c, p, g);
  RN hh[NC], dtg[NC], dh[3][NC];
#pragma unroll
  for (int n = 0; n < NC; ++n) {
    const RD& e = g[prow(n)][pcol(n)];
    hh[n] = e.v - RN(prow(n) == pcol(n) ? etad(prow(n)) : 0.0);
    dtg[n] = e.d[0];
    dh[0][n] = e.d[1];
    dh[1][n] = e.d[2];
    dh[2][n] = e.d[3];
  }
  RN alpha, beta[3], sqrtg;
  rn_metric_quantities(hh, alpha, beta, sqrtg);
  const RN f = sqrtg / alpha;
#pragma unroll
  for (int n = 0; n < NC; ++n) {
    h[n] = hh[n].v;
    Pi[n] = (f * (dtg[n] - beta[0] * dh[0][n] - beta[1] * dh[1][n] - beta[2] * dh[2][n])).v;
    if (dtg_out) dtg_out[n] = dtg[n].v;
  }
}

// the state the case puts at x (case_state_tuple): the background through the core rule
TGH_HD void exact_state(const Case& c, double t, const double* x, double* out) {
  double xc[3];
  core_position(c, t, x, xc);
  rn_background_state(c, t, xc, out, out + NC);
}

}  // namespace tgh
