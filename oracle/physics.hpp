// TEST INFRASTRUCTURE -- part of the CPU oracle (see stencils.hpp).
//
// Profiles and the sphere interior:
//   smoothstep, Interior, interior_profiles, _layer_profiles   src/interior.jl:117-120, 567-590
//   is_frozen / is_outside / core_follows / core_position      src/interior.jl:328-363, 615-625
//   core_rate, layer_rate_step, core_rate_weight               src/interior.jl:476-565
//   core_relaxation_rate, _adm_split                           src/interior.jl:420-470
//   ConstantDamping, GaussianDamping, HorizonDissipation       src/gauge.jl:1094-1266
//   background_state_rate, core_target_rate                    src/initialdata.jl:1721-1796
#pragma once
#include <cmath>
#include <limits>

#include "spacetime.hpp"

namespace orc {

static inline double clamp01(double s) { return s < 0.0 ? 0.0 : (s > 1.0 ? 1.0 : s); }
// src/interior.jl:117-120
static inline double smoothstep(double s) {
  double u = clamp01(s);
  return clamp01(u * u * u * (10.0 + u * (6.0 * u - 15.0)));
}

struct Interior {
  int variant = TGH_INT_NONE;
  double c0[3] = {0, 0, 0}, v[3] = {0, 0, 0};
  double r0 = 0, r1 = 0, rho_max = 0, w_ramp = 0.5, rho_ramp = 0.5;
  void center(double t, double c[3]) const {
    for (int i = 0; i < 3; ++i) c[i] = c0[i] + t * v[i];
  }
  double radius(double t, const double x[3]) const {
    double c[3];
    center(t, c);
    double d1 = x[0] - c[0], d2 = x[1] - c[1], d3 = x[2] - c[2];
    return std::sqrt(d1 * d1 + d2 * d2 + d3 * d3);
  }
  bool is_frozen(double r) const { return variant == TGH_INT_PASTED ? r < r1 : r < r0; }
  bool is_outside(double r) const { return r >= r1; }
  bool in_layer(double r) const { return r0 <= r && r < r1; }
  bool core_follows() const {
    return variant == TGH_INT_DAMPED && !(v[0] == 0.0 && v[1] == 0.0 && v[2] == 0.0);
  }
  void profiles(double r, double& w, double& rho) const {
    double s = (r - r0) / (r1 - r0);
    w = smoothstep(s / w_ramp);
    rho = variant == TGH_INT_FROZEN ? 0.0 : rho_max * smoothstep((1.0 - s) / rho_ramp);
  }
  double core_rate() const {
    double s = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    double k = 12.0 * s / r0;
    return rho_max > k ? rho_max : k;
  }
  double layer_rate_step() const { return std::cbrt(std::numeric_limits<double>::epsilon()) * r0; }
  double core_rate_weight(double r) const { return smoothstep(4.0 * r / r0 - 1.0); }
  // src/interior.jl:615-625 (no hole: the identity)
  void core_position(double t, const double x[3], double out[3]) const {
    if (variant == TGH_INT_NONE) {
      for (int i = 0; i < 3; ++i) out[i] = x[i];
      return;
    }
    double c[3];
    center(t, c);
    double d[3] = {x[0] - c[0], x[1] - c[1], x[2] - c[2]};
    double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (r >= r0) {
      for (int i = 0; i < 3; ++i) out[i] = x[i];
      return;
    }
    double n[3] = {0.0, 0.0, 1.0};
    if (r != 0.0)
      for (int i = 0; i < 3; ++i) n[i] = d[i] / r;
    for (int i = 0; i < 3; ++i) out[i] = c[i] + r0 * n[i];
  }
};

struct Profiles {
  int damping, dissipation;
  double gamma0, dn, df, dw, dc0[3], dv[3];
  double eps, eo, ei, er1, erh, ec0[3], ev[3];
  double damping_rate(double t, const double x[3]) const {
    if (damping == TGH_DAMP_CONSTANT) return gamma0;
    double d1 = x[0] - (dc0[0] + t * dv[0]), d2 = x[1] - (dc0[1] + t * dv[1]),
           d3 = x[2] - (dc0[2] + t * dv[2]);
    double r2 = d1 * d1 + d2 * d2 + d3 * d3;
    return df + (dn - df) * std::exp(-r2 / (2.0 * dw * dw));
  }
  double dissipation_rate(double t, const double x[3]) const {
    if (dissipation == TGH_DISS_CONSTANT) return eps;
    double d1 = x[0] - (ec0[0] + t * ev[0]), d2 = x[1] - (ec0[1] + t * ev[1]),
           d3 = x[2] - (ec0[2] + t * ev[2]);
    double r = std::sqrt(d1 * d1 + d2 * d2 + d3 * d3);
    if (r >= erh) return eo;
    if (r <= er1) return ei;
    double s = (erh - r) / (erh - er1);
    return eo + (ei - eo) * smoothstep(s);
  }
  bool has_dissipation() const {
    return dissipation == TGH_DISS_CONSTANT ? eps != 0.0 : !(eo == 0.0 && ei == 0.0);
  }
};

// src/initialdata.jl:1721-1729
static inline void background_state_rate(const tgh_background& bg, double t, const double x[3],
                                         double dl, double h[NC], double Pi[NC], double dth[NC],
                                         double dtPi[NC]) {
  double dh[3][NC], Pp[NC], Pm[NC], hx[NC], dgx[NC], dhx[3][NC];
  background_state(bg, t, x, h, Pi, dh, dth);
  double tp = t + dl, tm = t - dl;
  background_state(bg, tp, x, hx, Pp, dhx, dgx);
  background_state(bg, tm, x, hx, Pm, dhx, dgx);
  for (int n = 0; n < NC; ++n) dtPi[n] = (Pp[n] - Pm[n]) / (tp - tm);
}

// src/initialdata.jl:1784-1796
static inline void core_target_rate(const Interior& in, const tgh_background& bg, double t,
                                    const double x[3], double dl, double dth[NC], double dtPi[NC]) {
  double s = in.core_rate_weight(in.radius(t, x));
  if (s == 0.0) {
    for (int n = 0; n < NC; ++n) dth[n] = dtPi[n] = 0.0;
    return;
  }
  double tp = t + dl, tm = t - dl;
  double xp[3], xm[3], hp[NC], Pp[NC], hm[NC], Pm[NC], dh[3][NC], dg[NC];
  in.core_position(tp, x, xp);
  in.core_position(tm, x, xm);
  background_state(bg, tp, xp, hp, Pp, dh, dg);
  background_state(bg, tm, xm, hm, Pm, dh, dg);
  double f = s / (tp - tm);
  for (int n = 0; n < NC; ++n) {
    dth[n] = f * (hp[n] - hm[n]);
    dtPi[n] = f * (Pp[n] - Pm[n]);
  }
}

// _adm_split (src/interior.jl:462-470)
static inline void adm_split(const double* h, double& A, double bu[3], double bl[3], double g[3][3]) {
  g[0][0] = 1.0 + h[4]; g[0][1] = h[5]; g[0][2] = h[6];
  g[1][0] = h[5]; g[1][1] = 1.0 + h[7]; g[1][2] = h[8];
  g[2][0] = h[6]; g[2][1] = h[8]; g[2][2] = 1.0 + h[9];
  bl[0] = h[1]; bl[1] = h[2]; bl[2] = h[3];
  double gi[3][3];
  inv3(g, gi);
  for (int i = 0; i < 3; ++i) bu[i] = gi[i][0] * bl[0] + gi[i][1] * bl[1] + gi[i][2] * bl[2];
  A = (1.0 - h[0]) + (bu[0] * bl[0] + bu[1] * bl[1] + bu[2] * bl[2]);
}

// src/interior.jl:420-459
static inline void core_relaxation_rate(const double* h, const double* ht, double rho,
                                        const double* dtht, double out[NC]) {
  double A, bu[3], bl[3], g[3][3], At, but[3], blt[3], gt[3][3];
  adm_split(h, A, bu, bl, g);
  adm_split(ht, At, but, blt, gt);
  double dgt[3][3] = {{dtht[4], dtht[5], dtht[6]}, {dtht[5], dtht[7], dtht[8]}, {dtht[6], dtht[8], dtht[9]}};
  double gti[3][3];
  inv3(gt, gti);
  double dgtb[3];
  for (int i = 0; i < 3; ++i) dgtb[i] = dgt[i][0] * but[0] + dgt[i][1] * but[1] + dgt[i][2] * but[2];
  double rhs3[3] = {dtht[1] - dgtb[0], dtht[2] - dgtb[1], dtht[3] - dgtb[2]};
  double dbt[3];
  for (int i = 0; i < 3; ++i) dbt[i] = gti[i][0] * rhs3[0] + gti[i][1] * rhs3[1] + gti[i][2] * rhs3[2];
  double dAt = -dtht[0] + (but[0] * dgtb[0] + but[1] * dgtb[1] + but[2] * dgtb[2]) +
               2.0 * (blt[0] * dbt[0] + blt[1] * dbt[1] + blt[2] * dbt[2]);
  double dA = dAt - rho * (A - At);
  double db[3];
  for (int i = 0; i < 3; ++i) db[i] = dbt[i] - rho * (bu[i] - but[i]);
  double dh6[6] = {h[4] - ht[4], h[5] - ht[5], h[6] - ht[6], h[7] - ht[7], h[8] - ht[8], h[9] - ht[9]};
  double dg[3][3] = {{dgt[0][0] - rho * dh6[0], dgt[0][1] - rho * dh6[1], dgt[0][2] - rho * dh6[2]},
                     {dgt[1][0] - rho * dh6[1], dgt[1][1] - rho * dh6[3], dgt[1][2] - rho * dh6[4]},
                     {dgt[2][0] - rho * dh6[2], dgt[2][1] - rho * dh6[4], dgt[2][2] - rho * dh6[5]}};
  double dgb[3], gdb[3];
  for (int i = 0; i < 3; ++i) {
    dgb[i] = dg[i][0] * bu[0] + dg[i][1] * bu[1] + dg[i][2] * bu[2];
    gdb[i] = g[i][0] * db[0] + g[i][1] * db[1] + g[i][2] * db[2];
  }
  double dtt = -dA + (bu[0] * dgb[0] + bu[1] * dgb[1] + bu[2] * dgb[2]) +
               2.0 * (bl[0] * db[0] + bl[1] * db[1] + bl[2] * db[2]);
  out[0] = dtt;
  out[1] = dgb[0] + gdb[0];
  out[2] = dgb[1] + gdb[1];
  out[3] = dgb[2] + gdb[2];
  out[4] = dg[0][0];
  out[5] = dg[1][0];
  out[6] = dg[2][0];
  out[7] = dg[1][1];
  out[8] = dg[2][1];
  out[9] = dg[2][2];
}

}  // namespace orc
