// TEST INFRASTRUCTURE -- part of the CPU oracle (see stencils.hpp).
//
// The range projection of one point's state, restating src/bounds.jl:
//   _adm_split          src/bounds.jl:256-296
//   _surely_posdef      src/bounds.jl:298-318
//   _jacobi_rotation    src/bounds.jl:320-361
//   sym_eigen3          src/bounds.jl:365-393 (JACOBI_SWEEPS = 16)
//   _recompose          src/bounds.jl:395-398
//   _spectrum_clamp     src/bounds.jl:404-427 (BOUNDS_SLACK = 8)
//   _with_spatial / _with_shift / _with_lapse   src/bounds.jl:429-456
//   bounds_project      src/bounds.jl:458-527 (BOUNDS_PASSES = 4)
//   _project_once       src/bounds.jl:529-593
// Explicit scalar arithmetic in the reference's order; the file is compiled without
// floating-point contraction, as Julia evaluates it, so that a value recomputed from a stored
// state is the same bits at every call.
#pragma once
#include <cmath>
#include <limits>

namespace orc {

struct Bounds {
  double alpha_min, alpha_max, lambda_min, lambda_max, beta_max, K_max, r_gate;
};

static const double BEPS = std::numeric_limits<double>::epsilon();
static const int BOUNDS_SLACK = 8, BOUNDS_PASSES = 4, JACOBI_SWEEPS = 16;

// the offset metric as a 4x4 (row, column), from the packed (tt,tx,ty,tz,xx,xy,xz,yy,yz,zz)
static inline void sym4(const double* v, double m[4][4]) {
  static const int P[4][4] = {{0, 1, 2, 3}, {1, 4, 5, 6}, {2, 5, 7, 8}, {3, 6, 8, 9}};
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) m[a][b] = v[P[a][b]];
}
static inline void pack10(const double m[4][4], double* v) {
  v[0] = m[0][0]; v[1] = m[1][0]; v[2] = m[2][0]; v[3] = m[3][0];
  v[4] = m[1][1]; v[5] = m[2][1]; v[6] = m[3][1];
  v[7] = m[2][2]; v[8] = m[3][2]; v[9] = m[3][3];
}

struct AdmSplit {
  double g[6];  // gamma_11, 12, 13, 22, 23, 33
  double beta[3], detg, bb, a2;
};
static inline AdmSplit adm_split(const double hm[4][4]) {
  AdmSplit s;
  const double g11 = 1.0 + hm[1][1], g12 = hm[2][1], g13 = hm[3][1];
  const double g22 = 1.0 + hm[2][2], g23 = hm[3][2], g33 = 1.0 + hm[3][3];
  const double b1 = hm[1][0], b2 = hm[2][0], b3 = hm[3][0];
  const double c11 = g22 * g33 - g23 * g23;
  const double c12 = g13 * g23 - g12 * g33;
  const double c13 = g12 * g23 - g13 * g22;
  const double c22 = g11 * g33 - g13 * g13;
  const double c23 = g12 * g13 - g11 * g23;
  const double c33 = g11 * g22 - g12 * g12;
  s.detg = g11 * c11 + g12 * c12 + g13 * c13;
  const double qf = b1 * (c11 * b1 + c12 * b2 + c13 * b3) + b2 * (c12 * b1 + c22 * b2 + c23 * b3) +
                    b3 * (c13 * b1 + c23 * b2 + c33 * b3);
  s.bb = qf / s.detg;
  s.a2 = (1.0 - hm[0][0]) + s.bb;
  s.g[0] = g11; s.g[1] = g12; s.g[2] = g13; s.g[3] = g22; s.g[4] = g23; s.g[5] = g33;
  s.beta[0] = b1; s.beta[1] = b2; s.beta[2] = b3;
  return s;
}

static inline bool surely_posdef(double a11, double a12, double a13, double a22, double a23, double a33) {
  const double tol = 16 * BEPS;
  const double m2 = a11 * a22 - a12 * a12;
  const double e2 = std::fabs(a11 * a22) + a12 * a12;
  const double c1 = a22 * a33 - a23 * a23;
  const double c2 = a12 * a33 - a23 * a13;
  const double c3 = a12 * a23 - a22 * a13;
  const double m3 = a11 * c1 - a12 * c2 + a13 * c3;
  const double e3 = std::fabs(a11) * (std::fabs(a22 * a33) + a23 * a23) +
                    std::fabs(a12) * (std::fabs(a12 * a33) + std::fabs(a23 * a13)) +
                    std::fabs(a13) * (std::fabs(a12 * a23) + std::fabs(a22 * a13));
  return (a11 > 0.0) & (m2 > tol * e2) & (m3 > tol * e3);
}

// one rotation in the (p, q) plane (0-based) that annihilates A[p][q], accumulated into V
static inline void jacobi_rotation(double A[3][3], double V[3][3], int p, int q) {
  const double apq = A[p][q];
  if (apq == 0.0) return;
  const double app = A[p][p], aqq = A[q][q];
  const double tau = (aqq - app) / (2 * apq);
  const double t = std::fabs(tau) > 1.0 / std::sqrt(BEPS) ? 1.0 / (2 * tau)
                                                          : std::copysign(1.0, tau) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
  const double c = 1.0 / std::sqrt(1.0 + t * t);
  const double s = t * c;
  const int r = 3 - p - q;
  const double arp = A[r][p], arq = A[r][q];
  const double newp = app - t * apq, newq = aqq + t * apq;
  const double newrp = c * arp - s * arq, newrq = s * arp + c * arq;
  A[p][p] = newp;
  A[q][q] = newq;
  A[p][q] = A[q][p] = 0.0;
  A[r][p] = A[p][r] = newrp;
  A[r][q] = A[q][r] = newrq;
  for (int i = 0; i < 3; ++i) {
    const double vp = V[i][p], vq = V[i][q];
    V[i][p] = c * vp - s * vq;
    V[i][q] = s * vp + c * vq;
  }
}

static inline void sym_eigen3(double A[3][3], double lam[3], double V[3][3]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) V[i][j] = i == j ? 1.0 : 0.0;
  for (int sweep = 0; sweep < JACOBI_SWEEPS; ++sweep) {
    const double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
    const double on = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
    if (!(off > BEPS * BEPS * on)) break;
    jacobi_rotation(A, V, 0, 1);
    jacobi_rotation(A, V, 0, 2);
    jacobi_rotation(A, V, 1, 2);
  }
  lam[0] = A[0][0];
  lam[1] = A[1][1];
  lam[2] = A[2][2];
}

static inline double recompose(const double V[3][3], const double* l, int i, int j) {
  return V[i][0] * l[0] * V[j][0] + V[i][1] * l[1] * V[j][1] + V[i][2] * l[2] * V[j][2];
}
// Julia's clamp: x > hi ? hi : x < lo ? lo : x
static inline double jclamp(double x, double lo, double hi) { return x > hi ? hi : (x < lo ? lo : x); }

// gamma's spectrum clamped into [lmin, lmax]: g is left as it came unless an eigenvalue is
// outside by more than the slack, and then recomposed from the eigenvectors
static inline bool spectrum_clamp(const double g[6], double lmin, double lmax, double out[6]) {
  const double a11 = g[0], a12 = g[1], a13 = g[2], a22 = g[3], a23 = g[4], a33 = g[5];
  const bool lo = surely_posdef(a11 - lmin, a12, a13, a22 - lmin, a23, a33 - lmin);
  const bool hi = surely_posdef(lmax - a11, -a12, -a13, lmax - a22, -a23, lmax - a33);
  for (int n = 0; n < 6; ++n) out[n] = g[n];
  if (lo & hi) return false;
  double A[3][3] = {{a11, a12, a13}, {a12, a22, a23}, {a13, a23, a33}}, lam[3], V[3][3];
  sym_eigen3(A, lam, V);
  const double S = std::fmax(std::fmax(std::fabs(lam[0]), std::fabs(lam[1])), std::fabs(lam[2]));
  const double s = BOUNDS_SLACK * BEPS * S;
  bool inside = true;
  for (int k = 0; k < 3; ++k) inside = inside & ((lmin - s <= lam[k]) & (lam[k] <= lmax + s));
  if (inside) return false;
  double l2[3];
  for (int k = 0; k < 3; ++k) l2[k] = jclamp(lam[k], lmin, lmax);
  out[0] = recompose(V, l2, 0, 0);
  out[1] = recompose(V, l2, 0, 1);
  out[2] = recompose(V, l2, 0, 2);
  out[3] = recompose(V, l2, 1, 1);
  out[4] = recompose(V, l2, 1, 2);
  out[5] = recompose(V, l2, 2, 2);
  return true;
}

// one application of the five steps; h, Pi updated in place; returns hit, sets nonfinite
static inline bool project_once(double h[10], double Pi[10], const Bounds& bd, bool& nonfinite) {
  const double slack = BOUNDS_SLACK * BEPS;
  // (1) non-finite components take Minkowski's value
  bool fin = true;
  for (int v = 0; v < 10; ++v) fin = fin & std::isfinite(h[v]) & std::isfinite(Pi[v]);
  nonfinite = !fin;
  if (nonfinite)
    for (int v = 0; v < 10; ++v) {
      if (!std::isfinite(h[v])) h[v] = 0.0;
      if (!std::isfinite(Pi[v])) Pi[v] = 0.0;
    }
  double hm[4][4];
  sym4(h, hm);
  const AdmSplit s0 = adm_split(hm);
  // (2) the spectrum of gamma
  double g2[6];
  const bool gfire = spectrum_clamp(s0.g, bd.lambda_min, bd.lambda_max, g2);
  if (gfire) {
    hm[1][1] = g2[0] - 1.0; hm[2][1] = hm[1][2] = g2[1]; hm[3][1] = hm[1][3] = g2[2];
    hm[2][2] = g2[3] - 1.0; hm[3][2] = hm[2][3] = g2[4]; hm[3][3] = g2[5] - 1.0;
  }
  const AdmSplit s1 = gfire ? adm_split(hm) : s0;
  // (3) the shift, with the projected gamma
  const double bmax2 = bd.beta_max * bd.beta_max;
  const bool bfire = !(s1.bb <= bmax2 + slack * bmax2);
  if (bfire) {
    const double f = bd.beta_max / std::sqrt(s1.bb);
    for (int i = 0; i < 3; ++i) hm[i + 1][0] = hm[0][i + 1] = f * s1.beta[i];
  }
  const AdmSplit s2 = bfire ? adm_split(hm) : s1;
  // (4) the lapse, by moving g_tt alone
  const double lo2 = bd.alpha_min * bd.alpha_min, hi2 = bd.alpha_max * bd.alpha_max;
  const double sa = slack * (1.0 + std::fabs(hm[0][0]) + std::fabs(s2.bb));
  const bool alow = !(s2.a2 >= lo2 - sa);
  const bool ahigh = !(s2.a2 <= hi2 + sa);
  const bool afire = alow | ahigh;
  const double at2 = alow ? lo2 : hi2;
  if (afire) hm[0][0] = (1.0 - at2) + s2.bb;
  const AdmSplit s3 = afire ? adm_split(hm) : s2;
  const bool hfire = gfire | bfire | afire;
  // (5) the momentum: rescaled where a positive lapse was raised, then capped
  const bool raise = alow & (s0.a2 > 0.0) & (s0.detg > 0.0) & (s3.a2 > s0.a2);
  if (raise) {
    const double f = (std::sqrt(s0.a2) / std::sqrt(s3.a2)) * (std::sqrt(s3.detg) / std::sqrt(s0.detg));
    for (int v = 0; v < 10; ++v) Pi[v] = Pi[v] * f;
  }
  const double a = std::sqrt(s3.a2) / std::sqrt(s3.detg);
  double m = std::fabs(a * Pi[0]);
  for (int v = 1; v < 10; ++v) {
    const double x = std::fabs(a * Pi[v]);
    m = (x != x || m != m) ? std::numeric_limits<double>::quiet_NaN() : std::fmax(m, x);
  }
  const bool Kfire = !(m <= bd.K_max + slack * bd.K_max);
  if (Kfire) {
    const double f = bd.K_max / m;
    for (int v = 0; v < 10; ++v) Pi[v] = Pi[v] * f;
  }
  if (hfire) pack10(hm, h);
  return nonfinite | hfire | raise | Kfire;
}

// bounds_project: the projection, and where it fired, its result re-tested and re-projected by
// the same arithmetic (at most BOUNDS_PASSES times)
static inline bool bounds_project(double h[10], double Pi[10], const Bounds& bd, bool& nonfinite) {
  const bool hit = project_once(h, Pi, bd, nonfinite);
  if (hit)
    for (int pass = 0; pass < BOUNDS_PASSES; ++pass) {
      double h2[10], P2[10];
      for (int v = 0; v < 10; ++v) {
        h2[v] = h[v];
        P2[v] = Pi[v];
      }
      bool nf2;
      if (!project_once(h2, P2, bd, nf2)) break;
      for (int v = 0; v < 10; ++v) {
        h[v] = h2[v];
        Pi[v] = P2[v];
      }
    }
  return hit;
}

}  // namespace orc
