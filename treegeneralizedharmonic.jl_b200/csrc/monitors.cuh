// The two constraint monitors and their masked norms (src/constraints.jl):
//   gauge_constraint_kernel   gh_constraint_kernel!     src/constraints.jl:211-271
//   adm_constraint_kernel     adm_constraint_kernel!    src/constraints.jl:432-532
//                             adm_constraints_at_node   src/constraints.jl:136-190
//                             metric_derivatives_along  src/pointwise.jl:530-546
//   diag_norms_kernel         diag_norms / SlotNorms    src/constraints.jl:716-778
// They write a diag field set: per block NDIAG slots of (N+1)^3 points, slot-major like the
// state vector. One thread per owned point; a point the mask excludes writes zeros and reads
// nothing, as the reference's kernels do.
#pragma once
#include "rhs.cuh"

namespace tgh {

enum { NDIAG = 10, DG_CGH = 0, DG_HAM = 4, DG_MOM = 5, DG_MASK = 8, DG_TAU = 9 };

struct MonArgs {
  const double* work;    // the filled working array
  const double* Hsrc;    // sampled gauge source (N1^3 x 20 per block), or null
  const double* matter;  // (N1^3 x 10) per block, or null
  const double* blk;
  double* diag;          // NDIAG x N1^3 per block
  int N1, Wd, G, all;    // all: every point is evolved (the trivial mask)
  int Wx;                // the working array's row pitch (kernels.cuh Geo)
  long S, Wv, npts;
  double t;
};

// the owned point p: block, indices, position, the working-array pointer
struct MonPoint {
  int b;
  long ip;
  double x[3], h;
  const double* wk;
};
__device__ __forceinline__ MonPoint mon_point(const MonArgs& A, long p) {
  MonPoint m;
  m.b = (int)(p / A.S);
  m.ip = p - (long)m.b * A.S;
  const int k = (int)(m.ip / ((long)A.N1 * A.N1)), j = (int)((m.ip / A.N1) % A.N1), i = (int)(m.ip % A.N1);
  const double* bl = A.blk + 8 * m.b;
  m.h = bl[3];
  m.x[0] = __dadd_rn(bl[0], __dmul_rn(bl[4] + (double)i, m.h));
  m.x[1] = __dadd_rn(bl[1], __dmul_rn(bl[5] + (double)j, m.h));
  m.x[2] = __dadd_rn(bl[2], __dmul_rn(bl[6] + (double)k, m.h));
  m.wk = A.work + (long)m.b * NV * A.Wv + (i + A.G) + (long)A.Wx * ((j + A.G) + (long)A.Wd * (k + A.G));
  return m;
}

// The lowered gauge source and its gradient at a point (gauge_source, src/gauge.jl:156-212):
// zero, sampled (rows H_a, then d_c H_a at 4 + c + 4a), or the closed Kerr-Schild form, which
// reads d_t g (D[0], here without the dissipation) and the spatial gradients.
__device__ __forceinline__ void mon_gauge(const Case& cs, const MonArgs& A, const MonPoint& m, const double* hv,
                                          const double* const D[4], double Hl[4], double dHl[4][4]) {
  if (cs.gauge == TGH_GAUGE_NONE) {
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      Hl[a] = 0.0;
#pragma unroll
      for (int c = 0; c < 4; ++c) dHl[c][a] = 0.0;
    }
  } else if (cs.gauge == TGH_GAUGE_SAMPLED) {
    const double* q = A.Hsrc + (long)m.b * NV * A.S + m.ip;
#pragma unroll
    for (int a = 0; a < 4; ++a) Hl[a] = q[a * A.S];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int c = 0; c < 4; ++c) dHl[c][a] = q[(4 + c + 4 * a) * A.S];
  } else {
    ks_gauge_source<double>(cs, hv, D, Hl, dHl);
  }
}

// C_a = g_ab (Gamma^b + H^b) = g^{bc} Gamma_{a,bc} + H_a at one owned point, with d_t g from
// the first evolution equation without the dissipation. The reference raises with g^{-1} and
// lowers again; the lowered contraction V_a = g^{bc} d_b g_ac - g^{bc} d_a g_bc / 2 is the same
// number up to roundoff, and exactly zero on flat data.
template <int Q>
__global__ void __launch_bounds__(128) gauge_constraint_kernel(const Case cs, const MonArgs A) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= A.npts) return;
  const MonPoint m = mon_point(A, p);
  double* dg = A.diag + (long)m.b * NDIAG * A.S + m.ip;
  if (!A.all && !evolved(cs, A.t, m.x)) {
#pragma unroll
    for (int a = 0; a < 4; ++a) dg[(DG_CGH + a) * A.S] = 0.0;
    dg[DG_MASK * A.S] = 0.0;
    return;
  }
  const long s[3] = {1, A.Wx, (long)A.Wx * A.Wd};
  const double ih = 1.0 / m.h;
  double hv[NC], dth[NC], dh[3][NC];
#pragma unroll
  for (int v = 0; v < NC; ++v) {
    const double* pv = m.wk + v * A.Wv;
    hv[v] = pv[0];
#pragma unroll
    for (int d = 0; d < 3; ++d) dh[d][v] = ih * st_d1<Q, double>(pv, s[d]);
  }
  Coef<double> C;
  metric_quantities(hv, C);
  const double a_div = C.alpha / C.sqrtg;
#pragma unroll
  for (int v = 0; v < NC; ++v)
    dth[v] = C.beta[0] * dh[0][v] + C.beta[1] * dh[1][v] + C.beta[2] * dh[2][v] + a_div * m.wk[(NC + v) * A.Wv];
  const double* D[4] = {dth, dh[0], dh[1], dh[2]};
  double Hl[4], dHl[4][4];
  mon_gauge(cs, A, m, hv, D, Hl, dHl);
#pragma unroll
  for (int x = 0; x < 4; ++x) {
    double sv = 0.0, tr = 0.0;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) sv = fma(C.gu[pidx(a, b)], D[a][pidx(x, b)], sv);
#pragma unroll
    for (int n = 0; n < NC; ++n) tr = fma(prow(n) == pcol(n) ? C.gu[n] : 2.0 * C.gu[n], D[x][n], tr);
    dg[(DG_CGH + x) * A.S] = fma(-0.5, tr, sv) + Hl[x];
  }
  dg[DG_MASK * A.S] = 1.0;
}

// d alpha, d beta^j and d sqrt(gamma) along one direction whose d g is dgl (packed), the
// closed forms of metric_derivatives_along (src/pointwise.jl:530-546)
__device__ __forceinline__ void mon_along(const Coef<double>& C, const double* dgl, double& dal, double db[3],
                                          double& dsq) {
  double dgu[NC];  // -g^{-1} (d g) g^{-1}
#pragma unroll
  for (int n = 0; n < NC; ++n) {
    const int a = prow(n), b = pcol(n);
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      double r = 0.0;
#pragma unroll
      for (int d = 0; d < 4; ++d) r = fma(dgl[pidx(c, d)], C.gu[pidx(d, b)], r);
      s = fma(C.gu[pidx(a, c)], r, s);
    }
    dgu[n] = -s;
  }
  dal = C.alpha * C.alpha * C.alpha * dgu[0] * 0.5;
#pragma unroll
  for (int j = 0; j < 3; ++j) db[j] = -(dgu[pidx(0, j + 1)] + C.beta[j] * dgu[0]) / C.gu[0];
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int k = 0; k < 3; ++k) s = fma(C.gamu[sidx3(j, k)], dgl[pidx(j + 1, k + 1)], s);
  dsq = C.sqrtg * s * 0.5;
}

// The first-derivative terms of the four-dimensional Ricci tensor, R_ab for the packed a <= b:
//   (d_c g^{cd}) Gamma_{d,ab} - (d_b g^{cd}) Gamma_{d,ca} + Gamma^c_cd Gamma^d_ab - Gamma^c_bd Gamma^d_ca
// with d g^{-1} = -g^{-1} (d g) g^{-1} folded into the contractions: per b, U = g^{-1} d_b g
// (16 values); the first term is -w_f Gamma^f_ab with w_f = sum_c U_c[c][f]. R_ab is symmetric
// as a whole (not term by term), so each packed entry is formed once, with b its larger index.
__device__ __forceinline__ void ricci_first_order(const Coef<double>& C, const double* const D[4], double R[NC]) {
  double G4[4][NC];  // Gamma^a_bc
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int n = 0; n < NC; ++n) {
      const int b = prow(n), c = pcol(n);
      double s = 0.0;
#pragma unroll
      for (int x = 0; x < 4; ++x) s = fma(C.gu[pidx(a, x)], 0.5 * (D[b][pidx(x, c)] + D[c][pidx(x, b)] - D[x][n]), s);
      G4[a][n] = s;
    }
  double w[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    double U[4][4];  // U[c][f] = g^{ce} d_b g_ef
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        double s = 0.0;
#pragma unroll
        for (int e = 0; e < 4; ++e) s = fma(C.gu[pidx(c, e)], D[b][pidx(e, f)], s);
        U[c][f] = s;
      }
#pragma unroll
    for (int f = 0; f < 4; ++f) w[f] += U[b][f];
#pragma unroll
    for (int a = 0; a <= b; ++a) {
      double r = 0.0;
#pragma unroll
      for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int f = 0; f < 4; ++f) r = fma(U[c][f], G4[f][pidx(c, a)], r);
#pragma unroll
      for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int d = 0; d < 4; ++d) r = fma(-G4[c][pidx(b, d)], G4[d][pidx(c, a)], r);
      R[pidx(a, b)] = r;
    }
  }
  double tw[4];  // Gamma^c_cf - w_f
#pragma unroll
  for (int f = 0; f < 4; ++f)
    tw[f] = G4[0][pidx(0, f)] + G4[1][pidx(1, f)] + G4[2][pidx(2, f)] + G4[3][pidx(3, f)] - w[f];
#pragma unroll
  for (int n = 0; n < NC; ++n)
#pragma unroll
    for (int f = 0; f < 4; ++f) R[n] = fma(tw[f], G4[f][n], R[n]);
}

// The second-derivative terms of R_ab from the ten second derivatives dv[m] = d_mu d_nu g_v
// (m the packed (mu nu)) of one metric component v = (al be), added to the packed R:
//   R_ab += X_ab + X_ba - (1/2) g^{cd} d_c d_d g_ab - (1/2) g^{cd} d_a d_b g_cd,
//   X_ab = (1/2) g^{cd} d_c d_a g_db,
// the terms -(1/2) g^{cd} (d_c d_b g_da - d_b d_c g_da) of the full expansion cancelling.
template <int V>
__device__ __forceinline__ void ricci_second_order(const Coef<double>& C, const double dv[NC], double R[NC]) {
  constexpr int al = prow(V), be = pcol(V);
  const double c3 = (al == be ? -0.5 : -1.0) * C.gu[V];
  double tr = 0.0;
#pragma unroll
  for (int m = 0; m < NC; ++m) {
    R[m] = fma(c3, dv[m], R[m]);
    tr = fma(prow(m) == pcol(m) ? C.gu[m] : 2.0 * C.gu[m], dv[m], tr);
  }
  R[V] = fma(-0.5, tr, R[V]);
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    double y = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c) y = fma(C.gu[pidx(c, al)], dv[pidx(c, a)], y);
    R[pidx(a, be)] = fma(a == be ? 1.0 : 0.5, y, R[pidx(a, be)]);
    if (al != be) {
      double z = 0.0;
#pragma unroll
      for (int c = 0; c < 4; ++c) z = fma(C.gu[pidx(c, be)], dv[pidx(c, a)], z);
      R[pidx(a, al)] = fma(a == al ? 1.0 : 0.5, z, R[pidx(a, al)]);
    }
  }
}

// What the ten second derivatives of one component need besides its own stencils: the
// metric, the shift's and lapse's derivatives along x_i (i = 0..2) and t (3), the divergences
// and the d_t Pi terms that carry no second derivative.
struct AdmPoint {
  Coef<double> C;
  double phi, am, divb, divA[3];
  double dphi[4], db[4][3];
  const double* wk;
  long Wv, s[3];
  double ih, ih2;
};

// Component V's second derivatives d_mu d_nu g_V in packed (mu nu) order: the six spatial ones
// from the stencils; d_t d_i g and d_t d_t g from the first evolution equation differentiated
// once and twice, with d_t Pi_V from the reduced equation (src + the principal part).
template <int Q, int V>
__device__ __forceinline__ void adm_component(const AdmPoint& P, double src, double dv[NC]) {
  const double* ph = P.wk + V * P.Wv;
  const double* pp = ph + NC * P.Wv;
  const double hc = ph[0], pc = pp[0];
  // the component's first derivatives are formed again here (the same stencils) rather than
  // held for all ten components
  double dh[3], dP[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    dh[d] = P.ih * st_d1<Q, double>(ph, P.s[d]);
    dP[d] = P.ih * st_d1<Q, double>(pp, P.s[d]);
  }
  dv[4] = P.ih2 * st_d2<Q, double>(ph, P.s[0], hc);
  dv[5] = P.ih2 * st_mixed<Q, double>(ph, P.s[0], P.s[1]);
  dv[6] = P.ih2 * st_mixed<Q, double>(ph, P.s[0], P.s[2]);
  dv[7] = P.ih2 * st_d2<Q, double>(ph, P.s[1], hc);
  dv[8] = P.ih2 * st_mixed<Q, double>(ph, P.s[1], P.s[2]);
  dv[9] = P.ih2 * st_d2<Q, double>(ph, P.s[2], hc);
  const Coef<double>& C = P.C;
  double t0 = C.beta[0] * dP[0] + C.beta[1] * dP[1] + C.beta[2] * dP[2] + P.divb * pc;
  t0 += P.am * (C.gamu[0] * dv[4] + 2.0 * C.gamu[1] * dv[5] + 2.0 * C.gamu[2] * dv[6] + C.gamu[3] * dv[7] +
                2.0 * C.gamu[4] * dv[8] + C.gamu[5] * dv[9]);
  t0 += P.divA[0] * dh[0] + P.divA[1] * dh[1] + P.divA[2] * dh[2];
  const double dtP = src + t0;
#pragma unroll
  for (int i = 0; i < 3; ++i)
    dv[1 + i] = P.dphi[i] * pc + P.phi * dP[i] +
                (P.db[i][0] * dh[0] + P.db[i][1] * dh[1] + P.db[i][2] * dh[2]) +
                (C.beta[0] * dv[pidx(i + 1, 1)] + C.beta[1] * dv[pidx(i + 1, 2)] + C.beta[2] * dv[pidx(i + 1, 3)]);
  dv[0] = P.dphi[3] * pc + P.phi * dtP + (P.db[3][0] * dh[0] + P.db[3][1] * dh[1] + P.db[3][2] * dh[2]) +
          (C.beta[0] * dv[1] + C.beta[1] * dv[2] + C.beta[2] * dv[3]);
}

template <int Q, int V>
__device__ __forceinline__ void adm_components(const AdmPoint& P, const double src[NC], double R[NC]) {
  if constexpr (V < NC) {
    double dv[NC];
    adm_component<Q, V>(P, src[V], dv);
    ricci_second_order<V>(P.C, dv, R);
    adm_components<Q, V + 1>(P, src, R);
  }
}

// The ADM Hamiltonian and momentum constraints at one owned point: the four-dimensional Ricci
// tensor
//   R_ab = d_c Gamma^c_ab - d_b Gamma^c_ca + Gamma^c_cd Gamma^d_ab - Gamma^c_bd Gamma^d_ca
// from every second derivative of g (the spatial ones from the right-hand side's stencils,
// d_t d_i g and d_t d_t g from the first evolution equation differentiated once and twice, with
// d_t Pi from the reduced equation, source and damping included, no dissipation), then
// H = 2 R_nn + R, M_i = -n^a (R_ai - g_ai R / 2), n = (1, -beta) / alpha. With matter, H - 16 pi
// rho and M_i - 8 pi S_i. The first-derivative terms are formed first; the hundred second
// derivatives are then formed component by component and folded into the ten packed R_ab at
// once, so that no more than ten of them are held (the reference's kernel holds them all).
template <int Q>
__global__ void __launch_bounds__(128) adm_constraint_kernel(const Case cs, const MonArgs A) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= A.npts) return;
  const MonPoint m = mon_point(A, p);
  double* dgo = A.diag + (long)m.b * NDIAG * A.S + m.ip;
  if (!A.all && !evolved(cs, A.t, m.x)) {
    dgo[DG_HAM * A.S] = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) dgo[(DG_MOM + a) * A.S] = 0.0;
    dgo[DG_MASK * A.S] = 0.0;
    return;
  }
  AdmPoint P;
  P.wk = m.wk;
  P.Wv = A.Wv;
  P.s[0] = 1;
  P.s[1] = A.Wx;
  P.s[2] = (long)A.Wx * A.Wd;
  P.ih = 1.0 / m.h;
  P.ih2 = P.ih * P.ih;
  double hv[NC], dh[3][NC];
#pragma unroll
  for (int v = 0; v < NC; ++v) {
    const double* ph = m.wk + v * A.Wv;
    hv[v] = ph[0];
#pragma unroll
    for (int d = 0; d < 3; ++d) dh[d][v] = P.ih * st_d1<Q, double>(ph, P.s[d]);
  }
  metric_quantities(hv, P.C);
  const Coef<double>& C = P.C;
  P.phi = C.alpha / C.sqrtg;
  P.am = C.alpha * C.sqrtg;
  double R[NC], src[NC];
  {
    double dth[NC];
#pragma unroll
    for (int v = 0; v < NC; ++v)
      dth[v] = C.beta[0] * dh[0][v] + C.beta[1] * dh[1][v] + C.beta[2] * dh[2][v] + P.phi * m.wk[(NC + v) * A.Wv];
    const double* D[4] = {dth, dh[0], dh[1], dh[2]};
    // d_t Pi without its second-derivative terms: gh_node_rhs_expanded (src/pointwise.jl:818-850)
    // without the dissipation, the source and damping first
    {
      double Hl[4], dHl[4][4], dHs[NC];
      mon_gauge(cs, A, m, hv, D, Hl, dHl);
#pragma unroll
      for (int n = 0; n < NC; ++n) dHs[n] = dHl[prow(n)][pcol(n)] + dHl[pcol(n)][prow(n)];
      gh_source<double, true>(C, D, Hl, dHs, damping_rate(cs, A.t, m.x), cs.g2, src);
    }
    // d alpha, d beta, d sqrt(gamma) along x_i and t
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      double dal, dsq;
      mon_along(C, i < 3 ? dh[i] : dth, dal, P.db[i], dsq);
      P.dphi[i] = (dal - P.phi * dsq) / C.sqrtg;
    }
    const double* dhp[3] = {dh[0], dh[1], dh[2]};
    metric_divergences(C, dhp, P.divb, P.divA);
    ricci_first_order(C, D, R);
  }
  double rho = 0.0, Sm[3] = {0.0, 0.0, 0.0};
  if (A.matter) {
    const double* q = A.matter + (long)m.b * NC * A.S + m.ip;
    double mm[NC], ms[NC];
#pragma unroll
    for (int n = 0; n < NC; ++n) mm[n] = q[n * A.S];
    matter_source<double>(C, mm, ms);
#pragma unroll
    for (int v = 0; v < NC; ++v) src[v] += ms[v];
    rho = mm[0];
    Sm[0] = mm[1];
    Sm[1] = mm[2];
    Sm[2] = mm[3];
  }
  adm_components<Q, 0>(P, src, R);
  double Rs = 0.0;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) Rs = fma(C.gu[pidx(a, b)], R[pidx(a, b)], Rs);
  const double nv[4] = {1.0 / C.alpha, -C.beta[0] / C.alpha, -C.beta[1] / C.alpha, -C.beta[2] / C.alpha};
  double Rnn = 0.0;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) Rnn = fma(R[pidx(a, b)] * nv[a], nv[b], Rnn);
  double ham = 2.0 * Rnn + Rs;
  double mom[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double sm = 0.0;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      // g_a(i+1) = eta + h, read again
      const double g = m.wk[pidx(a, i + 1) * A.Wv] + (a == i + 1 ? 1.0 : 0.0);
      sm = fma(nv[a], R[pidx(a, i + 1)] - g * Rs * 0.5, sm);
    }
    mom[i] = -sm;
  }
  if (A.matter) {
    const double c8 = 8.0 * 3.14159265358979323846;
    ham -= 2.0 * (c8 * rho);
#pragma unroll
    for (int i = 0; i < 3; ++i) mom[i] -= c8 * Sm[i];
  }
  dgo[DG_HAM * A.S] = ham;
#pragma unroll
  for (int i = 0; i < 3; ++i) dgo[(DG_MOM + i) * A.S] = mom[i];
  dgo[DG_MASK * A.S] = 1.0;
}

// a maximum that keeps NaN (Julia's max), so that a blown-up run shows in the L-infinity norm
__device__ __forceinline__ double nan_max(double a, double b) { return (a != a || b != b) ? __longlong_as_double(0x7ff8000000000000LL) : fmax(a, b); }

// One fold of the slots C_a .. mask over the primary copies (each lattice point once): per
// CTA the evolved volume (mask x weight), per slot the sum of squares x weight and the largest
// magnitude; weight h^3 (volume) or 1 (points); with hsel > 0 only the blocks of spacing hsel
// (one refinement level: every spacing is h0 2^-l, exactly).
// part: 17 rows (volume, 8 sums, 8 maxima) of one value per CTA, folded in a fixed order.
static __global__ void __launch_bounds__(128) diag_norms_kernel(const double* __restrict__ diag,
                                                                const uint8_t* __restrict__ primary,
                                                                const double* __restrict__ blk, long S, long npts,
                                                                int volume, double hsel, double* part) {
  __shared__ double sh[17][128];
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double c[17];
#pragma unroll
  for (int n = 0; n < 17; ++n) c[n] = 0.0;
  if (p < npts && primary[p]) {
    const int b = (int)(p / S);
    const double h = blk[8 * b + 3];
    if (!(hsel > 0.0) || h == hsel) {
      const long ip = p - (long)b * S;
      const double w = volume ? h * h * h : 1.0;
      const double* q = diag + (long)b * NDIAG * S + ip;
      c[0] = q[DG_MASK * S] * w;
#pragma unroll
      for (int s = 0; s < 8; ++s) {
        const double u = q[s * S];
        c[1 + s] = u * u * w;
        c[9 + s] = fabs(u);
      }
    }
  }
#pragma unroll
  for (int n = 0; n < 17; ++n) sh[n][threadIdx.x] = c[n];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
#pragma unroll
      for (int n = 0; n < 9; ++n) sh[n][threadIdx.x] += sh[n][threadIdx.x + o];
#pragma unroll
      for (int n = 9; n < 17; ++n) sh[n][threadIdx.x] = nan_max(sh[n][threadIdx.x], sh[n][threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x < 17) part[(long)threadIdx.x * gridDim.x + blockIdx.x] = sh[threadIdx.x][0];
}

// the CTA partials folded, one CTA per quantity: each thread a strided run, then a tree, in the
// same order every time (deterministic)
static __global__ void __launch_bounds__(256) diag_norms_fold_kernel(const double* __restrict__ part, int npart,
                                                                     double* out) {
  __shared__ double sh[256];
  const int n = blockIdx.x;
  const bool sum = n < 9;
  const double* q = part + (long)n * npart;
  double acc = 0.0;
  for (int c = threadIdx.x; c < npart; c += 256) acc = sum ? acc + q[c] : nan_max(acc, q[c]);
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] = sum ? sh[threadIdx.x] + sh[threadIdx.x + o] : nan_max(sh[threadIdx.x], sh[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[n] = sh[0];
}

// ---- the masked Loehner indicator (src/refinement.jl:170-400) ----
// A non-negative double's bit pattern orders as the double does (and a positive NaN above +inf),
// so integer atomics give an order-independent maximum that keeps NaN.
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* a, double v) {
  atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

// field_scales: the largest |h_v| over the evolved owned points, per component (the
// reference amplitude of the indicator's noise floor); out[v] as bit patterns, zeroed before
static __global__ void __launch_bounds__(128) field_scales_kernel(const MonArgs A, const Case cs,
                                                                  unsigned long long* out) {
  __shared__ unsigned long long sh[NC];
  if (threadIdx.x < NC) sh[threadIdx.x] = 0ull;
  __syncthreads();
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < A.npts) {
    const MonPoint m = mon_point(A, p);
    if (A.all || evolved(cs, A.t, m.x)) {
#pragma unroll
      for (int v = 0; v < NC; ++v) atomicMax(&sh[v], (unsigned long long)__double_as_longlong(fabs(m.wk[v * A.Wv])));
    }
  }
  __syncthreads();
  if (threadIdx.x < NC) atomicMax(&out[threadIdx.x], sh[threadIdx.x]);
}

// lohner: |u+ - 2 u0 + u-| / (|u+ - u0| + |u0 - u-| + 4 eps scale), 0 where the denominator
// is; every operation rounded on its own, in the reference's order
__device__ __forceinline__ double lohner(double um, double u0, double up, double floor4) {
  const double num = fabs(__dadd_rn(__dsub_rn(up, __dmul_rn(2.0, u0)), um));
  const double den = __dadd_rn(__dadd_rn(fabs(__dsub_rn(up, u0)), fabs(__dsub_rn(u0, um))), floor4);
  return den == 0.0 ? 0.0 : __ddiv_rn(num, den);
}

// gh_tau_kernel!: tau at every owned point into the diag slot DG_TAU, the worst lohner over the
// ten components of h and the three axes, zero where the mask leaves the point out (asked
// before any value is read); its maximum over the mesh into *tmax (bit pattern)
static __global__ void __launch_bounds__(128) tau_kernel(const MonArgs A, const Case cs, double floor4,
                                                         unsigned long long* tmax) {
  __shared__ unsigned long long sh;
  if (threadIdx.x == 0) sh = 0ull;
  __syncthreads();
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < A.npts) {
    const MonPoint m = mon_point(A, p);
    double tau = 0.0;
    if (A.all || evolved(cs, A.t, m.x)) {
      const long s[3] = {1, A.Wx, (long)A.Wx * A.Wd};
#pragma unroll
      for (int v = 0; v < NC; ++v) {
        const double* q = m.wk + v * A.Wv;
        const double u0 = q[0];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const double t = lohner(q[-s[d]], u0, q[s[d]], floor4);
          tau = (t != t || tau != tau) ? __longlong_as_double(0x7ff8000000000000LL) : fmax(tau, t);
        }
      }
    }
    A.diag[(long)m.b * NDIAG * A.S + DG_TAU * A.S + m.ip] = tau;
    atomicMax(&sh, (unsigned long long)__double_as_longlong(tau));
  }
  __syncthreads();
  if (threadIdx.x == 0) atomicMax(tmax, sh);
}

// firing_boxes over the diag slot DG_TAU, for ntol thresholds at once: per block and threshold
// the number of owned points with tau > tol and the bounding box of their node indices.
// counts: nb x ntol (zeroed before); boxes: nb x ntol x 6 (lo i, j, k set to N1, hi to -1 before)
static __global__ void __launch_bounds__(128) firing_kernel(const MonArgs A, int ntol, const double* __restrict__ tol,
                                                            int* counts, int* boxes) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= A.npts) return;
  const int b = (int)(p / A.S);
  const long ip = p - (long)b * A.S;
  const int ijk[3] = {(int)(ip % A.N1), (int)((ip / A.N1) % A.N1), (int)(ip / ((long)A.N1 * A.N1))};
  const double tau = A.diag[(long)b * NDIAG * A.S + DG_TAU * A.S + ip];
  for (int n = 0; n < ntol; ++n) {
    if (!(tau > tol[n])) continue;
    const long o = (long)b * ntol + n;
    atomicAdd(&counts[o], 1);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      atomicMin(&boxes[6 * o + d], ijk[d]);
      atomicMax(&boxes[6 * o + 3 + d], ijk[d]);
    }
  }
}

static __global__ void firing_init_kernel(int n, int N1, int* counts, int* boxes) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= n) return;
  counts[id] = 0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    boxes[6 * id + d] = N1;
    boxes[6 * id + 3 + d] = -1;
  }
}

cudaError_t launch_gauge_constraint(int q, cudaStream_t s, const Case& cs, const MonArgs& a);
cudaError_t launch_adm_constraint(int q, cudaStream_t s, const Case& cs, const MonArgs& a);

}  // namespace tgh
