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
  m.wk = A.work + (long)m.b * NV * A.Wv + (i + A.G) + (long)A.Wd * ((j + A.G) + (long)A.Wd * (k + A.G));
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
  const long s[3] = {1, A.Wd, (long)A.Wd * A.Wd};
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

// The ADM Hamiltonian and momentum constraints at one owned point: every second derivative of
// g (the spatial ones from the right-hand side's stencils, d_t d_i g and d_t d_t g from the
// first evolution equation differentiated once and twice, with d_t Pi from the reduced equation,
// source and damping included, no dissipation), then the four-dimensional Ricci tensor
//   R_ab = d_c Gamma^c_ab - d_b Gamma^c_ca + Gamma^c_cd Gamma^d_ab - Gamma^c_bd Gamma^d_ca
// and H = 2 R_nn + R, M_i = -n^a (R_ai - g_ai R / 2), n = (1, -beta) / alpha. With matter, H - 16 pi
// rho and M_i - 8 pi S_i. A diagnostic: it holds the hundred second derivatives at once and
// spills, which is the reference's trade as well.
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
  const long s[3] = {1, A.Wd, (long)A.Wd * A.Wd};
  const double ih = 1.0 / m.h, ih2 = ih * ih;
  double hv[NC], Pv[NC], dh[3][NC], dP[3][NC], dd[NC][NC];  // dd[(mu nu)][(ab)] = d_mu d_nu g_ab
#pragma unroll
  for (int v = 0; v < NC; ++v) {
    const double* ph = m.wk + v * A.Wv;
    const double* pp = ph + NC * A.Wv;
    hv[v] = ph[0];
    Pv[v] = pp[0];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      dh[d][v] = ih * st_d1<Q, double>(ph, s[d]);
      dP[d][v] = ih * st_d1<Q, double>(pp, s[d]);
    }
    dd[4][v] = ih2 * st_d2<Q, double>(ph, s[0], hv[v]);
    dd[5][v] = ih2 * st_mixed<Q, double>(ph, s[0], s[1]);
    dd[6][v] = ih2 * st_mixed<Q, double>(ph, s[0], s[2]);
    dd[7][v] = ih2 * st_d2<Q, double>(ph, s[1], hv[v]);
    dd[8][v] = ih2 * st_mixed<Q, double>(ph, s[1], s[2]);
    dd[9][v] = ih2 * st_d2<Q, double>(ph, s[2], hv[v]);
  }
  Coef<double> C;
  metric_quantities(hv, C);
  const double phi = C.alpha / C.sqrtg;
  double dth[NC];
#pragma unroll
  for (int v = 0; v < NC; ++v)
    dth[v] = C.beta[0] * dh[0][v] + C.beta[1] * dh[1][v] + C.beta[2] * dh[2][v] + phi * Pv[v];
  const double* D[4] = {dth, dh[0], dh[1], dh[2]};
  // d_t Pi: gh_node_rhs_expanded (src/pointwise.jl:818-850) without the dissipation
  double dtP[NC];
  {
    double Hl[4], dHl[4][4], dHs[NC];
    mon_gauge(cs, A, m, hv, D, Hl, dHl);
#pragma unroll
    for (int n = 0; n < NC; ++n) dHs[n] = dHl[prow(n)][pcol(n)] + dHl[pcol(n)][prow(n)];
    gh_source<double, true>(C, D, Hl, dHs, damping_rate(cs, A.t, m.x), cs.g2, dtP);
    const double* dhp[3] = {dh[0], dh[1], dh[2]};
    double divb, divA[3];
    metric_divergences(C, dhp, divb, divA);
    const double am = C.alpha * C.sqrtg;
#pragma unroll
    for (int v = 0; v < NC; ++v) {
      double t0 = C.beta[0] * dP[0][v] + C.beta[1] * dP[1][v] + C.beta[2] * dP[2][v] + divb * Pv[v];
      t0 += am * (C.gamu[0] * dd[4][v] + 2.0 * C.gamu[1] * dd[5][v] + 2.0 * C.gamu[2] * dd[6][v] +
                  C.gamu[3] * dd[7][v] + 2.0 * C.gamu[4] * dd[8][v] + C.gamu[5] * dd[9][v]);
      t0 += divA[0] * dh[0][v] + divA[1] * dh[1][v] + divA[2] * dh[2][v];
      dtP[v] += t0;
    }
  }
  double rho = 0.0, Sm[3] = {0.0, 0.0, 0.0};
  if (A.matter) {
    const double* q = A.matter + (long)m.b * NC * A.S + m.ip;
    double mm[NC], ms[NC];
#pragma unroll
    for (int n = 0; n < NC; ++n) mm[n] = q[n * A.S];
    matter_source<double>(C, mm, ms);
#pragma unroll
    for (int v = 0; v < NC; ++v) dtP[v] += ms[v];
    rho = mm[0];
    Sm[0] = mm[1];
    Sm[1] = mm[2];
    Sm[2] = mm[3];
  }
  // d_t d_i g (slots tx, ty, tz) and d_t d_t g (slot tt)
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double dal, db[3], dsq;
    mon_along(C, dh[i], dal, db, dsq);
    const double dphi = (dal - phi * dsq) / C.sqrtg;
#pragma unroll
    for (int v = 0; v < NC; ++v)
      dd[1 + i][v] = dphi * Pv[v] + phi * dP[i][v] + (db[0] * dh[0][v] + db[1] * dh[1][v] + db[2] * dh[2][v]) +
                     (C.beta[0] * dd[pidx(i + 1, 1)][v] + C.beta[1] * dd[pidx(i + 1, 2)][v] +
                      C.beta[2] * dd[pidx(i + 1, 3)][v]);
  }
  {
    double dal, db[3], dsq;
    mon_along(C, dth, dal, db, dsq);
    const double dphi = (dal - phi * dsq) / C.sqrtg;
#pragma unroll
    for (int v = 0; v < NC; ++v)
      dd[0][v] = dphi * Pv[v] + phi * dtP[v] + (db[0] * dh[0][v] + db[1] * dh[1][v] + db[2] * dh[2][v]) +
                 (C.beta[0] * dd[1][v] + C.beta[1] * dd[2][v] + C.beta[2] * dd[3][v]);
  }
  // the Ricci assembly (adm_constraints_at_node), dg[e][(ab)] = D[e][(ab)]
  double dgu[4][NC], Gl[4][NC], G4[4][NC], Gtr[4];
#pragma unroll
  for (int e = 0; e < 4; ++e)
#pragma unroll
    for (int n = 0; n < NC; ++n) {
      const int a = prow(n), b = pcol(n);
      double sa = 0.0;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        double r = 0.0;
#pragma unroll
        for (int d = 0; d < 4; ++d) r = fma(D[e][pidx(c, d)], C.gu[pidx(d, b)], r);
        sa = fma(C.gu[pidx(a, c)], r, sa);
      }
      dgu[e][n] = -sa;
    }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int n = 0; n < NC; ++n) {
      const int b = prow(n), c = pcol(n);
      Gl[a][n] = 0.5 * (D[b][pidx(a, c)] + D[c][pidx(a, b)] - D[a][n]);
    }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int n = 0; n < NC; ++n) {
      double sa = 0.0;
#pragma unroll
      for (int x = 0; x < 4; ++x) sa = fma(C.gu[pidx(a, x)], Gl[x][n], sa);
      G4[a][n] = sa;
    }
#pragma unroll
  for (int d = 0; d < 4; ++d) Gtr[d] = G4[0][pidx(0, d)] + G4[1][pidx(1, d)] + G4[2][pidx(2, d)] + G4[3][pidx(3, d)];
  double R[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      double r = 0.0;
#pragma unroll
      for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int d = 0; d < 4; ++d) {
          const double gcd = C.gu[pidx(c, d)];
          // d_c Gamma^c_ab
          r = fma(dgu[c][pidx(c, d)], Gl[d][pidx(a, b)], r);
          r = fma(0.5 * gcd, dd[pidx(c, a)][pidx(d, b)] + dd[pidx(c, b)][pidx(d, a)] - dd[pidx(c, d)][pidx(a, b)], r);
          // - d_b Gamma^c_ca
          r = fma(-dgu[b][pidx(c, d)], Gl[d][pidx(c, a)], r);
          r = fma(-0.5 * gcd, dd[pidx(b, c)][pidx(d, a)] + dd[pidx(b, a)][pidx(d, c)] - dd[pidx(b, d)][pidx(c, a)], r);
          // - Gamma^c_bd Gamma^d_ca
          r = fma(-G4[c][pidx(b, d)], G4[d][pidx(c, a)], r);
        }
#pragma unroll
      for (int d = 0; d < 4; ++d) r = fma(Gtr[d], G4[d][pidx(a, b)], r);
      R[a][b] = r;
    }
  double Rs = 0.0;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) Rs = fma(C.gu[pidx(a, b)], R[a][b], Rs);
  const double nv[4] = {1.0 / C.alpha, -C.beta[0] / C.alpha, -C.beta[1] / C.alpha, -C.beta[2] / C.alpha};
  double Rnn = 0.0;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) Rnn = fma(R[a][b] * nv[a], nv[b], Rnn);
  double ham = 2.0 * Rnn + Rs;
  double mom[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double sm = 0.0;
#pragma unroll
    for (int a = 0; a < 4; ++a) sm = fma(nv[a], R[a][i + 1] - C.g[pidx(a, i + 1)] * Rs * 0.5, sm);
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
      const long s[3] = {1, A.Wd, (long)A.Wd * A.Wd};
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
