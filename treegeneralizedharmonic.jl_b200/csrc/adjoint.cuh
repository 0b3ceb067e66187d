// The adjoint (reverse mode) of the plain form's right-hand side gh_rhs! = prepare!; rhs!
// (src/evolution.jl:1327-1390): given a cotangent lambda of du, the cotangent of the state u,
// (d du / d u)^T lambda, and of the layer's and damping's parameters, lambda . d du / d theta.
//
// At an owned point p the right-hand side is a function of a few stencil features of the
// ghosted working array - per component v the values h_v, Pi_v, the first derivatives of h_v
// and Pi_v, the second and mixed derivatives of h_v, and the two dissipation sums - combined
// with coefficients that depend on h and its first derivatives (the metric, lapse, shift, the
// divergences and the source). With Phi = sum_v lambda_v du_v(p):
//   * the features that enter linearly (the derivatives of Pi, the second derivatives of h, the
//     dissipation of Pi) get their cotangents in closed form, coefficient x lambda;
//   * the 50 nonlinear inputs - h (10), its first derivatives (30) and d_t h (10) - get theirs
//     from 50 forward-mode passes of Phi in value-plus-derivative arithmetic (Tan), each seeding
//     one input; d_t h's cotangent is passed on to Pi, the dissipation of h and, through the
//     passes that seed h and its derivatives, the shift and lapse;
//   * three more passes seed the parameters (rho_max, the ramp width, the damping strength).
// adjoint_gather_kernel then applies the transposed stencils: every point of the working array,
// ghosts included, collects from the owned points whose stencils read it. The fill's transpose
// follows (prolongation level by level from the finest, then the copies into the primary
// state entries; the Dirichlet data do not depend on u and drop out).
//
// 16 feature cotangents per component and point are kept, each feature a field in the padded
// working layout (zero away from the owned points).
#pragma once
#include "kernels.cuh"
#include "tangent_rhs.cuh"

namespace tgh {

constexpr int ADJ_NF = 16;
// per component: h value, dh (x,y,z), d2h (xx,yy,zz), mixed (xy,xz,yz), KO(h); Pi value, dPi (x,y,z), KO(Pi)
enum { AF_HC = 0, AF_HD1 = 1, AF_HD2 = 4, AF_HMX = 7, AF_HKO = 10, AF_PC = 11, AF_PD1 = 12, AF_PKO = 15 };
constexpr int ADJ_PASSES = 53;  // h (10), dh (30), d_t h (10), rho_max, ramp, damping

struct AdjArgs {
  const double* lam;  // the cotangent of du, state layout
  double* cot;        // NC x ADJ_NF feature fields, cstride doubles each (padded working layout of one variable)
  long cstride;
  double* part;       // 3 per CTA: the parameters' cotangents
};

// Phi along one seeded input (m < 10: h_m; m < 40: dh; m < 50: d_t h; 50..52: the parameters)
template <bool DISS, bool INT>
__device__ __forceinline__ Tan adjoint_phi(int m, const Case& cs, const RhsArgs& A, const PointIdx& q, double r, bool layer,
                           const double* hv, const double* d1, const double* dth, const double* Pv,
                           const double* koh, double eh, double ih, double ih2, const double* lh, const double* lP,
                           const double* P1, double P0, const double* P2, double PKO, const double* he,
                           const double* Pe) {
  Tan hT[NC], dT[3][NC], dthT[NC];
#pragma unroll
  for (int v = 0; v < NC; ++v) hT[v] = Tan(hv[v], m == v ? 1.0 : 0.0);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int v = 0; v < NC; ++v) dT[i][v] = Tan(d1[i * NC + v], m == NC + i * NC + v ? 1.0 : 0.0);
  Coef<Tan> C;
  metric_quantities(hT, C);
  if (m >= 4 * NC && m < 5 * NC) {
#pragma unroll
    for (int v = 0; v < NC; ++v) dthT[v] = Tan(dth[v], m - 4 * NC == v ? 1.0 : 0.0);
  } else {
    const Tan adiv = C.alpha / C.sqrtg;
#pragma unroll
    for (int v = 0; v < NC; ++v) {
      Tan s = C.beta[0] * dT[0][v] + C.beta[1] * dT[1][v] + C.beta[2] * dT[2][v] + adiv * Tan(Pv[v]);
      if (DISS) s = fma(Tan(eh), Tan(koh[v]), s);
      dthT[v] = s;
    }
  }
  const int dir = m == 50 ? TAN_RHO_MAX : m == 51 ? TAN_RAMP : m == 52 ? TAN_DAMP_NEAR : TAN_STATE;
  Tan wT = Tan(1.0), rhoT = Tan(0.0);
  if (INT && layer) layer_profiles_t(cs, r, dir, wT, rhoT);
  const Tan* dh[3] = {dT[0], dT[1], dT[2]};
  Tan divb, divA[3];
  metric_divergences(C, dh, divb, divA);
  Tan msrc[NC];
  const Tan* D[4] = {dthT, dT[0], dT[1], dT[2]};
  rhs_source(cs, A, q.b, q.ip, damping_rate_t(cs, A.t, q.x, dir), hT, C, D, msrc);
  // the Pi half: source + the stencil part contracted with the coefficients
  Tan lin = C.beta[0] * Tan(ih * P1[0]) + C.beta[1] * Tan(ih * P1[1]) + C.beta[2] * Tan(ih * P1[2]) + divb * Tan(P0);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    Tan sd = Tan(0.0);
#pragma unroll
    for (int v = 0; v < NC; ++v) sd = fma(Tan(lP[v]), dT[i][v], sd);
    lin = fma(divA[i], sd, lin);
  }
  const Tan am = C.alpha * C.sqrtg;
  Tan a2 = am * C.gamu[0] * Tan(P2[0]) + am * C.gamu[3] * Tan(P2[1]) + am * C.gamu[5] * Tan(P2[2]);
  a2 = a2 + Tan(2.0) * am * (C.gamu[1] * Tan(P2[3]) + C.gamu[2] * Tan(P2[4]) + C.gamu[4] * Tan(P2[5]));
  lin = lin + Tan(ih2) * a2 + Tan(eh * PKO);
  Tan phiP = lin;
#pragma unroll
  for (int v = 0; v < NC; ++v) phiP = fma(Tan(lP[v]), msrc[v], phiP);
  Tan phi;
  if (INT && layer) {
    Tan relax = Tan(0.0);
#pragma unroll
    for (int v = 0; v < NC; ++v) relax = relax + Tan(lP[v] * (Pv[v] - Pe[v]));
    phi = wT * phiP - rhoT * relax;
#pragma unroll
    for (int v = 0; v < NC; ++v) phi = phi + Tan(lh[v]) * (wT * dthT[v] - rhoT * (hT[v] - Tan(he[v])));
  } else {
    phi = phiP;
#pragma unroll
    for (int v = 0; v < NC; ++v) phi = fma(Tan(lh[v]), dthT[v], phi);
  }
  return phi;
}

template <int Q, bool DISS, bool INT>
static __global__ void __launch_bounds__(128) adjoint_point_kernel(const Case cs, const RhsArgs A, const AdjArgs J) {
  __shared__ double sh[3][128];
  const long p = A.p0 + (long)blockIdx.x * blockDim.x + threadIdx.x;
  double th[3] = {0.0, 0.0, 0.0};
  if (p < A.p1) {
    const PointIdx q = point_index(A, p);
    const long S = (long)A.N1 * A.N1 * A.N1;
    const long sv = (long)A.Wx * A.Wd * A.Wd;
    const long s[3] = {1, A.Wx, (long)A.Wx * A.Wd};
    const double* wk = A.work + q.wo;
    const long loc = q.wo - (long)q.b * NV * sv + (long)q.b * sv;  // the point in one feature field
    auto cot = [&](int v, int f) -> double& { return J.cot[(long)(v * ADJ_NF + f) * J.cstride + loc]; };
    double r = 0.0, w = 1.0, rho = 0.0, he[NC], Pe[NC];
    bool layer = false;
    bool frozen = false;
    if (INT) {
      r = interior_radius(cs, A.t, q.x);
      frozen = cs.interior == TGH_INT_PASTED ? r < cs.r1 : r < cs.r0;
      layer = !frozen && r < cs.r1;
      if (layer) {
        layer_profiles(cs, r, w, rho);
        rn_background_state(cs, A.t, q.x, he, Pe);
      }
    }
    if (frozen) {
      // a core at rest: du = 0, nothing depends on the state
      for (int v = 0; v < NC; ++v)
        for (int f = 0; f < ADJ_NF; ++f) cot(v, f) = 0.0;
    } else {
      const double ih = 1.0 / q.h, ih2 = ih * ih;
      const double eh = DISS ? dissipation_rate(cs, A.t, q.x) * ih : 0.0;
      double lh[NC], lP[NC], hv[NC], Pv[NC], d1[3 * NC], koh[NC];
      const double* lam = J.lam + (long)q.b * NV * S + q.ip;
      for (int v = 0; v < NC; ++v) {
        lh[v] = lam[v * S];
        lP[v] = lam[(NC + v) * S];
        const double* ph = wk + v * sv;
        hv[v] = ph[0];
        Pv[v] = ph[NC * sv];
        for (int i = 0; i < 3; ++i) d1[i * NC + v] = ih * st_d1<Q, double>(ph, s[i]);
        koh[v] = DISS ? st_ko<Q, double>(ph, s[0], hv[v]) + st_ko<Q, double>(ph, s[1], hv[v]) +
                            st_ko<Q, double>(ph, s[2], hv[v])
                      : 0.0;
      }
      Coef<double> C;
      metric_quantities(hv, C);
      const double adiv = C.alpha / C.sqrtg;
      double dth[NC];
      for (int v = 0; v < NC; ++v) {
        double x = C.beta[0] * d1[v] + C.beta[1] * d1[NC + v] + C.beta[2] * d1[2 * NC + v] + adiv * Pv[v];
        if (DISS) x = fma(eh, koh[v], x);
        dth[v] = x;
      }
      const double* dh[3] = {d1, d1 + NC, d1 + 2 * NC};
      double divb, divA[3];
      metric_divergences(C, dh, divb, divA);
      const double am = C.alpha * C.sqrtg;
      const double Ad[6] = {am * C.gamu[0], am * C.gamu[3], am * C.gamu[5],
                            2.0 * am * C.gamu[1], 2.0 * am * C.gamu[2], 2.0 * am * C.gamu[4]};
      const double W = layer ? w : 1.0;
      // the linear features: their sums against lambda, and their cotangents
      double P1[3] = {0, 0, 0}, P0 = 0.0, P2[6] = {0, 0, 0, 0, 0, 0}, PKO = 0.0;
      for (int v = 0; v < NC; ++v) {
        const double* ph = wk + v * sv;
        const double* pp = ph + NC * sv;
        for (int i = 0; i < 3; ++i) P1[i] += lP[v] * st_d1<Q, double>(pp, s[i]);
        P0 += lP[v] * Pv[v];
        for (int i = 0; i < 3; ++i) P2[i] += lP[v] * st_d2<Q, double>(ph, s[i], hv[v]);
        P2[3] += lP[v] * st_mixed<Q, double>(ph, s[0], s[1]);
        P2[4] += lP[v] * st_mixed<Q, double>(ph, s[0], s[2]);
        P2[5] += lP[v] * st_mixed<Q, double>(ph, s[1], s[2]);
        if (DISS)
          PKO += lP[v] * (st_ko<Q, double>(pp, s[0], Pv[v]) + st_ko<Q, double>(pp, s[1], Pv[v]) +
                          st_ko<Q, double>(pp, s[2], Pv[v]));
        const double wl = W * lP[v];
        for (int i = 0; i < 3; ++i) cot(v, AF_PD1 + i) = wl * C.beta[i] * ih;
        for (int i = 0; i < 3; ++i) cot(v, AF_HD2 + i) = wl * ih2 * Ad[i];
        for (int i = 0; i < 3; ++i) cot(v, AF_HMX + i) = wl * ih2 * Ad[3 + i];
        cot(v, AF_PKO) = wl * eh;
      }
      // the nonlinear inputs, one forward pass each
      double g[ADJ_PASSES];
#pragma unroll 1
      for (int m = 0; m < ADJ_PASSES; ++m) {
        if ((m == 50 || m == 51) && !layer) {
          g[m] = 0.0;
          continue;
        }
        g[m] = adjoint_phi<DISS, INT>(m, cs, A, q, r, layer, hv, d1, dth, Pv, koh, eh, ih, ih2, lh, lP, P1, P0, P2,
                                      PKO, he, Pe)
                   .d;
      }
      for (int v = 0; v < NC; ++v) {
        cot(v, AF_HC) = g[v];
        for (int i = 0; i < 3; ++i) cot(v, AF_HD1 + i) = g[NC + i * NC + v] * ih;
        const double gd = g[4 * NC + v];
        cot(v, AF_HKO) = gd * eh;
        cot(v, AF_PC) = gd * adiv + W * lP[v] * divb - (layer ? rho * lP[v] : 0.0);
      }
      th[0] = g[50];
      th[1] = g[51];
      th[2] = g[52];
    }
  }
  // the parameters' cotangents: per CTA, in a fixed order
  for (int k = 0; k < 3; ++k) sh[k][threadIdx.x] = th[k];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int k = 0; k < 3; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) J.part[3 * blockIdx.x + k] = sh[k][0];
}

// The transposed stencils: mu at every point of every block's working array (ghosts included)
// for component v of h and of Pi, from the feature cotangents of the owned points that read it.
template <int Q, bool DISS>
static __global__ void __launch_bounds__(128) adjoint_gather_kernel(const double* __restrict__ cot, long cstride, Geo g,
                                                             int nb, double* __restrict__ mu) {
  const long cube = (long)g.Wd * g.Wd * g.Wd;
  const long id = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= cube * NC * nb) return;
  const int b = (int)(id / (cube * NC));
  const int v = (int)((id / cube) % NC);
  const long c = id % cube;
  const int x = (int)(c % g.Wd), y = (int)((c / g.Wd) % g.Wd), z = (int)(c / ((long)g.Wd * g.Wd));
  const int X[3] = {x, y, z};
  const long st[3] = {1, g.Wx, (long)g.Wx * g.Wd};
  const long base = (long)b * g.Wv + work_index(g, x, y, z);
  auto F = [&](int f, int dx, int dy, int dz) -> double {
    const int xx = x + dx, yy = y + dy, zz = z + dz;
    if (xx < 0 || yy < 0 || zz < 0 || xx >= g.Wd || yy >= g.Wd || zz >= g.Wd) return 0.0;
    return cot[(long)(v * ADJ_NF + f) * cstride + base + dx + g.Wx * (dy + (long)g.Wd * dz)];
  };
  auto off = [&](int axis, int k, int& dx, int& dy, int& dz) {
    dx = axis == 0 ? k : 0;
    dy = axis == 1 ? k : 0;
    dz = axis == 2 ? k : 0;
  };
  (void)X;
  (void)st;
  double mh = F(AF_HC, 0, 0, 0), mp = F(AF_PC, 0, 0, 0);
  for (int a = 0; a < 3; ++a) {
    int px, py, pz, mx, my, mz;
    for (int k = 1; k <= W<Q>::R; ++k) {
      off(a, k, px, py, pz);
      off(a, -k, mx, my, mz);
      // first derivatives: D(p) = sum_k w_k (u(p + k) - u(p - k))
      mh += W<Q>::d1(k) * (F(AF_HD1 + a, mx, my, mz) - F(AF_HD1 + a, px, py, pz));
      mp += W<Q>::d1(k) * (F(AF_PD1 + a, mx, my, mz) - F(AF_PD1 + a, px, py, pz));
      // second derivatives: w_0 u(p) + sum_k w_k (u(p + k) + u(p - k))
      mh += W<Q>::d2(k) * (F(AF_HD2 + a, mx, my, mz) + F(AF_HD2 + a, px, py, pz));
    }
    mh += W<Q>::d2(0) * F(AF_HD2 + a, 0, 0, 0);
    if (DISS) {
      for (int k = 1; k <= W<Q>::RD; ++k) {
        off(a, k, px, py, pz);
        off(a, -k, mx, my, mz);
        mh += W<Q>::ko(k) * (F(AF_HKO, mx, my, mz) + F(AF_HKO, px, py, pz));
        mp += W<Q>::ko(k) * (F(AF_PKO, mx, my, mz) + F(AF_PKO, px, py, pz));
      }
      mh += W<Q>::ko(0) * F(AF_HKO, 0, 0, 0);
      mp += W<Q>::ko(0) * F(AF_PKO, 0, 0, 0);
    }
  }
  // mixed: M(p) = sum_a w_a sum_e w_e ((u(p+a1+e2) - u(p+a1-e2)) - (u(p-a1+e2) - u(p-a1-e2)))
  const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  for (int k = 0; k < 3; ++k) {
    const int a1 = pairs[k][0], a2 = pairs[k][1];
    for (int a = 1; a <= W<Q>::R; ++a)
      for (int e = 1; e <= W<Q>::R; ++e) {
        int d[3];
        double s4 = 0.0;
        for (int sa = -1; sa <= 1; sa += 2)
          for (int se = -1; se <= 1; se += 2) {
            d[0] = d[1] = d[2] = 0;
            d[a1] = -sa * a;
            d[a2] = -se * e;
            // the point p = q - (sa a) e1 - (se e) e2 reads q with sign sa * se
            s4 += (double)(sa * se) * F(AF_HMX + k, d[0], d[1], d[2]);
          }
        mh += W<Q>::d1(a) * W<Q>::d1(e) * s4;
      }
  }
  const long o = (long)b * NV * g.Wv + work_index(g, x, y, z);
  mu[o + v * g.Wv] = mh;
  mu[o + (NC + v) * g.Wv] = mp;
}

// The fill's transpose, prolongation part: level l's prolonged ghost values pass their mu to the
// coarse stencil they were summed from (the finest level first).
template <int P>
static __global__ void prolong_adjoint_kernel(const ProlongPt* __restrict__ pts, int n, double* __restrict__ mu, Geo g) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= n * NV) return;
  const int pi = id % n, v = id / n;
  const ProlongPt p = pts[pi];
  const double m = mu[(long)p.dst_b * NV * g.Wv + (long)v * g.Wv + p.dst_w];
  if (m == 0.0) return;
  constexpr ProlongWeights<P> Wt = prolong_weights<P>();
  const int cx = (p.odd & 1) ? P : 1, cy = (p.odd & 2) ? P : 1, cz = (p.odd & 4) ? P : 1;
  double* src = mu + (long)p.src_b * NV * g.Wv + (long)v * g.Wv + p.src_w;
  const long sy = g.Wx, sz = (long)g.Wx * g.Wd;
  for (int kz = 0; kz < cz; ++kz)
    for (int ky = 0; ky < cy; ++ky)
      for (int kx = 0; kx < cx; ++kx) {
        const double wgt = (cx == 1 ? 1.0 : Wt.v[kx]) * (cy == 1 ? 1.0 : Wt.v[ky]) * (cz == 1 ? 1.0 : Wt.v[kz]);
        atomicAdd(src + kz * sz + ky * sy + kx, wgt * m);
      }
}

// The fill's transpose, copy part: every work point filled from the state vector hands its mu to
// that state entry (the primary copy of its lattice point).
static __global__ void copy_adjoint_kernel(const CopyRun* __restrict__ runs, int nruns, const double* __restrict__ mu,
                                    double* __restrict__ mu_u, Geo g) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= nruns) return;
  const CopyRun r = runs[warp];
  for (int e = lane; e < r.len; e += 32) {
    double* dst = mu_u + (long)r.src_b * NV * g.S + (r.si + e * r.step) + (long)g.N1 * (r.sj + (long)g.N1 * r.sk);
    const double* src = mu + (long)r.dst_b * NV * g.Wv + r.dst_w + e;
    for (int v = 0; v < NV; ++v) {
      const double m = src[v * g.Wv];
      if (m != 0.0) atomicAdd(dst + v * g.S, m);
    }
  }
}

// y = a x + y over n entries
static __global__ void axpy_kernel(long n, double a, const double* __restrict__ x, double* __restrict__ y) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    y[i] = fma(a, x[i], y[i]);
}
// z = a x + b y
static __global__ void axpby_kernel(long n, double a, const double* __restrict__ x, double b, const double* __restrict__ y,
                             double* __restrict__ z) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    z[i] = a * x[i] + b * y[i];
}

// the masked error's gradient: lambda = w (u - u_exact) / (L sum w) at the evolved primaries
// (zero elsewhere), given L and sum w
static __global__ void error_adjoint_kernel(const double* __restrict__ u, const double* __restrict__ blk,
                                     const uint8_t* __restrict__ primary, Geo g, long npts, const Case cs, double t,
                                     double scale, double* __restrict__ lam) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const int b = (int)(p / g.S);
  const long ip = p - (long)b * g.S;
  double* o = lam + (long)b * NV * g.S + ip;
  const double* q = u + (long)b * NV * g.S + ip;
  bool ev = primary[p] != 0;
  double ex[NV];
  if (ev) {
    const int k = (int)(ip / ((long)g.N1 * g.N1)), j = (int)((ip / g.N1) % g.N1), i = (int)(ip % g.N1);
    double x[3];
    point_pos(blk, b, i, j, k, x);
    ev = evolved(cs, t, x);
    if (ev) exact_state(cs, t, x, ex);
  }
  const double h = blk[8 * b + 3];
  for (int v = 0; v < NV; ++v) o[v * g.S] = ev ? scale * h * h * h * (q[v * g.S] - ex[v]) : 0.0;
}

cudaError_t launch_adjoint_point(int q, bool diss, bool intr, cudaStream_t s, const Case& cs, const RhsArgs& a,
                                 const AdjArgs& j);
cudaError_t launch_adjoint_gather(int q, bool diss, cudaStream_t s, const double* cot, long cstride, const Geo& g,
                                  int nb, double* mu);

}  // namespace tgh
