// Device spelling of the generalized-harmonic source algebra, kept in registers:
//   the reduced source with constraint damping   (src/pointwise.jl:612-741, gh_node_source_lean)
//   the coefficient divergences                  (src/pointwise.jl:754-778, metric_divergences)
//   the matter term                              (src/pointwise.jl:667-698, matter_source)
// Symmetric tensors are held by their 10 packed components; every loop is unrolled with
// compile-time indices so that nothing is addressed through local memory. The terms and
// their grouping follow the reference's lean spelling; the summation order inside a
// contraction is the compiler's (fused multiply-adds), which moves results by roundoff.
#pragma once
#include "analytic.cuh"

namespace tgh {

// msrc = -alpha sqrt(gamma) (S0 + Z) from the coefficients, D[c] = d_c g packed (c = t,x,y,z),
// the lowered gauge source Hl and dHs = d_a H_b + d_b H_a packed.
//
// The terms are formed in the order that keeps the fewest values live at one point (one
// thread holds them all in registers): first everything that reads D besides the
// Christoffels - the contracted Christoffel Gamma^c = g^{cx} (g^{ab} d_a g_xb - g^{ab} d_x g_ab / 2),
// the term Gamma^c d_c g_ab, and C2 + C2^T built one row of g^{-1} (d_a g) at a time - then
// the 40 Christoffels Gamma^a_bc, after which D is dead, then Gamma.Gamma, the gauge terms
// and the damping. Same terms as the reference's spelling, summed in another order.
template <class T, bool HAS_H>
TGH_HD void gh_source(const Coef<T>& C, const T* const D[4], const T Hl[4], const T dHs[NC], T g0, T g2,
                      T* msrc) {
  const T* Gp = C.gu;
  // (1) Gamma^c
  T Gup[4];
  {
    T V[4];
#pragma unroll
    for (int x = 0; x < 4; ++x) {
      T s = T(0.0), tr = T(0.0);
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) s = fma(Gp[pidx(a, b)], D[a][pidx(x, b)], s);
#pragma unroll
      for (int n = 0; n < NC; ++n) tr = fma(prow(n) == pcol(n) ? Gp[n] : T(2.0) * Gp[n], D[x][n], tr);
      V[x] = fma(T(-0.5), tr, s);
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      T s = Gp[pidx(c, 0)] * V[0];
#pragma unroll
      for (int x = 1; x < 4; ++x) s = fma(Gp[pidx(c, x)], V[x], s);
      Gup[c] = s;
    }
  }
  // (2) S = -(d_a H_b + d_b H_a) - Gamma^c d_c g_ab
  T S[NC];
#pragma unroll
  for (int n = 0; n < NC; ++n) {
    T t5 = Gup[0] * D[0][n];
#pragma unroll
    for (int c = 1; c < 4; ++c) t5 = fma(Gup[c], D[c][n], t5);
    S[n] = HAS_H ? -(dHs[n] + t5) : -t5;
  }
  // (3) C2 + C2^T with C2[a][b] = Cuu_{mn} d_m g_nb, Cuu = g^{-1} (d_a g) g^{-1} (symmetric):
  //     row m of E = g^{-1} d_a g, then Cuu_{mn} for n >= m, consumed at once
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    T C2[4];
#pragma unroll
    for (int b = 0; b < 4; ++b) C2[b] = T(0.0);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      T E[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        T s = Gp[pidx(m, 0)] * D[a][pidx(0, c)];
#pragma unroll
        for (int x = 1; x < 4; ++x) s = fma(Gp[pidx(m, x)], D[a][pidx(x, c)], s);
        E[c] = s;
      }
#pragma unroll
      for (int n = m; n < 4; ++n) {
        T cu = E[0] * Gp[pidx(0, n)];
#pragma unroll
        for (int y = 1; y < 4; ++y) cu = fma(E[y], Gp[pidx(y, n)], cu);
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          C2[b] = fma(cu, D[m][pidx(n, b)], C2[b]);
          if (n != m) C2[b] = fma(cu, D[n][pidx(m, b)], C2[b]);
        }
      }
    }
#pragma unroll
    for (int n = 0; n < NC; ++n) {
      const int i = prow(n), j = pcol(n);
      if (i == a) S[n] += C2[j];
      if (j == a) S[n] += C2[i];
    }
  }
  // (4) Christoffels Gamma^a_bc = g^{ax} (d_b g_xc + d_c g_xb - d_x g_bc)/2, packed over (bc)
  T G[4][NC];
#pragma unroll
  for (int n = 0; n < NC; ++n) {
    const int i = prow(n), j = pcol(n);
    T low[4];
#pragma unroll
    for (int x = 0; x < 4; ++x) low[x] = T(0.5) * (D[i][pidx(x, j)] + D[j][pidx(x, i)] - D[x][pidx(i, j)]);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      T s = Gp[pidx(a, 0)] * low[0];
#pragma unroll
      for (int x = 1; x < 4; ++x) s = fma(Gp[pidx(a, x)], low[x], s);
      G[a][n] = s;
    }
  }
  // (5) -2 Gamma^x_ya Gamma^y_xb and + 2 Gamma^c_ab H_c
#pragma unroll
  for (int n = 0; n < NC; ++n) {
    const int a = prow(n), b = pcol(n);
    T t2 = T(0.0);
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
      for (int y = 0; y < 4; ++y) t2 = fma(G[x][pidx(y, a)], G[y][pidx(x, b)], t2);
    T s = fma(T(-2.0), t2, S[n]);
    if (HAS_H) {
      T t4 = G[0][n] * Hl[0];
#pragma unroll
      for (int c = 1; c < 4; ++c) t4 = fma(G[c][n], Hl[c], t4);
      s = fma(T(2.0), t4, s);
    }
    S[n] = s;
  }
  // (6) Gundlach-Pretorius damping with t_a = -alpha delta_a^t
  if (g0 != T(0.0)) {
    T Cup[4], Cl[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      T s = Gup[c];
      if (HAS_H) {
#pragma unroll
        for (int x = 0; x < 4; ++x) s = fma(Gp[pidx(c, x)], Hl[x], s);
      }
      Cup[c] = s;
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      T s = C.g[pidx(c, 0)] * Cup[0];
#pragma unroll
      for (int x = 1; x < 4; ++x) s = fma(C.g[pidx(c, x)], Cup[x], s);
      Cl[c] = s;
    }
    T tC = Gp[pidx(0, 0)] * Cl[0];
#pragma unroll
    for (int x = 1; x < 4; ++x) tC = fma(Gp[pidx(0, x)], Cl[x], tC);
    tC = -C.alpha * tC;
    const T tl = -C.alpha;
    const T k = (T(1.0) + g2) * tC;
#pragma unroll
    for (int n = 0; n < NC; ++n) {
      const int a = prow(n), b = pcol(n);
      T z = T(0.0);
      if (a == 0) z = fma(tl, Cl[b], z);
      if (b == 0) z = fma(tl, Cl[a], z);
      z = z - k * C.g[n];
      S[n] = fma(g0, z, S[n]);
    }
  }
  const T f = -(C.alpha * C.sqrtg);
#pragma unroll
  for (int n = 0; n < NC; ++n) msrc[n] = f * S[n];
}

// row a of d g^{ab} = -g^{ac} (d g_cd) g^{db}
template <class T, int A>
TGH_HD void dgu_row(const T* Gp, const T* dg, T out[4]) {
  T v[4];
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    T s = Gp[pidx(A, 0)] * dg[pidx(0, d)];
#pragma unroll
    for (int c = 1; c < 4; ++c) s = fma(Gp[pidx(A, c)], dg[pidx(c, d)], s);
    v[d] = s;
  }
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    T s = v[0] * Gp[pidx(0, b)];
#pragma unroll
    for (int d = 1; d < 4; ++d) s = fma(v[d], Gp[pidx(d, b)], s);
    out[b] = -s;
  }
}

// d_i beta^i and d_i (alpha sqrt(gamma) gamma^{ij})
template <class T>
TGH_HD void metric_divergences(const Coef<T>& C, const T* const dh[3], T& divb, T divA[3]) {
  const T* Gp = C.gu;
  const T igutt = T(1.0) / Gp[0];
  T r1[3][4], ri[3][4];
  dgu_row<T, 0>(Gp, dh[0], r1[0]);
  dgu_row<T, 0>(Gp, dh[1], r1[1]);
  dgu_row<T, 0>(Gp, dh[2], r1[2]);
  dgu_row<T, 1>(Gp, dh[0], ri[0]);
  dgu_row<T, 2>(Gp, dh[1], ri[1]);
  dgu_row<T, 3>(Gp, dh[2], ri[2]);
  divb = T(0.0);
#pragma unroll
  for (int i = 0; i < 3; ++i) divb -= (r1[i][i + 1] + C.beta[i] * r1[i][0]) * igutt;
  const T a3h = T(0.5) * C.alpha * C.alpha * C.alpha;
  const T as = C.alpha * C.sqrtg;
  T fac[3];  // d_i (alpha sqrt(gamma)) = sqrt(gamma) d_i alpha + alpha d_i sqrt(gamma)
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    T s = T(0.0);
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int k = 0; k < 3; ++k) s = fma(C.gamu[sidx3(j, k)], dh[i][pidx(j + 1, k + 1)], s);
    const T ds = T(0.5) * C.sqrtg * s;
    fac[i] = a3h * r1[i][0] * C.sqrtg + C.alpha * ds;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    T s = T(0.0);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      T dgam = ri[i][k + 1] + C.beta[k] * r1[i][i + 1] + C.beta[i] * r1[i][k + 1] + C.beta[i] * C.beta[k] * r1[i][0];
      s = fma(fac[i], C.gamu[sidx3(i, k)], s);
      s = fma(as, dgam, s);
    }
    divA[k] = s;
  }
}

// the stress-energy term alpha sqrt(gamma) (16 pi T_ab - 8 pi g_ab T); m = (rho, S_i, S_ij packed)
template <class T>
TGH_HD void matter_source(const Coef<T>& C, const T* m, T* out) {
  const T c8 = T(8.0 * M_PI), c16 = T(16.0 * M_PI);
  const T* b = C.beta;
  const T rho = m[0];
  const T S1 = m[1], S2 = m[2], S3 = m[3];
  const T S11 = m[4], S21 = m[5], S31 = m[6], S22 = m[7], S32 = m[8], S33 = m[9];
  T Sb1 = S11 * b[0] + S21 * b[1] + S31 * b[2];
  T Sb2 = S21 * b[0] + S22 * b[1] + S32 * b[2];
  T Sb3 = S31 * b[0] + S32 * b[1] + S33 * b[2];
  T bS = b[0] * S1 + b[1] * S2 + b[2] * S3;
  T Ttt = C.alpha * C.alpha * rho - T(2.0) * (C.alpha * bS) + (b[0] * Sb1 + b[1] * Sb2 + b[2] * Sb3);
  T Tt[3] = {Sb1 - C.alpha * S1, Sb2 - C.alpha * S2, Sb3 - C.alpha * S3};
  T trS = C.gamu[0] * S11 + C.gamu[3] * S22 + C.gamu[5] * S33 +
          T(2.0) * (C.gamu[1] * S21 + C.gamu[2] * S31 + C.gamu[4] * S32);
  T tr8 = c8 * (trS - rho);
  T a = C.alpha * C.sqrtg;
  const T Tab[NC] = {Ttt, Tt[0], Tt[1], Tt[2], S11, S21, S31, S22, S32, S33};
#pragma unroll
  for (int n = 0; n < NC; ++n) out[n] = a * (c16 * Tab[n] - C.g[n] * tr8);
}

}  // namespace tgh
