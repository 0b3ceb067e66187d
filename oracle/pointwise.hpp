// TEST INFRASTRUCTURE -- part of the CPU oracle (see stencils.hpp).
//
// The pointwise generalized-harmonic algebra, restating src/pointwise.jl:
//   metric_quantities            src/pointwise.jl:145-184
//   gh_node_source               src/pointwise.jl:346-401   (reference spelling)
//   metric_derivatives           src/pointwise.jl:462-500
//   gh_node_source_lean          src/pointwise.jl:612-741   (the kernel's spelling)
//   metric_divergences, _dgu_row src/pointwise.jl:754-778
//   gh_node_rhs_expanded         src/pointwise.jl:818-850
//   matter_source                src/pointwise.jl:667-698
//   metric_derivatives_along     src/pointwise.jl:530-546
//   gauge_constraint_at_node     src/pointwise.jl:947-962
//   adm_constraints_at_node      src/constraints.jl:136-190
// Packed order (tt,tx,ty,tz,xx,xy,xz,yy,yz,zz); every index below is 0-based.
// Sums are left folds in the reference's order; the file is compiled without
// floating-point contraction so that each product is rounded, as Julia does by default.
#pragma once
#include <cmath>

namespace orc {

static const int NC = 10;

// _pairindex (src/pointwise.jl:102-105), 0-based
static inline int pairindex(int a, int b) {
  int i = a > b ? a : b, j = a > b ? b : a;
  return j * 4 - (j * (j - 1)) / 2 + (i - j);
}
// _unpair (src/pointwise.jl:569-574), 0-based (row >= col)
static inline void unpair(int n, int& a, int& b) {
  if (n < 4) { a = n; b = 0; }
  else if (n < 7) { a = n - 3; b = 1; }
  else if (n < 9) { a = n - 5; b = 2; }
  else { a = 3; b = 3; }
}

template <class T> static inline void sym4(const T* v, T m[4][4]) {
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) m[a][b] = v[pairindex(a, b)];
}
template <class T> static inline void pack10(const T m[4][4], T* v) {
  for (int n = 0; n < NC; ++n) {
    int a, b;
    unpair(n, a, b);
    v[n] = m[a][b];
  }
}
static inline double eta(int a) { return a == 0 ? -1.0 : 1.0; }

template <class T> static inline T det3(T a, T b, T c, T d, T e, T f, T g, T h, T i) {
  return a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
}
// 4x4 determinant and inverse by cofactors
template <class T> static inline T det4(const T m[4][4]) {
  T s = T(0);
  for (int j = 0; j < 4; ++j) {
    int c[3], k = 0;
    for (int jj = 0; jj < 4; ++jj)
      if (jj != j) c[k++] = jj;
    T minor = det3(m[1][c[0]], m[1][c[1]], m[1][c[2]], m[2][c[0]], m[2][c[1]], m[2][c[2]],
                   m[3][c[0]], m[3][c[1]], m[3][c[2]]);
    s = (j % 2 == 0) ? s + m[0][j] * minor : s - m[0][j] * minor;
  }
  return s;
}
template <class T> static inline void inv4(const T m[4][4], T out[4][4]) {
  T cof[4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      int r[3], c[3], kr = 0, kc = 0;
      for (int ii = 0; ii < 4; ++ii)
        if (ii != i) r[kr++] = ii;
      for (int jj = 0; jj < 4; ++jj)
        if (jj != j) c[kc++] = jj;
      T minor = det3(m[r[0]][c[0]], m[r[0]][c[1]], m[r[0]][c[2]], m[r[1]][c[0]], m[r[1]][c[1]],
                     m[r[1]][c[2]], m[r[2]][c[0]], m[r[2]][c[1]], m[r[2]][c[2]]);
      cof[i][j] = ((i + j) % 2 == 0) ? minor : -minor;
    }
  T det = m[0][0] * cof[0][0] + m[0][1] * cof[0][1] + m[0][2] * cof[0][2] + m[0][3] * cof[0][3];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) out[i][j] = cof[j][i] / det;
}
template <class T> static inline void inv3(const T m[3][3], T o[3][3]) {
  T c00 = m[1][1] * m[2][2] - m[1][2] * m[2][1];
  T c01 = m[1][2] * m[2][0] - m[1][0] * m[2][2];
  T c02 = m[1][0] * m[2][1] - m[1][1] * m[2][0];
  T det = m[0][0] * c00 + m[0][1] * c01 + m[0][2] * c02;
  o[0][0] = c00 / det;
  o[1][0] = c01 / det;
  o[2][0] = c02 / det;
  o[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) / det;
  o[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) / det;
  o[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) / det;
  o[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) / det;
  o[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) / det;
  o[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) / det;
}

template <class T> struct Coef {
  T g4[4][4], gu4[4][4], guo[4][4];
  T alpha, beta[3], gamu[3][3], sqrtg;
};

// src/pointwise.jl:145-184
template <class T> static inline void metric_quantities(const T* h10, Coef<T>& c) {
  T hm[4][4];
  sym4(h10, hm);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) c.g4[a][b] = (a == b ? T(eta(a)) : T(0)) + hm[a][b];
  T gi[4][4];
  inv4(c.g4, gi);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      T s = gi[a][0] * hm[0][b];
      for (int k = 1; k < 4; ++k) s = s + gi[a][k] * hm[k][b];
      c.guo[a][b] = -(s * T(eta(b)));
    }
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) c.gu4[a][b] = (a == b ? T(eta(a)) : T(0)) + c.guo[a][b];
  T gutt = c.gu4[0][0];
  T q1 = c.guo[0][0];
  c.alpha = T(1) / sqrt(T(1) - q1);
  for (int i = 0; i < 3; ++i) c.beta[i] = -c.gu4[0][i + 1] / gutt;
  for (int r = 0; r < 3; ++r)
    for (int s = 0; s < 3; ++s)
      c.gamu[r][s] = c.gu4[r + 1][s + 1] - c.gu4[0][r + 1] * c.gu4[0][s + 1] / gutt;
  T B[4][4];
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) B[a][b] = T(eta(a)) * hm[a][b];
  T B2[4][4], B3[4][4];
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      T s = B[a][0] * B[0][b];
      for (int k = 1; k < 4; ++k) s = s + B[a][k] * B[k][b];
      B2[a][b] = s;
    }
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      T s = B2[a][0] * B[0][b];
      for (int k = 1; k < 4; ++k) s = s + B2[a][k] * B[k][b];
      B3[a][b] = s;
    }
  T trB = ((B[0][0] + B[1][1]) + B[2][2]) + B[3][3];
  T trB2 = ((B2[0][0] + B2[1][1]) + B2[2][2]) + B2[3][3];
  T trB3 = ((B3[0][0] + B3[1][1]) + B3[2][2]) + B3[3][3];
  T e1 = trB;
  T e2 = (trB * trB - trB2) / T(2);
  T e3 = (trB * trB * trB - T(3) * trB * trB2 + T(2) * trB3) / T(6);
  T e4 = det4(B);
  T d1 = -(((e1 + e2) + e3) + e4);
  T detgm1 = -d1 - q1 + d1 * q1;
  c.sqrtg = sqrt(T(1) + detgm1);
}

// dg[a][b][c] = d_a g_bc (GHSO2 order) from d_t g and the three spatial gradients (_dg4)
template <class T> static inline void dg4(const T* dtg, const T* const dh[3], T dg[4][4][4]) {
  const T* D[4] = {dtg, dh[0], dh[1], dh[2]};
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b)
      for (int c = 0; c < 4; ++c) dg[a][b][c] = D[a][pairindex(b, c)];
}

// src/pointwise.jl:346-401, the reference spelling of msrc = -a sqrtg (S0 + Z)
template <class T>
static inline void gh_node_source(const Coef<T>& C, const T dg[4][4][4], const T Hl[4],
                                  const T dHl[4][4], T g0, T g2, T* msrc) {
  const T a_mul = C.alpha * C.sqrtg;
  T Clul[4][4][4], Cluu[4][4][4];
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b)
      for (int c = 0; c < 4; ++c) {
        T s = C.gu4[b][0] * dg[a][0][c];
        for (int x = 1; x < 4; ++x) s = s + C.gu4[b][x] * dg[a][x][c];
        Clul[a][b][c] = s;
      }
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b)
      for (int c = 0; c < 4; ++c) {
        T s = C.gu4[c][0] * Clul[a][b][0];
        for (int y = 1; y < 4; ++y) s = s + C.gu4[c][y] * Clul[a][b][y];
        Cluu[a][b][c] = s;
      }
  T C2[4][4];
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      bool first = true;
      T s = T(0);
      for (int y = 0; y < 4; ++y)
        for (int x = 0; x < 4; ++x) {
          T t = Cluu[a][x][y] * dg[x][y][b];
          s = first ? t : s + t;
          first = false;
        }
      C2[a][b] = s;
    }
  T Glll[4][4][4], G4[4][4][4];
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b)
      for (int c = 0; c < 4; ++c) Glll[a][b][c] = (dg[b][a][c] + dg[c][a][b] - dg[a][b][c]) / T(2);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b)
      for (int c = 0; c < 4; ++c) {
        T s = C.gu4[a][0] * Glll[0][b][c];
        for (int x = 1; x < 4; ++x) s = s + C.gu4[a][x] * Glll[x][b][c];
        G4[a][b][c] = s;
      }
  T G2[4][4];
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      bool first = true;
      T s = T(0);
      for (int y = 0; y < 4; ++y)
        for (int x = 0; x < 4; ++x) {
          T t = G4[x][y][a] * G4[y][x][b];
          s = first ? t : s + t;
          first = false;
        }
      G2[a][b] = s;
    }
  T Gup[4];
  for (int c = 0; c < 4; ++c) {
    bool first = true;
    T s = T(0);
    for (int e = 0; e < 4; ++e)
      for (int d = 0; d < 4; ++d) {
        T t = C.gu4[d][e] * G4[c][d][e];
        s = first ? t : s + t;
        first = false;
      }
    Gup[c] = s;
  }
  T S0[4][4];
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      T sH = G4[0][a][b] * Hl[0];
      for (int c = 1; c < 4; ++c) sH = sH + G4[c][a][b] * Hl[c];
      T sG = Gup[0] * dg[0][a][b];
      for (int c = 1; c < 4; ++c) sG = sG + Gup[c] * dg[c][a][b];
      S0[a][b] = (C2[a][b] + C2[b][a]) - T(2) * G2[a][b] - dHl[a][b] - dHl[b][a] + T(2) * sH - sG;
    }
  if (g0 != T(0)) {
    T Cup[4], Cl[4], tl[4] = {-C.alpha, T(0), T(0), T(0)}, tu[4];
    for (int c = 0; c < 4; ++c) {
      T s = C.gu4[c][0] * Hl[0];
      for (int x = 1; x < 4; ++x) s = s + C.gu4[c][x] * Hl[x];
      Cup[c] = Gup[c] + s;
    }
    for (int c = 0; c < 4; ++c) {
      T s = C.g4[c][0] * Cup[0];
      for (int x = 1; x < 4; ++x) s = s + C.g4[c][x] * Cup[x];
      Cl[c] = s;
    }
    for (int c = 0; c < 4; ++c) {
      T s = C.gu4[c][0] * tl[0];
      for (int x = 1; x < 4; ++x) s = s + C.gu4[c][x] * tl[x];
      tu[c] = s;
    }
    T tC = tu[0] * Cl[0];
    for (int x = 1; x < 4; ++x) tC = tC + tu[x] * Cl[x];
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b)
        S0[a][b] = S0[a][b] + g0 * (tl[a] * Cl[b] + tl[b] * Cl[a] - (T(1) + g2) * C.g4[a][b] * tC);
  }
  T p[NC];
  pack10(S0, p);
  for (int n = 0; n < NC; ++n) msrc[n] = -a_mul * p[n];
}

template <class T> static inline T slot(const T* v, int a, int b) { return v[pairindex(a, b)]; }
template <class T> static inline T fold4(const T t[4]) { return ((t[0] + t[1]) + t[2]) + t[3]; }
template <class T> static inline T foldn(const T* t, int n) {
  T s = t[0];
  for (int i = 1; i < n; ++i) s = s + t[i];
  return s;
}

// _lean_c2 (src/pointwise.jl:702-713)
template <class T> static inline void lean_c2(const T* Gp, const T* const D[4], int a, T* out) {
  const T* Da = D[a];
  T E[16];
  for (int n = 0; n < 16; ++n) {
    T t[4];
    for (int x = 0; x < 4; ++x) t[x] = slot(Gp, n % 4, x) * slot(Da, x, n / 4);
    E[n] = fold4(t);
  }
  T Cuu[NC];
  for (int n = 0; n < NC; ++n) {
    int i, j;
    unpair(n, i, j);
    T t[4];
    for (int y = 0; y < 4; ++y) t[y] = E[i + 4 * y] * slot(Gp, y, j);
    Cuu[n] = fold4(t);
  }
  T C2[4];
  for (int b = 0; b < 4; ++b) {
    T t[16];
    for (int m = 0; m < 16; ++m) t[m] = slot(Cuu, m % 4, m / 4) * slot(D[m % 4], m / 4, b);
    C2[b] = foldn(t, 16);
  }
  for (int n = 0; n < NC; ++n) {
    int i, j;
    unpair(n, i, j);
    out[n] = (i == a ? C2[j] : T(0)) + (j == a ? C2[i] : T(0));
  }
}

// _lean_christoffel (src/pointwise.jl:717-722): Gamma^a_bc packed over (bc)
template <class T> static inline void lean_christoffel(const T* Gp, const T* const D[4], int a, T* out) {
  for (int n = 0; n < NC; ++n) {
    int i, j;
    unpair(n, i, j);
    T t[4];
    for (int x = 0; x < 4; ++x)
      t[x] = slot(Gp, a, x) * ((slot(D[i], x, j) + slot(D[j], x, i) - slot(D[x], i, j)) / T(2));
    out[n] = fold4(t);
  }
}

// src/pointwise.jl:612-639 (+ _lean_gamma_terms :726-733, _lean_damping :736-741)
template <class T>
static inline void gh_node_source_lean(const Coef<T>& C, const T* dth, const T* const dh[3],
                                       const T Hl[4], const T dHl[4][4], T g0, T g2, T* msrc) {
  T Gp[NC], gp[NC];
  pack10(C.gu4, Gp);
  pack10(C.g4, gp);
  const T* D[4] = {dth, dh[0], dh[1], dh[2]};
  T c[4][NC];
  for (int a = 0; a < 4; ++a) lean_c2(Gp, D, a, c[a]);
  T S[NC];
  for (int n = 0; n < NC; ++n) S[n] = ((c[0][n] + c[1][n]) + c[2][n]) + c[3][n];
  T G[4][NC];
  for (int a = 0; a < 4; ++a) lean_christoffel(Gp, D, a, G[a]);
  T Gup[4];
  for (int cc = 0; cc < 4; ++cc) {
    T t[16];
    for (int n = 0; n < 16; ++n) t[n] = slot(Gp, n % 4, n / 4) * slot(G[cc], n % 4, n / 4);
    Gup[cc] = foldn(t, 16);
  }
  for (int n = 0; n < NC; ++n) {
    int a, b;
    unpair(n, a, b);
    T t[16];
    for (int m = 0; m < 16; ++m) t[m] = slot(G[m % 4], m / 4, a) * slot(G[m / 4], m % 4, b);
    T t2 = foldn(t, 16);
    T t4 = G[0][n] * Hl[0] + G[1][n] * Hl[1] + G[2][n] * Hl[2] + G[3][n] * Hl[3];
    T t5 = Gup[0] * D[0][n] + Gup[1] * D[1][n] + Gup[2] * D[2][n] + Gup[3] * D[3][n];
    S[n] = S[n] + (-T(2) * t2 - (dHl[a][b] + dHl[b][a]) + T(2) * t4 - t5);
  }
  if (g0 != T(0)) {
    T GH[4], Cup[4], Cl[4];
    for (int cc = 0; cc < 4; ++cc) {
      T t[4];
      for (int x = 0; x < 4; ++x) t[x] = slot(Gp, cc, x) * Hl[x];
      GH[cc] = fold4(t);
    }
    for (int cc = 0; cc < 4; ++cc) Cup[cc] = Gup[cc] + GH[cc];
    for (int cc = 0; cc < 4; ++cc) {
      T t[4];
      for (int x = 0; x < 4; ++x) t[x] = slot(gp, cc, x) * Cup[x];
      Cl[cc] = fold4(t);
    }
    T tt[4];
    for (int x = 0; x < 4; ++x) tt[x] = slot(Gp, 0, x) * Cl[x];
    T tC = -C.alpha * fold4(tt);
    T tl1 = -C.alpha;
    for (int n = 0; n < NC; ++n) {
      int a, b;
      unpair(n, a, b);
      T z = T(0);
      S[n] = S[n] + g0 * (((a == 0 ? tl1 * Cl[b] : z) + (b == 0 ? tl1 * Cl[a] : z)) -
                          (T(1) + g2) * gp[n] * tC);
    }
  }
  T f = -(C.alpha * C.sqrtg);
  for (int n = 0; n < NC; ++n) msrc[n] = f * S[n];
}

// _dgu_row (src/pointwise.jl:775-778)
template <class T> static inline void dgu_row(const T* Gp, const T* dg, int a, T out[4]) {
  T v[4];
  for (int d = 0; d < 4; ++d) {
    T t[4];
    for (int c = 0; c < 4; ++c) t[c] = slot(Gp, a, c) * slot(dg, c, d);
    v[d] = fold4(t);
  }
  for (int b = 0; b < 4; ++b) {
    T t[4];
    for (int d = 0; d < 4; ++d) t[d] = v[d] * slot(Gp, d, b);
    out[b] = -fold4(t);
  }
}

// src/pointwise.jl:754-771
template <class T>
static inline void metric_divergences(const Coef<T>& C, const T* const dh[3], T& divb, T divA[3]) {
  T Gp[NC];
  pack10(C.gu4, Gp);
  T gutt = C.gu4[0][0];
  T r1[3][4], ri[3][4];
  for (int i = 0; i < 3; ++i) {
    dgu_row(Gp, dh[i], 0, r1[i]);
    dgu_row(Gp, dh[i], i + 1, ri[i]);
  }
  T tb[3];
  for (int i = 0; i < 3; ++i) tb[i] = -(r1[i][i + 1] + C.beta[i] * r1[i][0]) / gutt;
  divb = (tb[0] + tb[1]) + tb[2];
  T da[3], ds[3];
  for (int i = 0; i < 3; ++i) da[i] = C.alpha * C.alpha * C.alpha * r1[i][0] / T(2);
  for (int i = 0; i < 3; ++i) {
    T t[9];
    for (int m = 0; m < 9; ++m) t[m] = C.gamu[m % 3][m / 3] * slot(dh[i], m % 3 + 1, m / 3 + 1);
    ds[i] = C.sqrtg * foldn(t, 9) / T(2);
  }
  for (int k = 0; k < 3; ++k) {
    T t[3];
    for (int i = 0; i < 3; ++i)
      t[i] = da[i] * C.sqrtg * C.gamu[i][k] + C.alpha * ds[i] * C.gamu[i][k] +
             C.alpha * C.sqrtg *
                 (ri[i][k + 1] + C.beta[k] * r1[i][i + 1] + C.beta[i] * r1[i][k + 1] +
                  C.beta[i] * C.beta[k] * r1[i][0]);
    divA[k] = (t[0] + t[1]) + t[2];
  }
}

// src/pointwise.jl:462-500: dbeta[i][j] = d_i beta^j, dA[i][j][k] = d_i (a sqrtg gamma^{jk})
template <class T>
static inline void metric_derivatives(const Coef<T>& C, const T* const dh[3], T dal[3],
                                      T dbeta[3][3], T dA[3][3][3]) {
  T gutt = C.gu4[0][0];
  T dgl[3][4][4], dgu[3][4][4];
  for (int i = 0; i < 3; ++i) {
    sym4(dh[i], dgl[i]);
    T tmp[4][4];
    for (int a = 0; a < 4; ++a)
      for (int d = 0; d < 4; ++d) {
        T s = C.gu4[a][0] * dgl[i][0][d];
        for (int c = 1; c < 4; ++c) s = s + C.gu4[a][c] * dgl[i][c][d];
        tmp[a][d] = s;
      }
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) {
        T s = tmp[a][0] * C.gu4[0][b];
        for (int d = 1; d < 4; ++d) s = s + tmp[a][d] * C.gu4[d][b];
        dgu[i][a][b] = -s;
      }
  }
  for (int i = 0; i < 3; ++i) dal[i] = C.alpha * C.alpha * C.alpha * dgu[i][0][0] / T(2);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) dbeta[i][j] = -(dgu[i][0][j + 1] + C.beta[j] * dgu[i][0][0]) / gutt;
  T ds[3];
  for (int i = 0; i < 3; ++i) {
    bool first = true;
    T s = T(0);
    for (int k = 0; k < 3; ++k)
      for (int j = 0; j < 3; ++j) {
        T t = C.gamu[j][k] * dgl[i][j + 1][k + 1];
        s = first ? t : s + t;
        first = false;
      }
    ds[i] = C.sqrtg * s / T(2);
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) {
        T dgu_jk = dgu[i][j + 1][k + 1] + C.beta[k] * dgu[i][0][j + 1] + C.beta[j] * dgu[i][0][k + 1] +
                   C.beta[j] * C.beta[k] * dgu[i][0][0];
        dA[i][j][k] = dal[i] * C.sqrtg * C.gamu[j][k] + C.alpha * ds[i] * C.gamu[j][k] +
                      C.alpha * C.sqrtg * dgu_jk;
      }
}

// src/pointwise.jl:818-850. ddh[n] in (xx,xy,xz,yy,yz,zz) order.
template <class T>
static inline void gh_node_rhs_expanded(const T* h, const T* Pi, const T* const dh[3],
                                        const T* const dPi[3], const T* const ddh[6],
                                        const T Hl[4], const T dHl[4][4], T g0, T g2, T* dth,
                                        T* dtPi) {
  Coef<T> C;
  metric_quantities(h, C);
  T a_div = C.alpha / C.sqrtg;
  T a_mul = C.alpha * C.sqrtg;
  T A[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) A[i][j] = a_mul * C.gamu[i][j];
  T dal[3], dbeta[3][3], dA[3][3][3];
  metric_derivatives(C, dh, dal, dbeta, dA);
  T divb = (dbeta[0][0] + dbeta[1][1]) + dbeta[2][2];
  T divA[3];
  for (int j = 0; j < 3; ++j) divA[j] = (dA[0][0][j] + dA[1][1][j]) + dA[2][2][j];
  for (int v = 0; v < NC; ++v)
    dth[v] = C.beta[0] * dh[0][v] + C.beta[1] * dh[1][v] + C.beta[2] * dh[2][v] + a_div * Pi[v];
  T dtPi0[NC];
  for (int v = 0; v < NC; ++v)
    dtPi0[v] = C.beta[0] * dPi[0][v] + C.beta[1] * dPi[1][v] + C.beta[2] * dPi[2][v] + divb * Pi[v] +
               A[0][0] * ddh[0][v] + T(2) * A[0][1] * ddh[1][v] + T(2) * A[0][2] * ddh[2][v] +
               A[1][1] * ddh[3][v] + T(2) * A[1][2] * ddh[4][v] + A[2][2] * ddh[5][v] +
               divA[0] * dh[0][v] + divA[1] * dh[1][v] + divA[2] * dh[2][v];
  T dg[4][4][4];
  dg4(dth, dh, dg);
  T msrc[NC];
  gh_node_source(C, dg, Hl, dHl, g0, g2, msrc);
  for (int v = 0; v < NC; ++v) dtPi[v] = dtPi0[v] + msrc[v];
}

// src/pointwise.jl:530-546: the chain rule of metric_derivatives along one direction, with
// d sqrt(gamma) and d gamma^{jk} returned apart (the monitors take them along time as well)
template <class T>
static inline void metric_derivatives_along(const Coef<T>& C, const T* dg10, T& dal, T dbeta[3], T& dsq,
                                            T dgamu[3][3]) {
  T gutt = C.gu4[0][0];
  T dgl[4][4], tmp[4][4], dgu[4][4];
  sym4(dg10, dgl);
  for (int a = 0; a < 4; ++a)
    for (int d = 0; d < 4; ++d) {
      T s = C.gu4[a][0] * dgl[0][d];
      for (int c = 1; c < 4; ++c) s = s + C.gu4[a][c] * dgl[c][d];
      tmp[a][d] = s;
    }
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      T s = tmp[a][0] * C.gu4[0][b];
      for (int d = 1; d < 4; ++d) s = s + tmp[a][d] * C.gu4[d][b];
      dgu[a][b] = -s;
    }
  dal = C.alpha * C.alpha * C.alpha * dgu[0][0] / T(2);
  for (int j = 0; j < 3; ++j) dbeta[j] = -(dgu[0][j + 1] + C.beta[j] * dgu[0][0]) / gutt;
  T s = T(0);
  bool first = true;
  for (int k = 0; k < 3; ++k)
    for (int j = 0; j < 3; ++j) {
      T t = C.gamu[j][k] * dgl[j + 1][k + 1];
      s = first ? t : s + t;
      first = false;
    }
  dsq = C.sqrtg * s / T(2);
  for (int j = 0; j < 3; ++j)
    for (int k = 0; k < 3; ++k)
      dgamu[j][k] = dgu[j + 1][k + 1] + C.beta[k] * dgu[0][j + 1] + C.beta[j] * dgu[0][k + 1] +
                    C.beta[j] * C.beta[k] * dgu[0][0];
}

// src/pointwise.jl:947-962: C^mu = g^{ab} Gamma^mu_{ab} + H^mu, with the inverse of g formed here
// (a general 4x4 inverse) and dgl[a][b][c] = d_c g_ab, the derivative axis last
template <class T>
static inline void gauge_constraint_at_node(const T g[4][4], const T dgl[4][4][4], const T Hup[4], T out[4]) {
  T gu[4][4];
  inv4(g, gu);
  T Gl[4][4][4], G[4][4][4];
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b)
      for (int c = 0; c < 4; ++c) Gl[a][b][c] = (dgl[a][c][b] + dgl[a][b][c] - dgl[b][c][a]) / T(2);
  for (int m = 0; m < 4; ++m)
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) {
        T s = gu[m][0] * Gl[0][a][b];
        for (int c = 1; c < 4; ++c) s = s + gu[m][c] * Gl[c][a][b];
        G[m][a][b] = s;
      }
  for (int m = 0; m < 4; ++m) {
    T s = T(0);
    bool first = true;
    for (int b = 0; b < 4; ++b)
      for (int a = 0; a < 4; ++a) {
        T t = gu[a][b] * G[m][a][b];
        s = first ? t : s + t;
        first = false;
      }
    out[m] = s + Hup[m];
  }
}

// src/constraints.jl:136-190: the ADM Hamiltonian and momentum constraints from the
// four-dimensional Ricci tensor, dg[a][b][c] = d_a g_bc and ddg[a][b][c][d] = d_a d_b g_cd
// (derivative axes first):
//   R_ab = d_c Gamma^c_ab - d_b Gamma^c_ca + Gamma^c_cd Gamma^d_ab - Gamma^c_bd Gamma^d_ca
//   H = 2 R_nn + R,   M_i = -n^a (R_ai - g_ai R / 2),   n = (1, -beta) / alpha
template <class T>
static inline void adm_constraints_at_node(const T g4[4][4], const T gu4[4][4], T alpha, const T beta[3],
                                           const T dg[4][4][4], const T ddg[4][4][4][4], T& ham, T mom[3]) {
  T dgu[4][4][4];
  for (int e = 0; e < 4; ++e) {
    T tmp[4][4];
    for (int a = 0; a < 4; ++a)
      for (int d = 0; d < 4; ++d) {
        T s = gu4[a][0] * dg[e][0][d];
        for (int c = 1; c < 4; ++c) s = s + gu4[a][c] * dg[e][c][d];
        tmp[a][d] = s;
      }
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) {
        T s = tmp[a][0] * gu4[0][b];
        for (int d = 1; d < 4; ++d) s = s + tmp[a][d] * gu4[d][b];
        dgu[e][a][b] = -s;
      }
  }
  T Gl[4][4][4], G4[4][4][4], Gtr[4];
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b)
      for (int c = 0; c < 4; ++c) Gl[a][b][c] = (dg[b][a][c] + dg[c][a][b] - dg[a][b][c]) / T(2);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b)
      for (int c = 0; c < 4; ++c) {
        T s = gu4[a][0] * Gl[0][b][c];
        for (int x = 1; x < 4; ++x) s = s + gu4[a][x] * Gl[x][b][c];
        G4[a][b][c] = s;
      }
  for (int d = 0; d < 4; ++d) Gtr[d] = ((G4[0][0][d] + G4[1][1][d]) + G4[2][2][d]) + G4[3][3][d];
  T R[4][4];
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      // A_ab = d_c Gamma^c_ab, B_ab = d_b Gamma^c_ca, each as its two sums (c fastest)
      T A1 = T(0), A2 = T(0), B1 = T(0), B2 = T(0);
      bool first = true;
      for (int d = 0; d < 4; ++d)
        for (int c = 0; c < 4; ++c) {
          T a1 = dgu[c][c][d] * Gl[d][a][b];
          T a2 = gu4[c][d] * (ddg[c][a][d][b] + ddg[c][b][d][a] - ddg[c][d][a][b]) / T(2);
          T b1 = dgu[b][c][d] * Gl[d][c][a];
          T b2 = gu4[c][d] * (ddg[b][c][d][a] + ddg[b][a][d][c] - ddg[b][d][c][a]) / T(2);
          A1 = first ? a1 : A1 + a1;
          A2 = first ? a2 : A2 + a2;
          B1 = first ? b1 : B1 + b1;
          B2 = first ? b2 : B2 + b2;
          first = false;
        }
      T q1 = Gtr[0] * G4[0][a][b];
      for (int d = 1; d < 4; ++d) q1 = q1 + Gtr[d] * G4[d][a][b];
      T q2 = T(0);
      first = true;
      for (int d = 0; d < 4; ++d)
        for (int c = 0; c < 4; ++c) {
          T t = G4[c][b][d] * G4[d][c][a];
          q2 = first ? t : q2 + t;
          first = false;
        }
      R[a][b] = (A1 + A2) - (B1 + B2) + q1 - q2;
    }
  T Rs = T(0);
  bool first = true;
  for (int b = 0; b < 4; ++b)
    for (int a = 0; a < 4; ++a) {
      T t = gu4[a][b] * R[a][b];
      Rs = first ? t : Rs + t;
      first = false;
    }
  T n[4] = {T(1) / alpha, -beta[0] / alpha, -beta[1] / alpha, -beta[2] / alpha};
  T Rnn = T(0);
  first = true;
  for (int b = 0; b < 4; ++b)
    for (int a = 0; a < 4; ++a) {
      T t = R[a][b] * n[a] * n[b];
      Rnn = first ? t : Rnn + t;
      first = false;
    }
  ham = T(2) * Rnn + Rs;
  for (int i = 0; i < 3; ++i) {
    T s = n[0] * (R[0][i + 1] - g4[0][i + 1] * Rs / T(2));
    for (int a = 1; a < 4; ++a) s = s + n[a] * (R[a][i + 1] - g4[a][i + 1] * Rs / T(2));
    mom[i] = -s;
  }
}

// src/pointwise.jl:667-698; Sij symmetric, S3 = (S_x, S_y, S_z)
template <class T>
static inline void matter_source(const Coef<T>& C, T rho, const T S3[3], const T Sij[3][3], T* out) {
  const T c8 = T(8) * T(M_PI);
  const T c16 = T(16) * T(M_PI);
  const T* b = C.beta;
  T S11 = Sij[0][0], S21 = Sij[1][0], S31 = Sij[2][0], S22 = Sij[1][1], S32 = Sij[2][1], S33 = Sij[2][2];
  T Sb1 = S11 * b[0] + S21 * b[1] + S31 * b[2];
  T Sb2 = S21 * b[0] + S22 * b[1] + S32 * b[2];
  T Sb3 = S31 * b[0] + S32 * b[1] + S33 * b[2];
  T bS = b[0] * S3[0] + b[1] * S3[1] + b[2] * S3[2];
  T Ttt = C.alpha * C.alpha * rho - T(2) * (C.alpha * bS) + (b[0] * Sb1 + b[1] * Sb2 + b[2] * Sb3);
  T Tt1 = Sb1 - C.alpha * S3[0];
  T Tt2 = Sb2 - C.alpha * S3[1];
  T Tt3 = Sb3 - C.alpha * S3[2];
  T trS = C.gamu[0][0] * S11 + C.gamu[1][1] * S22 + C.gamu[2][2] * S33 +
          T(2) * (C.gamu[1][0] * S21 + C.gamu[2][0] * S31 + C.gamu[2][1] * S32);
  T tr8 = c8 * (trS - rho);
  T a = C.alpha * C.sqrtg;
  const T* g = &C.g4[0][0];
  (void)g;
  out[0] = a * (c16 * Ttt - C.g4[0][0] * tr8);
  out[1] = a * (c16 * Tt1 - C.g4[1][0] * tr8);
  out[2] = a * (c16 * Tt2 - C.g4[2][0] * tr8);
  out[3] = a * (c16 * Tt3 - C.g4[3][0] * tr8);
  out[4] = a * (c16 * S11 - C.g4[1][1] * tr8);
  out[5] = a * (c16 * S21 - C.g4[2][1] * tr8);
  out[6] = a * (c16 * S31 - C.g4[3][1] * tr8);
  out[7] = a * (c16 * S22 - C.g4[2][2] * tr8);
  out[8] = a * (c16 * S32 - C.g4[3][2] * tr8);
  out[9] = a * (c16 * S33 - C.g4[3][3] * tr8);
}

}  // namespace orc
