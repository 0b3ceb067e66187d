// TEST INFRASTRUCTURE -- a companion of the CPU oracle, not the oracle of parity.
//
// The ADM Hamiltonian and momentum constraints at one point with the four-dimensional Ricci
// tensor contracted in the order of the GPU monitor kernel: the first-derivative terms
//   (d_c g^{cd}) Gamma_{d,ab} - (d_b g^{cd}) Gamma_{d,ca} + Gamma^c_cd Gamma^d_ab - Gamma^c_bd Gamma^d_ca
// with d g^{-1} = -g^{-1} (d g) g^{-1} folded into the contractions, then the ten second
// derivatives of each metric component folded into the ten packed R_ab,
//   R_ab += X_ab + X_ba - (1/2) g^{cd} d_c d_d g_ab - (1/2) g^{cd} d_a d_b g_cd,
//   X_ab = (1/2) g^{cd} d_c d_a g_db.
// It is the same tensor as adm_constraints_at_node (src/constraints.jl:136-190), which the
// monitors' parity is checked against; this restatement exists so that (1) the kernel's
// reformulation is checked against the reference's assembly on the CPU and (2) the floating-
// point operations the kernel's contraction does are counted (one multiply-add = 2 flops).
// Inputs and outputs as adm_constraints_at_node.
#pragma once
#include "pointwise.hpp"

namespace orc {

template <class T>
static inline void adm_constraints_streamed(const T g4[4][4], const T gu4[4][4], T alpha, const T beta[3],
                                            const T dg[4][4][4], const T ddg[4][4][4][4], T& ham, T mom[3]) {
  int PR[NC], PCl[NC];
  for (int n = 0; n < NC; ++n) unpair(n, PR[n], PCl[n]);
  auto gu = [&](int n) { return gu4[PR[n]][PCl[n]]; };
  auto D = [&](int e, int n) { return dg[e][PR[n]][PCl[n]]; };
  // first-derivative terms, R_ab for the packed a <= b with b the larger index
  T G4[4][NC], R[NC];
  for (int a = 0; a < 4; ++a)
    for (int n = 0; n < NC; ++n) {
      const int b = PR[n], c = PCl[n];
      T s = T(0);
      for (int x = 0; x < 4; ++x)
        s = s + gu4[a][x] * (T(0.5) * ((D(b, pairindex(x, c)) + D(c, pairindex(x, b))) - D(x, n)));
      G4[a][n] = s;
    }
  T w[4] = {T(0), T(0), T(0), T(0)};
  for (int b = 0; b < 4; ++b) {
    T U[4][4];
    for (int c = 0; c < 4; ++c)
      for (int f = 0; f < 4; ++f) {
        T s = T(0);
        for (int e = 0; e < 4; ++e) s = s + gu4[c][e] * D(b, pairindex(e, f));
        U[c][f] = s;
      }
    for (int f = 0; f < 4; ++f) w[f] = w[f] + U[b][f];
    for (int a = 0; a <= b; ++a) {
      T r = T(0);
      for (int c = 0; c < 4; ++c)
        for (int f = 0; f < 4; ++f) r = r + U[c][f] * G4[f][pairindex(c, a)];
      for (int c = 0; c < 4; ++c)
        for (int d = 0; d < 4; ++d) r = r - G4[c][pairindex(b, d)] * G4[d][pairindex(c, a)];
      R[pairindex(a, b)] = r;
    }
  }
  T tw[4];
  for (int f = 0; f < 4; ++f)
    tw[f] = (((G4[0][pairindex(0, f)] + G4[1][pairindex(1, f)]) + G4[2][pairindex(2, f)]) + G4[3][pairindex(3, f)]) - w[f];
  for (int n = 0; n < NC; ++n)
    for (int f = 0; f < 4; ++f) R[n] = R[n] + tw[f] * G4[f][n];
  // second-derivative terms, one metric component v = (al be) at a time
  for (int v = 0; v < NC; ++v) {
    const int al = PR[v], be = PCl[v];
    T dv[NC];
    for (int m = 0; m < NC; ++m) dv[m] = ddg[PR[m]][PCl[m]][al][be];
    const T c3 = T(al == be ? -0.5 : -1.0) * gu(v);
    T tr = T(0);
    for (int m = 0; m < NC; ++m) {
      R[m] = R[m] + c3 * dv[m];
      tr = tr + (PR[m] == PCl[m] ? gu(m) : T(2) * gu(m)) * dv[m];
    }
    R[v] = R[v] + T(-0.5) * tr;
    for (int a = 0; a < 4; ++a) {
      T y = T(0);
      for (int c = 0; c < 4; ++c) y = y + gu4[c][al] * dv[pairindex(c, a)];
      R[pairindex(a, be)] = R[pairindex(a, be)] + T(a == be ? 1.0 : 0.5) * y;
      if (al != be) {
        T z = T(0);
        for (int c = 0; c < 4; ++c) z = z + gu4[c][be] * dv[pairindex(c, a)];
        R[pairindex(a, al)] = R[pairindex(a, al)] + T(a == al ? 1.0 : 0.5) * z;
      }
    }
  }
  // the contractions
  T Rs = T(0);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) Rs = Rs + gu4[a][b] * R[pairindex(a, b)];
  const T n[4] = {T(1) / alpha, -beta[0] / alpha, -beta[1] / alpha, -beta[2] / alpha};
  T Rnn = T(0);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) Rnn = Rnn + (R[pairindex(a, b)] * n[a]) * n[b];
  ham = T(2) * Rnn + Rs;
  for (int i = 0; i < 3; ++i) {
    T s = T(0);
    for (int a = 0; a < 4; ++a) s = s + n[a] * (R[pairindex(a, i + 1)] - (g4[a][i + 1] * Rs) * T(0.5));
    mom[i] = -s;
  }
}

}  // namespace orc
