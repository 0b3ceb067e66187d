// TEST INFRASTRUCTURE -- part of the CPU oracle (see stencils.hpp).
//
// SIMD lanes for the oracle's right-hand side, the counterpart of the reference's CPU kernel
// on SIMD.jl's Vec{W,T} (src/lanes.jl:1-135, gh_rhs_lanes! src/evolution.jl:698-790): W
// neighbouring points along x evaluated as one, every operation lane by lane in the scalar
// order, so that (with no contraction into fused multiply-adds, as this oracle is built) each
// lane's numbers are the scalar code's bit for bit. W is the host's register width in doubles,
// fixed when the oracle is compiled (ORC_SIMD_W): 8 for an AVX-512 build, 4 for AVX2.
#pragma once
#include <cmath>

#ifndef ORC_SIMD_W
#define ORC_SIMD_W 4
#endif

namespace orc {

template <int W> struct VecOf;
template <> struct VecOf<4> {
  typedef double type __attribute__((vector_size(32)));
};
template <> struct VecOf<8> {
  typedef double type __attribute__((vector_size(64)));
};

template <int W> struct Lane {
  typedef typename VecOf<W>::type V;
  V v;
  Lane() : v{} {}
  Lane(double c) {
    for (int l = 0; l < W; ++l) v[l] = c;
  }
  static Lane load(const double* p) {
    Lane r;
    __builtin_memcpy(&r.v, p, sizeof(V));
    return r;
  }
  void store_lane(int l, double* p) const { *p = v[l]; }
};
template <int W> static inline Lane<W> mk(typename Lane<W>::V x) {
  Lane<W> r;
  r.v = x;
  return r;
}
template <int W> static inline Lane<W> operator+(const Lane<W>& a, const Lane<W>& b) { return mk<W>(a.v + b.v); }
template <int W> static inline Lane<W> operator-(const Lane<W>& a, const Lane<W>& b) { return mk<W>(a.v - b.v); }
template <int W> static inline Lane<W> operator*(const Lane<W>& a, const Lane<W>& b) { return mk<W>(a.v * b.v); }
template <int W> static inline Lane<W> operator/(const Lane<W>& a, const Lane<W>& b) { return mk<W>(a.v / b.v); }
template <int W> static inline Lane<W> operator-(const Lane<W>& a) { return mk<W>(-a.v); }
// a choice made for the group: the damping terms are formed where any lane has a nonzero rate
// (_anynonzero, src/lanes.jl); adding a zero rate's terms leaves a lane's value unchanged
template <int W> static inline bool operator!=(const Lane<W>& a, const Lane<W>& b) {
  for (int l = 0; l < W; ++l)
    if (a.v[l] != b.v[l]) return true;
  return false;
}
// lane by lane: a where c > 0, else b
template <int W> static inline Lane<W> select_pos(const Lane<W>& c, const Lane<W>& a, const Lane<W>& b) {
  Lane<W> r;
  for (int l = 0; l < W; ++l) r.v[l] = c.v[l] > 0 ? a.v[l] : b.v[l];
  return r;
}
template <int W> static inline Lane<W> sqrt(const Lane<W>& a) {
  Lane<W> r;
  for (int l = 0; l < W; ++l) r.v[l] = std::sqrt(a.v[l]);
  return r;
}

// a working-array or state value at p: one double, or W neighbouring ones along x
template <class T> struct Loader {
  static T at(const double* p) { return T(*p); }
};
template <int W> struct Loader<Lane<W>> {
  static Lane<W> at(const double* p) { return Lane<W>::load(p); }
};
template <class T> static inline T ldw(const double* p) { return Loader<T>::at(p); }

// a per-point profile at the group's points: f(l) is lane l's value
template <class T> struct PerLane {
  template <class F> static T make(F f) { return T(f(0)); }
};
template <int W> struct PerLane<Lane<W>> {
  template <class F> static Lane<W> make(F f) {
    Lane<W> r;
    for (int l = 0; l < W; ++l) r.v[l] = f(l);
    return r;
  }
};

}  // namespace orc
