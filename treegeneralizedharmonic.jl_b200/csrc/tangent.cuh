// A value with one directional derivative: forward-mode differentiation of the right-hand
// side, its dissipation and the RK4 step along one direction of the parameters (the interior
// layer's rho_max and ramp width, the damping strength) and of the initial data (the
// perturbation amplitudes). Exact to roundoff: each operation carries its derivative.
#pragma once
#include <cmath>

#ifndef TGH_HD
#define TGH_HD __host__ __device__ __forceinline__
#endif

namespace tgh {

// the scalar overloads stay visible beside the ones below
using ::exp;
using ::fma;
using ::sqrt;

struct Tan {
  double v, d;
  TGH_HD Tan() {}
  TGH_HD Tan(double c) : v(c), d(0.0) {}
  TGH_HD Tan(double a, double b) : v(a), d(b) {}
};
TGH_HD Tan operator+(const Tan& a, const Tan& b) { return Tan(a.v + b.v, a.d + b.d); }
TGH_HD Tan operator-(const Tan& a, const Tan& b) { return Tan(a.v - b.v, a.d - b.d); }
TGH_HD Tan operator-(const Tan& a) { return Tan(-a.v, -a.d); }
TGH_HD Tan operator*(const Tan& a, const Tan& b) { return Tan(a.v * b.v, fma(a.d, b.v, a.v * b.d)); }
TGH_HD Tan operator/(const Tan& a, const Tan& b) {
  const double q = a.v / b.v;
  return Tan(q, (a.d - q * b.d) / b.v);
}
TGH_HD Tan& operator+=(Tan& a, const Tan& b) { return a = a + b; }
TGH_HD Tan& operator-=(Tan& a, const Tan& b) { return a = a - b; }
TGH_HD Tan fma(const Tan& a, const Tan& b, const Tan& c) {
  return Tan(fma(a.v, b.v, c.v), fma(a.d, b.v, fma(a.v, b.d, c.d)));
}
TGH_HD Tan sqrt(const Tan& a) {
  const double s = sqrt(a.v);
  return Tan(s, a.d / (2.0 * s));
}
TGH_HD Tan dsqrt(const Tan& a) { return sqrt(a); }
TGH_HD Tan exp(const Tan& a) {
  const double e = exp(a.v);
  return Tan(e, e * a.d);
}
// branches follow the value
TGH_HD bool operator>(const Tan& a, const Tan& b) { return a.v > b.v; }
TGH_HD bool operator<(const Tan& a, const Tan& b) { return a.v < b.v; }
TGH_HD bool operator==(const Tan& a, const Tan& b) { return a.v == b.v; }
TGH_HD bool operator!=(const Tan& a, const Tan& b) { return a.v != b.v; }
TGH_HD double value(double a) { return a; }
TGH_HD double value(float a) { return a; }
TGH_HD double value(const Tan& a) { return a.v; }
TGH_HD double tangent(double) { return 0.0; }
TGH_HD double tangent(float) { return 0.0; }
TGH_HD double tangent(const Tan& a) { return a.d; }

// the element offset from the value working array to its tangent (set before a tangent launch)
__constant__ long c_tan_off;

}  // namespace tgh
