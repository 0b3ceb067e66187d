// TEST INFRASTRUCTURE -- part of the CPU oracle. Only tests/, __graft_entry__.smoke()
// and bench.py's cpu_baseline leg may load it; the product never links it.
//
// Exact-rational finite-difference and Kreiss-Oliger weights, restating
// src/stencils.jl:59-157 (lagrange_derivative_weights, rational_derivative_weights,
// rational_dissipation_weights) and the single rounding of src/stencils.jl:170-174
// (each weight is the correctly rounded quotient of its exact numerator and denominator).
#pragma once
#include <cstdint>
#include <stdexcept>
#include <vector>

namespace orc {

typedef __int128 i128;

static inline i128 i128_abs(i128 a) { return a < 0 ? -a : a; }
static inline i128 i128_gcd(i128 a, i128 b) {
  a = i128_abs(a);
  b = i128_abs(b);
  while (b != 0) {
    i128 t = a % b;
    a = b;
    b = t;
  }
  return a == 0 ? 1 : a;
}

struct Rat {
  i128 n, d;  // d > 0, reduced
  Rat(i128 n_ = 0, i128 d_ = 1) : n(n_), d(d_) { norm(); }
  void norm() {
    if (d < 0) { n = -n; d = -d; }
    i128 g = i128_gcd(n, d);
    n /= g;
    d /= g;
  }
};
static inline Rat operator+(Rat a, Rat b) { return Rat(a.n * b.d + b.n * a.d, a.d * b.d); }
static inline Rat operator-(Rat a, Rat b) { return Rat(a.n * b.d - b.n * a.d, a.d * b.d); }
static inline Rat operator*(Rat a, Rat b) { return Rat(a.n * b.n, a.d * b.d); }
static inline Rat operator/(Rat a, Rat b) { return Rat(a.n * b.d, a.d * b.n); }

// src/stencils.jl:89-110: the m-th derivative at 0 of the Lagrange basis on `nodes`.
static inline std::vector<Rat> lagrange_derivative_weights(const std::vector<Rat>& ns, int m) {
  const int n = (int)ns.size();
  std::vector<Rat> ws(n);
  for (int i = 0; i < n; ++i) {
    std::vector<Rat> c{Rat(1)};
    Rat den(1);
    for (int k = 0; k < n; ++k) {
      if (k == i) continue;
      // multiply the polynomial c (low to high) by (x - ns[k])  (_polymul_linear)
      Rat a = Rat(0) - ns[k];
      std::vector<Rat> out(c.size() + 1);
      out[0] = a * c[0];
      for (size_t j = 1; j < c.size(); ++j) out[j] = c[j - 1] + a * c[j];
      out[c.size()] = c.back();
      c = out;
      den = den * (ns[i] - ns[k]);
    }
    if (m < n) {
      i128 fact = 1;
      for (int j = 2; j <= m; ++j) fact *= j;
      ws[i] = Rat(fact) * c[m] / den;
    } else {
      ws[i] = Rat(0);
    }
  }
  return ws;
}

// src/stencils.jl:124-134: centered order-q weights of d^m on nodes -q/2..q/2.
static inline std::vector<Rat> rational_derivative_weights(int q, int m) {
  if (q < 2 || q % 2 != 0) throw std::invalid_argument("q must be even and >= 2");
  if (m != 1 && m != 2) throw std::invalid_argument("m must be 1 or 2");
  const int r = q / 2;
  std::vector<Rat> ns;
  for (int j = -r; j <= r; ++j) ns.push_back(Rat(j));
  return lagrange_derivative_weights(ns, m);
}

static inline i128 binom(int n, int k) {
  i128 b = 1;
  for (int j = 1; j <= k; ++j) b = b * (n - k + j) / j;
  return b;
}

// src/stencils.jl:148-157: (-1)^{r+1} 2^{-2r} (D+D-)^r on unit spacing.
static inline std::vector<Rat> rational_dissipation_weights(int r) {
  if (r < 1) throw std::invalid_argument("r must be >= 1");
  const int sgn = ((r + 1) % 2 == 0) ? 1 : -1;
  const i128 den = (i128)1 << (2 * r);
  std::vector<Rat> w;
  for (int j = -r; j <= r; ++j) {
    const int e = r - j;  // (-1)^(r-j)
    const int s = (e % 2 == 0) ? 1 : -1;
    w.push_back(Rat((i128)sgn * s * binom(2 * r, r - j), den));
  }
  return w;
}

// One rounding: T(num) / T(den) (src/stencils.jl:170-174).
static inline std::vector<double> to_double(const std::vector<Rat>& w) {
  std::vector<double> o;
  for (auto& x : w) o.push_back((double)(int64_t)x.n / (double)(int64_t)x.d);
  return o;
}

struct Stencils {
  int q = 0, r = 0, rD = 0;
  std::vector<double> w1, w2, wD;  // sizes q+1, q+1, 2 rD + 1
  explicit Stencils(int q_) : q(q_), r(q_ / 2), rD(q_ / 2 + 1) {
    w1 = to_double(rational_derivative_weights(q, 1));
    w2 = to_double(rational_derivative_weights(q, 2));
    wD = to_double(rational_dissipation_weights(rD));
  }
};

}  // namespace orc
