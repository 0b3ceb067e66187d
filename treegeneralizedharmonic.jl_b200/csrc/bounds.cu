// The range projection of the stage limiter (src/bounds.jl): gh_bounds_kernel! (:635-663)
// applying bounds_project (:458-593) at every owned point inside the gate r < r_gate, written
// back only where it fired.
//
// This unit is compiled without floating-point contraction (-fmad=false): the projection tests
// values that a previous call computed and stored, and its idempotence (a second call leaves a
// repaired state alone, bit for bit) rests on every product and sum being rounded on its own,
// as the reference's scalar arithmetic is. Division and square root are the IEEE ones.
#include <cfloat>

#include "bounds.cuh"

namespace tgh {

namespace {

constexpr double EPS = DBL_EPSILON;
constexpr int SLACK = 8, PASSES = 4, SWEEPS = 16;

// the 3+1 split of the offset metric m (4x4, row-major) in ADM variables
struct Split {
  double g[6], beta[3], detg, bb, a2;
};
__device__ Split split(const double m[16]) {
  Split s;
  const double g11 = 1.0 + m[5], g12 = m[9], g13 = m[13], g22 = 1.0 + m[10], g23 = m[14], g33 = 1.0 + m[15];
  const double b1 = m[4], b2 = m[8], b3 = m[12];
  const double c11 = g22 * g33 - g23 * g23, c12 = g13 * g23 - g12 * g33, c13 = g12 * g23 - g13 * g22;
  const double c22 = g11 * g33 - g13 * g13, c23 = g12 * g13 - g11 * g23, c33 = g11 * g22 - g12 * g12;
  s.detg = g11 * c11 + g12 * c12 + g13 * c13;
  const double qf = b1 * (c11 * b1 + c12 * b2 + c13 * b3) + b2 * (c12 * b1 + c22 * b2 + c23 * b3) +
                    b3 * (c13 * b1 + c23 * b2 + c33 * b3);
  s.bb = qf / s.detg;
  s.a2 = (1.0 - m[0]) + s.bb;
  s.g[0] = g11; s.g[1] = g12; s.g[2] = g13; s.g[3] = g22; s.g[4] = g23; s.g[5] = g33;
  s.beta[0] = b1; s.beta[1] = b2; s.beta[2] = b3;
  return s;
}

// Sylvester's criterion with each minor above 16 eps of its terms: true means certainly
// positive definite
__device__ bool certainly_posdef(double a11, double a12, double a13, double a22, double a23, double a33) {
  const double tol = 16 * EPS;
  const double m2 = a11 * a22 - a12 * a12, e2 = fabs(a11 * a22) + a12 * a12;
  const double c1 = a22 * a33 - a23 * a23, c2 = a12 * a33 - a23 * a13, c3 = a12 * a23 - a22 * a13;
  const double m3 = a11 * c1 - a12 * c2 + a13 * c3;
  const double e3 = fabs(a11) * (fabs(a22 * a33) + a23 * a23) + fabs(a12) * (fabs(a12 * a33) + fabs(a23 * a13)) +
                    fabs(a13) * (fabs(a12 * a23) + fabs(a22 * a13));
  return (a11 > 0.0) & (m2 > tol * e2) & (m3 > tol * e3);
}

// a cyclic-Jacobi rotation annihilating A[p][q] (A symmetric 3x3, row-major), accumulated in V
__device__ void rotate(double A[9], double V[9], int p, int q) {
  const double apq = A[3 * p + q];
  if (apq == 0.0) return;
  const double app = A[4 * p], aqq = A[4 * q];
  const double tau = (aqq - app) / (2 * apq);
  const double t = fabs(tau) > 1.0 / sqrt(EPS) ? 1.0 / (2 * tau) : copysign(1.0, tau) / (fabs(tau) + sqrt(1.0 + tau * tau));
  const double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
  const int r = 3 - p - q;
  const double arp = A[3 * r + p], arq = A[3 * r + q];
  A[4 * p] = app - t * apq;
  A[4 * q] = aqq + t * apq;
  A[3 * p + q] = A[3 * q + p] = 0.0;
  A[3 * r + p] = A[3 * p + r] = c * arp - s * arq;
  A[3 * r + q] = A[3 * q + r] = s * arp + c * arq;
  for (int i = 0; i < 3; ++i) {
    const double vp = V[3 * i + p], vq = V[3 * i + q];
    V[3 * i + p] = c * vp - s * vq;
    V[3 * i + q] = s * vp + c * vq;
  }
}

__device__ double clampj(double x, double lo, double hi) { return x > hi ? hi : (x < lo ? lo : x); }

// gamma's spectrum into [lmin, lmax]; g is kept unless an eigenvalue lies outside by more than
// the slack, and is then recomposed as V diag(clamped) V^T
__device__ bool clamp_spectrum(const double g[6], double lmin, double lmax, double out[6]) {
  for (int n = 0; n < 6; ++n) out[n] = g[n];
  const bool lo = certainly_posdef(g[0] - lmin, g[1], g[2], g[3] - lmin, g[4], g[5] - lmin);
  const bool hi = certainly_posdef(lmax - g[0], -g[1], -g[2], lmax - g[3], -g[4], lmax - g[5]);
  if (lo & hi) return false;
  double A[9] = {g[0], g[1], g[2], g[1], g[3], g[4], g[2], g[4], g[5]};
  double V[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int sweep = 0; sweep < SWEEPS; ++sweep) {
    const double off = A[1] * A[1] + A[2] * A[2] + A[5] * A[5];
    const double on = A[0] * A[0] + A[4] * A[4] + A[8] * A[8];
    if (!(off > EPS * EPS * on)) break;
    rotate(A, V, 0, 1);
    rotate(A, V, 0, 2);
    rotate(A, V, 1, 2);
  }
  const double lam[3] = {A[0], A[4], A[8]};
  const double S = fmax(fmax(fabs(lam[0]), fabs(lam[1])), fabs(lam[2]));
  const double sl = SLACK * EPS * S;
  bool inside = true;
  for (int k = 0; k < 3; ++k) inside = inside & ((lmin - sl <= lam[k]) & (lam[k] <= lmax + sl));
  if (inside) return false;
  double l2[3];
  for (int k = 0; k < 3; ++k) l2[k] = clampj(lam[k], lmin, lmax);
  auto rc = [&](int i, int j) {
    return V[3 * i] * l2[0] * V[3 * j] + V[3 * i + 1] * l2[1] * V[3 * j + 1] + V[3 * i + 2] * l2[2] * V[3 * j + 2];
  };
  out[0] = rc(0, 0);
  out[1] = rc(0, 1);
  out[2] = rc(0, 2);
  out[3] = rc(1, 1);
  out[4] = rc(1, 2);
  out[5] = rc(2, 2);
  return true;
}

// one application of the five steps (non-finite repair, spectrum, shift, lapse, momentum)
__device__ bool project_once(double h[10], double P[10], const BoundsArgs& B, bool& nonfinite) {
  const double slack = SLACK * EPS;
  bool fin = true;
  for (int v = 0; v < 10; ++v) fin = fin & isfinite(h[v]) & isfinite(P[v]);
  nonfinite = !fin;
  if (nonfinite)
    for (int v = 0; v < 10; ++v) {
      if (!isfinite(h[v])) h[v] = 0.0;
      if (!isfinite(P[v])) P[v] = 0.0;
    }
  // the offset metric as a 4x4, row-major, from the packed (tt,tx,ty,tz,xx,xy,xz,yy,yz,zz)
  double m[16] = {h[0], h[1], h[2], h[3], h[1], h[4], h[5], h[6], h[2], h[5], h[7], h[8], h[3], h[6], h[8], h[9]};
  const Split s0 = split(m);
  double g2[6];
  const bool gfire = clamp_spectrum(s0.g, B.lmin, B.lmax, g2);
  if (gfire) {
    m[5] = g2[0] - 1.0;
    m[6] = m[9] = g2[1];
    m[7] = m[13] = g2[2];
    m[10] = g2[3] - 1.0;
    m[11] = m[14] = g2[4];
    m[15] = g2[5] - 1.0;
  }
  const Split s1 = gfire ? split(m) : s0;
  const double bmax2 = B.bmax * B.bmax;
  const bool bfire = !(s1.bb <= bmax2 + slack * bmax2);
  if (bfire) {
    const double f = B.bmax / sqrt(s1.bb);
    for (int i = 0; i < 3; ++i) m[4 * (i + 1)] = m[i + 1] = f * s1.beta[i];
  }
  const Split s2 = bfire ? split(m) : s1;
  const double lo2 = B.amin * B.amin, hi2 = B.amax * B.amax;
  const double sa = slack * (1.0 + fabs(m[0]) + fabs(s2.bb));
  const bool alow = !(s2.a2 >= lo2 - sa), ahigh = !(s2.a2 <= hi2 + sa);
  const bool afire = alow | ahigh;
  if (afire) m[0] = (1.0 - (alow ? lo2 : hi2)) + s2.bb;
  const Split s3 = afire ? split(m) : s2;
  const bool hfire = gfire | bfire | afire;
  const bool raise = alow & (s0.a2 > 0.0) & (s0.detg > 0.0) & (s3.a2 > s0.a2);
  if (raise) {
    const double f = (sqrt(s0.a2) / sqrt(s3.a2)) * (sqrt(s3.detg) / sqrt(s0.detg));
    for (int v = 0; v < 10; ++v) P[v] = P[v] * f;
  }
  const double a = sqrt(s3.a2) / sqrt(s3.detg);
  double mx = fabs(a * P[0]);
  for (int v = 1; v < 10; ++v) {
    const double x = fabs(a * P[v]);
    mx = (x != x || mx != mx) ? __longlong_as_double(0x7ff8000000000000LL) : fmax(mx, x);
  }
  const bool kfire = !(mx <= B.kmax + slack * B.kmax);
  if (kfire) {
    const double f = B.kmax / mx;
    for (int v = 0; v < 10; ++v) P[v] = P[v] * f;
  }
  if (hfire) {
    h[0] = m[0]; h[1] = m[4]; h[2] = m[8]; h[3] = m[12]; h[4] = m[5];
    h[5] = m[9]; h[6] = m[13]; h[7] = m[10]; h[8] = m[14]; h[9] = m[15];
  }
  return nonfinite | hfire | raise | kfire;
}

__global__ void __launch_bounds__(128) bounds_kernel(const Case cs, const BoundsArgs B) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= B.npts) return;
  const int N1 = B.N1;
  const int b = (int)(p / B.S);
  const long ip = p - (long)b * B.S;
  const int k = (int)(ip / ((long)N1 * N1)), j = (int)((ip / N1) % N1), i = (int)(ip % N1);
  const double* bl = B.blk + 8 * b;
  double x[3];
  x[0] = __dadd_rn(bl[0], __dmul_rn(bl[4] + (double)i, bl[3]));
  x[1] = __dadd_rn(bl[1], __dmul_rn(bl[5] + (double)j, bl[3]));
  x[2] = __dadd_rn(bl[2], __dmul_rn(bl[6] + (double)k, bl[3]));
  const double r = interior_radius(cs, B.t, x);
  if (!(r < B.rgate)) return;
  double* q = B.u + (long)b * NV * B.S + ip;
  double h[10], P[10];
  for (int v = 0; v < 10; ++v) {
    h[v] = q[v * B.S];
    P[v] = q[(10 + v) * B.S];
  }
  bool nf = false;
  const bool hit = project_once(h, P, B, nf);
  if (hit)
    for (int pass = 0; pass < PASSES; ++pass) {
      double h2[10], P2[10];
      for (int v = 0; v < 10; ++v) {
        h2[v] = h[v];
        P2[v] = P[v];
      }
      bool nf2;
      if (!project_once(h2, P2, B, nf2)) break;
      for (int v = 0; v < 10; ++v) {
        h[v] = h2[v];
        P[v] = P2[v];
      }
    }
  if (hit)
    for (int v = 0; v < 10; ++v) {
      q[v * B.S] = h[v];
      q[(10 + v) * B.S] = P[v];
    }
  if (B.primary[p]) {
    if (hit) {
      atomicAdd(&B.counts[0], 1ull);
      atomicMax(&B.counts[2], (unsigned long long)__double_as_longlong(r));  // r >= 0: bits order as values
    }
    if (nf) atomicAdd(&B.counts[1], 1ull);
  }
}

}  // namespace

cudaError_t launch_bounds_projection(cudaStream_t s, const Case& cs, const BoundsArgs& a) {
  cudaError_t e = cudaMemsetAsync(a.counts, 0, 3 * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  bounds_kernel<<<(unsigned)((a.npts + 127) / 128), 128, 0, s>>>(cs, a);
  return cudaGetLastError();
}

}  // namespace tgh
