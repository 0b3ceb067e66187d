// The tangent-linear right-hand side: the plain form's gh_rhs! (src/evolution.jl:258-388, with
// the interior's :damped static-core branches, src/evolution.jl:489-695) at one point per
// thread in Tan arithmetic, the head and the Pi components fused in one kernel, so that the
// coefficients never leave registers. du receives the right-hand side, dut its derivative
// along one direction: of the state (dut from the tangent of u alone) or also of one
// parameter of the interior or the damping. The values follow the FP64 kernels' operations and
// agree with them to roundoff (a few products are contracted into FMAs differently).
#pragma once
#include "rhs.cuh"

namespace tgh {

// the parameter a tangent differentiates along (besides the state's own tangent)
enum { TAN_STATE = 0, TAN_RHO_MAX = 1, TAN_RAMP = 2, TAN_DAMP_NEAR = 3 };

struct TanArgs {
  double* dut;  // the derivative of du, state layout
  int dir;      // TAN_*
};

// the quintic ramp of the interior profiles (src/interior.jl) and its derivative 30 u^2 (1 - u)^2
__device__ __forceinline__ Tan smoothstep_t(const Tan& s) {
  const double u = s.v < 0.0 ? 0.0 : (s.v > 1.0 ? 1.0 : s.v);
  double p = u * u * u * (10.0 + u * (6.0 * u - 15.0));
  p = p < 0.0 ? 0.0 : (p > 1.0 ? 1.0 : p);
  const double dp = (s.v <= 0.0 || s.v >= 1.0) ? 0.0 : 30.0 * u * u * (1.0 - u) * (1.0 - u);
  return Tan(p, dp * s.d);
}

// layer_profiles with the layer's parameters as the direction asks: rho_max, or the ramp width
// (w_ramp and rho_ramp together)
__device__ __forceinline__ void layer_profiles_t(const Case& c, double r, int dir, Tan& w, Tan& rho) {
  const double s = (r - c.r0) / (c.r1 - c.r0);
  const double dr = dir == TAN_RAMP ? 1.0 : 0.0;
  w = smoothstep_t(Tan(s) / Tan(c.w_ramp, dr));
  rho = c.interior == TGH_INT_FROZEN
            ? Tan(0.0)
            : Tan(c.rho_max, dir == TAN_RHO_MAX ? 1.0 : 0.0) * smoothstep_t(Tan(1.0 - s) / Tan(c.rho_ramp, dr));
}

// damping_rate with the damping strength (gamma0, or the Gaussian's near value) as a parameter
__device__ __forceinline__ Tan damping_rate_t(const Case& c, double t, const double* x, int dir) {
  const double seed = dir == TAN_DAMP_NEAR ? 1.0 : 0.0;
  if (c.damping == TGH_DAMP_CONSTANT) return Tan(c.g0, seed);
  const double d1 = x[0] - (c.dc0[0] + t * c.dv[0]), d2 = x[1] - (c.dc0[1] + t * c.dv[1]),
               d3 = x[2] - (c.dc0[2] + t * c.dv[2]);
  const double r2 = d1 * d1 + d2 * d2 + d3 * d3;
  const double e = exp(-r2 / (2.0 * c.dwidth * c.dwidth));
  return Tan(c.dfar + (c.dnear - c.dfar) * e, seed * e);
}

template <int Q, bool DISS, bool INT>
__global__ void __launch_bounds__(128) rhs_tangent_kernel(const Case cs, const RhsArgs A, const TanArgs ta) {
  const long p = A.p0 + (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= A.p1) return;
  const PointIdx q = point_index(A, p);
  const long S = (long)A.N1 * A.N1 * A.N1;
  const long sv = (long)A.Wx * A.Wd * A.Wd;
  const long s1 = 1, s2 = A.Wx, s3 = (long)A.Wx * A.Wd;
  const double* wk = A.work + q.wo;
  const double inv_h = 1.0 / q.h;
  double* du = A.du + (long)q.b * NV * S + q.ip;
  double* dut = ta.dut + (long)q.b * NV * S + q.ip;
  auto put = [&](int v, const Tan& val) {
    du[v * S] = val.v;
    dut[v * S] = val.d;
  };
  Tan w = Tan(1.0), rho = Tan(0.0);
  double r = 0.0;
  if (INT) {
    r = interior_radius(cs, A.t, q.x);
    const bool frozen = cs.interior == TGH_INT_PASTED ? r < cs.r1 : r < cs.r0;
    if (frozen) {  // a core at rest: du = 0 (a moving core is refused before launch)
      for (int v = 0; v < NV; ++v) put(v, Tan(0.0));
      return;
    }
    if (r < cs.r1) layer_profiles_t(cs, r, ta.dir, w, rho);
  }
  const bool layer = INT && r < cs.r1;
  Tan hv[NC], dh0[NC], dh1[NC], dh2[NC], dth[NC], eh;
  Coef<Tan> C;
  rhs_dt<Q, DISS, Tan>(cs, A, wk, sv, q.x, inv_h, hv, dh0, dh1, dh2, C, dth, eh);
  double he[NC], Pe[NC];
  if (layer) rn_background_state(cs, A.t, q.x, he, Pe);
#pragma unroll 1
  for (int v = 0; v < NC; ++v) put(v, layer ? w * dth[v] - rho * (ld<Tan>(wk + v * sv) - Tan(he[v])) : dth[v]);
  // the Pi coefficients, kept in registers
  const Tan* dh[3] = {dh0, dh1, dh2};
  Tan divb, divA[3];
  metric_divergences(C, dh, divb, divA);
  const Tan am = C.alpha * C.sqrtg;
  const Tan Axx = am * C.gamu[0], Axy = Tan(2.0) * am * C.gamu[1], Axz = Tan(2.0) * am * C.gamu[2];
  const Tan Ayy = am * C.gamu[3], Ayz = Tan(2.0) * am * C.gamu[4], Azz = am * C.gamu[5];
  Tan msrc[NC];
  const Tan* D[4] = {dth, dh0, dh1, dh2};
  rhs_source(cs, A, q.b, q.ip, damping_rate_t(cs, A.t, q.x, ta.dir), hv, C, D, msrc);
  const Tan ih = Tan(inv_h), ih2 = Tan(inv_h * inv_h);
#pragma unroll 1
  for (int v = 0; v < NC; ++v) {
    const double* ph = wk + v * sv;
    const double* pp = ph + NC * sv;
    const Tan hc = ld<Tan>(ph), pc = ld<Tan>(pp);
    Tan s = C.beta[0] * (ih * st_d1<Q, Tan>(pp, s1));
    s = fma(C.beta[1], ih * st_d1<Q, Tan>(pp, s2), s);
    s = fma(C.beta[2], ih * st_d1<Q, Tan>(pp, s3), s);
    s = fma(divb, pc, s);
    s = fma(divA[0], ih * st_d1<Q, Tan>(ph, s1), s);
    s = fma(divA[1], ih * st_d1<Q, Tan>(ph, s2), s);
    s = fma(divA[2], ih * st_d1<Q, Tan>(ph, s3), s);
    Tan p2 = Axx * st_d2<Q, Tan>(ph, s1, hc);
    p2 = fma(Ayy, st_d2<Q, Tan>(ph, s2, hc), p2);
    p2 = fma(Azz, st_d2<Q, Tan>(ph, s3, hc), p2);
    p2 = fma(Axy, st_mixed<Q, Tan>(ph, s1, s2), p2);
    p2 = fma(Axz, st_mixed<Q, Tan>(ph, s1, s3), p2);
    p2 = fma(Ayz, st_mixed<Q, Tan>(ph, s2, s3), p2);
    s = fma(ih2, p2, s);
    if (DISS) s = fma(eh, st_ko<Q, Tan>(pp, s1, pc) + st_ko<Q, Tan>(pp, s2, pc) + st_ko<Q, Tan>(pp, s3, pc), s);
    if (layer) {
      const Tan m = w * msrc[v] - rho * (pc - Tan(Pe[v]));
      put(NC + v, fma(w, s, m));
    } else {
      put(NC + v, s + msrc[v]);
    }
  }
}

// the tangent-linear right-hand side at order q (defined in rhs_tangent.cu, where the tangent
// working array's offset is set)
cudaError_t launch_rhs_tangent(int q, bool diss, bool intr, cudaStream_t s, const Case& cs, const RhsArgs& a,
                               const TanArgs& ta, long tan_off);

}  // namespace tgh
