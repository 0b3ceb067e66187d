// The tangent-linear right-hand side's instantiations and its launcher, which sets the offset
// from the value working array to its tangent before the launch.
#include "tangent_rhs.cuh"

namespace tgh {

template <int Q, bool DISS>
static cudaError_t launch_tan_q(bool intr, cudaStream_t s, const Case& cs, const RhsArgs& a, const TanArgs& ta) {
  const int TH = 128;
  const unsigned nb = (unsigned)((a.p1 - a.p0 + TH - 1) / TH);
  if (intr) rhs_tangent_kernel<Q, DISS, true><<<nb, TH, 0, s>>>(cs, a, ta);
  else rhs_tangent_kernel<Q, DISS, false><<<nb, TH, 0, s>>>(cs, a, ta);
  return cudaGetLastError();
}

cudaError_t launch_rhs_tangent(int q, bool diss, bool intr, cudaStream_t s, const Case& cs, const RhsArgs& a,
                               const TanArgs& ta, long tan_off) {
  cudaError_t e = cudaMemcpyToSymbolAsync(c_tan_off, &tan_off, sizeof(long), 0, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return e;
  switch (q) {
    case 2: return diss ? launch_tan_q<2, true>(intr, s, cs, a, ta) : launch_tan_q<2, false>(intr, s, cs, a, ta);
    case 4: return diss ? launch_tan_q<4, true>(intr, s, cs, a, ta) : launch_tan_q<4, false>(intr, s, cs, a, ta);
    case 6: return diss ? launch_tan_q<6, true>(intr, s, cs, a, ta) : launch_tan_q<6, false>(intr, s, cs, a, ta);
    default: return diss ? launch_tan_q<8, true>(intr, s, cs, a, ta) : launch_tan_q<8, false>(intr, s, cs, a, ta);
  }
}

}  // namespace tgh
