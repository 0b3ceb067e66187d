// Launch entry points of the right-hand side (the head kernel, then the Pi kernel), one
// translation unit per order q (the instantiations are large; units compile in parallel).
#pragma once
#include <cuda_runtime.h>

#include "rhs.cuh"

namespace tgh {
cudaError_t launch_rhs_q2(bool diss, int mode, bool intr, long npts, cudaStream_t s, const Case& cs, const RhsArgs& a);
cudaError_t launch_rhs_q4(bool diss, int mode, bool intr, long npts, cudaStream_t s, const Case& cs, const RhsArgs& a);
cudaError_t launch_rhs_q6(bool diss, int mode, bool intr, long npts, cudaStream_t s, const Case& cs, const RhsArgs& a);
cudaError_t launch_rhs_q8(bool diss, int mode, bool intr, long npts, cudaStream_t s, const Case& cs, const RhsArgs& a);

template <int Q, bool DISS, int MODE, int N1S>
cudaError_t launch_rhs_n(bool intr, long npts, cudaStream_t s, const Case& cs, const RhsArgs& a) {
  const int T = 128;
  const unsigned nb = (unsigned)((npts + T - 1) / T);
  if (intr) rhs_head_kernel<Q, DISS, MODE, true, N1S><<<nb, T, 0, s>>>(cs, a);
  else rhs_head_kernel<Q, DISS, MODE, false, N1S><<<nb, T, 0, s>>>(cs, a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  rhs_pi_kernel<Q, DISS, MODE, double, N1S><<<nb, T, 0, s>>>(cs, a);
  return cudaGetLastError();
}

// blocks of N = 32 cells run the kernels compiled for that size, others the general ones
template <int Q, bool DISS, int MODE>
cudaError_t launch_rhs_t(bool intr, long npts, cudaStream_t s, const Case& cs, const RhsArgs& a) {
  if (a.N1 == 33) return launch_rhs_n<Q, DISS, MODE, 33>(intr, npts, s, cs, a);
  return launch_rhs_n<Q, DISS, MODE, 0>(intr, npts, s, cs, a);
}

#define TGH_DEFINE_RHS_LAUNCH(QQ)                                                                     \
  cudaError_t launch_rhs_q##QQ(bool diss, int mode, bool intr, long npts, cudaStream_t s, const Case& cs, \
                               const RhsArgs& a) {                                                   \
    if (diss) return mode == MODE_DU ? launch_rhs_t<QQ, true, MODE_DU>(intr, npts, s, cs, a)          \
                                     : launch_rhs_t<QQ, true, MODE_STAGE>(intr, npts, s, cs, a);      \
    return mode == MODE_DU ? launch_rhs_t<QQ, false, MODE_DU>(intr, npts, s, cs, a)                   \
                           : launch_rhs_t<QQ, false, MODE_STAGE>(intr, npts, s, cs, a);               \
  }
}  // namespace tgh
