// Launch entry points of the right-hand side (the head kernel, then the Pi kernel), one
// translation unit per order q (the instantiations are large; units compile in parallel).
#pragma once
#include <cuda_runtime.h>

#include "rhs.cuh"

namespace tgh {
// part 0: the head kernel, part 1: the Pi kernel, over the points [a.p0, a.p1)
cudaError_t launch_rhs_q2(int part, bool diss, int mode, bool intr, cudaStream_t s, const Case& cs, const RhsArgs& a);
cudaError_t launch_rhs_q4(int part, bool diss, int mode, bool intr, cudaStream_t s, const Case& cs, const RhsArgs& a);
cudaError_t launch_rhs_q6(int part, bool diss, int mode, bool intr, cudaStream_t s, const Case& cs, const RhsArgs& a);
cudaError_t launch_rhs_q8(int part, bool diss, int mode, bool intr, cudaStream_t s, const Case& cs, const RhsArgs& a);

template <int Q, bool DISS, int MODE, int N1S>
cudaError_t launch_rhs_n(int part, bool intr, cudaStream_t s, const Case& cs, const RhsArgs& a) {
  const int T = 128;
  const unsigned nb = (unsigned)((a.p1 - a.p0 + T - 1) / T);
  if (part == 0) {
    if (intr) rhs_head_kernel<Q, DISS, MODE, true, N1S><<<nb, T, 0, s>>>(cs, a);
    else rhs_head_kernel<Q, DISS, MODE, false, N1S><<<nb, T, 0, s>>>(cs, a);
  } else {
    rhs_pi_kernel<Q, DISS, MODE, double, N1S><<<nb, T, 0, s>>>(cs, a);
  }
  return cudaGetLastError();
}

// blocks of N = 32 cells run the kernels compiled for that size, others the general ones
template <int Q, bool DISS, int MODE>
cudaError_t launch_rhs_t(int part, bool intr, cudaStream_t s, const Case& cs, const RhsArgs& a) {
  if (a.N1 == 33) return launch_rhs_n<Q, DISS, MODE, 33>(part, intr, s, cs, a);
  return launch_rhs_n<Q, DISS, MODE, 0>(part, intr, s, cs, a);
}

#define TGH_DEFINE_RHS_LAUNCH(QQ)                                                                        \
  cudaError_t launch_rhs_q##QQ(int part, bool diss, int mode, bool intr, cudaStream_t s, const Case& cs, \
                               const RhsArgs& a) {                                                      \
    if (diss) return mode == MODE_DU ? launch_rhs_t<QQ, true, MODE_DU>(part, intr, s, cs, a)             \
                                     : launch_rhs_t<QQ, true, MODE_STAGE>(part, intr, s, cs, a);         \
    return mode == MODE_DU ? launch_rhs_t<QQ, false, MODE_DU>(part, intr, s, cs, a)                      \
                           : launch_rhs_t<QQ, false, MODE_STAGE>(part, intr, s, cs, a);                  \
  }
}  // namespace tgh
