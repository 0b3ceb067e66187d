// Launch entry points of the right-hand-side kernel, one translation unit per order q
// (the instantiations are large; separate units compile in parallel).
#pragma once
#include <cuda_runtime.h>

#include "rhs.cuh"

namespace tgh {
cudaError_t launch_rhs_q2(bool diss, int mode, bool intr, long npts, cudaStream_t s, const Case& cs, const RhsArgs& a);
cudaError_t launch_rhs_q4(bool diss, int mode, bool intr, long npts, cudaStream_t s, const Case& cs, const RhsArgs& a);
cudaError_t launch_rhs_q6(bool diss, int mode, bool intr, long npts, cudaStream_t s, const Case& cs, const RhsArgs& a);
cudaError_t launch_rhs_q8(bool diss, int mode, bool intr, long npts, cudaStream_t s, const Case& cs, const RhsArgs& a);

#define TGH_DEFINE_RHS_LAUNCH(QQ)                                                                        \
  cudaError_t launch_rhs_q##QQ(bool diss, int mode, bool intr, long npts, cudaStream_t s, const Case& cs,          \
                               const RhsArgs& a) {                                                      \
    const int T = 128;                                                                                  \
    const unsigned nb = (unsigned)((npts + T - 1) / T);                                                 \
    if (diss) {                                                                                         \
      if (mode == MODE_DU) {                                                                            \
        if (intr) rhs_kernel<QQ, true, MODE_DU, true><<<nb, T, 0, s>>>(cs, a);                          \
        else rhs_kernel<QQ, true, MODE_DU, false><<<nb, T, 0, s>>>(cs, a);                              \
      } else {                                                                                          \
        if (intr) rhs_kernel<QQ, true, MODE_STAGE, true><<<nb, T, 0, s>>>(cs, a);                       \
        else rhs_kernel<QQ, true, MODE_STAGE, false><<<nb, T, 0, s>>>(cs, a);                           \
      }                                                                                                 \
    } else {                                                                                            \
      if (mode == MODE_DU) {                                                                            \
        if (intr) rhs_kernel<QQ, false, MODE_DU, true><<<nb, T, 0, s>>>(cs, a);                         \
        else rhs_kernel<QQ, false, MODE_DU, false><<<nb, T, 0, s>>>(cs, a);                             \
      } else {                                                                                          \
        if (intr) rhs_kernel<QQ, false, MODE_STAGE, true><<<nb, T, 0, s>>>(cs, a);                      \
        else rhs_kernel<QQ, false, MODE_STAGE, false><<<nb, T, 0, s>>>(cs, a);                          \
      }                                                                                                 \
    }                                                                                                   \
    return cudaGetLastError();                                                                          \
  }
}  // namespace tgh
