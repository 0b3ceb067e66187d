// Launch entry points of the right-hand side (the head kernel, then the Pi kernel), one
// translation unit per order q (the instantiations are large; units compile in parallel).
#pragma once
#include <cuda_runtime.h>

#include "rhs.cuh"

namespace tgh {
// part 0: the head kernel, part 1: the Pi kernel, over the points [a.p0, a.p1); suffix f64 the
// FP64 form, f32 the mixed form (FP32 stencil sums and algebra on an FP64 state)
#define TGH_DECLARE_RHS_LAUNCH(QQ, SUF)                                                                    \
  cudaError_t launch_rhs_q##QQ##_##SUF(int part, bool diss, int mode, bool intr, cudaStream_t s, const Case& cs, \
                                       const RhsArgs& a);
TGH_DECLARE_RHS_LAUNCH(2, f64)
TGH_DECLARE_RHS_LAUNCH(4, f64)
TGH_DECLARE_RHS_LAUNCH(6, f64)
TGH_DECLARE_RHS_LAUNCH(8, f64)
TGH_DECLARE_RHS_LAUNCH(2, f32)
TGH_DECLARE_RHS_LAUNCH(4, f32)
TGH_DECLARE_RHS_LAUNCH(6, f32)
TGH_DECLARE_RHS_LAUNCH(8, f32)

template <int Q, bool DISS, int MODE, int N1S, class T>
cudaError_t launch_rhs_n(int part, bool intr, cudaStream_t s, const Case& cs, const RhsArgs& a) {
  const int TH = a.threads == 64 ? 64 : 128;
  const unsigned nb = (unsigned)((a.p1 - a.p0 + TH - 1) / TH);
  if (part == 0) {
    if (intr) rhs_head_kernel<Q, DISS, MODE, true, N1S, T><<<nb, TH, 0, s>>>(cs, a);
    else rhs_head_kernel<Q, DISS, MODE, false, N1S, T><<<nb, TH, 0, s>>>(cs, a);
  } else {
    // the FP64 kernels for N = 32 come with three launch bounds (3, 4, 5 resident CTAs per SM)
    if constexpr (N1S == 33 && !is_fp32<T>()) {
      if (a.pi_mb == 3) rhs_pi_kernel<Q, DISS, MODE, T, N1S, 3><<<nb, TH, 0, s>>>(cs, a);
      else if (a.pi_mb == 5) rhs_pi_kernel<Q, DISS, MODE, T, N1S, 5><<<nb, TH, 0, s>>>(cs, a);
      else rhs_pi_kernel<Q, DISS, MODE, T, N1S><<<nb, TH, 0, s>>>(cs, a);
    } else {
      rhs_pi_kernel<Q, DISS, MODE, T, N1S><<<nb, TH, 0, s>>>(cs, a);
    }
  }
  return cudaGetLastError();
}

// blocks of N = 32 cells run the kernels compiled for that size, others the general ones
template <int Q, bool DISS, int MODE, class T>
cudaError_t launch_rhs_t(int part, bool intr, cudaStream_t s, const Case& cs, const RhsArgs& a) {
  if (a.N1 == 33) return launch_rhs_n<Q, DISS, MODE, 33, T>(part, intr, s, cs, a);
  return launch_rhs_n<Q, DISS, MODE, 0, T>(part, intr, s, cs, a);
}

#define TGH_DEFINE_RHS_LAUNCH(QQ, SUF, TT)                                                                    \
  cudaError_t launch_rhs_q##QQ##_##SUF(int part, bool diss, int mode, bool intr, cudaStream_t s, const Case& cs, \
                                       const RhsArgs& a) {                                                   \
    if (diss) return mode == MODE_DU ? launch_rhs_t<QQ, true, MODE_DU, TT>(part, intr, s, cs, a)              \
                                     : launch_rhs_t<QQ, true, MODE_STAGE, TT>(part, intr, s, cs, a);          \
    return mode == MODE_DU ? launch_rhs_t<QQ, false, MODE_DU, TT>(part, intr, s, cs, a)                       \
                           : launch_rhs_t<QQ, false, MODE_STAGE, TT>(part, intr, s, cs, a);                   \
  }
}  // namespace tgh
