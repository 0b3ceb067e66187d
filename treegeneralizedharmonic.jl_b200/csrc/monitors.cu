// Launches of the constraint monitors, one instantiation per order q.
#include <cuda_runtime.h>

#include "monitors.cuh"

namespace tgh {

template <int Q> static cudaError_t launch_gauge_q(cudaStream_t s, const Case& cs, const MonArgs& a) {
  const unsigned nb = (unsigned)((a.npts + 127) / 128);
  gauge_constraint_kernel<Q><<<nb, 128, 0, s>>>(cs, a);
  return cudaGetLastError();
}
template <int Q> static cudaError_t launch_adm_q(cudaStream_t s, const Case& cs, const MonArgs& a) {
  const unsigned nb = (unsigned)((a.npts + 127) / 128);
  adm_constraint_kernel<Q><<<nb, 128, 0, s>>>(cs, a);
  return cudaGetLastError();
}

cudaError_t launch_gauge_constraint(int q, cudaStream_t s, const Case& cs, const MonArgs& a) {
  switch (q) {
    case 2: return launch_gauge_q<2>(s, cs, a);
    case 4: return launch_gauge_q<4>(s, cs, a);
    case 6: return launch_gauge_q<6>(s, cs, a);
    default: return launch_gauge_q<8>(s, cs, a);
  }
}
cudaError_t launch_adm_constraint(int q, cudaStream_t s, const Case& cs, const MonArgs& a) {
  switch (q) {
    case 2: return launch_adm_q<2>(s, cs, a);
    case 4: return launch_adm_q<4>(s, cs, a);
    case 6: return launch_adm_q<6>(s, cs, a);
    default: return launch_adm_q<8>(s, cs, a);
  }
}

}  // namespace tgh
