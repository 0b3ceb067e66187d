// Instantiations and launchers of the right-hand side's adjoint kernels (adjoint.cuh).
#include "adjoint.cuh"

namespace tgh {

template <int Q, bool DISS>
static cudaError_t adj_point_q(bool intr, cudaStream_t s, const Case& cs, const RhsArgs& a, const AdjArgs& j) {
  const unsigned nb = (unsigned)((a.p1 - a.p0 + 127) / 128);
  if (intr) adjoint_point_kernel<Q, DISS, true><<<nb, 128, 0, s>>>(cs, a, j);
  else adjoint_point_kernel<Q, DISS, false><<<nb, 128, 0, s>>>(cs, a, j);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_point(int q, bool diss, bool intr, cudaStream_t s, const Case& cs, const RhsArgs& a,
                                 const AdjArgs& j) {
  switch (q) {
    case 2: return diss ? adj_point_q<2, true>(intr, s, cs, a, j) : adj_point_q<2, false>(intr, s, cs, a, j);
    case 4: return diss ? adj_point_q<4, true>(intr, s, cs, a, j) : adj_point_q<4, false>(intr, s, cs, a, j);
    case 6: return diss ? adj_point_q<6, true>(intr, s, cs, a, j) : adj_point_q<6, false>(intr, s, cs, a, j);
    default: return diss ? adj_point_q<8, true>(intr, s, cs, a, j) : adj_point_q<8, false>(intr, s, cs, a, j);
  }
}

template <int Q, bool DISS>
static cudaError_t adj_gather_q(cudaStream_t s, const double* cot, long cstride, const Geo& g, int nb, double* mu) {
  const long n = (long)g.Wd * g.Wd * g.Wd * NC * nb;
  adjoint_gather_kernel<Q, DISS><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(cot, cstride, g, nb, mu);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_gather(int q, bool diss, cudaStream_t s, const double* cot, long cstride, const Geo& g,
                                  int nb, double* mu) {
  switch (q) {
    case 2: return diss ? adj_gather_q<2, true>(s, cot, cstride, g, nb, mu) : adj_gather_q<2, false>(s, cot, cstride, g, nb, mu);
    case 4: return diss ? adj_gather_q<4, true>(s, cot, cstride, g, nb, mu) : adj_gather_q<4, false>(s, cot, cstride, g, nb, mu);
    case 6: return diss ? adj_gather_q<6, true>(s, cot, cstride, g, nb, mu) : adj_gather_q<6, false>(s, cot, cstride, g, nb, mu);
    default: return diss ? adj_gather_q<8, true>(s, cot, cstride, g, nb, mu) : adj_gather_q<8, false>(s, cot, cstride, g, nb, mu);
  }
}

}  // namespace tgh
