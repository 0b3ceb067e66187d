// The range projection's launch (bounds.cu): arguments and entry.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "physics.cuh"

namespace tgh {

struct BoundsArgs {
  double* u;                    // state vector, (N1^3 x 20) per block
  const double* blk;            // per block: domain lo (3), h, integer corner (3), pad
  const uint8_t* primary;       // per owned point: 1 at the primary copy
  unsigned long long* counts;   // fired, non-finite, max radius (bits) over the primaries
  double amin, amax, lmin, lmax, bmax, kmax, rgate;
  double t;
  long S, npts;
  int N1;
};

// zeroes the counts, then one thread per owned point of u
cudaError_t launch_bounds_projection(cudaStream_t s, const Case& cs, const BoundsArgs& a);

}  // namespace tgh
