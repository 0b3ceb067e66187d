// tgh_max_speed_noalloc: the checked maximum characteristic speed for callers that cannot
// allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is off limits - inside another framework's
// memory pool that owns the whole device, in a process whose allocator must stay untouched
// between checkpoints, or in a driver loop that may not create device allocations at all -
// and that still wants the speed (hence the time step) of a state it already holds on the
// device. tgh_max_speed needs a problem handle, and building one allocates.
//
// How: every scratch byte this entry point touches lives in one file-scope __device__ array
// of fixed size (below). The caller passes the state and the mesh description; the mesh's
// block table (levels and corners) is copied into the array, and a variant of the speed
// kernel of tgh_max_speed - the same arithmetic per point - places each point from that table
// and reduces into the array's first words, which are cleared first. Nothing is allocated:
// no cudaMalloc, no cudaFree, no host heap.
//
// Limits and sharing: at most TGH_NOALLOC_MAX_BLOCKS blocks. Every GPU that loads the library
// holds the array (256 + 16 x TGH_NOALLOC_MAX_BLOCKS bytes = 131,328 bytes, about 0.13 MB)
// until the process exits. All calls on a device share it and
// it keeps the last call's contents; calls that overlap on the GPU (two streams, or two host
// threads) race on it. The first call on a device looks up the array's device address with
// that device current; make that first call before any stream capture.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>

#include "../../include/tgh.h"
#include "physics.cuh"

using namespace tgh;

namespace {

constexpr int kMaxBlocks = TGH_NOALLOC_MAX_BLOCKS;
constexpr int kMaxDevices = 64;
// layout: [0, 256) reduction words | level (int32 per block) | corner (3 int32 per block)
constexpr size_t kRedBytes = 256;
constexpr size_t kLevelOff = kRedBytes;
constexpr size_t kCornerOff = kLevelOff + sizeof(int32_t) * kMaxBlocks;
constexpr size_t kScratchBytes = kCornerOff + sizeof(int32_t) * 3 * kMaxBlocks;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// device address of g_noalloc_scratch, looked up once per device (the symbol's name in host
// code is only a host-side stand-in for it)
static unsigned char* g_scratch_ptr[kMaxDevices] = {nullptr};

// The speed of tgh_max_speed's kernel, lambda = alpha sqrt(tr gamma^{ij}) + |beta| over the
// evolved owned points (src/evolution.jl:932-949), with the point placed from the block table
// in the scratch array: lo + (corner + i) h, h = h0 / 2^level, each operation rounded. The
// maximum (as the ordered bits of a non-negative double, NaN above all) and the count of
// non-finite evolved values go to red[0] and red[1].
__global__ void speed_noalloc_kernel(const double* __restrict__ u, const int32_t* __restrict__ level,
                                     const int32_t* __restrict__ corner, double lo0, double lo1, double lo2,
                                     double h0, int N1, long npts, const Case cs, double t,
                                     unsigned long long* red) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long S = (long)N1 * N1 * N1;
  double lam = 0.0;
  unsigned long long bad = 0;
  if (p < npts) {
    const int b = (int)(p / S);
    const long ip = p - (long)b * S;
    const int k = (int)(ip / ((long)N1 * N1)), j = (int)((ip / N1) % N1), i = (int)(ip % N1);
    const double h = ldexp(h0, -level[b]);
    const double x[3] = {__dadd_rn(lo0, __dmul_rn((double)corner[3 * b] + (double)i, h)),
                         __dadd_rn(lo1, __dmul_rn((double)corner[3 * b + 1] + (double)j, h)),
                         __dadd_rn(lo2, __dmul_rn((double)corner[3 * b + 2] + (double)k, h))};
    const bool evolved = cs.interior == TGH_INT_NONE ? true : interior_radius(cs, t, x) >= cs.r1;
    if (evolved) {
      const double* q = u + (long)b * NV * S + ip;
      double hv[NC];
      for (int v = 0; v < NV; ++v) {
        const double a = q[v * S];
        if (!isfinite(a)) ++bad;
        if (v < NC) hv[v] = a;
      }
      Coef<double> C;
      metric_quantities(hv, C);
      lam = C.alpha * sqrt(C.gamu[0] + C.gamu[3] + C.gamu[5]) +
            sqrt(C.beta[0] * C.beta[0] + C.beta[1] * C.beta[1] + C.beta[2] * C.beta[2]);
    }
  }
  unsigned long long bits = isnan(lam) ? 0x7ff8000000000000ull : (unsigned long long)__double_as_longlong(lam);
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long ob = __shfl_down_sync(0xffffffffu, bits, o);
    const unsigned long long obad = __shfl_down_sync(0xffffffffu, bad, o);
    bits = ob > bits ? ob : bits;
    bad += obad;
  }
  if ((threadIdx.x & 31) == 0) {
    if (bits) atomicMax(red, bits);
    if (bad) atomicAdd(red + 1, bad);
  }
}

int set_error(char* errbuf, int errlen, int code, const char* msg) {
  if (errbuf && errlen > 0) {
    std::strncpy(errbuf, msg, (size_t)errlen - 1);
    errbuf[errlen - 1] = 0;
  }
  return code;
}

}  // namespace

extern "C" int tgh_max_speed_noalloc(const tgh_config* cfg, const tgh_mesh* mesh, const double* u, double t,
                                     void* cuda_stream, double* lambda, char* errbuf, int errlen) {
  char msg[256];
  if (!cfg || !mesh || !u || !lambda) return set_error(errbuf, errlen, TGH_ERR_ARG, "a required argument is null");
  if (cfg->q < 2 || cfg->q > 8 || cfg->q % 2) return set_error(errbuf, errlen, TGH_ERR_ARG, "q must be even in 2..8");
  if (mesh->nblocks < 1) return set_error(errbuf, errlen, TGH_ERR_ARG, "the mesh has no blocks");
  if (!mesh->level || !mesh->corner)
    return set_error(errbuf, errlen, TGH_ERR_ARG, "the mesh's level and corner tables must not be null");
  if (mesh->N < 1) return set_error(errbuf, errlen, TGH_ERR_ARG, "the block edge N must be at least 1");
  if (mesh->nblocks > kMaxBlocks) {
    std::snprintf(msg, sizeof(msg),
                  "the mesh has %d blocks; the allocation-free speed holds at most %d (use tgh_max_speed)",
                  mesh->nblocks, kMaxBlocks);
    return set_error(errbuf, errlen, TGH_ERR_ARG, msg);
  }
  // the checks tgh_problem_create makes on the block table (levels in range, corners on the
  // block lattice), on the host copy the caller passed
  for (int b = 0; b < mesh->nblocks; ++b) {
    if (mesh->level[b] < 0 || mesh->level[b] > 20) {
      std::snprintf(msg, sizeof(msg), "block %d: level %d out of range 0..20", b, (int)mesh->level[b]);
      return set_error(errbuf, errlen, TGH_ERR_ARG, msg);
    }
    for (int d = 0; d < 3; ++d)
      if (mesh->corner[3 * b + d] % mesh->N) {
        std::snprintf(msg, sizeof(msg), "block %d: a corner is not a multiple of N", b);
        return set_error(errbuf, errlen, TGH_ERR_ARG, msg);
      }
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return set_error(errbuf, errlen, TGH_ERR_CUDA, "no usable current CUDA device");
  if (!g_scratch_ptr[dev]) {
    void* ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) {
      std::snprintf(msg, sizeof(msg), "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      return set_error(errbuf, errlen, TGH_ERR_CUDA, msg);
    }
    g_scratch_ptr[dev] = (unsigned char*)ptr;
  }
  unsigned char* base = g_scratch_ptr[dev];
  cudaStream_t s = (cudaStream_t)cuda_stream;
  const int nb = mesh->nblocks;
  const int N1 = mesh->N + 1;
  const long npts = (long)N1 * N1 * N1 * nb;
  int32_t* lev = (int32_t*)(base + kLevelOff);
  int32_t* cor = (int32_t*)(base + kCornerOff);
  unsigned long long* red = (unsigned long long*)base;
  // the constants the speed reads: only the interior's mask
  Case cs;
  std::memset(&cs, 0, sizeof(cs));
  cs.interior = cfg->interior;
  for (int i = 0; i < 3; ++i) {
    cs.ic0[i] = cfg->int_c0[i];
    cs.iv[i] = cfg->int_v[i];
  }
  cs.r0 = cfg->r0;
  cs.r1 = cfg->r1;
  unsigned long long h[2] = {0, 0};
  if ((e = cudaMemcpyAsync(lev, mesh->level, sizeof(int32_t) * nb, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(cor, mesh->corner, sizeof(int32_t) * 3 * nb, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemsetAsync(red, 0, 2 * sizeof(unsigned long long), s)) != cudaSuccess) {
    std::snprintf(msg, sizeof(msg), "staging the block table: %s", cudaGetErrorString(e));
    return set_error(errbuf, errlen, TGH_ERR_CUDA, msg);
  }
  speed_noalloc_kernel<<<(unsigned)((npts + 127) / 128), 128, 0, s>>>(u, lev, cor, mesh->lo[0], mesh->lo[1],
                                                                     mesh->lo[2], mesh->h0, N1, npts, cs, t, red);
  if ((e = cudaGetLastError()) != cudaSuccess ||
      (e = cudaMemcpyAsync(h, red, sizeof(h), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess) {
    std::snprintf(msg, sizeof(msg), "the speed kernel: %s", cudaGetErrorString(e));
    return set_error(errbuf, errlen, TGH_ERR_CUDA, msg);
  }
  if (h[1] > 0) {
    std::snprintf(msg, sizeof(msg), "the state at t = %g is not finite where it is evolved: %llu values", t, h[1]);
    return set_error(errbuf, errlen, TGH_ERR_NONFINITE, msg);
  }
  double lam;
  std::memcpy(&lam, &h[0], sizeof(lam));
  *lambda = lam;
  if (!(std::isfinite(lam) && lam > 0.0)) {
    std::snprintf(msg, sizeof(msg), "the maximum characteristic speed came out as %g", lam);
    return set_error(errbuf, errlen, TGH_ERR_SPEED, msg);
  }
  return TGH_OK;
}
