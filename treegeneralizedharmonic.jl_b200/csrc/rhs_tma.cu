// Host side of the TMA-staged Pi kernel: the tensor maps of a working array and the launch.
#include <cudaTypedefs.h>

#include <cstring>
#include <string>

#include "rhs_pi_tma.cuh"

namespace tgh {

// The working array of nwb blocks viewed as a 4-d tensor (x: Wx = 40 with 39 used, y: 39,
// z: 39, block x 20 + variable), with the h box (50, 15, 6, 1) and the Pi box (50, 17, 8, 1).
// Rows are 320 bytes apart (a multiple of 16, as the copies need); a box starting at x = -2
// reads zeros left of the array and beyond x = 39 (the pad column, also zero).
bool make_pi_tma_maps(double* work, int nwb, PiTmaMaps* out, std::string& err) {
  using namespace pitma;
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
      err = "the driver offers no cuTensorMapEncodeTiled";
      return false;
    }
    encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  }
  const int Wd = N1 + 2 * G, Wx = Wd + 1;
  const cuuint64_t dims[4] = {(cuuint64_t)Wx, (cuuint64_t)Wd, (cuuint64_t)Wd, (cuuint64_t)NV * nwb};
  const cuuint64_t strides[3] = {(cuuint64_t)Wx * 8, (cuuint64_t)Wx * Wd * 8, (cuuint64_t)Wx * Wd * Wd * 8};
  const cuuint32_t ones[4] = {1, 1, 1, 1};
  const cuuint32_t hbox[4] = {XB, HY, HZ, 1}, pbox[4] = {XB, PY, PZ, 1};
  CUresult r = encode(&out->h, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, work, dims, strides, hbox, ones,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r == CUDA_SUCCESS)
    r = encode(&out->pi, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, work, dims, strides, pbox, ones,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    err = "cuTensorMapEncodeTiled refused the working array's map (error " + std::to_string((int)r) + ")";
    return false;
  }
  return true;
}

template <bool DISS, int MODE>
static cudaError_t launch_pi_tma_t(cudaStream_t s, const Case& cs, const RhsArgs& a, const PiTmaMaps& M,
                                   PiTmaStatus st, int b0, int nb) {
  using namespace pitma;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(rhs_pi_tma_kernel<DISS, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         SMEM);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  rhs_pi_tma_kernel<DISS, MODE><<<(unsigned)(nb * TILES), THREADS, SMEM, s>>>(cs, a, M, st, b0);
  return cudaGetLastError();
}

// The Pi kernel over the whole blocks b0 .. b0 + nb - 1 (q = 4, N = 32, FP64).
cudaError_t launch_pi_tma(bool diss, int mode, cudaStream_t s, const Case& cs, const RhsArgs& a,
                          const PiTmaMaps& M, PiTmaStatus st, int b0, int nb) {
  if (diss) return mode == MODE_DU ? launch_pi_tma_t<true, MODE_DU>(s, cs, a, M, st, b0, nb)
                                   : launch_pi_tma_t<true, MODE_STAGE>(s, cs, a, M, st, b0, nb);
  return mode == MODE_DU ? launch_pi_tma_t<false, MODE_DU>(s, cs, a, M, st, b0, nb)
                         : launch_pi_tma_t<false, MODE_STAGE>(s, cs, a, M, st, b0, nb);
}

}  // namespace tgh
