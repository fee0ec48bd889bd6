// Split-precision grouped GEMM (filled in by the tcgen05 implementation).
#include "kernels.cuh"

namespace tnt {

size_t split_scratch_bytes(const GemmJob*, int32_t, int64_t, int) { return 16; }

cudaError_t launch_gemm_split(const GemmJob*, const GemmJob*, int32_t, const GemmTile*, int32_t, double*, int64_t,
                              const double*, int64_t, const double*, int64_t, int64_t, double, double, int, void*,
                              size_t, cudaStream_t) {
  return cudaErrorNotSupported;
}

}  // namespace tnt
