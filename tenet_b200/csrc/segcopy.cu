// Strided block copies with optional row scaling, many blocks per launch.
//
// Used to publish truncated factorisation outputs in place: every segment
// copies a rows x cols column-major block (source leading dimension src_ld)
// into a destination block (leading dimension dst_ld), optionally scaling row
// i by scales[scale_off + i] (the S Vh product of a truncated SVD).
#include "kernels.cuh"

namespace tnt {

namespace {

__global__ void __launch_bounds__(256) segcopy_kernel(const SegCopy* __restrict__ segs, const double* __restrict__ src,
                                                      double* __restrict__ dst, const double* __restrict__ scales) {
  const SegCopy S = segs[blockIdx.x];
  const int64_t n = S.rows * S.cols;
  for (int64_t e = threadIdx.x; e < n; e += blockDim.x) {
    const int64_t i = e % S.rows, j = e / S.rows;
    double v = src[S.src_off + i + j * S.src_ld];
    if (S.scale_off >= 0) v *= scales[S.scale_off + i];
    dst[S.dst_off + i + j * S.dst_ld] = v;
  }
}

}  // namespace

cudaError_t launch_segcopy(const SegCopy* segs, int64_t nseg, const double* src, double* dst, const double* scales,
                           cudaStream_t stream) {
  if (nseg == 0) return cudaSuccess;
  if (nseg > 0x7fffffff) return cudaErrorInvalidValue;
  segcopy_kernel<<<(unsigned)nseg, 256, 0, stream>>>(segs, src, dst, scales);
  return cudaGetLastError();
}

}  // namespace tnt
