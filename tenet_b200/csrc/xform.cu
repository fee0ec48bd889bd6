// Recoupling transform kernel: dst = alpha * U . P(src) + beta * dst per group.
//
// Replaces the Host replay of tenet-operations/src/transform_replay.rs:
// Single blocks (4428-4517, a permuted strided copy times one coefficient) and
// Multi groups (4519-4800: pack every source block of a group into a column,
// one GEMM with U^T, scatter back).  Here a group is executed element-wise:
// each thread owns one element position of the group's common block shape,
// gathers that element from every source block, applies the ndst x nsrc
// coefficient matrix from shared memory, and writes every destination block.
// Threads walk destination axis 0 fastest, so writes are contiguous runs of
// the codomain extent; each source element is read exactly once.
#include "kernels.cuh"

namespace tnt {

namespace {

constexpr int kXThreads = 256;
constexpr int kRegSrc = 16;     // source blocks cached in registers
constexpr int kSmemCoef = 1024; // coefficients staged in shared memory

__device__ __forceinline__ void unravel(int64_t e, int rank, const int32_t* dims, int32_t* idx) {
  for (int k = 0; k < rank; ++k) {
    int32_t d = dims[k];
    int64_t q = e / d;
    idx[k] = (int32_t)(e - q * d);
    e = q;
  }
}

__device__ __forceinline__ int64_t place(const XEntry& en, int rank, const int32_t* idx) {
  int64_t off = en.offset;
  for (int k = 0; k < rank; ++k) off += (int64_t)idx[k] * en.strides[k];
  return off;
}

__global__ void __launch_bounds__(kXThreads) xform_kernel(const XTile* __restrict__ tiles, int32_t ntiles,
                                                          const XGroup* __restrict__ groups,
                                                          const XEntry* __restrict__ src_e,
                                                          const XEntry* __restrict__ dst_e,
                                                          const double* __restrict__ coef,
                                                          const double* __restrict__ src, double* __restrict__ dst,
                                                          double alpha, double beta) {
  __shared__ XGroup g;
  __shared__ XTile tile;
  __shared__ double U[kSmemCoef];
  for (int32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    __syncthreads();
    if (threadIdx.x == 0) {
      tile = tiles[t];
      g = groups[tile.group];
    }
    __syncthreads();
    const int nsrc = g.nsrc, ndst = g.ndst, rank = g.rank;
    const int ncoef = nsrc * ndst;
    const bool coef_in_smem = ncoef <= kSmemCoef;
    if (coef_in_smem)
      for (int i = threadIdx.x; i < ncoef; i += blockDim.x) U[i] = coef[g.coef_off + i];
    __syncthreads();
    const double* Ug = coef_in_smem ? U : coef + g.coef_off;
    for (int64_t e = tile.start + threadIdx.x; e < tile.start + tile.count; e += blockDim.x) {
      int32_t idx[kMaxRank];
      unravel(e, rank, g.dims, idx);
      if (nsrc == 0) {
        for (int d = 0; d < ndst; ++d) {
          int64_t o = place(dst_e[g.dst_first + d], rank, idx);
          dst[o] = beta == 0.0 ? 0.0 : beta * dst[o];
        }
        continue;
      }
      if (nsrc <= kRegSrc) {
        double v[kRegSrc];
#pragma unroll
        for (int s = 0; s < kRegSrc; ++s)
          if (s < nsrc) v[s] = __ldg(src + place(src_e[g.src_first + s], rank, idx));
        for (int d = 0; d < ndst; ++d) {
          double acc = 0.0;
#pragma unroll
          for (int s = 0; s < kRegSrc; ++s)
            if (s < nsrc) acc = fma(Ug[d * nsrc + s], v[s], acc);
          int64_t o = place(dst_e[g.dst_first + d], rank, idx);
          dst[o] = beta == 0.0 ? alpha * acc : fma(beta, dst[o], alpha * acc);
        }
      } else {
        for (int d = 0; d < ndst; ++d) {
          double acc = 0.0;
          for (int s = 0; s < nsrc; ++s)
            acc = fma(Ug[d * nsrc + s], __ldg(src + place(src_e[g.src_first + s], rank, idx)), acc);
          int64_t o = place(dst_e[g.dst_first + d], rank, idx);
          dst[o] = beta == 0.0 ? alpha * acc : fma(beta, dst[o], alpha * acc);
        }
      }
    }
  }
}

}  // namespace

cudaError_t launch_xform(const DevXform& x, double* dst, const double* src, double alpha, double beta,
                         cudaStream_t stream) {
  if (x.ntiles == 0) return cudaSuccess;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int grid = x.ntiles < sms * 8 ? x.ntiles : sms * 8;
  xform_kernel<<<grid, kXThreads, 0, stream>>>(x.tiles, x.ntiles, x.groups, x.src, x.dst, x.coef, src, dst, alpha,
                                              beta);
  return cudaGetLastError();
}

}  // namespace tnt
