// FP64 Krylov building blocks on the device: weighted inner products against
// many vectors, many-vector axpy, scaling and a small symmetric eigensolver.
//
// The reference's Krylov crate offers CG over the KrylovVector /
// LinearOperator traits (tenet-krylov/src/{cg,vector,operator}.rs); the
// inner product of block-sparse tensors is the quantum-dimension-weighted
// sum <x, y> = sum_c d_c tr(x_c^T y_c) (TensorKit semantics, as pinned by
// tenet/tests/semantic_suite.rs).  These kernels keep a Lanczos iteration
// resident on the GPU in FP64: orthogonalisation (weighted dots + axpy) and
// the tridiagonal eigenproblem (cyclic Jacobi in one CTA).
#include <cfloat>

#include "kernels.cuh"

namespace tnt {

namespace {

constexpr int kDotThreads = 256;
constexpr int kDotMaxVecs = 64;
constexpr int kChunk = 8192;  // elements per CTA of a weighted dot

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Partial weighted dots of chunk `blockIdx.x`: part[blockIdx.x * k + j] =
// sum_{e in chunk} w(e) V_j[e] y[e], with w constant per coupled sector.
__global__ void __launch_bounds__(kDotThreads) wdot_kernel(const SvdJob* __restrict__ sectors, int32_t nsectors,
                                                           const int64_t* __restrict__ chunk_sector,
                                                           const int64_t* __restrict__ chunk_start, int32_t k,
                                                           const double* __restrict__ V, int64_t ldv,
                                                           const double* __restrict__ y, double* __restrict__ part) {
  __shared__ double red[kDotMaxVecs][kDotThreads / 32];
  const int64_t c = blockIdx.x;
  const SvdJob S = sectors[chunk_sector[c]];
  const int64_t begin = chunk_start[c];
  const int64_t size = S.m * S.n;
  const int64_t end = begin + kChunk < size ? begin + kChunk : size;
  const double w = S.weight;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int j0 = 0; j0 < k; j0 += 8) {
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int64_t e = begin + threadIdx.x; e < end; e += blockDim.x) {
      const double ye = y[S.a_off + e];
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (j0 + j < k) acc[j] = fma(V[(int64_t)(j0 + j) * ldv + S.a_off + e], ye, acc[j]);
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const double v = warp_sum(acc[j]);
      if (lane == 0 && j0 + j < k) red[j0 + j][warp] = v;
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < k; j += blockDim.x) {
    double s = 0.0;
    for (int q = 0; q < kDotThreads / 32; ++q) s += red[j][q];
    part[c * k + j] = w * s;
  }
}

// out[j] = sum over chunks of part[c * k + j] (fixed order: deterministic).
__global__ void wdot_reduce_kernel(const double* __restrict__ part, int64_t nchunks, int32_t k,
                                   double* __restrict__ out) {
  const int j = blockIdx.x;
  double s = 0.0;
  for (int64_t c = threadIdx.x; c < nchunks; c += blockDim.x) s += part[c * k + j];
  __shared__ double red[32];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0) out[j] = t;
  }
}

// y = a * y + sum_j coef[j] V_j   (a = 1: Gram-Schmidt update with coef = -h).
__global__ void axpy_many_kernel(int64_t n, int32_t k, const double* __restrict__ V, int64_t ldv,
                                 const double* __restrict__ coef, double a, const double* __restrict__ a_dev,
                                 double* __restrict__ y) {
  const double aa = a_dev ? *a_dev : a;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    double v = aa * y[e];
    for (int j = 0; j < k; ++j) v = fma(coef[j], V[(int64_t)j * ldv + e], v);
    y[e] = v;
  }
}

// Cyclic Jacobi eigen-decomposition of a symmetric m x m matrix (m <= 48) in
// one CTA; eigenvalues ascending, eigenvectors as columns (column-major).
__global__ void __launch_bounds__(256) symeig_kernel(int32_t m, const double* __restrict__ Ain,
                                                     double* __restrict__ evals, double* __restrict__ evecs,
                                                     int32_t* __restrict__ status) {
  __shared__ double A[48][49];
  __shared__ double Q[48][49];
  __shared__ double ev[48];
  __shared__ int rot;
  const int tid = threadIdx.x;
  for (int i = tid; i < m * m; i += blockDim.x) {
    const int r = i % m, c = i / m;
    A[r][c] = Ain[i];
    Q[r][c] = r == c ? 1.0 : 0.0;
  }
  __syncthreads();
  int sweep = 0;
  for (; sweep < 60; ++sweep) {
    if (tid == 0) rot = 0;
    __syncthreads();
    for (int p = 0; p < m - 1; ++p) {
      for (int q = p + 1; q < m; ++q) {
        const double apq = A[p][q];
        const double app = A[p][p], aqq = A[q][q];
        __syncthreads();
        if (fabs(apq) > 1e-300 && fabs(apq) > 4.0 * sqrt((double)m) * DBL_EPSILON * sqrt(fabs(app * aqq)) + 1e-300) {
          const double theta = (aqq - app) / (2.0 * apq);
          const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
          const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
          // A <- J^T A J on rows/cols p, q; Q <- Q J
          for (int i = tid; i < m; i += blockDim.x) {
            const double aip = A[i][p], aiq = A[i][q];
            A[i][p] = c * aip - s * aiq;
            A[i][q] = s * aip + c * aiq;
          }
          __syncthreads();
          for (int i = tid; i < m; i += blockDim.x) {
            const double api = A[p][i], aqi = A[q][i];
            A[p][i] = c * api - s * aqi;
            A[q][i] = s * api + c * aqi;
            const double qip = Q[i][p], qiq = Q[i][q];
            Q[i][p] = c * qip - s * qiq;
            Q[i][q] = s * qip + c * qiq;
          }
          if (tid == 0) rot = 1;
        }
        __syncthreads();
      }
    }
    const int any = rot;
    __syncthreads();
    if (!any) break;
  }
  if (tid == 0 && sweep == 60) *status = 1;
  for (int i = tid; i < m; i += blockDim.x) ev[i] = A[i][i];
  __syncthreads();
  for (int i = tid; i < m; i += blockDim.x) {
    int pos = 0;
    for (int j = 0; j < m; ++j) pos += (ev[j] < ev[i] || (ev[j] == ev[i] && j < i)) ? 1 : 0;
    evals[pos] = ev[i];
    for (int r = 0; r < m; ++r) evecs[r + (int64_t)pos * m] = Q[r][i];
  }
}

}  // namespace

int64_t wdot_chunks(const SvdJob* host_sectors, int32_t nsectors, std::vector<int64_t>& sector_of_chunk,
                    std::vector<int64_t>& start_of_chunk) {
  sector_of_chunk.clear();
  start_of_chunk.clear();
  for (int32_t s = 0; s < nsectors; ++s) {
    const int64_t size = host_sectors[s].m * host_sectors[s].n;
    for (int64_t b = 0; b < size; b += kChunk) {
      sector_of_chunk.push_back(s);
      start_of_chunk.push_back(b);
    }
  }
  return (int64_t)sector_of_chunk.size();
}

cudaError_t launch_wdot(const SvdJob* sectors, int32_t nsectors, const int64_t* chunk_sector,
                        const int64_t* chunk_start, int64_t nchunks, int32_t k, const double* V, int64_t ldv,
                        const double* y, double* part, double* out, cudaStream_t stream) {
  if (k <= 0) return cudaSuccess;
  if (k > kDotMaxVecs) return cudaErrorInvalidValue;
  if (nchunks > 0)
    wdot_kernel<<<(unsigned)nchunks, kDotThreads, 0, stream>>>(sectors, nsectors, chunk_sector, chunk_start, k, V,
                                                              ldv, y, part);
  wdot_reduce_kernel<<<k, 256, 0, stream>>>(part, nchunks, k, out);
  return cudaGetLastError();
}

cudaError_t launch_axpy_many(int64_t n, int32_t k, const double* V, int64_t ldv, const double* coef, double a,
                             const double* a_dev, double* y, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t blocks = (n + 255) / 256;
  const unsigned grid = (unsigned)(blocks < (int64_t)sms * 16 ? blocks : (int64_t)sms * 16);
  axpy_many_kernel<<<grid, 256, 0, stream>>>(n, k, V, ldv, coef, a, a_dev, y);
  return cudaGetLastError();
}

cudaError_t launch_symeig(int32_t m, const double* A, double* evals, double* evecs, int32_t* status,
                          cudaStream_t stream) {
  if (m <= 0) return cudaSuccess;
  if (m > 48) return cudaErrorInvalidValue;
  symeig_kernel<<<1, 256, 0, stream>>>(m, A, evals, evecs, status);
  return cudaGetLastError();
}

}  // namespace tnt
