// FP64 grouped GEMM over every coupled sector of a compose, in one launch.
//
// Replaces the per-sector GEMM loop of FusionBlockContractPlan::execute_raw
// (tenet-operations/src/fusion_replay.rs:556) and its device twin
// execute_direct_on_storage (fusion_replay.rs:1168-1290, one cuBLAS call per
// sector).  Every (sector job, batch entry, output tile) is one work item of a
// persistent kernel.  Each tile carries its shape: interior tiles take the
// shape the autotuner picked for the sector (64x64, 64x32, 32x64 or 32x32,
// from the block-size histogram), and the last row and column blocks of a
// sector are trimmed to the remainder rounded up to 16, so ragged sectors
// waste little padding.  Tiles are pre-sorted longest first so the uneven
// sector sizes balance across the 148 SMs.  Math runs on the FP64 tensor
// cores (mma.sync m8n8k4 f64, which reaches the same 37 TFLOP/s on B200 as
// the m16n8k* shapes); operands are staged through shared memory by a
// three-deep cp.async ring.
#include "kernels.cuh"

namespace tnt {

namespace {

constexpr int BK = 16;
constexpr int SP = 68;  // padded row stride in doubles: conflict-free fragment loads
constexpr int kThreads = 128;
constexpr int kStages = 3;  // cp.async ring: two k-tiles in flight while one is multiplied
// Three CTAs per SM: the 64 x 64 tile body needs 168 registers, and capping it
// at 128 (four CTAs) spills and measured 7% slower on the 64-compose
// fZ2xU1xSU2 batch (21.2 against 22.8 TFLOP/s).
constexpr int kMinBlocks = 3;

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool pred) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int n = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// One BM x BN output tile (BM, BN in {16, 32, 48, 64}) whose first row and
// column are m0 and n0; 4 warps in a 2 x 2 layout, each computing
// (BM/2) x (BN/2) with m8n8k4 FP64 MMAs.  K runs in BK-deep k-tiles through a
// kStages-deep cp.async ring, one barrier per k-tile.
template <int BM, int BN>
__device__ __forceinline__ void tile_body(const GemmJob& J, int64_t m0, int64_t n0, int32_t batch,
                                          double* __restrict__ C, int64_t sc, const double* __restrict__ A,
                                          int64_t sa, const double* __restrict__ B, int64_t sb, double alpha,
                                          double beta, double (*As)[BK][SP], double (*Bs)[BK][SP]) {
  constexpr int WI = BM / 16, WJ = BN / 16;  // 8x8 MMA tiles per warp along M and N
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int g = lane >> 2, t4 = lane & 3;
  const double* a = A + batch * sa + J.a_off;
  const double* b = B + batch * sb + J.b_off;
  double* c = C + batch * sc + J.c_off;
  double acc[WI][WJ][2];
#pragma unroll
  for (int i = 0; i < WI; ++i)
#pragma unroll
    for (int j = 0; j < WJ; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  const int64_t nk = (J.k + BK - 1) / BK;
  auto load = [&](int64_t kt, int buf) {
    const int64_t k0 = kt * BK;
#pragma unroll
    for (int r = 0; r < (BM * BK) / kThreads; ++r) {
      int idx = tid + r * kThreads;
      int i = idx % BM, kk = idx / BM;
      int64_t gm = m0 + i, gk = k0 + kk;
      bool ok = gm < J.m && gk < J.k;
      cp_async8(&As[buf][kk][i], ok ? a + gm + gk * J.lda : a, ok);
    }
#pragma unroll
    for (int r = 0; r < (BN * BK) / kThreads; ++r) {
      int idx = tid + r * kThreads;
      int kk = idx % BK, j = idx / BK;
      int64_t gn = n0 + j, gk = k0 + kk;
      bool ok = gn < J.n && gk < J.k;
      cp_async8(&Bs[buf][kk][j], ok ? b + gk + gn * J.ldb : b, ok);
    }
  };

  // Prologue: k-tiles 0 .. kStages-2 in flight (empty groups keep the count).
#pragma unroll
  for (int s = 0; s < kStages - 1; ++s) {
    if (s < nk) load(s, s);
    cp_async_commit();
  }
  for (int64_t kt = 0; kt < nk; ++kt) {
    const int buf = (int)(kt % kStages);
    cp_async_wait<kStages - 2>();  // k-tile kt has landed
    __syncthreads();               // ... for every thread, and k-tile kt-1's buffer is free
    if (kt + kStages - 1 < nk) load(kt + kStages - 1, (int)((kt + kStages - 1) % kStages));
    cp_async_commit();
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double af[WI], bf[WJ];
#pragma unroll
      for (int i = 0; i < WI; ++i) af[i] = As[buf][kk + t4][wm * (BM / 2) + i * 8 + g];
#pragma unroll
      for (int j = 0; j < WJ; ++j) bf[j] = Bs[buf][kk + t4][wn * (BN / 2) + j * 8 + g];
#pragma unroll
      for (int i = 0; i < WI; ++i)
#pragma unroll
        for (int j = 0; j < WJ; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
  }
  cp_async_wait<0>();
  __syncthreads();  // the ring is reused by the CTA's next tile

#pragma unroll
  for (int i = 0; i < WI; ++i) {
    const int64_t row = m0 + wm * (BM / 2) + i * 8 + g;
    if (row >= J.m) continue;
#pragma unroll
    for (int j = 0; j < WJ; ++j) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int64_t col = n0 + wn * (BN / 2) + j * 8 + t4 * 2 + e;
        if (col >= J.n) continue;
        double* p = c + row + col * J.ldc;
        double v = alpha * acc[i][j][e];
        *p = beta == 0.0 ? v : fma(beta, *p, v);
      }
    }
  }
}

template <int BM>
__device__ __forceinline__ void tile_rows(int bn16, const GemmJob& J, int64_t m0, int64_t n0, int32_t batch,
                                          double* C, int64_t sc, const double* A, int64_t sa, const double* B,
                                          int64_t sb, double alpha, double beta, double (*As)[BK][SP],
                                          double (*Bs)[BK][SP]) {
  switch (bn16) {
    case 1: tile_body<BM, 16>(J, m0, n0, batch, C, sc, A, sa, B, sb, alpha, beta, As, Bs); break;
    case 2: tile_body<BM, 32>(J, m0, n0, batch, C, sc, A, sa, B, sb, alpha, beta, As, Bs); break;
    case 3: tile_body<BM, 48>(J, m0, n0, batch, C, sc, A, sa, B, sb, alpha, beta, As, Bs); break;
    default: tile_body<BM, 64>(J, m0, n0, batch, C, sc, A, sa, B, sb, alpha, beta, As, Bs); break;
  }
}

// One CTA per tile.  A tile's `shape` is its geometry code
// f64_tile_code(BM, BN) and (tm, tn) its first row and column in units of
// 16: interior tiles have the job's chosen shape, the last row and column
// blocks are trimmed to the remainder rounded up to 16.
__global__ void __launch_bounds__(kThreads, kMinBlocks) gemm_f64_kernel(const GemmJob* __restrict__ jobs,
                                                            const GemmTile* __restrict__ tiles, int32_t ntiles,
                                                            double* __restrict__ C, int64_t sc,
                                                            const double* __restrict__ A, int64_t sa,
                                                            const double* __restrict__ B, int64_t sb, double alpha,
                                                            double beta) {
  extern __shared__ __align__(16) double ring[];  // kStages x (A, B) k-tiles: 52 KB, above the static limit
  auto As = reinterpret_cast<double(*)[BK][SP]>(ring);
  auto Bs = reinterpret_cast<double(*)[BK][SP]>(ring + kStages * BK * SP);
  for (int32_t it = blockIdx.x; it < ntiles; it += gridDim.x) {
    const GemmTile tile = tiles[it];
    const GemmJob J = jobs[tile.job];
    const int64_t m0 = (int64_t)tile.tm * 16, n0 = (int64_t)tile.tn * 16;
    const int bm16 = (tile.shape >> 2) + 1, bn16 = (tile.shape & 3) + 1;
    switch (bm16) {
      case 1: tile_rows<16>(bn16, J, m0, n0, tile.batch, C, sc, A, sa, B, sb, alpha, beta, As, Bs); break;
      case 2: tile_rows<32>(bn16, J, m0, n0, tile.batch, C, sc, A, sa, B, sb, alpha, beta, As, Bs); break;
      case 3: tile_rows<48>(bn16, J, m0, n0, tile.batch, C, sc, A, sa, B, sb, alpha, beta, As, Bs); break;
      default: tile_rows<64>(bn16, J, m0, n0, tile.batch, C, sc, A, sa, B, sb, alpha, beta, As, Bs); break;
    }
  }
}

}  // namespace

cudaError_t launch_gemm_f64(const GemmJob* jobs, const GemmTile* tiles, int32_t ntiles, double* c, int64_t sc,
                            const double* a, int64_t sa, const double* b, int64_t sb, double alpha, double beta,
                            cudaStream_t stream) {
  if (ntiles == 0) return cudaSuccess;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // One CTA per tile (tiles are longest first): the hardware block scheduler
  // then balances the ragged sector mix as SMs free up (a grid-stride loop
  // over a fixed number of CTAs per SM measured 6-11% slower on the
  // 64-compose fZ2xU1xSU2 batch).
  int grid = ntiles;
  constexpr size_t smem = 2 * kStages * BK * SP * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(gemm_f64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  gemm_f64_kernel<<<grid, kThreads, smem, stream>>>(jobs, tiles, ntiles, c, sc, a, sa, b, sb, alpha, beta);
  return cudaGetLastError();
}

}  // namespace tnt
