// Split-precision grouped GEMM: FP64 blocks as BF16 slices on the tcgen05
// tensor cores, FP32 accumulation in TMEM, FP64 recombination.
//
// Replaces the per-sector FP64 GEMMs of FusionBlockContractPlan
// (tenet-operations/src/fusion_replay.rs:556, 1168-1290) with an emulated-FP64
// product whose error is set by the slice count.
//
// Splitting (pack_a_kernel / pack_b_kernel, one fused pass per operand):
// every row of A and every column of B is scaled by a power of two sigma so
// its largest magnitude is below 1, then cut into S fixed-point slices of 7
// bits, the balanced base-128 digits of one rounded integer:
//   a = sigma * sum_s a_s 2^{-7(s+1)},  a_0 in [-128, 128], a_s in [-64, 63].
// Each slice is an integer, exact in BF16.  A product a_s b_t has magnitude
// <= 2^14, so any FP32 sum of up to 2^10 such integer products is exact.
//
// Slices are stored pre-scaled, A_s = a_s 2^{-7s} (a power-of-two rescaling of
// an integer, still exact in BF16), so a b = sigma tau 2^{-14} sum_{s,t} A_s B_t.
//
// Multiplication (split_mma_kernel): the triangular product set s + t <= S-1
// (S(S+1)/2 MMAs per K step) accumulates in FP32 TMEM accumulators, one per
// diagonal d = s + t for d = 0, 1, 2 and one shared by every d >= 3.  K runs in
// chunks of 512: per k the worst-case integer diagonal sums are 2^14 (d = 0, 1)
// and 5 * 2^12 (d = 2), so over 512 terms those three accumulators hold exact
// integers (times 2^{-7d}); the d >= 3 accumulator sits 2^-21 below the result
// and its FP32 rounding stays below 1e-12 relative.  After each chunk the
// epilogue warps add the accumulators into FP64 registers.  The dropped
// diagonals d >= S bound the relative error by about (S+1) 2^{-7S}.
//
// The kernel is persistent (one CTA per SM walks a longest-K-first tile list).
// It keeps two accumulator sets in TMEM when they fit (2 x 4 x 64 columns), so
// the epilogue of one tile overlaps the MMAs of the next; at width 64 the
// epilogue releases TMEM as soon as its last columns are in registers.  The
// 8-bit-digit variant is described below.
//
// Data movement: the split pass writes the slices in 64-byte K rows
// ([slice][kblock][row][64 bytes] per job), already permuted into the
// SWIZZLE_64B pattern (16-byte chunk q of row r at chunk q ^ ((r >> 1) & 3)),
// so every operand tile of an MMA step (128 or TN rows of one slice and
// k-block) is one contiguous, pre-swizzled run: the producer moves it with one
// bulk copy (cp.async.bulk, no tensor map, no multicast) and the UMMA
// shared-memory descriptors use the SWIZZLE_64B K-major canonical layout.
// Warp roles per CTA (one 128 x TN output tile at a time): warp 0 issues the
// copies, warp 1 owns TMEM and issues tcgen05.mma from one thread, warps 2-9
// drain the accumulators (two warps per TMEM lane quarter, one per half of
// the columns) and write C.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "kernels.cuh"

namespace tnt {

namespace {

constexpr int TM = kSplitTileM;   // 128 rows per tile (TMEM lanes)
constexpr int KB = 32;            // K elements per block: one 64-byte swizzle row
constexpr int KCHUNK = 512;       // exact-accumulation chunk
constexpr int KB_PER_CHUNK = KCHUNK / KB;
constexpr int kEpiWarps = 8;  // two epilogue warps per TMEM lane quarter, one per half of the tile's columns
constexpr int kSplitThreads = 32 * (2 + kEpiWarps);
constexpr int A_TILE_BYTES = TM * KB * 2;  // 8 KiB
template <int TN>
__host__ __device__ constexpr int b_tile_bytes() { return TN * KB * 2; }  // 4 KiB (N = 64) or 8 KiB (N = 128)
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 2 GHz

// Per-sector packing record of the split operands (one batch entry).
struct SplitJob {
  int64_t m, n, k, a_off, b_off, c_off, lda, ldb, ldc;
  int64_t m_pad, n_pad, k_pad;
  int64_t a_pack, b_pack;          // element offset of slice 0 within one batch entry
  int64_t a_scale, b_scale;        // offset of the row / column scales within one batch entry
};

struct SplitDims {
  int64_t a_stride, b_stride;      // bf16 elements per batch entry
  int64_t as_stride, bs_stride;    // scales per batch entry (= rows of A / columns of B, padded)
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes));
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)));
}

// Bounded wait on phase `parity`; returns false after ~2 s (the caller records an error).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t addr = smem_u32(bar);
  long long start = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity));
    if (done) return true;
    if (clock64() - start > kWaitCycles) return false;
  }
}

// Contiguous global -> shared copy by the bulk-copy engine, completing on
// `bar` (both addresses 16-byte aligned, bytes a multiple of 16).  The packs
// are written pre-swizzled, so the plain copy lands in the SWIZZLE_64B
// layout the UMMA descriptors expect.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// UMMA shared-memory descriptor: K-major, SWIZZLE_64B, 8-row groups 512 B apart.
__device__ __forceinline__ uint64_t umma_desc_sw64(uint32_t smem_addr) {
  uint64_t d = 0;
  d |= (uint64_t)((smem_addr >> 4) & 0x3FFF);   // start address
  d |= (uint64_t)1 << 16;                        // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(512 >> 4) << 32;               // stride byte offset
  d |= (uint64_t)1 << 46;                        // descriptor version (tcgen05)
  d |= (uint64_t)4 << 61;                        // SWIZZLE_64B
  return d;
}

// Instruction descriptor: kind::f16, A = B = BF16, D = F32, K-major, M = 128, N = TN.
template <int TN>
__host__ __device__ constexpr uint32_t umma_idesc_bf16() {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// kind::i8: A = B = signed 8-bit, D = S32 (exact integer accumulation), M = 128, N = n.
__device__ __forceinline__ uint32_t umma_idesc_s8_n(int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
}

__device__ __forceinline__ void umma_s8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar)));
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 32 lanes x 16 columns of 32-bit words, no wait (pair with tmem_ld_wait).
__device__ __forceinline__ void tmem_ld16_raw(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// ---------------------------------------------------------------------------
// Split pass
// ---------------------------------------------------------------------------

__device__ __forceinline__ double pow2_scale(double amax) {
  if (!(amax > 0.0)) return 1.0;
  int e;
  frexp(amax, &e);  // amax = f 2^e, f in [0.5, 1)
  return ldexp(1.0, e);
}

// Cut 8 consecutive values (|x| < 1) into S slices of 7 bits each, 16 bytes
// (8 bf16) per slice: x ~ sum_s q_s 2^{-7(s+1)} with q_s the balanced
// base-128 digits of X = rint(x 2^{7S}) (one power-of-two scaling and one
// rounding): Y = X + 64 (1 + 128 + ... + 128^{S-1}), q_0 = floor(Y /
// 128^{S-1}) - 64 in [-128, 128], q_s = (floor(Y / 128^{S-1-s}) mod 128) - 64
// in [-64, 63], sum_s q_s 128^{S-1-s} = X.  Slice s is stored pre-scaled by
// 2^{-7s}: an integer of magnitude <= 128 times a power of two, exact in BF16.
template <int S>
__device__ __forceinline__ void cut8_store(const double (&x)[8], __nv_bfloat16* dst, int64_t slice_stride) {
  constexpr int kShift = 7 * S;
  constexpr long long kOffset = [] {
    long long c = 0;
    for (int j = 0; j < S; ++j) c = c * 128 + 64;
    return c;
  }();
  const double scale = (double)(1ull << kShift);
  long long y[8];
#pragma unroll
  for (int t = 0; t < 8; ++t) y[t] = __double2ll_rn(x[t] * scale) + kOffset;
  float w = 1.0f;  // 2^{-7s}
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const int sh = 7 * (S - 1 - s);
    uint32_t word[4];
#pragma unroll
    for (int t = 0; t < 8; t += 2) {
      const long long a = y[t] >> sh, b = y[t + 1] >> sh;  // arithmetic: floor division
      const int q0 = s == 0 ? (int)a - 64 : (int)(a & 127) - 64;
      const int q1 = s == 0 ? (int)b - 64 : (int)(b & 127) - 64;
      __nv_bfloat162 p = __floats2bfloat162_rn((float)q0 * w, (float)q1 * w);
      word[t / 2] = *reinterpret_cast<uint32_t*>(&p);
    }
    *reinterpret_cast<uint4*>(dst + s * slice_stride) = make_uint4(word[0], word[1], word[2], word[3]);
    w *= 0.0078125f;
  }
}

// ---------------------------------------------------------------------------
// 8-bit integer digits
// ---------------------------------------------------------------------------
//
// x' = x / sigma in (-1, 1) is cut into S signed digits of one rounded
// integer X = rint(x' 2^{8S-2}):
//   x' ~ sum_s d_s 2^{-6 - 8s},  d_0 in [-64, 64],  d_s in [-128, 127] (s >= 1),
// the balanced base-256 digits of X, stored as int8 without pre-scaling.  A
// digit product is at most 2^14, so the int32 sum of one diagonal d = s + t
// (at most d + 1 <= 6 pairs, at most 5 * 2^14 per k) stays exact over K
// chunks of 16384.  The epilogue forms sum_d 2^{-8d} acc_d exactly in
// integers (two parts below 2^53), rounds it to FP64 once and scales the tile
// by 2^{-12} sigma tau.  Relative error of the product (the dropped diagonals
// d >= S and the rounding of X): about (S + 1) 2^{2-8S}, 4e-11 at S = 5.

constexpr int KB8 = 64;  // int8 K elements per k-block: one 64-byte swizzle row
constexpr int kMaxI8Slices = 6;

// Exact int64 -> double for |x| < 2^51 with one 64-bit integer add and one
// FP64 add instead of a 64-bit conversion instruction (a quarter-rate pipe):
// adding x to the bit pattern of 1.5 2^52 gives the double 1.5 2^52 + x, and
// subtracting 1.5 2^52 leaves x exactly.
__device__ __forceinline__ double i51_to_f64(long long x) {
  return __longlong_as_double(x + 0x4338000000000000LL) - 6755399441055744.0;
}

// byte b (0..3) of each of w0..w3, packed into one word (value t in byte t).
__device__ __forceinline__ uint32_t gather_byte(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3, int b) {
  const uint32_t sel = (uint32_t)b | ((uint32_t)(b + 4) << 4);
  return __byte_perm(__byte_perm(w0, w1, sel), __byte_perm(w2, w3, sel), 0x5410);
}

// One FMA per value produces every digit: v = x' 2^{8S-2} + (1.5 2^52 + C)
// with C = 128 (1 + 256 + ... + 256^{S-2}) is exact up to the one rounding
// of X (the product is a power-of-two scaling; v lies in [2^52, 2^53), where
// doubles are the integers), and the low 52 bits of v are 2^51 + Y with
// Y = X + C.  For S <= 6, 2^51 is a multiple of 2^{8S}, so byte b of v is
// byte b of Y in two's complement: bytes 0..S-2 are u_s = d_s + 128 of the
// low digits (digit S-1-b; the int8 bits of d_s are u_s ^ 0x80), byte S-1 is
// the top digit d_0 itself (Y = d_0 256^{S-1} + sum u_s 256^{S-1-s}).  The
// digits are then a byte transpose of the eight values' low words.
template <int S>
__device__ __forceinline__ void cut8_store_s8(const double (&x)[8], int8_t* dst, int64_t slice_stride) {
  static_assert(S >= 1 && S <= kMaxI8Slices, "8-bit digits: 1..6 per value");
  constexpr unsigned long long kOffset = [] {
    unsigned long long c = 0;
    for (int j = 0; j < S - 1; ++j) c = c * 256 + 128;
    return c;
  }();
  constexpr unsigned long long kFlip = [] {
    unsigned long long m = 0;
    for (int j = 0; j < S - 1; ++j) m |= 0x80ull << (8 * j);
    return m;
  }();
  constexpr double kMagic = 6755399441055744.0 + (double)kOffset;  // 1.5 * 2^52 + C, an exact integer
  const double scale = (double)(1ull << (8 * S - 2));
  uint32_t w[2][S];  // digit s of values 0-3 (w[0]) and 4-7 (w[1])
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    uint32_t lo[4], hi[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const unsigned long long v = (unsigned long long)__double_as_longlong(fma(x[4 * h + t], scale, kMagic)) ^ kFlip;
      lo[t] = (uint32_t)v;
      hi[t] = (uint32_t)(v >> 32);
    }
#pragma unroll
    for (int s = 0; s < S; ++s) {
      const int b = S - 1 - s;  // byte of digit s
      w[h][s] = b < 4 ? gather_byte(lo[0], lo[1], lo[2], lo[3], b) : gather_byte(hi[0], hi[1], hi[2], hi[3], b - 4);
    }
  }
#pragma unroll
  for (int s = 0; s < S; ++s) *reinterpret_cast<uint2*>(dst + s * slice_stride) = make_uint2(w[0][s], w[1][s]);
}

// ---------------------------------------------------------------------------
// Fused scale-and-slice passes (one read of each operand from HBM)
// ---------------------------------------------------------------------------
//
// A: one CTA per (32-row group of a job, batch entry); lane = row, warp w
// takes k = 64 it + 8 w .. + 7.  Pass 1 reduces the row maxima over the whole
// K (across the 8 warps in shared memory) into the power-of-two scale; pass 2
// re-reads the same rows (now cached) and writes every slice.  B: one CTA per
// 32-column group; 8 threads per column, each taking 8 consecutive k (64
// contiguous doubles of a column per iteration), maxima reduced by shuffles
// within the 8-lane group.  BF16 slices fill two 32-wide k-blocks per
// iteration; int8 digits one 64-wide k-block.

// K-chunked packing of A (operands with few rows and a long K, whose fused
// pass would run one long sequential loop on a few CTAs): kPackAmax reduces
// each chunk's row maxima into `scales` (zeroed first) with an integer
// atomicMax on the bits of the non-negative maxima, kPackCut cuts each chunk
// with the scale derived from the full maxima, and pack_scale_kernel turns the
// maxima into the power-of-two scales.  kPackFused does all of it in one pass.
enum : int { kPackFused = 0, kPackAmax = 1, kPackCut = 2 };
constexpr int kPackChunkIts = 4;  // 64-k iterations per chunk

__global__ void pack_scale_kernel(double* __restrict__ scales, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    scales[i] = pow2_scale(scales[i]);
}

template <int S, bool I8, int MODE = kPackFused>
__global__ void __launch_bounds__(256, 4) pack_a_kernel(const SplitJob* __restrict__ jobs,
                                                     const int32_t* __restrict__ group_job, SplitDims dims,
                                                     const double* __restrict__ A, int64_t sa,
                                                     double* __restrict__ scales, void* __restrict__ pack) {
  __shared__ double red[8][32];
  __shared__ __align__(16) uint8_t tile[(I8 ? 1 : 2) * S * 2048];  // one iteration's slices
  const int64_t group = blockIdx.x, batch = blockIdx.y;
  const SplitJob J = jobs[group_job[group]];
  // A group made only of padding rows (m_pad rounds m up to the 128-row
  // tile) is skipped: an output row depends only on its own row of A, and the
  // multiply never writes rows beyond m, so those digits and scales are never
  // used.  Padding rows inside a live group still get zero digits.
  if (group * 32 - J.a_scale >= J.m) return;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t row = group * 32 - J.a_scale + lane;  // row within the job (padded rows beyond m read zero)
  const bool live = row < J.m;
  const double* a = A + batch * sa + J.a_off + row;
  const int64_t nit_all = J.k_pad / 64;
  // This CTA's 64-k iterations [it0, nit): all of them, or one chunk.
  const int64_t it0 = MODE == kPackFused ? 0 : (int64_t)blockIdx.z * kPackChunkIts;
  const int64_t nit = MODE == kPackFused ? nit_all : (nit_all < it0 + kPackChunkIts ? nit_all : it0 + kPackChunkIts);
  if (MODE != kPackFused && it0 >= nit) return;  // the whole CTA: this job's K ends before the chunk
  // Loads of one 64-k iteration of this thread: lane = row, k = 64 it + 8 w + i.
  // The address of k = 64 it + 8 w is formed once per iteration and stepped
  // by lda; an iteration wholly inside K needs no per-element bound checks.
  const int64_t lda = J.lda;
  auto load = [&](double (&v)[8], int64_t it) {
    const int64_t k0 = it * 64 + w * 8;
    const double* p = a + k0 * lda;
    if (live && k0 + 8 <= J.k) {
#pragma unroll
      for (int i = 0; i < 8; ++i, p += lda) v[i] = __ldg(p);
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i, p += lda) v[i] = (live && k0 + i < J.k) ? __ldg(p) : 0.0;
    }
  };
  double* srow = scales + batch * dims.as_stride + J.a_scale + row;
  double m = 0.0;
  if constexpr (MODE != kPackCut) {
    double amax = 0.0;
    if (live) {
      int64_t it = it0;
      for (; it + 1 < nit; it += 2) {  // two iterations of loads in flight
        double u[8], v[8];
        load(u, it);
        load(v, it + 1);
#pragma unroll
        for (int i = 0; i < 8; ++i) amax = fmax(amax, fmax(fabs(u[i]), fabs(v[i])));
      }
      if (it < nit) {
        double u[8];
        load(u, it);
#pragma unroll
        for (int i = 0; i < 8; ++i) amax = fmax(amax, fabs(u[i]));
      }
    }
    red[w][lane] = amax;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 8; ++i) m = fmax(m, red[i][lane]);
    if constexpr (MODE == kPackAmax) {
      // non-negative doubles order like their bit patterns
      if (w == 0 && m > 0.0)
        atomicMax(reinterpret_cast<unsigned long long*>(srow), (unsigned long long)__double_as_longlong(m));
      return;
    }
  } else {
    m = *srow;  // the full row maximum left by the kPackAmax launch
  }
  const double sigma = pow2_scale(m), inv = 1.0 / sigma;
  if (MODE == kPackFused && w == 0) *srow = sigma;
  // Pass 2.  Each iteration cuts 32 rows x 64 k into shared memory (lane =
  // row, coalesced reads) and writes every slice's 32 x 64-byte piece -- one
  // contiguous 2 KB run per slice and k-block -- with 16-byte stores.  The
  // loads of the next iteration are issued before this one is cut.  In the
  // tile, the 16-byte chunk q of row r sits at chunk q ^ ((r >> 1) & 3), so
  // the row-strided stores of a warp spread over all banks.
  const int64_t elem = I8 ? 1 : 2;
  const int64_t slice_bytes = J.m_pad * J.k_pad * elem;
  uint8_t* base = static_cast<uint8_t*>(pack) + (batch * dims.a_stride + J.a_pack) * elem +
                  (group * 32 - J.a_scale) * 64;  // row 0 of this group, k-block 0, slice 0
  const int swz = (lane >> 1) & 3;
  double x[8];
  if (nit > it0) load(x, it0);
  for (int64_t it = it0; it < nit; ++it) {
    double nx[8];
    if (it + 1 < nit) load(nx, it + 1);
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] *= inv;
    if constexpr (I8) {
      // tile[s][row][64 bytes]; warp w holds bytes 8w .. 8w + 7 of the row
      cut8_store_s8<S>(x, reinterpret_cast<int8_t*>(tile) + lane * 64 + ((((w >> 1) ^ swz) << 4) | ((w & 1) << 3)),
                       32 * 64);
    } else {
      // tile[s][kb 0..1][row][32 bf16]; warp w holds chunk w & 3 of k-block w >> 2
      cut8_store<S>(x, reinterpret_cast<__nv_bfloat16*>(tile) + (w >> 2) * 32 * 32 + lane * 32 + (((w & 3) ^ swz) << 3),
                    2 * 32 * 32);
    }
    __syncthreads();
    constexpr int kPieces = I8 ? S : 2 * S;  // 2 KB pieces per iteration
    const int c = threadIdx.x & 127;
    for (int p = threadIdx.x >> 7; p < kPieces; p += 2) {
      const int s = I8 ? p : p >> 1;
      const int64_t kb = I8 ? it : 2 * it + (p & 1);
      const uint4* src = reinterpret_cast<const uint4*>(tile + p * 2048);
      uint4* dst = reinterpret_cast<uint4*>(base + s * slice_bytes + kb * J.m_pad * 64);
      dst[c] = src[c];  // the tile is already in the 64-byte swizzle
    }
    __syncthreads();
    if (it + 1 < nit) {
#pragma unroll
      for (int i = 0; i < 8; ++i) x[i] = nx[i];
    }
  }
}

// B: one CTA per 32-column group, one warp per 4 columns, 8 lanes per
// column.  Loads are coalesced along K (lane j of a column reads
// k = 64 it + j + 8 i: 64 contiguous bytes per column per load); before the
// cut, each warp transposes its 4 x 64 values through shared memory so every
// lane holds 8 consecutive k (the 8-byte digit words).  The shared-memory
// index k ^ ((k >> 3) & 7) in the low three bits keeps both the strided
// writes and the consecutive reads at the 2-wavefront minimum.
template <int S, bool I8>
__global__ void __launch_bounds__(256, 4) pack_b_kernel(const SplitJob* __restrict__ jobs,
                                                     const int32_t* __restrict__ group_job, SplitDims dims,
                                                     const double* __restrict__ B, int64_t sb,
                                                     double* __restrict__ scales, void* __restrict__ pack) {
  __shared__ double tr[8][4][64];
  const int64_t group = blockIdx.x, batch = blockIdx.y;
  const SplitJob J = jobs[group_job[group]];
  if (group * 32 - J.b_scale >= J.n) return;  // only padding columns: never reach a written output column
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = lane >> 3, seg = lane & 7;
  const int64_t col = group * 32 - J.b_scale + (threadIdx.x >> 3);
  const bool live = col < J.n;
  const double* b = B + batch * sb + J.b_off + col * J.ldb;
  const int64_t nit = J.k_pad / 64;
  // Loads of one 64-k iteration of this thread: k = 64 it + seg + 8 i.
  auto load = [&](double (&v)[8], int64_t it) {
    const int64_t k0 = it * 64 + seg;
    const double* p = b + k0;
    if (live && it * 64 + 64 <= J.k) {
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] = __ldg(p + 8 * i);
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] = (live && k0 + 8 * i < J.k) ? __ldg(p + 8 * i) : 0.0;
    }
  };
  double amax = 0.0;
  if (live) {
    int64_t it = 0;
    for (; it + 1 < nit; it += 2) {  // two iterations of loads in flight
      double u[8], v[8];
      load(u, it);
      load(v, it + 1);
#pragma unroll
      for (int i = 0; i < 8; ++i) amax = fmax(amax, fmax(fabs(u[i]), fabs(v[i])));
    }
    if (it < nit) {
      double u[8];
      load(u, it);
#pragma unroll
      for (int i = 0; i < 8; ++i) amax = fmax(amax, fabs(u[i]));
    }
  }
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
  const double sigma = pow2_scale(amax), inv = 1.0 / sigma;
  if (seg == 0) scales[batch * dims.bs_stride + J.b_scale + col] = sigma;
  const int64_t slice_stride = J.n_pad * J.k_pad;
  double* t = &tr[warp][c][0];
  double x[8];
  if (nit > 0) load(x, 0);
  for (int64_t it = 0; it < nit; ++it) {
    double nx[8];  // the next iteration's loads, in flight while this one is cut
    if (it + 1 < nit) load(nx, it + 1);
#pragma unroll
    for (int i = 0; i < 8; ++i) t[8 * i + (seg ^ i)] = x[i] * inv;  // k = seg + 8 i
    __syncwarp();
    double y[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) y[j] = t[8 * seg + (j ^ seg)];  // k = 8 seg + j
    __syncwarp();
    if constexpr (I8) {
      int8_t* dst = static_cast<int8_t*>(pack) + batch * dims.b_stride + J.b_pack + it * J.n_pad * KB8 + col * KB8 +
                    ((((seg >> 1) ^ (int)((col >> 1) & 3)) << 4) | ((seg & 1) << 3));
      cut8_store_s8<S>(y, dst, slice_stride);
    } else {
      const int64_t kb = it * 2 + (seg >> 2);
      __nv_bfloat16* dst = static_cast<__nv_bfloat16*>(pack) + batch * dims.b_stride + J.b_pack +
                           kb * J.n_pad * KB + col * KB + (((seg & 3) ^ (int)((col >> 1) & 3)) << 3);
      cut8_store<S>(y, dst, slice_stride);
    }
    if (it + 1 < nit) {
#pragma unroll
      for (int i = 0; i < 8; ++i) x[i] = nx[i];
    }
  }
}

__host__ __device__ constexpr uint32_t tmem_cols_pow2(uint32_t c) {
  return c <= 32 ? 32 : c <= 64 ? 64 : c <= 128 ? 128 : c <= 256 ? 256 : 512;
}

// ---------------------------------------------------------------------------
// tcgen05 multiply
// ---------------------------------------------------------------------------

// I8 = false: BF16 slices, kind::f16, FP32 accumulators (diagonals 0-2 apart,
// the rest shared), K chunks of 512; one MMA per slice product.
// I8 = true: int8 digits, kind::i8, one exact S32 accumulator per diagonal d
// (columns d * TN .. of the set), K chunks of 16384.  The stage's B digits sit
// back to back in shared memory, B_0 .. B_{S-1} as one (S TN)-row K-major
// matrix, so A_i times the stacked [B_0 .. B_{S-1-i}] is ONE MMA of width
// (S - i) TN (two where that passes 256) written at columns i TN ..: the
// product A_i B_j lands on accumulator i + j.  The S(S+1)/2 digit products of
// a K step take S + 1 MMAs instead of S(S+1)/2, and A_i is read from shared
// memory once per K step instead of S - i times.
// Both formats move 64-byte K rows, so tiles, swizzle and descriptors are the
// same.  GemmTile::k carries the job's K, so the MMA issuer needs no job
// lookup; each role reads its next tile (and the producer its next job) one
// tile ahead.
template <int S, int TN, bool I8>
__global__ void __launch_bounds__(kSplitThreads, 1)
    split_mma_kernel(const uint8_t* __restrict__ apack, const uint8_t* __restrict__ bpack,
                     const SplitJob* __restrict__ jobs, const GemmTile* __restrict__ tiles, int32_t ntiles,
                     SplitDims dims, const double* __restrict__ a_scales, const double* __restrict__ b_scales,
                     double* __restrict__ C, int64_t sc, double alpha, double beta, int nstage,
                     int32_t* __restrict__ err) {
  constexpr int KBX = I8 ? KB8 : KB;                  // K elements per k-block
  constexpr int64_t kElem = I8 ? 1 : 2;               // bytes per pack element
  constexpr int KCH = I8 ? 16384 / KB8 : KB_PER_CHUNK;  // k-blocks per exact-accumulation chunk
  constexpr int NACC = I8 ? S : (S < 4 ? S : 4);      // accumulators per set
  constexpr int B_TILE_BYTES = b_tile_bytes<TN>();
  constexpr uint32_t SET_COLS = (I8 ? S : 4) * TN;    // columns per accumulator set
  constexpr int NSETS = 2 * SET_COLS <= 512 ? 2 : 1;  // double-buffered when two sets fit in TMEM
  constexpr uint32_t NCOLS = tmem_cols_pow2(NSETS * SET_COLS);
  constexpr int kStack = 256 / TN;                    // B digit tiles per stacked MMA (N <= 256)
  static_assert(NSETS * SET_COLS <= 512, "accumulators exceed TMEM");
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  constexpr int stage_bytes = S * (A_TILE_BYTES + b_tile_bytes<TN>());
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + nstage * stage_bytes);
  uint64_t* empty = full + nstage;
  uint64_t* acc_full = empty + nstage;   // [2]
  uint64_t* acc_empty = acc_full + 2;    // [2]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_empty + 2);
  volatile int* bail = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int32_t step = (int32_t)gridDim.x;
  auto nkb_of = [](const GemmTile& tl) { return (int64_t)((tl.k + 63) / 64) * (64 / KBX); };

  if (threadIdx.x == 0) {
    for (int s = 0; s < nstage; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int s = 0; s < 2; ++s) {
      mbar_init(&acc_full[s], 1);
      mbar_init(&acc_empty[s], 32 * kEpiWarps);
    }
    *bail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(NCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    // ---- bulk-copy producer ------------------------------------------------
    if (lane == 0) {
      int64_t it = 0;
      int32_t t = blockIdx.x;
      // Two tiles and one job ahead, so no load of the tile table waits at a tile boundary.
      GemmTile t1 = t < ntiles ? tiles[t] : GemmTile{};
      GemmTile t2 = t + step < ntiles ? tiles[t + step] : GemmTile{};
      SplitJob j1 = jobs[t < ntiles ? t1.job : 0];
      for (; t < ntiles && !*bail; t += step) {
        const GemmTile tile = t1;
        const SplitJob J = j1;
        t1 = t2;
        if (t + step < ntiles) j1 = jobs[t1.job];
        if (t + 2 * step < ntiles) t2 = tiles[t + 2 * step];
        const int64_t nkb = J.k_pad / KBX;
        const int64_t abase = tile.batch * dims.a_stride + J.a_pack + (int64_t)tile.tm * TM * KBX;
        const int64_t bbase = tile.batch * dims.b_stride + J.b_pack + (int64_t)tile.tn * TN * KBX;
        for (int64_t kb = 0; kb < nkb; ++kb, ++it) {
          const int st = (int)(it % nstage);
          if (!mbar_wait(&empty[st], (uint32_t)(((it / nstage) & 1) ^ 1))) {
            atomicExch(err, 1);
            *bail = 1;
            break;
          }
          uint8_t* sbase = smem + st * stage_bytes;
          mbar_expect_tx(&full[st], (uint32_t)stage_bytes);
#pragma unroll
          for (int s = 0; s < S; ++s) {
            const int64_t ea = abase + (int64_t)s * J.m_pad * J.k_pad + kb * J.m_pad * KBX;
            bulk_load(sbase + s * A_TILE_BYTES, apack + ea * kElem, A_TILE_BYTES, &full[st]);
            const int64_t eb = bbase + (int64_t)s * J.n_pad * J.k_pad + kb * J.n_pad * KBX;
            bulk_load(sbase + S * A_TILE_BYTES + s * B_TILE_BYTES, bpack + eb * kElem, B_TILE_BYTES, &full[st]);
          }
        }
      }
    }
  } else if (warp == 1) {
    // ---- MMA issuer (one thread) -------------------------------------------
    if (lane == 0) {
      int64_t it = 0, round = 0;
      int32_t t = blockIdx.x;
      GemmTile nxt = t < ntiles ? tiles[t] : GemmTile{};
      for (; t < ntiles && !*bail; t += step) {
        const GemmTile tile = nxt;
        if (t + step < ntiles) nxt = tiles[t + step];
        const int64_t nkb = nkb_of(tile);
        uint32_t tacc = 0;
        bool fresh[NACC];
#pragma unroll
        for (int a = 0; a < NACC; ++a) fresh[a] = true;
        for (int64_t kb = 0; kb < nkb; ++kb, ++it) {
          const int64_t kin = kb % KCH;
          if (kin == 0) {
            const int set = (int)(round % NSETS);
            if (round >= NSETS) {
              if (!mbar_wait(&acc_empty[set], (uint32_t)((round / NSETS - 1) & 1))) {
                atomicExch(err, 2);
                *bail = 1;
                break;
              }
            }
            tc_fence_after();
            tacc = tmem + (uint32_t)set * SET_COLS;
#pragma unroll
            for (int a = 0; a < NACC; ++a) fresh[a] = true;
          }
          const int st = (int)(it % nstage);
          if (!mbar_wait(&full[st], (uint32_t)((it / nstage) & 1))) {
            atomicExch(err, 3);
            *bail = 1;
            break;
          }
          tc_fence_after();
          const uint32_t sa = smem_u32(smem + st * stage_bytes);
          const uint32_t sbb = sa + S * A_TILE_BYTES;
          if constexpr (I8) {
#pragma unroll
            for (int kk = 0; kk < 2; ++kk) {  // two 32-byte K steps per 64-byte row
              // The first MMA of a chunk (i = 0 spans every accumulator) overwrites.
              const uint32_t first = (kin == 0 && kk == 0) ? 0u : 1u;
#pragma unroll
              for (int i = 0; i < S; ++i) {
                const uint64_t ad = umma_desc_sw64(sa + i * A_TILE_BYTES + kk * 32);
#pragma unroll
                for (int j0 = 0; j0 < S - i; j0 += kStack) {
                  const int nj = S - i - j0 < kStack ? S - i - j0 : kStack;
                  const uint64_t bd = umma_desc_sw64(sbb + j0 * B_TILE_BYTES + kk * 32);
                  umma_s8(tacc + (uint32_t)((i + j0) * TN), ad, bd, umma_idesc_s8_n(nj * TN), i == 0 ? first : 1u);
                }
              }
            }
          } else {
            const uint32_t idesc = umma_idesc_bf16<TN>();
#pragma unroll
            for (int d = 0; d < S; ++d) {
              const int acc = d < NACC - 1 ? d : NACC - 1;
#pragma unroll
              for (int i = 0; i <= d; ++i) {
                const int j = d - i;
#pragma unroll
                for (int kk = 0; kk < 2; ++kk) {  // two 32-byte K steps per 64-byte row
                  const uint64_t ad = umma_desc_sw64(sa + i * A_TILE_BYTES + kk * 32);
                  const uint64_t bd = umma_desc_sw64(sbb + j * B_TILE_BYTES + kk * 32);
                  umma_bf16(tacc + (uint32_t)(acc * TN), ad, bd, idesc, fresh[acc] ? 0u : 1u);
                  fresh[acc] = false;
                }
              }
            }
          }
          umma_commit(&empty[st]);
          if (kin == KCH - 1 || kb == nkb - 1) {
            umma_commit(&acc_full[round % NSETS]);
            ++round;
          }
        }
      }
    }
  } else {
    // ---- epilogue: warps 2..9; TMEM lane quarter = warp % 4, column half = (warp - 2) / 4
    // Each chunk's accumulators are summed in FP64 and added into C directly
    // (the first chunk applies alpha/beta), so no FP64 tile lives in registers.
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    constexpr int HC = TN / 2;  // columns per epilogue warp
    int64_t round = 0;
    int32_t t = blockIdx.x;
    GemmTile nxt = t < ntiles ? tiles[t] : GemmTile{};
    for (; t < ntiles; t += step) {
      if (*bail) break;
      const GemmTile tile = nxt;
      if (t + step < ntiles) nxt = tiles[t + step];
      const SplitJob J = jobs[tile.job];
      const int64_t nkb = J.k_pad / KBX;
      const int64_t nchunks = (nkb + KCH - 1) / KCH;
      const int64_t row = (int64_t)tile.tm * TM + q * 32 + lane;
      const bool live = row < J.m;
      // 2^-12 2^{-8(H-1)} (digits, H = min(S, 3) high diagonals) or 2^-14 (slices)
      constexpr double kTileScale = I8 ? (S == 1 ? 1.0 / 4096.0 : S == 2 ? 1.0 / 1048576.0 : 1.0 / 268435456.0)
                                       : 1.0 / 16384.0;
      const double sr = live ? a_scales[tile.batch * dims.as_stride + J.a_scale + row] * kTileScale * alpha : 0.0;
      const double* tcs = b_scales + tile.batch * dims.bs_stride + J.b_scale + (int64_t)tile.tn * TN;
      // The column scales of this warp's columns, one per lane (read before
      // the accumulators are ready; the writes fetch them by shuffle).
      constexpr int NTS = (HC + 31) / 32;
      double tsc[NTS];
#pragma unroll
      for (int u = 0; u < NTS; ++u) tsc[u] = (32 * u + lane < HC) ? __ldg(tcs + half * HC + 32 * u + lane) : 0.0;
      double* crow = C + tile.batch * sc + J.c_off + row;
      if (nchunks == 0) {  // k == 0: C = beta C on this warp's columns
        if (live)
          for (int cc = half * HC; cc < (half + 1) * HC; ++cc) {
            const int64_t col = (int64_t)tile.tn * TN + cc;
            if (col < J.n) {
              double* p = crow + col * J.ldc;
              *p = beta == 0.0 ? 0.0 : beta * *p;
            }
          }
        continue;
      }
      bool ok = true;
      for (int64_t chunk = 0; chunk < nchunks; ++chunk, ++round) {
        const int set = (int)(round % NSETS);
        if (!mbar_wait(&acc_full[set], (uint32_t)((round / NSETS) & 1))) {
          atomicExch(err, 4);
          *bail = 1;
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)set * SET_COLS;
        // Sum of the accumulators of columns [c0, c0 + 16) in FP64.
        auto drain16 = [&](int c0, double (&sum)[16]) {
          if constexpr (I8) {
            // The exact integer sum in two parts: hi = sum_{a<H} acc_a
            // 256^{H-1-a} (|hi| < 2^43) and lo = sum_{a<L} acc_{H+a}
            // 256^{L-1-a} (|lo| < 2^47), both exact as doubles; the value
            // hi + lo 2^{-8L} is rounded once (the FMA), and the remaining
            // 2^{-8(H-1)} sits in kTileScale.  The loads of up to three
            // accumulators are in flight before each wait.
            constexpr int H = NACC < 3 ? NACC : 3, L = NACC - H;
            uint32_t r[3][16];
#pragma unroll
            for (int a = 0; a < H; ++a) tmem_ld16_raw(tbase + (uint32_t)(a * TN + c0), r[a]);
            tmem_ld_wait();
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              long long h = 0;
#pragma unroll
              for (int a = 0; a < H; ++a) h = h * 256 + (long long)(int32_t)r[a][i];
              sum[i] = i51_to_f64(h);
            }
            if constexpr (L > 0) {
#pragma unroll
              for (int a = 0; a < L; ++a) tmem_ld16_raw(tbase + (uint32_t)((H + a) * TN + c0), r[a]);
              tmem_ld_wait();
              constexpr double kLo = L == 1 ? 1.0 / 256.0 : L == 2 ? 1.0 / 65536.0 : 1.0 / 16777216.0;
#pragma unroll
              for (int i = 0; i < 16; ++i) {
                long long l = 0;
#pragma unroll
                for (int a = 0; a < L; ++a) l = l * 256 + (long long)(int32_t)r[a][i];
                sum[i] = fma(i51_to_f64(l), kLo, sum[i]);
              }
            }
          } else {
#pragma unroll
            for (int i = 0; i < 16; ++i) sum[i] = 0.0;
#pragma unroll
            for (int a = 0; a < NACC; ++a) {
              float v[16];
              tmem_ld16(tbase + (uint32_t)(a * TN + c0), v);
#pragma unroll
              for (int i = 0; i < 16; ++i) sum[i] += (double)v[i];
            }
          }
        };
        auto write16 = [&](int c0, const double (&sum)[16]) {
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const int cw = c0 - half * HC + i;  // column within this warp's share (uniform)
            const double tau = __shfl_sync(0xffffffffu, tsc[cw >> 5], cw & 31);
            const int64_t col = (int64_t)tile.tn * TN + c0 + i;
            if (live && col < J.n) {
              double* p = crow + col * J.ldc;
              const double v = sr * tau * sum[i];
              if (chunk > 0) *p += v;
              else *p = beta == 0.0 ? v : fma(beta, *p, v);
            }
          }
        };
        if constexpr (HC == 32) {
          // Release the accumulators as soon as the second 16 columns are in
          // registers, so the next tile's MMAs run while they are written
          // (holding all 32 columns would spill at this block size).
          double sum[16];
          drain16(half * HC, sum);
          write16(half * HC, sum);
          drain16(half * HC + 16, sum);
          tc_fence_before();
          mbar_arrive(&acc_empty[set]);
          write16(half * HC + 16, sum);
        } else {
#pragma unroll 1
          for (int c0 = half * HC; c0 < (half + 1) * HC; c0 += 16) {
            double sum[16];
            drain16(c0, sum);
            write16(c0, sum);
          }
          tc_fence_before();
          mbar_arrive(&acc_empty[set]);
        }
      }
      if (!ok) break;
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(NCOLS));
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

struct Layout {
  std::vector<SplitJob> jobs;
  SplitDims dims;
  size_t off_jobs, off_apack, off_bpack, off_ascale, off_bscale, off_err, total;
};

// Slice packs of one format: kb K elements per k-block (a 64-byte row),
// `elem` bytes per element (BF16: 32 x 2; int8: 64 x 1).
Layout make_layout(const GemmJob* host_jobs, int32_t njobs, int64_t nbatch, int S, int TN, bool i8) {
  const int64_t kb = i8 ? KB8 : KB, elem = i8 ? 1 : 2;
  Layout L;
  int64_t ap = 0, bp = 0, as = 0, bs = 0;
  for (int32_t j = 0; j < njobs; ++j) {
    const GemmJob& g = host_jobs[j];
    SplitJob s{};
    s.m = g.m;
    s.n = g.n;
    s.k = g.k;
    s.a_off = g.a_off;
    s.b_off = g.b_off;
    s.c_off = g.c_off;
    s.lda = g.lda;
    s.ldb = g.ldb;
    s.ldc = g.ldc;
    s.m_pad = round_up(std::max<int64_t>(g.m, 1), TM);
    s.n_pad = round_up(std::max<int64_t>(g.n, 1), TN);  // TN: the layout's tile width
    s.k_pad = round_up(g.k, 64);  // whole 64-element iterations of the pack kernels
    s.a_pack = ap;
    s.b_pack = bp;
    s.a_scale = as;
    s.b_scale = bs;
    ap += (int64_t)S * s.m_pad * s.k_pad;
    bp += (int64_t)S * s.n_pad * s.k_pad;
    as += s.m_pad;
    bs += s.n_pad;
    L.jobs.push_back(s);
  }
  L.dims.a_stride = std::max<int64_t>(ap, kb);
  L.dims.b_stride = std::max<int64_t>(bp, kb);
  L.dims.as_stride = as;
  L.dims.bs_stride = bs;
  auto al = [](size_t x) { return (x + 1023) & ~size_t(1023); };
  size_t o = 0;
  L.off_jobs = o;
  o = al(o + L.jobs.size() * sizeof(SplitJob));
  L.off_apack = o;
  o = al(o + (size_t)nbatch * L.dims.a_stride * elem);
  L.off_bpack = o;
  o = al(o + (size_t)nbatch * L.dims.b_stride * elem);
  L.off_ascale = o;
  o = al(o + (size_t)nbatch * std::max<int64_t>(as, 1) * 8);
  L.off_bscale = o;
  o = al(o + (size_t)nbatch * std::max<int64_t>(bs, 1) * 8);
  L.off_err = o;
  o = al(o + 64);
  L.total = o;
  return L;
}

// The uploaded per-plan table: the SplitJob records, then the job index of
// every 32-row group of A and every 32-column group of B (so a pack CTA finds
// its job with one load).
struct TableLayout {
  size_t a_groups, b_groups, total;
};

TableLayout table_layout(const Layout& L) {
  auto al = [](size_t x) { return (x + 15) & ~size_t(15); };
  TableLayout T;
  T.a_groups = al(L.jobs.size() * sizeof(SplitJob));
  T.b_groups = al(T.a_groups + (size_t)(L.dims.as_stride / 32) * sizeof(int32_t));
  T.total = al(T.b_groups + (size_t)(L.dims.bs_stride / 32) * sizeof(int32_t));
  return T;
}

template <int S, bool I8>
void pack_a_launch(cudaStream_t st, const SplitJob* jobs, const int32_t* agj, SplitDims dims, const double* a, int64_t sa,
                   void* apack, double* ascale, int64_t nbatch, int kchunks) {
  const dim3 ga((unsigned)(dims.as_stride / 32), (unsigned)nbatch);
  if (kchunks <= 1) {
    pack_a_kernel<S, I8><<<ga, 256, 0, st>>>(jobs, agj, dims, a, sa, ascale, apack);
    return;
  }
  const dim3 gz(ga.x, ga.y, (unsigned)kchunks);
  const int64_t nscale = nbatch * dims.as_stride;
  cudaMemsetAsync(ascale, 0, (size_t)nscale * sizeof(double), st);
  pack_a_kernel<S, I8, kPackAmax><<<gz, 256, 0, st>>>(jobs, agj, dims, a, sa, ascale, apack);
  pack_a_kernel<S, I8, kPackCut><<<gz, 256, 0, st>>>(jobs, agj, dims, a, sa, ascale, apack);
  const int64_t blocks = (nscale + 255) / 256;
  pack_scale_kernel<<<(unsigned)(blocks < 4096 ? blocks : 4096), 256, 0, st>>>(ascale, nscale);
}

template <int S>
cudaError_t split_passes_t(cudaStream_t st, const SplitJob* jobs, const int32_t* agj, const int32_t* bgj, SplitDims dims,
                           const double* a,
                           int64_t sa, void* apack, double* ascale, const double* b, int64_t sb, void* bpack,
                           double* bscale, int64_t nbatch, bool i8, int kchunks) {
  // A null source skips that side (its packs were made beforehand).
  const dim3 gb((unsigned)(dims.bs_stride / 32), (unsigned)nbatch);
  if (i8) {
    if constexpr (S <= kMaxI8Slices) {
      if (a) pack_a_launch<S, true>(st, jobs, agj, dims, a, sa, apack, ascale, nbatch, kchunks);
      if (b) pack_b_kernel<S, true><<<gb, 256, 0, st>>>(jobs, bgj, dims, b, sb, bscale, bpack);
    } else {
      return cudaErrorInvalidValue;
    }
  } else {
    if (a) pack_a_launch<S, false>(st, jobs, agj, dims, a, sa, apack, ascale, nbatch, kchunks);
    if (b) pack_b_kernel<S, false><<<gb, 256, 0, st>>>(jobs, bgj, dims, b, sb, bscale, bpack);
  }
  return cudaGetLastError();
}

cudaError_t launch_split_passes(int S, cudaStream_t st, const SplitJob* jobs, const int32_t* agj, const int32_t* bgj,
                                SplitDims dims,
                                const double* a, int64_t sa, void* apack, double* ascale, const double* b, int64_t sb,
                                void* bpack, double* bscale, int64_t nbatch, bool i8, int kchunks) {
  switch (S) {
#define TNT_SPLIT_CASE(n) \
  case n:                 \
    return split_passes_t<n>(st, jobs, agj, bgj, dims, a, sa, apack, ascale, b, sb, bpack, bscale, nbatch, i8, kchunks);
    TNT_SPLIT_CASE(1) TNT_SPLIT_CASE(2) TNT_SPLIT_CASE(3) TNT_SPLIT_CASE(4)
    TNT_SPLIT_CASE(5) TNT_SPLIT_CASE(6) TNT_SPLIT_CASE(7) TNT_SPLIT_CASE(8)
#undef TNT_SPLIT_CASE
    default: return cudaErrorInvalidValue;
  }
}

template <int S, int TN, bool I8>
cudaError_t mma_t(int ntiles, size_t smem, cudaStream_t st, const uint8_t* ma, const uint8_t* mb,
                  const SplitJob* jobs, const GemmTile* tiles, SplitDims dims, const double* ascale,
                  const double* bscale, double* c, int64_t sc, double alpha, double beta, int nstage, int32_t* err) {
  cudaError_t e =
      cudaFuncSetAttribute(split_mma_kernel<S, TN, I8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = ntiles < sms ? ntiles : sms;
  split_mma_kernel<S, TN, I8><<<grid, kSplitThreads, smem, st>>>(ma, mb, jobs, tiles, ntiles, dims, ascale, bscale, c,
                                                                 sc, alpha, beta, nstage, err);
  return cudaGetLastError();
}

template <int S>
cudaError_t mma_i8(int ntiles, size_t smem, cudaStream_t st, const uint8_t* ma, const uint8_t* mb,
                   const SplitJob* jobs, const GemmTile* tiles, SplitDims dims, const double* ascale,
                   const double* bscale, double* c, int64_t sc, double alpha, double beta, int nstage, int32_t* err) {
  if constexpr (S <= kMaxI8Slices)
    return mma_t<S, 64, true>(ntiles, smem, st, ma, mb, jobs, tiles, dims, ascale, bscale, c, sc, alpha, beta, nstage,
                              err);
  return cudaErrorInvalidValue;
}

// BF16 slices at tile width 64 or 128; int8 digits at width 64 (one S32
// accumulator per diagonal: S x 64 TMEM columns).
cudaError_t launch_mma(int S, int TN, bool i8, int ntiles, size_t smem, cudaStream_t st, const uint8_t* ma,
                       const uint8_t* mb, const SplitJob* jobs, const GemmTile* tiles, SplitDims dims,
                       const double* ascale, const double* bscale, double* c, int64_t sc, double alpha, double beta,
                       int nstage, int32_t* err) {
#define TNT_MMA_CASE(n)                                                                                          \
  case n:                                                                                                        \
    if (i8)                                                                                                      \
      return mma_i8<n>(ntiles, smem, st, ma, mb, jobs, tiles, dims, ascale, bscale, c, sc, alpha, beta, nstage,   \
                       err);                                                                                     \
    return TN == 128 ? mma_t<n, 128, false>(ntiles, smem, st, ma, mb, jobs, tiles, dims, ascale, bscale, c, sc,  \
                                            alpha, beta, nstage, err)                                            \
                     : mma_t<n, 64, false>(ntiles, smem, st, ma, mb, jobs, tiles, dims, ascale, bscale, c, sc,   \
                                           alpha, beta, nstage, err);
  switch (S) {
    TNT_MMA_CASE(1) TNT_MMA_CASE(2) TNT_MMA_CASE(3) TNT_MMA_CASE(4)
    TNT_MMA_CASE(5) TNT_MMA_CASE(6) TNT_MMA_CASE(7) TNT_MMA_CASE(8)
    default: return cudaErrorInvalidValue;
  }
#undef TNT_MMA_CASE
}

}  // namespace

int split_tile_n(const GemmJob* host_jobs, int32_t njobs, double eff64) {
  // Tile-width pick keyed on the sector-size histogram: estimated MMA time of
  // every job's padded tiles at N = 64 and N = 128, with the measured per-MAC
  // throughput ratio of the two widths (eff64; N = 64 issues twice as many
  // MMAs for the same work).  Overridable with TNT_SPLIT_TILE_N=64|128.
  if (const char* env = getenv("TNT_SPLIT_TILE_N")) {
    const int v = atoi(env);
    if (v == 64 || v == 128) return v;
  }
  double t64 = 0.0, t128 = 0.0;
  for (int32_t j = 0; j < njobs; ++j) {
    const GemmJob& g = host_jobs[j];
    const double m = (double)round_up(std::max<int64_t>(g.m, 1), TM), k = (double)round_up(g.k, KB);
    t64 += m * k * (double)round_up(std::max<int64_t>(g.n, 1), 64) / eff64;
    t128 += m * k * (double)round_up(std::max<int64_t>(g.n, 1), 128);
  }
  return t128 < t64 ? 128 : 64;
}

size_t split_scratch_bytes(const GemmJob* host_jobs, int32_t njobs, int64_t nbatch, int slices, int tile_n,
                           bool i8) {
  return make_layout(host_jobs, njobs, nbatch, slices, tile_n, i8).total;
}

double split_padded_macs(const GemmJob* host_jobs, int32_t njobs, int tile_n) {
  double w = 0.0;
  for (int32_t j = 0; j < njobs; ++j) {
    const GemmJob& g = host_jobs[j];
    w += (double)round_up(std::max<int64_t>(g.m, 1), TM) * (double)round_up(g.k, KB) *
         (double)round_up(std::max<int64_t>(g.n, 1), tile_n);
  }
  return w;
}

std::vector<uint8_t> split_job_table(const GemmJob* host_jobs, int32_t njobs, int slices, int tile_n, bool i8) {
  const Layout L = make_layout(host_jobs, njobs, 1, slices, tile_n, i8);
  const TableLayout T = table_layout(L);
  std::vector<uint8_t> out(T.total, 0);
  if (!L.jobs.empty()) std::memcpy(out.data(), L.jobs.data(), L.jobs.size() * sizeof(SplitJob));
  // job of every 32-row group of A and 32-column group of B (one batch entry)
  int32_t* ag = reinterpret_cast<int32_t*>(out.data() + T.a_groups);
  int32_t* bg = reinterpret_cast<int32_t*>(out.data() + T.b_groups);
  for (size_t j = 0; j < L.jobs.size(); ++j) {
    for (int64_t g = L.jobs[j].a_scale / 32; g < (L.jobs[j].a_scale + L.jobs[j].m_pad) / 32; ++g) ag[g] = (int32_t)j;
    for (int64_t g = L.jobs[j].b_scale / 32; g < (L.jobs[j].b_scale + L.jobs[j].n_pad) / 32; ++g) bg[g] = (int32_t)j;
  }
  return out;
}

namespace {

// K chunks of the A pack: A with few 32-row groups and a long K is packed in
// chunks, so the work spreads over the GPU instead of a few long-running CTAs.
int pack_a_chunks(const Layout& L, int64_t nbatch) {
  int64_t max_nit = 0;
  for (const SplitJob& j : L.jobs) max_nit = std::max<int64_t>(max_nit, j.k_pad / 64);
  int dev_sm = 148, cur_dev = 0;
  cudaGetDevice(&cur_dev);
  cudaDeviceGetAttribute(&dev_sm, cudaDevAttrMultiProcessorCount, cur_dev);
  const int64_t a_ctas = (L.dims.as_stride / 32) * nbatch;
  if (a_ctas < (int64_t)dev_sm * 8 && max_nit > 2 * kPackChunkIts)
    return (int)std::min<int64_t>(65535, (max_nit + kPackChunkIts - 1) / kPackChunkIts);
  return 1;
}

// Byte offsets of one side's slices and scales inside a pre-packed operand
// (one batch entry): [slices][scales], each 1024-byte aligned.
struct OperandLayout {
  size_t pack, scale, total;
};

OperandLayout operand_layout(const Layout& L, int side, bool i8) {
  auto al = [](size_t x) { return (x + 1023) & ~size_t(1023); };
  const size_t elem = i8 ? 1 : 2;
  OperandLayout o;
  o.pack = 0;
  o.scale = al((size_t)(side == 0 ? L.dims.a_stride : L.dims.b_stride) * elem);
  o.total = al(o.scale + (size_t)std::max<int64_t>(side == 0 ? L.dims.as_stride : L.dims.bs_stride, 1) * 8);
  return o;
}

}  // namespace

size_t split_operand_bytes(const GemmJob* host_jobs, int32_t njobs, int slices, int tile_n, bool i8, int side) {
  return operand_layout(make_layout(host_jobs, njobs, 1, slices, tile_n, i8), side, i8).total;
}

cudaError_t launch_split_pack_operand(const void* job_table, const GemmJob* host_jobs, int32_t njobs, int side,
                                      const double* src, int slices, int tile_n, bool i8, void* packed,
                                      cudaStream_t stream) {
  if (njobs == 0) return cudaSuccess;
  if (slices < 1 || slices > (i8 ? kMaxI8Slices : 8) || (tile_n != 64 && tile_n != 128) || (i8 && tile_n != 64))
    return cudaErrorInvalidValue;
  const Layout L = make_layout(host_jobs, njobs, 1, slices, tile_n, i8);
  const OperandLayout o = operand_layout(L, side, i8);
  uint8_t* base = static_cast<uint8_t*>(packed);
  const SplitJob* djobs = static_cast<const SplitJob*>(job_table);
  const TableLayout T = table_layout(L);
  const int32_t* agj = reinterpret_cast<const int32_t*>(static_cast<const uint8_t*>(job_table) + T.a_groups);
  const int32_t* bgj = reinterpret_cast<const int32_t*>(static_cast<const uint8_t*>(job_table) + T.b_groups);
  double* scale = reinterpret_cast<double*>(base + o.scale);
  if (side == 0)
    return launch_split_passes(slices, stream, djobs, agj, bgj, L.dims, src, 0, base + o.pack, scale, nullptr, 0,
                               nullptr, nullptr, 1, i8, pack_a_chunks(L, 1));
  return launch_split_passes(slices, stream, djobs, agj, bgj, L.dims, nullptr, 0, nullptr, nullptr, src, 0,
                             base + o.pack, scale, 1, i8, 1);
}

cudaError_t launch_gemm_split(const void* job_table, const GemmJob* host_jobs, int32_t njobs, const GemmTile* tiles,
                              int32_t ntiles, double* c, int64_t sc, const double* a, int64_t sa, const double* b,
                              int64_t sb, int64_t nbatch, double alpha, double beta, int slices, int tile_n, bool i8,
                              void* scratch, size_t scratch_bytes, int32_t* err_word, cudaStream_t stream,
                              const void* pre_a, const void* pre_b) {
  if (ntiles == 0 || njobs == 0) return cudaSuccess;
  if (slices < 1 || slices > (i8 ? kMaxI8Slices : 8) || (tile_n != 64 && tile_n != 128) || (i8 && tile_n != 64))
    return cudaErrorInvalidValue;
  if ((pre_a || pre_b) && nbatch != 1) return cudaErrorInvalidValue;
  Layout L = make_layout(host_jobs, njobs, nbatch, slices, tile_n, i8);
  if (L.total > scratch_bytes) return cudaErrorInvalidValue;
  uint8_t* base = static_cast<uint8_t*>(scratch);
  // The per-job packing table is device-resident (uploaded once per plan by
  // the caller), so no host memory is read in stream order and the launch
  // sequence can be captured into a CUDA graph.
  const SplitJob* djobs = static_cast<const SplitJob*>(job_table);
  void* apack = base + L.off_apack;
  void* bpack = base + L.off_bpack;
  double* ascale = reinterpret_cast<double*>(base + L.off_ascale);
  double* bscale = reinterpret_cast<double*>(base + L.off_bscale);
  // A pre-packed side (one batch entry, split_operand_bytes long) replaces
  // that side's pack pass: the multiply reads its slices and scales directly.
  if (pre_a) {
    const OperandLayout o = operand_layout(L, 0, i8);
    apack = const_cast<uint8_t*>(static_cast<const uint8_t*>(pre_a)) + o.pack;
    ascale = reinterpret_cast<double*>(const_cast<uint8_t*>(static_cast<const uint8_t*>(pre_a)) + o.scale);
  }
  if (pre_b) {
    const OperandLayout o = operand_layout(L, 1, i8);
    bpack = const_cast<uint8_t*>(static_cast<const uint8_t*>(pre_b)) + o.pack;
    bscale = reinterpret_cast<double*>(const_cast<uint8_t*>(static_cast<const uint8_t*>(pre_b)) + o.scale);
  }
  // Pipeline waits that give up record their code in the caller's error word
  // (never cleared here: the caller reads and clears it when it synchronises).
  int32_t* err = err_word;
  if (nbatch > 65535 || L.dims.as_stride / 32 >= (1LL << 31) || L.dims.bs_stride / 32 >= (1LL << 31))
    return cudaErrorInvalidValue;
  const TableLayout T = table_layout(make_layout(host_jobs, njobs, 1, slices, tile_n, i8));
  const int32_t* agj = reinterpret_cast<const int32_t*>(static_cast<const uint8_t*>(job_table) + T.a_groups);
  const int32_t* bgj = reinterpret_cast<const int32_t*>(static_cast<const uint8_t*>(job_table) + T.b_groups);
  if (!pre_a || !pre_b) {
    cudaError_t e = launch_split_passes(slices, stream, djobs, agj, bgj, L.dims, pre_a ? nullptr : a, sa, apack,
                                        ascale, pre_b ? nullptr : b, sb, bpack, bscale, nbatch, i8,
                                        pre_a ? 1 : pack_a_chunks(L, nbatch));
    if (e != cudaSuccess) return e;
  }
  const uint8_t* ma = static_cast<const uint8_t*>(apack);
  const uint8_t* mb = static_cast<const uint8_t*>(bpack);
  const int stage_bytes = slices * (A_TILE_BYTES + tile_n * 64);
  const int max_smem = 227 * 1024;
  int nstage = std::min(4, (max_smem - 2048) / stage_bytes);
  if (nstage < 1) return cudaErrorInvalidValue;
  const size_t smem = 1024 + (size_t)nstage * stage_bytes + 256;
  return launch_mma(slices, tile_n, i8, ntiles, smem, stream, ma, mb, djobs, tiles, L.dims, ascale, bscale, c, sc,
                    alpha, beta, nstage, err);
}

}  // namespace tnt
