// Batched per-sector SVD and cross-sector truncation on the device.
//
// Replaces the serial sector loop of svd_compact_factors_dyn_with_direction
// (tenet-matrixalgebra/src/factorize.rs:1631-1760), which calls a dense SVD
// per coupled sector, the gauge fix svd_compact_gauge (factorize.rs:3836-3852)
// and the host-side select_truncation (tenet-matrixalgebra/src/truncation.rs:257-560).
//
// SVD: one CTA per coupled-sector matrix, one-sided (Hestenes) Jacobi.  The
// matrix (or its transpose when it is wide) is copied into a scratch panel W
// of k = min(m, n) columns; each sweep runs a round-robin tournament of
// disjoint column pairs, a group of 4-32 lanes per pair (several pairs per
// warp at once), rotating W and the accumulated
// right factor V until no pair's cosine exceeds 4 sqrt(rows) eps.  Singular values are the column
// norms, sorted descending; U columns are made largest-entry-positive.
// Truncation: one CTA evaluates the reference's sequential greedy rules in
// parallel -- every candidate singular value computes its position in the
// reference order by binary searches over the per-sector descending spectra.
#include <cfloat>

#include <map>
#include <mutex>

#include "kernels.cuh"

namespace tnt {

namespace {

constexpr int kSvdThreads = 1024;
constexpr size_t kSvdSmemBytes = 200 * 1024;  // panels up to this size stay in shared memory
constexpr int kMaxSweeps = 40;

__device__ __forceinline__ void cp_async8(double* smem_dst, const double* gmem_src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Round-robin (circle method) pairing: round r of a k2-player tournament
// (k2 even) pairs player k2-1 with r and (r+i) with (r-i) mod (k2-1).
__device__ __forceinline__ void tournament_pair(int r, int i, int k2, int& p, int& q) {
  int a, b;
  if (i == 0) {
    a = k2 - 1;
    b = r;
  } else {  // (r + i) mod (k2 - 1) and (r - i) mod (k2 - 1), with 0 <= r < k2 - 1 and 0 < i < k2 - 1
    a = r + i;
    if (a >= k2 - 1) a -= k2 - 1;
    b = r - i;
    if (b < 0) b += k2 - 1;
  }
  p = a < b ? a : b;
  q = a < b ? b : a;
}

}  // namespace

// Whether a sector's whole panel (W, V, values, ranks) fits the shared-memory
// budget, and the column-block width of the blocked path otherwise (0 when
// even two columns do not fit).  Shared by the kernels and the host, which
// sends sectors with at least kSvdCluster blocks to the cluster kernel.
__host__ __device__ bool svd_on_chip(int64_t rows, int64_t k) {
  return (size_t)(rows * k + k * k + 2 * k) * sizeof(double) <= kSvdSmemBytes;
}
__host__ __device__ int svd_block_width(int64_t rows, int64_t k) {
  const int64_t capd = (int64_t)(kSvdSmemBytes / sizeof(double));
  int bw = (int)(k < 64 ? k : 64);
  while (bw > 1 && 2 * bw * rows + 4 * (int64_t)bw * bw > capd) --bw;
  return bw < 2 ? 0 : bw;
}

namespace {

// Copy nc columns (length len, column gcol(c) of the column-major source)
// into the contiguous shared panel dst.  Incoherent: cp.async through L1,
// every load in flight at once.  Coherent: ld.global.cg (L2), eight loads in
// flight per thread before their shared-memory stores.
template <bool kCoherent, class F>
__device__ __forceinline__ void stage_columns(double* __restrict__ dst, const double* __restrict__ src, int64_t len,
                                              int nc, F gcol) {
  const int64_t total = (int64_t)nc * len;
  if constexpr (!kCoherent) {
    for (int64_t idx = threadIdx.x; idx < total; idx += blockDim.x) {
      const int c = (int)(idx / len);
      cp_async8(dst + idx, src + gcol(c) * len + (idx - (int64_t)c * len));
    }
    cp_async_commit_wait_all();
  } else {
    for (int64_t base = threadIdx.x; base < total; base += 8 * (int64_t)blockDim.x) {
      double v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int64_t idx = base + (int64_t)u * blockDim.x;
        v[u] = 0.0;
        if (idx < total) {
          const int c = (int)(idx / len);
          v[u] = __ldcg(src + gcol(c) * len + (idx - (int64_t)c * len));
        }
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int64_t idx = base + (int64_t)u * blockDim.x;
        if (idx < total) dst[idx] = v[u];
      }
    }
  }
}

// One step of the blocked one-sided Jacobi: columns [p0, p0 + np) and, for a
// cross step, [q0, q0 + nq) of W (rows x k) and V (k x k), both column-major
// in global memory, are staged into the shared panel Ws, every pair among
// them (within-block round robin when nq == 0, the np x nq cross pairs
// otherwise, np <= nq) is rotated there while the rotations accumulate in a
// 2 bw x 2 bw matrix Z, the columns go back and V's columns are multiplied by
// Z.  Sets *rotated when any pair rotated.  kCoherent: W and V may have been
// written by other CTAs (a cluster sharing one sector), so they are read at
// L2 (ld.global.cg) instead of through this SM's L1.
template <bool kCoherent>
__device__ void jacobi_block_step(double* __restrict__ W, double* __restrict__ V, double* __restrict__ Ws,
                                  int64_t rows, int64_t k, int64_t p0, int np, int64_t q0, int nq, int G, double tol,
                                  double noise2, double abs_floor, int* rotated) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const int gpw = 32 / G, sub = lane / G, gl = lane % G;
  const int nc = np + nq;
  double* Zs = Ws + (int64_t)nc * rows;
  auto gcol = [&](int c) { return c < np ? p0 + c : q0 + (c - np); };
  stage_columns<kCoherent>(Ws, W, rows, nc, [&](int c) { return gcol(c); });
  for (int idx = tid; idx < nc * nc; idx += blockDim.x) Zs[idx] = (idx % nc == idx / nc) ? 1.0 : 0.0;
  __syncthreads();
  const int n2 = (np + 1) & ~1;
  const int nrounds = nq == 0 ? n2 - 1 : nq;   // within-block round robin, or nq cross rounds
  const int ppr = nq == 0 ? n2 / 2 : np;       // pairs per round (np <= nq for cross steps)
  for (int r = 0; r < nrounds; ++r) {
    for (int base = warp * gpw; base < ppr; base += nwarps * gpw) {
      const int i = base + sub;
      int p = 0, q = 0;
      bool live = i < ppr;
      if (live) {
        if (nq == 0) {
          tournament_pair(r, i, n2, p, q);
          live = q < np;
        } else {
          p = i;
          q = np + (i + r) % nq;
        }
      }
      double* wp = Ws + (int64_t)p * rows;
      double* wq = Ws + (int64_t)q * rows;
      double al = 0.0, be = 0.0, ga = 0.0;
      if (live)
        for (int64_t x = gl; x < rows; x += G) {
          const double u = wp[x], v = wq[x];
          al = fma(u, u, al);
          be = fma(v, v, be);
          ga = fma(u, v, ga);
        }
      for (int o = G >> 1; o > 0; o >>= 1) {
        al += __shfl_xor_sync(0xffffffffu, al, o);
        be += __shfl_xor_sync(0xffffffffu, be, o);
        ga += __shfl_xor_sync(0xffffffffu, ga, o);
      }
      if (live && fabs(ga) > tol * sqrt(al * be) && fmin(al, be) > noise2 && fabs(ga) > abs_floor &&
          fabs(ga) > DBL_MIN) {
        const double zeta = (be - al) / (2.0 * ga);
        const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double cs = rsqrt(1.0 + t * t);
        const double sn = cs * t;
        for (int64_t x = gl; x < rows; x += G) {
          const double u = wp[x], v = wq[x];
          wp[x] = cs * u - sn * v;
          wq[x] = sn * u + cs * v;
        }
        double* zp = Zs + p * nc;
        double* zq = Zs + q * nc;
        for (int x = gl; x < nc; x += G) {
          const double u = zp[x], v = zq[x];
          zp[x] = cs * u - sn * v;
          zq[x] = sn * u + cs * v;
        }
        if (gl == 0) *rotated = 1;
      }
    }
    __syncthreads();
  }
  for (int64_t idx = tid; idx < (int64_t)nc * rows; idx += blockDim.x) {
    const int c = (int)(idx / rows);
    W[gcol(c) * rows + (idx - (int64_t)c * rows)] = Ws[idx];
  }
  __syncthreads();
  // V[:, cols] <- V[:, cols] Z, staging V's columns where W's were (k <= rows).
  stage_columns<kCoherent>(Ws, V, k, nc, [&](int c) { return gcol(c); });
  __syncthreads();
  // Each thread forms 8 outputs of one row: one shared-memory read of V
  // feeds 8 FMAs (Z entries are broadcast reads).
  const int ngrp = (nc + 7) >> 3;
  for (int64_t idx = tid; idx < (int64_t)ngrp * k; idx += blockDim.x) {
    const int g8 = (int)(idx / k);
    const int64_t r = idx - (int64_t)g8 * k;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int c = 0; c < nc; ++c) {
      const double v = Ws[(int64_t)c * k + r];
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (g8 * 8 + j < nc) acc[j] = fma(v, Zs[(g8 * 8 + j) * nc + c], acc[j]);
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (g8 * 8 + j < nc) V[gcol(g8 * 8 + j) * k + r] = acc[j];
  }
  __syncthreads();
}

// Scratch per job (doubles): W (rows x k), V (k x k), sorted values (k), rank (k).
__global__ void __launch_bounds__(kSvdThreads) svd_jacobi_kernel(const SvdJob* __restrict__ jobs,
                                                                 const double* __restrict__ A, double* __restrict__ U,
                                                                 double* __restrict__ S, double* __restrict__ VH,
                                                                 double* __restrict__ work,
                                                                 const int64_t* __restrict__ work_off,
                                                                 int32_t* __restrict__ status) {
  const SvdJob J = jobs[blockIdx.x];
  const int64_t m = J.m, n = J.n, k = J.k;
  if (k == 0) return;
  const bool wide = m < n;            // work on A^T so that the k columns are the short side
  const int64_t rows = wide ? n : m;  // length of each working column
  // Small sectors keep the panel and the rotations in shared memory.
  extern __shared__ __align__(16) double smem_panel[];
  const bool on_chip = svd_on_chip(rows, k);
  double* W = on_chip ? smem_panel : work + work_off[blockIdx.x];
  double* V = W + rows * k;  // k x k accumulated rotations, column-major
  double* sv = V + k * k;    // column norms
  double* rk = sv + k;       // descending rank of each column
  const double* a = A + J.a_off;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;

  for (int64_t idx = tid; idx < rows * k; idx += blockDim.x) {
    int64_t r = idx % rows, c = idx / rows;
    W[idx] = wide ? a[c + r * m] : a[r + c * m];
  }
  for (int64_t idx = tid; idx < k * k; idx += blockDim.x) V[idx] = (idx % k == idx / k) ? 1.0 : 0.0;
  __shared__ double red[32];
  double f2 = 0.0;
  for (int64_t idx = tid; idx < rows * k; idx += blockDim.x) f2 = fma(W[idx], W[idx], f2);
  f2 = warp_sum(f2);
  if (lane == 0) red[warp] = f2;
  __syncthreads();
  double frob2 = 0.0;
  for (int w = 0; w < nwarps; ++w) frob2 += red[w];
  // A pair is rotated only while (1) its cosine exceeds the orthogonality
  // tolerance, at the rounding level of a length-`rows` dot product (the
  // sqrt(rows) eps criterion of one-sided Jacobi codes), and (2) both columns
  // stand above the rounding-noise level rows * eps * ||A||_F.  In a
  // rank-deficient matrix the null-space columns shrink to that level, and
  // every rotation against a large column refills them with fresh rounding
  // noise whose cosine with it is O(1): without (2) they never settle.
  // Singular values below that level carry no accuracy in any backward-stable
  // SVD, so nothing is lost.
  const double abs_floor = 1e-28 * frob2;
  const double tol = 4.0 * sqrt((double)rows) * DBL_EPSILON;
  const double noise2 = ((double)rows * DBL_EPSILON) * ((double)rows * DBL_EPSILON) * frob2;

  __shared__ int rotated;
  const int k2 = (int)((k + 1) & ~1LL);
  // Lanes per pair: enough that each lane holds a handful of rows, whole
  // warps for long columns (coalesced global-memory panels).
  const int G = rows <= 64 ? 4 : rows <= 128 ? 8 : rows <= 256 ? 16 : 32;
  const int gpw = 32 / G, sub = lane / G, gl = lane % G;
  // In shared memory with even row and column counts every column starts on a
  // 16-byte boundary, so the pair loops move two rows per access.
  const bool vec2 = on_chip && (rows & 1) == 0 && (k & 1) == 0;
  const double tol2 = tol * tol;  // |ga| > tol sqrt(al be), compared squared
  const int rows2 = (int)(rows / 2), k2v = (int)(k / 2);
  int sweep = 0;
  // Panels too large for shared memory run blocked: column blocks of width bw
  // are staged in shared memory pairwise (2 bw columns and a 2 bw x 2 bw
  // rotation accumulator Z), every cross pair of the two blocks is rotated
  // there (bw rounds of disjoint pairs), the columns go back to global memory
  // and V's matching columns are multiplied by Z once.  One outer sweep visits
  // every pair exactly once (within-block pairs in a diagonal step per block),
  // like a cyclic sweep, but each rotation reads shared memory, not L2.
  // (bw == 0: columns too long even for two; unblocked global-memory sweeps)
  const int bw = on_chip ? 0 : svd_block_width(rows, k);
  double* Ws = smem_panel;  // blocked path: staged columns, column-major
  auto block_step = [&](int64_t p0, int np, int64_t q0, int nq) {
    jacobi_block_step<false>(W, V, Ws, rows, k, p0, np, q0, nq, G, tol, noise2, abs_floor, &rotated);
  };

  for (; sweep < kMaxSweeps && k > 1; ++sweep) {
    if (tid == 0) rotated = 0;
    __syncthreads();
    if (bw > 0) {
      const int nb = (int)((k + bw - 1) / bw);
      auto bsize = [&](int b) { return (int)((b + 1) * (int64_t)bw <= k ? bw : k - (int64_t)b * bw); };
      for (int b = 0; b < nb; ++b) block_step((int64_t)b * bw, bsize(b), 0, 0);
      for (int bi = 0; bi < nb; ++bi)
        for (int bj = bi + 1; bj < nb; ++bj) {
          // the smaller block takes the "p" side so the pairs of a round stay disjoint
          if (bsize(bi) <= bsize(bj)) block_step((int64_t)bi * bw, bsize(bi), (int64_t)bj * bw, bsize(bj));
          else block_step((int64_t)bj * bw, bsize(bj), (int64_t)bi * bw, bsize(bi));
        }
      const int done = rotated == 0;
      __syncthreads();
      if (done) break;
      continue;
    }
    for (int r = 0; r < k2 - 1; ++r) {
      // A group of G lanes works on one pair, 32/G pairs per warp at once:
      // the dot products, the G-lane reductions and the rotation chain of
      // those pairs overlap instead of running one after another.
      for (int base = warp * gpw; base < k2 / 2; base += nwarps * gpw) {
        const int i = base + sub;
        int p = 0, q = 0;
        bool live = i < k2 / 2;
        if (live) {
          tournament_pair(r, i, k2, p, q);
          live = q < k;  // q == k is the bye of an odd column count
        }
        double* wp = W + (int64_t)p * rows;
        double* wq = W + (int64_t)q * rows;
        double al = 0.0, be = 0.0, ga = 0.0;
        if (live && vec2) {
          // two rows per lane and step: 16-byte shared-memory accesses, 32-bit indices
          const double2* wp2 = reinterpret_cast<const double2*>(wp);
          const double2* wq2 = reinterpret_cast<const double2*>(wq);
          for (int x = gl; x < rows2; x += G) {
            const double2 u = wp2[x], v = wq2[x];
            al = fma(u.x, u.x, al);
            be = fma(v.x, v.x, be);
            ga = fma(u.x, v.x, ga);
            al = fma(u.y, u.y, al);
            be = fma(v.y, v.y, be);
            ga = fma(u.y, v.y, ga);
          }
        } else if (live)
          for (int64_t x = gl; x < rows; x += G) {
            const double u = wp[x], v = wq[x];
            al = fma(u, u, al);
            be = fma(v, v, be);
            ga = fma(u, v, ga);
          }
        for (int o = G >> 1; o > 0; o >>= 1) {  // every lane takes part in the shuffles
          al += __shfl_xor_sync(0xffffffffu, al, o);
          be += __shfl_xor_sync(0xffffffffu, be, o);
          ga += __shfl_xor_sync(0xffffffffu, ga, o);
        }
        if (live && ga * ga > tol2 * (al * be) && fmin(al, be) > noise2 && fabs(ga) > abs_floor &&
            fabs(ga) > DBL_MIN) {
          // t = sign(zeta) / (|zeta| + sqrt(1 + zeta^2)), zeta = (be - al) / (2 ga), with
          // numerator and denominator scaled by |2 ga|: one division, one root.
          const double d = be - al, g2 = 2.0 * ga;
          const double t = (d > 0.0 ? g2 : d < 0.0 ? -g2 : fabs(g2)) / (fabs(d) + sqrt(fma(d, d, g2 * g2)));
          const double cs = rsqrt(1.0 + t * t);
          const double sn = cs * t;
          double* vp = V + (int64_t)p * k;
          double* vq = V + (int64_t)q * k;
          if (vec2) {
            double2* wp2 = reinterpret_cast<double2*>(wp);
            double2* wq2 = reinterpret_cast<double2*>(wq);
            for (int x = gl; x < rows2; x += G) {
              const double2 u = wp2[x], v = wq2[x];
              wp2[x] = make_double2(cs * u.x - sn * v.x, cs * u.y - sn * v.y);
              wq2[x] = make_double2(sn * u.x + cs * v.x, sn * u.y + cs * v.y);
            }
            double2* vp2 = reinterpret_cast<double2*>(vp);
            double2* vq2 = reinterpret_cast<double2*>(vq);
            for (int x = gl; x < k2v; x += G) {
              const double2 u = vp2[x], v = vq2[x];
              vp2[x] = make_double2(cs * u.x - sn * v.x, cs * u.y - sn * v.y);
              vq2[x] = make_double2(sn * u.x + cs * v.x, sn * u.y + cs * v.y);
            }
          } else {
            for (int64_t x = gl; x < rows; x += G) {
              const double u = wp[x], v = wq[x];
              wp[x] = cs * u - sn * v;
              wq[x] = sn * u + cs * v;
            }
            for (int64_t x = gl; x < k; x += G) {
              const double u = vp[x], v = vq[x];
              vp[x] = cs * u - sn * v;
              vq[x] = sn * u + cs * v;
            }
          }
          if (gl == 0) rotated = 1;
        }
      }
      __syncthreads();
    }
    const int done = rotated == 0;
    __syncthreads();
    if (done) break;
  }
  if (tid == 0) {
    if (sweep == kMaxSweeps) atomicExch(status, 1);
    atomicMax(status + 1, sweep);  // sweeps of the slowest sector (diagnostic)
  }

  for (int c = warp; c < k; c += nwarps) {
    const double* wc = W + (int64_t)c * rows;
    double acc = 0.0;
    for (int64_t x = lane; x < rows; x += 32) acc = fma(wc[x], wc[x], acc);
    acc = warp_sum(acc);
    if (lane == 0) sv[c] = sqrt(acc);
  }
  __syncthreads();
  for (int c = tid; c < k; c += blockDim.x) {
    const double sc = sv[c];
    int64_t pos = 0;
    for (int64_t o = 0; o < k; ++o) {
      const double so = sv[o];
      pos += (so > sc || (so == sc && o < c)) ? 1 : 0;
    }
    rk[c] = (double)pos;
  }
  __syncthreads();

  double* s = S + J.s_off;
  double* u = U + J.u_off;
  double* vh = VH + J.v_off;
  for (int c = warp; c < k; c += nwarps) {
    const int64_t pos = (int64_t)rk[c];
    const double sc = sv[c];
    const double* wc = W + (int64_t)c * rows;
    const double* vc = V + (int64_t)c * k;
    const double inv = sc > 0.0 ? 1.0 / sc : 0.0;
    // Gauge (factorize.rs:3836-3852, 3945-3962): the largest-|.| entry of the
    // left singular vector is made positive; the first maximum wins.
    const double* lv = wide ? vc : wc;
    const int64_t llen = wide ? k : rows;
    double best = -1.0;
    int64_t bidx = 0;
    for (int64_t x = lane; x < llen; x += 32) {
      const double v = fabs(lv[x]);
      if (v > best) {
        best = v;
        bidx = x;
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, off);
      const int64_t oi = __shfl_xor_sync(0xffffffffu, bidx, off);
      if (ob > best || (ob == best && oi < bidx)) {
        best = ob;
        bidx = oi;
      }
    }
    const double sign = lv[bidx] < 0.0 ? -1.0 : 1.0;
    if (!wide) {
      for (int64_t x = lane; x < m; x += 32) u[x + pos * m] = sign * wc[x] * inv;
      for (int64_t x = lane; x < n; x += 32) vh[pos + x * k] = sign * vc[x];
    } else {
      for (int64_t x = lane; x < m; x += 32) u[x + pos * m] = sign * vc[x];
      for (int64_t x = lane; x < n; x += 32) vh[pos + x * k] = sign * wc[x] * inv;
    }
    if (lane == 0) s[pos] = sc;
  }
}

// ---------------------------------------------------------------------------
// Large sectors: one thread-block cluster per sector
// ---------------------------------------------------------------------------
//
// A sector with at least kSvdCluster column blocks runs the blocked Jacobi on
// a cluster of CL CTAs (one per SM, scheduled together; CL = 16 for sectors
// with at least 16 blocks where the device can co-schedule such clusters,
// else 8): each sweep
// runs the within-block steps of all blocks, then a round-robin tournament
// of block pairs, the pairs of a round (disjoint columns) spread over the
// CTAs, with a cluster barrier (barrier.cluster, release / acquire) between
// rounds so every CTA sees the columns the others wrote.  Columns are read at
// L2 (ld.global.cg), never from a stale L1.  Every CTA executes the same
// sequence of barriers: the loop bounds and the convergence decision (one
// flag in the sector's scratch, read after a barrier) are identical for all.
// One sweep visits every column pair once, as in the single-CTA kernel.

constexpr int kSvdCluster = 8;       // portable cluster size: sectors with >= 8 column blocks
constexpr int kSvdClusterWide = 16;  // non-portable, where the device can co-schedule it: >= 16 blocks

__device__ __forceinline__ void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

template <int CL>
__global__ void __launch_bounds__(kSvdThreads) svd_cluster_kernel(const SvdJob* __restrict__ jobs,
                                                                  const double* __restrict__ A,
                                                                  double* __restrict__ U, double* __restrict__ S,
                                                                  double* __restrict__ VH, double* __restrict__ work,
                                                                  const int64_t* __restrict__ work_off,
                                                                  int32_t* __restrict__ status) {
  const int64_t job = blockIdx.x / CL;
  const int rank = (int)(blockIdx.x % CL);  // 1-D clusters: the CTA's rank in its cluster
  const SvdJob J = jobs[job];
  const int64_t m = J.m, n = J.n, k = J.k;  // k >= CL blocks, so k > 1
  const bool wide = m < n;
  const int64_t rows = wide ? n : m;
  double* W = work + work_off[job];
  double* V = W + rows * k;
  double* sv = V + k * k;
  int* flag = reinterpret_cast<int*>(sv + k);  // the rank slots are free in this kernel
  extern __shared__ __align__(16) double smem_panel[];
  __shared__ int rotated, s_any;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const double* a = A + J.a_off;

  // W = A (or A^T), V = I, squared column norms into sv: columns split over the cluster.
  for (int64_t c = (int64_t)rank * nwarps + warp; c < k; c += (int64_t)CL * nwarps) {
    double f = 0.0;
    for (int64_t x = lane; x < rows; x += 32) {
      const double v = wide ? a[c + x * m] : a[x + c * m];
      W[c * rows + x] = v;
      f = fma(v, v, f);
    }
    for (int64_t x = lane; x < k; x += 32) V[c * k + x] = x == c ? 1.0 : 0.0;
    f = warp_sum(f);
    if (lane == 0) sv[c] = f;
  }
  cluster_barrier();
  double frob2 = 0.0;  // the same sum, in the same order, in every CTA
  for (int64_t o = 0; o < k; ++o) frob2 += __ldcg(sv + o);
  const double abs_floor = 1e-28 * frob2;
  const double tol = 4.0 * sqrt((double)rows) * DBL_EPSILON;
  const double noise2 = ((double)rows * DBL_EPSILON) * ((double)rows * DBL_EPSILON) * frob2;
  const int G = rows <= 64 ? 4 : rows <= 128 ? 8 : rows <= 256 ? 16 : 32;
  const int bw = svd_block_width(rows, k);
  const int nb = (int)((k + bw - 1) / bw);
  const int nb2 = (nb + 1) & ~1;
  auto bsize = [&](int b) { return (int)((b + 1) * (int64_t)bw <= k ? bw : k - (int64_t)b * bw); };

  int sweep = 0;
  for (; sweep < kMaxSweeps; ++sweep) {
    if (rank == 0 && tid == 0) atomicExch(flag, 0);
    if (tid == 0) rotated = 0;
    cluster_barrier();
    for (int b = rank; b < nb; b += CL)
      jacobi_block_step<true>(W, V, smem_panel, rows, k, (int64_t)b * bw, bsize(b), 0, 0, G, tol, noise2, abs_floor,
                              &rotated);
    cluster_barrier();
    for (int r = 0; r < nb2 - 1; ++r) {
      for (int i = rank; i < nb2 / 2; i += CL) {
        int bi, bj;
        tournament_pair(r, i, nb2, bi, bj);
        if (bj >= nb) continue;  // the bye of an odd block count
        if (bsize(bi) <= bsize(bj))
          jacobi_block_step<true>(W, V, smem_panel, rows, k, (int64_t)bi * bw, bsize(bi), (int64_t)bj * bw,
                                  bsize(bj), G, tol, noise2, abs_floor, &rotated);
        else
          jacobi_block_step<true>(W, V, smem_panel, rows, k, (int64_t)bj * bw, bsize(bj), (int64_t)bi * bw,
                                  bsize(bi), G, tol, noise2, abs_floor, &rotated);
      }
      cluster_barrier();
    }
    __syncthreads();
    if (tid == 0 && rotated) atomicOr(flag, 1);
    cluster_barrier();
    if (tid == 0) s_any = atomicOr(flag, 0);
    __syncthreads();
    const int any = s_any;
    cluster_barrier();  // every CTA has read the flag before rank 0 clears it
    if (!any) break;
  }
  if (rank == 0 && tid == 0) {
    if (sweep == kMaxSweeps) atomicExch(status, 1);
    atomicMax(status + 1, sweep);
  }

  // Singular values, order, gauge and outputs: columns split over the cluster.
  for (int64_t c = (int64_t)rank * nwarps + warp; c < k; c += (int64_t)CL * nwarps) {
    const double* wc = W + c * rows;
    double acc = 0.0;
    for (int64_t x = lane; x < rows; x += 32) {
      const double v = __ldcg(wc + x);
      acc = fma(v, v, acc);
    }
    acc = warp_sum(acc);
    if (lane == 0) sv[c] = sqrt(acc);
  }
  cluster_barrier();
  double* s_out = S + J.s_off;
  double* u = U + J.u_off;
  double* vh = VH + J.v_off;
  for (int64_t c = (int64_t)rank * nwarps + warp; c < k; c += (int64_t)CL * nwarps) {
    const double sc = __ldcg(sv + c);
    int64_t cnt = 0;
    for (int64_t o = lane; o < k; o += 32) {
      const double so = __ldcg(sv + o);
      cnt += (so > sc || (so == sc && o < c)) ? 1 : 0;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
    const int64_t pos = cnt;
    const double* wc = W + c * rows;
    const double* vc = V + c * k;
    const double inv = sc > 0.0 ? 1.0 / sc : 0.0;
    const double* lv = wide ? vc : wc;  // gauge: largest-|.| entry of the left vector positive, first maximum
    const int64_t llen = wide ? k : rows;
    double best = -1.0;
    int64_t bidx = 0;
    for (int64_t x = lane; x < llen; x += 32) {
      const double v = fabs(__ldcg(lv + x));
      if (v > best) {
        best = v;
        bidx = x;
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, off);
      const int64_t oi = __shfl_xor_sync(0xffffffffu, bidx, off);
      if (ob > best || (ob == best && oi < bidx)) {
        best = ob;
        bidx = oi;
      }
    }
    const double sign = __ldcg(lv + bidx) < 0.0 ? -1.0 : 1.0;
    if (!wide) {
      for (int64_t x = lane; x < m; x += 32) u[x + pos * m] = sign * __ldcg(wc + x) * inv;
      for (int64_t x = lane; x < n; x += 32) vh[pos + x * k] = sign * __ldcg(vc + x);
    } else {
      for (int64_t x = lane; x < m; x += 32) u[x + pos * m] = sign * __ldcg(vc + x);
      for (int64_t x = lane; x < n; x += 32) vh[pos + x * k] = sign * __ldcg(wc + x) * inv;
    }
    if (lane == 0) s_out[pos] = sc;
  }
}

// ---------------------------------------------------------------------------
// Truncation selection (one CTA)
// ---------------------------------------------------------------------------

// Number of entries of the descending array x[0..len) that are > v.
__device__ __forceinline__ int64_t count_greater(const double* x, int64_t len, double v) {
  int64_t lo = 0, hi = len;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (x[mid] > v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}
// Number of entries >= v.
__device__ __forceinline__ int64_t count_geq(const double* x, int64_t len, double v) {
  int64_t lo = 0, hi = len;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (x[mid] >= v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__device__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0) red[32] = t;
  }
  __syncthreads();
  return red[32];
}

// One CTA per segment of sectors (one tensor's spectra); seg_first == nullptr
// means a single segment over all njobs sectors.
__global__ void __launch_bounds__(1024) truncate_kernel(const SvdJob* __restrict__ all_jobs, int32_t all_njobs,
                                                        const int64_t* __restrict__ seg_first,
                                                        const double* __restrict__ S, int32_t policy, double p0,
                                                        double p1, const int64_t* __restrict__ all_ranks,
                                                        int64_t* __restrict__ all_kept, double* __restrict__ all_err) {
  __shared__ double red[33];
  const int64_t j0 = seg_first ? seg_first[blockIdx.x] : 0;
  const int64_t j1 = seg_first ? seg_first[blockIdx.x + 1] : all_njobs;
  const SvdJob* jobs = all_jobs + j0;
  const int32_t njobs = (int32_t)(j1 - j0);
  const int64_t* space_ranks = all_ranks ? all_ranks + j0 : nullptr;
  int64_t* kept = all_kept + j0;
  double* err = all_err + blockIdx.x;
  // Weighted norm of the full spectrum (for tolerance policies).
  double part = 0.0;
  for (int c = 0; c < njobs; ++c) {
    const double* s = S + jobs[c].s_off;
    double acc = 0.0;
    for (int64_t i = threadIdx.x; i < jobs[c].k; i += blockDim.x) acc = fma(s[i], s[i], acc);
    part = fma(jobs[c].weight, acc, part);
  }
  const double full2 = block_sum(part, red);

  for (int c = threadIdx.x; c < njobs; c += blockDim.x) kept[c] = 0;
  __syncthreads();

  if (policy == 0) {  // Full
    for (int c = threadIdx.x; c < njobs; c += blockDim.x) kept[c] = jobs[c].k;
  } else if (policy == 1) {  // Rank: greedy prefix of the descending candidate order
    const double budget = p0;
    for (int c = 0; c < njobs; ++c) {
      const double* sc = S + jobs[c].s_off;
      for (int64_t i = threadIdx.x; i < jobs[c].k; i += blockDim.x) {
        const double v = sc[i];
        double before = 0.0;  // weight of every candidate ahead of (c, i)
        for (int o = 0; o < njobs; ++o) {
          const double* so = S + jobs[o].s_off;
          int64_t cnt;
          if (o == c) cnt = i;
          else if (o < c) cnt = count_geq(so, jobs[o].k, v);
          else cnt = count_greater(so, jobs[o].k, v);
          before = fma((double)cnt, jobs[o].weight, before);
        }
        if (before + jobs[c].weight <= budget + 1e-12) atomicAdd((unsigned long long*)&kept[c], 1ull);
      }
    }
  } else if (policy == 2) {  // Tolerance: values >= max(atol, rtol * norm)
    const double thr = fmax(p0, p1 * sqrt(full2));
    for (int c = threadIdx.x; c < njobs; c += blockDim.x) kept[c] = count_geq(S + jobs[c].s_off, jobs[c].k, thr);
  } else if (policy == 3) {  // DiscardWeight: drop the smallest tails while the weighted sum fits
    const double budget = (p0 * sqrt(full2)) * (p0 * sqrt(full2));
    for (int c = 0; c < njobs; ++c) {
      const double* sc = S + jobs[c].s_off;
      for (int64_t i = threadIdx.x; i < jobs[c].k; i += blockDim.x) {
        const double v = sc[i];
        // candidates discarded before (c, i): smaller values, equal values of
        // lower sectors, and the deeper tail of its own sector.
        double before = 0.0;
        for (int o = 0; o < njobs; ++o) {
          const double* so = S + jobs[o].s_off;
          const int64_t len = jobs[o].k;
          if (o == c) {
            for (int64_t x = i + 1; x < len; ++x) before = fma(jobs[o].weight * so[x], so[x], before);
            continue;
          }
          const int64_t from = o < c ? count_greater(so, len, v) : count_geq(so, len, v);
          for (int64_t x = from; x < len; ++x) before = fma(jobs[o].weight * so[x], so[x], before);
        }
        const double mine = jobs[c].weight * v * v;
        if (!(before + mine <= budget + 1e-15)) atomicAdd((unsigned long long*)&kept[c], 1ull);
      }
    }
  } else {  // Space: per-sector prefix, clamped
    for (int c = threadIdx.x; c < njobs; c += blockDim.x) {
      int64_t r = space_ranks[c];
      kept[c] = r < jobs[c].k ? r : jobs[c].k;
    }
  }
  __syncthreads();
  // Discarded weighted norm.
  double d = 0.0;
  for (int c = 0; c < njobs; ++c) {
    const double* s = S + jobs[c].s_off;
    double acc = 0.0;
    for (int64_t i = kept[c] + threadIdx.x; i < jobs[c].k; i += blockDim.x) acc = fma(s[i], s[i], acc);
    d = fma(jobs[c].weight, acc, d);
  }
  const double tot = block_sum(d, red);
  if (threadIdx.x == 0) *err = sqrt(tot);
}

}  // namespace

cudaError_t launch_svd(const SvdJob* jobs, int32_t njobs, const double* a, double* u, double* s, double* vh,
                       double* work, const int64_t* work_off, int32_t* status, cudaStream_t stream) {
  if (njobs == 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(svd_jacobi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kSvdSmemBytes);
  if (e != cudaSuccess) return e;
  svd_jacobi_kernel<<<njobs, kSvdThreads, kSvdSmemBytes, stream>>>(jobs, a, u, s, vh, work, work_off, status);
  return cudaGetLastError();
}

int svd_cluster_size() { return kSvdCluster; }

namespace {

template <int CL>
cudaError_t launch_svd_clusters(const SvdJob* jobs, int32_t njobs, const double* a, double* u, double* s, double* vh,
                                double* work, const int64_t* work_off, int32_t* status, cudaStream_t stream) {
  cudaError_t e = cudaFuncSetAttribute(svd_cluster_kernel<CL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kSvdSmemBytes);
  if (e != cudaSuccess) return e;
  if (CL > 8) {
    e = cudaFuncSetAttribute(svd_cluster_kernel<CL>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(njobs * CL));
  cfg.blockDim = dim3(kSvdThreads);
  cfg.dynamicSmemBytes = kSvdSmemBytes;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, svd_cluster_kernel<CL>, jobs, a, u, s, vh, work, work_off, status);
}

}  // namespace

int svd_wide_cluster_size() {
  // 16-CTA clusters are non-portable: used only where the current device
  // reports room for at least one (one 1024-thread, 200 KB CTA per SM).
  static std::mutex mu;
  static std::map<int, int> known;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  std::lock_guard<std::mutex> g(mu);
  auto it = known.find(dev);
  if (it != known.end()) return it->second;
  int size = 0;
  if (cudaFuncSetAttribute(svd_cluster_kernel<kSvdClusterWide>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
          cudaSuccess &&
      cudaFuncSetAttribute(svd_cluster_kernel<kSvdClusterWide>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kSvdSmemBytes) == cudaSuccess) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kSvdClusterWide);
    cfg.blockDim = dim3(kSvdThreads);
    cfg.dynamicSmemBytes = kSvdSmemBytes;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kSvdClusterWide;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nc = 0;
    if (cudaOccupancyMaxActiveClusters(&nc, svd_cluster_kernel<kSvdClusterWide>, &cfg) == cudaSuccess && nc >= 1)
      size = kSvdClusterWide;
  }
  cudaGetLastError();  // a refused query leaves no sticky error behind
  known.emplace(dev, size);
  return size;
}

cudaError_t launch_svd_split(const SvdJob* jobs, int32_t n_cluster, int32_t njobs, const double* a, double* u,
                             double* s, double* vh, double* work, const int64_t* work_off, int32_t* status,
                             cudaStream_t stream, int32_t n_wide) {
  if (n_wide > 0) {
    cudaError_t e = launch_svd_clusters<kSvdClusterWide>(jobs, n_wide, a, u, s, vh, work, work_off, status, stream);
    if (e != cudaSuccess) return e;
  }
  if (n_cluster > n_wide) {
    cudaError_t e = launch_svd_clusters<kSvdCluster>(jobs + n_wide, n_cluster - n_wide, a, u, s, vh, work,
                                                     work_off + n_wide, status, stream);
    if (e != cudaSuccess) return e;
  }
  if (njobs > n_cluster)
    return launch_svd(jobs + n_cluster, njobs - n_cluster, a, u, s, vh, work, work_off + n_cluster, status, stream);
  return cudaGetLastError();
}

cudaError_t launch_truncate(const SvdJob* jobs, int32_t njobs, const double* s, int32_t policy, double p0, double p1,
                            const int64_t* space_ranks, int64_t* kept, double* err, cudaStream_t stream) {
  truncate_kernel<<<1, 1024, 0, stream>>>(jobs, njobs, nullptr, s, policy, p0, p1, space_ranks, kept, err);
  return cudaGetLastError();
}

cudaError_t launch_truncate_segments(const SvdJob* jobs, int32_t nseg, const int64_t* seg_first, const double* s,
                                     int32_t policy, double p0, double p1, const int64_t* space_ranks, int64_t* kept,
                                     double* err, cudaStream_t stream) {
  if (nseg == 0) return cudaSuccess;
  truncate_kernel<<<nseg, 1024, 0, stream>>>(jobs, 0, seg_first, s, policy, p0, p1, space_ranks, kept, err);
  return cudaGetLastError();
}

}  // namespace tnt
