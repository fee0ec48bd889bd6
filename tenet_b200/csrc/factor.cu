// Batched per-sector QR and Hermitian eigendecomposition on the device.
//
// Replace the serial sector loops of qr_compact (tenet-matrixalgebra/src/
// factorize.rs:5158, positive_diagonal_gauge :3789-3830) and eigh_full_dyn
// (factorize.rs:3041-3150: eigenvalues stable-sorted by descending |lambda|,
// eigenvector_gauge :3902-3913 makes each vector's largest-|.| entry
// positive), which call a dense factorisation per coupled sector.
//
// Both kernels run one CTA per coupled-sector matrix and share the SVD's
// per-sector scratch layout (rows*k + k*k + 2k doubles), keeping the working
// panel in shared memory when it fits.
//
// QR: Householder reflections H_j = I - tau_j v_j v_j^T (v_j(j) = 1) reduce
// the m x n panel to R in place, one warp per trailing column; Q (m x k,
// k = min(m, n)) is accumulated backwards from the identity.  Panels in
// global memory apply the reflectors 32 at a time in compact WY form.  The gauge
// negates column j of Q and row j of R when R_jj < 0 (zero keeps sign +1), so
// Q R is unchanged and the factorisation of a full-rank block is unique.
//
// eigh: cyclic two-sided Jacobi with a round-robin tournament of disjoint
// (p, q) pairs: per round every pair's rotation is computed from the current
// 2x2 principal block, then all column rotations A <- A J, V <- V J and all
// row rotations A <- J^T A are applied in parallel (one warp per pair).  A
// pair is skipped once |a_pq| is below 4 sqrt(n) eps sqrt(|a_pp a_qq|) or the
// rounding level eps ||A||_F.  Plans with a sector too large for shared
// memory run the whole eigendecomposition through the batched SVD instead
// (eigh_shift_kernel, eigh_from_svd_kernel below).
#include <cfloat>

#include "kernels.cuh"

namespace tnt {

namespace {

constexpr int kFacThreads = 512;
constexpr size_t kFacSmemBytes = 200 * 1024;
constexpr int kEighSweeps = 40;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0) red[32] = t;
  }
  __syncthreads();
  return red[32];
}

__device__ __forceinline__ void tournament_pair(int r, int i, int k2, int& p, int& q) {
  int a, b;
  if (i == 0) {
    a = k2 - 1;
    b = r;
  } else {
    a = (r + i) % (k2 - 1);
    b = (r - i + (k2 - 1)) % (k2 - 1);
  }
  p = a < b ? a : b;
  q = a < b ? b : a;
}

// Index of the first largest-|.| entry of x[0..len) across one warp.
__device__ __forceinline__ int64_t warp_argmax_abs(const double* x, int64_t len, int lane) {
  double best = -1.0;
  int64_t bidx = 0;
  for (int64_t i = lane; i < len; i += 32) {
    const double v = fabs(x[i]);
    if (v > best) {
      best = v;
      bidx = i;
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
  return bidx;
}

// ---------------------------------------------------------------------------
// QR
// ---------------------------------------------------------------------------

// Blocked QR for panels beyond shared memory with up to kQrBlockedMaxRows
// rows: the reflectors of 32 columns at a time are factored unblocked, kept
// in shared memory as V (unit diagonal, zeros above) with the upper
// triangular T of the compact WY form H_p ... H_{p+31} = I - V T V^T, and
// applied to every trailing column at once: a <- a - V T^T (V^T a), so each
// trailing column is read and written once per panel instead of once per
// reflector.  Q is accumulated backwards the same way with T.  Every T is
// kept in the sector's scratch (panel p at p * 32, leading dimension its
// width) for the Q pass.
constexpr int kQrBw = 32;
constexpr int64_t kQrBlockedMaxRows = 704;  // V (rows x 32) + T, Gram, per-warp vectors within 200 KB

// v[0..31] summed over the warp's lanes; lane L returns the sum of v[L].
__device__ __forceinline__ double warp_reduce_scatter32(double (&v)[kQrBw], int lane) {
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) {
    const bool upper = (lane & s) != 0;
#pragma unroll
    for (int i = 0; i < s; ++i) {
      const double send = upper ? v[i] : v[i + s];
      const double keep = upper ? v[i + s] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, s);
    }
  }
  return v[0];
}

// Panel p's reflectors into Vs (m x 32, column-major; columns beyond pw zero).
__device__ void qr_load_panel(const double* W, int64_t m, int64_t p, int pw, double* Vs) {
  for (int64_t idx = threadIdx.x; idx < (int64_t)kQrBw * m; idx += blockDim.x) {
    const int jj = (int)(idx / m);
    const int64_t i = idx - (int64_t)jj * m, j = p + jj;
    Vs[idx] = jj < pw ? (i > j ? W[i + j * m] : (i == j ? 1.0 : 0.0)) : 0.0;
  }
}

// Columns [c0, c1) of X (leading dimension m): x <- x - V M (V^T x) over rows
// p..m-1, with M = T^T (trans) or T; one warp per column, ws = 32 doubles of
// this warp's shared memory.
__device__ void qr_apply_block(double* X, int64_t m, int64_t p, int64_t c0, int64_t c1, const double* Vs,
                               const double* Ts, bool trans, double* ws) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int64_t c = c0 + warp; c < c1; c += nwarps) {
    double* xc = X + c * m;
    double w[kQrBw];
#pragma unroll
    for (int jj = 0; jj < kQrBw; ++jj) w[jj] = 0.0;
    for (int64_t i = p + lane; i < m; i += 32) {
      const double a = xc[i];
#pragma unroll
      for (int jj = 0; jj < kQrBw; ++jj) w[jj] = fma(Vs[jj * m + i], a, w[jj]);
    }
    ws[lane] = warp_reduce_scatter32(w, lane);
    __syncwarp();
    // (M w)[lane]: T^T w sums rows l <= lane of column lane; T w sums columns l >= lane of row lane.
    double mw = 0.0;
    if (trans) {
      for (int l = 0; l <= lane; ++l) mw = fma(Ts[l + lane * kQrBw], ws[l], mw);
    } else {
      for (int l = lane; l < kQrBw; ++l) mw = fma(Ts[lane + l * kQrBw], ws[l], mw);
    }
    __syncwarp();
    ws[lane] = mw;
    __syncwarp();
    for (int64_t i = p + lane; i < m; i += 32) {
      double s = 0.0;
#pragma unroll
      for (int jj = 0; jj < kQrBw; ++jj) s = fma(Vs[jj * m + i], ws[jj], s);
      xc[i] -= s;
    }
    __syncwarp();
  }
}

__global__ void __launch_bounds__(kFacThreads) qr_kernel(const SvdJob* __restrict__ jobs, const double* __restrict__ A,
                                                         double* __restrict__ Q, double* __restrict__ R,
                                                         double* __restrict__ work,
                                                         const int64_t* __restrict__ work_off) {
  const SvdJob J = jobs[blockIdx.x];
  const int64_t m = J.m, n = J.n, k = J.k;
  if (k == 0) return;
  extern __shared__ double smem_fac[];
  const bool on_chip = (size_t)(m * n + k) * sizeof(double) <= kFacSmemBytes;
  double* W = on_chip ? smem_fac : work + work_off[blockIdx.x];  // m x n panel, column-major
  double* tau = W + m * n;
  __shared__ double red[33];
  __shared__ double s_beta, s_inv;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const double* a = A + J.a_off;
  for (int64_t i = tid; i < m * n; i += blockDim.x) W[i] = a[i];
  __syncthreads();

  // Blocked (panels of 32 reflectors, compact WY) when the panel lives in
  // global memory and V fits in shared memory; otherwise one reflector at a time.
  const bool blocked = !on_chip && m <= kQrBlockedMaxRows;
  double* Vs = smem_fac;                  // blocked: m x 32 reflectors of the panel
  double* Ts = Vs + m * kQrBw;            // 32 x 32 T of the panel
  double* Zs = Ts + kQrBw * kQrBw;        // 32 x 32 Gram matrix V^T V
  double* wvs = Zs + kQrBw * kQrBw;       // 32 doubles per warp
  double* Tall = tau + k;                 // every panel's T, for the Q pass
  const int64_t step = blocked ? kQrBw : k;
  for (int64_t p = 0; p < k; p += step) {
  const int64_t pend = p + step < k ? p + step : k;  // this panel's reflectors [p, pend)
  const int64_t cend = blocked ? pend : n;           // columns H_j is applied to one at a time
  for (int64_t j = p; j < pend; ++j) {
    double* col = W + j * m;
    double ss = 0.0;
    for (int64_t i = j + 1 + tid; i < m; i += blockDim.x) ss = fma(col[i], col[i], ss);
    const double sigma = block_sum(ss, red);  // squared norm below the diagonal
    if (tid == 0) {
      const double alpha = col[j];
      double t = 0.0, beta = alpha;
      if (sigma > 0.0) {
        const double nrm = sqrt(alpha * alpha + sigma);
        beta = alpha >= 0.0 ? -nrm : nrm;
        t = (beta - alpha) / beta;
      }
      tau[j] = t;
      s_beta = beta;
      // scale factor for v below the diagonal: 1 / (alpha - beta)
      s_inv = (t != 0.0) ? 1.0 / (alpha - beta) : 0.0;
    }
    __syncthreads();
    const double inv = s_inv;
    const double t = tau[j];
    for (int64_t i = j + 1 + tid; i < m; i += blockDim.x) col[i] *= inv;
    __syncthreads();
    if (tid == 0) col[j] = s_beta;
    // Apply H_j to trailing columns (of the panel, when blocked): one warp per column.
    if (t != 0.0) {
      for (int64_t c = j + 1 + warp; c < cend; c += nwarps) {
        double* wc = W + c * m;
        double d = lane == 0 ? wc[j] : 0.0;
        for (int64_t i = j + 1 + lane; i < m; i += 32) d = fma(col[i], wc[i], d);
        d = warp_sum(d) * t;
        if (lane == 0) wc[j] -= d;
        for (int64_t i = j + 1 + lane; i < m; i += 32) wc[i] = fma(-d, col[i], wc[i]);
      }
    }
    __syncthreads();
  }
  if (blocked) {
    // T of the panel: T_jj = tau_j, T[0:jj, jj] = -tau_jj T[0:jj, 0:jj] (V^T v_jj)[0:jj].
    const int pw = (int)(pend - p);
    qr_load_panel(W, m, p, pw, Vs);
    for (int i = tid; i < 2 * kQrBw * kQrBw; i += blockDim.x) Ts[i] = 0.0;  // Ts and Zs
    __syncthreads();
    for (int e = warp; e < pw * pw; e += nwarps) {
      const int l = e % pw, jj = e / pw;
      if (l >= jj) continue;
      double d = 0.0;
      for (int64_t i = p + jj + lane; i < m; i += 32) d = fma(Vs[l * m + i], Vs[jj * m + i], d);
      d = warp_sum(d);
      if (lane == 0) Zs[l + jj * kQrBw] = d;
    }
    __syncthreads();
    for (int jj = 0; jj < pw; ++jj) {
      const double t = tau[p + jj];
      if (tid < jj) {
        double acc = 0.0;
        for (int l2 = tid; l2 < jj; ++l2) acc = fma(Ts[tid + l2 * kQrBw], Zs[l2 + jj * kQrBw], acc);
        Ts[tid + jj * kQrBw] = -t * acc;
      } else if (tid == jj) {
        Ts[jj + jj * kQrBw] = t;
      }
      __syncthreads();
    }
    for (int i = tid; i < pw * pw; i += blockDim.x) Tall[p * kQrBw + i] = Ts[(i % pw) + (i / pw) * kQrBw];
    // Trailing columns: a <- (H_p ... H_{pend-1})^T a = a - V T^T V^T a.
    qr_apply_block(W, m, p, pend, n, Vs, Ts, true, wvs + warp * kQrBw);
    __syncthreads();
  }
  }

  // Q = H_0 ... H_{k-1} [I; 0], accumulated backwards in the output.
  double* q = Q + J.u_off;
  for (int64_t i = tid; i < m * k; i += blockDim.x) q[i] = (i % m == i / m) ? 1.0 : 0.0;
  __syncthreads();
  if (blocked) {
    for (int64_t p = ((k - 1) / kQrBw) * kQrBw; p >= 0; p -= kQrBw) {
      const int pw = (int)(p + kQrBw < k ? kQrBw : k - p);
      qr_load_panel(W, m, p, pw, Vs);
      for (int i = tid; i < kQrBw * kQrBw; i += blockDim.x) {
        const int l = i % kQrBw, c = i / kQrBw;
        Ts[i] = (l < pw && c < pw) ? Tall[p * kQrBw + l + c * pw] : 0.0;
      }
      __syncthreads();
      // Columns c >= p: q <- (H_p ... H_{p+pw-1}) q = q - V T V^T q.
      qr_apply_block(q, m, p, p, k, Vs, Ts, false, wvs + warp * kQrBw);
      __syncthreads();
    }
  }
  for (int64_t j = blocked ? -1 : k - 1; j >= 0; --j) {
    const double t = tau[j];
    if (t != 0.0) {
      const double* v = W + j * m;
      for (int64_t c = j + warp; c < k; c += nwarps) {
        double* qc = q + c * m;
        double d = lane == 0 ? qc[j] : 0.0;
        for (int64_t i = j + 1 + lane; i < m; i += 32) d = fma(v[i], qc[i], d);
        d = warp_sum(d) * t;
        if (lane == 0) qc[j] -= d;
        for (int64_t i = j + 1 + lane; i < m; i += 32) qc[i] = fma(-d, v[i], qc[i]);
      }
    }
    __syncthreads();
  }

  // Positive-diagonal gauge and R (k x n, column-major).
  double* r = R + J.v_off;
  for (int64_t i = tid; i < k * n; i += blockDim.x) {
    const int64_t row = i % k, c = i / k;
    const double sgn = W[row + row * m] < 0.0 ? -1.0 : 1.0;
    r[i] = row <= c ? sgn * W[row + c * m] : 0.0;
  }
  for (int64_t i = tid; i < m * k; i += blockDim.x) {
    const int64_t c = i / m;
    if (W[c + c * m] < 0.0) q[i] = -q[i];
  }
}

// ---------------------------------------------------------------------------
// Hermitian (real symmetric) eigendecomposition
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(kFacThreads) eigh_kernel(const SvdJob* __restrict__ jobs,
                                                           const double* __restrict__ A, double* __restrict__ VEC,
                                                           double* __restrict__ VAL, double* __restrict__ MAG,
                                                           double* __restrict__ work,
                                                           const int64_t* __restrict__ work_off,
                                                           int32_t* __restrict__ status) {
  const SvdJob J = jobs[blockIdx.x];
  const int64_t n = J.m;
  if (n == 0) return;
  extern __shared__ double smem_fac[];
  const bool on_chip = (size_t)(2 * n * n + 2 * n) * sizeof(double) <= kFacSmemBytes;
  double* W = on_chip ? smem_fac : work + work_off[blockIdx.x];  // n x n, column-major
  double* V = W + n * n;
  double* lam = V + n * n;
  double* rk = lam + n;
  __shared__ double red[33];
  __shared__ int rotated;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  // Rotation (c, s) of every pair of the current round.
  __shared__ double rc[kFacThreads / 32 * 8], rs[kFacThreads / 32 * 8];
  __shared__ int rp[kFacThreads / 32 * 8], rq[kFacThreads / 32 * 8];
  const double* a = A + J.a_off;
  double f2 = 0.0, d2 = 0.0;
  int finite = 1;
  for (int64_t i = tid; i < n * n; i += blockDim.x) {
    const double v = a[i];
    const int64_t r = i % n, c = i / n;
    const double d = v - a[c + r * n];
    W[i] = v;
    V[i] = r == c ? 1.0 : 0.0;
    f2 = fma(v, v, f2);
    d2 = fma(d, d, d2);
    finite &= isfinite(v) ? 1 : 0;
  }
  const double frob = sqrt(block_sum(f2, red));
  const double asym = sqrt(block_sum(d2, red));
  const int all_finite = __syncthreads_and(finite);
  // Hermiticity check of the reference (normwise_hermitian, factorize.rs:5999-6021):
  // ||A - A^T||_F <= 2 * 64 eps ||A||_F, every entry finite.
  if (!all_finite || asym > 128.0 * DBL_EPSILON * frob) {
    if (tid == 0) atomicExch(status, 2);
    return;
  }
  // Off-diagonal entries at the rounding level eps ||A||_F are noise that
  // every rotation regenerates; rotating them again never settles.
  const double abs_floor = DBL_EPSILON * frob;
  const double tol = 4.0 * sqrt((double)n) * DBL_EPSILON;  // rounding level of a length-n rotation

  const int k2 = (int)((n + 1) & ~1LL);
  const int npairs = k2 / 2;
  int sweep = 0;
  for (; sweep < kEighSweeps && n > 1; ++sweep) {
    if (tid == 0) rotated = 0;
    __syncthreads();
    for (int r = 0; r < k2 - 1; ++r) {
      // Pairs are processed in batches of (warps * 8) so the rotation table stays in shared memory.
      for (int base = 0; base < npairs; base += nwarps * 8) {
        const int batch = min(npairs - base, nwarps * 8);
        for (int b = tid; b < batch; b += blockDim.x) {
          int p, q;
          tournament_pair(r, base + b, k2, p, q);
          double c = 1.0, s = 0.0;
          if (q < n) {
            const double apq = W[p + (int64_t)q * n];
            const double app = W[p + (int64_t)p * n], aqq = W[q + (int64_t)q * n];
            if (fabs(apq) > tol * sqrt(fabs(app * aqq)) && fabs(apq) > abs_floor && fabs(apq) > DBL_MIN) {
              const double zeta = (aqq - app) / (2.0 * apq);
              const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
              c = 1.0 / sqrt(1.0 + t * t);
              s = c * t;
              rotated = 1;
            }
          }
          rc[b] = c;
          rs[b] = s;
          rp[b] = p;
          rq[b] = q;
        }
        __syncthreads();
        // Columns: A <- A J, V <- V J.
        for (int b = warp; b < batch; b += nwarps) {
          const double c = rc[b], s = rs[b];
          if (s == 0.0) continue;
          int p, q;
          tournament_pair(r, base + b, k2, p, q);
          double* wp = W + (int64_t)p * n;
          double* wq = W + (int64_t)q * n;
          double* vp = V + (int64_t)p * n;
          double* vq = V + (int64_t)q * n;
          for (int64_t x = lane; x < n; x += 32) {
            const double u = wp[x], v = wq[x];
            wp[x] = c * u - s * v;
            wq[x] = s * u + c * v;
            const double g = vp[x], h = vq[x];
            vp[x] = c * g - s * h;
            vq[x] = s * g + c * h;
          }
        }
        __syncthreads();
        // Rows: A <- J^T A, one warp per column (lanes over the pairs), so a
        // warp's accesses stay inside one contiguous column instead of
        // striding by n down a row.  Every element is updated once per batch
        // with the same arithmetic as a row-by-row pass.
        for (int64_t x = warp; x < n; x += nwarps) {
          double* col = W + x * n;
          for (int b = lane; b < batch; b += 32) {
            const double c = rc[b], s = rs[b];
            if (s == 0.0) continue;
            const int p = rp[b], q = rq[b];
            const double u = col[p], v = col[q];
            col[p] = c * u - s * v;
            col[q] = s * u + c * v;
          }
        }
        __syncthreads();
      }
    }
    const int done = rotated == 0;
    __syncthreads();
    if (done) break;
  }
  if (tid == 0 && sweep == kEighSweeps) atomicExch(status, 1);

  for (int64_t i = tid; i < n; i += blockDim.x) lam[i] = W[i + i * n];
  __syncthreads();
  // Order: descending |lambda|; ties keep LAPACK's ascending-value order, then index.
  for (int64_t i = tid; i < n; i += blockDim.x) {
    const double li = lam[i], ai = fabs(li);
    int64_t pos = 0;
    for (int64_t o = 0; o < n; ++o) {
      const double lo = lam[o], ao = fabs(lo);
      pos += (ao > ai || (ao == ai && (lo < li || (lo == li && o < i)))) ? 1 : 0;
    }
    rk[i] = (double)pos;
  }
  __syncthreads();
  double* vec = VEC + J.u_off;
  double* val = VAL + J.s_off;
  for (int64_t c = warp; c < n; c += nwarps) {
    const int64_t pos = (int64_t)rk[c];
    const double* vc = V + c * n;
    const int64_t b = warp_argmax_abs(vc, n, lane);
    const double sgn = vc[b] < 0.0 ? -1.0 : 1.0;
    for (int64_t x = lane; x < n; x += 32) vec[x + pos * n] = sgn * vc[x];
    if (lane == 0) {
      val[pos] = lam[c];
      if (MAG) MAG[J.s_off + pos] = fabs(lam[c]);
    }
  }
}

// ---------------------------------------------------------------------------
// Eigendecomposition of large sectors through the batched SVD
// ---------------------------------------------------------------------------
//
// A sector too large for the on-chip two-sided Jacobi is shifted to
// B = A + c I with c = ||A||_F, at least the spectral radius, so B is
// positive semidefinite: its singular values are lambda + c and its right
// singular vectors are eigenvectors of A (for a repeated singular value they
// span the eigenspace).  The batched SVD, with thread-block clusters for the
// largest sectors, does the work; eigh_from_svd_kernel maps sigma back to
// lambda = sigma - c, orders by descending |lambda| (ties: ascending value,
// then index) and applies the largest-entry gauge, as eigh_kernel does.
// Eigenvalue error: about eps (||A||_2 + c) absolute, against eps ||A||_2 for
// the two-sided Jacobi.

__global__ void __launch_bounds__(kFacThreads) eigh_shift_kernel(const SvdJob* __restrict__ jobs,
                                                                 const double* __restrict__ A, double* __restrict__ B,
                                                                 double* __restrict__ shift, int32_t* __restrict__ bad) {
  const SvdJob J = jobs[blockIdx.x];
  const int64_t n = J.m;
  const int tid = threadIdx.x;
  if (n == 0) {
    if (tid == 0) shift[blockIdx.x] = 0.0;
    return;
  }
  __shared__ double red[33];
  const double* a = A + J.a_off;
  double* b = B + J.a_off;
  double f2 = 0.0, d2 = 0.0;
  int finite = 1;
  for (int64_t i = tid; i < n * n; i += blockDim.x) {
    const double v = a[i];
    const int64_t r = i % n, c = i / n;
    const double d = v - a[c + r * n];
    f2 = fma(v, v, f2);
    d2 = fma(d, d, d2);
    finite &= isfinite(v) ? 1 : 0;
  }
  const double frob = sqrt(block_sum(f2, red));
  const double asym = sqrt(block_sum(d2, red));
  const int all_finite = __syncthreads_and(finite);
  // The Hermiticity check of eigh_kernel (normwise_hermitian, factorize.rs:5999-6021).
  if ((!all_finite || asym > 128.0 * DBL_EPSILON * frob) && tid == 0) atomicExch(bad, 1);
  const double c = all_finite ? frob : 0.0;
  if (tid == 0) shift[blockIdx.x] = c;
  for (int64_t i = tid; i < n * n; i += blockDim.x) b[i] = a[i] + ((i % n) == (i / n) ? c : 0.0);
}

__global__ void __launch_bounds__(kFacThreads) eigh_from_svd_kernel(const SvdJob* __restrict__ jobs,
                                                                    const double* __restrict__ S,
                                                                    const double* __restrict__ VH,
                                                                    const double* __restrict__ shift,
                                                                    double* __restrict__ VEC, double* __restrict__ VAL,
                                                                    double* __restrict__ MAG) {
  const SvdJob J = jobs[blockIdx.x];
  const int64_t n = J.m, k = J.k;
  if (n == 0) return;
  extern __shared__ double smem_fac[];
  double* lam = smem_fac;
  double* rk = lam + n;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const double c = shift[blockIdx.x];
  for (int64_t i = tid; i < n; i += blockDim.x) lam[i] = S[J.s_off + i] - c;
  __syncthreads();
  for (int64_t i = tid; i < n; i += blockDim.x) {
    const double li = lam[i], ai = fabs(li);
    int64_t pos = 0;
    for (int64_t o = 0; o < n; ++o) {
      const double lo = lam[o], ao = fabs(lo);
      pos += (ao > ai || (ao == ai && (lo < li || (lo == li && o < i)))) ? 1 : 0;
    }
    rk[i] = (double)pos;
  }
  __syncthreads();
  const double* vh = VH + J.v_off;
  double* vec = VEC + J.u_off;
  for (int64_t i = warp; i < n; i += nwarps) {
    const int64_t pos = (int64_t)rk[i];
    // Right singular vector i is row i of vh (k x n, leading dimension k).
    double best = -1.0;
    int64_t bidx = 0;
    for (int64_t x = lane; x < n; x += 32) {
      const double v = fabs(vh[i + x * k]);
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
    const double sgn = vh[i + bidx * k] < 0.0 ? -1.0 : 1.0;
    for (int64_t x = lane; x < n; x += 32) vec[x + pos * n] = sgn * vh[i + x * k];
    if (lane == 0) {
      VAL[J.s_off + pos] = lam[i];
      if (MAG) MAG[J.s_off + pos] = fabs(lam[i]);
    }
  }
}

}  // namespace

cudaError_t launch_qr(const SvdJob* jobs, int32_t njobs, const double* a, double* q, double* r, double* work,
                      const int64_t* work_off, cudaStream_t stream) {
  if (njobs == 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(qr_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFacSmemBytes);
  if (e != cudaSuccess) return e;
  qr_kernel<<<njobs, kFacThreads, kFacSmemBytes, stream>>>(jobs, a, q, r, work, work_off);
  return cudaGetLastError();
}

cudaError_t launch_eigh(const SvdJob* jobs, int32_t njobs, const double* a, double* vecs, double* vals, double* mags,
                        double* work, const int64_t* work_off, int32_t* status, cudaStream_t stream) {
  if (njobs == 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(eigh_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFacSmemBytes);
  if (e != cudaSuccess) return e;
  eigh_kernel<<<njobs, kFacThreads, kFacSmemBytes, stream>>>(jobs, a, vecs, vals, mags, work, work_off, status);
  return cudaGetLastError();
}

bool eigh_on_chip(int64_t n) { return (size_t)(2 * n * n + 2 * n) * sizeof(double) <= kFacSmemBytes; }

cudaError_t launch_eigh_by_svd(const SvdJob* jobs, int32_t n_cluster, int32_t njobs, int64_t max_n, const double* a,
                               double* b, double* u, double* s, double* vh, double* shift, int32_t* bad,
                               double* vecs, double* vals, double* mags, double* work, const int64_t* work_off,
                               int32_t* status, cudaStream_t stream, int32_t n_wide) {
  if (njobs == 0) return cudaSuccess;
  const size_t post_smem = (size_t)2 * (size_t)max_n * sizeof(double);
  if (post_smem > kFacSmemBytes) return cudaErrorInvalidValue;
  eigh_shift_kernel<<<njobs, kFacThreads, 0, stream>>>(jobs, a, b, shift, bad);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = launch_svd_split(jobs, n_cluster, njobs, b, u, s, vh, work, work_off, status, stream, n_wide);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(eigh_from_svd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFacSmemBytes);
  if (e != cudaSuccess) return e;
  eigh_from_svd_kernel<<<njobs, kFacThreads, post_smem, stream>>>(jobs, s, vh, shift, vecs, vals, mags);
  return cudaGetLastError();
}

}  // namespace tnt
