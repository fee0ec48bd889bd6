// Recoupling transform kernel: dst = alpha * U . P(src) + beta * dst per group.
//
// Replaces the Host replay of tenet-operations/src/transform_replay.rs:
// Single blocks (4428-4517, a permuted strided copy times one coefficient) and
// Multi groups (4519-4800: pack every source block of a group into a column,
// one GEMM with U^T, scatter back).  Both compute, for every element position
// of the group's common block shape, dst_d = alpha * sum_s U[d, s] src_s (+ beta
// dst_d); here that sum is formed in registers, so each source element is read
// once and each destination element written once.
//
// A group's blocks are viewed as d0 x C matrices: d0 = the extent of
// destination axis 0 (stride 1 in every destination block, contiguous runs of
// the codomain), C = the product of the other extents ("columns").  A CTA
// takes a tile of columns; it stages the group's coefficients, the block
// offsets/strides and the multi-index of each of its columns in shared
// memory, then maps threads as (W lanes along axis 0) x (256/W columns), with
// W the power of two covering min(d0, 32).  Address arithmetic per element is
// a few multiply-adds from shared memory; no division in the element loop.
//
// Tiles come sorted by kernel path (xform_kind) and each path is its own
// kernel specialisation, so each gets the registers it needs: abelian copies
// with short rows unroll across columns; abelian copies with long rows and
// groups up to 4 x 4 (the SU(2) case) walk each column down axis 0 with
// paired 16-byte accesses where aligned; transposing abelian copies (source
// strided along axis 0, contiguous along another axis) stage planes through
// shared memory; everything else takes the general loop.
#include "kernels.cuh"

namespace tnt {

namespace {

constexpr int kXThreads = 256;
constexpr int kRegSrc = 8;        // source values cached in registers per element
constexpr int kSmemCoef = 1024;   // coefficients staged in shared memory
constexpr int kSmemEntries = 48;  // source + destination entries staged in shared memory
constexpr int kMaxTileCols = 256; // columns per tile (multi-indices staged in shared memory)
constexpr int kSmallGroup = 4;    // groups up to 4 x 4 take the register path

struct SmemEntry {
  int64_t offset;
  int64_t strides[kMaxRank];
};

template <int KIND>
__global__ void __launch_bounds__(kXThreads, 3) xform_kernel(const XTile* __restrict__ tiles, int32_t ntiles,
                                                          const XGroup* __restrict__ groups,
                                                          const XEntry* __restrict__ src_e,
                                                          const XEntry* __restrict__ dst_e,
                                                          const double* __restrict__ coef,
                                                          const double* __restrict__ src, double* __restrict__ dst,
                                                          double alpha, double beta) {
  __shared__ XGroup g;
  __shared__ XTile tile;
  __shared__ double U[kSmemCoef];
  __shared__ SmemEntry ent[kSmemEntries];
  __shared__ uint16_t cidx[kMaxTileCols][kMaxRank - 1];
  __shared__ int64_t cbase[kMaxTileCols][2];  // abelian groups: per-column source / destination base offsets

  const int tid = threadIdx.x;
  for (int32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    __syncthreads();
    if (tid == 0) {
      tile = tiles[t];
      g = groups[tile.group];
    }
    __syncthreads();
    const int nsrc = g.nsrc, ndst = g.ndst, rank = g.rank;
    const int ncoef = nsrc * ndst;
    const bool coef_smem = ncoef <= kSmemCoef;
    const bool ent_smem = nsrc + ndst <= kSmemEntries;
    const int d0 = rank > 0 ? g.dims[0] : 1;
    const int ncols = (int)tile.count;
    if (coef_smem)
      for (int i = tid; i < ncoef; i += kXThreads) U[i] = coef[g.coef_off + i];
    if (ent_smem) {
      for (int i = tid; i < nsrc + ndst; i += kXThreads) {
        const XEntry& e = i < nsrc ? src_e[g.src_first + i] : dst_e[g.dst_first + (i - nsrc)];
        ent[i].offset = e.offset;
#pragma unroll
        for (int k = 0; k < kMaxRank; ++k) ent[i].strides[k] = k < rank ? e.strides[k] : 0;
      }
    }
    const bool abelian = KIND == 0 || KIND == 3;
    for (int c = tid; c < (KIND == 4 ? 0 : ncols); c += kXThreads) {
      int64_t col = tile.start + c;
      int64_t sb = 0, db = 0;
      const XEntry* es = abelian ? &src_e[g.src_first] : nullptr;
      const XEntry* ed = abelian ? &dst_e[g.dst_first] : nullptr;
#pragma unroll
      for (int k = 1; k < kMaxRank; ++k) {
        uint16_t v = 0;
        if (k < rank) {
          const int32_t dk = g.dims[k];
          const int64_t q = col / dk;
          v = (uint16_t)(col - q * dk);
          col = q;
          if (abelian) {
            sb += (int64_t)v * es->strides[k];
            db += (int64_t)v * ed->strides[k];
          }
        }
        cidx[c][k - 1] = v;
      }
      if (abelian) {
        cbase[c][0] = es->offset + sb;
        cbase[c][1] = ed->offset + db;
      }
    }
    __syncthreads();

    const double* Ug = coef_smem ? U : coef + g.coef_off;
    int W = 1;
    while (W < d0 && W < 32) W <<= 1;
    const int H = kXThreads / W;
    const int tx = tid % W, ty = tid / W;

    if constexpr (KIND == 4) {
      // Transposing copies (one source and one destination block, source
      // stride 1 along a destination axis k* > 0, not along axis 0): the
      // block is a stack of planes (axis 0 x axis k*) over the remaining
      // axes; a tile is a range of planes.  Planes, cut into sub-planes of at
      // most 64 columns of k* and as many rows of axis 0 as shared memory
      // holds, are staged in batches: loaded with consecutive threads along
      // k* (contiguous in the source), written with consecutive threads along
      // axis 0 (contiguous in the destination), every lane active.
      constexpr int kTrCap = 4096;  // doubles of staging
      constexpr int kTrPlanes = 64;
      __shared__ double tbuf[kTrCap];
      __shared__ int64_t pbase[kTrPlanes][2];
      const double u = alpha * Ug[0];
      // k*: the first axis after 0 with source stride 1 and extent above 1
      // (the host assigns this path only when there is one).
      int ks = 1;
      while (ks < rank - 1 && !(ent[0].strides[ks] == 1 && g.dims[ks] > 1)) ++ks;
      const int64_t s0 = ent[0].strides[0], sks = ent[0].strides[ks], dks = ent[1].strides[ks];
      const int dj = g.dims[ks];
      const int J = dj < 64 ? dj : 64, Jp = J + 1;
      const int R = d0 < kTrCap / Jp ? d0 : kTrCap / Jp;
      const int64_t o_end = tile.start + tile.count;
      for (int i0 = 0; i0 < d0; i0 += R) {
        const int r = d0 - i0 < R ? d0 - i0 : R;
        for (int j0 = 0; j0 < dj; j0 += J) {
          const int jn = dj - j0 < J ? dj - j0 : J;
          const int ps = r * Jp;  // staging doubles per plane
          const int npmax = kTrCap / ps < kTrPlanes ? kTrCap / ps : kTrPlanes;  // >= 1: ps <= kTrCap
          for (int64_t o0 = tile.start; o0 < o_end; o0 += npmax) {
            const int np = o_end - o0 < npmax ? (int)(o_end - o0) : npmax;
            if (tid < np) {
              int64_t rem = o0 + tid, sb = ent[0].offset, db = ent[1].offset;
#pragma unroll
              for (int k = 1; k < kMaxRank; ++k) {
                if (k < rank && k != ks) {
                  const int32_t dk = g.dims[k];
                  const int64_t q = rem / dk;
                  const int64_t v = rem - q * dk;
                  rem = q;
                  sb += v * ent[0].strides[k];
                  db += v * ent[1].strides[k];
                }
              }
              pbase[tid][0] = sb + (int64_t)i0 * s0 + (int64_t)j0 * sks;
              pbase[tid][1] = db + i0 + (int64_t)j0 * dks;
            }
            __syncthreads();
            // Load: flat over (plane, row, k* column), k* fastest (contiguous in
            // the source); eight loads in flight per thread.  Quotients by
            // float reciprocal: exact here, since e < 4096 keeps the product's
            // error below 2^-11, under half of 1 / divisor for divisors below 1024.
            const int n_el = np * r * jn;
            const float inv_jn = 1.0f / (float)jn, inv_r = 1.0f / (float)r;
            for (int e0 = tid; e0 < n_el; e0 += 8 * kXThreads) {
              double v[8];
              int at[8];
#pragma unroll
              for (int q = 0; q < 8; ++q) {
                const int e = e0 + q * kXThreads;
                at[q] = -1;
                if (e < n_el) {
                  const int row = __float2int_rz(((float)e + 0.5f) * inv_jn), j = e - row * jn;
                  const int p = __float2int_rz(((float)row + 0.5f) * inv_r), i = row - p * r;
                  v[q] = __ldg(src + pbase[p][0] + (int64_t)i * s0 + (int64_t)j * sks);
                  at[q] = p * ps + i * Jp + j;
                }
              }
#pragma unroll
              for (int q = 0; q < 8; ++q)
                if (at[q] >= 0) tbuf[at[q]] = v[q];
            }
            __syncthreads();
            // Store: flat over (plane, k* column, row), rows fastest (contiguous
            // in the destination).
            for (int e = tid; e < n_el; e += kXThreads) {
              const int col = __float2int_rz(((float)e + 0.5f) * inv_r), i = e - col * r;
              const int p = __float2int_rz(((float)col + 0.5f) * inv_jn), j = col - p * jn;
              const double x = u * tbuf[p * ps + i * Jp + j];
              double* dp = dst + pbase[p][1] + (int64_t)j * dks + i;
              *dp = beta == 0.0 ? x : fma(beta, *dp, x);
            }
            __syncthreads();
          }
        }
      }
      continue;
    }

    if constexpr (KIND == 0) {
      // Abelian groups: a scaled permuted copy.  Each thread issues kUnroll
      // independent loads before its stores so enough bytes are in flight to
      // cover HBM latency; column bases come precomputed from shared memory.
      constexpr int kUnroll = 8;
      const double scale = alpha * Ug[0];
      const int64_t s0 = src_e[g.src_first].strides[0];
      for (int i0 = tx; i0 < d0; i0 += W) {
        const int64_t si = (int64_t)i0 * s0;
        for (int cl0 = ty; cl0 < ncols; cl0 += H * kUnroll) {
          double v[kUnroll];
          int64_t od[kUnroll];
#pragma unroll
          for (int u = 0; u < kUnroll; ++u) {
            const int cl = cl0 + u * H;
            od[u] = -1;
            if (cl < ncols) {
              v[u] = __ldg(src + cbase[cl][0] + si);
              od[u] = cbase[cl][1] + i0;
            }
          }
#pragma unroll
          for (int u = 0; u < kUnroll; ++u) {
            if (od[u] >= 0) {
              const double x = scale * v[u];
              dst[od[u]] = beta == 0.0 ? x : fma(beta, dst[od[u]], x);
            }
          }
        }
      }
      continue;
    }

    if constexpr (KIND == 3) {
      // Abelian groups with long rows: a scaled copy of each column down
      // destination axis 0 (column bases precomputed in shared memory).  Each
      // thread issues four loads before its stores, 16-byte pairs when the
      // source runs along that axis and both bases are 16-byte aligned.
      const double u = alpha * Ug[0];
      const int64_t s0 = src_e[g.src_first].strides[0];
      for (int cl = ty; cl < ncols; cl += H) {
        const int64_t sbase = cbase[cl][0], dbase = cbase[cl][1];
        const bool vec = s0 == 1 && (d0 & 1) == 0 &&
                         ((reinterpret_cast<uintptr_t>(src + sbase) | reinterpret_cast<uintptr_t>(dst + dbase)) & 15) == 0;
        if (vec) {
          const int np = d0 >> 1;
          const double2* sp = reinterpret_cast<const double2*>(src + sbase);
          double2* op = reinterpret_cast<double2*>(dst + dbase);
          for (int p0 = tx; p0 < np; p0 += 4 * W) {
            double2 v[4];
#pragma unroll
            for (int q = 0; q < 4; ++q)
              if (p0 + q * W < np) v[q] = __ldg(sp + p0 + q * W);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int p = p0 + q * W;
              if (p < np) {
                const double2 a = make_double2(u * v[q].x, u * v[q].y);
                if (beta == 0.0) {
                  op[p] = a;
                } else {
                  const double2 b = op[p];
                  op[p] = make_double2(fma(beta, b.x, a.x), fma(beta, b.y, a.y));
                }
              }
            }
          }
        } else {
          for (int i0 = tx; i0 < d0; i0 += 4 * W) {
            double v[4];
#pragma unroll
            for (int q = 0; q < 4; ++q)
              if (i0 + q * W < d0) v[q] = __ldg(src + sbase + (int64_t)(i0 + q * W) * s0);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int i = i0 + q * W;
              if (i < d0) {
                double* o = dst + dbase + i;
                *o = beta == 0.0 ? u * v[q] : fma(beta, *o, u * v[q]);
              }
            }
          }
        }
      }
      continue;
    }

    if constexpr (KIND == 1) {
      // Small recoupling groups (the SU(2) case, and abelian groups with long
      // rows): per column, the block base offsets are formed once and the loop
      // runs down destination axis 0 (stride 1 in every destination block).
      // When every source is contiguous along that axis and every base is
      // 16-byte aligned, elements move in pairs (16-byte loads and stores).
      for (int cl = ty; cl < ncols; cl += H) {
        int64_t sb[kSmallGroup], db[kSmallGroup];
        bool vec = (d0 & 1) == 0;
#pragma unroll
        for (int e = 0; e < kSmallGroup; ++e) {
          sb[e] = 0;
          db[e] = 0;
          if (e < nsrc) {
            const SmemEntry& en = ent[e];
            int64_t o = en.offset;
#pragma unroll
            for (int k = 1; k < kMaxRank; ++k) o += (int64_t)cidx[cl][k - 1] * en.strides[k];
            sb[e] = o;
            vec = vec && en.strides[0] == 1 && ((reinterpret_cast<uintptr_t>(src + o) & 15) == 0);
          }
          if (e < ndst) {
            const SmemEntry& en = ent[nsrc + e];
            int64_t o = en.offset;
#pragma unroll
            for (int k = 1; k < kMaxRank; ++k) o += (int64_t)cidx[cl][k - 1] * en.strides[k];
            db[e] = o;
            vec = vec && ((reinterpret_cast<uintptr_t>(dst + o) & 15) == 0);
          }
        }
        if (vec) {
          const int np = d0 >> 1;
          for (int p0 = tx; p0 < np; p0 += 2 * W) {
            const int p1 = p0 + W;
            const bool two = p1 < np;
            double2 v0[kSmallGroup], v1[kSmallGroup];
#pragma unroll
            for (int e = 0; e < kSmallGroup; ++e) {
              v0[e] = make_double2(0.0, 0.0);
              v1[e] = make_double2(0.0, 0.0);
              if (e < nsrc) {
                const double2* sp = reinterpret_cast<const double2*>(src + sb[e]);
                v0[e] = __ldg(sp + p0);
                if (two) v1[e] = __ldg(sp + p1);
              }
            }
#pragma unroll
            for (int d = 0; d < kSmallGroup; ++d) {
              if (d < ndst) {
                double2 a0 = make_double2(0.0, 0.0), a1 = make_double2(0.0, 0.0);
#pragma unroll
                for (int e = 0; e < kSmallGroup; ++e)
                  if (e < nsrc) {
                    const double u = alpha * Ug[d * nsrc + e];
                    a0.x = fma(u, v0[e].x, a0.x);
                    a0.y = fma(u, v0[e].y, a0.y);
                    a1.x = fma(u, v1[e].x, a1.x);
                    a1.y = fma(u, v1[e].y, a1.y);
                  }
                double2* o = reinterpret_cast<double2*>(dst + db[d]);
                if (beta == 0.0) {
                  o[p0] = a0;
                  if (two) o[p1] = a1;
                } else {
                  double2 b0 = o[p0];
                  o[p0] = make_double2(fma(beta, b0.x, a0.x), fma(beta, b0.y, a0.y));
                  if (two) {
                    double2 b1 = o[p1];
                    o[p1] = make_double2(fma(beta, b1.x, a1.x), fma(beta, b1.y, a1.y));
                  }
                }
              }
            }
          }
          continue;
        }
        for (int i0 = tx; i0 < d0; i0 += 2 * W) {
          const int i1 = i0 + W;
          const bool two = i1 < d0;
          double v0[kSmallGroup], v1[kSmallGroup];
#pragma unroll
          for (int e = 0; e < kSmallGroup; ++e) {
            v0[e] = 0.0;
            v1[e] = 0.0;
            if (e < nsrc) {
              const int64_t s0 = ent[e].strides[0];
              v0[e] = __ldg(src + sb[e] + (int64_t)i0 * s0);
              if (two) v1[e] = __ldg(src + sb[e] + (int64_t)i1 * s0);
            }
          }
#pragma unroll
          for (int d = 0; d < kSmallGroup; ++d) {
            if (d < ndst) {
              double a0 = 0.0, a1 = 0.0;
#pragma unroll
              for (int e = 0; e < kSmallGroup; ++e)
                if (e < nsrc) {
                  const double u = Ug[d * nsrc + e];
                  a0 = fma(u, v0[e], a0);
                  a1 = fma(u, v1[e], a1);
                }
              double* o = dst + db[d] + i0;
              if (beta == 0.0) {
                o[0] = alpha * a0;
                if (two) o[W] = alpha * a1;
              } else {
                o[0] = fma(beta, o[0], alpha * a0);
                if (two) o[W] = fma(beta, o[W], alpha * a1);
              }
            }
          }
        }
      }
      continue;
    }

    if constexpr (KIND == 2) {
    for (int cl = ty; cl < ncols; cl += H) {
      int32_t ci[kMaxRank - 1];
#pragma unroll
      for (int k = 0; k < kMaxRank - 1; ++k) ci[k] = cidx[cl][k];
      for (int i0 = tx; i0 < d0; i0 += W) {
        auto place = [&](int e, bool is_src) -> int64_t {
          if (ent_smem) {
            const SmemEntry& en = ent[is_src ? e : nsrc + e];
            int64_t off = en.offset + (int64_t)i0 * en.strides[0];
#pragma unroll
            for (int k = 1; k < kMaxRank; ++k) off += (int64_t)ci[k - 1] * en.strides[k];
            return off;
          }
          const XEntry& en = is_src ? src_e[g.src_first + e] : dst_e[g.dst_first + e];
          int64_t off = en.offset + (int64_t)i0 * en.strides[0];
          for (int k = 1; k < rank; ++k) off += (int64_t)ci[k - 1] * en.strides[k];
          return off;
        };
        if (nsrc == 1 && ndst == 1) {  // abelian groups: one scaled permuted copy
          const double v = alpha * Ug[0] * __ldg(src + place(0, true));
          const int64_t o = place(0, false);
          dst[o] = beta == 0.0 ? v : fma(beta, dst[o], v);
        } else if (nsrc == 0) {
          for (int d = 0; d < ndst; ++d) {
            const int64_t o = place(d, false);
            dst[o] = beta == 0.0 ? 0.0 : beta * dst[o];
          }
        } else if (nsrc <= kRegSrc) {
          double v[kRegSrc];
#pragma unroll
          for (int s = 0; s < kRegSrc; ++s)
            if (s < nsrc) v[s] = __ldg(src + place(s, true));
          for (int d = 0; d < ndst; ++d) {
            double acc = 0.0;
#pragma unroll
            for (int s = 0; s < kRegSrc; ++s)
              if (s < nsrc) acc = fma(Ug[d * nsrc + s], v[s], acc);
            const int64_t o = place(d, false);
            dst[o] = beta == 0.0 ? alpha * acc : fma(beta, dst[o], alpha * acc);
          }
        } else {
          for (int d = 0; d < ndst; ++d) {
            double acc = 0.0;
            for (int s = 0; s < nsrc; ++s) acc = fma(Ug[d * nsrc + s], __ldg(src + place(s, true)), acc);
            const int64_t o = place(d, false);
            dst[o] = beta == 0.0 ? alpha * acc : fma(beta, dst[o], alpha * acc);
          }
        }
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
  for (int k = 0; k < kXKinds; ++k) {
    const int32_t n = x.kind_count[k];
    if (n == 0) continue;
    const int grid = n < sms * 8 ? n : sms * 8;
    const XTile* t = x.tiles + x.kind_begin[k];
    if (k == 0)
      xform_kernel<0><<<grid, kXThreads, 0, stream>>>(t, n, x.groups, x.src, x.dst, x.coef, src, dst, alpha, beta);
    else if (k == 1)
      xform_kernel<1><<<grid, kXThreads, 0, stream>>>(t, n, x.groups, x.src, x.dst, x.coef, src, dst, alpha, beta);
    else if (k == 3)
      xform_kernel<3><<<grid, kXThreads, 0, stream>>>(t, n, x.groups, x.src, x.dst, x.coef, src, dst, alpha, beta);
    else if (k == 4)
      xform_kernel<4><<<grid, kXThreads, 0, stream>>>(t, n, x.groups, x.src, x.dst, x.coef, src, dst, alpha, beta);
    else
      xform_kernel<2><<<grid, kXThreads, 0, stream>>>(t, n, x.groups, x.src, x.dst, x.coef, src, dst, alpha, beta);
  }
  return cudaGetLastError();
}

}  // namespace tnt
