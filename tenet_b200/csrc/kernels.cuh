// Device-side plan tables and kernel launchers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "plan_tables.hpp"

namespace tnt {

// A recoupling transform resident on one device.
struct DevXform {
  XGroup* groups = nullptr;
  XEntry* src = nullptr;
  XEntry* dst = nullptr;
  double* coef = nullptr;
  XTile* tiles = nullptr;  // sorted by kind
  int32_t ntiles = 0;
  int32_t kind_begin[kXKinds] = {0, 0, 0, 0, 0}, kind_count[kXKinds] = {0, 0, 0, 0, 0};
  int32_t max_nsrc = 0, max_ndst = 0;
};

// One unit of grouped-GEMM work of job `job` of batch entry `batch`.
// FP64 tile lists: (tm, tn) is the tile's first row and column in units of
// 16 and `shape` its geometry, f64_tile_code(BM, BN) with BM, BN in
// {16, 32, 48, 64}.  Split tile lists: (tm, tn) is the tile index at the
// split tile shape, `shape` is unused and `k` is the job's K (0 in FP64 lists).
struct GemmTile {
  int32_t job, batch, tm, tn, shape, k;
};
// Interior FP64 tile shapes the autotuner chooses between.
enum : int32_t { kShape64x64 = 0, kShape64x32 = 1, kShape32x64 = 2, kShape32x32 = 3 };
constexpr int kShapeM[4] = {64, 64, 32, 32};
constexpr int kShapeN[4] = {64, 32, 64, 32};
inline int32_t f64_tile_code(int bm, int bn) { return (bm / 16 - 1) * 4 + (bn / 16 - 1); }

struct DevGemm {
  GemmJob* jobs = nullptr;
  int32_t njobs = 0;
};

cudaError_t launch_xform(const DevXform& x, double* dst, const double* src, double alpha, double beta,
                         cudaStream_t stream);

// FP64 grouped GEMM over tiles of mixed shapes (mma.sync f64 tensor-core path).
cudaError_t launch_gemm_f64(const GemmJob* jobs, const GemmTile* tiles, int32_t ntiles, double* c, int64_t sc,
                            const double* a, int64_t sa, const double* b, int64_t sb, double alpha, double beta,
                            cudaStream_t stream);

// Split-precision grouped GEMM (BF16 slices, tcgen05 FP32 accumulation, FP64 recombination).
constexpr int kSplitTileM = 128;
// Output tile width picked from the sector-size histogram (64 or 128), given
// the per-MAC throughput of 64-wide tiles relative to 128-wide ones.
int split_tile_n(const GemmJob* host_jobs, int32_t njobs, double eff64);
// Padded multiply-accumulates of one batch entry at the given tile width.
double split_padded_macs(const GemmJob* host_jobs, int32_t njobs, int tile_n);
// i8 selects 8-bit integer digits on kind::i8 (tile width 64) instead of
// BF16 slices on kind::f16.
size_t split_scratch_bytes(const GemmJob* host_jobs, int32_t njobs, int64_t nbatch, int slices, int tile_n,
                           bool i8);
// Per-job packing table of the split operands (bytes to upload once per
// plan, slice count, tile width and format; the layout does not depend on nbatch).
std::vector<uint8_t> split_job_table(const GemmJob* host_jobs, int32_t njobs, int slices, int tile_n, bool i8);
// pre_a / pre_b (nullable, nbatch == 1 only): a side packed beforehand by
// launch_split_pack_operand, whose pack pass is then skipped.
cudaError_t launch_gemm_split(const void* job_table, const GemmJob* host_jobs, int32_t njobs, const GemmTile* tiles,
                              int32_t ntiles, double* c, int64_t sc, const double* a, int64_t sa, const double* b,
                              int64_t sb, int64_t nbatch, double alpha, double beta, int slices, int tile_n, bool i8,
                              void* scratch, size_t scratch_bytes, int32_t* err_word, cudaStream_t stream,
                              const void* pre_a = nullptr, const void* pre_b = nullptr);
// One operand of a compose packed once for many composes (side 0: the left
// operand A, 1: the right operand B): split_operand_bytes bytes, the side's
// slices then its row (column) scales.
size_t split_operand_bytes(const GemmJob* host_jobs, int32_t njobs, int slices, int tile_n, bool i8, int side);
cudaError_t launch_split_pack_operand(const void* job_table, const GemmJob* host_jobs, int32_t njobs, int side,
                                      const double* src, int slices, int tile_n, bool i8, void* packed,
                                      cudaStream_t stream);

// Batched one-sided Jacobi SVD, one CTA per coupled sector.
cudaError_t launch_svd(const SvdJob* jobs, int32_t njobs, const double* a, double* u, double* s, double* vh,
                       double* work, const int64_t* work_off, int32_t* status, cudaStream_t stream);

// Batched per-sector Householder QR (positive-diagonal gauge) and Jacobi eigh
// (descending |lambda|, largest-entry-positive vectors), factor.cu.
cudaError_t launch_qr(const SvdJob* jobs, int32_t njobs, const double* a, double* q, double* r, double* work,
                      const int64_t* work_off, cudaStream_t stream);
cudaError_t launch_eigh(const SvdJob* jobs, int32_t njobs, const double* a, double* vecs, double* vals, double* mags,
                        double* work, const int64_t* work_off, int32_t* status, cudaStream_t stream);
// True when eigh_kernel keeps an n x n sector (matrix and vectors) in shared memory.
bool eigh_on_chip(int64_t n);
// Eigendecomposition through the batched SVD of B = A + ||A||_F I, for plans
// with sectors beyond eigh_on_chip: b (a's layout), u, s, vh (the SVD
// layouts of the plan) and shift (one double per job) are scratch; *bad is
// set to 1 for a non-Hermitian or non-finite sector (not cleared here).
cudaError_t launch_eigh_by_svd(const SvdJob* jobs, int32_t n_cluster, int32_t njobs, int64_t max_n, const double* a,
                               double* b, double* u, double* s, double* vh, double* shift, int32_t* bad,
                               double* vecs, double* vals, double* mags, double* work, const int64_t* work_off,
                               int32_t* status, cudaStream_t stream, int32_t n_wide = 0);

// Large sectors on thread-block clusters: the first n_cluster jobs (those with
// at least svd_cluster_size() column blocks of the blocked path) run one
// cluster each, the rest one CTA each.
// The first n_wide of those jobs (at least svd_wide_cluster_size() column
// blocks) run on 16-CTA clusters where the device allows them.
cudaError_t launch_svd_split(const SvdJob* jobs, int32_t n_cluster, int32_t njobs, const double* a, double* u,
                             double* s, double* vh, double* work, const int64_t* work_off, int32_t* status,
                             cudaStream_t stream, int32_t n_wide = 0);
int svd_cluster_size();
// 16 where the current device can co-schedule a 16-CTA cluster of the SVD kernel, else 0.
int svd_wide_cluster_size();
__host__ __device__ bool svd_on_chip(int64_t rows, int64_t k);
__host__ __device__ int svd_block_width(int64_t rows, int64_t k);

// tnt_svd with its scratch in a file-scope device array (svd_static.cu): no
// device allocation; rejects plans whose scratch exceeds the array.
cudaError_t svd_static(const std::vector<SvdJob>& jobs, const double* a, double* u, double* s, double* vh,
                       cudaStream_t stream, std::string& why);

// Krylov building blocks (krylov.cu): weighted dots against k vectors, many-vector axpy, small eigensolver.
int64_t wdot_chunks(const SvdJob* host_sectors, int32_t nsectors, std::vector<int64_t>& sector_of_chunk,
                    std::vector<int64_t>& start_of_chunk);
cudaError_t launch_wdot(const SvdJob* sectors, int32_t nsectors, const int64_t* chunk_sector,
                        const int64_t* chunk_start, int64_t nchunks, int32_t k, const double* V, int64_t ldv,
                        const double* y, double* part, double* out, cudaStream_t stream);
cudaError_t launch_axpy_many(int64_t n, int32_t k, const double* V, int64_t ldv, const double* coef, double a,
                             const double* a_dev, double* y, cudaStream_t stream);
cudaError_t launch_symeig(int32_t m, const double* A, double* evals, double* evecs, int32_t* status,
                          cudaStream_t stream);

// Many strided block copies in one launch (segcopy.cu).
struct SegCopy {
  int64_t src_off, dst_off, rows, cols, src_ld, dst_ld, scale_off;  // scale_off < 0: no scaling
};
cudaError_t launch_segcopy(const SegCopy* segs, int64_t nseg, const double* src, double* dst, const double* scales,
                           cudaStream_t stream);

// Cross-sector truncation selection: one CTA per segment of sectors.
cudaError_t launch_truncate_segments(const SvdJob* jobs, int32_t nseg, const int64_t* seg_first, const double* s,
                                     int32_t policy, double p0, double p1, const int64_t* space_ranks, int64_t* kept,
                                     double* err, cudaStream_t stream);

// Cross-sector truncation selection in one CTA.
cudaError_t launch_truncate(const SvdJob* jobs, int32_t njobs, const double* s, int32_t policy, double p0, double p1,
                            const int64_t* space_ranks, int64_t* kept, double* err, cudaStream_t stream);

}  // namespace tnt
