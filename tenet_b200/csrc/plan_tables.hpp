// Plain-old-data tables shared by the host structure compiler and the CUDA
// kernels.  Everything the device reads is one of these structs, uploaded
// once per plan and reused by every replay.
#pragma once

#include <cstdint>
#include <vector>

namespace tnt {

constexpr int kMaxRank = 8;

// One recoupling group: every source block shares the same uncoupled sectors,
// so all blocks of the group have one shape; the group maps nsrc source blocks
// to ndst destination blocks through the row-major ndst x nsrc matrix U
// (the TreeTransformGroupPlan U[dst, src] of tenet-operations/src/transform_plan.rs:642-705).
struct XGroup {
  int64_t nelem;             // elements per block
  int32_t nsrc, ndst;        // 0 sources: a destination block nothing maps to
  int32_t src_first;         // first entry in src_entries
  int32_t dst_first;         // first entry in dst_entries
  int32_t coef_off;          // first coefficient of U
  int32_t rank;
  int32_t dims[kMaxRank];    // block extents in destination axis order
};

// Kernel path of a group's tiles: 0 = abelian copy with short rows (column
// bases staged, unrolled across columns), 1 = groups up to 4 x 4 walked down
// destination axis 0 (paired 16-byte accesses where aligned), 2 = anything
// else, 3 = abelian copy with long rows (one source, one destination, d0 >=
// 64: each column walked down axis 0 with four 16-byte loads in flight),
// 4 = transposing abelian copy (assigned by the host tiler, which sees the
// entries: see xform_transposing_axis).  Shared by the host tiler and the
// device kernels.
constexpr int kXKinds = 5;
inline int xform_kind(const XGroup& g) {
  const int d0 = g.rank > 0 ? g.dims[0] : 1;
  if (g.nsrc == 1 && g.ndst == 1) return d0 < 64 ? 0 : 3;
  if (g.nsrc >= 1 && g.nsrc <= 4 && g.ndst <= 4) return 1;
  return 2;
}

// Placement of one block inside the flat payload.  Source strides are listed
// in destination axis order, so element (i0..i_{r-1}) of the destination block
// reads src[offset + sum_k i_k * strides[k]].
struct XEntry {
  int64_t offset;
  int64_t strides[kMaxRank];
};

// A contiguous range of columns (positions of every axis but destination
// axis 0) of one group, the unit of device work.
struct XTile {
  int32_t group;
  int32_t kind;  // xform_kind of the group
  int64_t start;
  int64_t count;
};

struct XformTables {
  std::vector<XGroup> groups;
  std::vector<XEntry> src_entries, dst_entries;
  std::vector<double> coef;
  std::vector<XTile> tiles;
  int64_t src_size = 0, dst_size = 0;
  int32_t max_nsrc = 0, max_ndst = 0;
};

// One dense GEMM of a coupled sector, column-major: C[m x n] = A[m x k] B[k x n]
// (a Rank2GemmBatchJob of tenet-operations/src/fusion_replay.rs:518-528).
struct GemmJob {
  int64_t m, n, k;
  int64_t a_off, b_off, c_off;
  int64_t lda, ldb, ldc;
};

struct GemmTables {
  std::vector<GemmJob> jobs;
  int64_t a_size = 0, b_size = 0, c_size = 0;
};

// One coupled-sector matrix to factorise: A[m x n] (column-major, lda = m) ->
// U[m x k], S[k], Vh[k x n] with k = min(m, n).
struct SvdJob {
  int64_t m, n, k;
  int64_t a_off, u_off, s_off, v_off;
  double weight;  // quantum dimension of the coupled sector
};

struct SvdTables {
  std::vector<SvdJob> jobs;
  int64_t a_size = 0, u_size = 0, s_size = 0, v_size = 0;
};

}  // namespace tnt
