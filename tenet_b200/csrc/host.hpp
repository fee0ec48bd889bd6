// Host-side structure compiler for the symmetric block-sparse path.
//
// Restates, in C++, the multiplicity-free structure layer of TeNeT:
//   - sector labels, SectorId codecs and F/R/B symbols
//     (tenet-sectors/src/{abelian,su2,product_rule,algebra}.rs),
//   - graded legs and fusion-tree enumeration
//     (tenet-core/src/sector.rs:147-237, fusion_tree.rs:491-560, 970-1130),
//   - the coupled-sector column-major block layout
//     (tenet-core/src/fusion_space.rs:2211-2262, 3953-4104),
//   - tree-pair recoupling (Artin braids, bends, repartition, permute;
//     fusion_tree.rs:2477-2507, 2763-2870, 3319-3355, 3785-3812, 8154-8253,
//     8744-9040),
//   - grouped transform plans (tenet-operations/src/transform_structure.rs:587-770)
//     and per-sector GEMM job tables (tenet-operations/src/fusion_replay.rs:457-530).
// The outputs are the plain tables the CUDA kernels consume (plan_tables.hpp).
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "plan_tables.hpp"

namespace tnt {

enum FactorKind : int32_t { FK_U1 = 0, FK_SU2 = 1, FK_FZ2 = 2, FK_Z2 = 3, FK_TABLE = 4 };
enum CodecKind : int32_t { CODEC_PACKED = 0, CODEC_CANTOR = 1 };

constexpr int kMaxFactors = 4;

struct Sector {
  int32_t v[kMaxFactors] = {0, 0, 0, 0};
  bool operator==(const Sector& o) const {
    return v[0] == o.v[0] && v[1] == o.v[1] && v[2] == o.v[2] && v[3] == o.v[3];
  }
  bool operator!=(const Sector& o) const { return !(*this == o); }
};

// A checked table provider: a multiplicity-free rule with real, symmetric
// braiding given by its tables (sector labels 0 .. n-1, 0 the vacuum, the
// SectorId of label i is i).  Validated once by check_table (the reference's
// CheckedGenericFusion / CheckedGenericRigidSymbols admission,
// tenet-sectors/src/algebra.rs:743-910).
struct TableData {
  int n = 0;
  std::vector<int32_t> dual;   // n
  std::vector<uint8_t> N;      // n^3, N[(a n + b) n + c] in {0, 1}
  std::vector<double> dims;    // n
  std::vector<double> fs;      // n
  std::vector<double> R;       // n^3
  std::vector<double> F;       // n^6, F(a, b, c; d; e, f)
  uint64_t identity = 0;       // content hash: equal tables, equal rules
  bool nsym(int a, int b, int c) const { return N[((size_t)a * n + b) * n + c] != 0; }
  double f(int a, int b, int c, int d, int e, int g) const {
    return F[((((((size_t)a * n + b) * n + c) * n + d) * n + e) * n) + g];
  }
};

// Throws std::invalid_argument naming the first law the tables break.
void check_table(const TableData& t, double tol);

struct Rule {
  int nf = 1;
  FactorKind kind[kMaxFactors] = {FK_U1, FK_U1, FK_U1, FK_U1};
  CodecKind codec = CODEC_PACKED;
  std::shared_ptr<const TableData> table;  // FK_TABLE (a single-factor rule)

  bool fermionic() const;
  bool unique() const;  // no SU(2) factor: every fusion has one channel
  uint64_t id(const Sector& s) const;
  Sector vacuum() const { return Sector{}; }
  Sector dual(const Sector& s) const;
  void channels(const Sector& a, const Sector& b, std::vector<Sector>& out) const;
  bool nsym(const Sector& a, const Sector& b, const Sector& c) const;
  double dim(const Sector& a) const;
  double twist(const Sector& a) const;
  double fs(const Sector& a) const;
  double R(const Sector& a, const Sector& b, const Sector& c) const;
  double F(const Sector& a, const Sector& b, const Sector& c, const Sector& d, const Sector& e,
           const Sector& f) const;
  double B(const Sector& a, const Sector& b, const Sector& c) const;
  bool operator==(const Rule& o) const;
};

// SU(2) F-symbol in the Condon-Shortley gauge, doubled spins.
double su2_fsymbol(int a, int b, int c, int d, int e, int f);

struct Leg {
  std::vector<Sector> sectors;  // as stored (dualized for a dual leg), sorted by id
  std::vector<int64_t> degs;
  bool dual = false;

  static Leg make(const Rule& r, const std::vector<Sector>& s, const std::vector<int64_t>& d, bool dual);
  Leg dualized(const Rule& r) const;
  int64_t deg(const Sector& s) const;
  bool operator==(const Leg& o) const;
};

struct Tree {
  std::vector<Sector> u;
  std::vector<uint8_t> d;
  Sector c;
  std::vector<Sector> inner;  // innermost first
};

struct TreePair {
  Tree cod, dom;
};

// Serialised tree pair used as a hash key.
std::string pair_key(const TreePair& p);

struct SectorInfo {
  Sector c;
  int64_t rows = 0, cols = 0, offset = 0;
};

struct BlockInfo {
  TreePair key;
  int32_t sector = 0;
  int64_t offset = 0;
  int64_t shape[kMaxRank] = {};
  int64_t strides[kMaxRank] = {};
  int64_t row_start = 0, col_start = 0;
};

struct Space {
  Rule rule;
  std::vector<Leg> cod, dom;
  std::vector<SectorInfo> sectors;
  std::vector<BlockInfo> blocks;
  std::unordered_map<std::string, int32_t> block_index;
  int64_t size = 0;

  int n1() const { return (int)cod.size(); }
  int n2() const { return (int)dom.size(); }
  int sector_of(const Sector& c) const;
  bool same_as(const Space& o) const;
};

std::shared_ptr<Space> make_space(const Rule& r, const std::vector<Leg>& cod, const std::vector<Leg>& dom);

// Recoupling terms of one tree pair.
using Terms = std::vector<std::pair<TreePair, double>>;
Terms artin_terms(const Rule& r, const Tree& t, int index, bool inverse);
Terms bendright(const Rule& r, const TreePair& p);
Terms bendleft(const Rule& r, const TreePair& p);
Terms repartition_terms(const Rule& r, const TreePair& p, int target);
Terms braid_pair_terms(const Rule& r, const TreePair& p, const std::vector<int>& p1,
                       const std::vector<int>& p2, const std::vector<int>& lv1, const std::vector<int>& lv2);

enum TransformKind : int32_t { XK_PERMUTE = 0, XK_BRAID = 1, XK_REPARTITION = 2, XK_ADJOINT = 3 };

// Host copy of a compiled recoupling transform (device tables: plan_tables.hpp).
struct TransformPlan {
  std::shared_ptr<Space> src, dst;
  std::vector<int> axes;  // dst axis k reads src axis axes[k]
  XformTables tables;
  int64_t moved_elements = 0;  // sum over groups of nelem * (nsrc + ndst)
};

// Group maxima and device tiles of tables whose groups and entries are set
// (for tables compiled elsewhere).
void finish_transform_tables(XformTables& t);

// One step of a recoupling chain.  twist_axes (this step's destination flat
// axes) and supertrace (>= 0: the fermionic supertrace twist on the first
// `supertrace` codomain positions, see supertrace_axes) multiply each
// destination block by the product of the named ribbon twists.
struct TransformStep {
  TransformKind kind = XK_PERMUTE;
  std::vector<int> p1, p2, levels;
  int nrep = 0;
  std::vector<int> twist_axes;
  int supertrace = -1;
};

// Several steps replayed as one transform: per source tree pair the terms of
// every step are multiplied through, so the payload is read and written once.
std::shared_ptr<TransformPlan> make_transform_chain(const std::shared_ptr<Space>& src,
                                                    const std::vector<TransformStep>& steps);

// Spaces after each step of a chain (geometry only, no coefficients).
std::vector<std::shared_ptr<Space>> chain_spaces(const std::shared_ptr<Space>& src,
                                                 const std::vector<TransformStep>& steps);
// A step that changes nothing on `src`: a permute keeping every axis in place
// with no twist that acts on it.
bool step_is_noop(const Space& src, const TransformStep& st);

// twist_axes (destination flat axes, codomain first) multiplies every
// destination block by the product of the ribbon twists of its uncoupled
// sectors on those axes (TensorKit twist; typed.rs:4599), fused into the
// plan's coefficients.
std::shared_ptr<TransformPlan> make_transform(const std::shared_ptr<Space>& src, TransformKind kind,
                                              const std::vector<int>& p1, const std::vector<int>& p2,
                                              const std::vector<int>& levels, int nrep,
                                              const std::vector<int>& twist_axes = {});

// Destination axes of a contraction's right operand, permuted to
// (contracted ; open), that carry the fermionic supertrace twist: the
// contracted codomain positions whose leg is dual
// (tenet-tensors/src/contract/fusion/block_specs.rs:683-716,
// contract/dynamic.rs:2697-2760).  Empty for non-fermionic rules.
std::vector<int> supertrace_axes(const Space& dst, int n_contracted);

// Per-sector GEMM batch of C = A o B.
struct ComposePlan {
  std::shared_ptr<Space> lhs, rhs, dst;
  GemmTables tables;
  double flops = 0;  // 2 m n k summed over jobs
};

std::shared_ptr<ComposePlan> make_compose(const std::shared_ptr<Space>& lhs, const std::shared_ptr<Space>& rhs);

// Per-sector factorisation layout (SVD of every coupled-sector matrix).
struct FactorPlan {
  std::shared_ptr<Space> src;
  SvdTables tables;
};
std::shared_ptr<FactorPlan> make_factor(const std::shared_ptr<Space>& src);

}  // namespace tnt
