/*
 * tenet_b200.h -- C ABI of the B200-native symmetric block-sparse backend.
 *
 * Plain pointers and sizes only.  Every call returns a tnt_status and never
 * aborts; on failure nothing is published into caller-owned output (the
 * reference's all-or-nothing rule, README.md:93-94 of TeNeT) and
 * tnt_last_error() returns a message for the calling thread.
 *
 * Reference seams replaced (paths relative to the TeNeT workspace):
 *   structure:  tenet-core/src/block_structure.rs:1692 (BlockStructure),
 *               tenet-core/src/fusion_space.rs:3953-4104 (coupled layout)
 *   transform:  tenet-operations/src/replay_backend.rs:28-79
 *               (TreeTransformBackend::tree_transform_structure_into_raw)
 *   compose:    tenet-operations/src/fusion_replay.rs:1302-1380 (StorageGemm),
 *               tenet-dense/src/executor.rs:217 (matmul_batch_axpby_into)
 *   factorize:  tenet-dense/src/executor.rs:34-300 (svd_into),
 *               tenet-matrixalgebra/src/factorize.rs:1409 (svd_trunc_factors_dyn),
 *               tenet-matrixalgebra/src/truncation.rs:257 (select_truncation)
 *
 * Device pointers are plain CUDA global-memory pointers (double*) on the
 * context's device; `stream` is a cudaStream_t passed as void* (NULL = the
 * legacy default stream).  Plans are immutable after creation and may be
 * shared across threads.
 *
 * Threading and streams.  A context owns one set of grow-only scratch
 * buffers (split-precision slice packs, staging for host tables, segment
 * tables, dot partials) and one set of status words, shared by every call on
 * it; the context's mutex guards them on the host.  Calls on one context may
 * come from several threads and several streams: a call that uses the
 * scratch on a stream other than the previous user's first makes its stream
 * wait for that user's work (a CUDA event), so such calls are correct but
 * their scratch-using work does not overlap on the device.  For device
 * overlap, give each stream its own context (contexts share nothing but
 * plans), or pass caller scratch (tnt_compose_ws, tnt_svd_ws).  Two
 * exceptions: (1) a call made while its stream captures a CUDA graph is not
 * tracked, so the caller orders the graph's replays against other calls on
 * the same context; (2) the factorisation entry points (tnt_svd, tnt_svd_ws,
 * tnt_qr, tnt_eigh, tnt_symeig, tnt_truncate_segments, and tnt_truncate with
 * space ranks) synchronise their stream before returning.
 */
#ifndef TENET_B200_H
#define TENET_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  TNT_OK = 0,
  TNT_INVALID_ARGUMENT = 1,
  TNT_OUT_OF_MEMORY = 2,
  TNT_UNSUPPORTED = 3,
  TNT_CUDA_ERROR = 4,
  TNT_DEVICE_TIMEOUT = 5,
  TNT_INTERNAL = 6
} tnt_status;

/* Fusion-rule factors and SectorId codecs. */
enum { TNT_U1 = 0, TNT_SU2 = 1, TNT_FZ2 = 2, TNT_Z2 = 3 };
enum { TNT_CODEC_PACKED = 0, TNT_CODEC_CANTOR = 1 };

/* Compose arithmetic: FP64 tensor cores, BF16 slices (kind::f16, FP32
 * accumulation), one cuBLAS DGEMM per sector, or 8-bit integer digits
 * (kind::i8, exact int32 accumulation per product diagonal). */
enum { TNT_PREC_FP64 = 0, TNT_PREC_BF16X = 1, TNT_PREC_CUBLAS_FP64 = 2, TNT_PREC_INT8X = 3 };

/* Truncation policies (tenet-matrixalgebra/src/truncation.rs:69-93). */
enum { TNT_TRUNC_FULL = 0, TNT_TRUNC_RANK = 1, TNT_TRUNC_TOL = 2, TNT_TRUNC_DISCARD = 3, TNT_TRUNC_SPACE = 4 };

typedef struct tnt_rule_s tnt_rule;
typedef struct tnt_space_s tnt_space;
typedef struct tnt_xplan_s tnt_xplan;
typedef struct tnt_cplan_s tnt_cplan;
typedef struct tnt_fplan_s tnt_fplan;
typedef struct tnt_ctx_s tnt_ctx;

/* Last error message of the calling thread (empty after success). */
tnt_status tnt_last_error(char* buf, size_t len);

/* Library version, e.g. "0.1.0"; never fails. */
const char* tnt_version(void);

/* ---- fusion rules (tenet-sectors/src/product_rule.rs:80-140) ------------ */
/* A product of `nfactors` factors (TNT_U1/SU2/FZ2/Z2), first factor first.  */
tnt_status tnt_rule_create(int32_t nfactors, const int32_t* kinds, int32_t codec, tnt_rule** out);
/* A fusion rule given by a checked table provider (the reference's checked
 * Generic providers, tenet-sectors/src/algebra.rs:743-910, and the transform
 * path they feed, tenet-tensors/src/tree_context.rs:38-110,
 * tree_transform/plan.rs:250-330), restricted to multiplicity-free rules with
 * real, symmetric braiding.  Sectors are labels 0 .. n-1 (0 the vacuum; one
 * int32 per label, SectorId = label).  Tables, row-major: dual[n],
 * nsym[n^3] (N(a,b,c) in {0,1}), dims[n], fs[n], rsym[n^3] (R(a,b,c)),
 * fsym[n^6] (F(a,b,c;d;e,f): the coefficient of a (x) (b (x) c -> f) -> d in
 * (a (x) b -> e) (x) c -> d).  Before the rule exists the tables are checked
 * to `tol`: vacuum and dual laws, no outer multiplicity, d_a d_b =
 * sum_c N d_c, orthogonal F blocks, the pentagon, R(a,b,c) R(b,a,c) = 1, the
 * hexagon and fs_a = d_a F(a,a,a;a;0,0); the first broken law is returned as
 * TNT_INVALID_ARGUMENT.  n <= 16. */
tnt_status tnt_rule_create_table(int32_t n, const int32_t* dual, const uint8_t* nsym, const double* dims,
                                 const double* fs, const double* rsym, const double* fsym, double tol,
                                 tnt_rule** out);
void tnt_rule_destroy(tnt_rule* rule);
/* SectorId of one label (nfactors ints: U1 charge, SU2 2j, parity). */
tnt_status tnt_rule_sector_id(const tnt_rule* rule, const int32_t* label, uint64_t* id);
/* F(a,b,c;d;e,f), R(a,b;c), quantum dimension, twist, Frobenius-Schur phase
 * (tenet-sectors/src/algebra.rs:552-623). */
tnt_status tnt_rule_fsymbol(const tnt_rule* rule, const int32_t* abcdef, double* value);
tnt_status tnt_rule_rsymbol(const tnt_rule* rule, const int32_t* abc, double* value);
tnt_status tnt_rule_dim(const tnt_rule* rule, const int32_t* label, double* dim);

/* ---- hom spaces: GradedSpace legs -> BlockStructure --------------------- */
/* Legs are listed codomain first.  Leg i has leg_nsectors[i] sectors whose
 * labels (nfactors ints each, already dualized for a dual leg) and
 * degeneracies follow consecutively in leg_labels / leg_degeneracies; its
 * dual flag is leg_is_dual[i] (tenet-core/src/sector.rs:147-237). */
tnt_status tnt_space_create(const tnt_rule* rule, int32_t n_codomain, int32_t n_domain,
                            const int32_t* leg_nsectors, const int32_t* leg_labels,
                            const int64_t* leg_degeneracies, const uint8_t* leg_is_dual, tnt_space** out);
void tnt_space_destroy(tnt_space* space);
tnt_status tnt_space_info(const tnt_space* space, int64_t* size, int32_t* nsectors, int32_t* nblocks,
                          int32_t* n_codomain, int32_t* n_domain);
/* Coupled sectors in storage order: labels (nsectors*nfactors), rows, cols, offsets. */
tnt_status tnt_space_sectors(const tnt_space* space, int32_t* labels, int64_t* rows, int64_t* cols,
                             int64_t* offsets);
/* Blocks in storage order: offsets, shapes/strides (nblocks*rank), sector index. */
tnt_status tnt_space_blocks(const tnt_space* space, int64_t* offsets, int64_t* shapes, int64_t* strides,
                            int32_t* sector_index);
/* Block keys as int32 records: per block, per tree (codomain then domain):
 * rank, uncoupled labels, dual flags, coupled label, inner labels
 * (FusionTreeKey fields, tenet-core/src/fusion_tree.rs:1225).  Pass
 * keys == NULL to query the length. */
tnt_status tnt_space_block_keys(const tnt_space* space, int32_t* keys, int64_t capacity, int64_t* length);
/* One leg of a space: axis counts codomain first. */
tnt_status tnt_space_leg(const tnt_space* space, int32_t axis, int32_t* nsectors, int32_t* labels,
                         int64_t* degeneracies, uint8_t* is_dual);

/* ---- recoupling plans (TreeTransformStructure, transform_structure.rs:587-770) */
/* TensorMap::permute (tenet/src/typed.rs:13163). */
tnt_status tnt_permute_plan(const tnt_space* src, int32_t n_codomain, const int32_t* codomain_axes,
                            int32_t n_domain, const int32_t* domain_axes, tnt_xplan** out);
/* TensorMap::braid with one level per source axis (typed.rs:13204). */
tnt_status tnt_braid_plan(const tnt_space* src, int32_t n_codomain, const int32_t* codomain_axes,
                          int32_t n_domain, const int32_t* domain_axes, const int32_t* levels, tnt_xplan** out);
/* TensorMap::repartition (typed.rs:13250). */
tnt_status tnt_repartition_plan(const tnt_space* src, int32_t n_codomain, tnt_xplan** out);
/* TensorMap::adjoint materialised: codomain and domain swap, every block is
 * transposed (block(t', c) = block(t, c)^T; tenet-tensors/src/adjoint.rs). */
tnt_status tnt_adjoint_plan(const tnt_space* src, tnt_xplan** out);
/* TensorMap::twist / twist_inverse (typed.rs:4599-4606): every block times
 * the product of the ribbon twists of its uncoupled sectors on `legs` (flat
 * axes, codomain first).  The twists in scope are +-1, so `inverse` changes
 * nothing; the destination space equals the source space. */
tnt_status tnt_twist_plan(const tnt_space* src, int32_t n_legs, const int32_t* legs, int32_t inverse,
                          tnt_xplan** out);
/* Right operand of TensorMap::contract (typed.rs:13653): permute to
 * (contracted_axes ; open_axes) with the fermionic supertrace twist of each
 * dual contracted leg folded into the coefficients
 * (tenet-tensors/src/contract/dynamic.rs:330-390, 2697-2760).  Equal to
 * tnt_permute_plan for bosonic rules. */
tnt_status tnt_contract_rhs_plan(const tnt_space* src, int32_t n_contracted, const int32_t* contracted_axes,
                                 int32_t n_open, const int32_t* open_axes, tnt_xplan** out);
/* Several recoupling steps fused into one transform (one read and one write
 * of the payload): the coefficients of each source tree pair are multiplied
 * through every step.  `program` holds, per step, a kind and its arguments:
 *   0 permute: n_codomain, codomain[...], n_domain, domain[...]
 *   1 braid:   n_codomain, codomain[...], n_domain, domain[...], levels[rank]
 *   2 repartition: n_codomain
 *   3 adjoint
 *   4 twist:   n_legs, legs[...]
 * each on the space the previous step produced (typed.rs:4599, 13163-13250). */
tnt_status tnt_transform_chain_plan(const tnt_space* src, int32_t nsteps, const int32_t* program, int64_t len,
                                    tnt_xplan** out);
void tnt_xplan_destroy(tnt_xplan* plan);
/* The destination space (new handle, owned by the caller). */
tnt_status tnt_xplan_dst_space(const tnt_xplan* plan, tnt_space** out);
/* groups, total coefficient count, algorithmic bytes moved per replay. */
tnt_status tnt_xplan_info(const tnt_xplan* plan, int64_t* ngroups, int64_t* ncoef, int64_t* bytes_moved);
/* Export the compiled tables (for inspection and host replay in tests).
 * groups: 6 + 8 int64 per group (nelem, nsrc, ndst, src_first, dst_first,
 * coef_off, dims[8]); src/dst entries: 9 int64 each (offset, strides[8]);
 * coef: ncoef doubles.  Sizes come from tnt_xplan_info / tnt_xplan_entries. */
tnt_status tnt_xplan_entries(const tnt_xplan* plan, int64_t* nsrc_entries, int64_t* ndst_entries);
/* A transform plan from tables compiled elsewhere, in the tnt_xplan_export
 * layout: the reference's TreeTransformStructure (transform_structure.rs:
 * 82-95, 807-811) lowered to groups of same-shape blocks with a row-major
 * U[dst, src] coefficient matrix each; source strides are listed in
 * destination axis order.  Every group has `rank` axes.  Checked: entry and
 * coefficient ranges, block extents 1..65535, blocks inside their payloads,
 * and every destination element written by exactly one group.  The plan has
 * no spaces (tnt_xplan_dst_space fails on it). */
tnt_status tnt_xplan_from_tables(int32_t rank, int64_t ngroups, const int64_t* groups, int64_t nsrc_entries,
                                 const int64_t* src_entries, int64_t ndst_entries, const int64_t* dst_entries,
                                 int64_t ncoef, const double* coef, int64_t src_size, int64_t dst_size,
                                 tnt_xplan** out);
tnt_status tnt_xplan_export(const tnt_xplan* plan, int64_t* groups, int64_t* src_entries, int64_t* dst_entries,
                            double* coef);

/* ---- compose plans (FusionBlockContractPlan, fusion_replay.rs:216-530) --- */
tnt_status tnt_compose_plan(const tnt_space* lhs, const tnt_space* rhs, tnt_cplan** out);
void tnt_cplan_destroy(tnt_cplan* plan);
tnt_status tnt_cplan_dst_space(const tnt_cplan* plan, tnt_space** out);
/* jobs (coupled sectors) and 2*m*n*k flops per compose. */
tnt_status tnt_cplan_info(const tnt_cplan* plan, int64_t* njobs, double* flops);
/* Export the job table: 9 int64 per job (m, n, k, a_off, b_off, c_off, lda, ldb, ldc). */
tnt_status tnt_cplan_export(const tnt_cplan* plan, int64_t* jobs);
/* Table-driven seam: a GEMM batch compiled elsewhere (Rank2GemmBatchJob
 * records: m, n, k, a_off, b_off, c_off, lda, ldb, ldc; 9 int64 per job). */
tnt_status tnt_cplan_from_jobs(int64_t njobs, const int64_t* jobs, int64_t a_size, int64_t b_size,
                               int64_t c_size, tnt_cplan** out);

/* ---- factorisation plans (per coupled sector) --------------------------- */
tnt_status tnt_factor_plan(const tnt_space* src, tnt_fplan** out);
void tnt_fplan_destroy(tnt_fplan* plan);
/* Flat sizes of U, S and Vh for a compact SVD of every sector. */
tnt_status tnt_fplan_info(const tnt_fplan* plan, int32_t* nsectors, int64_t* u_size, int64_t* s_size,
                          int64_t* v_size);
/* Export the per-sector records: 8 int64 each (m, n, k, a_off, u_off, s_off, v_off, 0) plus weights. */
tnt_status tnt_fplan_export(const tnt_fplan* plan, int64_t* records, double* weights);

/* ---- device execution ----------------------------------------------------- */
tnt_status tnt_ctx_create(int32_t device, tnt_ctx** out);
void tnt_ctx_destroy(tnt_ctx* ctx);

/* dst = alpha * T(src) + beta * dst  (replay_backend.rs:28-79). */
tnt_status tnt_transform(tnt_ctx* ctx, const tnt_xplan* plan, double* dst, const double* src, double alpha,
                         double beta, void* stream);

/* dst = alpha * (lhs o rhs) + beta * dst, one GEMM per coupled sector, for
 * `nbatch` operand triples stored back to back (element strides
 * stride_dst/lhs/rhs).  precision: TNT_PREC_FP64 (FP64 tensor-core grouped
 * kernel), TNT_PREC_BF16X (split-precision: `slices` BF16 slices per
 * operand, FP32 tensor-core accumulation, FP64 recombination) or
 * TNT_PREC_INT8X (`slices` signed 7-bit digits per operand in int8, exact
 * int32 accumulation per product diagonal, FP64 recombination), or
 * TNT_PREC_CUBLAS_FP64 (one cuBLAS DGEMM per sector: the reference's own
 * device route, typed.rs:11438-11480, kept as the comparison baseline). */
tnt_status tnt_compose(tnt_ctx* ctx, const tnt_cplan* plan, int64_t nbatch, double* dst, int64_t stride_dst,
                       const double* lhs, int64_t stride_lhs, const double* rhs, int64_t stride_rhs,
                       double alpha, double beta, int32_t precision, int32_t slices, void* stream);

/* Device scratch a split-precision compose of this plan needs (bytes; 0 for
 * the FP64 precisions), an upper bound over the tile widths the autotuner
 * may pick. */
tnt_status tnt_cplan_scratch_bytes(const tnt_cplan* plan, int64_t nbatch, int32_t precision, int32_t slices,
                                   size_t* bytes);
/* tnt_compose with the slice packs in a caller-provided device buffer of at
 * least tnt_cplan_scratch_bytes bytes (no allocation in the context), for
 * callers that account device memory themselves; it takes the tile width
 * from the device's current autotuner state without timing anything. */
tnt_status tnt_compose_ws(tnt_ctx* ctx, const tnt_cplan* plan, int64_t nbatch, double* dst, int64_t stride_dst,
                          const double* lhs, int64_t stride_lhs, const double* rhs, int64_t stride_rhs, double alpha,
                          double beta, int32_t precision, int32_t slices, void* scratch, size_t scratch_bytes,
                          void* stream);

/* Constant operands packed once (no counterpart in the reference, whose
 * compose is plain FP64): in an iterative solver one operand of a compose is
 * often the same on every call (the environments and the MPO tensor of an
 * effective Hamiltonian across Lanczos iterations), so its 8-bit digit packs
 * and scales can be made once.  tnt_split_operand_bytes gives the size of one
 * packed side (0: the left operand, 1: the right) of `plan` at `slices`
 * digits; tnt_split_pack_operand writes it into caller memory;
 * tnt_compose_packed runs one compose (no batch) with either side taken from
 * such a buffer (pass the packed pointer and NULL for the plain one, or the
 * plain pointer and NULL).  TNT_PREC_INT8X only; the result is bit-identical
 * to tnt_compose on the same operands. */
tnt_status tnt_split_operand_bytes(const tnt_cplan* plan, int32_t side, int32_t precision, int32_t slices,
                                   size_t* bytes);
tnt_status tnt_split_pack_operand(tnt_ctx* ctx, const tnt_cplan* plan, int32_t side, const double* operand,
                                  int32_t precision, int32_t slices, void* packed, size_t packed_bytes, void* stream);
tnt_status tnt_compose_packed(tnt_ctx* ctx, const tnt_cplan* plan, double* dst, const double* lhs,
                              const void* lhs_packed, const double* rhs, const void* rhs_packed, double alpha,
                              double beta, int32_t precision, int32_t slices, void* stream);

/* Tile-shape autotuning of tnt_compose.  FP64: every coupled-sector job gets
 * one output-tile shape (0: 64x64, 1: 64x32, 2: 32x64, 3: 32x32) minimising
 * ntiles * (ceil(k/16) + 1) * cost[shape]; split precision: tile width 64 or
 * 128 from the per-MAC throughput ratio eff64.  The per-device costs are
 * measured on the first compose with beta == 0, at least 2e8 flops and no
 * stream capture in progress (it times each candidate on the caller's own
 * operands, so make that call before any capture); TNT_AUTOTUNE=0 keeps the
 * model defaults.  No counterpart in the reference (per-sector GEMM calls).
 * tnt_cplan_tile_shapes: the per-job shapes for the given four costs;
 * tnt_tuning_info: the device's current costs and calibration state. */
tnt_status tnt_cplan_tile_shapes(const tnt_cplan* plan, const double* costs, int32_t* shapes);
tnt_status tnt_tuning_info(int32_t device, double* f64_costs, int32_t* f64_calibrated, double* split_eff64,
                           int32_t* split_calibrated);

/* Same as tnt_compose with HOST buffers: copies operands in, computes, copies
 * the result out, synchronising `stream` before returning.  A batch runs as a
 * pipeline of up to 8 chunks on two context-owned copy streams, so copies in,
 * composes and copies out overlap (full overlap needs pinned host buffers). */
tnt_status tnt_compose_host(tnt_ctx* ctx, const tnt_cplan* plan, int64_t nbatch, double* dst_host,
                            const double* lhs_host, const double* rhs_host, int32_t precision, int32_t slices,
                            void* stream);

/* Compact SVD of every coupled sector: u (m x k), s (k), vh (k x n) per
 * sector at the offsets of tnt_fplan_info, largest-|U| column gauge
 * (factorize.rs:3836-3852). */
tnt_status tnt_svd(tnt_ctx* ctx, const tnt_fplan* plan, const double* a, double* u, double* s, double* vh,
                   void* stream);

/* tnt_svd without any device allocation, for callers that cannot allocate
 * device memory at the point of use: a serving loop that admits work against
 * a fixed device-memory budget, or a foreign host whose own allocator owns
 * every device byte.  No counterpart in the reference (its factorisations
 * always allocate their outputs and workspaces).  Scratch lives in a
 * library-owned static device array of 8 MiB per device (held until process
 * exit); plans needing more are rejected with TNT_INVALID_ARGUMENT.  Runs on
 * the calling thread's current device and synchronises `stream`.  Calls that
 * overlap on one device share that array and race: serialise them.  The
 * first call on a device looks the array up, and (CUDA loading the module
 * lazily) is when its 8 MiB are committed on that device: make it at set-up,
 * before a device-memory budget is fixed and before any stream capture
 * begins.  Every sector runs on one CTA, largest first; tnt_svd's
 * thread-block clusters for sectors of many column blocks are not used, so
 * sectors of several hundred rows run several times slower than through
 * tnt_svd. */
tnt_status tnt_svd_static(const tnt_fplan* plan, const double* a, double* u, double* s, double* vh, void* stream);

/* Compact QR of every coupled sector (qr_compact, factorize.rs:5158): q
 * (m x k) at the plan's U offsets, r (k x n, upper trapezoidal) at its Vh
 * offsets, k = min(m, n); positive-diagonal gauge (R_jj >= 0,
 * positive_diagonal_gauge, factorize.rs:3789-3830).  Synchronises `stream`. */
tnt_status tnt_qr(tnt_ctx* ctx, const tnt_fplan* plan, const double* a, double* q, double* r, void* stream);
/* Real symmetric eigendecomposition of every coupled sector of an
 * endomorphism (eigh_full, factorize.rs:3041-3150): eigenvalues (signed) at
 * the plan's S offsets, stable-sorted by descending |lambda|; eigenvectors
 * (n x n, columns) at its U offsets with each vector's largest-|.| entry
 * positive.  mags (nullable, S layout) receives |lambda| for tnt_truncate.
 * Non-Hermitian blocks (||A - A^T||_F > 128 eps ||A||_F) return
 * TNT_INVALID_ARGUMENT.  Plans whose sectors all fit in shared memory (n up
 * to 111) run a two-sided Jacobi per sector; a plan with a larger sector runs
 * every sector through the batched SVD of A + ||A||_F I (positive
 * semidefinite: singular values lambda + ||A||_F, right singular vectors the
 * eigenvectors), with absolute eigenvalue error about eps (||A||_2 +
 * ||A||_F), and grows a context scratch of the plan's A, U, S and Vh sizes
 * on first use.  Synchronises `stream`. */
tnt_status tnt_eigh(tnt_ctx* ctx, const tnt_fplan* plan, const double* a, double* vecs, double* vals, double* mags,
                    void* stream);

/* Synchronise `stream` and report device-side failures since the last call:
 * TNT_DEVICE_TIMEOUT when a bounded pipeline wait of the split-precision
 * kernel gave up (the compose results of that launch are invalid; the
 * context stays usable).  Kernels never trap or hang on such a failure. */
tnt_status tnt_ctx_sync(tnt_ctx* ctx, void* stream);
/* Jacobi sweeps the slowest sector of the last tnt_svd / tnt_svd_ws on this
 * context needed (diagnostic). */
tnt_status tnt_ctx_svd_sweeps(const tnt_ctx* ctx, int32_t* sweeps);
/* Doubles of SVD workspace a plan needs (tnt_svd_ws). */
tnt_status tnt_fplan_work(const tnt_fplan* plan, int64_t* work_elems);
/* tnt_svd with a caller-provided device workspace of tnt_fplan_work doubles
 * (the workspace offsets of a concatenated plan are relative to `work`). */
tnt_status tnt_svd_ws(tnt_ctx* ctx, const tnt_fplan* plan, const double* a, double* u, double* s, double* vh,
                      double* work, void* stream);

/* tnt_svd_ws without any host synchronisation, for callers that keep several
 * streams busy (the serving loop's lanes): status (2 int32, device memory)
 * receives [0] non-zero if a sector did not converge within the sweep limit
 * and [1] the Jacobi sweeps of the slowest sector; read it once the stream
 * has passed this call. */
tnt_status tnt_svd_ws_async(tnt_ctx* ctx, const tnt_fplan* plan, const double* a, double* u, double* s, double* vh,
                            double* work, int32_t* status, void* stream);

/* Cross-sector truncation chosen on the device (select_truncation,
 * truncation.rs:257-560).  `s` are the device singular values of tnt_svd;
 * kept (nsectors int64, device memory) and err (1 double, device memory)
 * are written.  policy: TNT_TRUNC_*; p0/p1: rank budget or atol/rtol;
 * space_ranks: per-sector ranks (host array, TNT_TRUNC_SPACE only). */
tnt_status tnt_truncate(tnt_ctx* ctx, const tnt_fplan* plan, const double* s, int32_t policy, double p0,
                        double p1, const int64_t* space_ranks, int64_t* kept, double* err, void* stream);
/* tnt_truncate with space_ranks in device memory (int64 per sector) and no
 * host synchronisation. */
tnt_status tnt_truncate_async(tnt_ctx* ctx, const tnt_fplan* plan, const double* s, int32_t policy, double p0,
                              double p1, const int64_t* space_ranks, int64_t* kept, double* err, void* stream);

/* ---- grouped launches across many tensors -------------------------------- */
/* One plan running n plans in a single launch over shared arenas: the
 * operands of plan i sit at element offsets src/dst (transform), a/b/c
 * (compose) or a/u/s/v (factorisation) of the arena pointers passed at
 * execution.  Lets a scheduler batch uneven tensors of many independent
 * simulations into one grouped kernel.  For factorisations, w_offs (may be
 * NULL) places each plan's SVD workspace in the caller's buffer for
 * tnt_svd_ws. */
tnt_status tnt_xplan_concat(int32_t n, const tnt_xplan* const* plans, const int64_t* src_offs,
                            const int64_t* dst_offs, tnt_xplan** out);
tnt_status tnt_cplan_concat(int32_t n, const tnt_cplan* const* plans, const int64_t* a_offs, const int64_t* b_offs,
                            const int64_t* c_offs, tnt_cplan** out);
tnt_status tnt_fplan_concat(int32_t n, const tnt_fplan* const* plans, const int64_t* a_offs, const int64_t* u_offs,
                            const int64_t* s_offs, const int64_t* v_offs, const int64_t* w_offs, tnt_fplan** out);
/* Truncation of a concatenated factorisation, independently per segment:
 * segment i owns sectors [seg_first[i], seg_first[i+1]) (seg_first has nseg+1
 * host entries); space_ranks (host, one per sector, TNT_TRUNC_SPACE) as in
 * tnt_truncate; kept (per sector) and err (per segment) are device memory. */
tnt_status tnt_truncate_segments(tnt_ctx* ctx, const tnt_fplan* plan, int32_t nseg, const int32_t* seg_first,
                                 const double* s, int32_t policy, double p0, double p1, const int64_t* space_ranks,
                                 int64_t* kept, double* err, void* stream);

/* Copy nseg column-major blocks in one launch.  table holds 7 int64 per
 * block (host memory): src_off, dst_off, rows, cols, src_ld, dst_ld,
 * scale_off; row i is multiplied by scales[scale_off + i] when scale_off >= 0
 * (publishes S Vh of a truncated SVD).  The table travels through the
 * context's staging buffer in stream order: use one stream per context. */
tnt_status tnt_copy_segments(tnt_ctx* ctx, int64_t nseg, const int64_t* table, const double* src, double* dst,
                             const double* scales, void* stream);
/* tnt_copy_segments with the table (7 int64 per segment, same fields) in
 * device memory and no host synchronisation.  The offsets are not checked:
 * the caller builds them inside its buffers. */
tnt_status tnt_copy_segments_async(tnt_ctx* ctx, int64_t nseg, const int64_t* table, const double* src, double* dst,
                                   const double* scales, void* stream);

/* ---- FP64 Krylov building blocks (Lanczos on the device) ---------------- */
/* out[j] = <V_j, y> for j < k, the quantum-dimension-weighted inner product
 * sum_c d_c tr(V_j,c^T y_c) over the coupled sectors of the plan's space;
 * V_j = V + j * ldv.  out is device memory.  k <= 64.  (The reference's
 * KrylovVector inner product, tenet-krylov/src/vector.rs.) */
tnt_status tnt_wdot(tnt_ctx* ctx, const tnt_fplan* plan, int32_t k, const double* V, int64_t ldv, const double* y,
                    double* out, void* stream);
/* y = a * y + sum_j coef[j] V_j over n elements; coef is device memory; if
 * a_dev is non-NULL the scale is read from the device instead of `a`. */
tnt_status tnt_axpy_many(tnt_ctx* ctx, int64_t n, int32_t k, const double* V, int64_t ldv, const double* coef,
                         double a, const double* a_dev, double* y, void* stream);
/* Eigen-decomposition of a symmetric m x m matrix (m <= 48, device,
 * column-major): ascending eigenvalues and eigenvector columns; synchronises
 * `stream`. */
tnt_status tnt_symeig(tnt_ctx* ctx, int32_t m, const double* A, double* evals, double* evecs, void* stream);

/* ---- network schedules (tenet-network/src/network.rs:919-941, 1467-1560) ----
 * A pairwise contraction schedule lowered to device work.  Slots
 * 0..n_inputs-1 hold the inputs (their adjoint where conj[i] != 0); step s
 * contracts two live slots (TensorMap::contract semantics, supertrace twist
 * included) into result_slot, then applies its optional result permutation.
 * `steps` is a flat int32 program, per step:
 *   lhs_slot, rhs_slot, result_slot,
 *   k, lhs_axes[k], rhs_axes[k],
 *   n_out, contract_output_axes[n_out],
 *   n_codomain (-1: no result permutation), codomain[n_codomain], n_domain, domain[n_domain]
 * final_perm (length 0: none): n_codomain, codomain[...], n_domain, domain[...].
 * Every transform an operand needs before its compose (adjoint, pending
 * output permutations, the contraction permute and twist) is fused into one
 * recoupling pass; intermediates live in a caller-provided workspace. */
typedef struct tnt_nplan_s tnt_nplan;
tnt_status tnt_network_plan(int32_t n_inputs, const tnt_space* const* inputs, const uint8_t* conj, int32_t n_steps,
                            const int32_t* steps, int64_t steps_len, int32_t final_slot, const int32_t* final_perm,
                            int64_t final_perm_len, tnt_nplan** out);
void tnt_nplan_destroy(tnt_nplan* plan);
/* The space of the network's result (new handle, owned by the caller). */
tnt_status tnt_nplan_output_space(const tnt_nplan* plan, tnt_space** out);
/* Fused transforms and composes per execution, compose flops, transform
 * bytes moved and workspace elements for intermediates. */
tnt_status tnt_nplan_info(const tnt_nplan* plan, int64_t* n_transforms, int64_t* n_composes, double* flops,
                          int64_t* bytes_moved, int64_t* workspace_elems);
/* Workspace bytes tnt_network_execute needs at this compose precision. */
tnt_status tnt_nplan_workspace_bytes(const tnt_nplan* plan, int32_t precision, int32_t slices, size_t* bytes);
/* Run the schedule on `stream`: inputs[i] hold the payloads of the planned
 * input spaces (read only), output receives the result and must not overlap
 * an input or the workspace.  No device allocation; capturable in a CUDA
 * graph after the first call at the same precision. */
tnt_status tnt_network_execute(tnt_ctx* ctx, const tnt_nplan* plan, int32_t n_inputs, const double* const* inputs,
                               double* output, void* workspace, size_t workspace_bytes, int32_t precision,
                               int32_t slices, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TENET_B200_H */
