// extern "C" boundary of libtenet_b200 (declared in include/tenet_b200.h).
#include "tenet_b200.h"

#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "autotune.hpp"
#include "host.hpp"
#include "kernels.cuh"

using namespace tnt;

namespace {

thread_local std::string g_error;

struct Failure : std::runtime_error {
  tnt_status code;
  Failure(tnt_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    tnt_status code = e == cudaErrorMemoryAllocation ? TNT_OUT_OF_MEMORY : TNT_CUDA_ERROR;
    throw Failure(code, std::string(what) + ": " + cudaGetErrorString(e));
  }
}

template <class F>
tnt_status guarded(F&& f) {
  try {
    f();
    g_error.clear();
    return TNT_OK;
  } catch (const Failure& e) {
    g_error = e.what();
    return e.code;
  } catch (const std::invalid_argument& e) {
    g_error = e.what();
    return TNT_INVALID_ARGUMENT;
  } catch (const std::bad_alloc&) {
    g_error = "host allocation failed";
    return TNT_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    g_error = e.what();
    return TNT_INTERNAL;
  }
}

void need(bool ok, const char* msg) {
  if (!ok) throw std::invalid_argument(msg);
}

template <class T>
T* upload(const std::vector<T>& v) {
  if (v.empty()) return nullptr;
  T* d = nullptr;
  cuda_check(cudaMalloc(&d, v.size() * sizeof(T)), "cudaMalloc(plan table)");
  cuda_check(cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "upload plan table");
  return d;
}

int current_device() {
  int d = -1;
  cuda_check(cudaGetDevice(&d), "cudaGetDevice");
  return d;
}

}  // namespace

struct tnt_rule_s {
  Rule r;
};

struct tnt_space_s {
  std::shared_ptr<Space> s;
};

struct tnt_ctx_s {
  int device = 0;
  void* split_buf = nullptr;  // split-precision slice packs (grow-only)
  size_t split_bytes = 0;
  SegCopy* seg_stage = nullptr;  // copy-segment tables
  size_t seg_stage_elems = 0;
  double* dot_part = nullptr;  // partial sums of weighted dots
  size_t dot_part_elems = 0;
  cublasHandle_t cublas = nullptr;
  // Recursive: host-buffer entry points hold it across the device-buffer
  // entry point they call, which takes it again for its own scratch.
  std::recursive_mutex mu;
  double* stage = nullptr;  // device staging for host-buffer entry points
  size_t stage_elems = 0;
  double* svd_work = nullptr;
  size_t svd_work_elems = 0;
  double* eigh_tmp = nullptr;  // eigh of large sectors: shifted copy, SVD outputs, shifts, flag
  size_t eigh_tmp_elems = 0;
  int32_t* status = nullptr;  // device: [0] error flags, [1] Jacobi sweeps of the last SVD,
                              // [2] split-kernel pipeline timeouts since the last tnt_ctx_sync
  int32_t last_sweeps = 0;     // host copy of status[1] after each tnt_svd / tnt_svd_ws
  // tnt_compose_host pipeline: copy-in and copy-out streams and per-chunk events
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  std::vector<cudaEvent_t> chunk_events;
  // Ordering of the shared scratch across streams: the last stream whose
  // work used it, and an event recorded after that work.
  cudaEvent_t scratch_done = nullptr;
  cudaStream_t scratch_user = nullptr;
  bool scratch_user_valid = false;
};

struct tnt_xplan_s {
  std::shared_ptr<TransformPlan> p;
  std::mutex mu;
  std::map<int, DevXform> dev;
  ~tnt_xplan_s() {
    for (auto& kv : dev) {
      int prev = -1;
      cudaGetDevice(&prev);
      cudaSetDevice(kv.first);
      cudaFree(kv.second.groups);
      cudaFree(kv.second.src);
      cudaFree(kv.second.dst);
      cudaFree(kv.second.coef);
      cudaFree(kv.second.tiles);
      if (prev >= 0) cudaSetDevice(prev);
    }
  }
  const DevXform& on_device() {
    int d = current_device();
    std::lock_guard<std::mutex> g(mu);
    auto it = dev.find(d);
    if (it != dev.end()) return it->second;
    const XformTables& t = p->tables;
    DevXform x;
    x.groups = upload(t.groups);
    x.src = upload(t.src_entries);
    x.dst = upload(t.dst_entries);
    x.coef = upload(t.coef);
    // One launch per kernel path: tiles grouped by kind (stable within a kind).
    std::vector<XTile> tiles(t.tiles);
    std::stable_sort(tiles.begin(), tiles.end(), [](const XTile& a, const XTile& b) { return a.kind < b.kind; });
    for (const XTile& tl : tiles) x.kind_count[tl.kind] += 1;
    for (int k = 1; k < kXKinds; ++k) x.kind_begin[k] = x.kind_begin[k - 1] + x.kind_count[k - 1];
    x.tiles = upload(tiles);
    x.ntiles = (int32_t)tiles.size();
    x.max_nsrc = t.max_nsrc;
    x.max_ndst = t.max_ndst;
    return dev.emplace(d, x).first->second;
  }
};

struct CplanDevice {
  GemmJob* jobs = nullptr;
  std::map<int64_t, std::pair<GemmTile*, int32_t>> f64_tiles;    // per nbatch
  std::map<int64_t, std::pair<GemmTile*, int32_t>> split_tiles;  // per nbatch and tile width
  std::map<int64_t, void*> split_jobs;                             // per slice count and tile width
};

struct tnt_cplan_s {
  std::shared_ptr<ComposePlan> p;
  std::mutex mu;
  std::map<int, CplanDevice> dev;
  ~tnt_cplan_s() {
    for (auto& kv : dev) {
      int prev = -1;
      cudaGetDevice(&prev);
      cudaSetDevice(kv.first);
      cudaFree(kv.second.jobs);
      for (auto& t : kv.second.f64_tiles) cudaFree(t.second.first);
      for (auto& t : kv.second.split_tiles) cudaFree(t.second.first);
      for (auto& t : kv.second.split_jobs) cudaFree(t.second);
      if (prev >= 0) cudaSetDevice(prev);
    }
  }
  // Tiles of every (job, batch entry) output tile, longest K first; each
  // carries its job's K.
  std::vector<GemmTile> make_tiles(int64_t nbatch, int tm, int tn) const {
    std::vector<std::pair<int64_t, GemmTile>> v;
    const auto& jobs = p->tables.jobs;
    for (int64_t b = 0; b < nbatch; ++b)
      for (size_t j = 0; j < jobs.size(); ++j) {
        const GemmJob& J = jobs[j];
        int64_t mt = (J.m + tm - 1) / tm, nt = (J.n + tn - 1) / tn;
        for (int64_t x = 0; x < mt; ++x)
          for (int64_t y = 0; y < nt; ++y)
            v.push_back({J.k, GemmTile{(int32_t)j, (int32_t)b, (int32_t)x, (int32_t)y, 0, (int32_t)J.k}});
      }
    std::stable_sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    std::vector<GemmTile> out;
    out.reserve(v.size());
    for (auto& x : v) out.push_back(x.second);
    return out;
  }
  CplanDevice& on_device(int d) {
    auto it = dev.find(d);
    if (it != dev.end()) return it->second;
    CplanDevice c;
    c.jobs = upload(p->tables.jobs);
    return dev.emplace(d, c).first->second;
  }
  GemmJob* jobs_dev() {
    int d = current_device();
    std::lock_guard<std::mutex> g(mu);
    return on_device(d).jobs;
  }
};

struct FplanChunks {
  int64_t* sector = nullptr;
  int64_t* start = nullptr;
  int64_t n = 0;
};

struct tnt_fplan_s {
  std::shared_ptr<FactorPlan> p;
  std::mutex mu;
  std::map<int, std::pair<SvdJob*, int64_t*>> dev;  // jobs, work offsets (sector order)
  std::map<int, std::pair<SvdJob*, int64_t*>> lpt;  // the same, cluster jobs then largest first
  int32_t n_cluster = 0;                            // leading jobs of the lpt tables run on clusters
  int32_t n_wide = 0;                               // ... the first n_wide of them on 16-CTA clusters
  std::map<int, FplanChunks> chunks;                // weighted-dot chunk tables
  int64_t work_elems = 0;
  std::vector<int64_t> work_off;
  ~tnt_fplan_s() {
    for (auto& kv : dev) {
      int prev = -1;
      cudaGetDevice(&prev);
      cudaSetDevice(kv.first);
      cudaFree(kv.second.first);
      cudaFree(kv.second.second);
      auto lt = lpt.find(kv.first);
      if (lt != lpt.end()) {
        cudaFree(lt->second.first);
        cudaFree(lt->second.second);
      }
      auto it = chunks.find(kv.first);
      if (it != chunks.end()) {
        cudaFree(it->second.sector);
        cudaFree(it->second.start);
      }
      if (prev >= 0) cudaSetDevice(prev);
    }
  }
  FplanChunks chunks_on_device() {
    int d = current_device();
    std::lock_guard<std::mutex> g(mu);
    auto it = chunks.find(d);
    if (it != chunks.end()) return it->second;
    std::vector<int64_t> sec, st;
    FplanChunks c;
    c.n = wdot_chunks(p->tables.jobs.data(), (int32_t)p->tables.jobs.size(), sec, st);
    c.sector = upload(sec);
    c.start = upload(st);
    chunks.emplace(d, c);
    return c;
  }
  std::pair<SvdJob*, int64_t*> on_device() {
    int d = current_device();
    std::lock_guard<std::mutex> g(mu);
    auto it = dev.find(d);
    if (it != dev.end()) return it->second;
    auto r = std::make_pair(upload(p->tables.jobs), upload(work_off));
    dev.emplace(d, r);
    return r;
  }
  // Job and work-offset tables ordered longest-first (rows * k^2 descending)
  // for the one-CTA-per-sector factorisation kernels: each job carries its
  // own output offsets, so the order only changes which CTA starts first,
  // and the largest sectors no longer start in the last wave.
  std::pair<SvdJob*, int64_t*> lpt_on_device() {
    on_device();  // sector-order tables first (needed by truncation and dots)
    int d = current_device();
    std::lock_guard<std::mutex> g(mu);
    auto it = lpt.find(d);
    if (it != lpt.end()) return it->second;
    const auto& jobs = p->tables.jobs;
    std::vector<size_t> order(jobs.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    auto cost = [&](size_t i) {
      const double r = (double)std::max(jobs[i].m, jobs[i].n), k = (double)jobs[i].k;
      return r * k * k;
    };
    // Sectors whose blocked Jacobi has at least one column block per cluster
    // CTA run on a thread-block cluster (svd_cluster_kernel); they go first,
    // those with a block for each of 16 CTAs (where the device allows such
    // clusters) ahead of the 8-CTA ones.
    const int wide = svd_wide_cluster_size();
    auto clustered = [&](size_t i) {
      const int64_t rows = std::max(jobs[i].m, jobs[i].n), k = jobs[i].k;
      if (svd_on_chip(rows, k)) return 0;
      const int bw = svd_block_width(rows, k);
      if (bw <= 0) return 0;
      const int64_t nb = (k + bw - 1) / bw;
      return wide > 0 && nb >= wide ? 2 : nb >= svd_cluster_size() ? 1 : 0;
    };
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
      const int ca = clustered(a), cb = clustered(b);
      if (ca != cb) return ca > cb;
      return cost(a) > cost(b);
    });
    n_cluster = 0;
    n_wide = 0;
    for (size_t i = 0; i < order.size(); ++i) {
      n_cluster += clustered(order[i]) > 0 ? 1 : 0;
      n_wide += clustered(order[i]) == 2 ? 1 : 0;
    }
    std::vector<SvdJob> sj(jobs.size());
    std::vector<int64_t> sw(jobs.size());
    for (size_t i = 0; i < order.size(); ++i) {
      sj[i] = jobs[order[i]];
      sw[i] = work_off[order[i]];
    }
    auto r = std::make_pair(upload(sj), upload(sw));
    lpt.emplace(d, r);
    return r;
  }
};

extern "C" {

tnt_status tnt_last_error(char* buf, size_t len) {
  if (buf && len) {
    size_t n = std::min(len - 1, g_error.size());
    std::memcpy(buf, g_error.data(), n);
    buf[n] = 0;
  }
  return TNT_OK;
}

const char* tnt_version(void) { return "0.1.0"; }

// ---- rules -----------------------------------------------------------------

tnt_status tnt_rule_create(int32_t nfactors, const int32_t* kinds, int32_t codec, tnt_rule** out) {
  return guarded([&] {
    need(out != nullptr && kinds != nullptr, "null argument");
    need(nfactors >= 1 && nfactors <= kMaxFactors, "1..4 factors supported");
    need(codec == TNT_CODEC_PACKED || codec == TNT_CODEC_CANTOR, "unknown codec");
    Rule r;
    r.nf = nfactors;
    r.codec = (CodecKind)codec;
    for (int i = 0; i < nfactors; ++i) {
      need(kinds[i] >= 0 && kinds[i] <= 3, "unknown factor kind");
      r.kind[i] = (FactorKind)kinds[i];
    }
    *out = new tnt_rule{r};
  });
}

tnt_status tnt_rule_create_table(int32_t n, const int32_t* dual, const uint8_t* nsym, const double* dims,
                                 const double* fs, const double* rsym, const double* fsym, double tol,
                                 tnt_rule** out) {
  return guarded([&] {
    need(out && dual && nsym && dims && fs && rsym && fsym, "null argument");
    need(n >= 1 && n <= 16, "table providers hold 1..16 sectors");
    need(tol > 0.0 && tol < 1e-3, "tolerance must be in (0, 1e-3)");
    auto t = std::make_shared<TableData>();
    const size_t n3 = (size_t)n * n * n, n6 = n3 * n3;
    t->n = n;
    t->dual.assign(dual, dual + n);
    t->N.assign(nsym, nsym + n3);
    t->dims.assign(dims, dims + n);
    t->fs.assign(fs, fs + n);
    t->R.assign(rsym, rsym + n3);
    t->F.assign(fsym, fsym + n6);
    for (double v : t->F) need(std::isfinite(v), "non-finite F symbol");
    for (double v : t->R) need(std::isfinite(v), "non-finite R symbol");
    check_table(*t, tol);
    // identity: FNV-1a over every table (equal tables compare equal)
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](const void* p, size_t bytes) {
      const uint8_t* b = static_cast<const uint8_t*>(p);
      for (size_t i = 0; i < bytes; ++i) h = (h ^ b[i]) * 1099511628211ull;
    };
    mix(&n, sizeof(n));
    mix(t->dual.data(), n * sizeof(int32_t));
    mix(t->N.data(), n3);
    mix(t->dims.data(), n * sizeof(double));
    mix(t->fs.data(), n * sizeof(double));
    mix(t->R.data(), n3 * sizeof(double));
    mix(t->F.data(), n6 * sizeof(double));
    t->identity = h;
    Rule r;
    r.nf = 1;
    r.kind[0] = FK_TABLE;
    r.table = t;
    *out = new tnt_rule{r};
  });
}

void tnt_rule_destroy(tnt_rule* rule) { delete rule; }

static Sector read_label(const Rule& r, const int32_t* p) {
  Sector s;
  for (int i = 0; i < r.nf; ++i) {
    s.v[i] = p[i];
    if (r.kind[i] == FK_TABLE) need(p[i] >= 0 && p[i] < r.table->n, "table sector label out of range");
    if (r.kind[i] == FK_SU2) need(p[i] >= 0 && p[i] <= 254, "SU(2) doubled spin must be in 0..254");
    if (r.kind[i] == FK_FZ2 || r.kind[i] == FK_Z2) need(p[i] == 0 || p[i] == 1, "parity must be 0 or 1");
  }
  return s;
}

tnt_status tnt_rule_sector_id(const tnt_rule* rule, const int32_t* label, uint64_t* id) {
  return guarded([&] {
    need(rule && label && id, "null argument");
    *id = rule->r.id(read_label(rule->r, label));
  });
}

tnt_status tnt_rule_fsymbol(const tnt_rule* rule, const int32_t* x, double* value) {
  return guarded([&] {
    need(rule && x && value, "null argument");
    const Rule& r = rule->r;
    int nf = r.nf;
    *value = r.F(read_label(r, x), read_label(r, x + nf), read_label(r, x + 2 * nf), read_label(r, x + 3 * nf),
                 read_label(r, x + 4 * nf), read_label(r, x + 5 * nf));
  });
}

tnt_status tnt_rule_rsymbol(const tnt_rule* rule, const int32_t* x, double* value) {
  return guarded([&] {
    need(rule && x && value, "null argument");
    const Rule& r = rule->r;
    *value = r.R(read_label(r, x), read_label(r, x + r.nf), read_label(r, x + 2 * r.nf));
  });
}

tnt_status tnt_rule_dim(const tnt_rule* rule, const int32_t* label, double* dim) {
  return guarded([&] {
    need(rule && label && dim, "null argument");
    *dim = rule->r.dim(read_label(rule->r, label));
  });
}

// ---- spaces ----------------------------------------------------------------

tnt_status tnt_space_create(const tnt_rule* rule, int32_t n_codomain, int32_t n_domain, const int32_t* leg_nsectors,
                            const int32_t* leg_labels, const int64_t* leg_degeneracies, const uint8_t* leg_is_dual,
                            tnt_space** out) {
  return guarded([&] {
    need(rule && out, "null argument");
    need(n_codomain >= 0 && n_domain >= 0 && n_codomain + n_domain <= kMaxRank, "rank must be 0..8");
    int n = n_codomain + n_domain;
    need(n == 0 || (leg_nsectors && leg_labels && leg_degeneracies && leg_is_dual), "null leg arrays");
    const Rule& r = rule->r;
    std::vector<Leg> legs;
    int64_t pos = 0;
    for (int i = 0; i < n; ++i) {
      need(leg_nsectors[i] >= 0, "negative sector count");
      std::vector<Sector> s;
      std::vector<int64_t> d;
      for (int j = 0; j < leg_nsectors[i]; ++j, ++pos) {
        s.push_back(read_label(r, leg_labels + pos * r.nf));
        d.push_back(leg_degeneracies[pos]);
      }
      legs.push_back(Leg::make(r, s, d, leg_is_dual[i] != 0));
    }
    std::vector<Leg> cod(legs.begin(), legs.begin() + n_codomain), dom(legs.begin() + n_codomain, legs.end());
    *out = new tnt_space{make_space(r, cod, dom)};
  });
}

void tnt_space_destroy(tnt_space* space) { delete space; }

tnt_status tnt_space_info(const tnt_space* space, int64_t* size, int32_t* nsectors, int32_t* nblocks,
                          int32_t* n_codomain, int32_t* n_domain) {
  return guarded([&] {
    need(space != nullptr, "null space");
    const Space& s = *space->s;
    if (size) *size = s.size;
    if (nsectors) *nsectors = (int32_t)s.sectors.size();
    if (nblocks) *nblocks = (int32_t)s.blocks.size();
    if (n_codomain) *n_codomain = s.n1();
    if (n_domain) *n_domain = s.n2();
  });
}

tnt_status tnt_space_sectors(const tnt_space* space, int32_t* labels, int64_t* rows, int64_t* cols,
                             int64_t* offsets) {
  return guarded([&] {
    need(space != nullptr, "null space");
    const Space& s = *space->s;
    int nf = s.rule.nf;
    for (size_t i = 0; i < s.sectors.size(); ++i) {
      if (labels)
        for (int f = 0; f < nf; ++f) labels[i * nf + f] = s.sectors[i].c.v[f];
      if (rows) rows[i] = s.sectors[i].rows;
      if (cols) cols[i] = s.sectors[i].cols;
      if (offsets) offsets[i] = s.sectors[i].offset;
    }
  });
}

tnt_status tnt_space_blocks(const tnt_space* space, int64_t* offsets, int64_t* shapes, int64_t* strides,
                            int32_t* sector_index) {
  return guarded([&] {
    need(space != nullptr, "null space");
    const Space& s = *space->s;
    int rank = s.n1() + s.n2();
    for (size_t b = 0; b < s.blocks.size(); ++b) {
      const BlockInfo& bi = s.blocks[b];
      if (offsets) offsets[b] = bi.offset;
      for (int k = 0; k < rank; ++k) {
        if (shapes) shapes[b * rank + k] = bi.shape[k];
        if (strides) strides[b * rank + k] = bi.strides[k];
      }
      if (sector_index) sector_index[b] = bi.sector;
    }
  });
}

static void emit_tree(const Rule& r, const Tree& t, std::vector<int32_t>& o) {
  o.push_back((int32_t)t.u.size());
  for (auto& s : t.u)
    for (int f = 0; f < r.nf; ++f) o.push_back(s.v[f]);
  for (auto d : t.d) o.push_back(d);
  for (int f = 0; f < r.nf; ++f) o.push_back(t.c.v[f]);
  for (auto& s : t.inner)
    for (int f = 0; f < r.nf; ++f) o.push_back(s.v[f]);
}

tnt_status tnt_space_block_keys(const tnt_space* space, int32_t* keys, int64_t capacity, int64_t* length) {
  return guarded([&] {
    need(space != nullptr && length != nullptr, "null argument");
    const Space& s = *space->s;
    std::vector<int32_t> o;
    for (auto& b : s.blocks) {
      emit_tree(s.rule, b.key.cod, o);
      emit_tree(s.rule, b.key.dom, o);
    }
    *length = (int64_t)o.size();
    if (keys) {
      need(capacity >= (int64_t)o.size(), "key buffer too small");
      std::memcpy(keys, o.data(), o.size() * sizeof(int32_t));
    }
  });
}

tnt_status tnt_space_leg(const tnt_space* space, int32_t axis, int32_t* nsectors, int32_t* labels,
                         int64_t* degeneracies, uint8_t* is_dual) {
  return guarded([&] {
    need(space != nullptr, "null space");
    const Space& s = *space->s;
    need(axis >= 0 && axis < s.n1() + s.n2(), "axis out of range");
    const Leg& l = axis < s.n1() ? s.cod[axis] : s.dom[axis - s.n1()];
    if (nsectors) *nsectors = (int32_t)l.sectors.size();
    if (is_dual) *is_dual = l.dual ? 1 : 0;
    for (size_t i = 0; i < l.sectors.size(); ++i) {
      if (labels)
        for (int f = 0; f < s.rule.nf; ++f) labels[i * s.rule.nf + f] = l.sectors[i].v[f];
      if (degeneracies) degeneracies[i] = l.degs[i];
    }
  });
}

// ---- transform plans ---------------------------------------------------------

static tnt_status make_xplan(const tnt_space* src, TransformKind kind, int32_t n1, const int32_t* p1, int32_t n2,
                             const int32_t* p2, const int32_t* levels, int32_t nrep, tnt_xplan** out) {
  return guarded([&] {
    need(src && out, "null argument");
    std::vector<int> a, b, lv;
    if (kind == XK_PERMUTE || kind == XK_BRAID) {
      need(n1 >= 0 && n2 >= 0 && (n1 == 0 || p1) && (n2 == 0 || p2), "null axis list");
      a.assign(p1, p1 + n1);
      b.assign(p2, p2 + n2);
      if (kind == XK_BRAID) {
        need(levels != nullptr, "null levels");
        lv.assign(levels, levels + n1 + n2);
      }
    }
    auto x = new tnt_xplan_s();
    try {
      x->p = make_transform(src->s, kind, a, b, lv, nrep);
    } catch (...) {
      delete x;
      throw;
    }
    *out = x;
  });
}

tnt_status tnt_permute_plan(const tnt_space* src, int32_t n_codomain, const int32_t* codomain_axes, int32_t n_domain,
                            const int32_t* domain_axes, tnt_xplan** out) {
  return make_xplan(src, XK_PERMUTE, n_codomain, codomain_axes, n_domain, domain_axes, nullptr, 0, out);
}

tnt_status tnt_braid_plan(const tnt_space* src, int32_t n_codomain, const int32_t* codomain_axes, int32_t n_domain,
                          const int32_t* domain_axes, const int32_t* levels, tnt_xplan** out) {
  return make_xplan(src, XK_BRAID, n_codomain, codomain_axes, n_domain, domain_axes, levels, 0, out);
}

tnt_status tnt_repartition_plan(const tnt_space* src, int32_t n_codomain, tnt_xplan** out) {
  return make_xplan(src, XK_REPARTITION, 0, nullptr, 0, nullptr, nullptr, n_codomain, out);
}

tnt_status tnt_adjoint_plan(const tnt_space* src, tnt_xplan** out) {
  return make_xplan(src, XK_ADJOINT, 0, nullptr, 0, nullptr, nullptr, 0, out);
}

tnt_status tnt_twist_plan(const tnt_space* src, int32_t n_legs, const int32_t* legs, int32_t inverse,
                          tnt_xplan** out) {
  (void)inverse;  // every twist in scope is +-1, its own inverse
  return guarded([&] {
    need(src && out, "null argument");
    need(n_legs >= 0 && (n_legs == 0 || legs), "null leg list");
    int n1 = src->s->n1(), n = n1 + src->s->n2();
    std::vector<int> a, b, tw(legs, legs + n_legs);
    for (int i = 0; i < n1; ++i) a.push_back(i);
    for (int i = n1; i < n; ++i) b.push_back(i);
    auto x = new tnt_xplan_s();
    try {
      x->p = make_transform(src->s, XK_PERMUTE, a, b, {}, 0, tw);
    } catch (...) {
      delete x;
      throw;
    }
    *out = x;
  });
}

tnt_status tnt_contract_rhs_plan(const tnt_space* src, int32_t n_contracted, const int32_t* contracted_axes,
                                 int32_t n_open, const int32_t* open_axes, tnt_xplan** out) {
  return guarded([&] {
    need(src && out, "null argument");
    need(n_contracted >= 0 && n_open >= 0 && (n_contracted == 0 || contracted_axes) && (n_open == 0 || open_axes),
         "null axis list");
    std::vector<int> a(contracted_axes, contracted_axes + n_contracted), b(open_axes, open_axes + n_open);
    auto x = new tnt_xplan_s();
    try {
      auto plain = make_transform(src->s, XK_PERMUTE, a, b, {}, 0);
      std::vector<int> tw = supertrace_axes(*plain->dst, n_contracted);
      x->p = tw.empty() ? plain : make_transform(src->s, XK_PERMUTE, a, b, {}, 0, tw);
    } catch (...) {
      delete x;
      throw;
    }
    *out = x;
  });
}

tnt_status tnt_transform_chain_plan(const tnt_space* src, int32_t nsteps, const int32_t* program, int64_t len,
                                    tnt_xplan** out) {
  return guarded([&] {
    need(src && out, "null argument");
    need(nsteps >= 1 && program && len > 0, "empty chain");
    int64_t pos = 0;
    auto next = [&]() -> int32_t {
      if (pos >= len) throw std::invalid_argument("chain program ends early");
      return program[pos++];
    };
    auto list = [&](int32_t n) {
      if (n < 0 || n > 64) throw std::invalid_argument("bad axis count in chain program");
      std::vector<int> v;
      for (int32_t i = 0; i < n; ++i) v.push_back(next());
      return v;
    };
    std::vector<TransformStep> steps;
    std::shared_ptr<Space> cur = src->s;
    for (int32_t i = 0; i < nsteps; ++i) {
      TransformStep st;
      const int32_t kind = next();
      const int n = cur->n1() + cur->n2();
      if (kind == XK_PERMUTE || kind == XK_BRAID) {
        st.kind = (TransformKind)kind;
        st.p1 = list(next());
        st.p2 = list(next());
        if (kind == XK_BRAID) st.levels = list(n);
      } else if (kind == XK_REPARTITION) {
        st.kind = XK_REPARTITION;
        st.nrep = next();
      } else if (kind == XK_ADJOINT) {
        st.kind = XK_ADJOINT;
      } else if (kind == 4) {  // twist: identity permute with twisted legs
        st.kind = XK_PERMUTE;
        for (int a = 0; a < cur->n1(); ++a) st.p1.push_back(a);
        for (int a = cur->n1(); a < n; ++a) st.p2.push_back(a);
        st.twist_axes = list(next());
      } else {
        throw std::invalid_argument("unknown step kind in chain program");
      }
      cur = chain_spaces(cur, {st}).back();
      steps.push_back(st);
    }
    need(pos == len, "chain program has trailing entries");
    auto x = new tnt_xplan_s();
    try {
      x->p = make_transform_chain(src->s, steps);
    } catch (...) {
      delete x;
      throw;
    }
    *out = x;
  });
}

void tnt_xplan_destroy(tnt_xplan* plan) { delete plan; }

tnt_status tnt_xplan_dst_space(const tnt_xplan* plan, tnt_space** out) {
  return guarded([&] {
    need(plan && out, "null argument");
    need(plan->p->dst != nullptr, "plan built from tables has no destination space");
    *out = new tnt_space{plan->p->dst};
  });
}

tnt_status tnt_xplan_info(const tnt_xplan* plan, int64_t* ngroups, int64_t* ncoef, int64_t* bytes_moved) {
  return guarded([&] {
    need(plan != nullptr, "null plan");
    if (ngroups) *ngroups = (int64_t)plan->p->tables.groups.size();
    if (ncoef) *ncoef = (int64_t)plan->p->tables.coef.size();
    if (bytes_moved) *bytes_moved = plan->p->moved_elements * (int64_t)sizeof(double);
  });
}

tnt_status tnt_xplan_entries(const tnt_xplan* plan, int64_t* nsrc_entries, int64_t* ndst_entries) {
  return guarded([&] {
    need(plan != nullptr, "null plan");
    if (nsrc_entries) *nsrc_entries = (int64_t)plan->p->tables.src_entries.size();
    if (ndst_entries) *ndst_entries = (int64_t)plan->p->tables.dst_entries.size();
  });
}

tnt_status tnt_xplan_export(const tnt_xplan* plan, int64_t* groups, int64_t* src_entries, int64_t* dst_entries,
                            double* coef) {
  return guarded([&] {
    need(plan != nullptr, "null plan");
    const XformTables& t = plan->p->tables;
    if (groups)
      for (size_t i = 0; i < t.groups.size(); ++i) {
        const XGroup& g = t.groups[i];
        int64_t* r = groups + 14 * i;
        r[0] = g.nelem;
        r[1] = g.nsrc;
        r[2] = g.ndst;
        r[3] = g.src_first;
        r[4] = g.dst_first;
        r[5] = g.coef_off;
        for (int k = 0; k < kMaxRank; ++k) r[6 + k] = k < g.rank ? g.dims[k] : 1;
      }
    auto put = [](const std::vector<XEntry>& v, int64_t* o) {
      for (size_t i = 0; i < v.size(); ++i) {
        o[9 * i] = v[i].offset;
        for (int k = 0; k < kMaxRank; ++k) o[9 * i + 1 + k] = v[i].strides[k];
      }
    };
    if (src_entries) put(t.src_entries, src_entries);
    if (dst_entries) put(t.dst_entries, dst_entries);
    if (coef) std::memcpy(coef, t.coef.data(), t.coef.size() * sizeof(double));
  });
}

tnt_status tnt_xplan_from_tables(int32_t rank, int64_t ngroups, const int64_t* groups, int64_t nsrc_entries,
                                 const int64_t* src_entries, int64_t ndst_entries, const int64_t* dst_entries,
                                 int64_t ncoef, const double* coef, int64_t src_size, int64_t dst_size,
                                 tnt_xplan** out) {
  return guarded([&] {
    need(out != nullptr, "null argument");
    need(rank >= 0 && rank <= kMaxRank, "rank must be 0..8");
    need(ngroups >= 0 && nsrc_entries >= 0 && ndst_entries >= 0 && ncoef >= 0, "negative table length");
    need(src_size >= 0 && dst_size >= 0, "negative payload size");
    need((ngroups == 0 || groups) && (nsrc_entries == 0 || src_entries) && (ndst_entries == 0 || dst_entries) &&
             (ncoef == 0 || coef),
         "null table");
    need(nsrc_entries < INT32_MAX && ndst_entries < INT32_MAX && ncoef < INT32_MAX, "table too long");
    auto tp = std::make_shared<TransformPlan>();
    XformTables& T = tp->tables;
    T.src_size = src_size;
    T.dst_size = dst_size;
    auto entry = [&](const int64_t* r) {
      XEntry e{};
      e.offset = r[0];
      for (int k = 0; k < kMaxRank; ++k) e.strides[k] = k < rank ? r[1 + k] : 0;
      return e;
    };
    for (int64_t i = 0; i < nsrc_entries; ++i) T.src_entries.push_back(entry(src_entries + 9 * i));
    for (int64_t i = 0; i < ndst_entries; ++i) T.dst_entries.push_back(entry(dst_entries + 9 * i));
    T.coef.assign(coef, coef + ncoef);
    // Every destination element is written by exactly one group (the kernel
    // writes without atomics, and an element nothing writes would keep stale data).
    std::vector<bool> written(dst_size > 0 ? (size_t)dst_size : 0, false);
    auto span = [&](const XEntry& e, const int32_t* dims, int64_t size, const char* what) {
      int64_t hi = e.offset;
      need(e.offset >= 0, what);
      for (int k = 0; k < rank; ++k) {
        need(e.strides[k] >= 0, what);
        hi += (int64_t)(dims[k] - 1) * e.strides[k];
      }
      need(hi < size, what);
    };
    for (int64_t gi = 0; gi < ngroups; ++gi) {
      const int64_t* r = groups + 14 * gi;
      XGroup g{};
      g.nelem = r[0];
      need(r[1] >= 0 && r[1] < INT32_MAX && r[2] >= 1 && r[2] < INT32_MAX, "group source / destination counts");
      g.nsrc = (int32_t)r[1];
      g.ndst = (int32_t)r[2];
      need(r[3] >= 0 && r[3] + g.nsrc <= nsrc_entries, "group source entries out of range");
      need(r[4] >= 0 && r[4] + g.ndst <= ndst_entries, "group destination entries out of range");
      need(r[5] >= 0 && r[5] + (int64_t)g.nsrc * g.ndst <= ncoef, "group coefficients out of range");
      g.src_first = (int32_t)r[3];
      g.dst_first = (int32_t)r[4];
      g.coef_off = (int32_t)r[5];
      g.rank = rank;
      int64_t n = 1;
      for (int k = 0; k < kMaxRank; ++k) {
        const int64_t d = k < rank ? r[6 + k] : 1;
        need(d >= 1 && d <= 65535, "block extents must be 1..65535");
        g.dims[k] = (int32_t)d;
        n *= d;
      }
      need(n == g.nelem && n > 0, "group element count differs from its extents");
      for (int32_t s = 0; s < g.nsrc; ++s) span(T.src_entries[g.src_first + s], g.dims, src_size, "source block outside the source");
      for (int32_t d = 0; d < g.ndst; ++d) {
        const XEntry& e = T.dst_entries[g.dst_first + d];
        span(e, g.dims, dst_size, "destination block outside the destination");
        for (int64_t idx = 0; idx < n; ++idx) {
          int64_t pos = e.offset, rem = idx;
          for (int k = 0; k < rank; ++k) {
            pos += (rem % g.dims[k]) * e.strides[k];
            rem /= g.dims[k];
          }
          need(!written[(size_t)pos], "two destination blocks overlap");
          written[(size_t)pos] = true;
        }
      }
      tp->moved_elements += g.nelem * (g.nsrc + g.ndst);
      T.groups.push_back(g);
    }
    for (int64_t i = 0; i < dst_size; ++i) need(written[(size_t)i], "a destination element is written by no group");
    finish_transform_tables(T);
    auto x = new tnt_xplan_s();
    x->p = tp;
    *out = x;
  });
}

// ---- compose plans -----------------------------------------------------------

tnt_status tnt_compose_plan(const tnt_space* lhs, const tnt_space* rhs, tnt_cplan** out) {
  return guarded([&] {
    need(lhs && rhs && out, "null argument");
    auto c = new tnt_cplan_s();
    try {
      c->p = make_compose(lhs->s, rhs->s);
    } catch (...) {
      delete c;
      throw;
    }
    *out = c;
  });
}

void tnt_cplan_destroy(tnt_cplan* plan) { delete plan; }

tnt_status tnt_cplan_dst_space(const tnt_cplan* plan, tnt_space** out) {
  return guarded([&] {
    need(plan && out, "null argument");
    need(plan->p->dst != nullptr, "plan built from raw jobs has no destination space");
    *out = new tnt_space{plan->p->dst};
  });
}

tnt_status tnt_cplan_info(const tnt_cplan* plan, int64_t* njobs, double* flops) {
  return guarded([&] {
    need(plan != nullptr, "null plan");
    if (njobs) *njobs = (int64_t)plan->p->tables.jobs.size();
    if (flops) *flops = plan->p->flops;
  });
}

tnt_status tnt_cplan_export(const tnt_cplan* plan, int64_t* jobs) {
  return guarded([&] {
    need(plan && jobs, "null argument");
    const auto& v = plan->p->tables.jobs;
    for (size_t i = 0; i < v.size(); ++i) {
      const GemmJob& j = v[i];
      int64_t r[9] = {j.m, j.n, j.k, j.a_off, j.b_off, j.c_off, j.lda, j.ldb, j.ldc};
      std::memcpy(jobs + 9 * i, r, sizeof(r));
    }
  });
}

tnt_status tnt_cplan_from_jobs(int64_t njobs, const int64_t* jobs, int64_t a_size, int64_t b_size, int64_t c_size,
                               tnt_cplan** out) {
  return guarded([&] {
    need(out && (njobs == 0 || jobs), "null argument");
    auto plan = std::make_shared<ComposePlan>();
    for (int64_t i = 0; i < njobs; ++i) {
      const int64_t* r = jobs + 9 * i;
      GemmJob j{r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7], r[8]};
      need(j.m >= 0 && j.n >= 0 && j.k >= 0, "negative extent");
      need(j.lda >= std::max<int64_t>(1, j.m) && j.ldc >= std::max<int64_t>(1, j.m) &&
               j.ldb >= std::max<int64_t>(1, j.k),
           "leading dimension too small");
      if (j.m && j.k) need(j.a_off >= 0 && j.a_off + j.lda * (j.k - 1) + j.m <= a_size, "A region out of bounds");
      if (j.k && j.n) need(j.b_off >= 0 && j.b_off + j.ldb * (j.n - 1) + j.k <= b_size, "B region out of bounds");
      if (j.m && j.n) need(j.c_off >= 0 && j.c_off + j.ldc * (j.n - 1) + j.m <= c_size, "C region out of bounds");
      plan->tables.jobs.push_back(j);
      plan->flops += 2.0 * (double)j.m * (double)j.n * (double)j.k;
    }
    plan->tables.a_size = a_size;
    plan->tables.b_size = b_size;
    plan->tables.c_size = c_size;
    auto c = new tnt_cplan_s();
    c->p = plan;
    *out = c;
  });
}

// ---- factor plans ------------------------------------------------------------

tnt_status tnt_factor_plan(const tnt_space* src, tnt_fplan** out) {
  return guarded([&] {
    need(src && out, "null argument");
    auto f = new tnt_fplan_s();
    f->p = make_factor(src->s);
    int64_t off = 0;
    for (auto& j : f->p->tables.jobs) {
      f->work_off.push_back(off);
      int64_t rows = std::max(j.m, j.n);
      off += rows * j.k + j.k * j.k + 2 * j.k;
    }
    f->work_elems = off;
    *out = f;
  });
}

void tnt_fplan_destroy(tnt_fplan* plan) { delete plan; }

tnt_status tnt_fplan_info(const tnt_fplan* plan, int32_t* nsectors, int64_t* u_size, int64_t* s_size,
                          int64_t* v_size) {
  return guarded([&] {
    need(plan != nullptr, "null plan");
    const SvdTables& t = plan->p->tables;
    if (nsectors) *nsectors = (int32_t)t.jobs.size();
    if (u_size) *u_size = t.u_size;
    if (s_size) *s_size = t.s_size;
    if (v_size) *v_size = t.v_size;
  });
}

tnt_status tnt_fplan_export(const tnt_fplan* plan, int64_t* records, double* weights) {
  return guarded([&] {
    need(plan != nullptr, "null plan");
    const auto& v = plan->p->tables.jobs;
    for (size_t i = 0; i < v.size(); ++i) {
      const SvdJob& j = v[i];
      if (records) {
        int64_t r[8] = {j.m, j.n, j.k, j.a_off, j.u_off, j.s_off, j.v_off, 0};
        std::memcpy(records + 8 * i, r, sizeof(r));
      }
      if (weights) weights[i] = j.weight;
    }
  });
}

// ---- device execution ----------------------------------------------------------

tnt_status tnt_ctx_create(int32_t device, tnt_ctx** out) {
  return guarded([&] {
    need(out != nullptr, "null argument");
    int count = 0;
    cuda_check(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
    need(device >= 0 && device < count, "device ordinal out of range");
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    auto c = new tnt_ctx_s();
    c->device = device;
    cudaError_t e = cudaMalloc(&c->status, 16 * sizeof(int32_t));  // [0] error flags, [1] SVD sweeps
    if (e != cudaSuccess) {
      delete c;
      cuda_check(e, "cudaMalloc(status)");
    }
    cudaMemset(c->status, 0, 16 * sizeof(int32_t));
    e = cudaEventCreateWithFlags(&c->scratch_done, cudaEventDisableTiming);
    if (e != cudaSuccess) {
      cudaFree(c->status);
      delete c;
      cuda_check(e, "cudaEventCreate(scratch order)");
    }
    *out = c;
  });
}

void tnt_ctx_destroy(tnt_ctx* ctx) {
  if (!ctx) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(ctx->device);
  if (ctx->cublas) cublasDestroy(ctx->cublas);
  cudaFree(ctx->stage);
  cudaFree(ctx->svd_work);
  cudaFree(ctx->eigh_tmp);
  cudaFree(ctx->dot_part);
  cudaFree(ctx->split_buf);
  cudaFree(ctx->seg_stage);
  cudaFree(ctx->status);
  if (ctx->copy_in) cudaStreamDestroy(ctx->copy_in);
  if (ctx->copy_out) cudaStreamDestroy(ctx->copy_out);
  for (cudaEvent_t e : ctx->chunk_events) cudaEventDestroy(e);
  if (ctx->scratch_done) cudaEventDestroy(ctx->scratch_done);
  if (prev >= 0) cudaSetDevice(prev);
  delete ctx;
}

static void enter(tnt_ctx* ctx) {
  need(ctx != nullptr, "null context");
  cuda_check(cudaSetDevice(ctx->device), "cudaSetDevice");
}

tnt_status tnt_transform(tnt_ctx* ctx, const tnt_xplan* plan, double* dst, const double* src, double alpha,
                         double beta, void* stream) {
  return guarded([&] {
    enter(ctx);
    need(plan != nullptr, "null plan");
    const XformTables& t = plan->p->tables;
    need(t.dst_size == 0 || dst, "null destination");
    need(t.src_size == 0 || src, "null source");
    const DevXform& x = const_cast<tnt_xplan*>(plan)->on_device();
    cuda_check(launch_xform(x, dst, src, alpha, beta, (cudaStream_t)stream), "transform kernel launch");
  });
}

static void compose_cublas(tnt_ctx* ctx, tnt_cplan* plan, int64_t nbatch, double* dst, int64_t sd, const double* lhs,
                           int64_t sl, const double* rhs, int64_t sr, double alpha, double beta, cudaStream_t st) {
  std::lock_guard<std::recursive_mutex> g(ctx->mu);  // one cuBLAS handle per context, bound to st below
  if (!ctx->cublas) {
    if (cublasCreate(&ctx->cublas) != CUBLAS_STATUS_SUCCESS) throw Failure(TNT_CUDA_ERROR, "cublasCreate failed");
  }
  cublasSetStream(ctx->cublas, st);
  for (int64_t b = 0; b < nbatch; ++b)
    for (auto& j : plan->p->tables.jobs) {
      if (j.m == 0 || j.n == 0) continue;
      double* c = dst + b * sd + j.c_off;
      if (j.k == 0) {
        // sector present in only one operand: C = beta * C
        for (int64_t col = 0; col < j.n; ++col) {
          if (beta == 0.0)
            cuda_check(cudaMemsetAsync(c + col * j.ldc, 0, j.m * sizeof(double), st), "memset");
          else if (cublasDscal(ctx->cublas, (int)j.m, &beta, c + col * j.ldc, 1) != CUBLAS_STATUS_SUCCESS)
            throw Failure(TNT_CUDA_ERROR, "cublasDscal failed");
        }
        continue;
      }
      if (cublasDgemm(ctx->cublas, CUBLAS_OP_N, CUBLAS_OP_N, (int)j.m, (int)j.n, (int)j.k, &alpha,
                      lhs + b * sl + j.a_off, (int)j.lda, rhs + b * sr + j.b_off, (int)j.ldb, &beta, c,
                      (int)j.ldc) != CUBLAS_STATUS_SUCCESS)
        throw Failure(TNT_CUDA_ERROR, "cublasDgemm failed");
    }
}

}  // extern "C"

namespace {

bool stream_capturing(cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  return cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone;
}

// The context's scratch (split packs, staging, segment tables, dot partials)
// is shared by every call on the context.  A call that uses it on stream st
// first makes st wait for the previous user's work when that ran on another
// stream, and records the context's event after its own launches
// (scratch_acquire / scratch_release, with ctx->mu held in between).  Calls
// on different streams of one context are therefore correct, and their
// scratch-using work runs one after the other.  Calls made while st captures
// a graph are not tracked (a captured event cannot order work outside the
// graph): the replays of such a graph are ordered by the caller.
void scratch_acquire(tnt_ctx* ctx, cudaStream_t st) {
  if (stream_capturing(st)) return;
  if (ctx->scratch_user_valid && ctx->scratch_user != st)
    cuda_check(cudaStreamWaitEvent(st, ctx->scratch_done, 0), "order the context scratch after its last user");
}

void scratch_release(tnt_ctx* ctx, cudaStream_t st) {
  if (stream_capturing(st)) {
    ctx->scratch_user_valid = false;
    return;
  }
  cuda_check(cudaEventRecord(ctx->scratch_done, st), "record the context scratch user");
  ctx->scratch_user = st;
  ctx->scratch_user_valid = true;
}

// Average milliseconds of `reps` launches after one untimed launch.
template <class F>
double time_ms(cudaStream_t st, int reps, F&& launch) {
  launch();
  cudaEvent_t a, b;
  cuda_check(cudaEventCreate(&a), "cudaEventCreate");
  cuda_check(cudaEventCreate(&b), "cudaEventCreate");
  cuda_check(cudaEventRecord(a, st), "cudaEventRecord");
  for (int r = 0; r < reps; ++r) launch();
  cuda_check(cudaEventRecord(b, st), "cudaEventRecord");
  cuda_check(cudaEventSynchronize(b), "cudaEventSynchronize");
  float ms = 0.f;
  cuda_check(cudaEventElapsedTime(&ms, a, b), "cudaEventElapsedTime");
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return (double)ms / reps;
}

// Timing-based calibration needs: autotuning on, an overwriting compose
// (beta == 0, so repeated launches leave the same result), no stream capture
// in progress, and enough work for the timing to mean something.
bool can_calibrate(const tnt_cplan_s* plan, int64_t nbatch, double beta, cudaStream_t st) {
  return autotune_enabled() && beta == 0.0 && !stream_capturing(st) && plan->p->flops * (double)nbatch >= 2e8;
}

struct ComposeArgs {
  int64_t nbatch;
  double* dst;
  int64_t sd;
  const double* lhs;
  int64_t sl;
  const double* rhs;
  int64_t sr;
  double alpha, beta;
};

// The FP64 tile list of this plan and batch count on the current device:
// per-job shapes from the device's measured per-shape costs, calibrated on
// the first eligible compose by timing every uniform shape.
std::pair<GemmTile*, int32_t> f64_tiles(tnt_cplan_s* plan, const ComposeArgs& x, cudaStream_t st) {
  const int d = current_device();
  GemmJob* jobs_dev;
  {
    std::lock_guard<std::mutex> g(plan->mu);
    CplanDevice& c = plan->on_device(d);
    auto it = c.f64_tiles.find(x.nbatch);
    if (it != c.f64_tiles.end()) return it->second;
    jobs_dev = c.jobs;
  }
  const std::vector<GemmJob>& jobs = plan->p->tables.jobs;
  double cost[4];
  bool calibrated;
  {
    std::lock_guard<std::mutex> g(tuning_mutex());
    DeviceTuning& T = device_tuning(d);
    std::copy(T.f64_cost, T.f64_cost + 4, cost);
    calibrated = T.f64_calibrated;
  }
  if (!calibrated && can_calibrate(plan, x.nbatch, x.beta, st)) {
    double measured[4];
    for (int s = 0; s < 4; ++s) {
      std::vector<int32_t> uniform(jobs.size(), s);
      std::vector<GemmTile> tv = build_f64_tiles(jobs, x.nbatch, uniform, cost);
      GemmTile* td = upload(tv);
      const double ms = time_ms(st, 3, [&] {
        cuda_check(launch_gemm_f64(jobs_dev, td, (int32_t)tv.size(), x.dst, x.sd, x.lhs, x.sl, x.rhs, x.sr, x.alpha,
                                   x.beta, st),
                   "fp64 grouped gemm launch");
      });
      cudaFree(td);
      measured[s] = ms / std::max(1.0, f64_tile_units(jobs, tv));
    }
    std::lock_guard<std::mutex> g(tuning_mutex());
    DeviceTuning& T = device_tuning(d);
    std::copy(measured, measured + 4, T.f64_cost);
    T.f64_calibrated = true;
    std::copy(measured, measured + 4, cost);
  }
  std::vector<GemmTile> tv = build_f64_tiles(jobs, x.nbatch, choose_f64_shapes(jobs, cost), cost);
  std::pair<GemmTile*, int32_t> r(upload(tv), (int32_t)tv.size());
  std::lock_guard<std::mutex> g(plan->mu);
  CplanDevice& c = plan->on_device(d);
  auto ins = c.f64_tiles.emplace(x.nbatch, r);
  if (!ins.second) cudaFree(r.first);  // another thread built it first
  return ins.first->second;
}

// The plan's device-resident split packing table for (slices, width, format).
void* split_table_on_device(tnt_cplan_s* plan, int slices, int tile_n, bool i8) {
  const GemmTables& t = plan->p->tables;
  std::lock_guard<std::mutex> g(plan->mu);
  CplanDevice& c = plan->on_device(current_device());
  const int64_t jkey = ((int64_t)slices * 1024 + tile_n) * 2 + (i8 ? 1 : 0);
  auto jt = c.split_jobs.find(jkey);
  if (jt == c.split_jobs.end())
    jt = c.split_jobs.emplace(jkey, (void*)upload(split_job_table(t.jobs.data(), (int32_t)t.jobs.size(), slices,
                                                                  tile_n, i8))).first;
  return jt->second;
}

// One split-precision compose at tile width tile_n (tiles and slice scratch
// built or grown on first use); pre_a / pre_b are sides packed beforehand
// (tnt_split_pack_operand, nbatch 1).
void compose_split(tnt_ctx* ctx, tnt_cplan_s* plan, const ComposeArgs& x, int slices, int tile_n, bool i8,
                   cudaStream_t st, void* ext_scratch = nullptr, size_t ext_bytes = 0, const void* pre_a = nullptr,
                   const void* pre_b = nullptr) {
  const GemmTables& t = plan->p->tables;
  for (const GemmJob& j : t.jobs) need(j.k < INT32_MAX, "split precision: K must stay below 2^31");
  const int d = current_device();
  std::pair<GemmTile*, int32_t> tiles;
  void* job_table = split_table_on_device(plan, slices, tile_n, i8);
  {
    std::lock_guard<std::mutex> g(plan->mu);
    CplanDevice& c = plan->on_device(d);
    const int64_t tkey = x.nbatch * 1024 + tile_n;
    auto it = c.split_tiles.find(tkey);
    if (it == c.split_tiles.end()) {
      auto tv = plan->make_tiles(x.nbatch, kSplitTileM, tile_n);
      it = c.split_tiles.emplace(tkey, std::make_pair(upload(tv), (int32_t)tv.size())).first;
    }
    tiles = it->second;
  }
  std::pair<void*, size_t> scratch;
  const size_t need_bytes = split_scratch_bytes(t.jobs.data(), (int32_t)t.jobs.size(), x.nbatch, slices, tile_n, i8);
  if (ext_scratch) {
    need(ext_bytes >= need_bytes, "scratch buffer smaller than tnt_cplan_scratch_bytes");
    scratch = std::make_pair(ext_scratch, ext_bytes);
  } else {
    // Slice packs live in a grow-only context buffer shared by every plan,
    // ordered across streams by scratch_acquire / scratch_release.  The pack
    // kernels rewrite every byte whose value reaches a result (padding-only
    // row and column groups feed only outputs that are never written), so no
    // clearing is needed.
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    if (ctx->split_bytes < need_bytes) {
      cudaFree(ctx->split_buf);
      ctx->split_buf = nullptr;
      ctx->split_bytes = 0;
      cuda_check(cudaMalloc(&ctx->split_buf, need_bytes), "cudaMalloc(split scratch)");
      ctx->split_bytes = need_bytes;
    }
    scratch_acquire(ctx, st);
    cuda_check(launch_gemm_split(job_table, t.jobs.data(), (int32_t)t.jobs.size(), tiles.first, tiles.second, x.dst,
                                 x.sd, x.lhs, x.sl, x.rhs, x.sr, x.nbatch, x.alpha, x.beta, slices, tile_n, i8,
                                 ctx->split_buf, ctx->split_bytes, ctx->status + 2, st, pre_a, pre_b),
               "split-precision gemm launch");
    scratch_release(ctx, st);
    return;
  }
  cuda_check(launch_gemm_split(job_table, t.jobs.data(), (int32_t)t.jobs.size(), tiles.first, tiles.second, x.dst, x.sd,
                               x.lhs, x.sl, x.rhs, x.sr, x.nbatch, x.alpha, x.beta, slices, tile_n, i8, scratch.first,
                               scratch.second, ctx->status + 2, st, pre_a, pre_b),
             "split-precision gemm launch");
}

// Split tile width for this plan: the device's measured 64-vs-128 per-MAC
// throughput ratio (calibrated on the first eligible compose by timing both
// widths) applied to the plan's padded work at each width.
int split_width(tnt_ctx* ctx, tnt_cplan_s* plan, const ComposeArgs& x, int slices, cudaStream_t st) {
  const GemmTables& t = plan->p->tables;
  const int d = current_device();
  double eff64;
  bool calibrated;
  {
    std::lock_guard<std::mutex> g(tuning_mutex());
    DeviceTuning& T = device_tuning(d);
    eff64 = T.split_eff64;
    calibrated = T.split_calibrated;
  }
  if (!calibrated && !getenv("TNT_SPLIT_TILE_N") && can_calibrate(plan, x.nbatch, x.beta, st)) {
    const double t64 = time_ms(st, 2, [&] { compose_split(ctx, plan, x, slices, 64, false, st); });
    const double t128 = time_ms(st, 2, [&] { compose_split(ctx, plan, x, slices, 128, false, st); });
    const double w64 = split_padded_macs(t.jobs.data(), (int32_t)t.jobs.size(), 64);
    const double w128 = split_padded_macs(t.jobs.data(), (int32_t)t.jobs.size(), 128);
    eff64 = (w64 / t64) / (w128 / t128);
    std::lock_guard<std::mutex> g(tuning_mutex());
    DeviceTuning& T = device_tuning(d);
    T.split_eff64 = eff64;
    T.split_calibrated = true;
  }
  return split_tile_n(t.jobs.data(), (int32_t)t.jobs.size(), eff64);
}

}  // namespace

extern "C" {

tnt_status tnt_compose(tnt_ctx* ctx, const tnt_cplan* cplan, int64_t nbatch, double* dst, int64_t stride_dst,
                       const double* lhs, int64_t stride_lhs, const double* rhs, int64_t stride_rhs, double alpha,
                       double beta, int32_t precision, int32_t slices, void* stream) {
  return guarded([&] {
    enter(ctx);
    need(cplan != nullptr, "null plan");
    need(nbatch >= 0, "negative batch");
    auto* plan = const_cast<tnt_cplan*>(cplan);
    const GemmTables& t = plan->p->tables;
    if (nbatch == 0 || t.jobs.empty()) return;
    need(dst && lhs && rhs, "null operand");
    if (nbatch > 1)
      need(stride_dst >= t.c_size && stride_lhs >= t.a_size && stride_rhs >= t.b_size, "batch stride too small");
    cudaStream_t st = (cudaStream_t)stream;
    const ComposeArgs x{nbatch, dst, stride_dst, lhs, stride_lhs, rhs, stride_rhs, alpha, beta};
    if (precision == TNT_PREC_FP64) {
      auto tiles = f64_tiles(plan, x, st);
      cuda_check(launch_gemm_f64(plan->jobs_dev(), tiles.first, tiles.second, dst, stride_dst, lhs, stride_lhs, rhs,
                                 stride_rhs, alpha, beta, st),
                 "fp64 grouped gemm launch");
    } else if (precision == TNT_PREC_CUBLAS_FP64) {
      compose_cublas(ctx, plan, nbatch, dst, stride_dst, lhs, stride_lhs, rhs, stride_rhs, alpha, beta, st);
    } else if (precision == TNT_PREC_BF16X) {
      need(slices >= 1 && slices <= 8, "slices must be 1..8");
      compose_split(ctx, plan, x, slices, split_width(ctx, plan, x, slices, st), false, st);
    } else if (precision == TNT_PREC_INT8X) {
      need(slices >= 1 && slices <= 6, "8-bit digits: slices must be 1..6");
      compose_split(ctx, plan, x, slices, 64, true, st);
    } else {
      throw std::invalid_argument("unknown precision");
    }
  });
}

tnt_status tnt_ctx_sync(tnt_ctx* ctx, void* stream) {
  return guarded([&] {
    enter(ctx);
    cudaStream_t st = (cudaStream_t)stream;
    int32_t code = 0;
    cuda_check(cudaMemcpyAsync(&code, ctx->status + 2, sizeof(int32_t), cudaMemcpyDeviceToHost, st),
               "read device error word");
    cuda_check(cudaStreamSynchronize(st), "stream synchronize");
    if (code != 0) {
      cuda_check(cudaMemset(ctx->status + 2, 0, sizeof(int32_t)), "clear device error word");
      throw Failure(TNT_DEVICE_TIMEOUT, "split-precision kernel: a pipeline wait gave up (stage code " +
                                            std::to_string(code) + "); its results are invalid");
    }
  });
}

tnt_status tnt_ctx_svd_sweeps(const tnt_ctx* ctx, int32_t* sweeps) {
  return guarded([&] {
    need(ctx && sweeps, "null argument");
    *sweeps = ctx->last_sweeps;
  });
}

tnt_status tnt_cplan_scratch_bytes(const tnt_cplan* cplan, int64_t nbatch, int32_t precision, int32_t slices,
                                   size_t* bytes) {
  return guarded([&] {
    need(cplan && bytes, "null argument");
    need(nbatch >= 0, "negative batch");
    const GemmTables& t = cplan->p->tables;
    *bytes = 0;
    if (nbatch == 0 || t.jobs.empty()) return;
    if (precision == TNT_PREC_BF16X) {
      need(slices >= 1 && slices <= 8, "slices must be 1..8");
      *bytes = std::max(split_scratch_bytes(t.jobs.data(), (int32_t)t.jobs.size(), nbatch, slices, 64, false),
                        split_scratch_bytes(t.jobs.data(), (int32_t)t.jobs.size(), nbatch, slices, 128, false));
    } else if (precision == TNT_PREC_INT8X) {
      need(slices >= 1 && slices <= 6, "8-bit digits: slices must be 1..6");
      *bytes = split_scratch_bytes(t.jobs.data(), (int32_t)t.jobs.size(), nbatch, slices, 64, true);
    } else {
      need(precision == TNT_PREC_FP64 || precision == TNT_PREC_CUBLAS_FP64, "unknown precision");
    }
  });
}

tnt_status tnt_compose_ws(tnt_ctx* ctx, const tnt_cplan* cplan, int64_t nbatch, double* dst, int64_t stride_dst,
                          const double* lhs, int64_t stride_lhs, const double* rhs, int64_t stride_rhs, double alpha,
                          double beta, int32_t precision, int32_t slices, void* scratch, size_t scratch_bytes,
                          void* stream) {
  if (precision != TNT_PREC_BF16X && precision != TNT_PREC_INT8X)
    return tnt_compose(ctx, cplan, nbatch, dst, stride_dst, lhs, stride_lhs, rhs, stride_rhs, alpha, beta, precision,
                       slices, stream);
  return guarded([&] {
    enter(ctx);
    need(cplan != nullptr, "null plan");
    need(nbatch >= 0, "negative batch");
    auto* plan = const_cast<tnt_cplan*>(cplan);
    const GemmTables& t = plan->p->tables;
    if (nbatch == 0 || t.jobs.empty()) return;
    need(dst && lhs && rhs && scratch, "null operand");
    need(slices >= 1 && slices <= (precision == TNT_PREC_INT8X ? 6 : 8),
         precision == TNT_PREC_INT8X ? "8-bit digits: slices must be 1..6" : "slices must be 1..8");
    if (nbatch > 1)
      need(stride_dst >= t.c_size && stride_lhs >= t.a_size && stride_rhs >= t.b_size, "batch stride too small");
    const ComposeArgs x{nbatch, dst, stride_dst, lhs, stride_lhs, rhs, stride_rhs, alpha, beta};
    const bool i8 = precision == TNT_PREC_INT8X;
    int width = 64;
    if (!i8) {  // the device's current tile-width model; no timing here
      std::lock_guard<std::mutex> g(tuning_mutex());
      width = split_tile_n(t.jobs.data(), (int32_t)t.jobs.size(), device_tuning(current_device()).split_eff64);
    }
    compose_split(ctx, plan, x, slices, width, i8, (cudaStream_t)stream, scratch, scratch_bytes);
  });
}

tnt_status tnt_split_operand_bytes(const tnt_cplan* cplan, int32_t side, int32_t precision, int32_t slices,
                                   size_t* bytes) {
  return guarded([&] {
    need(cplan && bytes, "null argument");
    need(side == 0 || side == 1, "side must be 0 (left operand) or 1 (right operand)");
    need(precision == TNT_PREC_INT8X, "pre-packed operands exist for TNT_PREC_INT8X");
    need(slices >= 1 && slices <= 6, "8-bit digits: slices must be 1..6");
    const GemmTables& t = cplan->p->tables;
    *bytes = t.jobs.empty() ? 0 : split_operand_bytes(t.jobs.data(), (int32_t)t.jobs.size(), slices, 64, true, side);
  });
}

tnt_status tnt_split_pack_operand(tnt_ctx* ctx, const tnt_cplan* cplan, int32_t side, const double* operand,
                                  int32_t precision, int32_t slices, void* packed, size_t packed_bytes,
                                  void* stream) {
  return guarded([&] {
    enter(ctx);
    size_t need_bytes = 0;
    const tnt_status st0 = tnt_split_operand_bytes(cplan, side, precision, slices, &need_bytes);
    if (st0 != TNT_OK) throw Failure(st0, "bad split operand request");
    auto* plan = const_cast<tnt_cplan*>(cplan);
    const GemmTables& t = plan->p->tables;
    if (t.jobs.empty()) return;
    need(operand && packed, "null operand");
    need(packed_bytes >= need_bytes, "packed buffer smaller than tnt_split_operand_bytes");
    for (const GemmJob& j : t.jobs) need(j.k < INT32_MAX, "split precision: K must stay below 2^31");
    void* table = split_table_on_device(plan, slices, 64, true);
    cuda_check(launch_split_pack_operand(table, t.jobs.data(), (int32_t)t.jobs.size(), side, operand, slices, 64, true,
                                         packed, (cudaStream_t)stream),
               "split operand pack launch");
  });
}

tnt_status tnt_compose_packed(tnt_ctx* ctx, const tnt_cplan* cplan, double* dst, const double* lhs,
                              const void* lhs_packed, const double* rhs, const void* rhs_packed, double alpha,
                              double beta, int32_t precision, int32_t slices, void* stream) {
  return guarded([&] {
    enter(ctx);
    need(cplan != nullptr, "null plan");
    need(precision == TNT_PREC_INT8X, "pre-packed operands exist for TNT_PREC_INT8X");
    need(slices >= 1 && slices <= 6, "8-bit digits: slices must be 1..6");
    auto* plan = const_cast<tnt_cplan*>(cplan);
    const GemmTables& t = plan->p->tables;
    if (t.jobs.empty()) return;
    need(dst && (lhs || lhs_packed) && (rhs || rhs_packed), "null operand");
    const ComposeArgs x{1, dst, t.c_size, lhs, t.a_size, rhs, t.b_size, alpha, beta};
    compose_split(ctx, plan, x, slices, 64, true, (cudaStream_t)stream, nullptr, 0, lhs_packed, rhs_packed);
  });
}

tnt_status tnt_cplan_tile_shapes(const tnt_cplan* plan, const double* costs, int32_t* shapes) {
  return guarded([&] {
    need(plan && costs && shapes, "null argument");
    const auto v = choose_f64_shapes(plan->p->tables.jobs, costs);
    std::copy(v.begin(), v.end(), shapes);
  });
}

tnt_status tnt_tuning_info(int32_t device, double* f64_costs, int32_t* f64_calibrated, double* split_eff64,
                           int32_t* split_calibrated) {
  return guarded([&] {
    std::lock_guard<std::mutex> g(tuning_mutex());
    const DeviceTuning& T = device_tuning(device);
    if (f64_costs) std::copy(T.f64_cost, T.f64_cost + 4, f64_costs);
    if (f64_calibrated) *f64_calibrated = T.f64_calibrated ? 1 : 0;
    if (split_eff64) *split_eff64 = T.split_eff64;
    if (split_calibrated) *split_calibrated = T.split_calibrated ? 1 : 0;
  });
}

tnt_status tnt_compose_host(tnt_ctx* ctx, const tnt_cplan* cplan, int64_t nbatch, double* dst_host,
                            const double* lhs_host, const double* rhs_host, int32_t precision, int32_t slices,
                            void* stream) {
  tnt_status st_code = guarded([&] {
    enter(ctx);
    need(cplan != nullptr, "null plan");
    const GemmTables& t = cplan->p->tables;
    need(nbatch >= 0, "negative batch");
    if (nbatch == 0) return;
    need(dst_host && lhs_host && rhs_host, "null host buffer");
    size_t na = (size_t)(t.a_size * nbatch), nb = (size_t)(t.b_size * nbatch), nc = (size_t)(t.c_size * nbatch);
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    if (ctx->stage_elems < na + nb + nc) {
      cudaFree(ctx->stage);
      ctx->stage = nullptr;
      ctx->stage_elems = 0;
      cuda_check(cudaMalloc(&ctx->stage, (na + nb + nc) * sizeof(double)), "cudaMalloc(stage)");
      ctx->stage_elems = na + nb + nc;
    }
    double* da = ctx->stage;
    double* db = da + na;
    double* dc = db + nb;
    cudaStream_t st = (cudaStream_t)stream;
    // Batches of several tensors run as a pipeline of chunks: the operands of
    // chunk c + 1 cross PCIe (copy-in stream) while chunk c is composed on
    // `stream` and chunk c - 1 returns (copy-out stream), so the step costs
    // about the larger transfer instead of the sum of both and the compose.
    const int64_t nchunks = std::min<int64_t>(nbatch, 8);
    if (!ctx->copy_in) {
      cuda_check(cudaStreamCreateWithFlags(&ctx->copy_in, cudaStreamNonBlocking), "create copy-in stream");
      cuda_check(cudaStreamCreateWithFlags(&ctx->copy_out, cudaStreamNonBlocking), "create copy-out stream");
    }
    while ((int64_t)ctx->chunk_events.size() < 2 * nchunks + 1) {
      cudaEvent_t e;
      cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "create event");
      ctx->chunk_events.push_back(e);
    }
    cudaEvent_t* ev = ctx->chunk_events.data();
    // Order the copies after work already queued on `stream`.
    cuda_check(cudaEventRecord(ev[2 * nchunks], st), "record event");
    cuda_check(cudaStreamWaitEvent(ctx->copy_in, ev[2 * nchunks], 0), "wait event");
    try {
      for (int64_t c = 0; c < nchunks; ++c) {
        const int64_t b0 = nbatch * c / nchunks, b1 = nbatch * (c + 1) / nchunks, nbc = b1 - b0;
        cuda_check(cudaMemcpyAsync(da + b0 * t.a_size, lhs_host + b0 * t.a_size, nbc * t.a_size * sizeof(double),
                                   cudaMemcpyHostToDevice, ctx->copy_in),
                   "H2D lhs");
        cuda_check(cudaMemcpyAsync(db + b0 * t.b_size, rhs_host + b0 * t.b_size, nbc * t.b_size * sizeof(double),
                                   cudaMemcpyHostToDevice, ctx->copy_in),
                   "H2D rhs");
        cuda_check(cudaEventRecord(ev[2 * c], ctx->copy_in), "record event");
        cuda_check(cudaStreamWaitEvent(st, ev[2 * c], 0), "wait event");
        tnt_status s = tnt_compose(ctx, cplan, nbc, dc + b0 * t.c_size, t.c_size, da + b0 * t.a_size, t.a_size,
                                   db + b0 * t.b_size, t.b_size, 1.0, 0.0, precision, slices, stream);
        if (s != TNT_OK) throw Failure(s, g_error);
        cuda_check(cudaEventRecord(ev[2 * c + 1], st), "record event");
        cuda_check(cudaStreamWaitEvent(ctx->copy_out, ev[2 * c + 1], 0), "wait event");
        cuda_check(cudaMemcpyAsync(dst_host + b0 * t.c_size, dc + b0 * t.c_size, nbc * t.c_size * sizeof(double),
                                   cudaMemcpyDeviceToHost, ctx->copy_out),
                   "D2H dst");
      }
    } catch (...) {
      // No copy of the caller's host buffers may outlive the call.
      cudaStreamSynchronize(ctx->copy_in);
      cudaStreamSynchronize(ctx->copy_out);
      throw;
    }
    cuda_check(cudaStreamSynchronize(ctx->copy_out), "stream synchronize");
    cuda_check(cudaStreamSynchronize(st), "stream synchronize");
  });
  return st_code;
}

tnt_status tnt_svd(tnt_ctx* ctx, const tnt_fplan* fplan, const double* a, double* u, double* s, double* vh,
                   void* stream) {
  return guarded([&] {
    enter(ctx);
    need(fplan != nullptr, "null plan");
    auto* plan = const_cast<tnt_fplan*>(fplan);
    const SvdTables& t = plan->p->tables;
    if (t.jobs.empty()) return;
    need(a && u && s && vh, "null operand");
    auto dev = plan->lpt_on_device();
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    if (ctx->svd_work_elems < (size_t)plan->work_elems) {
      cudaFree(ctx->svd_work);
      ctx->svd_work = nullptr;
      ctx->svd_work_elems = 0;
      cuda_check(cudaMalloc(&ctx->svd_work, plan->work_elems * sizeof(double)), "cudaMalloc(svd work)");
      ctx->svd_work_elems = plan->work_elems;
    }
    cudaStream_t st = (cudaStream_t)stream;
    cuda_check(cudaMemsetAsync(ctx->status, 0, 2 * sizeof(int32_t), st), "memset status");
    cuda_check(launch_svd_split(dev.first, plan->n_cluster, (int32_t)t.jobs.size(), a, u, s, vh, ctx->svd_work,
                                dev.second, ctx->status, st, plan->n_wide),
               "svd kernel launch");
    int32_t hs[2] = {0, 0};
    cuda_check(cudaMemcpyAsync(hs, ctx->status, sizeof(hs), cudaMemcpyDeviceToHost, st), "read svd status");
    cuda_check(cudaStreamSynchronize(st), "stream synchronize");
    ctx->last_sweeps = hs[1];
    if (hs[0] != 0) throw Failure(TNT_INTERNAL, "Jacobi SVD did not converge within the sweep limit");
  });
}

tnt_status tnt_svd_ws_async(tnt_ctx* ctx, const tnt_fplan* fplan, const double* a, double* u, double* s, double* vh,
                            double* work, int32_t* status, void* stream) {
  return guarded([&] {
    enter(ctx);
    need(fplan != nullptr, "null plan");
    auto* plan = const_cast<tnt_fplan*>(fplan);
    const SvdTables& t = plan->p->tables;
    if (t.jobs.empty()) return;
    need(a && u && s && vh && work && status, "null operand");
    auto dev = plan->lpt_on_device();
    cudaStream_t st = (cudaStream_t)stream;
    cuda_check(cudaMemsetAsync(status, 0, 2 * sizeof(int32_t), st), "memset status");
    cuda_check(launch_svd_split(dev.first, plan->n_cluster, (int32_t)t.jobs.size(), a, u, s, vh, work, dev.second,
                                status, st, plan->n_wide),
               "svd kernel launch");
  });
}

tnt_status tnt_fplan_work(const tnt_fplan* plan, int64_t* work_elems) {
  return guarded([&] {
    need(plan && work_elems, "null argument");
    *work_elems = plan->work_elems;
  });
}

tnt_status tnt_svd_ws(tnt_ctx* ctx, const tnt_fplan* fplan, const double* a, double* u, double* s, double* vh,
                      double* work, void* stream) {
  return guarded([&] {
    enter(ctx);
    need(fplan != nullptr, "null plan");
    auto* plan = const_cast<tnt_fplan*>(fplan);
    const SvdTables& t = plan->p->tables;
    if (t.jobs.empty()) return;
    need(a && u && s && vh && work, "null operand");
    auto dev = plan->lpt_on_device();
    cudaStream_t st = (cudaStream_t)stream;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);  // the status words are the context's
    cuda_check(cudaMemsetAsync(ctx->status, 0, 2 * sizeof(int32_t), st), "memset status");
    cuda_check(launch_svd_split(dev.first, plan->n_cluster, (int32_t)t.jobs.size(), a, u, s, vh, work, dev.second,
                                ctx->status, st, plan->n_wide),
               "svd kernel launch");
    int32_t hs[2] = {0, 0};
    cuda_check(cudaMemcpyAsync(hs, ctx->status, sizeof(hs), cudaMemcpyDeviceToHost, st), "read svd status");
    cuda_check(cudaStreamSynchronize(st), "stream synchronize");
    ctx->last_sweeps = hs[1];
    if (hs[0] != 0) throw Failure(TNT_INTERNAL, "Jacobi SVD did not converge within the sweep limit");
  });
}

namespace {
// Grow the context's factorisation scratch to the plan's size (SVD, QR and
// eigh share the per-sector layout of tnt_fplan_work).
double* factor_work(tnt_ctx* ctx, const tnt_fplan_s* plan) {
  if (ctx->svd_work_elems < (size_t)plan->work_elems) {
    cudaFree(ctx->svd_work);
    ctx->svd_work = nullptr;
    ctx->svd_work_elems = 0;
    cuda_check(cudaMalloc(&ctx->svd_work, plan->work_elems * sizeof(double)), "cudaMalloc(factor work)");
    ctx->svd_work_elems = plan->work_elems;
  }
  return ctx->svd_work;
}
}  // namespace

tnt_status tnt_qr(tnt_ctx* ctx, const tnt_fplan* fplan, const double* a, double* q, double* r, void* stream) {
  return guarded([&] {
    enter(ctx);
    need(fplan != nullptr, "null plan");
    auto* plan = const_cast<tnt_fplan*>(fplan);
    const SvdTables& t = plan->p->tables;
    if (t.jobs.empty()) return;
    need(a && q && r, "null operand");
    auto dev = plan->lpt_on_device();
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    double* work = factor_work(ctx, plan);
    cudaStream_t st = (cudaStream_t)stream;
    cuda_check(launch_qr(dev.first, (int32_t)t.jobs.size(), a, q, r, work, dev.second, st), "qr kernel launch");
    cuda_check(cudaStreamSynchronize(st), "stream synchronize");
  });
}

tnt_status tnt_eigh(tnt_ctx* ctx, const tnt_fplan* fplan, const double* a, double* vecs, double* vals, double* mags,
                    void* stream) {
  return guarded([&] {
    enter(ctx);
    need(fplan != nullptr, "null plan");
    auto* plan = const_cast<tnt_fplan*>(fplan);
    const SvdTables& t = plan->p->tables;
    if (t.jobs.empty()) return;
    need(a && vecs && vals, "null operand");
    for (const SvdJob& j : t.jobs)
      need(j.m == j.n, "eigh requires an endomorphism (square coupled-sector blocks)");
    auto dev = plan->lpt_on_device();
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    double* work = factor_work(ctx, plan);
    cudaStream_t st = (cudaStream_t)stream;
    int64_t max_n = 0;
    for (const SvdJob& j : t.jobs) max_n = std::max<int64_t>(max_n, j.m);
    if (!eigh_on_chip(max_n)) {
      // Sectors beyond the on-chip two-sided Jacobi go through the batched
      // SVD of the shifted, positive semidefinite A + ||A||_F I.
      const size_t njobs = t.jobs.size();
      const size_t elems = (size_t)(t.a_size + t.u_size + t.s_size + t.v_size) + njobs + 1;
      if (ctx->eigh_tmp_elems < elems) {
        cudaFree(ctx->eigh_tmp);
        ctx->eigh_tmp = nullptr;
        ctx->eigh_tmp_elems = 0;
        cuda_check(cudaMalloc(&ctx->eigh_tmp, elems * sizeof(double)), "cudaMalloc(eigh scratch)");
        ctx->eigh_tmp_elems = elems;
      }
      double* b = ctx->eigh_tmp;
      double* u = b + t.a_size;
      double* sv = u + t.u_size;
      double* vh = sv + t.s_size;
      double* shift = vh + t.v_size;
      int32_t* bad = reinterpret_cast<int32_t*>(shift + njobs);
      cuda_check(cudaMemsetAsync(ctx->status, 0, 2 * sizeof(int32_t), st), "memset status");
      cuda_check(cudaMemsetAsync(bad, 0, sizeof(int32_t), st), "memset eigh flag");
      cuda_check(launch_eigh_by_svd(dev.first, plan->n_cluster, (int32_t)njobs, max_n, a, b, u, sv, vh, shift, bad,
                                    vecs, vals, mags, work, dev.second, ctx->status, st, plan->n_wide),
                 "eigh (shifted SVD) launch");
      int32_t hs[2] = {0, 0};
      cuda_check(cudaMemcpyAsync(&hs[0], ctx->status, sizeof(int32_t), cudaMemcpyDeviceToHost, st), "read svd status");
      cuda_check(cudaMemcpyAsync(&hs[1], bad, sizeof(int32_t), cudaMemcpyDeviceToHost, st), "read eigh flag");
      cuda_check(cudaStreamSynchronize(st), "stream synchronize");
      if (hs[1] != 0) throw std::invalid_argument("eigh requires Hermitian coupled-sector blocks");
      if (hs[0] != 0) throw Failure(TNT_INTERNAL, "Jacobi SVD did not converge within the sweep limit");
      return;
    }
    cuda_check(cudaMemsetAsync(ctx->status, 0, sizeof(int32_t), st), "memset status");
    cuda_check(launch_eigh(dev.first, (int32_t)t.jobs.size(), a, vecs, vals, mags, work, dev.second, ctx->status, st),
               "eigh kernel launch");
    int32_t hs = 0;
    cuda_check(cudaMemcpyAsync(&hs, ctx->status, sizeof(int32_t), cudaMemcpyDeviceToHost, st), "read eigh status");
    cuda_check(cudaStreamSynchronize(st), "stream synchronize");
    if (hs & 2) throw std::invalid_argument("eigh requires Hermitian coupled-sector blocks");
    if (hs != 0) throw Failure(TNT_INTERNAL, "Jacobi eigensolver did not converge within the sweep limit");
  });
}

tnt_status tnt_svd_static(const tnt_fplan* fplan, const double* a, double* u, double* s, double* vh, void* stream) {
  return guarded([&] {
    need(fplan != nullptr, "null plan");
    const SvdTables& t = fplan->p->tables;
    if (t.jobs.empty()) return;
    need(a && u && s && vh, "null operand");
    std::string why;
    cudaError_t e = svd_static(t.jobs, a, u, s, vh, (cudaStream_t)stream, why);
    if (e == cudaErrorInvalidValue && !why.empty()) throw std::invalid_argument(why);
    if (e == cudaErrorUnknown && !why.empty()) throw Failure(TNT_INTERNAL, why);
    cuda_check(e, "static-scratch svd");
  });
}

tnt_status tnt_truncate(tnt_ctx* ctx, const tnt_fplan* fplan, const double* s, int32_t policy, double p0, double p1,
                        const int64_t* space_ranks, int64_t* kept, double* err, void* stream) {
  return guarded([&] {
    enter(ctx);
    need(fplan && kept && err, "null argument");
    need(policy >= TNT_TRUNC_FULL && policy <= TNT_TRUNC_SPACE, "unknown truncation policy");
    if (policy == TNT_TRUNC_RANK) need(p0 >= 0.0, "rank must be non-negative");
    if (policy == TNT_TRUNC_TOL) need(p0 >= 0.0 && p1 >= 0.0 && std::isfinite(p0) && std::isfinite(p1), "bad tolerance");
    if (policy == TNT_TRUNC_DISCARD) need(p0 >= 0.0 && std::isfinite(p0), "bad discard tolerance");
    auto* plan = const_cast<tnt_fplan*>(fplan);
    const SvdTables& t = plan->p->tables;
    auto dev = plan->on_device();
    cudaStream_t st = (cudaStream_t)stream;
    int64_t* dranks = nullptr;
    if (policy == TNT_TRUNC_SPACE) {
      need(space_ranks != nullptr, "space truncation needs per-sector ranks");
      std::lock_guard<std::recursive_mutex> g(ctx->mu);
      // ranks travel in the staging buffer's head
      size_t need_elems = t.jobs.size() + 1;
      if (ctx->stage_elems < need_elems) {
        cudaFree(ctx->stage);
        ctx->stage = nullptr;
        ctx->stage_elems = 0;
        cuda_check(cudaMalloc(&ctx->stage, need_elems * sizeof(double)), "cudaMalloc(stage)");
        ctx->stage_elems = need_elems;
      }
      dranks = (int64_t*)ctx->stage;
      scratch_acquire(ctx, st);
      cuda_check(cudaMemcpyAsync(dranks, space_ranks, t.jobs.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st),
                 "H2D ranks");
      cuda_check(launch_truncate(dev.first, (int32_t)t.jobs.size(), s, policy, p0, p1, dranks, kept, err, st),
                 "truncate kernel launch");
      scratch_release(ctx, st);
      cuda_check(cudaStreamSynchronize(st), "stream synchronize");
      return;
    }
    cuda_check(launch_truncate(dev.first, (int32_t)t.jobs.size(), s, policy, p0, p1, dranks, kept, err, st),
               "truncate kernel launch");
  });
}

tnt_status tnt_truncate_async(tnt_ctx* ctx, const tnt_fplan* fplan, const double* s, int32_t policy, double p0,
                              double p1, const int64_t* space_ranks, int64_t* kept, double* err, void* stream) {
  return guarded([&] {
    enter(ctx);
    need(fplan && kept && err && s, "null argument");
    need(policy >= TNT_TRUNC_FULL && policy <= TNT_TRUNC_SPACE, "unknown truncation policy");
    if (policy == TNT_TRUNC_RANK) need(p0 >= 0.0, "rank must be non-negative");
    if (policy == TNT_TRUNC_TOL) need(p0 >= 0.0 && p1 >= 0.0 && std::isfinite(p0) && std::isfinite(p1), "bad tolerance");
    if (policy == TNT_TRUNC_DISCARD) need(p0 >= 0.0 && std::isfinite(p0), "bad discard tolerance");
    if (policy == TNT_TRUNC_SPACE) need(space_ranks != nullptr, "space truncation needs per-sector ranks");
    auto* plan = const_cast<tnt_fplan*>(fplan);
    const SvdTables& t = plan->p->tables;
    auto dev = plan->on_device();
    cuda_check(launch_truncate(dev.first, (int32_t)t.jobs.size(), s, policy, p0, p1,
                               policy == TNT_TRUNC_SPACE ? space_ranks : nullptr, kept, err, (cudaStream_t)stream),
               "truncate kernel launch");
  });
}

tnt_status tnt_xplan_concat(int32_t n, const tnt_xplan* const* plans, const int64_t* src_offs,
                            const int64_t* dst_offs, tnt_xplan** out) {
  return guarded([&] {
    need(out && n >= 0 && (n == 0 || (plans && src_offs && dst_offs)), "null argument");
    auto tp = std::make_shared<TransformPlan>();
    XformTables& T = tp->tables;
    for (int32_t i = 0; i < n; ++i) {
      need(plans[i] != nullptr, "null plan");
      const XformTables& t = plans[i]->p->tables;
      const int32_t sbase = (int32_t)T.src_entries.size(), dbase = (int32_t)T.dst_entries.size();
      const int32_t cbase = (int32_t)T.coef.size(), gbase = (int32_t)T.groups.size();
      for (XGroup g : t.groups) {
        g.src_first += sbase;
        g.dst_first += dbase;
        g.coef_off += cbase;
        T.groups.push_back(g);
      }
      for (XEntry e : t.src_entries) {
        e.offset += src_offs[i];
        T.src_entries.push_back(e);
      }
      for (XEntry e : t.dst_entries) {
        e.offset += dst_offs[i];
        T.dst_entries.push_back(e);
      }
      T.coef.insert(T.coef.end(), t.coef.begin(), t.coef.end());
      for (XTile tile : t.tiles) {
        tile.group += gbase;
        T.tiles.push_back(tile);
      }
      T.src_size = std::max(T.src_size, src_offs[i] + t.src_size);
      T.dst_size = std::max(T.dst_size, dst_offs[i] + t.dst_size);
      T.max_nsrc = std::max(T.max_nsrc, t.max_nsrc);
      T.max_ndst = std::max(T.max_ndst, t.max_ndst);
      tp->moved_elements += plans[i]->p->moved_elements;
    }
    auto x = new tnt_xplan_s();
    x->p = tp;
    *out = x;
  });
}

tnt_status tnt_cplan_concat(int32_t n, const tnt_cplan* const* plans, const int64_t* a_offs, const int64_t* b_offs,
                            const int64_t* c_offs, tnt_cplan** out) {
  return guarded([&] {
    need(out && n >= 0 && (n == 0 || (plans && a_offs && b_offs && c_offs)), "null argument");
    auto cp = std::make_shared<ComposePlan>();
    GemmTables& T = cp->tables;
    for (int32_t i = 0; i < n; ++i) {
      need(plans[i] != nullptr, "null plan");
      const GemmTables& t = plans[i]->p->tables;
      for (GemmJob j : t.jobs) {
        j.a_off += a_offs[i];
        j.b_off += b_offs[i];
        j.c_off += c_offs[i];
        T.jobs.push_back(j);
      }
      T.a_size = std::max(T.a_size, a_offs[i] + t.a_size);
      T.b_size = std::max(T.b_size, b_offs[i] + t.b_size);
      T.c_size = std::max(T.c_size, c_offs[i] + t.c_size);
      cp->flops += plans[i]->p->flops;
    }
    auto c = new tnt_cplan_s();
    c->p = cp;
    *out = c;
  });
}

tnt_status tnt_fplan_concat(int32_t n, const tnt_fplan* const* plans, const int64_t* a_offs, const int64_t* u_offs,
                            const int64_t* s_offs, const int64_t* v_offs, const int64_t* w_offs, tnt_fplan** out) {
  return guarded([&] {
    need(out && n >= 0 && (n == 0 || (plans && a_offs && u_offs && s_offs && v_offs)), "null argument");
    auto fp = std::make_shared<FactorPlan>();
    SvdTables& T = fp->tables;
    for (int32_t i = 0; i < n; ++i) {
      need(plans[i] != nullptr, "null plan");
      const SvdTables& t = plans[i]->p->tables;
      for (SvdJob j : t.jobs) {
        j.a_off += a_offs[i];
        j.u_off += u_offs[i];
        j.s_off += s_offs[i];
        j.v_off += v_offs[i];
        T.jobs.push_back(j);
      }
      T.a_size = std::max(T.a_size, a_offs[i] + t.a_size);
      T.u_size = std::max(T.u_size, u_offs[i] + t.u_size);
      T.s_size = std::max(T.s_size, s_offs[i] + t.s_size);
      T.v_size = std::max(T.v_size, v_offs[i] + t.v_size);
    }
    auto f = new tnt_fplan_s();
    f->p = fp;
    if (w_offs) {
      int64_t top = 0;
      for (int32_t i = 0; i < n; ++i) {
        for (size_t q = 0; q < plans[i]->work_off.size(); ++q) f->work_off.push_back(w_offs[i] + plans[i]->work_off[q]);
        top = std::max(top, w_offs[i] + plans[i]->work_elems);
      }
      f->work_elems = top;
    } else {
      int64_t off = 0;
      for (auto& j : T.jobs) {
        f->work_off.push_back(off);
        off += std::max(j.m, j.n) * j.k + j.k * j.k + 2 * j.k;
      }
      f->work_elems = off;
    }
    *out = f;
  });
}

tnt_status tnt_truncate_segments(tnt_ctx* ctx, const tnt_fplan* fplan, int32_t nseg, const int32_t* seg_first,
                                 const double* s, int32_t policy, double p0, double p1, const int64_t* space_ranks,
                                 int64_t* kept, double* err, void* stream) {
  return guarded([&] {
    enter(ctx);
    need(fplan && seg_first && kept && err && s, "null argument");
    need(nseg >= 0, "negative segment count");
    need(policy >= TNT_TRUNC_FULL && policy <= TNT_TRUNC_SPACE, "unknown truncation policy");
    auto* plan = const_cast<tnt_fplan*>(fplan);
    const int32_t nj = (int32_t)plan->p->tables.jobs.size();
    need(seg_first[0] == 0 && seg_first[nseg] == nj, "segments must cover every sector");
    for (int32_t i = 0; i < nseg; ++i) need(seg_first[i] <= seg_first[i + 1], "segments must be ascending");
    auto dev = plan->on_device();
    cudaStream_t st = (cudaStream_t)stream;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    const size_t need_elems = (size_t)(nseg + 1) + (policy == TNT_TRUNC_SPACE ? (size_t)nj : 0);
    if (ctx->stage_elems < need_elems) {
      cudaFree(ctx->stage);
      ctx->stage = nullptr;
      ctx->stage_elems = 0;
      cuda_check(cudaMalloc(&ctx->stage, need_elems * sizeof(double)), "cudaMalloc(stage)");
      ctx->stage_elems = need_elems;
    }
    int64_t* dseg = (int64_t*)ctx->stage;
    std::vector<int64_t> seg64(seg_first, seg_first + nseg + 1);
    scratch_acquire(ctx, st);
    cuda_check(cudaMemcpyAsync(dseg, seg64.data(), seg64.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st),
               "H2D segments");
    int64_t* dranks = nullptr;
    if (policy == TNT_TRUNC_SPACE) {
      need(space_ranks != nullptr, "space truncation needs per-sector ranks");
      dranks = dseg + nseg + 1;
      cuda_check(cudaMemcpyAsync(dranks, space_ranks, nj * sizeof(int64_t), cudaMemcpyHostToDevice, st), "H2D ranks");
    }
    cuda_check(launch_truncate_segments(dev.first, nseg, dseg, s, policy, p0, p1, dranks, kept, err, st),
               "segmented truncate launch");
    scratch_release(ctx, st);
    cuda_check(cudaStreamSynchronize(st), "stream synchronize");
  });
}

tnt_status tnt_copy_segments(tnt_ctx* ctx, int64_t nseg, const int64_t* table, const double* src, double* dst,
                             const double* scales, void* stream) {
  return guarded([&] {
    enter(ctx);
    need(nseg >= 0, "negative segment count");
    if (nseg == 0) return;
    need(table && src && dst, "null argument");
    std::vector<SegCopy> segs(nseg);
    for (int64_t i = 0; i < nseg; ++i) {
      const int64_t* r = table + 7 * i;
      SegCopy sc{r[0], r[1], r[2], r[3], r[4], r[5], r[6]};
      need(sc.rows >= 0 && sc.cols >= 0 && sc.src_off >= 0 && sc.dst_off >= 0, "negative extent or offset");
      need(sc.src_ld >= sc.rows && sc.dst_ld >= sc.rows, "leading dimension smaller than rows");
      need(sc.scale_off < 0 || scales != nullptr, "row scaling needs scales");
      segs[i] = sc;
    }
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    if (ctx->seg_stage_elems < (size_t)nseg) {
      cudaFree(ctx->seg_stage);
      ctx->seg_stage = nullptr;
      ctx->seg_stage_elems = 0;
      cuda_check(cudaMalloc(&ctx->seg_stage, (size_t)nseg * sizeof(SegCopy)), "cudaMalloc(segment table)");
      ctx->seg_stage_elems = (size_t)nseg;
    }
    cudaStream_t st = (cudaStream_t)stream;
    scratch_acquire(ctx, st);
    cuda_check(cudaMemcpyAsync(ctx->seg_stage, segs.data(), (size_t)nseg * sizeof(SegCopy), cudaMemcpyHostToDevice, st),
               "H2D segment table");
    cuda_check(launch_segcopy(ctx->seg_stage, nseg, src, dst, scales, st), "segment copy launch");
    scratch_release(ctx, st);
  });
}

tnt_status tnt_copy_segments_async(tnt_ctx* ctx, int64_t nseg, const int64_t* table, const double* src, double* dst,
                                   const double* scales, void* stream) {
  return guarded([&] {
    enter(ctx);
    need(nseg >= 0, "negative segment count");
    if (nseg == 0) return;
    need(table && src && dst, "null argument");
    static_assert(sizeof(SegCopy) == 7 * sizeof(int64_t), "segment records are 7 int64");
    cuda_check(launch_segcopy(reinterpret_cast<const SegCopy*>(table), nseg, src, dst, scales, (cudaStream_t)stream),
               "segment copy launch");
  });
}

tnt_status tnt_wdot(tnt_ctx* ctx, const tnt_fplan* fplan, int32_t k, const double* V, int64_t ldv, const double* y,
                    double* out, void* stream) {
  return guarded([&] {
    enter(ctx);
    need(fplan != nullptr, "null plan");
    need(k >= 0 && k <= 64, "k must be 0..64");
    if (k == 0) return;
    need(V && y && out, "null operand");
    need(k == 1 || ldv >= fplan->p->tables.a_size, "ldv smaller than the vector length");
    auto* plan = const_cast<tnt_fplan*>(fplan);
    auto dev = plan->on_device();
    FplanChunks ch = plan->chunks_on_device();
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    const size_t need_elems = (size_t)std::max<int64_t>(1, ch.n) * (size_t)k;
    if (ctx->dot_part_elems < need_elems) {
      cudaFree(ctx->dot_part);
      ctx->dot_part = nullptr;
      ctx->dot_part_elems = 0;
      cuda_check(cudaMalloc(&ctx->dot_part, need_elems * sizeof(double)), "cudaMalloc(dot partials)");
      ctx->dot_part_elems = need_elems;
    }
    scratch_acquire(ctx, (cudaStream_t)stream);
    cuda_check(launch_wdot(dev.first, (int32_t)plan->p->tables.jobs.size(), ch.sector, ch.start, ch.n, k, V, ldv, y,
                           ctx->dot_part, out, (cudaStream_t)stream),
               "weighted dot launch");
    scratch_release(ctx, (cudaStream_t)stream);
  });
}

tnt_status tnt_axpy_many(tnt_ctx* ctx, int64_t n, int32_t k, const double* V, int64_t ldv, const double* coef,
                         double a, const double* a_dev, double* y, void* stream) {
  return guarded([&] {
    enter(ctx);
    need(n >= 0 && k >= 0, "negative size");
    if (n == 0) return;
    need(y != nullptr && (k == 0 || (V && coef)), "null operand");
    need(k <= 1 || ldv >= n, "ldv smaller than n");
    cuda_check(launch_axpy_many(n, k, V, ldv, coef, a, a_dev, y, (cudaStream_t)stream), "axpy launch");
  });
}

tnt_status tnt_symeig(tnt_ctx* ctx, int32_t m, const double* A, double* evals, double* evecs, void* stream) {
  return guarded([&] {
    enter(ctx);
    need(m >= 0 && m <= 48, "m must be 0..48");
    if (m == 0) return;
    need(A && evals && evecs, "null operand");
    cudaStream_t st = (cudaStream_t)stream;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);  // the status words are the context's
    cuda_check(cudaMemsetAsync(ctx->status, 0, sizeof(int32_t), st), "memset status");
    cuda_check(launch_symeig(m, A, evals, evecs, ctx->status, st), "symeig launch");
    int32_t hs = 0;
    cuda_check(cudaMemcpyAsync(&hs, ctx->status, sizeof(int32_t), cudaMemcpyDeviceToHost, st), "read status");
    cuda_check(cudaStreamSynchronize(st), "stream synchronize");
    if (hs != 0) throw Failure(TNT_INTERNAL, "symmetric eigensolver did not converge");
  });
}

}  // extern "C"

// ---- network schedules ---------------------------------------------------------
// A compiled pairwise contraction schedule (tenet-network/src/network.rs:919-941)
// lowered to device work.  Every operand transform a step needs (adjoint of a
// conjugated input, the pending output permutations of the step that produced
// it, the permute into (open ; contracted) or (contracted ; open) order and the
// supertrace twist) is multiplied into ONE recoupling plan, so each
// intermediate is written once by a compose and read once by a transform (or
// read directly by the next compose when the chain is a no-op).
// Intermediates live in one caller-provided workspace at offsets planned from
// their lifetimes.

namespace {

struct NetBuf {
  int64_t elems = 0;
  int input = -1;       // >= 0: the caller's input pointer
  bool output = false;  // the caller's output pointer
  int64_t offset = 0;   // elements into the workspace
  int def = -1, last = -1;
};

struct NetOp {
  int kind = 0;  // 0 transform, 1 compose, 2 device copy
  std::shared_ptr<tnt_xplan_s> x;
  std::shared_ptr<tnt_cplan_s> c;
  int src = -1, dst = -1, a = -1, b = -1;
};

struct NetSlot {
  bool live = false;
  int buf = -1;
  std::shared_ptr<Space> base;          // space of the stored payload
  std::vector<TransformStep> pending;   // steps not yet applied to it
  std::shared_ptr<Space> logical;       // space after the pending steps
};

TransformStep permute_step(const std::vector<int>& p1, const std::vector<int>& p2, int supertrace = -1) {
  TransformStep st;
  st.kind = XK_PERMUTE;
  st.p1 = p1;
  st.p2 = p2;
  st.supertrace = supertrace;
  return st;
}

}  // namespace

struct tnt_nplan_s {
  std::vector<std::shared_ptr<Space>> inputs;
  std::vector<NetBuf> bufs;
  std::vector<NetOp> ops;
  std::shared_ptr<Space> out;
  int64_t work_elems = 0;
  double flops = 0;
  int64_t moved = 0;  // bytes moved by the transforms per execution
};

namespace {

int net_new_buf(tnt_nplan_s& p, int64_t elems) {
  NetBuf b;
  b.elems = elems;
  p.bufs.push_back(b);
  return (int)p.bufs.size() - 1;
}

// Apply `slot.pending + extra` (no-op steps dropped) and return the buffer and
// space holding the result; no op when nothing is left to do.
std::pair<int, std::shared_ptr<Space>> net_materialize(tnt_nplan_s& p, NetSlot& slot,
                                                       const std::vector<TransformStep>& extra) {
  std::vector<TransformStep> all = slot.pending;
  all.insert(all.end(), extra.begin(), extra.end());
  std::vector<TransformStep> steps;
  std::shared_ptr<Space> cur = slot.base;
  for (auto& st : all) {
    auto next = chain_spaces(cur, {st}).back();
    if (!step_is_noop(*cur, st)) steps.push_back(st);
    cur = next;
  }
  if (steps.empty()) return {slot.buf, slot.base};
  auto plan = std::make_shared<tnt_xplan_s>();
  plan->p = make_transform_chain(slot.base, steps);
  NetOp op;
  op.kind = 0;
  op.x = plan;
  op.src = slot.buf;
  op.dst = net_new_buf(p, plan->p->dst->size);
  p.moved += plan->p->moved_elements * (int64_t)sizeof(double);
  p.ops.push_back(op);
  return {op.dst, plan->p->dst};
}

void net_check_axes(const std::vector<int>& axes, int n, const char* what) {
  std::vector<int> seen(n, 0);
  for (int a : axes)
    if (a < 0 || a >= n || seen[a]++) throw std::invalid_argument(what);
}

// Lifetimes, then first-fit offsets (256-byte aligned) in op order.
void net_plan_memory(tnt_nplan_s& p) {
  for (size_t i = 0; i < p.ops.size(); ++i) {
    const NetOp& op = p.ops[i];
    for (int r : {op.src, op.a, op.b})
      if (r >= 0) p.bufs[r].last = (int)i;
    if (op.dst >= 0 && p.bufs[op.dst].def < 0) p.bufs[op.dst].def = (int)i;
  }
  const int64_t align = 32;  // doubles
  std::vector<std::pair<int64_t, int64_t>> live;  // (offset, end) of live intermediates
  std::vector<int> live_ids;
  int64_t peak = 0;
  for (size_t i = 0; i < p.ops.size(); ++i) {
    int d = p.ops[i].dst;
    if (d >= 0 && p.bufs[d].input < 0 && !p.bufs[d].output && p.bufs[d].def == (int)i) {
      int64_t need_elems = (p.bufs[d].elems + align - 1) / align * align;
      std::vector<std::pair<int64_t, int64_t>> sorted = live;
      std::sort(sorted.begin(), sorted.end());
      int64_t at = 0;
      for (auto& iv : sorted) {
        if (iv.first - at >= need_elems) break;
        at = std::max(at, iv.second);
      }
      p.bufs[d].offset = at;
      live.push_back({at, at + need_elems});
      live_ids.push_back(d);
      peak = std::max(peak, at + need_elems);
    }
    for (size_t k = 0; k < live_ids.size();) {
      if (p.bufs[live_ids[k]].last <= (int)i && p.bufs[live_ids[k]].last >= 0) {
        live.erase(live.begin() + k);
        live_ids.erase(live_ids.begin() + k);
      } else {
        ++k;
      }
    }
  }
  p.work_elems = peak;
}

void net_throw_status(tnt_status s) {
  if (s != TNT_OK) throw Failure(s, g_error);
}

}  // namespace

extern "C" {

tnt_status tnt_network_plan(int32_t n_inputs, const tnt_space* const* inputs, const uint8_t* conj, int32_t n_steps,
                            const int32_t* steps, int64_t steps_len, int32_t final_slot, const int32_t* final_perm,
                            int64_t final_perm_len, tnt_nplan** out) {
  return guarded([&] {
    need(out != nullptr, "null argument");
    need(n_inputs >= 1 && inputs != nullptr, "a network needs at least one input");
    need(n_steps >= 0 && (n_steps == 0 || (steps && steps_len > 0)), "null step program");
    auto plan = std::make_unique<tnt_nplan_s>();
    const int nslots = n_inputs + n_steps;
    std::vector<NetSlot> slots(nslots);
    for (int i = 0; i < n_inputs; ++i) {
      need(inputs[i] != nullptr, "null input space");
      auto sp = inputs[i]->s;
      need(i == 0 || sp->rule == plan->inputs[0]->rule, "inputs use different fusion rules");
      plan->inputs.push_back(sp);
      NetSlot& s = slots[i];
      s.live = true;
      s.buf = net_new_buf(*plan, sp->size);
      plan->bufs[s.buf].input = i;
      s.base = sp;
      if (conj && conj[i]) {
        TransformStep adj;
        adj.kind = XK_ADJOINT;
        s.pending.push_back(adj);
        s.logical = chain_spaces(sp, s.pending).back();
      } else {
        s.logical = sp;
      }
    }
    int64_t pos = 0;
    auto next = [&]() -> int32_t {
      if (pos >= steps_len) throw std::invalid_argument("step program ends early");
      return steps[pos++];
    };
    auto take_list = [&](int32_t n) {
      if (n < 0 || n > 64) throw std::invalid_argument("bad axis count in step program");
      std::vector<int> v;
      for (int32_t i = 0; i < n; ++i) v.push_back(next());
      return v;
    };
    for (int32_t si = 0; si < n_steps; ++si) {
      int ls = next(), rs = next(), res = next();
      need(ls >= 0 && ls < nslots && rs >= 0 && rs < nslots && res >= 0 && res < nslots, "slot out of range");
      need(ls != rs, "a step contracts a slot with itself");
      need(slots[ls].live && slots[rs].live, "operand slot is empty or already consumed");
      int32_t k = next();
      auto la = take_list(k), ra = take_list(k);
      auto oa = take_list(next());
      int32_t npc = next();
      bool has_perm = npc >= 0;
      std::vector<int> pc, pd;
      if (has_perm) {
        pc = take_list(npc);
        pd = take_list(next());
      }
      NetSlot& L = slots[ls];
      NetSlot& R = slots[rs];
      int nl = L.logical->n1() + L.logical->n2(), nr = R.logical->n1() + R.logical->n2();
      net_check_axes(la, nl, "lhs contraction axes are not distinct axes of the operand");
      net_check_axes(ra, nr, "rhs contraction axes are not distinct axes of the operand");
      std::vector<int> open_a, open_b;
      for (int i = 0; i < nl; ++i)
        if (std::find(la.begin(), la.end(), i) == la.end()) open_a.push_back(i);
      for (int i = 0; i < nr; ++i)
        if (std::find(ra.begin(), ra.end(), i) == ra.end()) open_b.push_back(i);
      int nout = (int)(open_a.size() + open_b.size());
      need((int)oa.size() == nout, "contract output axes must list every open axis");
      net_check_axes(oa, nout, "contract output axes are not a permutation");
      auto A = net_materialize(*plan, L, {permute_step(open_a, la)});
      auto B = net_materialize(*plan, R, {permute_step(ra, open_b, k)});
      auto cp = std::make_shared<tnt_cplan_s>();
      cp->p = make_compose(A.second, B.second);
      NetOp op;
      op.kind = 1;
      op.c = cp;
      op.a = A.first;
      op.b = B.first;
      op.dst = net_new_buf(*plan, cp->p->dst->size);
      plan->flops += cp->p->flops;
      plan->ops.push_back(op);
      L = NetSlot{};
      R = NetSlot{};
      NetSlot& C = slots[res];
      need(!C.live, "result slot is still holding a tensor");
      C.live = true;
      C.buf = op.dst;
      C.base = cp->p->dst;
      int na = (int)open_a.size();
      std::vector<int> o1(oa.begin(), oa.begin() + na), o2(oa.begin() + na, oa.end());
      C.pending.push_back(permute_step(o1, o2));
      if (has_perm) C.pending.push_back(permute_step(pc, pd));
      C.logical = chain_spaces(C.base, C.pending).back();
    }
    need(pos == steps_len, "step program has trailing entries");
    need(final_slot >= 0 && final_slot < nslots && slots[final_slot].live, "final slot holds no tensor");
    for (int i = 0; i < nslots; ++i)
      need(i == final_slot || !slots[i].live, "a tensor is left uncontracted outside the final slot");
    NetSlot& F = slots[final_slot];
    std::vector<TransformStep> fin;
    if (final_perm_len > 0) {
      need(final_perm != nullptr, "null final permutation");
      int64_t q = 0;
      auto fnext = [&]() -> int32_t {
        if (q >= final_perm_len) throw std::invalid_argument("final permutation ends early");
        return final_perm[q++];
      };
      int32_t nc = fnext();
      need(nc >= 0 && nc <= 64, "bad final codomain count");
      std::vector<int> c1, c2;
      for (int32_t i = 0; i < nc; ++i) c1.push_back(fnext());
      int32_t nd = fnext();
      need(nd >= 0 && nd <= 64, "bad final domain count");
      for (int32_t i = 0; i < nd; ++i) c2.push_back(fnext());
      need(q == final_perm_len, "final permutation has trailing entries");
      fin.push_back(permute_step(c1, c2));
    }
    size_t nops = plan->ops.size();
    auto R = net_materialize(*plan, F, fin);
    if (plan->ops.size() > nops) {
      plan->bufs[R.first].output = true;  // the last transform writes the caller's output
    } else if (plan->bufs[R.first].input < 0) {
      plan->bufs[R.first].output = true;  // the last compose writes it
    } else {
      NetOp cp;
      cp.kind = 2;
      cp.src = R.first;
      cp.dst = net_new_buf(*plan, R.second->size);
      plan->bufs[cp.dst].output = true;
      plan->ops.push_back(cp);
    }
    plan->out = R.second;
    net_plan_memory(*plan);
    *out = plan.release();
  });
}

void tnt_nplan_destroy(tnt_nplan* plan) { delete plan; }

tnt_status tnt_nplan_output_space(const tnt_nplan* plan, tnt_space** out) {
  return guarded([&] {
    need(plan && out, "null argument");
    *out = new tnt_space{plan->out};
  });
}

tnt_status tnt_nplan_info(const tnt_nplan* plan, int64_t* n_transforms, int64_t* n_composes, double* flops,
                          int64_t* bytes_moved, int64_t* workspace_elems) {
  return guarded([&] {
    need(plan != nullptr, "null plan");
    int64_t nx = 0, nc = 0;
    for (auto& op : plan->ops) (op.kind == 1 ? nc : nx) += 1;
    if (n_transforms) *n_transforms = nx;
    if (n_composes) *n_composes = nc;
    if (flops) *flops = plan->flops;
    if (bytes_moved) *bytes_moved = plan->moved;
    if (workspace_elems) *workspace_elems = plan->work_elems;
  });
}

tnt_status tnt_nplan_workspace_bytes(const tnt_nplan* plan, int32_t precision, int32_t slices, size_t* bytes) {
  return guarded([&] {
    need(plan && bytes, "null argument");
    size_t scratch = 0;
    if (precision == TNT_PREC_BF16X || precision == TNT_PREC_INT8X) {
      for (auto& op : plan->ops) {
        if (op.kind != 1) continue;
        size_t b = 0;
        net_throw_status(tnt_cplan_scratch_bytes(op.c.get(), 1, precision, slices, &b));
        scratch = std::max(scratch, b);
      }
    }
    *bytes = (size_t)plan->work_elems * sizeof(double) + (scratch + 255) / 256 * 256;
  });
}

tnt_status tnt_network_execute(tnt_ctx* ctx, const tnt_nplan* plan, int32_t n_inputs, const double* const* inputs,
                               double* output, void* workspace, size_t workspace_bytes, int32_t precision,
                               int32_t slices, void* stream) {
  return guarded([&] {
    need(ctx && plan, "null argument");
    need(n_inputs == (int32_t)plan->inputs.size() && inputs != nullptr, "input count differs from the plan");
    for (int i = 0; i < n_inputs; ++i) need(plan->inputs[i]->size == 0 || inputs[i], "null input payload");
    need(plan->out->size == 0 || output, "null output payload");
    size_t need_bytes = 0;
    net_throw_status(tnt_nplan_workspace_bytes(plan, precision, slices, &need_bytes));
    need(need_bytes == 0 || (workspace != nullptr && workspace_bytes >= need_bytes), "workspace too small");
    char* ws = (char*)workspace;
    const size_t work_bytes = (size_t)plan->work_elems * sizeof(double);
    auto ptr = [&](int b) -> double* {
      const NetBuf& nb = plan->bufs[b];
      if (nb.input >= 0) return const_cast<double*>(inputs[nb.input]);
      if (nb.output) return output;
      return (double*)(ws + nb.offset * (int64_t)sizeof(double));
    };
    cudaStream_t st = (cudaStream_t)stream;
    for (auto& op : plan->ops) {
      if (op.kind == 0) {
        net_throw_status(tnt_transform(ctx, op.x.get(), ptr(op.dst), ptr(op.src), 1.0, 0.0, stream));
      } else if (op.kind == 1) {
        net_throw_status(tnt_compose_ws(ctx, op.c.get(), 1, ptr(op.dst), 0, ptr(op.a), 0, ptr(op.b), 0, 1.0, 0.0,
                                        precision, slices, ws ? ws + work_bytes : nullptr,
                                        workspace_bytes > work_bytes ? workspace_bytes - work_bytes : 0, stream));
      } else {
        size_t n = (size_t)plan->bufs[op.dst].elems * sizeof(double);
        if (n) cuda_check(cudaMemcpyAsync(ptr(op.dst), ptr(op.src), n, cudaMemcpyDeviceToDevice, st), "copy");
      }
    }
  });
}

}  // extern "C"
