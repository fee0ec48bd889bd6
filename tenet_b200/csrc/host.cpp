// Host structure compiler: sectors, fusion trees, layouts and recoupling plans.
// See host.hpp for the reference correspondence of each part.
#include "host.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <stdexcept>

namespace tnt {

// ---------------------------------------------------------------------------
// Sectors and symbols
// ---------------------------------------------------------------------------

static uint64_t u1_zigzag(int32_t q) { return (uint64_t)(((uint32_t)q << 1) ^ (uint32_t)(q >> 31)); }

static int packed_bits(FactorKind k) {
  switch (k) {
    case FK_U1: return 32;   // U1SectorLayout (tenet-sectors/src/algebra.rs:1530-1545)
    case FK_SU2: return 8;   // Su2SectorLayout (algebra.rs:1547-1562)
    default: return 1;       // Fz2SectorLayout (algebra.rs:1513-1528)
  }
}

bool Rule::fermionic() const {
  for (int i = 0; i < nf; ++i)
    if (kind[i] == FK_FZ2) return true;
  return false;
}

bool Rule::unique() const {
  for (int i = 0; i < nf; ++i)
    if (kind[i] == FK_SU2 || kind[i] == FK_TABLE) return false;
  return true;
}

bool Rule::operator==(const Rule& o) const {
  if (nf != o.nf || codec != o.codec) return false;
  for (int i = 0; i < nf; ++i)
    if (kind[i] != o.kind[i]) return false;
  if (kind[0] == FK_TABLE) return table && o.table && table->identity == o.table->identity;
  return true;
}

uint64_t Rule::id(const Sector& s) const {
  uint64_t leaf[kMaxFactors];
  for (int i = 0; i < nf; ++i) leaf[i] = kind[i] == FK_U1 ? u1_zigzag(s.v[i]) : (uint64_t)s.v[i];  // table: the label
  if (nf == 1) return leaf[0];
  if (codec == CODEC_PACKED) {  // PackedProductCodec (algebra.rs:1581-1620): first factor in the low bits
    uint64_t out = 0;
    int shift = 0;
    for (int i = 0; i < nf; ++i) {
      out |= leaf[i] << shift;
      shift += packed_bits(kind[i]);
    }
    return out;
  }
  uint64_t out = leaf[0];  // left-nested Cantor pairing (algebra.rs:1436-1447)
  for (int i = 1; i < nf; ++i) {
    uint64_t sum = out + leaf[i];
    out = sum * (sum + 1) / 2 + out;
  }
  return out;
}

Sector Rule::dual(const Sector& s) const {
  Sector d = s;
  if (kind[0] == FK_TABLE) {
    d.v[0] = table->dual[s.v[0]];
    return d;
  }
  for (int i = 0; i < nf; ++i)
    if (kind[i] == FK_U1) d.v[i] = -s.v[i];
  return d;
}

// Product channels: Cartesian product with the first factor fastest
// (tenet-sectors/src/product_rule.rs:287-302); SU(2) channels ascending.
void Rule::channels(const Sector& a, const Sector& b, std::vector<Sector>& out) const {
  out.clear();
  if (kind[0] == FK_TABLE) {  // ascending label = ascending SectorId
    for (int c = 0; c < table->n; ++c)
      if (table->nsym(a.v[0], b.v[0], c)) {
        Sector x;
        x.v[0] = c;
        out.push_back(x);
      }
    return;
  }
  int lo[kMaxFactors], hi[kMaxFactors], step[kMaxFactors];
  for (int i = 0; i < nf; ++i) {
    switch (kind[i]) {
      case FK_U1: lo[i] = hi[i] = a.v[i] + b.v[i]; step[i] = 1; break;
      case FK_SU2: lo[i] = std::abs(a.v[i] - b.v[i]); hi[i] = a.v[i] + b.v[i]; step[i] = 2; break;
      default: lo[i] = hi[i] = a.v[i] ^ b.v[i]; step[i] = 1; break;
    }
  }
  Sector cur;
  for (int i = 0; i < nf; ++i) cur.v[i] = lo[i];
  while (true) {
    out.push_back(cur);
    int i = 0;
    for (; i < nf; ++i) {
      if (cur.v[i] + step[i] <= hi[i]) {
        cur.v[i] += step[i];
        break;
      }
      cur.v[i] = lo[i];
    }
    if (i == nf) break;
  }
}

bool Rule::nsym(const Sector& a, const Sector& b, const Sector& c) const {
  if (kind[0] == FK_TABLE) return table->nsym(a.v[0], b.v[0], c.v[0]);
  for (int i = 0; i < nf; ++i) {
    switch (kind[i]) {
      case FK_U1:
        if (c.v[i] != a.v[i] + b.v[i]) return false;
        break;
      case FK_SU2:
        if (c.v[i] < std::abs(a.v[i] - b.v[i]) || c.v[i] > a.v[i] + b.v[i] || ((a.v[i] + b.v[i] + c.v[i]) & 1))
          return false;
        break;
      default:
        if (c.v[i] != (a.v[i] ^ b.v[i])) return false;
    }
  }
  return true;
}

double Rule::dim(const Sector& a) const {
  if (kind[0] == FK_TABLE) return table->dims[a.v[0]];
  double d = 1.0;
  for (int i = 0; i < nf; ++i)
    if (kind[i] == FK_SU2) d *= (double)(a.v[i] + 1);
  return d;
}

double Rule::twist(const Sector& a) const {
  double t = 1.0;  // fermion parity twist (abelian.rs:503-509)
  for (int i = 0; i < nf; ++i)
    if (kind[i] == FK_FZ2 && a.v[i] == 1) t = -t;
  return t;
}

double Rule::fs(const Sector& a) const {
  if (kind[0] == FK_TABLE) return table->fs[a.v[0]];
  double t = 1.0;  // SU(2): (-1)^(2j) (su2.rs:366-369)
  for (int i = 0; i < nf; ++i)
    if (kind[i] == FK_SU2 && (a.v[i] & 1)) t = -t;
  return t;
}

double Rule::R(const Sector& a, const Sector& b, const Sector& c) const {
  if (kind[0] == FK_TABLE) {
    const TableData& t = *table;
    return t.nsym(a.v[0], b.v[0], c.v[0]) ? t.R[((size_t)a.v[0] * t.n + b.v[0]) * t.n + c.v[0]] : 0.0;
  }
  double r = 1.0;
  for (int i = 0; i < nf; ++i) {
    if (kind[i] == FK_FZ2) {
      if (a.v[i] == 1 && b.v[i] == 1) r = -r;  // abelian.rs:477-484
    } else if (kind[i] == FK_SU2) {
      int x = a.v[i], y = b.v[i], z = c.v[i];
      if (z < std::abs(x - y) || z > x + y || ((x + y + z) & 1)) return 0.0;
      if (((x + y - z) / 2) & 1) r = -r;  // (-1)^(ja + jb - jc)
    }
  }
  return r;
}

double Rule::F(const Sector& a, const Sector& b, const Sector& c, const Sector& d, const Sector& e,
               const Sector& f) const {
  if (kind[0] == FK_TABLE) return table->f(a.v[0], b.v[0], c.v[0], d.v[0], e.v[0], f.v[0]);
  double v = 1.0;
  for (int i = 0; i < nf; ++i) {
    if (kind[i] == FK_SU2) {
      v *= su2_fsymbol(a.v[i], b.v[i], c.v[i], d.v[i], e.v[i], f.v[i]);
      if (v == 0.0) return 0.0;
    }
  }
  return v;
}

// B(a,b,c) = sqrt(d_a d_b / d_c) F(a, b, dual b, a; c, 1)  (algebra.rs:615-623)
double Rule::B(const Sector& a, const Sector& b, const Sector& c) const {
  return std::sqrt(dim(a)) * std::sqrt(dim(b)) / std::sqrt(dim(c)) * F(a, b, dual(b), a, c, vacuum());
}

// --- checked table providers ------------------------------------------------
//
// The laws a table must satisfy before any plan is compiled on it, in the
// F(a, b, c; d; e, f) convention the recoupling code uses (the same forms hold
// for the built-in SU(2) symbols):
//   vacuum:     N(0, a, a) = N(a, 0, a) = N(a, dual a, 0) = 1, dual(dual a) = a;
//   no outer multiplicity (N in {0, 1});
//   dimensions: d_a d_b = sum_c N(a, b, c) d_c;
//   F moves:    every F(a, b, c; d) block is square and orthogonal;
//   pentagon:   F(f,c,d;e;g,l) F(a,b,l;e;f,k) = sum_h F(a,b,c;g;f,h) F(a,h,d;e;g,k) F(b,c,d;k;h,l);
//   symmetric braiding: R(a, b, c) R(b, a, c) = 1;
//   hexagon:    R(c,a,e) F(a,c,b;d;e,g) R(c,b,g) = sum_f F(c,a,b;d;e,f) R(c,f,d) F(a,b,c;d;f,g);
//   Frobenius-Schur: fs_a = d_a F(a, dual a, a; a; 0, 0) for self-dual a.
void check_table(const TableData& t, double tol) {
  const int n = t.n;
  auto fail = [](const std::string& what) { throw std::invalid_argument("table provider: " + what); };
  auto R = [&](int a, int b, int c) { return t.R[((size_t)a * n + b) * n + c]; };
  for (int a = 0; a < n; ++a) {
    if (t.dual[a] < 0 || t.dual[a] >= n || t.dual[t.dual[a]] != a) fail("dual is not an involution");
    if (!t.nsym(0, a, a) || !t.nsym(a, 0, a)) fail("vacuum law");
    if (!t.nsym(a, t.dual[a], 0)) fail("dual law: a (x) dual(a) must contain the vacuum");
    for (int c = 0; c < n; ++c)
      if (c != a && (t.nsym(0, a, c) || t.nsym(a, 0, c))) fail("vacuum law");
    if (!(t.dims[a] > 0.0) || !std::isfinite(t.dims[a])) fail("quantum dimensions must be positive");
  }
  if (t.dual[0] != 0) fail("the vacuum must be self-dual");
  for (uint8_t v : t.N)
    if (v > 1) fail("outer multiplicity (N > 1) is not supported: the provider must be multiplicity free");
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b) {
      double s = 0.0;
      for (int c = 0; c < n; ++c) s += t.nsym(a, b, c) ? t.dims[c] : 0.0;
      if (std::fabs(s - t.dims[a] * t.dims[b]) > tol * t.dims[a] * t.dims[b]) fail("dimensions");
    }
  std::vector<int> es, fs;
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b)
      for (int c = 0; c < n; ++c)
        for (int d = 0; d < n; ++d) {
          es.clear();
          fs.clear();
          for (int e = 0; e < n; ++e)
            if (t.nsym(a, b, e) && t.nsym(e, c, d)) es.push_back(e);
          for (int f = 0; f < n; ++f)
            if (t.nsym(b, c, f) && t.nsym(a, f, d)) fs.push_back(f);
          if (es.size() != fs.size()) fail("F block not square");
          for (size_t i = 0; i < es.size(); ++i)
            for (size_t j = 0; j < es.size(); ++j) {
              double s = 0.0;
              for (size_t k = 0; k < fs.size(); ++k) s += t.f(a, b, c, d, es[i], fs[k]) * t.f(a, b, c, d, es[j], fs[k]);
              if (std::fabs(s - (i == j ? 1.0 : 0.0)) > tol) fail("F moves are not orthogonal");
            }
        }
  // both sides vanish unless f in a (x) b, g in f (x) c and e in g (x) d
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b)
      for (int f = 0; f < n; ++f)
        if (t.nsym(a, b, f))
          for (int c = 0; c < n; ++c)
            for (int g = 0; g < n; ++g)
              if (t.nsym(f, c, g))
                for (int d = 0; d < n; ++d)
                  for (int e = 0; e < n; ++e)
                    if (t.nsym(g, d, e))
                      for (int k = 0; k < n; ++k)
                        for (int l = 0; l < n; ++l) {
                    const double lhs = t.f(f, c, d, e, g, l) * t.f(a, b, l, e, f, k);
                    double rhs = 0.0;
                    for (int h = 0; h < n; ++h) rhs += t.f(a, b, c, g, f, h) * t.f(a, h, d, e, g, k) * t.f(b, c, d, k, h, l);
                    if (std::fabs(lhs - rhs) > tol) fail("pentagon equation");
                  }
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b)
      for (int c = 0; c < n; ++c)
        if (t.nsym(a, b, c) && std::fabs(R(a, b, c) * R(b, a, c) - 1.0) > tol)
          fail("braiding must be symmetric (R(a,b,c) R(b,a,c) = 1)");
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b)
      for (int c = 0; c < n; ++c)
        for (int d = 0; d < n; ++d)
          for (int e = 0; e < n; ++e)
            for (int g = 0; g < n; ++g) {
              const double lhs = R(c, a, e) * t.f(a, c, b, d, e, g) * R(c, b, g);
              double rhs = 0.0;
              for (int f = 0; f < n; ++f) rhs += t.f(c, a, b, d, e, f) * R(c, f, d) * t.f(a, b, c, d, f, g);
              if (std::fabs(lhs - rhs) > tol) fail("hexagon equation");
            }
  for (int a = 0; a < n; ++a)
    if (t.dual[a] == a && std::fabs(t.fs[a] - t.dims[a] * t.f(a, a, a, a, 0, 0)) > tol)
      fail("Frobenius-Schur phase differs from d_a F(a, a, a; a; 0, 0)");
}

// --- SU(2) 6j via Racah's single sum, in long double ------------------------

static long double lfact(int n) {
  static std::vector<long double> table = [] {
    std::vector<long double> t(1200);
    t[0] = 1.0L;
    for (size_t i = 1; i < t.size(); ++i) t[i] = t[i - 1] * (long double)i;
    return t;
  }();
  if (n < 0 || n >= (int)table.size()) throw std::runtime_error("SU(2) label out of supported range");
  return table[n];
}

static bool triad(int a, int b, int c) {
  return a + b - c >= 0 && a - b + c >= 0 && -a + b + c >= 0 && ((a + b + c) & 1) == 0;
}

static long double delta2(int a, int b, int c) {
  return lfact((a + b - c) / 2) * lfact((a - b + c) / 2) * lfact((-a + b + c) / 2) / lfact((a + b + c) / 2 + 1);
}

static double su2_fsymbol_uncached(int a, int b, int c, int d, int e, int f) {
  if (!(triad(a, b, e) && triad(e, c, d) && triad(b, c, f) && triad(a, f, d))) return 0.0;
  // {j1 j2 j3; j4 j5 j6} = {a b e; c d f}
  int j1 = a, j2 = b, j3 = e, j4 = c, j5 = d, j6 = f;
  int a1 = (j1 + j2 + j3) / 2, a2 = (j1 + j5 + j6) / 2, a3 = (j4 + j2 + j6) / 2, a4 = (j4 + j5 + j3) / 2;
  int b1 = (j1 + j2 + j4 + j5) / 2, b2 = (j2 + j3 + j5 + j6) / 2, b3 = (j3 + j1 + j6 + j4) / 2;
  int zmin = std::max(std::max(a1, a2), std::max(a3, a4));
  int zmax = std::min(b1, std::min(b2, b3));
  long double s = 0.0L;
  for (int z = zmin; z <= zmax; ++z) {
    long double term = lfact(z + 1) / (lfact(z - a1) * lfact(z - a2) * lfact(z - a3) * lfact(z - a4) *
                                      lfact(b1 - z) * lfact(b2 - z) * lfact(b3 - z));
    s += (z & 1) ? -term : term;
  }
  long double q = delta2(j1, j2, j3) * delta2(j1, j5, j6) * delta2(j4, j2, j6) * delta2(j4, j5, j3);
  long double v = s * sqrtl(q * (long double)(e + 1) * (long double)(f + 1));
  if (((a + b + c + d) / 2) & 1) v = -v;
  return (double)v;
}

double su2_fsymbol(int a, int b, int c, int d, int e, int f) {
  static std::mutex mu;
  static std::unordered_map<uint64_t, double> cache;
  auto in = [](int x) { return x >= 0 && x < 1024; };
  if (!(in(a) && in(b) && in(c) && in(d) && in(e) && in(f))) throw std::runtime_error("SU(2) label out of range");
  uint64_t key = ((uint64_t)a) | ((uint64_t)b << 10) | ((uint64_t)c << 20) | ((uint64_t)d << 30) |
                 ((uint64_t)e << 40) | ((uint64_t)f << 50);
  {
    std::lock_guard<std::mutex> g(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  double v = su2_fsymbol_uncached(a, b, c, d, e, f);
  std::lock_guard<std::mutex> g(mu);
  cache.emplace(key, v);
  return v;
}

// ---------------------------------------------------------------------------
// Legs
// ---------------------------------------------------------------------------

Leg Leg::make(const Rule& r, const std::vector<Sector>& s, const std::vector<int64_t>& d, bool dual) {
  if (s.size() != d.size()) throw std::invalid_argument("sector/degeneracy length mismatch");
  std::vector<size_t> order(s.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](size_t x, size_t y) { return r.id(s[x]) < r.id(s[y]); });
  Leg leg;
  leg.dual = dual;
  for (size_t i = 0; i < order.size(); ++i) {
    if (i > 0 && r.id(s[order[i]]) == r.id(s[order[i - 1]]))
      throw std::invalid_argument("sector appears multiple times on one leg");  // sector.rs:160-168
    if (d[order[i]] < 0) throw std::invalid_argument("negative degeneracy");
    if (d[order[i]] == 0) continue;
    leg.sectors.push_back(s[order[i]]);
    leg.degs.push_back(d[order[i]]);
  }
  return leg;
}

Leg Leg::dualized(const Rule& r) const {
  std::vector<Sector> s;
  for (auto& x : sectors) s.push_back(r.dual(x));
  return make(r, s, degs, !dual);
}

int64_t Leg::deg(const Sector& s) const {
  for (size_t i = 0; i < sectors.size(); ++i)
    if (sectors[i] == s) return degs[i];
  return 0;
}

bool Leg::operator==(const Leg& o) const {
  if (dual != o.dual || sectors.size() != o.sectors.size()) return false;
  for (size_t i = 0; i < sectors.size(); ++i)
    if (!(sectors[i] == o.sectors[i]) || degs[i] != o.degs[i]) return false;
  return true;
}

// ---------------------------------------------------------------------------
// Fusion trees
// ---------------------------------------------------------------------------

static void append_sector(std::string& k, const Sector& s) { k.append((const char*)s.v, sizeof(s.v)); }

static void append_tree(std::string& k, const Tree& t) {
  uint32_t n = (uint32_t)t.u.size();
  k.append((const char*)&n, sizeof(n));
  for (auto& s : t.u) append_sector(k, s);
  for (auto x : t.d) k.push_back((char)x);
  append_sector(k, t.c);
  for (auto& s : t.inner) append_sector(k, s);
}

std::string pair_key(const TreePair& p) {
  std::string k;
  k.reserve(256);
  append_tree(k, p.cod);
  k.push_back('|');
  append_tree(k, p.dom);
  return k;
}

static std::string tree_key(const Tree& t) {
  std::string k;
  append_tree(k, t);
  return k;
}

// fusion_tree.rs:970-990
static std::vector<Sector> reachable_coupled(const Rule& r, const std::vector<Sector>& eff) {
  std::vector<Sector> acc;
  if (eff.empty()) {
    acc.push_back(r.vacuum());
    return acc;
  }
  acc.push_back(eff[0]);
  std::vector<Sector> ch;
  for (size_t i = 1; i < eff.size(); ++i) {
    std::map<uint64_t, Sector> next;
    for (auto& f : acc) {
      r.channels(f, eff[i], ch);
      for (auto& c : ch) next.emplace(r.id(c), c);
    }
    acc.clear();
    for (auto& kv : next) acc.push_back(kv.second);
  }
  std::sort(acc.begin(), acc.end(), [&](const Sector& x, const Sector& y) { return r.id(x) < r.id(y); });
  return acc;
}

// visit_fusion_trees_where (fusion_tree.rs:1076-1130): inner line adjacent to
// the coupled sector is the outermost loop; emitted innermost-first.
static void visit_trees(const Rule& r, const std::vector<Sector>& eff, size_t n, const Sector& coupled,
                        std::vector<Sector>& inner_rev, std::vector<std::vector<Sector>>& out) {
  if (n == 0) {
    if (coupled == r.vacuum()) out.emplace_back(inner_rev.rbegin(), inner_rev.rend());
    return;
  }
  if (n == 1) {
    if (eff[0] == coupled) out.emplace_back(inner_rev.rbegin(), inner_rev.rend());
    return;
  }
  if (n == 2) {
    if (r.nsym(eff[0], eff[1], coupled)) out.emplace_back(inner_rev.rbegin(), inner_rev.rend());
    return;
  }
  const Sector& last = eff[n - 1];
  std::vector<Sector> ch;
  r.channels(coupled, r.dual(last), ch);
  for (auto& front : ch) {
    if (!r.nsym(front, last, coupled)) continue;
    inner_rev.push_back(front);
    visit_trees(r, eff, n - 1, front, inner_rev, out);
    inner_rev.pop_back();
  }
}

struct CoupledGroup {
  Sector c;
  std::vector<Tree> trees;
};

// fusion_trees_by_coupled_for_space (fusion_tree.rs:512-560)
static std::vector<CoupledGroup> trees_by_coupled(const Rule& r, const std::vector<Leg>& legs) {
  std::vector<CoupledGroup> groups;
  std::unordered_map<uint64_t, size_t> index;
  size_t n = legs.size();
  std::vector<uint8_t> duals(n);
  for (size_t i = 0; i < n; ++i) duals[i] = legs[i].dual ? 1 : 0;
  std::vector<size_t> ctr(n, 0);
  for (auto& l : legs)
    if (l.sectors.empty()) return groups;
  std::vector<Sector> tup(n);
  std::vector<Sector> inner_rev;
  while (true) {
    for (size_t i = 0; i < n; ++i) tup[i] = legs[i].sectors[ctr[i]];
    for (auto& c : reachable_coupled(r, tup)) {
      std::vector<std::vector<Sector>> inners;
      inner_rev.clear();
      visit_trees(r, tup, n, c, inner_rev, inners);
      uint64_t id = r.id(c);
      auto it = index.find(id);
      size_t gi;
      if (it == index.end()) {
        gi = groups.size();
        index.emplace(id, gi);
        groups.push_back(CoupledGroup{c, {}});
      } else {
        gi = it->second;
      }
      for (auto& in : inners) groups[gi].trees.push_back(Tree{tup, duals, c, in});
    }
    // first leg fastest (fusion_tree.rs:491-510)
    size_t i = 0;
    for (; i < n; ++i) {
      if (++ctr[i] < legs[i].sectors.size()) break;
      ctr[i] = 0;
    }
    if (i == n) break;
  }
  std::sort(groups.begin(), groups.end(),
            [&](const CoupledGroup& x, const CoupledGroup& y) { return r.id(x.c) < r.id(y.c); });
  return groups;
}

static int64_t tree_dim(const std::vector<Leg>& legs, const Tree& t, int64_t* shape) {
  int64_t p = 1;
  for (size_t i = 0; i < legs.size(); ++i) {
    int64_t d = legs[i].deg(t.u[i]);
    if (shape) shape[i] = d;
    p *= d;
  }
  return p;
}

int Space::sector_of(const Sector& c) const {
  for (size_t i = 0; i < sectors.size(); ++i)
    if (sectors[i].c == c) return (int)i;
  return -1;
}

bool Space::same_as(const Space& o) const {
  if (!(rule == o.rule) || cod.size() != o.cod.size() || dom.size() != o.dom.size()) return false;
  for (size_t i = 0; i < cod.size(); ++i)
    if (!(cod[i] == o.cod[i])) return false;
  for (size_t i = 0; i < dom.size(); ++i)
    if (!(dom[i] == o.dom[i])) return false;
  return true;
}

// fusion_space.rs:2211-2262 and 3953-4104
std::shared_ptr<Space> make_space(const Rule& r, const std::vector<Leg>& cod, const std::vector<Leg>& dom) {
  if (cod.size() + dom.size() > (size_t)kMaxRank) throw std::invalid_argument("tensor rank exceeds 8");
  auto sp = std::make_shared<Space>();
  sp->rule = r;
  sp->cod = cod;
  sp->dom = dom;
  auto cg = trees_by_coupled(r, cod);
  auto dg = trees_by_coupled(r, dom);
  size_t ci = 0, di = 0;
  int64_t offset = 0;
  int n1 = (int)cod.size(), n2 = (int)dom.size();
  while (ci < cg.size() && di < dg.size()) {
    uint64_t a = r.id(cg[ci].c), b = r.id(dg[di].c);
    if (a < b) {
      ++ci;
      continue;
    }
    if (a > b) {
      ++di;
      continue;
    }
    auto& rt = cg[ci].trees;
    auto& ct = dg[di].trees;
    ++ci;
    ++di;
    if (rt.empty() || ct.empty()) continue;
    std::vector<int64_t> rs(rt.size()), cs(ct.size());
    int64_t rows = 0, cols = 0;
    for (size_t i = 0; i < rt.size(); ++i) {
      rs[i] = rows;
      rows += tree_dim(cod, rt[i], nullptr);
    }
    for (size_t j = 0; j < ct.size(); ++j) {
      cs[j] = cols;
      cols += tree_dim(dom, ct[j], nullptr);
    }
    int32_t sidx = (int32_t)sp->sectors.size();
    sp->sectors.push_back(SectorInfo{rt[0].c, rows, cols, offset});
    for (size_t j = 0; j < ct.size(); ++j) {
      for (size_t i = 0; i < rt.size(); ++i) {
        BlockInfo b;
        b.key = TreePair{rt[i], ct[j]};
        b.sector = sidx;
        tree_dim(cod, rt[i], b.shape);
        tree_dim(dom, ct[j], b.shape + n1);
        int64_t s = 1;
        for (int k = 0; k < n1; ++k) {
          b.strides[k] = s;
          s *= b.shape[k];
        }
        s = rows;
        for (int k = 0; k < n2; ++k) {
          b.strides[n1 + k] = s;
          s *= b.shape[n1 + k];
        }
        b.row_start = rs[i];
        b.col_start = cs[j];
        b.offset = offset + rs[i] + rows * cs[j];
        sp->block_index.emplace(pair_key(b.key), (int32_t)sp->blocks.size());
        sp->blocks.push_back(std::move(b));
      }
    }
    offset += rows * cols;
  }
  sp->size = offset;
  return sp;
}

// ---------------------------------------------------------------------------
// Recoupling of tree pairs
// ---------------------------------------------------------------------------

namespace {

// FusionTermAccumulator (fusion_tree.rs:3888-3980): merge equal keys in first-seen order.
struct Acc {
  Terms items;
  std::unordered_map<std::string, size_t> idx;
  void push(const TreePair& p, double c) {
    std::string k = pair_key(p);
    auto it = idx.find(k);
    if (it == idx.end()) {
      idx.emplace(std::move(k), items.size());
      items.emplace_back(p, c);
    } else {
      items[it->second].second += c;
    }
  }
};

Sector ext(const Tree& t, int index, const Sector& first) {
  int rank = (int)t.u.size();
  if (index == 0) return first;
  if (index + 1 == rank) return t.c;
  return t.inner[index - 1];
}

}  // namespace

// PreparedMultiplicityFreeArtin::apply (fusion_tree.rs:8154-8253)
Terms artin_terms(const Rule& r, const Tree& t, int index, bool inverse) {
  Terms out;
  int rank = (int)t.u.size();
  Sector left = t.u[index], right = t.u[index + 1];
  Tree nt = t;
  std::swap(nt.u[index], nt.u[index + 1]);
  std::swap(nt.d[index], nt.d[index + 1]);
  Sector first = nt.u[0];
  Sector vac = r.vacuum();
  TreePair tp;
  if (left == vac || right == vac) {
    if (index > 0) nt.inner[index - 1] = left == vac ? ext(t, index + 1, first) : ext(t, index - 1, first);
    tp.cod = nt;
    out.emplace_back(tp, 1.0);
    return out;
  }
  if (index == 0) {
    Sector c = rank > 2 ? t.inner[0] : t.c;
    double coef = inverse ? r.R(right, left, c) : r.R(left, right, c);
    tp.cod = nt;
    out.emplace_back(tp, coef);
    return out;
  }
  Sector a = ext(t, index - 1, first), b = left, c = ext(t, index, first), d = right, e = ext(t, index + 1, first);
  std::vector<Sector> ch;
  r.channels(a, d, ch);
  for (auto& cp : ch) {
    if (!r.nsym(cp, b, e)) continue;
    Tree o = nt;
    o.inner[index - 1] = cp;
    double f = r.F(d, a, b, e, cp, c);
    double coef = inverse ? (r.R(d, c, e) * f) * r.R(d, a, cp) : r.R(c, d, e) * (f * r.R(a, d, cp));
    tp.cod = o;
    out.emplace_back(tp, coef);
  }
  return out;
}

// PreparedMultiplicityFreeBendRight (fusion_tree.rs:8744-8921)
Terms bendright(const Rule& r, const TreePair& p) {
  const Tree& cod = p.cod;
  const Tree& dom = p.dom;
  int n1 = (int)cod.u.size(), n2 = (int)dom.u.size();
  if (n1 == 0) throw std::runtime_error("bendright requires at least one codomain leg");
  Sector b = cod.u[n1 - 1];
  bool bdual = cod.d[n1 - 1] != 0;
  Sector a = n1 == 1 ? r.vacuum() : (n1 == 2 ? cod.u[0] : cod.inner.back());
  TreePair o;
  o.cod.u.assign(cod.u.begin(), cod.u.end() - 1);
  o.cod.d.assign(cod.d.begin(), cod.d.end() - 1);
  o.cod.c = a;
  if (n1 > 2) o.cod.inner.assign(cod.inner.begin(), cod.inner.end() - 1);
  o.dom = dom;
  o.dom.u.push_back(r.dual(b));
  o.dom.d.push_back(bdual ? 0 : 1);
  o.dom.c = a;
  if (n2 > 1) o.dom.inner.push_back(cod.c);
  double coef = std::sqrt(r.dim(cod.c)) / std::sqrt(r.dim(a)) * r.B(a, b, cod.c);
  if (bdual) coef *= r.fs(r.dual(b));
  return Terms{{o, coef}};
}

// fusion_tree.rs:8923-8998
Terms bendleft(const Rule& r, const TreePair& p) {
  TreePair sw{p.dom, p.cod};
  Terms t = bendright(r, sw);
  TreePair o{t[0].first.dom, t[0].first.cod};
  return Terms{{o, t[0].second}};
}

static Terms compose_terms(const Rule& r, const Terms& in, Terms (*op)(const Rule&, const TreePair&)) {
  Acc acc;
  for (auto& kv : in)
    for (auto& kv2 : op(r, kv.first)) acc.push(kv2.first, kv.second * kv2.second);
  return acc.items;
}

// fusion_tree.rs:3785-3812
Terms repartition_terms(const Rule& r, const TreePair& p, int target) {
  Terms cur{{p, 1.0}};
  int n1 = (int)p.cod.u.size();
  while (n1 < target) {
    cur = compose_terms(r, cur, bendleft);
    ++n1;
  }
  while (n1 > target) {
    cur = compose_terms(r, cur, bendright);
    --n1;
  }
  return cur;
}

// PreparedTreeBraid::new (fusion_tree.rs:2477-2507)
static std::vector<std::pair<int, bool>> artin_steps(const std::vector<int>& perm, const std::vector<int>& levels) {
  int rank = (int)perm.size();
  std::vector<int> work = perm, lv = levels;
  std::vector<std::pair<int, bool>> steps;
  for (int target = 0; target + 1 < rank; ++target) {
    int source = work[target];
    for (int index = source - 1; index >= target; --index) {
      steps.emplace_back(index, lv[index] > lv[index + 1]);
      std::swap(lv[index], lv[index + 1]);
    }
    for (int k = target + 1; k < rank; ++k)
      if (work[k] < source) work[k] += 1;
    work[target] = target;
  }
  return steps;
}

// prepare_braid_lowered (fusion_tree.rs:2763-2870) + execute (fusion_tree.rs:3319-3355)
Terms braid_pair_terms(const Rule& r, const TreePair& p, const std::vector<int>& p1, const std::vector<int>& p2,
                       const std::vector<int>& lv1, const std::vector<int>& lv2) {
  int n1 = (int)p.cod.u.size(), n2 = (int)p.dom.u.size(), n = n1 + n2;
  bool ident = (int)p1.size() == n1;
  for (int i = 0; ident && i < (int)p1.size(); ++i) ident = p1[i] == i;
  for (int i = 0; ident && i < (int)p2.size(); ++i) ident = p2[i] == n1 + i;
  if (ident) return Terms{{p, 1.0}};
  auto lin = [&](int a) { return a < n1 ? a : n2 + 2 * n1 - 1 - a; };
  std::vector<int> perm;
  for (int a : p1) perm.push_back(lin(a));
  for (int i = (int)p2.size() - 1; i >= 0; --i) perm.push_back(lin(p2[i]));
  bool linear_ident = true;
  for (int i = 0; i < n; ++i) linear_ident = linear_ident && perm[i] == i;
  if (linear_ident) return repartition_terms(r, p, (int)p1.size());
  std::vector<int> levels = lv1;
  for (int i = (int)lv2.size() - 1; i >= 0; --i) levels.push_back(lv2[i]);
  auto steps = artin_steps(perm, levels);
  Acc braided;
  for (auto& kv : repartition_terms(r, p, n)) {
    Terms cur{{kv.first, kv.second}};
    for (auto& st : steps) {
      Acc acc;
      for (auto& t : cur)
        for (auto& t2 : artin_terms(r, t.first.cod, st.first, st.second)) {
          TreePair q{t2.first.cod, t.first.dom};
          acc.push(q, t.second * t2.second);
        }
      cur = std::move(acc.items);
    }
    for (auto& t : cur) braided.push(t.first, t.second);
  }
  Acc out;
  for (auto& kv : braided.items)
    for (auto& kv2 : repartition_terms(r, kv.first, (int)p1.size())) out.push(kv2.first, kv.second * kv2.second);
  return out.items;
}

// ---------------------------------------------------------------------------
// Tensor-level transform plans
// ---------------------------------------------------------------------------

// Work tiles of whole columns (all axes but destination axis 0).  Each
// kernel path is its own launch, and its tiles are sized to fill whole waves
// of the transform kernel's resident CTAs (three per SM on the 148 SMs of a
// B200): a path is counted in waves of tiles of at most 32768 elements plus
// one partial tile per group, and the per-tile target divides the path's
// elements over that many waves, less one slot per group for the group's last,
// partial tile.  Small paths get one wave of tiles (at least 512 elements
// each); a tile holds at most 256 columns (the kernel stages their
// multi-indices in shared memory).  Within each path the largest tiles come
// first, so partial tiles fill the last slots.
//
// A single-block group whose source is strided along destination axis 0 but
// contiguous along another axis k* (extent above 1) is a transposing copy
// (kernel path 4): its tiles are ranges of planes (axis 0 x axis k*) over the
// remaining axes instead of ranges of columns.
static int xform_transposing_axis(const XformTables& t, const XGroup& g) {
  if (g.nsrc != 1 || g.ndst != 1 || g.rank < 2 || g.dims[0] < 4) return 0;
  const XEntry& e = t.src_entries[g.src_first];
  if (e.strides[0] == 1) return 0;
  for (int k = 1; k < g.rank; ++k)
    if (e.strides[k] == 1 && g.dims[k] > 1) return g.dims[k] >= 4 ? k : 0;
  return 0;
}

static void split_tiles(XformTables& t) {
  t.tiles.clear();
  const int64_t slots = 148 * 3;
  auto kind_of = [&](const XGroup& g) { return xform_transposing_axis(t, g) > 0 ? 4 : xform_kind(g); };
  int64_t total[kXKinds] = {}, ngroups[kXKinds] = {}, target[kXKinds] = {};
  for (auto& g : t.groups) {
    total[kind_of(g)] += g.nelem;
    ngroups[kind_of(g)] += 1;
  }
  for (int k = 0; k < kXKinds; ++k) {
    const int64_t waves = std::max<int64_t>(1, ((total[k] + 32767) / 32768 + ngroups[k] + slots - 1) / slots);
    target[k] = std::min<int64_t>(
        32768, std::max<int64_t>(512, total[k] / std::max<int64_t>(1, waves * slots - ngroups[k])));
  }
  for (size_t gi = 0; gi < t.groups.size(); ++gi) {
    const XGroup& g = t.groups[gi];
    for (int k = 0; k < g.rank; ++k)
      if (g.dims[k] > 65535) throw std::invalid_argument("a block extent above 65535 is not supported");
    const int kind = kind_of(g);
    const int ks = kind == 4 ? xform_transposing_axis(t, g) : 0;
    // work units: columns (all axes but 0), or planes (all axes but 0 and k*)
    const int64_t unit = (g.rank > 0 ? g.dims[0] : 1) * (kind == 4 ? g.dims[ks] : 1);
    const int64_t cols = g.nelem / unit;
    const int64_t per =
        std::max<int64_t>(1, kind == 4 ? target[kind] / unit : std::min<int64_t>(256, target[kind] / unit));
    for (int64_t s = 0; s < cols; s += per) {
      XTile tile;
      tile.group = (int32_t)gi;
      tile.kind = kind;
      tile.start = s;
      tile.count = std::min(per, cols - s);
      t.tiles.push_back(tile);
    }
  }
  auto elems = [&](const XTile& x) {
    const XGroup& g = t.groups[x.group];
    const int64_t unit = (g.rank > 0 ? (int64_t)g.dims[0] : 1) * (x.kind == 4 ? g.dims[xform_transposing_axis(t, g)] : 1);
    return x.count * unit;
  };
  std::stable_sort(t.tiles.begin(), t.tiles.end(), [&](const XTile& a, const XTile& b) {
    if (a.kind != b.kind) return a.kind < b.kind;
    return elems(a) > elems(b);
  });
}

void finish_transform_tables(XformTables& t) {
  t.max_nsrc = t.max_ndst = 0;
  for (auto& g : t.groups) {
    t.max_nsrc = std::max(t.max_nsrc, g.nsrc);
    t.max_ndst = std::max(t.max_ndst, g.ndst);
  }
  split_tiles(t);
}

// Product of the ribbon twists of a block's uncoupled sectors on the given
// flat axes (codomain first); real and +-1 for every rule in scope.
static double block_twist(const Rule& r, const Space& sp, const TreePair& key, const std::vector<int>& axes) {
  double f = 1.0;
  int n1 = sp.n1();
  for (int a : axes) f *= a < n1 ? r.twist(key.cod.u[a]) : r.twist(key.dom.u[a - n1]);
  return f;
}

std::vector<int> supertrace_axes(const Space& dst, int n_contracted) {
  std::vector<int> axes;
  bool fermionic = false;
  for (int i = 0; i < dst.rule.nf; ++i) fermionic |= dst.rule.kind[i] == FK_FZ2;
  if (!fermionic) return axes;
  for (int p = 0; p < n_contracted && p < dst.n1(); ++p)
    if (dst.cod[p].dual) axes.push_back(p);
  return axes;
}

// Geometry of one transform step on a given source space.
struct StepGeom {
  std::shared_ptr<Space> dst;
  std::vector<int> p1, p2, lv1, lv2, axes, twist;
};

static StepGeom step_geometry(const std::shared_ptr<Space>& src, const TransformStep& st) {
  const Rule& r = src->rule;
  int n1 = src->n1(), n2 = src->n2(), n = n1 + n2;
  StepGeom g;
  g.p1 = st.p1;
  g.p2 = st.p2;
  if (st.kind == XK_REPARTITION) {
    if (st.nrep < 0 || st.nrep > n) throw std::invalid_argument("repartition split exceeds the rank");
    std::vector<int> planar;
    for (int i = 0; i < n1; ++i) planar.push_back(i);
    for (int i = n - 1; i >= n1; --i) planar.push_back(i);
    g.p1.assign(planar.begin(), planar.begin() + st.nrep);
    g.p2.assign(planar.rbegin(), planar.rend() - st.nrep);
  }
  if (st.kind == XK_ADJOINT) {
    // block(t', c) = block(t, c)^T: swap codomain and domain, transpose every
    // block (TensorKit adjoint; real payloads need no conjugation).
    g.p1.clear();
    g.p2.clear();
    for (int i = n1; i < n; ++i) g.p1.push_back(i);
    for (int i = 0; i < n1; ++i) g.p2.push_back(i);
  }
  if ((int)(g.p1.size() + g.p2.size()) != n) throw std::invalid_argument("axis lists do not cover the rank");
  std::vector<int> seen(n, 0);
  for (int a : g.p1) {
    if (a < 0 || a >= n || seen[a]++) throw std::invalid_argument("axis lists are not a permutation");
  }
  for (int a : g.p2) {
    if (a < 0 || a >= n || seen[a]++) throw std::invalid_argument("axis lists are not a permutation");
  }
  if (st.kind == XK_BRAID && (int)st.levels.size() != n) throw std::invalid_argument("braid needs one level per axis");
  for (int a : st.twist_axes)
    if (a < 0 || a >= n) throw std::invalid_argument("twist leg out of range");

  std::vector<Leg> all = src->cod;
  for (auto& l : src->dom) all.push_back(l.dualized(r));
  std::vector<Leg> ncod, ndom;
  if (st.kind == XK_ADJOINT) {
    ncod = src->dom;
    ndom = src->cod;
  } else {
    for (int a : g.p1) ncod.push_back(all[a]);
    for (int a : g.p2) ndom.push_back(all[a].dualized(r));
  }
  g.dst = make_space(r, ncod, ndom);
  g.axes = g.p1;
  g.axes.insert(g.axes.end(), g.p2.begin(), g.p2.end());
  if (st.kind == XK_BRAID) {
    g.lv1.assign(st.levels.begin(), st.levels.begin() + n1);
    g.lv2.assign(st.levels.begin() + n1, st.levels.end());
  } else {
    for (int i = 0; i < n1; ++i) g.lv1.push_back(i);
    for (int i = n1; i < n; ++i) g.lv2.push_back(i);
  }
  g.twist = st.twist_axes;
  if (st.supertrace >= 0) {
    auto extra = supertrace_axes(*g.dst, st.supertrace);
    g.twist.insert(g.twist.end(), extra.begin(), extra.end());
  }
  return g;
}

// Destination tree pairs and coefficients of one source tree pair under one step.
static Terms step_terms(const Rule& r, const TransformStep& st, const StepGeom& g, const TreePair& key) {
  Terms terms = st.kind == XK_REPARTITION ? repartition_terms(r, key, st.nrep)
                : st.kind == XK_ADJOINT   ? Terms{{TreePair{key.dom, key.cod}, 1.0}}
                                          : braid_pair_terms(r, key, g.p1, g.p2, g.lv1, g.lv2);
  if (!g.twist.empty())
    for (auto& t : terms) t.second *= block_twist(r, *g.dst, t.first, g.twist);
  return terms;
}

std::vector<std::shared_ptr<Space>> chain_spaces(const std::shared_ptr<Space>& src,
                                                 const std::vector<TransformStep>& steps) {
  std::vector<std::shared_ptr<Space>> out;
  std::shared_ptr<Space> cur = src;
  for (auto& st : steps) {
    cur = step_geometry(cur, st).dst;
    out.push_back(cur);
  }
  return out;
}

bool step_is_noop(const Space& src, const TransformStep& st) {
  int n1 = src.n1(), n = n1 + src.n2();
  if (st.kind != XK_PERMUTE || !st.twist_axes.empty()) return false;
  if ((int)st.p1.size() != n1 || (int)(st.p1.size() + st.p2.size()) != n) return false;
  for (int i = 0; i < n1; ++i)
    if (st.p1[i] != i) return false;
  for (int i = n1; i < n; ++i)
    if (st.p2[i - n1] != i) return false;
  return st.supertrace < 0 || supertrace_axes(src, st.supertrace).empty();
}

std::shared_ptr<TransformPlan> make_transform(const std::shared_ptr<Space>& src, TransformKind kind,
                                              const std::vector<int>& p1, const std::vector<int>& p2,
                                              const std::vector<int>& levels, int nrep,
                                              const std::vector<int>& twist_axes) {
  TransformStep st;
  st.kind = kind;
  st.p1 = p1;
  st.p2 = p2;
  st.levels = levels;
  st.nrep = nrep;
  st.twist_axes = twist_axes;
  return make_transform_chain(src, {st});
}

std::shared_ptr<TransformPlan> make_transform_chain(const std::shared_ptr<Space>& src,
                                                    const std::vector<TransformStep>& steps) {
  if (steps.empty()) throw std::invalid_argument("empty transform chain");
  const Rule& r = src->rule;
  int n = src->n1() + src->n2();
  std::vector<StepGeom> geo;
  std::shared_ptr<Space> cur = src;
  std::vector<int> axes_total;
  for (size_t i = 0; i < steps.size(); ++i) {
    geo.push_back(step_geometry(cur, steps[i]));
    const auto& g = geo.back();
    if (i == 0) {
      axes_total = g.axes;
    } else {
      std::vector<int> next(n);
      for (int k = 0; k < n; ++k) next[k] = axes_total[g.axes[k]];
      axes_total = next;
    }
    cur = g.dst;
  }

  auto plan = std::make_shared<TransformPlan>();
  plan->src = src;
  plan->dst = cur;
  plan->axes = axes_total;
  const Space& dst = *plan->dst;

  // Terms of a source tree pair through every step; zero terms are dropped
  // between steps and kept after the last (as a single step keeps them).
  auto chain_terms = [&](const TreePair& key) {
    Terms acc{{key, 1.0}};
    for (size_t i = 0; i < steps.size(); ++i) {
      Terms next;
      std::unordered_map<std::string, size_t> at;
      for (auto& t : acc) {
        if (i > 0 && t.second == 0.0) continue;
        for (auto& u : step_terms(r, steps[i], geo[i], t.first)) {
          std::string k = pair_key(u.first);
          auto it = at.find(k);
          if (it == at.end()) {
            at.emplace(k, next.size());
            next.emplace_back(u.first, t.second * u.second);
          } else {
            next[it->second].second += t.second * u.second;
          }
        }
      }
      acc.swap(next);
    }
    return acc;
  };

  // Group source blocks by their uncoupled sectors (one block shape per group).
  std::unordered_map<std::string, size_t> gindex;
  std::vector<std::vector<int32_t>> gsrc;
  for (size_t b = 0; b < src->blocks.size(); ++b) {
    const auto& k = src->blocks[b].key;
    std::string key;
    for (auto& s : k.cod.u) append_sector(key, s);
    key.push_back('|');
    for (auto& s : k.dom.u) append_sector(key, s);
    auto it = gindex.find(key);
    if (it == gindex.end()) {
      gindex.emplace(key, gsrc.size());
      gsrc.push_back({(int32_t)b});
    } else {
      gsrc[it->second].push_back((int32_t)b);
    }
  }

  XformTables& T = plan->tables;
  T.src_size = src->size;
  T.dst_size = dst.size;
  std::vector<uint8_t> covered(dst.blocks.size(), 0);
  for (auto& members : gsrc) {
    std::vector<int32_t> dsts;
    std::unordered_map<int32_t, size_t> dpos;
    std::vector<std::vector<double>> rows;  // rows[d][s]
    for (size_t si = 0; si < members.size(); ++si) {
      const auto& sb = src->blocks[members[si]];
      Terms terms = chain_terms(sb.key);
      for (auto& t : terms) {
        auto it = dst.block_index.find(pair_key(t.first));
        if (it == dst.block_index.end()) {
          if (t.second == 0.0) continue;
          throw std::runtime_error("recoupling produced a tree pair outside the destination space");
        }
        int32_t d = it->second;
        auto jt = dpos.find(d);
        size_t di;
        if (jt == dpos.end()) {
          di = dsts.size();
          dpos.emplace(d, di);
          dsts.push_back(d);
          rows.emplace_back(members.size(), 0.0);
        } else {
          di = jt->second;
        }
        rows[di][si] += t.second;
      }
    }
    if (dsts.empty()) continue;
    XGroup g{};
    g.nsrc = (int32_t)members.size();
    g.ndst = (int32_t)dsts.size();
    g.rank = n;
    const auto& d0 = dst.blocks[dsts[0]];
    g.nelem = 1;
    for (int k = 0; k < n; ++k) {
      g.dims[k] = (int32_t)d0.shape[k];
      g.nelem *= d0.shape[k];
    }
    g.src_first = (int32_t)T.src_entries.size();
    g.dst_first = (int32_t)T.dst_entries.size();
    g.coef_off = (int32_t)T.coef.size();
    for (int32_t sbi : members) {
      const auto& sb = src->blocks[sbi];
      XEntry e{};
      e.offset = sb.offset;
      for (int k = 0; k < n; ++k) e.strides[k] = sb.strides[plan->axes[k]];
      T.src_entries.push_back(e);
    }
    for (int32_t dbi : dsts) {
      const auto& db = dst.blocks[dbi];
      for (int k = 0; k < n; ++k)
        if (db.shape[k] != g.dims[k]) throw std::runtime_error("destination block shape mismatch in a group");
      XEntry e{};
      e.offset = db.offset;
      for (int k = 0; k < n; ++k) e.strides[k] = db.strides[k];
      T.dst_entries.push_back(e);
      covered[dbi] = 1;
    }
    for (auto& row : rows) T.coef.insert(T.coef.end(), row.begin(), row.end());
    T.max_nsrc = std::max(T.max_nsrc, g.nsrc);
    T.max_ndst = std::max(T.max_ndst, g.ndst);
    plan->moved_elements += g.nelem * (g.nsrc + g.ndst);
    T.groups.push_back(g);
  }
  // Destination blocks no source reaches are written as zeros.
  for (size_t d = 0; d < dst.blocks.size(); ++d) {
    if (covered[d]) continue;
    const auto& db = dst.blocks[d];
    XGroup g{};
    g.nsrc = 0;
    g.ndst = 1;
    g.rank = n;
    g.nelem = 1;
    for (int k = 0; k < n; ++k) {
      g.dims[k] = (int32_t)db.shape[k];
      g.nelem *= db.shape[k];
    }
    g.src_first = (int32_t)T.src_entries.size();
    g.dst_first = (int32_t)T.dst_entries.size();
    g.coef_off = (int32_t)T.coef.size();
    XEntry e{};
    e.offset = db.offset;
    for (int k = 0; k < n; ++k) e.strides[k] = db.strides[k];
    T.dst_entries.push_back(e);
    plan->moved_elements += g.nelem;
    T.groups.push_back(g);
  }
  split_tiles(T);
  return plan;
}

// ---------------------------------------------------------------------------
// Compose and factorisation plans
// ---------------------------------------------------------------------------

// FusionBlockContractPlan::try_from_canonical_coupled_regions_impl (fusion_replay.rs:457-530)
std::shared_ptr<ComposePlan> make_compose(const std::shared_ptr<Space>& lhs, const std::shared_ptr<Space>& rhs) {
  if (!(lhs->rule == rhs->rule)) throw std::invalid_argument("compose: operands use different fusion rules");
  if (lhs->dom.size() != rhs->cod.size()) throw std::invalid_argument("compose: domain/codomain rank mismatch");
  for (size_t i = 0; i < lhs->dom.size(); ++i)
    if (!(lhs->dom[i] == rhs->cod[i])) throw std::invalid_argument("compose: domain of lhs != codomain of rhs");
  auto plan = std::make_shared<ComposePlan>();
  plan->lhs = lhs;
  plan->rhs = rhs;
  plan->dst = make_space(lhs->rule, lhs->cod, rhs->dom);
  const Space& d = *plan->dst;
  GemmTables& T = plan->tables;
  T.a_size = lhs->size;
  T.b_size = rhs->size;
  T.c_size = d.size;
  for (auto& s : d.sectors) {
    int ia = lhs->sector_of(s.c), ib = rhs->sector_of(s.c);
    GemmJob j{};
    j.m = s.rows;
    j.n = s.cols;
    j.c_off = s.offset;
    j.ldc = s.rows;
    if (ia >= 0 && ib >= 0) {
      const auto& a = lhs->sectors[ia];
      const auto& b = rhs->sectors[ib];
      if (a.rows != s.rows || b.cols != s.cols || a.cols != b.rows)
        throw std::runtime_error("compose: coupled-sector extents disagree");
      j.k = a.cols;
      j.a_off = a.offset;
      j.b_off = b.offset;
      j.lda = a.rows;
      j.ldb = b.rows;
    } else {
      j.k = 0;  // a sector only one operand carries: C block is zero
      j.lda = std::max<int64_t>(1, s.rows);
      j.ldb = 1;
    }
    plan->flops += 2.0 * (double)j.m * (double)j.n * (double)j.k;
    T.jobs.push_back(j);
  }
  return plan;
}

std::shared_ptr<FactorPlan> make_factor(const std::shared_ptr<Space>& src) {
  auto plan = std::make_shared<FactorPlan>();
  plan->src = src;
  SvdTables& T = plan->tables;
  T.a_size = src->size;
  for (auto& s : src->sectors) {
    SvdJob j{};
    j.m = s.rows;
    j.n = s.cols;
    j.k = std::min(s.rows, s.cols);
    j.a_off = s.offset;
    j.u_off = T.u_size;
    j.s_off = T.s_size;
    j.v_off = T.v_size;
    j.weight = src->rule.dim(s.c);
    T.u_size += j.m * j.k;
    T.s_size += j.k;
    T.v_size += j.k * j.n;
    T.jobs.push_back(j);
  }
  return plan;
}

}  // namespace tnt
