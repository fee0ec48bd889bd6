// Tile-shape autotuner state and per-job shape choice (see autotune.hpp).
#include "autotune.hpp"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>

namespace tnt {

namespace {

constexpr int64_t kF64Bk = 16;

int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

int64_t ksteps(const GemmJob& j) { return ceil_div(j.k, kF64Bk) + 1; }

}  // namespace

std::mutex& tuning_mutex() {
  static std::mutex m;
  return m;
}

DeviceTuning& device_tuning(int device) {
  static std::map<int, DeviceTuning> table;
  return table[device];
}

bool autotune_enabled() {
  const char* e = getenv("TNT_AUTOTUNE");
  return !(e && std::strcmp(e, "0") == 0);
}

std::vector<int32_t> choose_f64_shapes(const std::vector<GemmJob>& jobs, const double cost[4]) {
  std::vector<int32_t> shapes(jobs.size(), kShape64x64);
  for (size_t j = 0; j < jobs.size(); ++j) {
    const GemmJob& J = jobs[j];
    double best = 0.0;
    for (int s = 0; s < 4; ++s) {
      const double t = (double)(ceil_div(std::max<int64_t>(J.m, 1), kShapeM[s]) *
                                ceil_div(std::max<int64_t>(J.n, 1), kShapeN[s])) *
                       (double)ksteps(J) * cost[s];
      if (s == 0 || t < best) {
        best = t;
        shapes[j] = s;
      }
    }
  }
  return shapes;
}

std::vector<GemmTile> build_f64_tiles(const std::vector<GemmJob>& jobs, int64_t nbatch,
                                      const std::vector<int32_t>& shapes, const double cost[4]) {
  std::vector<std::pair<double, GemmTile>> v;
  for (int64_t b = 0; b < nbatch; ++b)
    for (size_t j = 0; j < jobs.size(); ++j) {
      const GemmJob& J = jobs[j];
      const int s = shapes[j];
      const int64_t BM = kShapeM[s], BN = kShapeN[s];
      const int64_t mt = ceil_div(J.m, BM), nt = ceil_div(J.n, BN);
      for (int64_t x = 0; x < mt; ++x) {
        const int64_t h = std::min<int64_t>(BM, ceil_div(J.m - x * BM, 16) * 16);  // last block: trimmed
        for (int64_t y = 0; y < nt; ++y) {
          const int64_t w = std::min<int64_t>(BN, ceil_div(J.n - y * BN, 16) * 16);
          // one cost per job (not per trimmed tile), so a job's tiles stay
          // adjacent in the list and its operands are read from HBM once
          const double c = (double)ksteps(J) * cost[s];
          v.push_back({c, GemmTile{(int32_t)j, (int32_t)b, (int32_t)(x * BM / 16), (int32_t)(y * BN / 16),
                                   f64_tile_code((int)h, (int)w), 0}});
        }
      }
    }
  std::stable_sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
  std::vector<GemmTile> out;
  out.reserve(v.size());
  for (auto& x : v) out.push_back(x.second);
  return out;
}

double f64_tile_units(const std::vector<GemmJob>& jobs, const std::vector<GemmTile>& tiles) {
  double u = 0.0;
  for (const GemmTile& t : tiles) u += (double)ksteps(jobs[t.job]);
  return u;
}

}  // namespace tnt
