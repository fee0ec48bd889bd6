// Tile-shape autotuner for the grouped GEMMs, keyed on the block-size
// histogram of a compose plan.
//
// FP64 path: every coupled-sector job picks one of four output-tile shapes
// (64x64, 64x32, 32x64, 32x32).  The pick minimises the job's estimated time
//   ntiles(shape) * (ceil(k / 16) + 1) * cost[shape]
// where cost[shape] is the measured time of one tile k-step of that shape on
// this device.  The costs are calibrated once per device by timing the first
// sufficiently large compose with each uniform shape; before that they take
// model defaults.  Large sectors keep 64x64 tiles, small and ragged sectors
// trade tile efficiency for less padding.
//
// Split path: the output tile width (64 or 128 columns) is picked by the
// measured time per padded multiply-accumulate of each width.
#pragma once

#include <cstdint>
#include <mutex>
#include <vector>

#include "kernels.cuh"

namespace tnt {

struct DeviceTuning {
  bool f64_calibrated = false;
  double f64_cost[4] = {1.0, 0.6, 0.6, 0.4};  // relative time per tile k-step, kShape* order
  bool split_calibrated = false;
  double split_eff64 = 0.8;  // per-MAC throughput of 64-wide tiles relative to 128-wide
};

// Per-device tuning state (process-wide); lock tuning_mutex() around access.
DeviceTuning& device_tuning(int device);
std::mutex& tuning_mutex();

// Autotuning is on unless TNT_AUTOTUNE=0.
bool autotune_enabled();

// Per-job FP64 tile shapes for the given per-shape costs.
std::vector<int32_t> choose_f64_shapes(const std::vector<GemmJob>& jobs, const double cost[4]);

// The FP64 tile list of `nbatch` batch entries with per-job shapes, sorted by
// estimated cost (longest first) for the persistent kernel's greedy balance.
std::vector<GemmTile> build_f64_tiles(const std::vector<GemmJob>& jobs, int64_t nbatch,
                                      const std::vector<int32_t>& shapes, const double cost[4]);

// Sum over the list of (k-steps + 1): the work unit the costs are quoted in.
double f64_tile_units(const std::vector<GemmJob>& jobs, const std::vector<GemmTile>& tiles);

}  // namespace tnt
