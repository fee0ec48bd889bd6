// Allocation-free variant of the batched per-sector SVD (tnt_svd_static).
//
// Some callers cannot allocate device memory when they need a factorisation:
// a serving loop that admits work against a fixed device-memory budget must
// not grow its footprint between admissions, and a foreign host (for example
// a Rust runtime reaching this library over FFI) may own every device byte
// through its own allocator, so a cudaMalloc here would bypass its
// accounting.  This entry point serves them: it runs the same Jacobi SVD
// kernel as tnt_svd, but its scratch (the sector job table, per-sector work
// panels and the convergence flag) lives in the file-scope device array
// below, so the call performs no cudaMalloc/cudaFree and uses no allocating
// library routine.  Inputs and outputs stay caller-owned device buffers.
//
// Limits and sharing rules:
//   * the array holds kStaticSvdDoubles doubles (8 MiB) on every device that
//     loads this library, for the life of the process; a plan whose tables
//     plus work panels exceed it is rejected with TNT_INVALID_ARGUMENT;
//   * every call shares the one array, and it keeps the previous call's
//     contents: calls whose kernels overlap on the GPU (different streams,
//     threads or contexts on one device) race on it and must be serialised
//     by the caller;
//   * the first call on each device looks up the array's device address with
//     that device current (cudaGetSymbolAddress) and caches it; CUDA loads
//     this file's module lazily, so that first call is also when the 8 MiB
//     are committed on the device.  Make it at set-up, before a memory budget
//     is fixed and before any stream capture begins;
//   * every sector runs on one CTA (the in-shared-memory or blocked Jacobi
//     kernel), largest sectors first; tnt_svd's thread-block clusters for
//     the largest sectors are not used here, so sectors of several hundred
//     rows factorise several times slower than through tnt_svd (6.4x at a
//     586 x 586 sector).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "kernels.cuh"

namespace tnt {

constexpr size_t kStaticSvdDoubles = size_t(1) << 20;  // 8 MiB

static __device__ __align__(256) double g_svd_scratch[kStaticSvdDoubles];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
double* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_svd_scratch on the current device (looked up once per device).
cudaError_t scratch_address(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> g(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_svd_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}

size_t doubles_for(size_t bytes) { return (bytes + sizeof(double) - 1) / sizeof(double); }

}  // namespace

// Layout inside the static array (in doubles, each region 256-byte aligned):
//   [status flag][job table][work offsets][work panels].
cudaError_t svd_static(const std::vector<SvdJob>& jobs, const double* a, double* u, double* s, double* vh,
                       cudaStream_t stream, std::string& why) {
  const size_t njobs = jobs.size();
  if (njobs == 0) return cudaSuccess;
  auto align32 = [](size_t x) { return (x + 31) & ~size_t(31); };  // 32 doubles = 256 bytes
  const size_t off_status = 0;
  const size_t off_jobs = align32(off_status + 1);
  const size_t off_offs = align32(off_jobs + doubles_for(njobs * sizeof(SvdJob)));
  const size_t off_work = align32(off_offs + njobs);
  // Largest sectors first (rows * k^2 descending): each job carries its own
  // output offsets, so the order only decides which CTA starts first.
  std::vector<SvdJob> order(jobs);
  std::stable_sort(order.begin(), order.end(), [](const SvdJob& x, const SvdJob& y) {
    const double cx = (double)std::max(x.m, x.n) * (double)x.k * (double)x.k;
    const double cy = (double)std::max(y.m, y.n) * (double)y.k * (double)y.k;
    return cx > cy;
  });
  std::vector<int64_t> work_off(njobs);
  size_t work = 0;
  for (size_t i = 0; i < njobs; ++i) {
    const SvdJob& j = order[i];
    work_off[i] = (int64_t)work;
    const size_t rows = (size_t)std::max(j.m, j.n);
    work += rows * (size_t)j.k + (size_t)j.k * (size_t)j.k + 2 * (size_t)j.k;
  }
  if (off_work + work > kStaticSvdDoubles) {
    why = "plan needs " + std::to_string(off_work + work) + " doubles of scratch; the static array holds " +
          std::to_string(kStaticSvdDoubles);
    return cudaErrorInvalidValue;
  }
  double* base = nullptr;
  cudaError_t e = scratch_address(&base);
  if (e != cudaSuccess) return e;
  int32_t* status = reinterpret_cast<int32_t*>(base + off_status);
  SvdJob* djobs = reinterpret_cast<SvdJob*>(base + off_jobs);
  int64_t* doffs = reinterpret_cast<int64_t*>(base + off_offs);
  // The kernel overwrites every work panel before reading it; only the flag
  // and the sweep counter beside it must start at zero.
  if ((e = cudaMemsetAsync(status, 0, 2 * sizeof(int32_t), stream)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(djobs, order.data(), njobs * sizeof(SvdJob), cudaMemcpyHostToDevice, stream)) != cudaSuccess)
    return e;
  if ((e = cudaMemcpyAsync(doffs, work_off.data(), njobs * sizeof(int64_t), cudaMemcpyHostToDevice, stream)) !=
      cudaSuccess)
    return e;
  if ((e = launch_svd(djobs, (int32_t)njobs, a, u, s, vh, base + off_work, doffs, status, stream)) != cudaSuccess)
    return e;
  int32_t hs = 0;
  if ((e = cudaMemcpyAsync(&hs, status, sizeof(int32_t), cudaMemcpyDeviceToHost, stream)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;
  if (hs != 0) {
    why = "Jacobi SVD did not converge within the sweep limit";
    return cudaErrorUnknown;
  }
  return cudaSuccess;
}

}  // namespace tnt
