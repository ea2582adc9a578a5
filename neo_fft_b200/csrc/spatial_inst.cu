// Instantiates the single-frame tile kernel for one block shape (NF_BH x NF_BW,
// 0 = runtime shape) and its three sample storages.
#include "launch.hpp"

#include <algorithm>
#include "tile_spatial.cuh"
#include "kalman.cuh"

#ifndef NF_BH
#error "compile with -DNF_BH=<rows> -DNF_BW=<cols>"
#endif

namespace nfd {
namespace {
template <class K>
cudaError_t prepare(K k, size_t smem) {
  return set_smem_limit(k, smem);
}
template <int ST, int ALGO>
cudaError_t launch_one(const DevPlan& d, const StripShape& S, dim3 grid, size_t smem, const PlaneJobs& job,
                       cudaStream_t st) {
  auto k = spatial_strip_kernel<NF_BH, NF_BW, ST, ALGO>;
  cudaError_t e = prepare(k, smem);
  if (e != cudaSuccess) return e;
  k<<<grid, 256, smem, st>>>(d, S, job);
  return cudaGetLastError();
}
template <int ST>
cudaError_t launch_render(const DevPlan& d, const StripShape& S, dim3 grid, size_t smem, const PlaneJobs& job,
                          cudaStream_t st) {
  auto k = kalman_render_kernel<NF_BH, NF_BW, ST>;
  cudaError_t e = prepare(k, smem);
  if (e != cudaSuccess) return e;
  k<<<grid, 256, smem, st>>>(d, S, job);
  return cudaGetLastError();
}
template <int ST, int ALGO>
cudaError_t launch_batch(const BatchWork& w, int ctas, size_t smem, cudaStream_t st) {
  auto k = spatial_batch_kernel<NF_BH, NF_BW, ST, ALGO>;
  cudaError_t e = prepare(k, smem);
  if (e != cudaSuccess) return e;
  k<<<ctas, 256, smem, st>>>(w);
  return cudaGetLastError();
}
// Kalman advance: runs of nb blocks of one block row per CTA of about nb * bh threads
// (whole warps, 64..256). The run length minimises the modelled launch time: waves of the
// grid over the resident CTAs (the occupancy the kernel really gets) times the CTA's
// rounds of threads over rows, columns and bins (eight bins per thread and round) plus
// one of setup; longer runs on ties.
template <int ST>
cudaError_t launch_kalman_one(const DevPlan& d, const void* src, ptrdiff_t ss, const KalmanArgs& args,
                              cudaStream_t st) {
  // Kalman step (a.synth set): the same run geometry, the run's estimate DCs after its
  // spectra, and the render's inverse columns and rows in the cost of a run. Runs stage
  // their old state in shared memory by bulk copies when every run's slice of the state
  // arrays starts on 16 bytes (a bin count that is a multiple of four).
  KalmanArgs a = args;
  const uintptr_t arrays = reinterpret_cast<uintptr_t>(a.last) |
                           (a.fp64 ? reinterpret_cast<uintptr_t>(a.cov64) | reinterpret_cast<uintptr_t>(a.proc64)
                                   : reinterpret_cast<uintptr_t>(a.cov32) | reinterpret_cast<uintptr_t>(a.proc32));
  a.staged = (d.bins & 3) == 0 && (arrays & 15) == 0;
  // Large blocks keep the state in global memory: one block's spectra and staged state must
  // fit the run's shared-memory budget (128x128 blocks in binary64 variance need 266 KB).
  if (a.staged && kalman_smem(d.bins, 1, a.synth != nullptr, a.fp64, 1).bytes > size_t(200) * 1024) a.staged = 0;
  const bool step = a.synth != nullptr;
  auto k = step ? kalman_advance_kernel<NF_BH, NF_BW, ST, true> : kalman_advance_kernel<NF_BH, NF_BW, ST, false>;
  auto smem_of = [&](int r) { return kalman_smem(d.bins, r, step, a.fp64, a.staged).bytes; };
  int nb_max = std::max(1, std::min(8, d.gx.count));
  while (nb_max > 1 && smem_of(nb_max) > size_t(200) * 1024) --nb_max;
  cudaError_t e = prepare(k, smem_of(nb_max));
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  // the choice of the last geometry this thread launched (frames of a clip repeat it)
  struct Choice {
    int dev = -1, cx = 0, cy = 0, bh = 0, bw = 0, st = 0, step = 0, fp64 = 0, nb = 0, threads = 0;
  };
  thread_local Choice last;
  if (last.dev == dev && last.cx == d.gx.count && last.cy == d.gy.count && last.bh == d.bh && last.bw == d.bw &&
      last.st == ST && last.step == int(step) && last.fp64 == a.fp64) {
    const dim3 grid((d.gx.count + last.nb - 1) / last.nb, d.gy.count);
    k<<<grid, last.threads, smem_of(last.nb), st>>>(d, last.nb, static_cast<const unsigned char*>(src), ss, a);
    return cudaGetLastError();
  }
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  auto rounds = [](long long tasks, int threads) { return (tasks + threads - 1) / threads; };
  int nb = nb_max, threads = 256;
  long long best = -1;
  for (int r = nb_max; r >= 1; --r) {
    const int t = std::min(256, std::max(64, (r * d.bh + 31) / 32 * 32));
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, t, smem_of(r)) != cudaSuccess || occ < 1)
      continue;
    const long long ctas = (long long)((d.gx.count + r - 1) / r) * d.gy.count;
    const long long slots = (long long)occ * sms;
    const long long per_run = 1 + rounds((long long)r * d.bh, t) + rounds((long long)r * d.K, t) +
                              rounds((long long)r * d.bins, 8 * t) +
                              (step ? rounds((long long)r * d.K, t) + rounds((long long)r * d.bh, t) : 0);
    const long long cost = (ctas + slots - 1) / slots * per_run;
    if (best < 0 || cost < best) {
      best = cost;
      nb = r;
      threads = t;
    }
  }
  last = Choice{dev, d.gx.count, d.gy.count, d.bh, d.bw, ST, int(step), a.fp64, nb, threads};
  const dim3 grid((d.gx.count + nb - 1) / nb, d.gy.count);
  k<<<grid, threads, smem_of(nb), st>>>(d, nb, static_cast<const unsigned char*>(src), ss, a);
  return cudaGetLastError();
}
} // namespace

#define NF_DEFINE(BH, BW) NF_DEFINE_(BH, BW)
#define NF_DEFINE_(BH, BW)                                                                                        \
  cudaError_t launch_spatial_##BH##x##BW(const DevPlan& d, const StripShape& S, dim3 grid, size_t smem,          \
                                         const PlaneJobs& job, cudaStream_t st) {                                \
    if (d.algo == 0) {                                                                                           \
      if (d.storage == kStoreU8) return launch_one<kStoreU8, 0>(d, S, grid, smem, job, st);                     \
      if (d.storage == kStoreU16) return launch_one<kStoreU16, 0>(d, S, grid, smem, job, st);                   \
      return launch_one<kStoreF32, 0>(d, S, grid, smem, job, st);                                                \
    }                                                                                                            \
    if (d.storage == kStoreU8) return launch_one<kStoreU8, 1>(d, S, grid, smem, job, st);                       \
    if (d.storage == kStoreU16) return launch_one<kStoreU16, 1>(d, S, grid, smem, job, st);                     \
    return launch_one<kStoreF32, 1>(d, S, grid, smem, job, st);                                                  \
  }                                                                                                              \
  cudaError_t launch_spatial_batch_##BH##x##BW(int storage, int algo, const BatchWork& w, int ctas, size_t smem, \
                                               cudaStream_t st) {                                                \
    if (algo == 0) {                                                                                             \
      if (storage == kStoreU8) return launch_batch<kStoreU8, 0>(w, ctas, smem, st);                             \
      if (storage == kStoreU16) return launch_batch<kStoreU16, 0>(w, ctas, smem, st);                           \
      return launch_batch<kStoreF32, 0>(w, ctas, smem, st);                                                      \
    }                                                                                                            \
    if (storage == kStoreU8) return launch_batch<kStoreU8, 1>(w, ctas, smem, st);                               \
    if (storage == kStoreU16) return launch_batch<kStoreU16, 1>(w, ctas, smem, st);                             \
    return launch_batch<kStoreF32, 1>(w, ctas, smem, st);                                                        \
  }                                                                                                              \
  cudaError_t launch_kalman_render_##BH##x##BW(const DevPlan& d, const StripShape& S, dim3 grid, size_t smem,   \
                                               const PlaneJobs& job, cudaStream_t st) {                         \
    if (d.storage == kStoreU8) return launch_render<kStoreU8>(d, S, grid, smem, job, st);                       \
    if (d.storage == kStoreU16) return launch_render<kStoreU16>(d, S, grid, smem, job, st);                     \
    return launch_render<kStoreF32>(d, S, grid, smem, job, st);                                                  \
  }                                                                                                              \
  cudaError_t launch_kalman_##BH##x##BW(const DevPlan& d, const void* src, ptrdiff_t ss, const KalmanArgs& a,    \
                                        cudaStream_t st) {                                                      \
    if (d.storage == kStoreU8) return launch_kalman_one<kStoreU8>(d, src, ss, a, st);                           \
    if (d.storage == kStoreU16) return launch_kalman_one<kStoreU16>(d, src, ss, a, st);                         \
    return launch_kalman_one<kStoreF32>(d, src, ss, a, st);                                                      \
  }
NF_DEFINE(NF_BH, NF_BW)
} // namespace nfd
