// Instantiates the single-frame tile kernel for one block shape (NF_BH x NF_BW,
// 0 = runtime shape) and its three sample storages.
#include "launch.hpp"
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
template <int ST, int ALGO>
cudaError_t launch_batch(const BatchWork& w, int ctas, size_t smem, cudaStream_t st) {
  auto k = spatial_batch_kernel<NF_BH, NF_BW, ST, ALGO>;
  cudaError_t e = prepare(k, smem);
  if (e != cudaSuccess) return e;
  k<<<ctas, 256, smem, st>>>(w);
  return cudaGetLastError();
}
template <int ST>
cudaError_t launch_kalman_one(const DevPlan& d, int nb, dim3 grid, size_t smem, const void* src, ptrdiff_t ss,
                              const KalmanArgs& a, cudaStream_t st) {
  auto k = kalman_advance_kernel<NF_BH, NF_BW, ST>;
  cudaError_t e = prepare(k, smem);
  if (e != cudaSuccess) return e;
  k<<<grid, 256, smem, st>>>(d, nb, static_cast<const unsigned char*>(src), ss, a);
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
  cudaError_t launch_kalman_##BH##x##BW(const DevPlan& d, int nb, dim3 grid, size_t smem, const void* src,       \
                                        ptrdiff_t ss, const KalmanArgs& a, cudaStream_t st) {                   \
    if (d.storage == kStoreU8) return launch_kalman_one<kStoreU8>(d, nb, grid, smem, src, ss, a, st);           \
    if (d.storage == kStoreU16) return launch_kalman_one<kStoreU16>(d, nb, grid, smem, src, ss, a, st);         \
    return launch_kalman_one<kStoreF32>(d, nb, grid, smem, src, ss, a, st);                                      \
  }
NF_DEFINE(NF_BH, NF_BW)
} // namespace nfd
