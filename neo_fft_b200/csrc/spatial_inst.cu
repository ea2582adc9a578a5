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
template <int ST>
cudaError_t launch_one(const DevPlan& d, const TileShape& S, dim3 grid, size_t smem, const void* src, ptrdiff_t ss,
                       void* dst, ptrdiff_t ds, const cf* L, cudaStream_t st) {
  auto k = spatial_tile_kernel<NF_BH, NF_BW, ST>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  k<<<grid, S.threads, smem, st>>>(d, S, static_cast<const unsigned char*>(src), ss, static_cast<unsigned char*>(dst),
                                   ds, L);
  return cudaGetLastError();
}
template <int ST>
cudaError_t launch_kalman_one(const DevPlan& d, int nb, dim3 grid, size_t smem, const void* src, ptrdiff_t ss,
                              const KalmanArgs& a, cudaStream_t st) {
  auto k = kalman_advance_kernel<NF_BH, NF_BW, ST>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  k<<<grid, 256, smem, st>>>(d, nb, static_cast<const unsigned char*>(src), ss, a);
  return cudaGetLastError();
}
} // namespace

#define NF_DEFINE(BH, BW) NF_DEFINE_(BH, BW)
#define NF_DEFINE_(BH, BW)                                                                                        \
  cudaError_t launch_spatial_##BH##x##BW(const DevPlan& d, const TileShape& S, dim3 grid, size_t smem,           \
                                         const void* src, ptrdiff_t ss, void* dst, ptrdiff_t ds, const cf* L,    \
                                         cudaStream_t st) {                                                      \
    if (d.storage == kStoreU8) return launch_one<kStoreU8>(d, S, grid, smem, src, ss, dst, ds, L, st);          \
    if (d.storage == kStoreU16) return launch_one<kStoreU16>(d, S, grid, smem, src, ss, dst, ds, L, st);        \
    return launch_one<kStoreF32>(d, S, grid, smem, src, ss, dst, ds, L, st);                                     \
  }
NF_DEFINE(NF_BH, NF_BW)

#define NF_DEFINE_KALMAN(BH, BW) NF_DEFINE_KALMAN_(BH, BW)
#define NF_DEFINE_KALMAN_(BH, BW)                                                                                \
  cudaError_t launch_kalman_##BH##x##BW(const DevPlan& d, int nb, dim3 grid, size_t smem, const void* src,       \
                                        ptrdiff_t ss, const KalmanArgs& a, cudaStream_t st) {                   \
    if (d.storage == kStoreU8) return launch_kalman_one<kStoreU8>(d, nb, grid, smem, src, ss, a, st);           \
    if (d.storage == kStoreU16) return launch_kalman_one<kStoreU16>(d, nb, grid, smem, src, ss, a, st);         \
    return launch_kalman_one<kStoreF32>(d, nb, grid, smem, src, ss, a, st);                                      \
  }
NF_DEFINE_KALMAN(NF_BH, NF_BW)
} // namespace nfd
