// Instantiates the multi-frame volume kernel for one block shape (NF_BH x NF_BW,
// 0 = runtime shape) and its three sample storages.
#include "launch.hpp"
#include "tile_volume.cuh"

#ifndef NF_BH
#error "compile with -DNF_BH=<rows> -DNF_BW=<cols>"
#endif

namespace nfd {
namespace {
template <int ST>
cudaError_t launch_one(const DevPlan& d, const VolumeShape& S, dim3 grid, size_t smem, const VolumeSources& v,
                       void* dst, ptrdiff_t ds, cudaStream_t st) {
  auto k = volume_tile_kernel<NF_BH, NF_BW, ST>;
  const cudaError_t e = set_smem_limit(k, smem);
  if (e != cudaSuccess) return e;
  k<<<grid, S.threads, smem, st>>>(d, S, v, static_cast<unsigned char*>(dst), ds);
  return cudaGetLastError();
}
} // namespace

#define NF_DEFINE(BH, BW) NF_DEFINE_(BH, BW)
#define NF_DEFINE_(BH, BW)                                                                                        \
  cudaError_t launch_volume_##BH##x##BW(const DevPlan& d, const VolumeShape& S, dim3 grid, size_t smem,          \
                                        const VolumeSources& v, void* dst, ptrdiff_t ds, cudaStream_t st) {      \
    if (d.storage == kStoreU8) return launch_one<kStoreU8>(d, S, grid, smem, v, dst, ds, st);                   \
    if (d.storage == kStoreU16) return launch_one<kStoreU16>(d, S, grid, smem, v, dst, ds, st);                 \
    return launch_one<kStoreF32>(d, S, grid, smem, v, dst, ds, st);                                              \
  }
NF_DEFINE(NF_BH, NF_BW)
} // namespace nfd
