// Instantiates the FFT3D temporal clip kernels (pass 1 spectra, pass 2 strips) for one
// block shape (NF_BH x NF_BW, 0 = runtime shape) and its three sample storages.
#include "launch.hpp"
#include "tile_temporal.cuh"

#ifndef NF_BH
#error "compile with -DNF_BH=<rows> -DNF_BW=<cols>"
#endif

namespace nfd {
namespace {
template <class K>
cudaError_t prepare(K k, size_t smem) {
  return set_smem_limit(k, smem);
}
template <int ST>
cudaError_t spectra(const SpectraWork& w, int items, size_t smem, cudaStream_t st) {
  auto k = spectra_batch_kernel<NF_BH, NF_BW, ST>;
  cudaError_t e = prepare(k, smem);
  if (e != cudaSuccess) return e;
  k<<<items, 256, smem, st>>>(w);
  return cudaGetLastError();
}
template <int ST>
cudaError_t volume_spectra(const VolumeSpectraWork& w, int items, size_t smem, cudaStream_t st) {
  auto k = volume_spectra_batch_kernel<NF_BH, NF_BW, ST>;
  cudaError_t e = prepare(k, smem);
  if (e != cudaSuccess) return e;
  k<<<items, 256, smem, st>>>(w);
  return cudaGetLastError();
}
template <int ST, int SRC>
cudaError_t temporal(const BatchWork& w, int ctas, size_t smem, cudaStream_t st) {
  auto k = temporal_batch_kernel<NF_BH, NF_BW, ST, SRC>;
  cudaError_t e = prepare(k, smem);
  if (e != cudaSuccess) return e;
  k<<<ctas, TemporalThreads<NF_BH, NF_BW, SRC>::value, smem, st>>>(w);
  return cudaGetLastError();
}
} // namespace

#define NF_DEFINE(BH, BW) NF_DEFINE_(BH, BW)
#define NF_DEFINE_(BH, BW)                                                                                        \
  cudaError_t launch_spectra_batch_##BH##x##BW(int storage, const SpectraWork& w, int items, size_t smem,        \
                                               cudaStream_t st) {                                                \
    if (storage == kStoreU8) return spectra<kStoreU8>(w, items, smem, st);                                       \
    if (storage == kStoreU16) return spectra<kStoreU16>(w, items, smem, st);                                     \
    return spectra<kStoreF32>(w, items, smem, st);                                                                \
  }                                                                                                              \
  cudaError_t launch_volume_spectra_batch_##BH##x##BW(int storage, const VolumeSpectraWork& w, int items,       \
                                                      size_t smem, cudaStream_t st) {                            \
    if (storage == kStoreU8) return volume_spectra<kStoreU8>(w, items, smem, st);                                \
    if (storage == kStoreU16) return volume_spectra<kStoreU16>(w, items, smem, st);                              \
    return volume_spectra<kStoreF32>(w, items, smem, st);                                                         \
  }                                                                                                              \
  cudaError_t launch_temporal_batch_##BH##x##BW(int storage, int slice, const BatchWork& w, int ctas,            \
                                                size_t smem, cudaStream_t st) {                                  \
    if (slice) {                                                                                                 \
      if (storage == kStoreU8) return temporal<kStoreU8, kSrcSlice>(w, ctas, smem, st);                          \
      if (storage == kStoreU16) return temporal<kStoreU16, kSrcSlice>(w, ctas, smem, st);                        \
      return temporal<kStoreF32, kSrcSlice>(w, ctas, smem, st);                                                   \
    }                                                                                                            \
    if (storage == kStoreU8) return temporal<kStoreU8, kSrcTemporal>(w, ctas, smem, st);                         \
    if (storage == kStoreU16) return temporal<kStoreU16, kSrcTemporal>(w, ctas, smem, st);                       \
    return temporal<kStoreF32, kSrcTemporal>(w, ctas, smem, st);                                                  \
  }
NF_DEFINE(NF_BH, NF_BW)
} // namespace nfd
