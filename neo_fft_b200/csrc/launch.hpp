// Kernel launchers, one translation unit per block shape (spatial_inst.cu is
// compiled once per shape with -DNF_BH/-DNF_BW; 0 = runtime shape).
#pragma once
#include "device_plan.cuh"

#include <cuda_runtime.h>

#include <map>
#include <mutex>

namespace nfd {
// Every kernel's dynamic shared-memory limit is set to the most it can take (the device's
// opt-in maximum less the kernel's static shared memory), so any launch size up to it is
// valid and host threads launching the same kernel with different sizes set the same
// value (a per-launch value would race with another thread's launch).
inline int dynamic_smem_max(const void* kernel) {
  static std::mutex mu;
  static std::map<const void*, int> cache;
  std::lock_guard<std::mutex> lock(mu);
  const auto it = cache.find(kernel);
  if (it != cache.end()) return it->second;
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa{};
  if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) return 0;
  const int m = optin - int(fa.sharedSizeBytes);
  cache.emplace(kernel, m);
  return m;
}
template <class K>
cudaError_t set_smem_limit(K k, size_t smem) {
  const int m = dynamic_smem_max(reinterpret_cast<const void*>(k));
  if (m <= 0 || smem > size_t(m)) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, m);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  return e;
}
struct StripShape;
struct PlaneJobs;
struct BatchWork;
#define NF_DECLARE_SPATIAL(BH, BW)                                                                              \
  cudaError_t launch_spatial_##BH##x##BW(const DevPlan& d, const StripShape& s, dim3 grid, size_t smem,         \
                                         const PlaneJobs& job, cudaStream_t st);                                \
  cudaError_t launch_spatial_batch_##BH##x##BW(int storage, int algo, const BatchWork& w, int ctas, size_t smem, \
                                               cudaStream_t st);                                                \
  cudaError_t launch_kalman_render_##BH##x##BW(const DevPlan& d, const StripShape& s, dim3 grid, size_t smem,   \
                                               const PlaneJobs& job, cudaStream_t st);
NF_DECLARE_SPATIAL(8, 8)
NF_DECLARE_SPATIAL(16, 16)
NF_DECLARE_SPATIAL(32, 32)
NF_DECLARE_SPATIAL(12, 12)
NF_DECLARE_SPATIAL(48, 48)
NF_DECLARE_SPATIAL(0, 0)
#undef NF_DECLARE_SPATIAL
struct SpectraWork;
struct VolumeSpectraWork;
#define NF_DECLARE_TEMPORAL(BH, BW)                                                                             \
  cudaError_t launch_spectra_batch_##BH##x##BW(int storage, const SpectraWork& w, int items, size_t smem,        \
                                               cudaStream_t st);                                                \
  cudaError_t launch_volume_spectra_batch_##BH##x##BW(int storage, const VolumeSpectraWork& w, int items,       \
                                                      size_t smem, cudaStream_t st);                            \
  cudaError_t launch_temporal_batch_##BH##x##BW(int storage, int slice, const BatchWork& w, int ctas,            \
                                                size_t smem, cudaStream_t st);
NF_DECLARE_TEMPORAL(8, 8)
NF_DECLARE_TEMPORAL(16, 16)
NF_DECLARE_TEMPORAL(32, 32)
NF_DECLARE_TEMPORAL(12, 12)
NF_DECLARE_TEMPORAL(48, 48)
NF_DECLARE_TEMPORAL(0, 0)
#undef NF_DECLARE_TEMPORAL
struct KalmanArgs;
struct AdjointShape;
struct AdjointBatch;
cudaError_t launch_adjoint_16x16(const DevPlan& d, const AdjointShape& S, const AdjointBatch& b, size_t smem,
                                 cudaStream_t st);
cudaError_t launch_adjoint_0x0(const DevPlan& d, const AdjointShape& S, const AdjointBatch& b, size_t smem,
                               cudaStream_t st);
struct VolumeShape;
struct VolumeSources;
#define NF_DECLARE_VOLUME(BH, BW)                                                                               \
  cudaError_t launch_volume_##BH##x##BW(const DevPlan& d, const VolumeShape& s, dim3 grid, size_t smem,         \
                                        const VolumeSources& v, void* dst, ptrdiff_t ds, cudaStream_t st);
NF_DECLARE_VOLUME(8, 8)
NF_DECLARE_VOLUME(16, 16)
NF_DECLARE_VOLUME(32, 32)
NF_DECLARE_VOLUME(12, 12)
NF_DECLARE_VOLUME(48, 48)
NF_DECLARE_VOLUME(0, 0)
#undef NF_DECLARE_VOLUME
#define NF_DECLARE_KALMAN(BH, BW)                                                                               \
  cudaError_t launch_kalman_##BH##x##BW(const DevPlan& d, const void* src, ptrdiff_t ss, const KalmanArgs& a,   \
                                        cudaStream_t st);
NF_DECLARE_KALMAN(8, 8)
NF_DECLARE_KALMAN(16, 16)
NF_DECLARE_KALMAN(32, 32)
NF_DECLARE_KALMAN(12, 12)
NF_DECLARE_KALMAN(48, 48)
NF_DECLARE_KALMAN(0, 0)
#undef NF_DECLARE_KALMAN
} // namespace nfd
