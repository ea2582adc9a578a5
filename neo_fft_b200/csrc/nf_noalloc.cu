// Allocation-free form of the DFTTest backward (nf_dft_backward_device): the scratch
// lives in a file-scope device buffer of fixed size, so a call allocates nothing.
// Every scratch word the backward reads is written earlier in the same call (cover
// gradients are retired row by row, table partials tile by tile), so nothing in the
// buffer has to start at zero and the buffer is never cleared.
#include "neo_fft_b200.h"
#include "plan_info.hpp"

#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

namespace {

constexpr size_t kStaticScratchBytes = size_t(16) << 20;  // 16 MiB per device
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_backward_scratch[kStaticScratchBytes];

std::mutex g_setup_lock;
void* g_scratch_addr[kMaxDevices] = {};

nf_status report(char* err, size_t len, nf_status st, const char* msg) {
  if (err && len) std::snprintf(err, len, "%s", msg);
  return st;
}

// Device address of the static buffer on device `dev`, which must be the current device
// (a symbol's address is per device); looked up once per device.
nf_status scratch_address(int dev, void** out, char* err, size_t len) {
  if (dev < 0 || dev >= kMaxDevices) return report(err, len, NF_DEVICE_ERROR, "device ordinal out of range");
  cudaError_t e = cudaSuccess;
  std::lock_guard<std::mutex> lock(g_setup_lock);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_backward_scratch);
    if (e != cudaSuccess || !p) {
      char msg[256];
      std::snprintf(msg, sizeof msg, "static backward scratch lookup failed: %s", cudaGetErrorString(e));
      return report(err, len, NF_DEVICE_ERROR, msg);
    }
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return NF_OK;
}

} // namespace

extern "C" size_t nf_dft_backward_static_capacity(void) { return kStaticScratchBytes; }

extern "C" nf_status nf_dft_backward_device_static(const nf_plan* plan, const nf_const_plane* sources,
                                                   const nf_const_plane* grad_out, const nf_plane* grad_sources,
                                                   int nplanes, float* grad_primary, void* stream, char* err,
                                                   size_t err_len) {
  // The plan and plane count are checked first, so the capacity message below is only
  // given to calls that the caller-scratch form would accept.
  nf_status st = nfi::check_backward_call(plan, nplanes, err, err_len);
  if (st != NF_OK) return st;
  // The buffer's address is the one on the plan's device, which must be current: the
  // kernels run on the current device and read the plan's tables there.
  int dev = 0;
  const cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return report(err, err_len, NF_DEVICE_ERROR, cudaGetErrorString(e));
  const int plan_dev = nfi::plan_info(plan).device;
  if (dev != plan_dev) {
    char msg[160];
    std::snprintf(msg, sizeof msg, "the plan lives on device %d but device %d is current", plan_dev, dev);
    return report(err, err_len, NF_INVALID_ARGUMENT, msg);
  }
  size_t need = 0;
  st = nf_dft_backward_scratch_bytes(plan, nplanes, &need);
  if (st != NF_OK) return report(err, err_len, st, "backward scratch size query failed");
  if (need > kStaticScratchBytes) {
    char msg[256];
    std::snprintf(msg, sizeof msg,
                  "backward needs %zu scratch bytes for %d planes, above the %zu-byte static buffer; "
                  "pass fewer planes per call or use nf_dft_backward_device",
                  need, nplanes, kStaticScratchBytes);
    return report(err, err_len, NF_INVALID_ARGUMENT, msg);
  }
  void* scratch = nullptr;
  if ((st = scratch_address(dev, &scratch, err, err_len)) != NF_OK) return st;
  return nf_dft_backward_device(plan, sources, grad_out, grad_sources, nplanes, grad_primary, scratch,
                                kStaticScratchBytes, stream, err, err_len);
}
