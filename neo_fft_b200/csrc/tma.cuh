// Tensor-memory-accelerator staging of source rows for the batched strip kernel.
//
// A persistent CTA prefetches the `step` source rows that block row by + 1 adds while
// block row by is transformed: one elected thread issues 2-D tiled bulk-tensor copies
// (this GPU's own memory, no cluster sharing; boxes 256 bytes wide, side by side) into
// one of two raw buffers in shared memory and an mbarrier counts their bytes; at block
// row by + 1 every thread waits on that barrier (bounded by a clock limit) and converts
// the raw samples to the staging ring.
// A wait that runs out sets kErrStaging in the plan's error word, marks the pipeline
// dead for the rest of the launch and stages that row from global memory instead; the
// kernel waits once more, again bounded, for copies still in flight before it exits.
#pragma once
#include <cstdint>

namespace nfd {

enum : int { kErrStaging = 2 };  // error-word bit: a staging copy did not complete

// Width of one staging box in bytes (256 / element size samples): a staged window takes
// one or more boxes side by side, each stored [row][sample] in shared memory.
constexpr int kStagingBoxBytes = 256;

// Per-CTA pipeline state: barriers and the dead flag in shared memory; the parity
// bits (one per buffer, flipped after each completed wait) and the copies thread 0
// has issued but not yet seen complete live in registers.
struct TmaPipe {
  unsigned long long* mbar;  // [2]
  int* dead;                 // shared: nonzero once a wait has run out
  unsigned phase;            // bit b: parity of buffer b's next completion
  unsigned pending;          // thread 0: bit b set while buffer b has a copy in flight
};

// About one second at the B200's clocks.
constexpr long long kStagingWaitCycles = 2000000000LL;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}

// Makes barrier initialisation visible to the bulk-copy unit.
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}

// true once the phase with `parity` has completed; false if `limit` cycles pass first.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* b, unsigned parity, long long limit) {
  const long long t0 = clock64();
  while (!mbar_try_wait(b, parity))
    if (clock64() - t0 > limit) return false;
  return true;
}

// Box (x, y) of the 2-D tensor map into shared memory; completion is counted on `b`.
// x * element size must be a multiple of 16 bytes (the caller rounds x down).
__device__ __forceinline__ void tma_load_2d(void* dst, const void* tmap, int x, int y, unsigned long long* b) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_u32(dst)),
      "l"(tmap), "r"(x), "r"(y), "r"(smem_u32(b))
      : "memory");
}

// `bytes` bytes from global `src` into shared `dst` with one bulk copy (both addresses
// 16-byte aligned, `bytes` a multiple of 16); completion is counted on `b`. This GPU's
// own memory only, no cluster sharing.
__device__ __forceinline__ void bulk_load_1d(void* dst, const void* src, unsigned bytes, unsigned long long* b) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(b))
               : "memory");
}

}  // namespace nfd
