// Instantiates the DFTTest and FFT3D adjoints for one block shape (NF_BH x NF_BW,
// 0 = runtime).
#include "adjoint.cuh"
#include "launch.hpp"

#ifndef NF_BH
#error "compile with -DNF_BH=<rows> -DNF_BW=<cols>"
#endif

namespace nfd {
#define NF_DEFINE(BH, BW) NF_DEFINE_(BH, BW)
#define NF_DEFINE_(BH, BW)                                                                                        \
  cudaError_t launch_adjoint_##BH##x##BW(const DevPlan& d, const AdjointShape& S, const AdjointBatch& b,          \
                                         size_t smem, cudaStream_t st) {                                         \
    auto k = d.algo == 0 ? fft3d_adjoint_kernel<BH, BW> : dft_adjoint_kernel<BH, BW>;                         \
    const cudaError_t e = set_smem_limit(k, smem);                                                              \
    if (e != cudaSuccess) return e;                                                                              \
    k<<<b.n * S.tiles_x * S.tiles_y, 256, smem, st>>>(d, S, b);                                                  \
    return cudaGetLastError();                                                                                   \
  }
NF_DEFINE(NF_BH, NF_BW)
} // namespace nfd
