// Kalman advance (FFT3D bt=0): forward spectrum of every block of the new frame
// and the per-bin recursion on the HBM-resident state (src/algorithms/plan.cpp:301-321,
// src/kernels/scalar/kalman.cpp:3-24).
//
// Each CTA owns a run of NB consecutive blocks of one block row; every block is
// visited exactly once, so each state bin has a single owner thread per frame and
// the update is race-free. Rows: thread = (block, row) -> reflected, windowed row
// transform into shared memory. Columns: thread = (block, column) -> transform
// along y in registers, written back in place. Recursion: thread = bin of the run,
// over the state arrays in their own order.
#pragma once
#include "tile_spatial.cuh"

namespace nfd {

struct KalmanArgs {
  cf* last;
  float* cov32;
  float* proc32;
  double* cov64;
  double* proc64;
  const float* pattern;  // per-bin noise table or nullptr (uniform r0)
  int fp64;
};

template <int BHC, int BWC, int STORAGE>
__global__ void __launch_bounds__(256) kalman_advance_kernel(DevPlan P, int nb_per_cta, const unsigned char* src,
                                                             ptrdiff_t src_stride, KalmanArgs A) {
  extern __shared__ float smem[];
  const int BH = BHC > 0 ? BHC : P.bh;
  const int BW = BWC > 0 ? BWC : P.bw;
  const int K = BW / 2 + 1;
  constexpr int CAPH = BHC > 0 ? BHC : nf::kMaxProject;
  constexpr int CAPW = BWC > 0 ? BWC : nf::kMaxProject;
  constexpr int UH = BHC > 0 ? CAPH : 1, UW = BWC > 0 ? CAPW : 1;
  // Square 8/16/32 blocks always use the codelet networks; sized instantiations
  // know it at compile time, so only one transform family is generated.
  constexpr bool kCodelet = BHC == BWC && (BWC == 8 || BWC == 16 || BWC == 32);
  const bool codelet = kCodelet || (BHC == 0 && P.codelet != 0);
  const DevAxis gx = P.gx, gy = P.gy;
  cf* spec = reinterpret_cast<cf*>(smem);
  const int by = blockIdx.y;
  const int bx0 = blockIdx.x * nb_per_cta;
  const int nb = min(nb_per_cta, gx.count - bx0);
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int oy = by * gy.step;
  bool bad = false;
  // Legacy pad_source decodes without a finiteness check (src/algorithms/pad.hpp:47-82);
  // the recursion checks every consumed value instead.
  for (int task = tid; task < nb * BH; task += nthr) {
    const int b = task / BH, y = task - b * BH;
    const int ox = (bx0 + b) * gx.step;
    const unsigned char* srow = src + ptrdiff_t(reflect_axis(oy + y, gy)) * src_stride;
    float row[CAPW];
#pragma unroll UW
    for (int x = 0; x < CAPW; ++x) {
      if (x < BW) {
        const float s = load_sample<STORAGE>(srow, reflect_axis(ox + x, gx));
        const float v = fsub(s, P.dec_base);
        row[x] = fmul(fmul(v, P.wya[y]), P.wxa[x]);
      }
    }
    nf::row_forward<BWC>(row, BW, spec + (size_t(b) * BH + y) * K, P.tww, codelet);
  }
  __syncthreads();
  for (int task = tid; task < nb * K; task += nthr) {
    const int b = task / K, k = task - b * K;
    cf col[CAPH];
    cf* sp = spec + size_t(b) * BH * K + k;
#pragma unroll UH
    for (int y = 0; y < CAPH; ++y)
      if (y < BH) col[y] = sp[size_t(y) * K];
    nf::fft_1d<true, BHC>(col, BH, P.twh, codelet);
#pragma unroll UH
    for (int y = 0; y < CAPH; ++y)
      if (y < BH) sp[size_t(y) * K] = col[y];
  }
  __syncthreads();
  // The recursion, one thread per bin: spec holds the run's blocks as [block][y*K + k],
  // the state's own layout, and the run's blocks are consecutive in the state, so bin i
  // of the run is state element base + i (coalesced; the arrays never alias).
  const int bins = BH * K;
  const int n = nb * bins;
  const size_t base = (size_t(by) * gx.count + bx0) * size_t(bins);
  cf* __restrict__ last = A.last + base;
  const float* __restrict__ pattern = A.pattern;
  // Eight bins per thread and step: their loads are issued together before the first
  // recursion, so each thread keeps several state reads in flight.
  constexpr int kStep = 8;
  if (A.fp64) {
    double* __restrict__ cov = A.cov64 + base;
    double* __restrict__ proc = A.proc64 + base;
    for (int i0 = tid; i0 < n; i0 += kStep * nthr) {
      cf L[kStep];
      double c[kStep], q[kStep];
#pragma unroll
      for (int j = 0; j < kStep; ++j) {
        const int i = i0 + j * nthr;
        if (i < n) {
          L[j] = last[i];
          c[j] = cov[i];
          q[j] = proc[i];
        }
      }
#pragma unroll
      for (int j = 0; j < kStep; ++j) {
        const int i = i0 + j * nthr;
        if (i < n) {
          const int kk = i - (i / bins) * bins;
          if (!kalman_bin_fp64(spec[i], L[j], c[j], q[j], pattern, kk, P.kalman_r0, P.kalman_ratio2)) bad = true;
          last[i] = L[j];
          cov[i] = c[j];
          proc[i] = q[j];
        }
      }
    }
  } else {
    float* __restrict__ cov = A.cov32 + base;
    float* __restrict__ proc = A.proc32 + base;
    for (int i0 = tid; i0 < n; i0 += kStep * nthr) {
      cf L[kStep];
      float c[kStep], q[kStep];
#pragma unroll
      for (int j = 0; j < kStep; ++j) {
        const int i = i0 + j * nthr;
        if (i < n) {
          L[j] = last[i];
          c[j] = cov[i];
          q[j] = proc[i];
        }
      }
#pragma unroll
      for (int j = 0; j < kStep; ++j) {
        const int i = i0 + j * nthr;
        if (i < n) {
          const int kk = i - (i / bins) * bins;
          if (!kalman_bin(spec[i], L[j], c[j], q[j], pattern, kk, P.kalman_r0, P.kalman_ratio2)) bad = true;
          last[i] = L[j];
          cov[i] = c[j];
          proc[i] = q[j];
        }
      }
    }
  }
  if (bad) atomicOr(P.err, kErrNonFinite);
}

} // namespace nfd
