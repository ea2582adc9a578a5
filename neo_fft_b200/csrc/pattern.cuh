// FFT3D sampled noise model (pfactor) and its preview (pshow): the pattern search of
// src/algorithms/plan.cpp:227-288. The plane's block spectra come from the clip spectra
// pass (spectra_batch_kernel, analysis window applied); these kernels score every
// candidate block, extract the chosen block's power and render the preview block.
#pragma once
#include "tile_spatial.cuh"

namespace nfd {

// select_pattern (plan.cpp:248-269): per candidate, the template ratio of its DC, the
// power of the mean-removed spectrum and the weighted sum over bins in bin order.
__global__ void pattern_score_kernel(const DevPlan* plan, const cf* spectra, const float* weights, int x0, int y0,
                                     int nx, int ny, float* scores) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nx * ny) return;
  const DevPlan& P = *plan;
  const int by = y0 + c / nx, bx = x0 + c % nx;
  const size_t cnt = size_t(P.gx.count);
  const cf* S = spectra + size_t(by) * P.bins * cnt + bx;
  const float g = P.grid ? fdiv(fmul(P.mean_scale, S[0].r), P.grid[0].r) : 0.0f;
  float sum = 0.0f;
  for (int k = 0; k < P.bins; ++k) {
    const cf x = S[size_t(k) * cnt];
    const float re = fsub(x.r, P.grid ? fmul(g, P.grid[k].r) : 0.0f);
    const float im = fsub(x.i, P.grid ? fmul(g, P.grid[k].i) : 0.0f);
    const float q = fadd(fmul(re, re), fmul(im, im));
    sum = fadd(sum, fmul(q, weights[k]));
  }
  scores[c] = sum;
}

// The chosen block's unscaled power per bin (model power, kernels/scalar/model.cpp:21-29).
__global__ void pattern_power_kernel(const DevPlan* plan, const cf* spectra, int bx, int by, float* power) {
  const DevPlan& P = *plan;
  const size_t cnt = size_t(P.gx.count);
  const cf* S = spectra + size_t(by) * P.bins * cnt + bx;
  const float g = P.grid ? fdiv(fmul(P.mean_scale, S[0].r), P.grid[0].r) : 0.0f;
  for (int k = threadIdx.x; k < P.bins; k += blockDim.x) {
    const cf x = S[size_t(k) * cnt];
    const float re = fsub(x.r, P.grid ? fmul(g, P.grid[k].r) : 0.0f);
    const float im = fsub(x.i, P.grid ? fmul(g, P.grid[k].i) : 0.0f);
    power[k] = fadd(fmul(re, re), fmul(im, im));
  }
}

// pshow preview (plan.cpp:409-418): the chosen block gathered without window, forward
// and inverse transformed. One thread: a single block.
template <int STORAGE>
__global__ void pattern_block_kernel(const DevPlan* plan, const unsigned char* src, long long stride, int ox, int oy,
                                     cf* work, float* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const DevPlan& P = *plan;
  const int BH = P.bh, BW = P.bw, K = BW / 2 + 1;
  const bool codelet = P.codelet != 0;
  bool bad = false;
  float row[nf::kMaxProject];
  for (int y = 0; y < BH; ++y) {
    const unsigned char* srow = src + ptrdiff_t(reflect_axis(oy + y, P.gy)) * stride;
    for (int x = 0; x < BW; ++x) {
      const float v = fmul(fsub(load_sample<STORAGE>(srow, reflect_axis(ox + x, P.gx)), P.dec_base), P.dec_scale);
      if (!isfin(v)) bad = true;
      row[x] = v;
    }
    nf::row_forward<0>(row, BW, work + size_t(y) * K, P.tww, codelet);
  }
  cf col[nf::kMaxProject];
  for (int k = 0; k < K; ++k) {
    for (int y = 0; y < BH; ++y) col[y] = work[size_t(y) * K + k];
    nf::fft_1d<true, 0>(col, BH, P.twh, codelet);
    for (int y = 0; y < BH; ++y) work[size_t(y) * K + k] = col[y];
  }
  for (int k = 0; k < K; ++k) {
    for (int y = 0; y < BH; ++y) col[y] = work[size_t(y) * K + k];
    nf::fft_1d<false, 0>(col, BH, P.twh, codelet);
    for (int y = 0; y < BH; ++y) work[size_t(y) * K + k] = col[y];
  }
  const float fct = fdiv(1.0f, fmul(float(BW), float(BH)));
  for (int y = 0; y < BH; ++y) {
    nf::row_inverse<0>(work + size_t(y) * K, BW, fct, row, P.tww, codelet);
    for (int x = 0; x < BW; ++x) {
      if (!isfin(row[x])) bad = true;
      out[size_t(y) * BW + x] = row[x];
    }
  }
  if (bad) atomicOr(P.err, kErrNonFinite);
}

// Preview output: the accumulator is zero except for the block at cover (ox, oy).
template <int STORAGE>
__global__ void pattern_fill_kernel(const DevPlan* plan, unsigned char* dst, long long stride, int ox, int oy,
                                    const float* block) {
  const DevPlan& P = *plan;
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= P.gx.length || y >= P.gy.length) return;
  const int cy = y + P.gy.offset - oy, cx = x + P.gx.offset - ox;
  const float v = (cy >= 0 && cy < P.bh && cx >= 0 && cx < P.bw) ? block[size_t(cy) * P.bw + cx] : 0.0f;
  store_sample<STORAGE>(dst + ptrdiff_t(y) * stride, x, v, P);
}

} // namespace nfd
