// Single-frame tile kernel: FFT3D bt=1/-1 (and Kalman render) and DFTTest tbsize=1.
//
// One CTA owns an output tile of the visible plane and computes every block that
// touches it, one block row at a time (rows of the reference's `by` loop,
// src/algorithms/plan.cpp:432-537 and 553-605):
//
//   A  row transforms   thread = (block, row): reflect+decode the source samples,
//                       apply the analysis window, real forward transform of the
//                       row into K = bw/2+1 bins (shared memory).
//   B  column pass      thread = (block, column): forward transform along y in
//                       registers; the DC of each block is exchanged through
//                       shared memory; per-bin filter; inverse transform along y.
//   C  row inverses     thread = (block, row): inverse real transform of the row,
//                       non-finite check, synthesis weighting into a block buffer.
//   D  overlap-add      thread = output pixel: contributions are added in the
//                       reference's order (block row ascending, then block column
//                       ascending; FFT3D sums a row strip first and applies the
//                       vertical synthesis weight once per block row), so every
//                       output is owner-written and deterministic without atomics.
//
// After the last block row the tile is quantised and stored.
#pragma once
#include "device_plan.cuh"

namespace nfd {

// Sample loads (u8/u16 integer, or f32).
template <int STORAGE>
__device__ __forceinline__ float load_sample(const unsigned char* row, int x) {
  if (STORAGE == kStoreU8) return float(row[x]);
  if (STORAGE == kStoreU16) return float(reinterpret_cast<const unsigned short*>(row)[x]);
  return reinterpret_cast<const float*>(row)[x];
}

__device__ __forceinline__ int reflect_axis(int c, const DevAxis& a) {
  const int j = c - a.offset;
  return j < 0 ? -j : (j < a.length ? j : 2 * a.length - 2 - j);
}

__device__ __forceinline__ int floor_div_i(int v, int d) { return v >= 0 ? v / d : -((-v + d - 1) / d); }

// Output conversion (kernels/scalar/spatial.cpp:89-129): FFT3D integer
// (acc+0.5)+base, DFTTest integer acc*scale+0.5, clipped to [0, peak] and
// truncated; FFT3D float clipped to [0,1]; DFTTest float acc*scale unclipped.
template <int STORAGE>
__device__ __forceinline__ void store_sample(unsigned char* row, int x, float acc, const DevPlan& P) {
  if (STORAGE == kStoreF32) {
    float v;
    if (P.algo == 0) v = acc < 0.0f ? 0.0f : (1.0f < acc ? 1.0f : acc);
    else v = fmul(acc, P.out_scale);
    reinterpret_cast<float*>(row)[x] = v;
    return;
  }
  const float v = P.algo == 0 ? fadd(fadd(acc, 0.5f), P.out_base) : fadd(fmul(acc, P.out_scale), 0.5f);
  const float c = v < 0.0f ? 0.0f : (P.out_peak < v ? P.out_peak : v);
  if (STORAGE == kStoreU8) row[x] = (unsigned char)(c);
  else reinterpret_cast<unsigned short*>(row)[x] = (unsigned short)(c);
}

struct TileShape {
  int tw, th;    // output tile (plane pixels)
  int nbx_max;   // blocks per block row that can touch a tile
  int threads;
};

// Shared-memory layout (floats): spec [nbx][bh][K] complex | obuf [nbx][bh][bw]
// | acc [th][tw] | dc [2*nbx].
__host__ __device__ inline size_t tile_smem_bytes(int bh, int bw, const TileShape& s) {
  const size_t K = size_t(bw / 2 + 1);
  return sizeof(float) * (size_t(s.nbx_max) * bh * K * 2 + size_t(s.nbx_max) * bh * bw + size_t(s.th) * s.tw +
                          2 * size_t(s.nbx_max));
}

template <int BHC, int BWC, int STORAGE>
__global__ void __launch_bounds__(256) spatial_tile_kernel(DevPlan P, TileShape S, const unsigned char* src,
                                                           ptrdiff_t src_stride, unsigned char* dst,
                                                           ptrdiff_t dst_stride, const cf* kalman_L) {
  extern __shared__ float smem[];
  const int BH = BHC > 0 ? BHC : P.bh;
  const int BW = BWC > 0 ? BWC : P.bw;
  const int K = BW / 2 + 1;
  constexpr int CAPH = BHC > 0 ? BHC : nf::kMaxProject;
  constexpr int CAPW = BWC > 0 ? BWC : nf::kMaxProject;
  constexpr int UH = BHC > 0 ? CAPH : 1, UW = BWC > 0 ? CAPW : 1;  // unroll compile-time sizes only
  // Square 8/16/32 blocks always use the codelet networks; sized instantiations
  // know it at compile time, so only one transform family is generated.
  constexpr bool kCodelet = BHC == BWC && (BWC == 8 || BWC == 16 || BWC == 32);
  const bool codelet = kCodelet || (BHC == 0 && P.codelet != 0);
  const DevAxis gx = P.gx, gy = P.gy;

  cf* spec = reinterpret_cast<cf*>(smem);
  float* obuf = smem + size_t(S.nbx_max) * BH * K * 2;
  float* acc = obuf + size_t(S.nbx_max) * BH * BW;
  float* dc = acc + size_t(S.th) * S.tw;

  const int tid = threadIdx.x, nthr = blockDim.x;
  // Tile in plane coordinates and in cover coordinates.
  const int px0 = blockIdx.x * S.tw, py0 = blockIdx.y * S.th;
  const int tw = min(S.tw, gx.length - px0), th = min(S.th, gy.length - py0);
  const int X0 = px0 + gx.offset, Y0 = py0 + gy.offset;
  const int bx_lo = max(0, floor_div_i(X0 - BW, gx.step) + 1);
  const int bx_hi = min(gx.count - 1, floor_div_i(X0 + tw - 1, gx.step));
  const int by_lo = max(0, floor_div_i(Y0 - BH, gy.step) + 1);
  const int by_hi = min(gy.count - 1, floor_div_i(Y0 + th - 1, gy.step));
  const int nbx = bx_hi - bx_lo + 1;
  bool bad = false;

  for (int i = tid; i < S.th * S.tw; i += nthr) acc[i] = 0.0f;

  const float fct = fdiv(1.0f, fmul(float(BW), float(BH)));

  for (int by = by_lo; by <= by_hi; ++by) {
    const int oy = by * gy.step;
    // ---- A: row transforms -------------------------------------------------
    if (!kalman_L) {
      for (int task = tid; task < nbx * BH; task += nthr) {
        const int b = task / BH, y = task - b * BH;
        const int ox = (bx_lo + b) * gx.step;
        const unsigned char* srow = src + ptrdiff_t(reflect_axis(oy + y, gy)) * src_stride;
        float row[CAPW];
#pragma unroll UW
        for (int x = 0; x < CAPW; ++x) {
          if (x < BW) {
            const float s = load_sample<STORAGE>(srow, reflect_axis(ox + x, gx));
            const float v = fmul(fsub(s, P.dec_base), P.dec_scale);
            if (!isfin(v)) bad = true;
            row[x] = P.algo == 0 ? fmul(fmul(v, P.wya[y]), P.wxa[x]) : fmul(v, P.h[y * BW + x]);
          }
        }
        nf::row_forward<BWC>(row, BW, spec + (size_t(b) * BH + y) * K, P.tww, codelet);
      }
      __syncthreads();
    }
    // ---- B: column forward, filter, column inverse --------------------------
    const int ncol = nbx * K;
    for (int base = 0; base < ncol; base += nthr) {
      const int task = base + tid;
      const bool active = task < ncol;
      const int b = active ? task / K : 0, k = active ? task - b * K : 0;
      cf col[CAPH];
      if (active) {
        cf* sp = spec + size_t(b) * BH * K + k;
        if (kalman_L) {
          const cf* L = kalman_L + (size_t(by) * gx.count + (bx_lo + b)) * P.bins + k;
#pragma unroll UH
          for (int y = 0; y < CAPH; ++y)
            if (y < BH) col[y] = L[size_t(y) * K];
        } else {
#pragma unroll UH
          for (int y = 0; y < CAPH; ++y)
            if (y < BH) col[y] = sp[size_t(y) * K];
          nf::fft_1d<true, BHC>(col, BH, P.twh, codelet);
        }
        if (k == 0) dc[b] = col[0].r;
      }
      __syncthreads();
      if (active) {
        const float g = P.grid ? fdiv(fmul(P.mean_scale, dc[b]), P.grid[0].r) : 0.0f;
        if (P.algo == 1 || P.fft3d_mode != kEnhanceOnly) {
#pragma unroll UH
          for (int y = 0; y < CAPH; ++y)
            if (y < BH) col[y] = spectral_bin(col[y], P.grid, y * K + k, g, P.filt, bad);
        }
        if (P.algo == 0 && P.fft3d_mode == kWienerThenEnh && k == 0) dc[nbx + b] = col[0].r;
      }
      if (P.algo == 0 && P.fft3d_mode != kWienerFused && P.enh.enh) {
        // enhance(): template ratio recomputed from the spectrum being enhanced
        // (plan.cpp:325-329).
        if (P.fft3d_mode == kWienerThenEnh) __syncthreads();
        if (active) {
          const float dcv = P.fft3d_mode == kWienerThenEnh ? dc[nbx + b] : dc[b];
          const float g2 = P.grid ? fdiv(fmul(P.mean_scale, dcv), P.grid[0].r) : 0.0f;
#pragma unroll UH
          for (int y = 0; y < CAPH; ++y)
            if (y < BH) col[y] = spectral_bin(col[y], P.grid, y * K + k, g2, P.enh, bad);
        }
      }
      if (active) {
        nf::fft_1d<false, BHC>(col, BH, P.twh, codelet);
        cf* sp = spec + size_t(b) * BH * K + k;
#pragma unroll UH
        for (int y = 0; y < CAPH; ++y)
          if (y < BH) sp[size_t(y) * K] = col[y];
      }
      __syncthreads();
    }
    // ---- C: row inverses and synthesis weighting ----------------------------
    for (int task = tid; task < nbx * BH; task += nthr) {
      const int b = task / BH, y = task - b * BH;
      if (P.center && y != BH / 2) continue;
      float row[CAPW];
      nf::row_inverse<BWC>(spec + (size_t(b) * BH + y) * K, BW, fct, row, P.tww, codelet);
      float* ob = obuf + (size_t(b) * BH + y) * BW;
#pragma unroll UW
      for (int x = 0; x < CAPW; ++x) {
        if (x < BW) {
          if (!isfin(row[x])) bad = true;
          ob[x] = P.algo == 0 ? fmul(row[x], P.wxs[x]) : fmul(row[x], P.hsyn[y * BW + x]);
        }
      }
    }
    __syncthreads();
    // ---- D: ordered overlap-add into the tile accumulator --------------------
    const int ylo = max(oy, Y0), yhi = min(oy + BH, Y0 + th);
    const int band = yhi - ylo;
    if (band > 0) {
      for (int i = tid; i < band * tw; i += nthr) {
        const int yy = i / tw, xx = i - yy * tw;
        const int Y = ylo + yy, X = X0 + xx;
        const int ly = Y - oy;
        float* a = acc + size_t(Y - Y0) * S.tw + xx;
        if (P.center) {
          const int bc = X - BW / 2;  // block whose centre is X (step 1)
          if (ly == BH / 2 && bc >= bx_lo && bc <= bx_hi)
            *a = obuf[(size_t(bc - bx_lo) * BH + ly) * BW + BW / 2];
          continue;
        }
        const int b0 = max(bx_lo, floor_div_i(X - BW, gx.step) + 1), b1 = min(bx_hi, floor_div_i(X, gx.step));
        if (P.algo == 0) {
          float r = 0.0f;
          for (int bb = b0; bb <= b1; ++bb) r = fadd(r, obuf[(size_t(bb - bx_lo) * BH + ly) * BW + (X - bb * gx.step)]);
          *a = fadd(*a, fmul(r, P.wys[ly]));
        } else {
          float s = *a;
          for (int bb = b0; bb <= b1; ++bb) s = fadd(s, obuf[(size_t(bb - bx_lo) * BH + ly) * BW + (X - bb * gx.step)]);
          *a = s;
        }
      }
    }
    __syncthreads();
  }
  // ---- store -----------------------------------------------------------------
  for (int i = tid; i < th * tw; i += nthr) {
    const int yy = i / tw, xx = i - yy * tw;
    const float v = acc[size_t(yy) * S.tw + xx];
    if (!isfin(v)) bad = true;
    store_sample<STORAGE>(dst + ptrdiff_t(py0 + yy) * dst_stride, px0 + xx, v, P);
  }
  if (bad) atomicOr(P.err, kErrNonFinite);
}

} // namespace nfd
