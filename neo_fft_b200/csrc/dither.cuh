// DFTTest 8-bit dither (dither > 0; src/kernels/scalar/dither.cpp:4-41 with the noise of
// kernels/scalar/rows.cpp:6-8): error diffusion over the unconverted accumulator, left
// to right within a row, each pixel depending on its left neighbour and on the row
// above up to one column to the right.
//
// One CTA runs the rows of a band as a wavefront in lockstep: at step s, thread r
// (row r of the band) handles column s - 2r, so row r-1 has finished column x+1 one
// step earlier. The diffusion into the next row (3/16, 5/16, 1/16 of the error) lives
// in a four-entry ring per row (columns x-2 .. x+1 are the only live ones), the right
// neighbour's 7/16 in a register; every sum is formed with the reference's operands
// in the reference's order. The last row of a band leaves its diffusion row in
// `boundary` for the first row of the next band.
#pragma once
#include "device_plan.cuh"

namespace nfd {

__device__ __forceinline__ unsigned dither_mix(unsigned v) {
  v ^= v >> 16;
  v *= 0x7feb352du;
  v ^= v >> 15;
  v *= 0x846ca68bu;
  return v ^ (v >> 16);
}

__device__ __forceinline__ unsigned dither_hash(unsigned seed, unsigned n, unsigned p, unsigned y, unsigned x) {
  return dither_mix(dither_mix(dither_mix(dither_mix(dither_mix(seed ^ 0xa511e9b3u) ^ n) ^ p) ^ y) ^ x);
}

constexpr int kDitherRows = 1024;

__global__ void __launch_bounds__(kDitherRows) dither_kernel(const float* src, long long src_stride, unsigned char* dst,
                                                             long long dst_stride, int W, int H, int mode, unsigned seed,
                                                             unsigned frame, unsigned plane, float* boundary, int* err) {
  __shared__ float ring[kDitherRows][4];
  const int r = threadIdx.x, R = blockDim.x;
  const float scale = fadd(float(mode - 1), 0.5f), off = fmul(scale, 0.5f);
  bool bad = false;
  for (int band = 0; band * R < H; ++band) {
    const int y = band * R + r;
    const int rows = min(R, H - band * R);
    const bool active = r < rows;
    const float* srow = src + ptrdiff_t(active ? y : 0) * src_stride;
    unsigned char* drow = dst + ptrdiff_t(active ? y : 0) * dst_stride;
    float carry = 0.0f;  // 7/16 of the left neighbour's error, added to this row's incoming value
    const int steps = W + 2 * (rows - 1);
    for (int s = 0; s < steps; ++s) {
      const int x = s - 2 * r;
      if (active && x >= 0 && x < W) {
        // incoming diffusion of the row above (zero for the image's first row)
        float in = 0.0f;
        if (r > 0) in = ring[r - 1][x & 3];
        else if (band > 0) in = boundary[x];
        const float cur = x > 0 ? fadd(in, carry) : in;
        const float e = srow[x];
        if (!isfin(e)) bad = true;
        float v;
        if (mode == 1) {
          v = fadd(fadd(e, cur), 0.5f);
        } else {
          const float u = float(dither_hash(seed, frame, plane, unsigned(y), unsigned(x)) >> 8) * 0x1p-24f;
          v = fadd(fadd(fsub(fadd(e, fmul(u, scale)), off), cur), 0.5f);
        }
        if (!isfin(v)) bad = true;
        const unsigned char d = v <= 0.0f ? 0 : (v >= 255.0f ? 255 : (unsigned char)(v));
        drow[x] = d;
        const float error = fsub(e, float(d));
        float* own = ring[r];
        if (x > 0) own[(x - 1) & 3] = fadd(own[(x - 1) & 3], fmul(error, 0.1875f));
        own[x & 3] = x > 0 ? fadd(own[x & 3], fmul(error, 0.3125f)) : fadd(0.0f, fmul(error, 0.3125f));
        if (x + 1 < W) {
          carry = fmul(error, 0.4375f);
          own[(x + 1) & 3] = fadd(0.0f, fmul(error, 0.0625f));
        }
        if (r == rows - 1) {  // last row of the band: hand the finished diffusion to the next band
          if (x > 0) boundary[x - 1] = own[(x - 1) & 3];
          if (x == W - 1) boundary[x] = own[x & 3];
        }
      }
      __syncthreads();
    }
    __syncthreads();
  }
  if (bad) atomicOr(err, kErrNonFinite);
}

} // namespace nfd
