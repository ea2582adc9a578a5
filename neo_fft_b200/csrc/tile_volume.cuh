// Multi-frame tile kernel: FFT3D bt=2..5 (temporal Wiener) and DFTTest tbsize>1
// (3-D volumes, tmode 0 centre slice and tmode 1 temporal overlap-add).
//
// Like the single-frame kernel, one CTA owns an output tile and computes every
// block touching it; blocks are processed per block row in chunks of `nbc`
// columns. Per chunk:
//
//   A   rows       thread = (block, slot, row): reflect+decode+window, row transform
//   B1  columns    thread = (block, slot, column): forward transform along y
//   T   time       thread = (block, row, column) bin:
//                    FFT3D   — T-point DFT with the reference's float twiddles,
//                              Wiener on every temporal frequency against the
//                              current frame's degrid template, inverse at the
//                              centre slot only (src/kernels/scalar/spectral.cpp:90-160);
//                    DFTTest — forward project transform along time (the DC of
//                              the whole volume is exchanged through shared memory),
//                              ftype filter over the T*bins spectrum, full inverse
//                              along time, keep the target slice (plan.cpp:568-589).
//   B2  columns    thread = (block, column): FFT3D enhancement of the recovered
//                  spectrum (plan.cpp:516), inverse transform along y
//   C   rows       thread = (block, row): inverse row transform of the one output
//                  slice, synthesis weighting
//   D   overlap    thread = pixel, reference order: temporal block, block row,
//                  block column (DFTTest); FFT3D keeps the row strip across chunks
//                  and applies the vertical weight when the block row completes.
#pragma once
#include "tile_spatial.cuh"

namespace nfd {

constexpr int kMaxSlots = 225;  // tmode 1: up to 15 covering blocks of 15 slots

struct VolumeSources {
  const unsigned char* ptr[kMaxSlots];
  long long stride[kMaxSlots];
  int target[15];  // target slice per temporal block (DFTTest)
  int nblocks;     // temporal blocks (1 unless DFTTest tmode 1)
  int ola;         // DFTTest tmode 1
};

struct VolumeShape {
  int tw, th, nbc;  // output tile and blocks per chunk
  int threads;
};

// Shared layout: spec [nbc][T][bh][K] complex | obuf [nbc][bh][bw] | strip [bh][tw]
// | acc [th][tw] | dc [nbc].
__host__ __device__ inline size_t volume_smem_bytes(int bh, int bw, int T, const VolumeShape& s) {
  const size_t K = size_t(bw / 2 + 1);
  return sizeof(float) * (size_t(s.nbc) * T * bh * K * 2 + size_t(s.nbc) * bh * bw + size_t(bh) * s.tw +
                          size_t(s.th) * s.tw + size_t(s.nbc));
}

template <int BHC, int BWC, int STORAGE>
__global__ void __launch_bounds__(256) volume_tile_kernel(DevPlan P, VolumeShape S, VolumeSources V,
                                                          unsigned char* dst, ptrdiff_t dst_stride) {
  extern __shared__ float smem[];
  const int BH = BHC > 0 ? BHC : P.bh;
  const int BW = BWC > 0 ? BWC : P.bw;
  const int K = BW / 2 + 1;
  const int T = P.T;
  constexpr int CAPH = BHC > 0 ? BHC : nf::kMaxProject;
  constexpr int CAPW = BWC > 0 ? BWC : nf::kMaxProject;
  constexpr int UH = BHC > 0 ? CAPH : 1, UW = BWC > 0 ? CAPW : 1;
  constexpr bool kCodelet = BHC == BWC && (BWC == 8 || BWC == 16 || BWC == 32);
  const bool codelet = kCodelet || (BHC == 0 && P.codelet != 0);
  const DevAxis gx = P.gx, gy = P.gy;
  const bool fft3d = P.algo == 0;

  cf* spec = reinterpret_cast<cf*>(smem);
  float* obuf = smem + size_t(S.nbc) * T * BH * K * 2;
  float* strip = obuf + size_t(S.nbc) * BH * BW;
  float* acc = strip + size_t(BH) * S.tw;
  float* dc = acc + size_t(S.th) * S.tw;
  const size_t slot_bins = size_t(BH) * K;        // one slice of one block
  const size_t blk_bins = size_t(T) * slot_bins;  // one volume

  const int tid = threadIdx.x, nthr = blockDim.x;
  const int px0 = blockIdx.x * S.tw, py0 = blockIdx.y * S.th;
  const int tw = min(S.tw, gx.length - px0), th = min(S.th, gy.length - py0);
  const int X0 = px0 + gx.offset, Y0 = py0 + gy.offset;
  const int bx_lo = max(0, floor_div_i(X0 - BW, gx.step) + 1);
  const int bx_hi = min(gx.count - 1, floor_div_i(X0 + tw - 1, gx.step));
  const int by_lo = max(0, floor_div_i(Y0 - BH, gy.step) + 1);
  const int by_hi = min(gy.count - 1, floor_div_i(Y0 + th - 1, gy.step));
  const int c = T / 2;
  const float fct = fdiv(1.0f, fmul(float(BW), float(BH)));
  const float fct3 = fdiv(1.0f, fmul(fmul(float(T), float(BH)), float(BW)));
  const float volume = fmul(fmul(float(T), float(BW)), float(BH));
  bool bad = false;

  for (int i = tid; i < S.th * S.tw; i += nthr) acc[i] = 0.0f;

  for (int tb = 0; tb < V.nblocks; ++tb) {
    const int zt = fft3d ? c : (V.ola ? V.target[tb] : c);  // output slice
    for (int by = by_lo; by <= by_hi; ++by) {
      const int oy = by * gy.step;
      for (int i = tid; i < BH * S.tw; i += nthr) strip[i] = 0.0f;
      for (int cb = bx_lo; cb <= bx_hi; cb += S.nbc) {
        const int nb = min(S.nbc, bx_hi - cb + 1);
        __syncthreads();
        // ---- A: rows of every slice ----------------------------------------
        for (int task = tid; task < nb * T * BH; task += nthr) {
          const int b = task / (T * BH), r = task - b * T * BH, z = r / BH, y = r - z * BH;
          const int ox = (cb + b) * gx.step;
          const unsigned char* srow = V.ptr[tb * T + z] + ptrdiff_t(reflect_axis(oy + y, gy)) * V.stride[tb * T + z];
          float row[CAPW];
#pragma unroll UW
          for (int x = 0; x < CAPW; ++x) {
            if (x < BW) {
              const float s = load_sample<STORAGE>(srow, reflect_axis(ox + x, gx));
              const float v = fmul(fsub(s, P.dec_base), P.dec_scale);
              if (!isfin(v)) bad = true;
              row[x] = fft3d ? fmul(fmul(v, P.wya[y]), P.wxa[x]) : fmul(v, P.h[(z * BH + y) * BW + x]);
            }
          }
          nf::row_forward<BWC>(row, BW, spec + b * blk_bins + size_t(z) * slot_bins + size_t(y) * K, P.tww, codelet);
        }
        __syncthreads();
        // ---- B1: forward columns of every slice ----------------------------
        for (int task = tid; task < nb * T * K; task += nthr) {
          const int b = task / (T * K), r = task - b * T * K, z = r / K, k = r - z * K;
          cf* sp = spec + b * blk_bins + size_t(z) * slot_bins + k;
          cf col[CAPH];
#pragma unroll UH
          for (int y = 0; y < CAPH; ++y)
            if (y < BH) col[y] = sp[size_t(y) * K];
          nf::fft_1d<true, BHC>(col, BH, P.twh, codelet);
#pragma unroll UH
          for (int y = 0; y < CAPH; ++y)
            if (y < BH) sp[size_t(y) * K] = col[y];
        }
        __syncthreads();
        // ---- T: temporal transform and filter per bin ------------------------
        const int nbin = nb * BH * K;
        if (fft3d) {
          // each block's template scale from the centre slot's DC, once per block
          for (int b = tid; b < nb; b += nthr) {
            const float g = P.grid ? fdiv(fmul(P.mean_scale, spec[b * blk_bins + size_t(c) * slot_bins].r), P.grid[0].r)
                                   : 0.0f;
            if (P.grid && !isfin(g)) bad = true;
            dc[b] = g;
          }
          __syncthreads();
          for (int task = tid; task < nbin; task += nthr) {
            const int b = task / int(slot_bins), kk = task - b * int(slot_bins);
            cf* bp = spec + b * blk_bins + kk;
            const float g = dc[b];
            const cf M = P.grid ? cf{fmul(g, P.grid[kk].r), fmul(g, P.grid[kk].i)} : cf{0.0f, 0.0f};
            const cf gT = {fmul(M.r, float(T)), fmul(M.i, float(T))};
            cf Fv[5];
            for (int m = 0; m < T; ++m) {
              cf sum = {0.0f, 0.0f};
              for (int j = 0; j < T; ++j) sum = nf::cadd(sum, nf::cmul_plain(bp[size_t(j) * slot_bins], P.tfwd[m * T + j]));
              Fv[m] = sum;
            }
            const float noise =
                P.filt.primary ? fmul(P.filt.primary[kk], P.noise_mult) : P.noise_uniform;
            if (!isfin(noise)) bad = true;
            cf y = {0.0f, 0.0f};
            for (int m = 0; m < T; ++m) {
              const cf R = m == 0 ? nf::csub(Fv[0], gT) : Fv[m];
              const float power = fadd(fmul(R.r, R.r), fmul(R.i, R.i));
              if (!isfin(power)) bad = true;
              const float q = fadd(power, 1e-15f);
              const float gr = fdiv(fsub(q, noise), q);
              const float gain = gr < P.lower ? P.lower : gr;
              cf Rf = {fmul(gain, R.r), fmul(gain, R.i)};
              if (m == 0) Rf = nf::cadd(Rf, gT);
              y = nf::cadd(y, nf::cmul_plain(Rf, P.tinv[m]));
            }
            const float invT = fdiv(1.0f, float(T));
            bp[0] = {fmul(y.r, invT), fmul(y.i, invT)};  // output spectrum in slot 0
          }
          __syncthreads();
        } else {
          // forward along time; the volume DC is bin 0 of slot 0 afterwards
          for (int task = tid; task < nbin; task += nthr) {
            const int b = task / int(slot_bins), kk = task - b * int(slot_bins);
            cf* bp = spec + b * blk_bins + kk;
            cf line[15];
            for (int z = 0; z < T; ++z) line[z] = bp[size_t(z) * slot_bins];
            nf::fft_project<true, 0, 16>(line, T, P.twt);
            for (int z = 0; z < T; ++z) bp[size_t(z) * slot_bins] = line[z];
            // the block's template scale from its volume DC, once per block (the filter reads it per bin)
            if (kk == 0)
              dc[b] = (P.grid && P.mean_scale != 0.0f && P.grid[0].r != 0.0f) ? fdiv(fmul(P.mean_scale, line[0].r), P.grid[0].r)
                                                                              : 0.0f;
          }
          __syncthreads();
          // The filter type fixed at compile time per branch (no switch per element).
          auto filter_lines = [&](auto ft) {
            constexpr int FT = decltype(ft)::value;
            for (int task = tid; task < nbin; task += nthr) {
              const int b = task / int(slot_bins), kk = task - b * int(slot_bins);
              cf* bp = spec + b * blk_bins + kk;
              const float g = dc[b];  // the block's template scale
              cf line[15];
              for (int z = 0; z < T; ++z)
                line[z] = spectral_bin<FT>(bp[size_t(z) * slot_bins], P.grid, z * int(slot_bins) + kk, g, P.filt, bad);
              nf::fft_project<false, 0, 16>(line, T, P.twt);
              bp[0] = line[zt];  // target slice in slot 0
            }
          };
          switch (P.filt.type) {
            case -1: filter_lines(std::integral_constant<int, -1>{}); break;
            case 0:  // the exponent mode fixed too
              if (P.filt.emode == 0) filter_lines(std::integral_constant<int, kFt0Ratio>{});
              else if (P.filt.emode == 1) filter_lines(std::integral_constant<int, kFt0Sqrt>{});
              else filter_lines(std::integral_constant<int, kFt0Pow>{});
              break;
            case 1: filter_lines(std::integral_constant<int, 1>{}); break;
            case 2: filter_lines(std::integral_constant<int, 2>{}); break;
            case 3: filter_lines(std::integral_constant<int, 3>{}); break;
            case 4: filter_lines(std::integral_constant<int, 4>{}); break;
            default: filter_lines(std::integral_constant<int, -3>{}); break;
          }
          __syncthreads();
        }
        // ---- B2: enhancement (FFT3D) and inverse columns --------------------
        for (int task = tid; task < nb * K; task += nthr) {
          const int b = task / K, k = task - b * K;
          cf* sp = spec + b * blk_bins + k;
          cf col[CAPH];
#pragma unroll UH
          for (int y = 0; y < CAPH; ++y)
            if (y < BH) col[y] = sp[size_t(y) * K];
          if (fft3d && P.enh.enh) {
            const float g2 = P.grid ? fdiv(fmul(P.mean_scale, spec[b * blk_bins].r), P.grid[0].r) : 0.0f;
#pragma unroll UH
            for (int y = 0; y < CAPH; ++y)
              if (y < BH) col[y] = spectral_bin<-2>(col[y], P.grid, y * K + k, g2, P.enh, bad);
          }
          nf::fft_1d<false, BHC>(col, BH, P.twh, codelet);
          // Slot 0 keeps the recovered spectrum whose DC other threads still read
          // for the enhancement ratio; the inverse goes to the dead slot 1.
          cf* dstc = spec + b * blk_bins + slot_bins + k;
#pragma unroll UH
          for (int y = 0; y < CAPH; ++y)
            if (y < BH) dstc[size_t(y) * K] = col[y];
        }
        __syncthreads();
        // ---- C: inverse rows of the output slice -----------------------------
        for (int task = tid; task < nb * BH; task += nthr) {
          const int b = task / BH, y = task - b * BH;
          if (P.center && y != BH / 2) continue;
          const cf* srcb = spec + b * blk_bins + slot_bins + size_t(y) * K;
          float row[CAPW];
          nf::row_inverse<BWC>(srcb, BW, fft3d ? fct : fct3, row, P.tww, codelet);
          float* ob = obuf + (size_t(b) * BH + y) * BW;
#pragma unroll UW
          for (int x = 0; x < CAPW; ++x) {
            if (x < BW) {
              if (!isfin(row[x])) bad = true;
              float v;
              if (fft3d) v = fmul(row[x], P.wxs[x]);
              else if (V.ola) v = fmul(fmul(volume, row[x]), P.h[(zt * BH + y) * BW + x]);
              else v = fmul(row[x], P.hsyn[(zt * BH + y) * BW + x]);
              ob[x] = v;
            }
          }
        }
        __syncthreads();
        // ---- D: ordered overlap-add of this chunk -----------------------------
        const int ylo = max(oy, Y0), yhi = min(oy + BH, Y0 + th);
        const int band = yhi - ylo;
        for (int i = tid; band > 0 && i < band * tw; i += nthr) {
          const int yy = i / tw, xx = i - yy * tw;
          const int Y = ylo + yy, X = X0 + xx, ly = Y - oy;
          if (P.center) {
            const int bc = X - BW / 2;
            if (ly == BH / 2 && bc >= cb && bc < cb + nb) {
              float* a = acc + size_t(Y - Y0) * S.tw + xx;
              const float v = obuf[(size_t(bc - cb) * BH + ly) * BW + BW / 2];
              *a = V.ola ? fadd(*a, v) : v;
            }
            continue;
          }
          const int b0 = max(cb, floor_div_i(X - BW, gx.step) + 1), b1 = min(cb + nb - 1, floor_div_i(X, gx.step));
          if (fft3d) {
            float* r = strip + size_t(ly) * S.tw + xx;
            float s = *r;
            for (int bb = b0; bb <= b1; ++bb) s = fadd(s, obuf[(size_t(bb - cb) * BH + ly) * BW + (X - bb * gx.step)]);
            *r = s;
          } else {
            float* a = acc + size_t(Y - Y0) * S.tw + xx;
            float s = *a;
            for (int bb = b0; bb <= b1; ++bb) s = fadd(s, obuf[(size_t(bb - cb) * BH + ly) * BW + (X - bb * gx.step)]);
            *a = s;
          }
        }
      }
      if (fft3d) {
        __syncthreads();
        const int ylo = max(oy, Y0), yhi = min(oy + BH, Y0 + th);
        for (int i = tid; yhi > ylo && i < (yhi - ylo) * tw; i += nthr) {
          const int yy = i / tw, xx = i - yy * tw;
          const int Y = ylo + yy, ly = Y - oy;
          float* a = acc + size_t(Y - Y0) * S.tw + xx;
          *a = fadd(*a, fmul(strip[size_t(ly) * S.tw + xx], P.wys[ly]));
        }
      }
      __syncthreads();
    }
  }
  for (int i = tid; i < th * tw; i += nthr) {
    const int yy = i / tw, xx = i - yy * tw;
    const float v = acc[size_t(yy) * S.tw + xx];
    if (!isfin(v)) bad = true;
    store_sample<STORAGE>(dst + ptrdiff_t(py0 + yy) * dst_stride, px0 + xx, v, P);
  }
  if (bad) atomicOr(P.err, kErrNonFinite);
}

} // namespace nfd
