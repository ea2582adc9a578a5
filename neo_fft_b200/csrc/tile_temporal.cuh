// FFT3D temporal clips (bt=2..5) in two passes over HBM:
//   pass 1 (spectra_batch_kernel): windowed spatial r2c of every block of a frame,
//     computed once per frame and written to a per-plane ring of T frame spectra —
//     the device counterpart of the reference's raw-spectrum cache (SpectraCache,
//     src/algorithms/plan.cpp:437-447);
//   pass 2 (temporal_batch_kernel): the streaming strip (strip_tile in temporal mode)
//     reads the T spectra of each block, filters across time and reconstructs.
// Clip edges, where the host layer falls back to a single frame (filter.hpp:407-421),
// run as pixel-mode strips of the batched spatial kernel beside pass 2.
#pragma once
#include "tile_spatial.cuh"

namespace nfd {

// Spectrum layout of one frame: [block row][bin][block column] complex, so the
// threads of a warp (consecutive block columns) read and write consecutive words.
struct SpectraJob {
  const unsigned char* src;
  long long src_stride;
  cf* out;
  int plan;
  int chunks_x;  // block-column chunks per block row
};

struct SpectraWork {
  const DevPlan* plans;
  const SpectraJob* jobs;
  const int* item_base;  // prefix sums of (block rows x chunks) per job (njobs+1)
  int njobs;
  int nbc;               // block columns per chunk
};

// Shared layout (floats): wxa[bw] wya[bh] | ring [bh][pitch] | spec [bh][K][nbc] complex.
__host__ __device__ inline size_t spectra_smem_bytes(int bh, int bw, int step, int nbc) {
  const size_t K = size_t(bw / 2 + 1);
  const size_t win = size_t(nbc - 1) * step + bw;
  const size_t pitch = (win + 3) & ~size_t(3);
  return sizeof(float) * (((size_t(bw + bh) + 3) & ~size_t(3)) + size_t(bh) * pitch + 2 * size_t(bh) * K * nbc);
}

// Two CTAs per SM for compile-time shapes: one CTA's staging loads overlap the other's
// transforms (the host keeps a chunk within half the SM's shared memory).
template <int BHC, int BWC>
struct SpectraOccupancy {
  static constexpr int value = BHC > 0 ? 2 : 1;
};

template <int BHC, int BWC, int STORAGE>
__global__ void __launch_bounds__(256, SpectraOccupancy<BHC, BWC>::value) spectra_batch_kernel(SpectraWork W) {
  extern __shared__ float smem[];
  const int BH = BHC > 0 ? BHC : W.plans[0].bh;
  const int BW = BWC > 0 ? BWC : W.plans[0].bw;
  const int K = BW / 2 + 1;
  constexpr int CAPH = BHC > 0 ? BHC : nf::kMaxProject;
  constexpr int CAPW = BWC > 0 ? BWC : nf::kMaxProject;
  constexpr int UH = BHC > 0 ? CAPH : 1, UW = BWC > 0 ? CAPW : 1;
  constexpr bool kCodelet = BHC == BWC && (BWC == 8 || BWC == 16 || BWC == 32);

  const int item = blockIdx.x;
  int lo = 0, hi = W.njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (W.item_base[mid] <= item) lo = mid;
    else hi = mid - 1;
  }
  __shared__ SpectraJob sJ;
  __shared__ DevPlan sP;
  if (threadIdx.x == 0) {
    sJ = W.jobs[lo];
    sP = W.plans[sJ.plan];
  }
  __syncthreads();
  const DevPlan& P = sP;
  const bool codelet = kCodelet || (BHC == 0 && P.codelet != 0);
  const DevAxis gx = P.gx, gy = P.gy;
  const int local = item - W.item_base[lo];
  const int by = local / sJ.chunks_x, chunk = local - by * sJ.chunks_x;
  const int nbc = W.nbc;
  const int bx0 = chunk * nbc, nb = min(nbc, gx.count - bx0);
  const int oy = by * gy.step, cx0 = bx0 * gx.step;
  const int win = (nb - 1) * gx.step + BW;
  const int pitch = ((nbc - 1) * gx.step + BW + 3) & ~3;
  const int tid = threadIdx.x, nthr = blockDim.x;

  float* wxa = smem;
  float* wya = wxa + BW;
  float* ring = smem + ((BW + BH + 3) & ~3);
  cf* spec = reinterpret_cast<cf*>(ring + size_t(BH) * pitch);
  for (int i = tid; i < BW; i += nthr) wxa[i] = P.wxa[i];
  for (int i = tid; i < BH; i += nthr) wya[i] = P.wya[i];
  bool bad = false;
  // stage the block row's samples (decoded, reflected) with coalesced loads
  for (Cursor2 c(tid, nthr, win); c.y < BH; c.next()) {
    const int y = c.y, xx = c.x;
    const unsigned char* srow = sJ.src + ptrdiff_t(reflect_axis(oy + y, gy)) * sJ.src_stride;
    const float sv = load_sample<STORAGE>(srow, reflect_axis(cx0 + xx, gx));
    const float v = fmul(fsub(sv, P.dec_base), P.dec_scale);
    if (STORAGE == kStoreF32 && !isfin(v)) bad = true;  // decoded integers are finite
    ring[size_t(y) * pitch + xx] = v;
  }
  __syncthreads();
  for (Cursor2 c(tid, nthr, nb); c.y < BH; c.next()) {
    const int y = c.y, b = c.x;
    const float* in = ring + size_t(y) * pitch + b * gx.step;
    float row[CAPW];
#pragma unroll UW
    for (int x = 0; x < CAPW; ++x)
      if (x < BW) row[x] = fmul(fmul(in[x], wya[y]), wxa[x]);
    nf::row_forward<BWC>(row, BW, spec + size_t(y) * K * nbc + b, P.tww, codelet, nbc);
  }
  __syncthreads();
  const size_t cnt = size_t(gx.count);
  cf* out = sJ.out + size_t(by) * P.bins * cnt + bx0;
  for (Cursor2 c(tid, nthr, nb); c.y < K; c.next()) {
    const int k = c.y, b = c.x;
    cf col[CAPH];
    const cf* sp = spec + size_t(k) * nbc + b;
#pragma unroll UH
    for (int y = 0; y < CAPH; ++y)
      if (y < BH) col[y] = sp[size_t(y) * K * nbc];
    nf::fft_1d<true, BHC>(col, BH, P.twh, codelet);
#pragma unroll UH
    for (int y = 0; y < CAPH; ++y)
      if (y < BH) out[size_t(y * K + k) * cnt + b] = col[y];
  }
  if (bad) atomicOr(P.err, kErrNonFinite);
}

// DFTTest tmode 1 with tosize 0 (temporal_grid.hpp:5-40): every output frame lies in
// exactly one temporal block, so a block's volume is transformed, filtered and inverted
// along time once, and all T filtered slice spectra are kept for the T outputs.
constexpr int kMaxVolumeSlots = 15;
struct VolumeSpectraJob {
  const unsigned char* src[kMaxVolumeSlots];
  long long src_stride[kMaxVolumeSlots];
  cf* out[kMaxVolumeSlots];
  int plan;
  int chunks_x;
};

struct VolumeSpectraWork {
  const DevPlan* plans;
  const VolumeSpectraJob* jobs;
  const int* item_base;  // prefix sums of (block rows x chunks) per job (njobs+1)
  int njobs;
  int nbc;
};

// Shared layout (floats): h [T][bh][bw] | ring [bh][pitch] | spec [T][bh][K][nbc] complex
// | dc [nbc].
__host__ __device__ inline size_t volume_spectra_smem_bytes(int bh, int bw, int T, int step, int nbc) {
  const size_t K = size_t(bw / 2 + 1);
  const size_t win = size_t(nbc - 1) * step + bw;
  const size_t pitch = (win + 3) & ~size_t(3);
  const size_t h = (size_t(T) * bh * bw + 3) & ~size_t(3);
  return sizeof(float) * (h + size_t(bh) * pitch + 2 * size_t(T) * bh * K * nbc + nbc);
}

// Time axis of the volume pass for T slices (TC = T at compile time, 0 = runtime): the
// forward transform along time per bin (the volume DC is bin 0 of slice 0 afterwards),
// then the spectral filter on all T x bins and the inverse along time, every slice
// written out.
template <int TC>
__device__ __forceinline__ void volume_time(const DevPlan& P, const VolumeSpectraJob& J, cf* spec, size_t slot,
                                            int nbc, int nb, int bins, int T_rt, size_t row_base, float* dc,
                                            bool& bad) {
  const int T = TC > 0 ? TC : T_rt;
  constexpr int CAP = TC > 0 ? TC : kMaxVolumeSlots;
  const int tid = threadIdx.x, nthr = blockDim.x;
  for (Cursor2 c(tid, nthr, nb); c.y < bins; c.next()) {
    const int kk = c.y, b = c.x;
    cf* bp = spec + size_t(kk) * nbc + b;
    cf line[CAP];
#pragma unroll
    for (int z = 0; z < CAP; ++z)
      if (z < T) line[z] = bp[size_t(z) * slot];
    nf::fft_project<true, TC, 16>(line, T, P.twt);
#pragma unroll
    for (int z = 0; z < CAP; ++z)
      if (z < T) bp[size_t(z) * slot] = line[z];
    // the block's template scale from its volume DC, once per block (the filter reads it per bin)
    if (kk == 0)
      dc[b] = (P.grid && P.mean_scale != 0.0f && P.grid[0].r != 0.0f) ? fdiv(fmul(P.mean_scale, line[0].r), P.grid[0].r)
                                                                      : 0.0f;
  }
  __syncthreads();
  const size_t cnt = size_t(P.gx.count);
  // The ftype is fixed at compile time per branch (one uniform branch per launch item
  // instead of a switch per element).
  auto filter_lines = [&](auto ft) {
    constexpr int FT = decltype(ft)::value;
    for (Cursor2 c(tid, nthr, nb); c.y < bins; c.next()) {
      const int kk = c.y, b = c.x;
      const cf* bp = spec + size_t(kk) * nbc + b;
      const float g = dc[b];  // the block's template scale
      cf line[CAP];
#pragma unroll
      for (int z = 0; z < CAP; ++z)
        if (z < T) line[z] = spectral_bin<FT>(bp[size_t(z) * slot], P.grid, z * bins + kk, g, P.filt, bad);
      nf::fft_project<false, TC, 16>(line, T, P.twt);
#pragma unroll
      for (int z = 0; z < CAP; ++z)
        if (z < T) J.out[z][row_base + size_t(kk) * cnt + b] = line[z];
    }
  };
  switch (P.filt.type) {
    case 0:  // the exponent mode fixed too
      if (P.filt.emode == 0) filter_lines(std::integral_constant<int, kFt0Ratio>{});
      else if (P.filt.emode == 1) filter_lines(std::integral_constant<int, kFt0Sqrt>{});
      else filter_lines(std::integral_constant<int, kFt0Pow>{});
      break;
    case 1: filter_lines(std::integral_constant<int, 1>{}); break;
    case 2: filter_lines(std::integral_constant<int, 2>{}); break;
    case 3: filter_lines(std::integral_constant<int, 3>{}); break;
    default: filter_lines(std::integral_constant<int, 4>{}); break;
  }
}

// Pass 1 of the DFTTest slice form: per block row chunk, the 3-D forward transform of
// each volume (spatial per slice, then time; the volume tile's phases A, B1 and T),
// the spectral filter and the inverse along time; all T slices written out.
template <int BHC, int BWC, int STORAGE>
__global__ void __launch_bounds__(256) volume_spectra_batch_kernel(VolumeSpectraWork W) {
  extern __shared__ float smem[];
  const int BH = BHC > 0 ? BHC : W.plans[0].bh;
  const int BW = BWC > 0 ? BWC : W.plans[0].bw;
  const int K = BW / 2 + 1;
  constexpr int CAPH = BHC > 0 ? BHC : nf::kMaxProject;
  constexpr int CAPW = BWC > 0 ? BWC : nf::kMaxProject;
  constexpr int UH = BHC > 0 ? CAPH : 1, UW = BWC > 0 ? CAPW : 1;
  constexpr bool kCodelet = BHC == BWC && (BWC == 8 || BWC == 16 || BWC == 32);

  const int item = blockIdx.x;
  int lo = 0, hi = W.njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (W.item_base[mid] <= item) lo = mid;
    else hi = mid - 1;
  }
  __shared__ DevPlan sP;
  __shared__ int s_chunks, s_plan;
  if (threadIdx.x == 0) {
    s_plan = W.jobs[lo].plan;
    s_chunks = W.jobs[lo].chunks_x;
    sP = W.plans[s_plan];
  }
  __syncthreads();
  const VolumeSpectraJob& J = W.jobs[lo];
  const DevPlan& P = sP;
  const bool codelet = kCodelet || (BHC == 0 && P.codelet != 0);
  const DevAxis gx = P.gx, gy = P.gy;
  const int T = P.T;
  const int local = item - W.item_base[lo];
  const int by = local / s_chunks, chunk = local - by * s_chunks;
  const int nbc = W.nbc;
  const int bx0 = chunk * nbc, nb = min(nbc, gx.count - bx0);
  const int oy = by * gy.step, cx0 = bx0 * gx.step;
  const int win = (nb - 1) * gx.step + BW;
  const int pitch = ((nbc - 1) * gx.step + BW + 3) & ~3;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int bins = BH * K;
  const size_t slot = size_t(bins) * nbc;  // complex per slice in spec

  float* h = smem;
  float* ring = smem + ((size_t(T) * BH * BW + 3) & ~size_t(3));
  cf* spec = reinterpret_cast<cf*>(ring + size_t(BH) * pitch);
  float* dc = reinterpret_cast<float*>(spec + size_t(T) * slot);
  for (int i = tid; i < T * BH * BW; i += nthr) h[i] = P.h[i];
  bool bad = false;
  for (int z = 0; z < T; ++z) {
    __syncthreads();
    for (Cursor2 c(tid, nthr, win); c.y < BH; c.next()) {
      const int y = c.y, xx = c.x;
      const unsigned char* srow = J.src[z] + ptrdiff_t(reflect_axis(oy + y, gy)) * J.src_stride[z];
      const float sv = load_sample<STORAGE>(srow, reflect_axis(cx0 + xx, gx));
      const float v = fmul(fsub(sv, P.dec_base), P.dec_scale);
      if (STORAGE == kStoreF32 && !isfin(v)) bad = true;  // decoded integers are finite
      ring[size_t(y) * pitch + xx] = v;
    }
    __syncthreads();
    for (Cursor2 c(tid, nthr, nb); c.y < BH; c.next()) {
      const int y = c.y, b = c.x;
      const float* in = ring + size_t(y) * pitch + b * gx.step;
      float row[CAPW];
#pragma unroll UW
      for (int x = 0; x < CAPW; ++x)
        if (x < BW) row[x] = fmul(in[x], h[(z * BH + y) * BW + x]);
      nf::row_forward<BWC>(row, BW, spec + size_t(z) * slot + size_t(y) * K * nbc + b, P.tww, codelet, nbc);
    }
  }
  __syncthreads();
  for (Cursor2 c(tid, nthr, nb); c.y < T * K; c.next()) {
    const int z = c.y / K, k = c.y - z * K, b = c.x;  // rows of (slot, bin); K is small
    cf col[CAPH];
    cf* sp = spec + size_t(z) * slot + size_t(k) * nbc + b;
#pragma unroll UH
    for (int y = 0; y < CAPH; ++y)
      if (y < BH) col[y] = sp[size_t(y) * K * nbc];
    nf::fft_1d<true, BHC>(col, BH, P.twh, codelet);
#pragma unroll UH
    for (int y = 0; y < CAPH; ++y)
      if (y < BH) sp[size_t(y) * K * nbc] = col[y];
  }
  __syncthreads();
  const size_t row_base = size_t(by) * bins * size_t(gx.count) + size_t(bx0);
  switch (T) {  // compile-time lengths keep the temporal line in registers
    case 2: volume_time<2>(P, J, spec, slot, nbc, nb, bins, T, row_base, dc, bad); break;
    case 3: volume_time<3>(P, J, spec, slot, nbc, nb, bins, T, row_base, dc, bad); break;
    case 4: volume_time<4>(P, J, spec, slot, nbc, nb, bins, T, row_base, dc, bad); break;
    case 5: volume_time<5>(P, J, spec, slot, nbc, nb, bins, T, row_base, dc, bad); break;
    case 6: volume_time<6>(P, J, spec, slot, nbc, nb, bins, T, row_base, dc, bad); break;
    case 7: volume_time<7>(P, J, spec, slot, nbc, nb, bins, T, row_base, dc, bad); break;
    default: volume_time<0>(P, J, spec, slot, nbc, nb, bins, T, row_base, dc, bad); break;
  }
  if (bad) atomicOr(P.err, kErrNonFinite);
}

// Pass 2: persistent strips over the step's jobs. FFT3D (SRC = kSrcTemporal): every job
// carries the slot spectra of its frame (clip-edge frames, which filter their single
// source frame, run as pixel strips in the batched spatial kernel). DFTTest (SRC =
// kSrcSlice): every job reconstructs one slice spectrum.
// Threads of a pass-2 CTA: 512 for FFT3D temporal strips of 48x48 blocks (their team
// transforms fit in 128 registers, so one CTA per SM runs 16 warps), 256 otherwise.
template <int BHC, int BWC, int SRC>
struct TemporalThreads {
  static constexpr int value = (SRC == kSrcTemporal && team_block<BHC, BWC>()) ? 512 : 256;
};

template <int BHC, int BWC, int STORAGE, int SRC>
__global__ void __launch_bounds__(TemporalThreads<BHC, BWC, SRC>::value, StripOccupancy<BHC, BWC>::value)
    temporal_batch_kernel(BatchWork W) {
  extern __shared__ float smem[];
  __shared__ int item;
  const int total = W.job_tile_base[W.njobs];
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) item = atomicAdd(W.counter, 1);
    __syncthreads();
    const int t = item;
    if (t >= total) break;
    int lo = 0, hi = W.njobs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (W.job_tile_base[mid] <= t) lo = mid;
      else hi = mid - 1;
    }
    __shared__ DevPlan sP;
    __shared__ PlaneJob sJ;
    __shared__ StripShape sS;
    if (threadIdx.x == 0) {
      sJ = W.jobs[lo];
      sP = W.plans[sJ.plan];
      sS = W.shapes[sJ.plan];
    }
    __syncthreads();
    const int local = t - W.job_tile_base[lo];
    const int sx = local % W.job_tiles_x[lo], sy = local / W.job_tiles_x[lo];
    if constexpr (SRC == kSrcSlice) {
      strip_tile<BHC, BWC, STORAGE, kSrcSlice, 1>(sP, sJ, sS, sx * sS.tw, sy * sS.th, smem);
    } else {
      strip_tile<BHC, BWC, STORAGE, kSrcTemporal, 0>(sP, sJ, sS, sx * sS.tw, sy * sS.th, smem);
    }
  }
}

} // namespace nfd
