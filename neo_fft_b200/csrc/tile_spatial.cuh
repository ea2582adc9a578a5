// Single-frame strip kernel: FFT3D bt=1/-1 (and Kalman render) and DFTTest tbsize=1.
//
// A CTA owns a column strip of the visible plane (TW columns, TH rows) and walks
// down it one block row at a time (the reference's `by` loop,
// src/algorithms/plan.cpp:432-537 and 553-605). Per block row:
//
//   0  stage    the source rows the block row adds are reflected, decoded and
//               checked once per sample into a shared ring of BH rows
//   A  rows     thread = (block, row): analysis window, real forward transform of
//               the row into K = bw/2+1 bins (shared memory)
//   B  columns  thread = (block, column): forward transform along y in registers,
//               the block's DC is exchanged through shared memory, per-bin filter,
//               inverse transform along y
//   C  rows     thread = (block, row): inverse real transform, non-finite check,
//               synthesis weighting (written in place over the row's bins)
//   D  overlap  thread = output pixel: contributions are added in the reference's
//               order (block row ascending, then block column ascending; FFT3D sums
//               the row strip first and applies the vertical synthesis weight once
//               per block row), into a ring accumulator of BH rows
//   E  retire   rows no later block row can touch are quantised and stored
//
// Outputs are owner-written and deterministic without atomics. Blocks overlapping
// two strips are computed by both (the horizontal halo); vertically the strip is
// tall, so little work is repeated.
#pragma once
#include <type_traits>
#include "device_plan.cuh"
#include "tma.cuh"

namespace nfd {

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
// ALGO: 0 FFT3D, 1 DFTTest known at compile time, -1 read from the plan.
// `P`: the plan, or an OutConv copy of its conversion fields taken before a loop.
template <int STORAGE, int ALGO = -1, class Conv = DevPlan>
__device__ __forceinline__ void store_sample(unsigned char* row, int x, float acc, const Conv& P) {
  const bool fft3d = ALGO >= 0 ? ALGO == 0 : P.algo == 0;
  if (STORAGE == kStoreU8 && P.raw_out) {  // dithered u8 output: the dither pass converts
    reinterpret_cast<float*>(row)[x] = acc;
    return;
  }
  if (STORAGE == kStoreF32) {
    float v;
    if (fft3d) v = acc < 0.0f ? 0.0f : (1.0f < acc ? 1.0f : acc);
    else v = fmul(acc, P.out_scale);
    reinterpret_cast<float*>(row)[x] = v;
    return;
  }
  const float v = fft3d ? fadd(fadd(acc, 0.5f), P.out_base) : fadd(fmul(acc, P.out_scale), 0.5f);
  const float c = v < 0.0f ? 0.0f : (P.out_peak < v ? P.out_peak : v);
  if (STORAGE == kStoreU8) row[x] = (unsigned char)(c);
  else reinterpret_cast<unsigned short*>(row)[x] = (unsigned short)(c);
}

// The output conversion fields of a plan, read once before a loop of stores.
struct OutConv {
  int algo, raw_out;
  float out_base, out_scale, out_peak;
};
__device__ __forceinline__ OutConv out_conv(const DevPlan& P) {
  return {P.algo, P.raw_out, P.out_base, P.out_scale, P.out_peak};
}

// One plane to filter: source/destination (device memory, signed byte strides) and
// for Kalman render the state's estimate L ([block][bins]) instead of a source.
struct PlaneJob {
  const unsigned char* src;
  long long src_stride;
  unsigned char* dst;
  long long dst_stride;
  const cf* kalman_L;
  int plan;  // index into the batch's plan table
  int zt;    // DFTTest slice form: the output's slice of its temporal block
  // Spectra computed beforehand, layout [block row][bin][block column]: FFT3D temporal
  // form, the T slots' spatial spectra (the strip filters across them); DFTTest slice
  // form, tspec[0] = the filtered spatial spectrum of slice zt (the strip reconstructs it).
  const cf* const* tspec;
  // Batched pixel strips: 2-D tensor map of the source plane (boxes of tma_box_w x
  // step samples) for the prefetched staging of interior block rows, or nullptr.
  const void* tmap;
};

// Source of a strip's block spectra.
constexpr int kSrcPixels = 0;    // source pixels
constexpr int kSrcTemporal = 1;  // FFT3D bt=2..5 slot spectra, filtered across time here
constexpr int kSrcSlice = 2;     // DFTTest tmode 1 filtered slice spectra
constexpr int kSrcKalman = 3;    // FFT3D Kalman render: the state's estimate L (PlaneJob::kalman_L)

struct StripShape {
  int tw, th;     // strip width and segment height (plane pixels)
  int nbx_max;    // block columns that can touch a strip (spectrum/overlap stride)
  int win_max;    // staged input columns: (nbx_max-1)*step + bw
  int ring_pitch; // floats per staged row: a multiple of 4 with an odd float4 count
  int tab_floats; // per-plan tables staged in shared memory
  int tma_box_w;  // bulk-tensor staging: staged width in samples, whole boxes (0: none)
  int raw_bytes;  // bytes of each of the two raw buffers (a multiple of 128)
};

// Floats of the per-plan tables a strip stages in shared memory (strip_tile).
__host__ __device__ inline int strip_table_floats(const DevPlan& P) {
  const int K = P.bw / 2 + 1, bins = P.bh * K;
  int n = P.algo == 0 ? 2 * (P.bw + P.bh) : 2 * P.bh * P.bw;
  if (P.grid) n += 2 * bins;
  if (P.filt.primary) n += bins;
  if (P.enh.sharpen_w) n += bins;
  if (P.enh.halo_w) n += bins;
  return (n + 3) & ~3;
}

// Shared layout (floats): tables | ring_in [bh][ring_pitch] | spec [bh][K][nbx]
// complex (block fastest) | ob [bh][nbx][bw+4] (synthesised rows, x fastest) |
// acc [bh][tw] | dc [2*nbx] | colmap [tw] (overlap-add blocks of each strip column) |
// raw [2][raw_bytes] source boxes of the bulk-tensor staging (128-byte aligned).
__host__ __device__ inline size_t strip_smem_bytes(int bh, int bw, const StripShape& s) {
  const size_t K = size_t(bw / 2 + 1);
  const size_t spec_cf = (size_t(s.nbx_max) * bh * K + 1) & ~size_t(1);  // keeps ob 16-byte aligned
  return sizeof(float) * (size_t(s.tab_floats) + size_t(bh) * s.ring_pitch + spec_cf * 2 +
                          size_t(bh) * s.nbx_max * (bw + 4) + size_t(bh) * s.tw + 2 * size_t(s.nbx_max) +
                          size_t(s.tw)) +
         (s.raw_bytes > 0 ? 2 * size_t(s.raw_bytes) + 128 : 0);
}

// Walks the linear indices start, start + step, ... of a rows x width range as (y, x)
// pairs with one division at the start: each step adds the step's quotient and
// remainder and carries once. `i < rows * width` is `y < rows`; width must be positive.
struct Cursor2 {
  int y, x, dq, dr, w;
  __device__ __forceinline__ Cursor2(int start, int step, int width) : w(width) {
    y = start / width;
    x = start - y * width;
    dq = step / width;
    dr = step - dq * width;
  }
  __device__ __forceinline__ void next() {
    y += dq;
    x += dr;
    if (x >= w) {
      x -= w;
      ++y;
    }
  }
};

// Warm L2 with one block row of slot spectra (nslots x bins runs of nbx values at
// `at` + bin * cnt in each slot) while the current row is filtered and reconstructed:
// one prefetch per 128-byte line, each at an element address inside its run.
// `walk` is the thread's walk over rows of prefetch_lines(nbx) lines.
__host__ __device__ inline int prefetch_lines(int nbx) { return (nbx * int(sizeof(cf)) + 127) / 128 + 1; }
__device__ __forceinline__ void prefetch_row_l2(const cf* const* slots, int nslots, size_t at, int bins, size_t cnt,
                                                int nbx, const Cursor2& walk) {
  for (Cursor2 q = walk; q.y < nslots * bins; q.next()) {
    const int z = q.y / bins, kk = q.y - z * bins;
    const uintptr_t lo = reinterpret_cast<uintptr_t>(slots[z] + at + size_t(kk) * cnt);
    const uintptr_t hi = lo + size_t(nbx) * sizeof(cf);
    const uintptr_t a = max(lo, (lo & ~uintptr_t(127)) + uintptr_t(q.x) * 128);
    if (a < hi) asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
  }
}

// FFT3D bt=2..5 filter of one block row's (bin, block) elements across the T slot
// spectra (spectral.cpp:90-160) with T = TC known at compile time; writes the recovered
// spectrum into spec [bin][block].
template <int TC>
__device__ __forceinline__ void temporal_filter_elements(const DevPlan& P, const PlaneJob& J, const DevSpectral& filt,
                                                         const cf* grid, float grid0, cf* spec, const float* dc, int NB,
                                                         int nbx, int nel, size_t row_base, size_t cnt, int T,
                                                         float invT, bool& bad, const Cursor2& walk) {
  // loop invariants in registers: slot pointers, temporal twiddles, scalars
  const cf* slot[TC];
  cf tf[TC * TC], ti[TC];
#pragma unroll
  for (int j = 0; j < TC; ++j) {
    slot[j] = J.tspec[j];
    ti[j] = P.tinv[j];
  }
#pragma unroll
  for (int i = 0; i < TC * TC; ++i) tf[i] = P.tfwd[i];
  const float lower = P.lower, noise_mult = P.noise_mult, noise_uniform = P.noise_uniform;
  const float* primary = filt.primary;
  const float fT = float(TC);
  (void)T;
  const int nrow_e = nel / nbx;  // bins
#pragma unroll 2
  for (Cursor2 c = walk; c.y < nrow_e; c.next()) {
    const int kk = c.y, b = c.x;
    const size_t at = row_base + size_t(kk) * cnt + b;
    cf v[TC];
#pragma unroll
    for (int j = 0; j < TC; ++j) v[j] = slot[j][at];
    cf gT = {0.0f, 0.0f};
    if (grid) {
      const float g = dc[b];  // the block's template scale
      const cf M = {fmul(g, grid[kk].r), fmul(g, grid[kk].i)};
      gT = {fmul(M.r, fT), fmul(M.i, fT)};
    }
    const float noise = primary ? fmul(primary[kk], noise_mult) : noise_uniform;
    if (!isfin(noise)) bad = true;
    cf yv = {0.0f, 0.0f};
#pragma unroll
    for (int m = 0; m < TC; ++m) {
      cf F = {0.0f, 0.0f};
#pragma unroll
      for (int j = 0; j < TC; ++j) F = nf::cadd(F, nf::cmul_plain(v[j], tf[m * TC + j]));
      const cf R = m == 0 ? nf::csub(F, gT) : F;
      const float power = fadd(fmul(R.r, R.r), fmul(R.i, R.i));
      if (!isfin(power)) bad = true;
      const float q = fadd(power, 1e-15f);
      const float gr = fdiv(fsub(q, noise), q);
      const float gain = gr < lower ? lower : gr;
      cf Rf = {fmul(gain, R.r), fmul(gain, R.i)};
      if (m == 0) Rf = nf::cadd(Rf, gT);
      yv = nf::cadd(yv, nf::cmul_plain(Rf, ti[m]));
    }
    spec[kk * NB + b] = {fmul(yv.r, invT), fmul(yv.i, invT)};
  }
}

// Block shapes whose temporal strips use team transforms (nf::TeamFFT over four lanes):
// square 48x48, the largest non-codelet shape instantiated.
template <int BHC, int BWC>
__host__ __device__ constexpr bool team_block() {
  return BHC == 48 && BWC == 48;
}
// Floats of team scratch a temporal strip of `threads` threads needs in its staging ring:
// per team of four lanes, bw + 4 complex values (four runs of bw/4 + 1).
__host__ __device__ inline int team_scratch_floats(int bw, int threads) { return (threads / 4) * 2 * (bw + 4); }

// ALGO: 0 FFT3D, 1 DFTTest (the launch knows the plan's algorithm, so the other
// algorithm's branches are compiled out), -1 read from the plan.
template <int BHC, int BWC, int STORAGE, int SRC = kSrcPixels, int ALGO = -1>
__device__ __forceinline__ void strip_tile(const DevPlan& P, const PlaneJob& J, const StripShape& S, int px0, int py0,
                                           float* smem, TmaPipe* pipe = nullptr) {
  const bool fft3d = ALGO >= 0 ? ALGO == 0 : P.algo == 0;
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
  const cf* kalman_L = J.kalman_L;
  (void)kalman_L;
  const int NB = S.nbx_max;   // block stride of spec and ob
  const int OBW = BW + 4;     // ob row pitch (conflict-free float4 stores and overlap reads)
  // FFT3D temporal tiles of 48x48 blocks share each 48-point transform among a team of
  // four lanes (nf::TeamFFT): a lane holds 12 values instead of 48.
  constexpr bool kTeam = SRC == kSrcTemporal && team_block<BHC, BWC>();
  const int lane = threadIdx.x & 3, team = threadIdx.x >> 2, nteams = blockDim.x >> 2;
  const unsigned team_mask = 0xFu << (threadIdx.x & 28);
  (void)lane; (void)team; (void)nteams; (void)team_mask;

  const int tw = min(S.tw, gx.length - px0), th = min(S.th, gy.length - py0);
  const int X0 = px0 + gx.offset, Y0 = py0 + gy.offset;
  const int bx_lo = max(0, floor_div_i(X0 - BW, gx.step) + 1);
  const int bx_hi = min(gx.count - 1, floor_div_i(X0 + tw - 1, gx.step));
  const int by_lo = max(0, floor_div_i(Y0 - BH, gy.step) + 1);
  const int by_hi = min(gy.count - 1, floor_div_i(Y0 + th - 1, gy.step));
  const int nbx = bx_hi - bx_lo + 1;
  const int cx0 = bx_lo * gx.step;           // first staged cover column
  const int win = (nbx - 1) * gx.step + BW;  // staged columns

  float* tab = smem;
  float* ring_in = tab + S.tab_floats;
  // Shared-memory offsets are 32-bit: the whole layout is below 227 KB.
  const int KNB = K * NB;  // complex stride between spectrum rows
  cf* spec = reinterpret_cast<cf*>(ring_in + BH * S.ring_pitch);
  float* ob = reinterpret_cast<float*>(spec + ((BH * KNB + 1) & ~1));
  float* acc = ob + BH * NB * OBW;
  float* dc = acc + BH * S.tw;
  int* colmap = reinterpret_cast<int*>(dc + 2 * NB);
  const int tid = threadIdx.x, nthr = blockDim.x;
  bool bad = false;
  // Raw boxes of the bulk-tensor staging, 128-byte aligned after colmap.
  unsigned char* raw = reinterpret_cast<unsigned char*>(colmap + S.tw);
  raw += (128 - (smem_u32(raw) & 127)) & 127;

  __syncthreads();  // shared memory may still be read by a previous work item
  // ---- per-plan tables into shared memory --------------------------------------
  const int bins = BH * K;
  float* t_wa = tab;  // FFT3D: wxa[BW] wya[BH] wxs[BW] wys[BH]; DFTTest: h[BH*BW] hsyn[BH*BW]
  int off = 0;
  auto stage = [&](const float* src, int n) {
    float* d = tab + off;
    for (int i = tid; i < n; i += nthr) d[i] = src[i];
    off += n;
    return d;
  };
  const float *wxa = nullptr, *wya = nullptr, *wxs = nullptr, *wys = nullptr, *h = nullptr, *hsyn = nullptr;
  if (fft3d) {
    wxa = stage(P.wxa, BW);
    wya = stage(P.wya, BH);
    wxs = stage(P.wxs, BW);
    wys = stage(P.wys, BH);
  } else {
    h = stage(P.h + (SRC == kSrcSlice ? size_t(J.zt) * BH * BW : 0), BH * BW);
    hsyn = stage(P.hsyn, BH * BW);
  }
  (void)t_wa;
  const cf* grid = P.grid ? reinterpret_cast<const cf*>(stage(reinterpret_cast<const float*>(P.grid), 2 * bins)) : nullptr;
  // Filter parameters with their tables redirected to shared memory. They live in
  // shared memory too (a per-thread copy would sit on the local-memory stack).
  __shared__ DevSpectral s_filt, s_enh;
  const float* prim = P.filt.primary ? stage(P.filt.primary, bins) : nullptr;
  const float* shw = P.enh.sharpen_w ? stage(P.enh.sharpen_w, bins) : nullptr;
  const float* hlw = P.enh.halo_w ? stage(P.enh.halo_w, bins) : nullptr;
  if (tid == 0) {
    s_filt = P.filt;
    s_enh = P.enh;
    if (prim) s_filt.primary = prim;
    if (shw) s_filt.sharpen_w = s_enh.sharpen_w = shw;
    if (hlw) s_filt.halo_w = s_enh.halo_w = hlw;
  }
  const DevSpectral& filt = s_filt;
  const DevSpectral& enh = s_enh;
  for (int i = tid; i < BH * S.tw; i += nthr) acc[i] = 0.0f;
  // Per strip column: the first overlapping block (relative to bx_lo), the number of
  // overlapping blocks and the column's offset inside the first one; the same for every
  // block row, so the overlap-add below needs no divisions.
  for (int xx = tid; xx < tw; xx += nthr) {
    const int X = X0 + xx;
    const int b0 = max(bx_lo, floor_div_i(X - BW, gx.step) + 1), b1 = min(bx_hi, floor_div_i(X, gx.step));
    const int nblk = max(0, b1 - b0 + 1);
    colmap[xx] = (b0 - bx_lo) | (nblk << 10) | ((nblk > 0 ? X - b0 * gx.step : 0) << 20);
  }
  __syncthreads();
  const float grid0 = grid ? grid[0].r : 1.0f;
  const float fct = fdiv(1.0f, fmul(float(BW), float(BH)));
  // DFTTest slice form: 3-D normalisation and the temporal-OLA synthesis weight
  // volume * h[zt] (plan.cpp:594-601).
  const float fct3 = fdiv(1.0f, fmul(fmul(float(P.T), float(BH)), float(BW)));
  const float volume = fmul(fmul(float(P.T), float(BW)), float(BH));
  const bool vec4 = (gx.step & 3) == 0 && (BW & 3) == 0;
  const bool ola4 = !P.center && vec4 && (S.tw & 3) == 0 && (tw & 3) == 0 && (X0 & 3) == 0;

  // One source sample in cover coordinates (cy, cx): rows and columns inside the visible
  // plane are read directly, the margins through the single reflection.
  auto source_sample = [&](int cy, int cx) -> float {
    const int sy = cy - gy.offset, sx = cx - gx.offset;
    const bool in = unsigned(sy) < unsigned(gy.length) && unsigned(sx) < unsigned(gx.length);
    const int ry = in ? sy : reflect_axis(cy, gy), rx = in ? sx : reflect_axis(cx, gx);
    return load_sample<STORAGE>(J.src + ptrdiff_t(ry) * J.src_stride, rx);
  };
  // Bulk-tensor staging (batched pixel strips with a tensor map): the strip's staged
  // columns lie inside the plane, and a block row after the tile's first whose `step` new
  // rows lie inside it too is copied by the elected thread one block row ahead. The box
  // starts at the staged columns rounded down to 16 bytes (xa); tma_shift is the
  // remainder in samples.
  constexpr int kElem = STORAGE == kStoreU8 ? 1 : (STORAGE == kStoreU16 ? 2 : 4);
  constexpr int kBox = kStagingBoxBytes / kElem;  // samples per box row
  const int sx0 = cx0 - gx.offset;
  const bool tma_cols = SRC == kSrcPixels && pipe != nullptr && J.tmap != nullptr && S.tma_box_w > 0 && sx0 >= 0 &&
                        sx0 + win <= gx.length;
  const int tma_xa = sx0 & ~(16 / kElem - 1), tma_shift = sx0 - tma_xa;
  const unsigned tma_bytes = unsigned(S.tma_box_w) * unsigned(gy.step) * kElem;
  auto tma_rows = [&](int b) {  // first plane row of block row b's new rows, or -1
    const int y = b * gy.step + BH - gy.step - gy.offset;
    return y >= 0 && y + gy.step <= gy.length ? y : -1;
  };
  // The dead flag is written only inside a staging phase and read only right after a
  // barrier that no staging phase separates from the next, so every thread of the CTA
  // takes the same staging path in a block row.
  bool tma_on = tma_cols && *pipe->dead == 0;
  // The phases' thread-to-(row, column) walks, divided once per tile: the widths do not
  // change between block rows, and a division left in the loop is not hoisted by the
  // compiler (it cannot prove the divisor nonzero).
  const Cursor2 walk_nbx(tid, nthr, nbx), walk_tw(tid, nthr, tw), walk_tw4(tid, nthr, max(tw >> 2, 1));
  const Cursor2 walk_win(tid, nthr, win), walk_q4(tid, nthr, (win + 3) >> 2);
  const Cursor2 walk_lines(tid, nthr, prefetch_lines(nbx)), walk_team(team, nteams, nbx);
  // No barrier between a block row's retire phase (accumulator ring and the output) and the
  // next block row's first phase (staging ring, or the column phase's spectrum and DC
  // buffers): they touch disjoint shared memory, and every later phase is behind a barrier.
  for (int by = by_lo; by <= by_hi; ++by) {
    const int oy = by * gy.step;
    if constexpr (SRC == kSrcPixels) {
      // ---- 0: stage the rows this block row adds ----------------------------
      // Prefetch block row by + 1 into buffer (by + 1) & 1, last read while staging
      // block row by - 1 (behind that phase's barrier).
      if (tma_on && tid == 0 && by < by_hi) {
        const int y1 = tma_rows(by + 1);
        if (y1 >= 0) {
          const int nb1 = (by + 1) & 1;
          mbar_expect_tx(pipe->mbar + nb1, tma_bytes);
          for (int k = 0; k * kBox < S.tma_box_w; ++k)
            tma_load_2d(raw + nb1 * S.raw_bytes + k * kStagingBoxBytes * gy.step, J.tmap, tma_xa + k * kBox, y1,
                        pipe->mbar + nb1);
          pipe->pending |= 1u << nb1;
        }
      }
      const int r0 = by == by_lo ? oy : max(oy, oy + BH - gy.step);
      const int nrows = oy + BH - r0;
      const float dec_base = P.dec_base, dec_scale = P.dec_scale;  // read once, not per sample
      bool staged = false;
      if (tma_on && by > by_lo && tma_rows(by) >= 0) {
        const int b0 = by & 1;
        const bool ok = mbar_wait_bounded(pipe->mbar + b0, (pipe->phase >> b0) & 1u, kStagingWaitCycles);
        if (ok) {
          pipe->phase ^= 1u << b0;
          if (tid == 0) pipe->pending &= ~(1u << b0);
        } else {  // the copy did not arrive: report it, stop prefetching, read directly
          *pipe->dead = 1;
          atomicOr(P.err, kErrStaging);
        }
        // Four samples per thread. Plane row tma_rows(by) + r, column tma_xa + i is sample
        // (i / kBox) * kBox * step + r * kBox + i % kBox of the raw boxes. A thread whose
        // wait ran out reads its samples directly.
        const unsigned char* rb = raw + b0 * S.raw_bytes;
        for (Cursor2 c = walk_q4; c.y < nrows; c.next()) {
          const int x = c.x * 4;
          float v[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) v[j] = 0.0f;
          const int i0 = x + tma_shift;
          if (ok && (tma_shift & 3) == 0) {
            // the quad lies inside one box row: one 4-, 8- or 16-byte shared load
            const int at = (i0 / kBox) * kBox * gy.step + c.y * kBox + i0 % kBox;
            if constexpr (STORAGE == kStoreU8) {
              const unsigned w = *reinterpret_cast<const unsigned*>(rb + at);
#pragma unroll
              for (int j = 0; j < 4; ++j) v[j] = float((w >> (8 * j)) & 0xffu);
            } else if constexpr (STORAGE == kStoreU16) {
              const uint2 w = *reinterpret_cast<const uint2*>(rb + 2 * at);
              v[0] = float(w.x & 0xffffu);
              v[1] = float(w.x >> 16);
              v[2] = float(w.y & 0xffffu);
              v[3] = float(w.y >> 16);
            } else {
              const float4 w = *reinterpret_cast<const float4*>(rb + 4 * at);
              v[0] = w.x;
              v[1] = w.y;
              v[2] = w.z;
              v[3] = w.w;
            }
          } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int i = i0 + j;
              if (ok) v[j] = load_sample<STORAGE>(rb, (i / kBox) * kBox * gy.step + c.y * kBox + i % kBox);
              else if (x + j < win) v[j] = source_sample(r0 + c.y, cx0 + x + j);
            }
          }
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            v[j] = fmul(fsub(v[j], dec_base), dec_scale);
            if (STORAGE == kStoreF32 && x + j < win && !isfin(v[j])) bad = true;
          }
          *reinterpret_cast<float4*>(ring_in + int(unsigned(r0 + c.y) % unsigned(BH)) * S.ring_pitch + x) =
              make_float4(v[0], v[1], v[2], v[3]);
        }
        staged = true;
      }
      if (!staged) {
        for (Cursor2 c = walk_win; c.y < nrows; c.next()) {
          const int cy = r0 + c.y;
          const float sv = source_sample(cy, cx0 + c.x);
          const float v = fmul(fsub(sv, dec_base), dec_scale);
          if (STORAGE == kStoreF32 && !isfin(v)) bad = true;  // decoded integers are finite
          ring_in[int(unsigned(cy) % unsigned(BH)) * S.ring_pitch + c.x] = v;
        }
      }
      __syncthreads();
      tma_on = tma_on && *pipe->dead == 0;
      // ---- A: row transforms (block index fastest) --------------------------
      for (Cursor2 c = walk_nbx; c.y < BH; c.next()) {
        const int y = c.y, b = c.x;
        const float* in = ring_in + int(unsigned(oy + y) % unsigned(BH)) * S.ring_pitch + b * gx.step;
        float row[CAPW];
        if (vec4) {
#pragma unroll UW
          for (int x = 0; x < CAPW; x += 4) {
            if (x < BW) {
              const float4 q = *reinterpret_cast<const float4*>(in + x);
              row[x] = q.x;
              row[x + 1] = q.y;
              row[x + 2] = q.z;
              row[x + 3] = q.w;
            }
          }
        } else {
#pragma unroll UW
          for (int x = 0; x < CAPW; ++x)
            if (x < BW) row[x] = in[x];
        }
#pragma unroll UW
        for (int x = 0; x < CAPW; ++x)
          if (x < BW) row[x] = fft3d ? fmul(fmul(row[x], wya[y]), wxa[x]) : fmul(row[x], h[y * BW + x]);
        nf::row_forward<BWC>(row, BW, spec + y * KNB + b, P.tww, codelet, NB);
      }
      __syncthreads();
    }
    // ---- B: column forward, filter, column inverse --------------------------
    const int ncol = nbx * K;
    if constexpr (SRC == kSrcSlice) {
      // DFTTest tmode 1 (plan.cpp:544-601): the slice's spectrum was filtered in 3-D by
      // the volume pass; only the column inverses remain.
      const cf* S = J.tspec[0] + size_t(by) * bins * size_t(gx.count) + size_t(bx_lo);
      if (by < by_hi)
        prefetch_row_l2(J.tspec, 1, size_t(by + 1) * bins * size_t(gx.count) + size_t(bx_lo), bins,
                        size_t(gx.count), nbx, walk_lines);
      for (Cursor2 c = walk_nbx; c.y < K; c.next()) {
        const int k = c.y, b = c.x;
        cf col[CAPH];
#pragma unroll UH
        for (int y = 0; y < CAPH; ++y)
          if (y < BH) col[y] = S[size_t(y * K + k) * gx.count + b];
        nf::fft_1d<false, BHC>(col, BH, P.twh, codelet);
        cf* sp = spec + k * NB + b;
#pragma unroll UH
        for (int y = 0; y < CAPH; ++y)
          if (y < BH) sp[y * KNB] = col[y];
      }
      __syncthreads();
    } else if constexpr (SRC == kSrcTemporal) {
      // FFT3D bt=2..5 (spectral.cpp:90-160): per bin, T-point DFT across the slots'
      // spatial spectra, Wiener per temporal frequency, inverse DFT at the centre
      // slot; then enhancement with the recovered spectrum's template ratio. The
      // filter runs element-parallel over (bin, block) so the slots' loads overlap;
      // the column inverses follow as in pixel mode.
      const int T = P.T, c = T / 2;
      const size_t cnt = size_t(gx.count);
      const size_t row_base = size_t(by) * bins * cnt + size_t(bx_lo);
      const float invT = fdiv(1.0f, float(T));
      if (by < by_hi) prefetch_row_l2(J.tspec, T, row_base + size_t(bins) * cnt, bins, cnt, nbx, walk_lines);
      // each block's template scale, mean_scale * DC(centre slot) / grid DC, once per block
      // (the filter below reads it for every bin of the block)
      for (int b = tid; b < nbx; b += nthr) {
        float g = 0.0f;
        if (grid) {
          g = fdiv(fmul(P.mean_scale, J.tspec[c][row_base + b].r), grid0);
          if (!isfin(g)) bad = true;
        }
        dc[b] = g;
      }
      __syncthreads();
      const int nel = bins * nbx;
      switch (T) {  // compile-time slot counts keep the slot values in registers
        case 2: temporal_filter_elements<2>(P, J, filt, grid, grid0, spec, dc, NB, nbx, nel, row_base, cnt, T, invT, bad, walk_nbx); break;
        case 3: temporal_filter_elements<3>(P, J, filt, grid, grid0, spec, dc, NB, nbx, nel, row_base, cnt, T, invT, bad, walk_nbx); break;
        case 4: temporal_filter_elements<4>(P, J, filt, grid, grid0, spec, dc, NB, nbx, nel, row_base, cnt, T, invT, bad, walk_nbx); break;
        default: temporal_filter_elements<5>(P, J, filt, grid, grid0, spec, dc, NB, nbx, nel, row_base, cnt, T, invT, bad, walk_nbx); break;
      }
      __syncthreads();
      if (enh.enh) {
        // template scale of each block's recovered spectrum, once per block
        for (int b = tid; b < nbx; b += nthr) dc[NB + b] = grid ? fdiv(fmul(P.mean_scale, spec[b].r), grid0) : 0.0f;
        __syncthreads();
        for (Cursor2 c = walk_nbx; c.y < bins; c.next()) {
          const int kk = c.y, b = c.x;
          const float g2 = dc[NB + b];
          cf* sp = spec + kk * NB + b;
          *sp = spectral_bin<-2>(*sp, grid, kk, g2, enh, bad);  // enh is always type -2
        }
        __syncthreads();
      }
      if constexpr (kTeam) {
        // Column inverses shared by teams of lanes, in place on the spectrum column: each
        // lane gathers and transforms its run, the runs go back into the column, and each
        // lane finishes the outermost butterflies of its own positions.
        using TH = nf::TeamFFT<false, BHC>;
        for (Cursor2 c = walk_team; c.y < K; c.next()) {
          cf* sp = spec + c.y * NB + c.x;
          cf run[TH::M];
          TH::run(lane, run, P.twh, [&](int y) { return sp[y * KNB]; });
          __syncwarp(team_mask);  // every lane has gathered before any run is written back
#pragma unroll
          for (int i = 0; i < TH::M; ++i) sp[(lane * TH::M + i) * KNB] = run[i];
          __syncwarp(team_mask);
          TH::outer(lane, P.twh, [&](int j, int i) { return sp[(j * TH::M + i) * KNB]; },
                    [&](int y, cf v) { sp[y * KNB] = v; });
        }
      } else {
        for (Cursor2 c = walk_nbx; c.y < K; c.next()) {
          const int k = c.y, b = c.x;
          cf col[CAPH];
          cf* sp = spec + k * NB + b;
#pragma unroll UH
          for (int y = 0; y < CAPH; ++y)
            if (y < BH) col[y] = sp[y * KNB];
          nf::fft_1d<false, BHC>(col, BH, P.twh, codelet);
#pragma unroll UH
          for (int y = 0; y < CAPH; ++y)
            if (y < BH) sp[y * KNB] = col[y];
        }
      }
      __syncthreads();
    } else {
    Cursor2 cb = walk_nbx;
    for (int base = 0; base < ncol; base += nthr, cb.next()) {
      const bool active = cb.y < K;  // task < ncol
      const int k = active ? cb.y : 0, b = active ? cb.x : 0;
      cf col[CAPH];
      cf* sp = spec + k * NB + b;  // + y*KNB
      if (active) {
        if constexpr (SRC == kSrcKalman) {
          const cf* L = kalman_L + (size_t(by) * gx.count + (bx_lo + b)) * P.bins + k;
#pragma unroll UH
          for (int y = 0; y < CAPH; ++y)
            if (y < BH) col[y] = L[size_t(y) * K];
        } else {
#pragma unroll UH
          for (int y = 0; y < CAPH; ++y)
            if (y < BH) col[y] = sp[y * KNB];
          nf::fft_1d<true, BHC>(col, BH, P.twh, codelet);
        }
        if (k == 0) dc[b] = col[0].r;
      }
      __syncthreads();
      if (active) {
        const float g = grid ? fdiv(fmul(P.mean_scale, dc[b]), grid0) : 0.0f;
        // The filter type is fixed at compile time per branch: one uniform branch per
        // column instead of a switch per bin.
        auto filter_column = [&](auto ft) {
          constexpr int FT = decltype(ft)::value;
          if constexpr (FT == kFt0Ratio) {
            float guard = 0.0f;
#pragma unroll UH
            for (int y = 0; y < CAPH; ++y)
              if (y < BH) col[y] = ratio_bin(col[y], grid, y * K + k, g, filt, guard);
            if (guard != guard) bad = true;
          } else {
#pragma unroll UH
            for (int y = 0; y < CAPH; ++y)
              if (y < BH) col[y] = spectral_bin<FT>(col[y], grid, y * K + k, g, filt, bad);
          }
        };
        if (ALGO == 1) {
          switch (filt.type) {
            case 0:  // the exponent mode fixed too
              if (filt.emode == 0) filter_column(std::integral_constant<int, kFt0Ratio>{});
              else if (filt.emode == 1) filter_column(std::integral_constant<int, kFt0Sqrt>{});
              else filter_column(std::integral_constant<int, kFt0Pow>{});
              break;
            case 1: filter_column(std::integral_constant<int, 1>{}); break;
            case 2: filter_column(std::integral_constant<int, 2>{}); break;
            case 3: filter_column(std::integral_constant<int, 3>{}); break;
            default: filter_column(std::integral_constant<int, 4>{}); break;
          }
        } else if (!fft3d || P.fft3d_mode != kEnhanceOnly) {
          if (filt.type == -1) filter_column(std::integral_constant<int, -1>{});
          else filter_column(std::integral_constant<int, -3>{});
        }
        if (fft3d && P.fft3d_mode == kWienerThenEnh && k == 0) dc[NB + b] = col[0].r;
      }
      if (fft3d && P.fft3d_mode != kWienerFused && enh.enh) {
        // enhance(): template ratio recomputed from the spectrum being enhanced
        // (plan.cpp:325-329).
        if (P.fft3d_mode == kWienerThenEnh) __syncthreads();
        if (active) {
          const float dcv = P.fft3d_mode == kWienerThenEnh ? dc[NB + b] : dc[b];
          const float g2 = grid ? fdiv(fmul(P.mean_scale, dcv), grid0) : 0.0f;
#pragma unroll UH
          for (int y = 0; y < CAPH; ++y)
            if (y < BH) col[y] = spectral_bin<-2>(col[y], grid, y * K + k, g2, enh, bad);
        }
      }
      if (active) {
        nf::fft_1d<false, BHC>(col, BH, P.twh, codelet);
#pragma unroll UH
        for (int y = 0; y < CAPH; ++y)
          if (y < BH) sp[y * KNB] = col[y];
      }
      __syncthreads();
    }
    }
    // ---- C: row inverses and synthesis weighting -----------------------------
    if constexpr (kTeam) {
      // Row inverses shared by teams of lanes; the runs are exchanged through the team's
      // scratch (the staging ring, which temporal tiles do not use).
      // Scratch rows of M + 1 values, T + N values per team: a lane's run stores and the
      // outer butterflies' reads then fall in distinct banks across the warp's teams.
      using TW = nf::TeamFFT<false, BWC>;
      cf* xs = reinterpret_cast<cf*>(ring_in) + team * (BWC + TW::T);
      for (Cursor2 c = walk_team; c.y < BH; c.next()) {
        const int y = c.y, b = c.x;
        const cf* bins = spec + y * KNB + b;
        cf run[TW::M];
        // the half spectrum mirrored as row_inverse does: conjugates above BW/2 (0 - im),
        // the DC and Nyquist imaginary parts cleared
        TW::run(lane, run, P.tww, [&](int x) {
          cf v = bins[(x <= BW / 2 ? x : BW - x) * NB];
          if (x > BW / 2) v.i = fsub(0.0f, v.i);
          if (x == 0 || x == BW / 2) v.i = 0.0f;
          return v;
        });
#pragma unroll
        for (int i = 0; i < TW::M; ++i) xs[lane * (TW::M + 1) + i] = run[i];
        __syncwarp(team_mask);
        float* o = ob + (y * NB + b) * OBW;
        float guard = 0.0f;
        TW::outer(lane, P.tww, [&](int j, int i) { return xs[j * (TW::M + 1) + i]; }, [&](int x, cf v) {
          const float r = fmul(v.r, fct);
          guard = __fmaf_rn(r, 0.0f, guard);
          o[x] = fmul(r, wxs[x]);
        });
        __syncwarp(team_mask);  // the scratch is reused by the team's next row
        if (guard != guard) bad = true;
      }
    } else {
    const int center = P.center;
    for (Cursor2 c = walk_nbx; c.y < BH; c.next()) {
      const int y = c.y, b = c.x;
      if (center && y != BH / 2) continue;
      float row[CAPW];
      nf::row_inverse<BWC>(spec + y * KNB + b, BW, SRC == kSrcSlice ? fct3 : fct, row, P.tww, codelet, NB);
      float* o = ob + (y * NB + b) * OBW;
      // NaN once any inverse sample is non-finite (x * 0 is NaN for inf and NaN, and a
      // signed zero otherwise): one multiply-add per sample instead of a compare.
      float guard = 0.0f;
#pragma unroll UW
      for (int x = 0; x < CAPW; ++x) {
        if (x < BW) {
          guard = __fmaf_rn(row[x], 0.0f, guard);
          if constexpr (SRC == kSrcSlice) row[x] = fmul(fmul(volume, row[x]), h[y * BW + x]);
          else row[x] = fft3d ? fmul(row[x], wxs[x]) : fmul(row[x], hsyn[y * BW + x]);
        }
      }
      if (guard != guard) bad = true;
      if ((BW & 3) == 0) {
#pragma unroll UW
        for (int x = 0; x < CAPW; x += 4)
          if (x < BW) *reinterpret_cast<float4*>(o + x) = make_float4(row[x], row[x + 1], row[x + 2], row[x + 3]);
      } else {
#pragma unroll UW
        for (int x = 0; x < CAPW; ++x)
          if (x < BW) o[x] = row[x];
      }
    }
    }
    __syncthreads();
    // ---- D: ordered overlap-add into the ring accumulator --------------------
    const int ylo = max(oy, Y0), yhi = min(oy + BH, Y0 + th);
    if (ola4) {
      // Four consecutive columns per thread (X0, tw and the step multiples of 4): they
      // share their first block and block count, so one 16-byte load per block serves
      // all four, each component summed in the same block order as the scalar path.
      const int adv4 = (OBW - gx.step) >> 2;
      for (Cursor2 c = walk_tw4; c.y < yhi - ylo; c.next()) {
        const int Y = ylo + c.y, xx = c.x << 2, ly = Y - oy;
        float4* a = reinterpret_cast<float4*>(acc + int(unsigned(Y) % unsigned(BH)) * S.tw + xx);
        const int cm = colmap[xx], nblk = (cm >> 10) & 1023;
        const float4* ov = reinterpret_cast<const float4*>(ob + (ly * NB + (cm & 1023)) * OBW + (cm >> 20));
        if (fft3d) {
          float4 r = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
          for (int j = 0; j < nblk; ++j, ov += adv4) {
            const float4 o = *ov;
            r = make_float4(fadd(r.x, o.x), fadd(r.y, o.y), fadd(r.z, o.z), fadd(r.w, o.w));
          }
          const float w = wys[ly];
          const float4 v = *a;
          *a = make_float4(fadd(v.x, fmul(r.x, w)), fadd(v.y, fmul(r.y, w)), fadd(v.z, fmul(r.z, w)),
                           fadd(v.w, fmul(r.w, w)));
        } else {
          float4 sacc = *a;
          int j = 0;
          for (; j + 4 <= nblk; j += 4, ov += 4 * adv4) {  // four blocks per step, added in block order
            const float4 o0 = ov[0], o1 = ov[adv4], o2 = ov[2 * adv4], o3 = ov[3 * adv4];
            sacc = make_float4(fadd(fadd(fadd(fadd(sacc.x, o0.x), o1.x), o2.x), o3.x),
                               fadd(fadd(fadd(fadd(sacc.y, o0.y), o1.y), o2.y), o3.y),
                               fadd(fadd(fadd(fadd(sacc.z, o0.z), o1.z), o2.z), o3.z),
                               fadd(fadd(fadd(fadd(sacc.w, o0.w), o1.w), o2.w), o3.w));
          }
          for (; j < nblk; ++j, ov += adv4) {
            const float4 o = *ov;
            sacc = make_float4(fadd(sacc.x, o.x), fadd(sacc.y, o.y), fadd(sacc.z, o.z), fadd(sacc.w, o.w));
          }
          *a = sacc;
        }
      }
    }
    for (Cursor2 c = walk_tw; !ola4 && c.y < yhi - ylo; c.next()) {
      const int yy = c.y, xx = c.x;
      const int Y = ylo + yy, X = X0 + xx, ly = Y - oy;
      float* a = acc + int(unsigned(Y) % unsigned(BH)) * S.tw + xx;
      const float* orow = ob + ly * NB * OBW;
      if (P.center) {
        const int bc = X - BW / 2;  // block whose centre is X (step 1)
        if (ly == BH / 2 && bc >= bx_lo && bc <= bx_hi) *a = orow[(bc - bx_lo) * OBW + BW / 2];
        continue;
      }
      // blocks b0.. in ascending order; block b0+j holds column X at offset xo - j*step
      const int cm = colmap[xx], nblk = (cm >> 10) & 1023;
      const float* ov = orow + (cm & 1023) * OBW + (cm >> 20);
      const int adv = OBW - gx.step;
      if (fft3d) {
        float r = 0.0f;
        for (int j = 0; j < nblk; ++j, ov += adv) r = fadd(r, *ov);
        *a = fadd(*a, fmul(r, wys[ly]));
      } else {
        float sacc = *a;
        for (int j = 0; j < nblk; ++j, ov += adv) sacc = fadd(sacc, *ov);
        *a = sacc;
      }
    }
    __syncthreads();
    // ---- E: retire rows that no later block row touches ---------------------
    const int rlo = max(oy, Y0), rhi = min(by == by_hi ? Y0 + th : oy + gy.step, Y0 + th);
    const OutConv oc = out_conv(P);
    for (Cursor2 c = walk_tw; c.y < rhi - rlo; c.next()) {
      const int yy = c.y, xx = c.x;
      const int Y = rlo + yy;
      float* a = acc + int(unsigned(Y) % unsigned(BH)) * S.tw + xx;
      const float v = *a;
      if (!isfin(v)) bad = true;
      store_sample<STORAGE, ALGO>(J.dst + ptrdiff_t(Y - gy.offset) * J.dst_stride, px0 + xx, v, oc);
      *a = 0.0f;
    }
  }
  if (bad) atomicOr(P.err, kErrNonFinite);
}

// Resident CTAs per SM the register budget allows: blocks up to 16x16 keep two
// 256-thread CTAs per SM (128 registers per thread); larger transforms need the
// full 255-register budget.
template <int BHC, int BWC>
struct StripOccupancy {
  static constexpr int value = (BHC > 0 && BHC * BWC <= 256) ? 2 : 1;
};

// Plain launch: grid (strips, segments, planes) over up to kMaxPlaneJobs planes of
// one plan (one plane for the drop-in call; several for multi-plane calls).
constexpr int kMaxPlaneJobs = 32;
struct PlaneJobs {
  PlaneJob job[kMaxPlaneJobs];
  int n;
};

template <int BHC, int BWC, int STORAGE, int ALGO>
__global__ void __launch_bounds__(256, StripOccupancy<BHC, BWC>::value)
    spatial_strip_kernel(DevPlan P, StripShape S, const __grid_constant__ PlaneJobs J) {
  extern __shared__ float smem[];
  strip_tile<BHC, BWC, STORAGE, kSrcPixels, ALGO>(P, J.job[blockIdx.z], S, blockIdx.x * S.tw, blockIdx.y * S.th,
                                                  smem);
}

// Kalman render (plan.cpp:471-477): the inverse transforms of the state's estimate and
// the enhancement, per plain strip tile. Blocks up to 32x32 run two CTAs per SM (the
// render holds one column transform at a time, with no staging ring or forward rows).
template <int BHC, int BWC>
struct RenderOccupancy {
  static constexpr int value = (BHC > 0 && BHC * BWC <= 1024) ? 2 : 1;
};

template <int BHC, int BWC, int STORAGE>
__global__ void __launch_bounds__(256, RenderOccupancy<BHC, BWC>::value)
    kalman_render_kernel(DevPlan P, StripShape S, const __grid_constant__ PlaneJobs J) {
  extern __shared__ float smem[];
  strip_tile<BHC, BWC, STORAGE, kSrcKalman, 0>(P, J.job[blockIdx.z], S, blockIdx.x * S.tw, blockIdx.y * S.th, smem);
}

// Batched launch: a persistent grid pulls (plane, strip, segment) work items from
// a device queue; planes may come from different plans of the same block shape
// (luma and chroma, or clips of several resolutions).
struct BatchWork {
  const DevPlan* plans;
  const StripShape* shapes;  // per plan
  const PlaneJob* jobs;
  const int* job_tile_base;  // prefix sums of tiles per job (njobs+1)
  const int* job_tiles_x;    // strips per job
  int njobs;
  int* counter;              // work-queue head, reset by the host before launch
};

// Batched launch over planes of one algorithm (ALGO 0 FFT3D, 1 DFTTest).
template <int BHC, int BWC, int STORAGE, int ALGO>
__global__ void __launch_bounds__(256, StripOccupancy<BHC, BWC>::value) spatial_batch_kernel(BatchWork W) {
  extern __shared__ float smem[];
  __shared__ int item;
  __shared__ alignas(8) unsigned long long s_mbar[2];
  __shared__ int s_dead;
  if (threadIdx.x == 0) {
    mbar_init(s_mbar, 1);
    mbar_init(s_mbar + 1, 1);
    mbar_init_fence();
    s_dead = 0;
  }
  TmaPipe pipe{s_mbar, &s_dead, 0u, 0u};
  const int total = W.job_tile_base[W.njobs];
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) item = atomicAdd(W.counter, 1);
    __syncthreads();
    const int t = item;
    if (t >= total) break;
    int lo = 0, hi = W.njobs - 1;  // job containing tile t
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (W.job_tile_base[mid] <= t) lo = mid;
      else hi = mid - 1;
    }
    // The work item's plan, job and shape are read once into shared memory (a
    // per-thread copy of the plan would live on the local-memory stack).
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
    strip_tile<BHC, BWC, STORAGE, kSrcPixels, ALGO>(sP, sJ, sS, sx * sS.tw, sy * sS.th, smem, &pipe);
  }
  // Copies still in flight after a wait ran out: wait for them once more (bounded)
  // before the CTA's shared memory is released.
  if (threadIdx.x == 0)
    for (int b = 0; b < 2; ++b)
      if (pipe.pending & (1u << b)) mbar_wait_bounded(s_mbar + b, (pipe.phase >> b) & 1u, kStagingWaitCycles);
}

} // namespace nfd
