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
//
// The Kalman step (advance, then render of the same frame: plan.cpp:301-321 followed by
// the Kalman branch of plan.cpp:471-490) keeps each block's new estimate L in shared
// memory after the recursion and renders it there: enhancement with the template ratio
// of L's DC, inverse columns, inverse rows and the horizontal synthesis weight. The
// synthesised 32x32 (bh x bw) blocks go to a buffer in the state's block order, and
// kalman_ola_kernel adds them per pixel in the reference's order. So each block is
// transformed forward once and back once, the state is read once and written once, and
// no block is transformed twice (a strip tile would redo its halo blocks).
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
  float* synth;  // Kalman step: synthesised blocks [block row][block column][bh][bw], else nullptr
  int staged;    // runs copy their old state into shared memory (bins a multiple of 4)
};

// Shared memory of a run of nb blocks of `bins` bins (byte offsets, 16-byte aligned):
// spectra [nb][bins] complex | estimate DCs [nb] floats (step) | staged old state: L
// [nb][bins] complex, C and Q [nb][bins] in the state's precision.
struct KalmanSmem {
  size_t dcs, last, cov, proc, bytes;
};
__host__ __device__ inline KalmanSmem kalman_smem(int bins, int nb, bool step, int fp64, int staged) {
  auto up = [](size_t v) { return (v + 15) & ~size_t(15); };
  KalmanSmem m;
  const size_t cnt = size_t(nb) * bins, cs = fp64 ? 8 : 4;
  m.dcs = up(cnt * 8);
  m.last = up(m.dcs + (step ? size_t(nb) * 4 : 0));
  m.cov = up(m.last + (staged ? cnt * 8 : 0));
  m.proc = up(m.cov + (staged ? cnt * cs : 0));
  m.bytes = up(m.proc + (staged ? cnt * cs : 0));
  return m;
}

// STEP: advance and render (A.synth receives the synthesised blocks). Shared memory: the
// run's spectra [block][bins] complex, then (STEP) the run's estimate DCs [nb].
template <int BHC, int BWC, int STORAGE, bool STEP>
__global__ void __launch_bounds__(256) kalman_advance_kernel(DevPlan P, int nb_per_cta, const unsigned char* src,
                                                             ptrdiff_t src_stride, KalmanArgs A) {
  extern __shared__ __align__(16) unsigned char kalman_shared[];  // bulk copies land on 16 bytes
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
  const int by = blockIdx.y;
  const int bx0 = blockIdx.x * nb_per_cta;
  const int nb = min(nb_per_cta, gx.count - bx0);
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int oy = by * gy.step;
  bool bad = false;
  const KalmanSmem lay = kalman_smem(BH * K, nb_per_cta, STEP, A.fp64, A.staged);
  unsigned char* sbase = kalman_shared;
  cf* spec = reinterpret_cast<cf*>(sbase);
  float* dcs = reinterpret_cast<float*>(sbase + lay.dcs);
  (void)dcs;
  const cf* st_last = reinterpret_cast<const cf*>(sbase + lay.last);
  const unsigned char* st_c = sbase + lay.cov;
  const unsigned char* st_q = sbase + lay.proc;
  // The run's old state is contiguous in each array: one elected thread copies it into
  // shared memory with three bulk copies (this GPU's own memory) while the transforms run.
  __shared__ alignas(8) unsigned long long s_mbar;
  const bool staged = A.staged != 0;
  if (staged && tid == 0) {
    const size_t cs = A.fp64 ? sizeof(double) : sizeof(float);
    const size_t first = (size_t(by) * gx.count + bx0) * size_t(BH * K), cnt = size_t(nb) * BH * K;
    const void* gc = A.fp64 ? static_cast<const void*>(A.cov64 + first) : static_cast<const void*>(A.cov32 + first);
    const void* gq = A.fp64 ? static_cast<const void*>(A.proc64 + first) : static_cast<const void*>(A.proc32 + first);
    mbar_init(&s_mbar, 1);
    mbar_init_fence();
    mbar_expect_tx(&s_mbar, unsigned(cnt * (sizeof(cf) + 2 * cs)));
    bulk_load_1d(sbase + lay.last, A.last + first, unsigned(cnt * sizeof(cf)), &s_mbar);
    bulk_load_1d(sbase + lay.cov, gc, unsigned(cnt * cs), &s_mbar);
    bulk_load_1d(sbase + lay.proc, gq, unsigned(cnt * cs), &s_mbar);
  }
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
  // of the run is state element base + i (coalesced; the arrays never alias). A staged
  // run reads its old state from the shared copy the bulk copies brought in while the
  // transforms ran; a run whose wait runs out reads it from global memory (the same values:
  // only this thread writes its bins) and reports kErrStaging.
  const int bins = BH * K;
  const int n = nb * bins;
  const size_t base = (size_t(by) * gx.count + bx0) * size_t(bins);
  cf* __restrict__ last = A.last + base;
  const float* __restrict__ pattern = A.pattern;
  bool from_stage = false;
  if (staged) {
    from_stage = mbar_wait_bounded(&s_mbar, 0u, kStagingWaitCycles);
    if (!from_stage) atomicOr(P.err, kErrStaging);
  }
  // Eight bins per thread and step: their loads are issued together before the first
  // recursion, so each thread keeps several state reads in flight.
  constexpr int kStep = 8;
  auto recursion = [&](auto* cov, auto* proc, const auto* st_cov, const auto* st_proc) {
    using Var = typename std::remove_pointer<decltype(cov)>::type;
    const cf* L_in = from_stage ? st_last : last;
    const Var* C_in = from_stage ? st_cov : cov;
    const Var* Q_in = from_stage ? st_proc : proc;
    for (int i0 = tid; i0 < n; i0 += kStep * nthr) {
      cf L[kStep];
      Var c[kStep], q[kStep];
#pragma unroll
      for (int j = 0; j < kStep; ++j) {
        const int i = i0 + j * nthr;
        if (i < n) {
          L[j] = L_in[i];
          c[j] = C_in[i];
          q[j] = Q_in[i];
        }
      }
#pragma unroll
      for (int j = 0; j < kStep; ++j) {
        const int i = i0 + j * nthr;
        if (i < n) {
          const int blk = i / bins, kk = i - blk * bins;
          bool ok;
          if constexpr (sizeof(Var) == 8) ok = kalman_bin_fp64(spec[i], L[j], c[j], q[j], pattern, kk, P.kalman_r0, P.kalman_ratio2);
          else ok = kalman_bin(spec[i], L[j], c[j], q[j], pattern, kk, P.kalman_r0, P.kalman_ratio2);
          if (!ok) bad = true;
          last[i] = L[j];
          if constexpr (STEP) {  // the estimate stays in shared memory for the render
            spec[i] = L[j];
            if (kk == 0) dcs[blk] = L[j].r;
          }
          cov[i] = c[j];
          proc[i] = q[j];
        }
      }
    }
  };
  if (A.fp64)
    recursion(A.cov64 + base, A.proc64 + base, reinterpret_cast<const double*>(st_c),
              reinterpret_cast<const double*>(st_q));
  else
    recursion(A.cov32 + base, A.proc32 + base, reinterpret_cast<const float*>(st_c),
              reinterpret_cast<const float*>(st_q));
  if constexpr (STEP) {
    // Render of the run's new estimates (the Kalman branch of plan.cpp:471-490): enhancement
    // with the template ratio of the estimate's DC (plan.cpp:325-329), inverse columns,
    // inverse rows with the non-finite check, horizontal synthesis weight.
    __syncthreads();
    const cf* grid = P.grid;
    const float grid0 = grid ? grid[0].r : 1.0f;
    const DevSpectral& enh = P.enh;
    for (int task = tid; task < nb * K; task += nthr) {
      const int b = task / K, k = task - b * K;
      cf col[CAPH];
      cf* sp = spec + size_t(b) * bins + k;
#pragma unroll UH
      for (int y = 0; y < CAPH; ++y)
        if (y < BH) col[y] = sp[size_t(y) * K];
      if (enh.enh) {
        const float g2 = grid ? fdiv(fmul(P.mean_scale, dcs[b]), grid0) : 0.0f;
#pragma unroll UH
        for (int y = 0; y < CAPH; ++y)
          if (y < BH) col[y] = spectral_bin<-2>(col[y], grid, y * K + k, g2, enh, bad);
      }
      nf::fft_1d<false, BHC>(col, BH, P.twh, codelet);
#pragma unroll UH
      for (int y = 0; y < CAPH; ++y)
        if (y < BH) sp[size_t(y) * K] = col[y];
    }
    __syncthreads();
    const float fct = fdiv(1.0f, fmul(float(BW), float(BH)));
    float* out = A.synth + (size_t(by) * gx.count + bx0) * size_t(BH) * BW;
    for (int task = tid; task < nb * BH; task += nthr) {
      const int b = task / BH, y = task - b * BH;
      float row[CAPW];
      nf::row_inverse<BWC>(spec + size_t(b) * bins + size_t(y) * K, BW, fct, row, P.tww, codelet);
      float guard = 0.0f;  // NaN once a sample is non-finite (x * 0 is NaN for inf and NaN)
      float* o = out + (size_t(b) * BH + y) * BW;
#pragma unroll UW
      for (int x = 0; x < CAPW; ++x) {
        if (x < BW) {
          guard = __fmaf_rn(row[x], 0.0f, guard);
          row[x] = fmul(row[x], P.wxs[x]);
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
  // A wait that ran out: wait once more (bounded) for the copies still in flight before the
  // CTA's shared memory is released.
  if (staged && !from_stage && tid == 0) mbar_wait_bounded(&s_mbar, 0u, kStagingWaitCycles);
  if (bad) atomicOr(P.err, kErrNonFinite);
}

// Overlap-add of the Kalman step's synthesised blocks in the order of the FFT3D branch of
// plan.cpp:520-535: per covering block row (ascending) the covering blocks' samples are
// summed from zero in block-column order, the sum is weighted by the vertical synthesis
// window and added to the pixel's accumulator; then the output conversion
// (kernels/scalar/spatial.cpp:89-129). FFT3D overlaps are at most half a block, so at most
// two block rows and two block columns cover a pixel: every load is issued before the
// sums. V = 4 (2): a thread owns four (two) adjacent pixels, which share their covering
// blocks when the step, the block width and the cover offset are multiples of four (two):
// one 16-byte (8-byte) load per block; V = 1 otherwise.
template <int STORAGE, int V>
__global__ void __launch_bounds__(256) kalman_ola_kernel(DevPlan P, const float* __restrict__ synth, unsigned char* dst,
                                                         long long dst_stride) {
  const DevAxis gx = P.gx, gy = P.gy;
  const int BH = P.bh, BW = P.bw;
  // the last covering block is the one starting at or before the pixel; the one before it
  // covers the pixel too when the pixel lies within its block length (one division per axis)
  const int Y = blockIdx.y, cy = Y + gy.offset;
  const int by1 = min(gy.count - 1, cy / gy.step);
  const int by0 = by1 > 0 && cy - (by1 - 1) * gy.step < BH ? by1 - 1 : by1;
  const int X = (blockIdx.x * blockDim.x + threadIdx.x) * V;
  if (X >= gx.length) return;
  const int cx = X + gx.offset;
  const int bx1 = min(gx.count - 1, cx / gx.step);
  const int bx0 = bx1 > 0 && cx - (bx1 - 1) * gx.step < BW ? bx1 - 1 : bx1;
  using Vec = typename std::conditional<V == 4, float4, typename std::conditional<V == 2, float2, float>::type>::type;
  Vec v[2][2];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int by = by0 + i, bx = bx0 + j;
      if (by <= by1 && bx <= bx1) {
        const size_t at = ((size_t(by) * gx.count + bx) * BH + (cy - by * gy.step)) * BW + (cx - bx * gx.step);
        v[i][j] = *reinterpret_cast<const Vec*>(synth + at);
      }
    }
  }
  float acc[V];
#pragma unroll
  for (int e = 0; e < V; ++e) acc[e] = 0.0f;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int by = by0 + i;
    if (by > by1) break;
    const float w = P.wys[cy - by * gy.step];
#pragma unroll
    for (int e = 0; e < V; ++e) {
      float r = 0.0f;
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        if (bx0 + j <= bx1) {
          const float* f = reinterpret_cast<const float*>(&v[i][j]);
          r = fadd(r, f[e]);
        }
      }
      acc[e] = fadd(acc[e], fmul(r, w));
    }
  }
  unsigned char* row = dst + ptrdiff_t(Y) * dst_stride;
  bool bad = false;
#pragma unroll
  for (int e = 0; e < V; ++e) {
    if (X + e < gx.length) {
      if (!isfin(acc[e])) bad = true;
      store_sample<STORAGE, 0>(row, X + e, acc[e], P);
    }
  }
  if (bad) atomicOr(P.err, kErrNonFinite);
}

} // namespace nfd
