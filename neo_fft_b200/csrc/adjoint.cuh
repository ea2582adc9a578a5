// Adjoint (backward) of the single-frame pipelines for float planes, with respect to
// the source pixels and to the per-bin primary table A (the learnable sigma table):
// DFTTest (tbsize=1, smode=1, ftype 0/1/2, zmean on or off) and FFT3D (bt=1: Wiener
// gain with the beta floor, degrid template, sharpen/dehalo fused into the gain, output
// clamped to [0, 1]).
//
// Forward per block (src/algorithms/plan.cpp:538-607, kernels/scalar/spectral.cpp):
//   v = 255*s (decode), b = v*h, X = r2c(b), g = mean*Re X0 / Re G0, M = g*G,
//   R = X - M, p = |R|^2, gain(p, A), Y = gain*R + M, y = c2r(Y)/N, acc += y*hsyn,
//   out = acc/255.
// Backward per block, with the forward spectra recomputed (nothing is stored):
//   d_acc = d_out/255 -> dy = d_acc*hsyn (transposed overlap-add, gathered)
//   dY = (m_kx/N) * r2c(dy)          adjoint of the half-complex inverse
//                                     (m_kx = 1 for the DC/Nyquist columns, else 2)
//   per bin: dR = gain*dY + 2*dgain/dp*<dY,R>*R, dM = dY - dR, dX = dR,
//            dA += <dY,R>*dgain/dA; dg = sum_k <dM_k, G_k>; dX0.re += dg*mean/Re G0
//   db = c2r_unnormalised(dX')        adjoint of r2c (dX' halves interior columns)
//   dv = db*h -> d_cover (ordered gather, like the forward overlap-add)
// FFT3D differs only in the windows and the gain (src/algorithms/plan.cpp:432-537,
// kernels/scalar/spectral.cpp:18-22, algorithms/fft3d_profile.cpp:69-81):
//   b = (v*wy)*wx, gain = max((q - A)/q, floor) * S(q) * D(q) with q = p + 1e-15,
//   acc += (y*wxs)*wys, out = clamp(acc, 0, 1): the upstream gradient passes only where
//   the forward output lies strictly inside (0, 1).
// A second kernel folds the cover gradient onto the source through the single
// reflection and multiplies by the decode scale; a third reduces the per-tile table
// gradients in a fixed order. Every sum has a fixed order, so gradients are deterministic.
#pragma once
#include "tile_spatial.cuh"

namespace nfd {

struct AdjointShape {
  int tw, th;       // tile of the cover plane
  int nbx_max, win_max, ring_pitch, tab_floats;
  int tiles_x, tiles_y;
};

struct AdjointJob {
  const float* src;     // forward input plane (float samples)
  long long src_stride; // bytes
  const float* gout;    // gradient of the output plane
  long long gout_stride;
  float* dcov;          // scratch: cover-plane gradient [cover_h][cover_w]
  float* partial;       // scratch: per-tile table gradients [tiles][bins]
  const float* fwd;     // FFT3D: the forward output plane (clamp mask); nullptr for DFTTest
  long long fwd_stride;
};

__host__ __device__ inline size_t adjoint_smem_bytes(int bh, int bw, const AdjointShape& s) {
  const size_t K = size_t(bw / 2 + 1), bins = size_t(bh) * K;
  const size_t spec_cf = (size_t(s.nbx_max) * bh * K + 1) & ~size_t(1);
  return sizeof(float) * (size_t(s.tab_floats) + 2 * size_t(bh) * s.ring_pitch + 2 * spec_cf * 2 +
                          size_t(bh) * s.nbx_max * (bw + 4) + size_t(bh) * s.tw + 2 * size_t(s.nbx_max) +
                          size_t(s.nbx_max | 1) * bins + bins + 2 * size_t(s.nbx_max) * K + size_t(s.tw));
}

// Per-bin backward of spectral_bin for ftype 0 (Wiener, any exponent), 1 (hard
// threshold), 2 (constant gain) and -1 (FFT3D Wiener with floor, enhancement fused).
// x: forward spectrum bin; dy: incoming complex gradient. Returns dX; adds the template
// gradient to dg and the table gradient to da. FT fixes the type at compile time.
template <int FT>
__device__ __forceinline__ cf spectral_bin_adjoint(cf x, cf dy, const cf* grid, int k, float g, const DevSpectral& p,
                                                   float& dg, float& da) {
  const int type = FT;
  const float a = p.primary ? p.primary[k] : p.a;
  const float mr = grid ? g * grid[k].r : 0.0f;
  const float mi = grid ? g * grid[k].i : 0.0f;
  const float re = x.r - mr, im = x.i - mi;
  const float power = re * re + im * im;
  float gain = 0.0f, dgain_dp = 0.0f, dgain_da = 0.0f;
  if (type == 0) {
    const float q = power + 1e-15f;
    const float r = (power - a) / q;
    if (r > 0.0f) {
      float dw;  // d gain / d r
      if (p.emode == 0) {  // the forward's exponent test (spectral.cpp:25-27), made once per plan
        gain = r;
        dw = 1.0f;
      } else if (p.emode == 1) {
        gain = sqrtf(r);
        dw = 0.5f / gain;
      } else {
        gain = powf(r, p.exponent);
        dw = p.exponent * gain / r;
      }
      dgain_dp = dw * (a + 1e-15f) / (q * q);
      dgain_da = -dw / q;
    }
  } else if (type == -1) {
    // wiener = max((q - a)/q, floor); the ratio wins ties, as in the forward
    const float q = power + 1e-15f;
    const float r = (q - a) / q;
    float w = p.floor, dw_dq = 0.0f, dw_da = 0.0f;
    if (!(r < p.floor)) {
      w = r;
      dw_dq = a / (q * q);
      dw_da = -1.0f / q;
    }
    float e = 1.0f, de_dq = 0.0f;
    if (p.enh) {  // S(q) * D(q) and its derivative (fft3d_profile.cpp:69-81)
      float sv = 1.0f, ds = 0.0f, dv = 1.0f, dd = 0.0f;
      if (p.sharpen != 0.0f && p.eb != 0.0f) {
        const float qa = q + p.ea, qb = q + p.eb;
        const float u = q * p.eb / (qa * qb);
        const float str = p.sharpen * p.sharpen_w[k];
        const float su = sqrtf(u);
        sv = 1.0f + str * su;
        // du/dq = eb (ea eb - q^2) / ((q+ea)(q+eb))^2
        const float du = p.eb * (p.ea * p.eb - q * q) / ((qa * qb) * (qa * qb));
        ds = su > 0.0f ? str * du / (2.0f * su) : 0.0f;
      }
      if (p.dehalo != 0.0f) {
        const float hd = p.dehalo * p.halo_w[k];
        const float qc = q + p.ec, den = qc + hd * q;
        dv = qc / den;
        dd = -hd * p.ec / (den * den);
      }
      e = sv * dv;
      de_dq = ds * dv + sv * dd;
    }
    gain = w * e;
    dgain_dp = dw_dq * e + w * de_dq;
    dgain_da = dw_da * e;
  } else if (type == 1) {
    gain = power < a ? 0.0f : 1.0f;
  } else {
    gain = a;
    dgain_da = 1.0f;
  }
  const float dgain = dy.r * re + dy.i * im;  // <dY, R>
  da += dgain * dgain_da;
  const float dp = dgain * dgain_dp;
  const cf dr = {gain * dy.r + 2.0f * dp * re, gain * dy.i + 2.0f * dp * im};
  if (grid) dg += (dy.r - dr.r) * grid[k].r + (dy.i - dr.i) * grid[k].i;
  return dr;
}

// ALGO: 0 FFT3D, 1 DFTTest.
template <int BHC, int BWC, int ALGO>
__device__ __forceinline__ void adjoint_tile(const DevPlan& P, const AdjointJob& J, const AdjointShape& S, int tile,
                                             float* smem) {
  constexpr bool kFft3d = ALGO == 0;
  const int BH = BHC > 0 ? BHC : P.bh;
  const int BW = BWC > 0 ? BWC : P.bw;
  const int K = BW / 2 + 1;
  constexpr int CAPH = BHC > 0 ? BHC : nf::kMaxProject;
  constexpr int CAPW = BWC > 0 ? BWC : nf::kMaxProject;
  constexpr int UH = BHC > 0 ? CAPH : 1, UW = BWC > 0 ? CAPW : 1;
  constexpr bool kCodelet = BHC == BWC && (BWC == 8 || BWC == 16 || BWC == 32);
  const bool codelet = kCodelet || (BHC == 0 && P.codelet != 0);
  const DevAxis gx = P.gx, gy = P.gy;
  const int NB = S.nbx_max, OBW = BW + 4, bins = BH * K;
  const int tid = threadIdx.x, nthr = blockDim.x;

  // Tile of the cover plane (cover coordinates).
  const int X0 = (tile % S.tiles_x) * S.tw, Y0 = (tile / S.tiles_x) * S.th;
  const int tw = min(S.tw, gx.cover - X0), th = min(S.th, gy.cover - Y0);
  const int bx_lo = max(0, floor_div_i(X0 - BW, gx.step) + 1);
  const int bx_hi = min(gx.count - 1, floor_div_i(X0 + tw - 1, gx.step));
  const int by_lo = max(0, floor_div_i(Y0 - BH, gy.step) + 1);
  const int by_hi = min(gy.count - 1, floor_div_i(Y0 + th - 1, gy.step));
  const int nbx = bx_hi - bx_lo + 1;
  const int cx0 = bx_lo * gx.step;
  const int win = (nbx - 1) * gx.step + BW;

  float* tab = smem;
  float* ring = tab + S.tab_floats;
  float* gring = ring + size_t(BH) * S.ring_pitch;
  const size_t spec_cf = (size_t(NB) * BH * K + 1) & ~size_t(1);
  cf* spec = reinterpret_cast<cf*>(gring + size_t(BH) * S.ring_pitch);
  cf* gspec = spec + spec_cf;
  float* ob = reinterpret_cast<float*>(gspec + spec_cf);
  float* acc = ob + size_t(BH) * NB * OBW;
  float* dc = acc + size_t(BH) * S.tw;
  // Per-block table gradients [bin][block] with an odd block stride: the column threads
  // (consecutive blocks) write consecutive words and the per-bin sums read rows whose
  // starts fall in distinct banks.
  const int NBp = NB | 1;
  float* da_blk = dc + 2 * size_t(NB);
  float* da_tile = da_blk + size_t(NBp) * bins;
  float* dg_part = da_tile + bins;  // [NB][K]
  int* colmap = reinterpret_cast<int*>(dg_part + 2 * size_t(NB) * K);  // [tw], as in strip_tile
  const bool ola4 = (gx.step & 3) == 0 && (BW & 3) == 0 && (S.tw & 3) == 0 && (tw & 3) == 0 && (X0 & 3) == 0;

  // tables
  int off = 0;
  auto stage = [&](const float* src, int n) {
    float* d = tab + off;
    for (int i = tid; i < n; i += nthr) d[i] = src[i];
    off += n;
    return d;
  };
  const float *h = nullptr, *hsyn = nullptr, *wxa = nullptr, *wya = nullptr, *wxs = nullptr, *wys = nullptr;
  if constexpr (kFft3d) {
    wxa = stage(P.wxa, BW);
    wya = stage(P.wya, BH);
    wxs = stage(P.wxs, BW);
    wys = stage(P.wys, BH);
  } else {
    h = stage(P.h, BH * BW);
    hsyn = stage(P.hsyn, BH * BW);
  }
  const cf* grid = P.grid ? reinterpret_cast<const cf*>(stage(reinterpret_cast<const float*>(P.grid), 2 * bins)) : nullptr;
  __shared__ DevSpectral s_filt;
  const float* prim = P.filt.primary ? stage(P.filt.primary, bins) : nullptr;
  const float* shw = kFft3d && P.filt.enh && P.filt.sharpen_w ? stage(P.filt.sharpen_w, bins) : nullptr;
  const float* hlw = kFft3d && P.filt.enh && P.filt.halo_w ? stage(P.filt.halo_w, bins) : nullptr;
  if (tid == 0) {
    s_filt = P.filt;
    if (prim) s_filt.primary = prim;
    if (shw) s_filt.sharpen_w = shw;
    if (hlw) s_filt.halo_w = hlw;
  }
  for (int i = tid; i < BH * S.tw; i += nthr) acc[i] = 0.0f;
  for (int i = tid; i < bins; i += nthr) da_tile[i] = 0.0f;
  for (int xx = tid; xx < tw; xx += nthr) {  // first overlapping block, count, offset in it
    const int X = X0 + xx;
    const int b0 = max(bx_lo, floor_div_i(X - BW, gx.step) + 1), b1 = min(bx_hi, floor_div_i(X, gx.step));
    const int nblk = max(0, b1 - b0 + 1);
    colmap[xx] = (b0 - bx_lo) | (nblk << 10) | ((nblk > 0 ? X - b0 * gx.step : 0) << 20);
  }
  __syncthreads();
  const DevSpectral& filt = s_filt;
  const float grid0 = grid ? grid[0].r : 1.0f;
  const float invN = 1.0f / (float(BW) * float(BH));
  const float out_scale = P.out_scale;

  // No barrier between a block row's retire phase (accumulator ring and the cover gradient) and
  // the next block row's staging (source and gradient rings): they touch disjoint shared memory,
  // and every later phase is behind a barrier.
  // The phases' thread-to-(row, column) walks, divided once per tile (a division inside the
  // block-row loop is not hoisted by the compiler).
  const Cursor2 walk_win(tid, nthr, win), walk_nbx(tid, nthr, nbx), walk_tw(tid, nthr, tw),
      walk_tw4(tid, nthr, max(tw >> 2, 1));
  for (int by = by_lo; by <= by_hi; ++by) {
    const int oy = by * gy.step;
    // ---- stage source rows (decoded) and upstream-gradient rows -------------
    const int r0 = by == by_lo ? oy : max(oy, oy + BH - gy.step);
    const int nrows = oy + BH - r0;
    for (Cursor2 c = walk_win; c.y < nrows; c.next()) {
      const int rr = c.y, xx = c.x;
      const int cy = r0 + rr, cx = cx0 + xx;
      const float* srow = reinterpret_cast<const float*>(reinterpret_cast<const unsigned char*>(J.src) +
                                                         ptrdiff_t(reflect_axis(cy, gy)) * J.src_stride);
      ring[size_t(cy % BH) * S.ring_pitch + xx] = srow[reflect_axis(cx, gx)] * P.dec_scale;
      const int py = cy - gy.offset, px = cx - gx.offset;
      float gv = 0.0f;
      if (py >= 0 && py < gy.length && px >= 0 && px < gx.length) {
        gv = reinterpret_cast<const float*>(reinterpret_cast<const unsigned char*>(J.gout) +
                                            ptrdiff_t(py) * J.gout_stride)[px] * out_scale;
        if constexpr (kFft3d) {  // out = clamp(acc, 0, 1)
          const float y = reinterpret_cast<const float*>(reinterpret_cast<const unsigned char*>(J.fwd) +
                                                         ptrdiff_t(py) * J.fwd_stride)[px];
          if (!(y > 0.0f && y < 1.0f)) gv = 0.0f;
        }
      }
      gring[size_t(cy % BH) * S.ring_pitch + xx] = gv;
    }
    __syncthreads();
    // ---- rows: forward spectrum rows and gradient rows ----------------------
    for (Cursor2 c = walk_nbx; c.y < 2 * BH; c.next()) {
      const int which = c.y >= BH ? 1 : 0, y = c.y - which * BH, b = c.x;
      const float* in = (which ? gring : ring) + size_t((oy + y) % BH) * S.ring_pitch + b * gx.step;
      float row[CAPW];
#pragma unroll UW
      for (int x = 0; x < CAPW; ++x)
        if (x < BW) {
          if constexpr (kFft3d)  // the forward's (v*wy)*wx; the synthesis weight wxs*wys
            row[x] = which ? in[x] * (wxs[x] * wys[y]) : fmul(fmul(in[x], wya[y]), wxa[x]);
          else
            row[x] = which ? in[x] * hsyn[y * BW + x] : fmul(in[x], h[y * BW + x]);
        }
      nf::row_forward<BWC>(row, BW, (which ? gspec : spec) + size_t(y) * K * NB + b, P.tww, codelet, NB);
    }
    __syncthreads();
    // ---- columns: forward transforms, DC exchange, per-bin adjoint -----------
    // (k = 0 tasks come first, so every block's DC is exchanged in the first pass)
    const int ncol = nbx * K;
    Cursor2 cb = walk_nbx;
    for (int base = 0; base < ncol; base += nthr, cb.next()) {
      const bool active = cb.y < K;  // task < ncol
      const int k = active ? cb.y : 0, b = active ? cb.x : 0;
      cf x[CAPH], gcol[CAPH];
      cf* sp = spec + size_t(k) * NB + b;
      cf* gp = gspec + size_t(k) * NB + b;
      float dg = 0.0f;
      if (active) {
#pragma unroll UH
        for (int y = 0; y < CAPH; ++y)
          if (y < BH) {
            x[y] = sp[size_t(y) * K * NB];
            gcol[y] = gp[size_t(y) * K * NB];
          }
        nf::fft_1d<true, BHC>(x, BH, P.twh, codelet);
        nf::fft_1d<true, BHC>(gcol, BH, P.twh, codelet);
        if (k == 0) dc[b] = x[0].r;
      }
      __syncthreads();
      if (active) {
        const float g = grid ? fmul(P.mean_scale, dc[b]) / grid0 : 0.0f;
        const float mk = (k == 0 || (BW % 2 == 0 && k == BW / 2)) ? invN : 2.0f * invN;
        const bool own = (bx_lo + b) * gx.step >= X0 && (bx_lo + b) * gx.step < X0 + tw && oy >= Y0 && oy < Y0 + th;
        // The ftype fixed at compile time per branch (no switch per bin).
        auto adjoint_column = [&](auto ft) {
          constexpr int FT = decltype(ft)::value;
#pragma unroll UH
          for (int y = 0; y < CAPH; ++y)
            if (y < BH) {
              float da = 0.0f;
              const cf dY = {gcol[y].r * mk, gcol[y].i * mk};
              sp[size_t(y) * K * NB] = spectral_bin_adjoint<FT>(x[y], dY, grid, y * K + k, g, filt, dg, da);
              da_blk[size_t(y * K + k) * NBp + b] = own ? da : 0.0f;
            }
        };
        if constexpr (kFft3d) adjoint_column(std::integral_constant<int, -1>{});
        else if (filt.type == 0) adjoint_column(std::integral_constant<int, 0>{});
        else if (filt.type == 1) adjoint_column(std::integral_constant<int, 1>{});
        else adjoint_column(std::integral_constant<int, 2>{});
        dg_part[size_t(b) * K + k] = dg;
      }
    }
    __syncthreads();
    // ---- columns: template-ratio gradient, adjoint of r2c, inverse -----------
    for (Cursor2 c = walk_nbx; c.y < K; c.next()) {
      const int k = c.y, b = c.x;
      cf x[CAPH];
      cf* sp = spec + size_t(k) * NB + b;
#pragma unroll UH
      for (int y = 0; y < CAPH; ++y)
        if (y < BH) x[y] = sp[size_t(y) * K * NB];
      if (k == 0 && grid) {  // g = mean * Re X0 / Re G0
        float dgs = 0.0f;
        for (int kk = 0; kk < K; ++kk) dgs += dg_part[size_t(b) * K + kk];
        x[0].r += dgs * P.mean_scale / grid0;
      }
      // adjoint of r2c: halve interior columns, unnormalised inverse
      const float half = (k == 0 || (BW % 2 == 0 && k == BW / 2)) ? 1.0f : 0.5f;
#pragma unroll UH
      for (int y = 0; y < CAPH; ++y)
        if (y < BH) x[y] = {x[y].r * half, x[y].i * half};
      nf::fft_1d<false, BHC>(x, BH, P.twh, codelet);
#pragma unroll UH
      for (int y = 0; y < CAPH; ++y)
        if (y < BH) sp[size_t(y) * K * NB] = x[y];
    }
    __syncthreads();
    // ---- table gradient of owned blocks, in block order ----------------------
    for (int i = tid; i < bins; i += nthr) {
      float s = da_tile[i];
      for (int b = 0; b < nbx; ++b) s += da_blk[size_t(i) * NBp + b];
      da_tile[i] = s;
    }
    // ---- rows: unnormalised inverse, analysis-window weighting ---------------
    for (Cursor2 c = walk_nbx; c.y < BH; c.next()) {
      const int y = c.y, b = c.x;
      float row[CAPW];
      nf::row_inverse<BWC>(spec + size_t(y) * K * NB + b, BW, 1.0f, row, P.tww, codelet, NB);
      float* o = ob + (size_t(y) * NB + b) * OBW;
#pragma unroll UW
      for (int x = 0; x < CAPW; ++x)
        if (x < BW) o[x] = kFft3d ? row[x] * (wya[y] * wxa[x]) : row[x] * h[y * BW + x];
    }
    __syncthreads();
    // ---- ordered gather into the cover-gradient ring; retire rows -------------
    const int ylo = max(oy, Y0), yhi = min(oy + BH, Y0 + th);
    if (ola4) {  // four columns per thread, one 16-byte load per block (as in strip_tile)
      const int adv4 = (OBW - gx.step) >> 2;
      for (Cursor2 c = walk_tw4; c.y < yhi - ylo; c.next()) {
        const int Y = ylo + c.y, xx = c.x << 2, ly = Y - oy;
        float4* a = reinterpret_cast<float4*>(acc + size_t(Y % BH) * S.tw + xx);
        const int cm = colmap[xx], nblk = (cm >> 10) & 1023;
        const float4* ov =
            reinterpret_cast<const float4*>(ob + size_t(ly) * NB * OBW + size_t(cm & 1023) * OBW + (cm >> 20));
        float4 sacc = *a;
        for (int j = 0; j < nblk; ++j, ov += adv4) {
          const float4 o = *ov;
          sacc = make_float4(sacc.x + o.x, sacc.y + o.y, sacc.z + o.z, sacc.w + o.w);
        }
        *a = sacc;
      }
    }
    for (Cursor2 c = walk_tw; !ola4 && c.y < yhi - ylo; c.next()) {
      const int yy = c.y, xx = c.x;
      const int Y = ylo + yy, ly = Y - oy;
      float* a = acc + size_t(Y % BH) * S.tw + xx;
      // blocks b0.. in ascending order; block b0+j holds column X at offset xo - j*step
      const int cm = colmap[xx], nblk = (cm >> 10) & 1023;
      const float* ov = ob + size_t(ly) * NB * OBW + size_t(cm & 1023) * OBW + (cm >> 20);
      float sacc = *a;
      for (int j = 0; j < nblk; ++j, ov += OBW - gx.step) sacc += *ov;
      *a = sacc;
    }
    __syncthreads();
    const int rlo = max(oy, Y0), rhi = min(by == by_hi ? Y0 + th : oy + gy.step, Y0 + th);
    for (Cursor2 c = walk_tw; c.y < rhi - rlo; c.next()) {
      const int yy = c.y, xx = c.x;
      const int Y = rlo + yy;
      float* a = acc + size_t(Y % BH) * S.tw + xx;
      J.dcov[size_t(Y) * gx.cover + X0 + xx] = *a;
      *a = 0.0f;
    }
  }
  __syncthreads();
  for (int i = tid; i < bins; i += nthr) J.partial[size_t(tile) * bins + i] = da_tile[i];
}

constexpr int kAdjointMaxPlanes = 32;
struct AdjointBatch {  // passed by value: no per-call uploads, capturable in graphs
  AdjointJob job[kAdjointMaxPlanes];
  float* gsrc[kAdjointMaxPlanes];
  long long gsrc_stride[kAdjointMaxPlanes];
  int n;
};

template <int BHC, int BWC>
__global__ void __launch_bounds__(256, 2) dft_adjoint_kernel(DevPlan P, AdjointShape S, AdjointBatch B) {
  extern __shared__ float smem[];
  const int tiles = S.tiles_x * S.tiles_y;
  adjoint_tile<BHC, BWC, 1>(P, B.job[blockIdx.x / tiles], S, blockIdx.x % tiles, smem);
}

template <int BHC, int BWC>
__global__ void __launch_bounds__(256, 2) fft3d_adjoint_kernel(DevPlan P, AdjointShape S, AdjointBatch B) {
  extern __shared__ float smem[];
  const int tiles = S.tiles_x * S.tiles_y;
  adjoint_tile<BHC, BWC, 0>(P, B.job[blockIdx.x / tiles], S, blockIdx.x % tiles, smem);
}

#ifdef NF_ADJOINT_AUX_KERNELS  // defined by the one unit that launches them (nf_api.cu)
// Source gradient: each source pixel gathers the cover positions that reflect onto
// it (single reflection per axis, ascending cover row then column) times the decode
// scale (255 for DFTTest, 1 for FFT3D).
__global__ void dft_adjoint_fold_kernel(DevPlan P, AdjointBatch B) {
  const AdjointJob& J = B.job[blockIdx.z];
  const DevAxis gx = P.gx, gy = P.gy;
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= gx.length || y >= gy.length) return;
  int cxs[3], cys[3], nx = 0, ny = 0;
  // cover c reflects to source j: c = off + j, or c = off - j (j >= 1), or
  // c = off + 2L - 2 - j (j <= L - 2); keep those inside the cover, ascending.
  auto axis = [](int j, const DevAxis& a, int* out, int& n) {
    const int c1 = a.offset - j, c0 = a.offset + j, c2 = a.offset + 2 * a.length - 2 - j;
    if (j >= 1 && c1 >= 0) out[n++] = c1;
    out[n++] = c0;
    if (j <= a.length - 2 && c2 < a.cover && c2 - a.offset >= a.length) out[n++] = c2;
  };
  axis(x, gx, cxs, nx);
  axis(y, gy, cys, ny);
  float s = 0.0f;
  for (int i = 0; i < ny; ++i)
    for (int j = 0; j < nx; ++j) s += J.dcov[size_t(cys[i]) * gx.cover + cxs[j]];
  float* row = reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(B.gsrc[blockIdx.z]) +
                                        ptrdiff_t(y) * B.gsrc_stride[blockIdx.z]);
  row[x] = s * P.dec_scale;
}

// Table gradient: sum of all tiles' partials of all planes. Block (32, 32): x = bin
// within a chunk of 32, y = residue class of the tile index; each thread sums its
// class in ascending tile order, then the 32 class sums are added in a fixed tree.
// The order never depends on timing, so the result is deterministic.
__global__ void __launch_bounds__(1024) dft_adjoint_reduce_kernel(const float* partial, int ntiles, int bins,
                                                                  float* out) {
  __shared__ float part[32][33];
  const int k = blockIdx.x * 32 + threadIdx.x;
  float s = 0.0f;
  if (k < bins)
    for (int t = threadIdx.y; t < ntiles; t += 32) s += partial[size_t(t) * bins + k];
  part[threadIdx.y][threadIdx.x] = s;
  __syncthreads();
  for (int w = 16; w > 0; w >>= 1) {
    if (threadIdx.y < w) part[threadIdx.y][threadIdx.x] += part[threadIdx.y + w][threadIdx.x];
    __syncthreads();
  }
  if (threadIdx.y == 0 && k < bins) out[k] = part[0][threadIdx.x];
}
#endif

} // namespace nfd
