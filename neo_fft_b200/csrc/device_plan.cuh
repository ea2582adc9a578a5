// Device-side plan descriptor and per-bin spectral arithmetic.
//
// DevPlan is passed by value to every tile kernel; its pointers reference the
// plan's immutable tables in device memory (uploaded once at creation). The
// per-bin functions restate the reference's scalar kernels operation by operation:
//   spectral_bin  — detail::spectral_prevalidated (src/kernels/scalar/spectral.cpp:5-53)
//   enhancement   — enhancement_gain (src/algorithms/fft3d_profile.cpp:69-81)
//   kalman_bin    — kalman_scalar (src/kernels/scalar/kalman.cpp:3-24)
#pragma once
#include "fft_core.cuh"

#include <cstddef>
#include <cstdint>

namespace nfd {

using nf::cf;
using nf::fadd;
using nf::fdiv;
using nf::fmul;
using nf::fsqrt;
using nf::fsub;

// Error bits OR-ed into DevPlan::err.
enum : int { kErrNonFinite = 1 };

struct DevAxis {
  int length, block, overlap, step, count, cover, offset;
};

struct DevSpectral {
  int type;  // -2 enhancement only, -1 FFT3D Wiener, 0..4 DFTTest ftype
  float a, b, low, high, exponent, floor;
  const float* primary;  // per-bin primary table, or nullptr for uniform a
  int enh;               // enhancement applied inside this call
  float sharpen, dehalo, ea, eb, ec;
  const float* sharpen_w;
  const float* halo_w;
  int emode;  // ftype 0 gain from the exponent: 0 the Wiener ratio, 1 its square root, 2 its power
};

enum StoreKind : int { kStoreU8 = 1, kStoreU16 = 2, kStoreF32 = 4 };

// FFT3D per-bin pipeline of the T=1 path (src/algorithms/plan.cpp:476-481).
enum Fft3dMode : int {
  kWienerFused = 0,    // uniform noise: Wiener with enhancement fused
  kWienerThenEnh = 1,  // table noise: Wiener, then enhancement on the result
  kEnhanceOnly = 2     // bt=-1 and Kalman render: enhancement only
};

struct DevPlan {
  int algo;  // 0 FFT3D, 1 DFTTest
  DevAxis gx, gy;
  int bh, bw, K, bins, T;
  int storage;  // input/output sample storage (1, 2, 4 bytes)
  float dec_base, dec_scale;
  const float *wxa, *wya, *wxs, *wys;  // FFT3D windows
  const float *h, *hsyn;               // DFTTest h and h*V
  const cf* grid;                      // degrid / zmean template or nullptr
  float mean_scale;
  DevSpectral filt;  // FFT3D Wiener (+fused enhancement) or DFTTest ftype
  DevSpectral enh;   // FFT3D stand-alone enhancement (type -2)
  int fft3d_mode;
  int codelet;                 // square 8/16/32 block: codelet networks
  const cf *twh, *tww, *twt;   // project twiddles for H, W and T
  float out_base, out_scale, out_peak;
  int center;  // DFTTest smode 0 (emit block centres)
  int* err;
  // FFT3D temporal (bt=2..5)
  const cf* tfwd;  // [T][T] forward temporal twiddles fwd[m][j]
  const cf* tinv;  // [T] inverse twiddles inv[c][m] for the centre slot
  float noise_uniform, noise_mult, lower;
  int kalman_fp64;
  float kalman_r0, kalman_ratio2;
  int raw_out;  // u8 output: store the unconverted accumulator as float (input of the dither pass)
};

NF_HD bool isfin(float v) {
#if defined(__CUDA_ARCH__)
  return isfinite(v);
#else
  return std::isfinite(v);
#endif
}

// enhancement_gain(q, k, e): sharpen S(q) and dehalo D(q), both on the residual
// power q (fft3d_profile.cpp:69-81).
NF_HD float enhancement_gain(float q, int k, const DevSpectral& e) {
  float s = 1.0f, d = 1.0f;
  if (e.sharpen != 0.0f && e.eb != 0.0f) {
    const float num = fmul(q, e.eb), den = fmul(fadd(q, e.ea), fadd(q, e.eb));
    const float strength = fmul(e.sharpen, e.sharpen_w[k]);
    s = fadd(1.0f, fmul(strength, fsqrt(fdiv(num, den))));
  }
  if (e.dehalo != 0.0f) {
    const float qc = fadd(q, e.ec);
    d = fdiv(qc, fadd(qc, fmul(fmul(e.dehalo, e.halo_w[k]), q)));
  }
  return fmul(s, d);
}

// Compile-time filter codes beyond the types: DFTTest ftype 0 with its exponent mode
// fixed as well (the Wiener ratio, its square root, its power), so the common ratio
// path carries no square-root or power code.
constexpr int kFt0Ratio = 10, kFt0Sqrt = 11, kFt0Pow = 12;

// One bin of spectral_prevalidated: residual against the scaled template, gain
// by type, optional enhancement, restore the template. Returns the new bin and
// flags non-finite intermediates through `bad`.
// FT >= 0 fixes the filter type at compile time (a DFTTest ftype: no enhancement;
// kFt0Ratio..kFt0Pow fix ftype 0's exponent mode too).
template <int FT = -3>
NF_HD cf spectral_bin(cf x, const cf* grid, int k, float scale, const DevSpectral& p, bool& bad) {
  constexpr int kType = FT >= kFt0Ratio ? 0 : FT;
  const float a = p.primary ? p.primary[k] : p.a;
  const float mr = grid ? fmul(scale, grid[k].r) : 0.0f;
  const float mi = grid ? fmul(scale, grid[k].i) : 0.0f;
  const float re = fsub(x.r, mr), im = fsub(x.i, mi);
  const float power = fadd(fmul(re, re), fmul(im, im));
  float gain = 0.0f;
  switch (kType >= -2 ? kType : p.type) {
    case -2:
      gain = 1.0f;
      break;
    case -1: {
      const float q = fadd(power, 1e-15f);
      const float g = fdiv(fsub(q, a), q);
      gain = g < p.floor ? p.floor : g;  // std::max(g, floor)
      break;
    }
    case 0: {
      const float r = fdiv(fsub(power, a), fadd(power, 1e-15f));
      const float wiener = r < 0.0f ? 0.0f : r;
      const int em = FT >= kFt0Ratio ? FT - kFt0Ratio : p.emode;
      if (em == 0) gain = wiener;
      else if (em == 1) gain = fsqrt(wiener);
      else gain = powf(wiener, p.exponent);
      break;
    }
    case 1:
      gain = power < a ? 0.0f : 1.0f;
      break;
    case 2:
      gain = a;
      break;
    case 3:
      gain = (power >= p.low && power <= p.high) ? a : p.b;
      break;
    case 4: {
      const float q = fadd(power, 1e-15f);
      const float num = fmul(q, p.high), den = fmul(fadd(q, p.low), fadd(q, p.high));
      gain = fmul(a, fsqrt(fdiv(num, den)));
      break;
    }
  }
  if (FT < 0 && p.enh) gain = fmul(gain, enhancement_gain(fadd(power, 1e-15f), k, p));
  const cf out = {fadd(fmul(gain, re), mr), fadd(fmul(gain, im), mi)};
  // The reference checks mr, mi, re, im, power, gain and both outputs. A non-finite mr,
  // re or gain always makes out.r non-finite (inf or NaN propagate through the product
  // and the sum; inf * 0 is NaN), and mi, im or gain out.i, so power and the two
  // outputs decide the same error.
  if (!isfin(power) || !isfin(out.r) || !isfin(out.i)) bad = true;
  return out;
}

// spectral_bin<kFt0Ratio> (DFTTest ftype 0, plain Wiener ratio) with its error test
// folded into one multiply-add: the gain is max((power - a)/(power + 1e-15), 0) with
// a finite table value a >= 0, so it lies in [0, 1] and each output, a point between
// the bin and the template term, is finite whenever the bin, the template term and the
// power are. A non-finite bin, template term, power or table value makes the gain NaN,
// and a NaN gain turns `guard` NaN (x * 0 is NaN for inf and NaN): the caller tests
// guard once instead of three compares per bin.
NF_HD cf ratio_bin(cf x, const cf* grid, int k, float scale, const DevSpectral& p, float& guard) {
  const float a = p.primary ? p.primary[k] : p.a;
  const float mr = grid ? fmul(scale, grid[k].r) : 0.0f;
  const float mi = grid ? fmul(scale, grid[k].i) : 0.0f;
  const float re = fsub(x.r, mr), im = fsub(x.i, mi);
  const float power = fadd(fmul(re, re), fmul(im, im));
  const float r = fdiv(fsub(power, a), fadd(power, 1e-15f));
  const float gain = r < 0.0f ? 0.0f : r;
  guard = nf::ffma(gain, 0.0f, guard);
  return {fadd(fmul(gain, re), mr), fadd(fmul(gain, im), mi)};
}

// One bin of kalman_scalar (src/kernels/scalar/kalman.cpp:3-24) in binary32, the
// reference's specified operation order. Returns false on a non-finite value.
NF_HD bool kalman_bin(cf x, cf& last, float& cov, float& proc, const float* pattern, int k, float uniform,
                      float ratio2) {
  const float r = pattern ? (pattern[k] < 1e-15f ? 1e-15f : pattern[k]) : uniform;
  const float threshold = fmul(r, ratio2);
  bool ok = isfin(r) && isfin(threshold) && isfin(x.r) && isfin(x.i) && isfin(last.r) && isfin(last.i) &&
            isfin(cov) && isfin(proc);
  const float dr = fsub(x.r, last.r), di = fsub(x.i, last.i);
  if ((!pattern && r == 0.0f) || fmul(dr, dr) > threshold || fmul(di, di) > threshold) {
    last = x;
    cov = proc = r;
    return ok;
  }
  const float sum = fadd(cov, proc);
  const float gain = fdiv(sum, fadd(sum, r));
  const float complement = fsub(1.0f, gain);
  const float nq = fmul(fmul(gain, gain), r), nc = fmul(complement, sum);
  const float nr = fadd(fmul(gain, x.r), fmul(complement, last.r));
  const float ni = fadd(fmul(gain, x.i), fmul(complement, last.i));
  ok = ok && isfin(sum) && isfin(gain) && isfin(nq) && isfin(nc) && isfin(nr) && isfin(ni);
  last = {nr, ni};
  cov = nc;
  proc = nq;
  return ok;
}

// Binary64 variance variant: C and Q are carried in binary64 and the gain and the
// estimate update are evaluated in binary64 (the long recursion accumulates no
// binary32 rounding in C/Q); the motion test keeps the binary32 order above.
NF_HD bool kalman_bin_fp64(cf x, cf& last, double& cov, double& proc, const float* pattern, int k, float uniform,
                           float ratio2) {
  const float r = pattern ? (pattern[k] < 1e-15f ? 1e-15f : pattern[k]) : uniform;
  const float threshold = fmul(r, ratio2);
  bool ok = isfin(r) && isfin(threshold) && isfin(x.r) && isfin(x.i) && isfin(last.r) && isfin(last.i);
  const float dr = fsub(x.r, last.r), di = fsub(x.i, last.i);
  if ((!pattern && r == 0.0f) || fmul(dr, dr) > threshold || fmul(di, di) > threshold) {
    last = x;
    cov = proc = double(r);
    return ok;
  }
  const double sum = cov + proc;
  const double gain = sum / (sum + double(r));
  const double complement = 1.0 - gain;
  proc = gain * gain * double(r);
  cov = complement * sum;
  last = {float(gain * double(x.r) + complement * double(last.r)), float(gain * double(x.i) + complement * double(last.i))};
  return ok && isfin(last.r) && isfin(last.i) && isfin(float(cov)) && isfin(float(proc));
}

} // namespace nfd
