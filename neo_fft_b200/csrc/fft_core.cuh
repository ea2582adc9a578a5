// FFT arithmetic shared by the sm_100a tile kernels and the host-side table builders.
//
// Every floating-point operation is spelled out with round-to-nearest intrinsics
// (device) or plain operators compiled with -ffp-contract=off (host), so the same
// source produces bit-identical results on both sides.
//
// Two families live here:
//
//  * Codelet-order transforms for 8, 16 and 32 points (fft8/fft16/fft32). The
//    neo-fft reference computes 8x8, 16x16 and 32x32 real 2-D FFTs with hand
//    written AVX2 codelets (src/spectral/codelets/fft8x8_avx2.cpp:42-138,
//    fft16x16_avx2.cpp:29-194, fft32x32_avx2.cpp:96-260; dispatched from
//    src/spectral/fft_backend.cpp:260-367). Parity with the reference's rounding
//    requires the same butterfly network, so these functions follow the codelets'
//    stage order, twiddle constants and fused multiply-adds step for step.
//
//  * A project mixed-radix decimation-in-time FFT for every other length (the
//    reference uses PocketFFT there, which is not available to restate). Factors
//    are taken outermost-first as 4,4,...,(2),3,...,5,..., then remaining primes by
//    direct DFT. Radix-3 and radix-5 butterflies use the same formulas as the
//    reference's temporal butterflies (src/spectral/fft_backend.cpp:396-420).
//
// Conventions (docs/knowledge/en/shared/fft-conventions.md): forward is
// unnormalised with exp(-2*pi*i*jk/N); inverse uses exp(+...) and the caller
// applies the 1/V scale once.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define NF_HD __host__ __device__ __forceinline__
#else
#define NF_HD inline
#endif

#if !defined(__CUDACC__)
#include <cmath>
#endif

namespace nf {

// 8-byte aligned, so a complex value moves with one 64-bit access: consecutive
// threads touching consecutive values hit distinct shared-memory banks.
struct alignas(8) cf {
  float r, i;
};

// Round-to-nearest float primitives that are never contracted.
NF_HD float fadd(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fadd_rn(a, b);
#else
  return a + b;
#endif
}
NF_HD float fsub(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fsub_rn(a, b);
#else
  return a - b;
#endif
}
NF_HD float fmul(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fmul_rn(a, b);
#else
  return a * b;
#endif
}
NF_HD float ffma(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
  return __fmaf_rn(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}
NF_HD float fdiv(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fdiv_rn(a, b);
#else
  return a / b;
#endif
}
NF_HD float fsqrt(float a) {
#if defined(__CUDA_ARCH__)
  return __fsqrt_rn(a);
#else
  return std::sqrt(a);
#endif
}

NF_HD cf cadd(cf a, cf b) { return {fadd(a.r, b.r), fadd(a.i, b.i)}; }
NF_HD cf csub(cf a, cf b) { return {fsub(a.r, b.r), fsub(a.i, b.i)}; }

// ---------------------------------------------------------------------------
// Codelet-order transforms (8/16/32 points).
// ---------------------------------------------------------------------------

// cos/sin(k*pi/8) and cos/sin(k*pi/16) rounded to binary32: the codelets' tables
// (fft16x16_avx2.cpp:12-24, fft32x32_avx2.cpp:12-46), which evaluate cos/sin of
// float(pi)*k/8 and float(pi)*k/16. Literal values; a host test checks them against
// the same expressions evaluated by the host compiler.
NF_HD float tw16r(int k) {
  const float t[8] = {0x1p+0f,         0x1.d906bcp-1f, 0x1.6a09e6p-1f,  0x1.87de2ap-2f,
                      -0x1.777a5cp-25f, -0x1.87de3p-2f, -0x1.6a09e6p-1f, -0x1.d906cp-1f};
  return t[k];
}
NF_HD float tw16i(int k) {
  const float t[8] = {0x0p+0f, 0x1.87de2cp-2f, 0x1.6a09e6p-1f, 0x1.d906bcp-1f,
                      0x1p+0f, 0x1.d906bcp-1f, 0x1.6a09e6p-1f, 0x1.87de2p-2f};
  return t[k];
}
NF_HD float tw32r(int k) {
  const float t[16] = {0x1p+0f,         0x1.f6297cp-1f,  0x1.d906bcp-1f,  0x1.a9b662p-1f,
                       0x1.6a09e6p-1f,  0x1.1c73b2p-1f,  0x1.87de2ap-2f,  0x1.8f8b78p-3f,
                       -0x1.777a5cp-25f, -0x1.8f8b84p-3f, -0x1.87de3p-2f, -0x1.1c73b8p-1f,
                       -0x1.6a09e6p-1f, -0x1.a9b664p-1f, -0x1.d906cp-1f, -0x1.f6297ep-1f};
  return t[k];
}
NF_HD float tw32i(int k) {
  const float t[16] = {0x0p+0f,        0x1.8f8b84p-3f, 0x1.87de2cp-2f, 0x1.1c73b4p-1f,
                       0x1.6a09e6p-1f, 0x1.a9b664p-1f, 0x1.d906bcp-1f, 0x1.f6297ep-1f,
                       0x1p+0f,        0x1.f6297cp-1f, 0x1.d906bcp-1f, 0x1.a9b66p-1f,
                       0x1.6a09e6p-1f, 0x1.1c73b2p-1f, 0x1.87de2p-2f,  0x1.8f8b82p-3f};
  return t[k];
}

// (in * w) with w = (wr, FORWARD ? -wi : wi), using the codelets' fused form:
// re = fma(in.r, wr, -(in.i*wi)), im = fma(in.r, wi, in.i*wr).
template <bool FORWARD>
NF_HD cf cmul_codelet(cf in, float wr, float wi_raw) {
  const float wi = FORWARD ? -wi_raw : wi_raw;
  return {ffma(in.r, wr, -fmul(in.i, wi)), ffma(in.r, wi, fmul(in.i, wr))};
}
// Multiplication by -j (forward) or +j (inverse); the negation is 0-x.
template <bool FORWARD>
NF_HD cf mul_j(cf z) {
  return FORWARD ? cf{z.i, fsub(0.0f, z.r)} : cf{fsub(0.0f, z.i), z.r};
}
NF_HD void bfly2(cf& x, cf& y) {
  const cf u = x, v = y;
  x = cadd(u, v);
  y = csub(u, v);
}

// 8-point transform, codelet order (fft8x8_avx2.cpp:42-138). The codelets are
// built with -ffp-contract=fast (CMakeLists.txt:91-101), which fuses the W8^1 and
// W8^3 products by sqrt(1/2) into the following butterfly's sum and difference;
// the fused form is written out here (checked bit-exact against the codelet).
template <bool FORWARD>
NF_HD void fft8(cf* v) {
  const float s = 0.70710678118654752440f;
  cf a0 = v[0], a1 = v[4], a2 = v[2], a3 = v[6], a4 = v[1], a5 = v[5], a6 = v[3], a7 = v[7];
  bfly2(a0, a1);
  bfly2(a2, a3);
  bfly2(a4, a5);
  bfly2(a6, a7);
  bfly2(a0, a2);
  bfly2(a4, a6);
  a3 = mul_j<FORWARD>(a3);
  a7 = mul_j<FORWARD>(a7);
  bfly2(a1, a3);
  bfly2(a5, a7);
  bfly2(a0, a4);
  {
    // a5*W8 then the (a1, a5) butterfly; the product is fused into both sums.
    const cf u = a5, x = a1;
    const float tr = FORWARD ? fadd(u.r, u.i) : fsub(u.r, u.i);
    const float ti = FORWARD ? fsub(u.i, u.r) : fadd(u.i, u.r);
    a1 = {ffma(s, tr, x.r), ffma(s, ti, x.i)};
    a5 = {ffma(-s, tr, x.r), ffma(-s, ti, x.i)};
  }
  a6 = mul_j<FORWARD>(a6);
  bfly2(a2, a6);
  {
    // a7*W8^3 then the (a3, a7) butterfly, fused the same way.
    const cf u = a7, x = a3;
    const float tr = FORWARD ? fsub(u.i, u.r) : fsub(fsub(0.0f, u.r), u.i);
    const float ti = FORWARD ? fsub(fsub(0.0f, u.r), u.i) : fsub(u.r, u.i);
    a3 = {ffma(s, tr, x.r), ffma(s, ti, x.i)};
    a7 = {ffma(-s, tr, x.r), ffma(-s, ti, x.i)};
  }
  v[0] = a0; v[1] = a1; v[2] = a2; v[3] = a3; v[4] = a4; v[5] = a5; v[6] = a6; v[7] = a7;
}

// 16-point transform, codelet order (fft16x16_avx2.cpp:29-194): bit-reversed
// load, radix-2 stages of span 2, 4, 8 and 16 with the W16 table.
template <bool FORWARD>
NF_HD void fft16(cf* v) {
  cf a[16] = {v[0], v[8], v[4], v[12], v[2], v[10], v[6], v[14], v[1], v[9], v[5], v[13], v[3], v[11], v[7], v[15]};
#pragma unroll
  for (int k = 0; k < 16; k += 2) bfly2(a[k], a[k + 1]);
  // span 4: (x0,x2) plain, (x1, j*x3)
#pragma unroll
  for (int g = 0; g < 16; g += 4) {
    bfly2(a[g], a[g + 2]);
    const cf v1 = mul_j<FORWARD>(a[g + 3]);
    const cf u1 = a[g + 1];
    a[g + 1] = cadd(u1, v1);
    a[g + 3] = csub(u1, v1);
  }
  // span 8: (x0,x4) plain, (x1, W2*x5), (x2, j*x6), (x3, W6*x7)
#pragma unroll
  for (int g = 0; g < 16; g += 8) {
    bfly2(a[g], a[g + 4]);
    {
      const cf v1 = cmul_codelet<FORWARD>(a[g + 5], tw16r(2), tw16i(2));
      const cf u1 = a[g + 1];
      a[g + 1] = cadd(u1, v1);
      a[g + 5] = csub(u1, v1);
    }
    {
      const cf v2 = mul_j<FORWARD>(a[g + 6]);
      const cf u2 = a[g + 2];
      a[g + 2] = cadd(u2, v2);
      a[g + 6] = csub(u2, v2);
    }
    {
      const cf v3 = cmul_codelet<FORWARD>(a[g + 7], tw16r(6), tw16i(6));
      const cf u3 = a[g + 3];
      a[g + 3] = cadd(u3, v3);
      a[g + 7] = csub(u3, v3);
    }
  }
  // span 16: (x0,x8) plain, (xk, Wk*x(k+8)) with x12 using j.
  bfly2(a[0], a[8]);
#pragma unroll
  for (int k = 1; k < 8; ++k) {
    const cf vk = (k == 4) ? mul_j<FORWARD>(a[12]) : cmul_codelet<FORWARD>(a[k + 8], tw16r(k), tw16i(k));
    const cf uk = a[k];
    a[k] = cadd(uk, vk);
    a[k + 8] = csub(uk, vk);
  }
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = a[k];
}

// 32-point transform, codelet order (fft32x32_avx2.cpp:220-240): two 16-point
// transforms of the even and odd samples combined with the W32 table.
template <bool FORWARD>
NF_HD void fft32(cf* v) {
  cf e[16], o[16];
#pragma unroll
  for (int m = 0; m < 16; ++m) {
    e[m] = v[2 * m];
    o[m] = v[2 * m + 1];
  }
  fft16<FORWARD>(e);
  fft16<FORWARD>(o);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const cf w = cmul_codelet<FORWARD>(o[k], tw32r(k), tw32i(k));
    v[k] = cadd(e[k], w);
    v[k + 16] = csub(e[k], w);
  }
}

// Real-row forms of the 16-point codelet transform. The codelet transforms a real
// row as complex data with zero imaginary parts and inverts a half spectrum after
// mirroring it into a full conjugate-symmetric array (fft16x16_avx2.cpp:239-262 and
// 400-430). On such data many of fft16's operations add or subtract an exact zero,
// negate a value (0 - x), or recompute another operation's result with its sign or
// its real and imaginary parts exchanged: with c = cos(pi/4) = sin(pi/4) in the
// table, W16^6 * conj(z) = (-re, im) of W16^2 * z, and round(-a) = -round(a) under
// round-to-nearest. These forms keep every other operation of fft16, in its order
// and with its rounding, and skip those. Each result equals fft16's: an exactly
// zero result may carry the other sign, and nothing else differs (a signed zero
// changes no later nonzero value: every divisor in the pipeline is positive).

// Bins 0..8 (at `stride`) of the forward transform of 16 real samples; the DC and
// Nyquist imaginary parts are 0, as the codelet stores them. ALL: bins 9..15 too (the
// halves of the 32-point transform).
template <bool ALL = false>
NF_HD void fft16_real_forward(const float* x, cf* X, int stride) {
  // span 2 on the bit-reversed pairs
  float s[16];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int p = ((j & 1) << 2) | (j & 2) | ((j & 4) >> 2);  // bit-reversed j (3 bits)
    s[2 * j] = fadd(x[p], x[p + 8]);
    s[2 * j + 1] = fsub(x[p], x[p + 8]);
  }
  // span 4, group g (positions 4g..4g+3): (R0, (p,-q), R2, (p,q)) with p = s[4g+1],
  // q = s[4g+3]; the j-rotation of the real q only moves it into the imaginary part.
  float R0[4], R2[4];
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    R0[g] = fadd(s[4 * g], s[4 * g + 2]);
    R2[g] = fsub(s[4 * g], s[4 * g + 2]);
  }
  // span 8, half h (groups 2h and 2h+1, positions 8h..8h+7):
  // (e0, c1, (R2, -R2'), c3, e4, conj(c3), (R2, R2'), conj(c1)).
  float e0[2], e4[2];
  cf c1[2], c3[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int g0 = 2 * h, g1 = 2 * h + 1;
    e0[h] = fadd(R0[g0], R0[g1]);
    e4[h] = fsub(R0[g0], R0[g1]);
    const float p = s[4 * g0 + 1], q = s[4 * g0 + 3];
    const cf v1 = cmul_codelet<true>(cf{s[4 * g1 + 1], -s[4 * g1 + 3]}, tw16r(2), tw16i(2));
    c1[h] = {fadd(p, v1.r), fadd(-q, v1.i)};
    c3[h] = {fsub(p, v1.r), fadd(q, v1.i)};  // W16^6 * (p',q') = (-v1.r, v1.i)
  }
  // span 16: X[k] = A[k] + W16^k B[k] for the two halves A and B.
  const float ra = R2[0], rb = R2[1], ra2 = R2[2], rb2 = R2[3];
  X[0] = {fadd(e0[0], e0[1]), 0.0f};
  X[8 * stride] = {fsub(e0[0], e0[1]), 0.0f};
  const cf t1 = cmul_codelet<true>(c1[1], tw16r(1), tw16i(1));
  const cf t2 = cmul_codelet<true>(cf{ra2, -rb2}, tw16r(2), tw16i(2));
  const cf t3 = cmul_codelet<true>(c3[1], tw16r(3), tw16i(3));
  const cf t5 = cmul_codelet<true>(cf{c3[1].r, -c3[1].i}, tw16r(5), tw16i(5));
  const cf t7 = cmul_codelet<true>(cf{c1[1].r, -c1[1].i}, tw16r(7), tw16i(7));
  const cf a5 = {c3[0].r, -c3[0].i}, a7 = {c1[0].r, -c1[0].i};
  X[stride] = cadd(c1[0], t1);
  X[2 * stride] = {fadd(ra, t2.r), fadd(-rb, t2.i)};
  X[3 * stride] = cadd(c3[0], t3);
  X[4 * stride] = {e4[0], -e4[1]};
  X[5 * stride] = cadd(a5, t5);
  X[6 * stride] = {fsub(ra, t2.r), fadd(rb, t2.i)};  // W16^6 * conj(B2) = (-t2.r, t2.i)
  X[7 * stride] = cadd(a7, t7);
  if constexpr (ALL) {  // X[k + 8] = A[k] - W16^k B[k]
    X[9 * stride] = csub(c1[0], t1);
    X[10 * stride] = {fsub(ra, t2.r), fsub(-rb, t2.i)};
    X[11 * stride] = csub(c3[0], t3);
    X[12 * stride] = {e4[0], e4[1]};
    X[13 * stride] = csub(a5, t5);
    X[14 * stride] = {fadd(ra, t2.r), fsub(rb, t2.i)};
    X[15 * stride] = csub(a7, t7);
  }
}

// Inverse of one real row from bins 0..8 (at `stride`): the 16 real outputs of fft16
// over the mirrored half spectrum, times fct (SCALE) or unscaled (the even half of the
// 32-point inverse). The imaginary parts of the DC and Nyquist bins reach only
// imaginary outputs and are not read.
template <bool SCALE = true>
NF_HD void fft16_real_inverse(const cf* Y, int stride, float fct, float* out) {
  const cf y0 = Y[0], y1 = Y[stride], y2 = Y[2 * stride], y3 = Y[3 * stride], y4 = Y[4 * stride],
           y5 = Y[5 * stride], y6 = Y[6 * stride], y7 = Y[7 * stride], y8 = Y[8 * stride];
  // span 2 over (Y0,Y8) (Y4,~Y4) (Y2,~Y6) (Y6,~Y2) (Y1,~Y7) (Y5,~Y3) (Y3,~Y5) (Y7,~Y1)
  const float s0 = fadd(y0.r, y8.r), s1 = fsub(y0.r, y8.r);
  const float y4r2 = fadd(y4.r, y4.r), y4i2 = fadd(y4.i, y4.i);
  const cf P = {fadd(y2.r, y6.r), fsub(y2.i, y6.i)}, M = {fsub(y2.r, y6.r), fadd(y2.i, y6.i)};
  const cf Q = {fadd(y1.r, y7.r), fsub(y1.i, y7.i)}, N = {fsub(y1.r, y7.r), fadd(y1.i, y7.i)};
  const cf S = {fadd(y5.r, y3.r), fsub(y5.i, y3.i)}, T = {fsub(y5.r, y3.r), fadd(y5.i, y3.i)};
  // span 4. Group 0: real parts only (these positions are never rotated later).
  const float e0 = fadd(s0, y4r2), e2 = fsub(s0, y4r2), e1 = fsub(s1, y4i2), e3 = fadd(s1, y4i2);
  // group 1: (2P.r, 0), (D, -D), (0, 2P.i), (Sg, Sg)
  const float p2r = fadd(P.r, P.r), p2i = fadd(P.i, P.i);
  const float D = fsub(M.r, M.i), Sg = fadd(M.r, M.i);
  // group 2; group 3 is (~q8, (-q9.i, -q9.r), (-q10.r, q10.i), (q11.i, q11.r))
  const cf q8 = cadd(Q, S), q10 = csub(Q, S);
  const cf q9 = {fsub(N.r, T.i), fadd(N.i, T.r)}, q11 = {fadd(N.r, T.i), fsub(N.i, T.r)};
  // span 8, half 0 (real parts)
  const float b0 = fadd(e0, p2r), b4 = fsub(e0, p2r);
  const float v1r = ffma(D, tw16r(2), fmul(D, tw16i(2)));
  const float b1 = fadd(e1, v1r), b5 = fsub(e1, v1r);
  const float b2 = fsub(e2, p2i), b6 = fadd(e2, p2i);
  const float v3r = ffma(Sg, tw16r(6), -fmul(Sg, tw16i(6)));
  const float b3 = fadd(e3, v3r), b7 = fsub(e3, v3r);
  // span 8, half 1: f0 = (2 q8.r, 0), f4 = (0, 2 q8.i), f2 = (D2, -D2), f6 = (S2, S2)
  const float f0r = fadd(q8.r, q8.r), f4i = fadd(q8.i, q8.i);
  const cf w1 = cmul_codelet<false>(cf{-q9.i, -q9.r}, tw16r(2), tw16i(2));
  const cf f1 = cadd(q9, w1), f5 = csub(q9, w1);
  const float D2 = fsub(q10.r, q10.i), S2 = fadd(q10.r, q10.i);
  const cf w3 = cmul_codelet<false>(cf{q11.i, q11.r}, tw16r(6), tw16i(6));
  const cf f3 = cadd(q11, w3), f7 = csub(q11, w3);
  // span 16, real parts: x[k] = b[k] + re(W16^k f[k]), x[k+8] = b[k] - re(W16^k f[k])
  auto rot = [](cf f, float wr, float wi) { return ffma(f.r, wr, -fmul(f.i, wi)); };
  const float t1 = rot(f1, tw16r(1), tw16i(1)), t3 = rot(f3, tw16r(3), tw16i(3));
  const float t5 = rot(f5, tw16r(5), tw16i(5)), t7 = rot(f7, tw16r(7), tw16i(7));
  const float t2 = ffma(D2, tw16r(2), fmul(D2, tw16i(2)));
  const float t6 = ffma(S2, tw16r(6), -fmul(S2, tw16i(6)));
  auto put = [fct](float v) { return SCALE ? fmul(v, fct) : v; };
  out[0] = put(fadd(b0, f0r));
  out[8] = put(fsub(b0, f0r));
  out[1] = put(fadd(b1, t1));
  out[9] = put(fsub(b1, t1));
  out[2] = put(fadd(b2, t2));
  out[10] = put(fsub(b2, t2));
  out[3] = put(fadd(b3, t3));
  out[11] = put(fsub(b3, t3));
  out[4] = put(fsub(b4, f4i));
  out[12] = put(fadd(b4, f4i));
  out[5] = put(fadd(b5, t5));
  out[13] = put(fsub(b5, t5));
  out[6] = put(fadd(b6, t6));
  out[14] = put(fsub(b6, t6));
  out[7] = put(fadd(b7, t7));
  out[15] = put(fsub(b7, t7));
}

// Real-row forms of the 32-point codelet transform, on the same terms as the 16-point
// ones. Forward: fft32's even and odd halves of a real row are real 16-point
// transforms (fft16_real_forward<true>), combined with the W32 table as fft32 does; the
// DC term's twiddle is (1, 0) and W32^8 multiplies a real value. Bins 0..16 at
// `stride`, the Nyquist imaginary part 0.
NF_HD void fft32_real_forward(const float* x, cf* X, int stride) {
  float xe[16], xo[16];
#pragma unroll
  for (int m = 0; m < 16; ++m) {
    xe[m] = x[2 * m];
    xo[m] = x[2 * m + 1];
  }
  cf E[16], O[16];
  fft16_real_forward<true>(xe, E, 1);
  fft16_real_forward<true>(xo, O, 1);
  // W32^0 * O[0] = (O0, O0 * -0 + 0): the imaginary part is +0, or NaN for inf and NaN
  X[0] = {fadd(E[0].r, O[0].r), ffma(O[0].r, -0.0f, 0.0f)};
  X[16 * stride] = {fsub(E[0].r, O[0].r), 0.0f};
#pragma unroll
  for (int k = 1; k < 16; ++k) {
    if (k == 8) {  // O[8] is real: W32^8 * O[8] = (O8 * cos, -O8)
      X[8 * stride] = {fadd(E[8].r, fmul(O[8].r, tw32r(8))), -O[8].r};
    } else {
      X[k * stride] = cadd(E[k], cmul_codelet<true>(O[k], tw32r(k), tw32i(k)));
    }
  }
}

// Inverse of one real row from bins 0..16 (at `stride`), times fct. fft32's even half of
// the mirrored spectrum is itself a mirrored 16-point half spectrum (bins 0, 2, .., 16),
// whose real outputs fft16_real_inverse gives; the odd half is transformed as fft32 does,
// and only the real parts of its W32 products are formed.
NF_HD void fft32_real_inverse(const cf* Y, int stride, float fct, float* out) {
  float ev[16];
  fft16_real_inverse<false>(Y, 2 * stride, 1.0f, ev);
  cf o[16];
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    const cf y = Y[(2 * m + 1) * stride];
    o[m] = y;
    o[15 - m] = {y.r, -y.i};
  }
  fft16<false>(o);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const float t = ffma(o[k].r, tw32r(k), -fmul(o[k].i, tw32i(k)));
    out[k] = fmul(fadd(ev[k], t), fct);
    out[k + 16] = fmul(fsub(ev[k], t), fct);
  }
}

// ---------------------------------------------------------------------------
// Project mixed-radix DIT transform for arbitrary lengths.
// ---------------------------------------------------------------------------

// Twiddle table entry w_N^m = (cos(2*pi*m/N), -sin(2*pi*m/N)) for the forward
// direction, evaluated in binary64 and rounded once to binary32. The inverse uses
// the conjugate. Tables are built on the host and copied to the device verbatim.
NF_HD cf cmul_plain(cf a, cf w) {
  return {fsub(fmul(a.r, w.r), fmul(a.i, w.i)), fadd(fmul(a.r, w.i), fmul(a.i, w.r))};
}
template <bool FORWARD>
NF_HD cf rot_j(cf z) {
  // forward: multiply by -j; inverse: by +j.
  return FORWARD ? cf{z.i, -z.r} : cf{-z.i, z.r};
}

// Radix-3/5 butterflies on t[0..r-1] (in place). Formulas follow the reference's
// temporal butterflies (fft_backend.cpp:400-419).
template <bool FORWARD>
NF_HD void radix3(cf* t) {
  const float s60 = 0.86602540378443864676f;
  const cf sum = cadd(t[1], t[2]), diff = csub(t[1], t[2]);
  const cf center = csub(t[0], cf{fmul(sum.r, 0.5f), fmul(sum.i, 0.5f)});
  const cf side = rot_j<FORWARD>(cf{fmul(diff.r, s60), fmul(diff.i, s60)});
  t[0] = cadd(t[0], sum);
  t[1] = cadd(center, side);
  t[2] = csub(center, side);
}
template <bool FORWARD>
NF_HD void radix5(cf* v) {
  const float c1 = 0.30901699437494742410f, c2 = 0.80901699437494742410f;
  const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;
  const cf a = cadd(v[1], v[4]), b = cadd(v[2], v[3]), c = csub(v[1], v[4]), d = csub(v[2], v[3]);
  const cf base1 = csub(cadd(v[0], cf{fmul(a.r, c1), fmul(a.i, c1)}), cf{fmul(b.r, c2), fmul(b.i, c2)});
  const cf base2 = cadd(csub(v[0], cf{fmul(a.r, c2), fmul(a.i, c2)}), cf{fmul(b.r, c1), fmul(b.i, c1)});
  const cf side1 = rot_j<FORWARD>(cadd(cf{fmul(c.r, s1), fmul(c.i, s1)}, cf{fmul(d.r, s2), fmul(d.i, s2)}));
  const cf side2 = rot_j<FORWARD>(csub(cf{fmul(c.r, s2), fmul(c.i, s2)}, cf{fmul(d.r, s1), fmul(d.i, s1)}));
  const cf v0 = cadd(cadd(v[0], a), b);
  v[0] = v0;
  v[1] = cadd(base1, side1);
  v[4] = csub(base1, side1);
  v[2] = cadd(base2, side2);
  v[3] = csub(base2, side2);
}
template <bool FORWARD>
NF_HD void radix4(cf* t) {
  const cf s02 = cadd(t[0], t[2]), d02 = csub(t[0], t[2]);
  const cf s13 = cadd(t[1], t[3]), d13 = rot_j<FORWARD>(csub(t[1], t[3]));
  t[0] = cadd(s02, s13);
  t[2] = csub(s02, s13);
  t[1] = cadd(d02, d13);
  t[3] = csub(d02, d13);
}

// ---------------------------------------------------------------------------
// Factorisation and the iterative DIT driver.
//
// Definition (recursive form): a length-N transform with outermost radix r and
// M = N/r computes r length-M transforms of x[j::r] (j = 0..r-1), then for each
// k1 < M multiplies sub_j[k1] by w_N^(j*k1) (skipped when j*k1 == 0) and applies a
// radix-r butterfly, writing X[k1 + M*q]. The iterative form below performs the
// same butterflies (digit-reversed load, innermost level first), so its rounding
// is identical. Twiddles for every level come from the length-N table:
// w_n^e = table[e * (N/n)].
// ---------------------------------------------------------------------------
constexpr int kMaxFactors = 16;
struct Factors {
  int count;
  int r[kMaxFactors];
};
NF_HD constexpr int pick_radix(int n) {
  if (n % 4 == 0) return 4;
  if (n % 2 == 0) return 2;
  if (n % 3 == 0) return 3;
  if (n % 5 == 0) return 5;
  for (int p = 7; p * p <= n; p += 2)
    if (n % p == 0) return p;
  return n;
}
// Outermost factor first.
NF_HD constexpr Factors factorize(int n) {
  Factors f{0, {}};
  while (n > 1 && f.count < kMaxFactors) {
    const int r = pick_radix(n);
    f.r[f.count++] = r;
    n /= r;
  }
  return f;
}

// Table of w_N^m for one length, m = 0..N-1 (forward sign).
struct TwiddleView {
  const cf* w;  // w[m] = exp(-2*pi*i*m/N)
  int n;
};

// Direct radix-p DFT on t[0..p-1] using the length-p twiddles embedded in a
// length-N table (stride N/p). Sum order is j = 0..p-1.
template <bool FORWARD>
NF_HD void radix_direct(cf* t, int p, TwiddleView tw, cf* scratch) {
  const int stride = tw.n / p;
  for (int q = 0; q < p; ++q) {
    cf acc = t[0];
    for (int j = 1; j < p; ++j) {
      cf w = tw.w[((j * q) % p) * stride];
      if (!FORWARD) w.i = -w.i;
      acc = cadd(acc, cmul_plain(t[j], w));
    }
    scratch[q] = acc;
  }
  for (int q = 0; q < p; ++q) t[q] = scratch[q];
}

template <bool FORWARD>
NF_HD void butterfly(cf* t, int r, const cf* table, int n_top, cf* scratch) {
  if (r == 2) {
    bfly2(t[0], t[1]);
  } else if (r == 3) {
    radix3<FORWARD>(t);
  } else if (r == 4) {
    radix4<FORWARD>(t);
  } else if (r == 5) {
    radix5<FORWARD>(t);
  } else {
    radix_direct<FORWARD>(t, r, TwiddleView{table, n_top}, scratch);
  }
}

// Compile-time form: constexpr factorisation and digit-reversal table, one
// template instance per level; every index is a constant, so the transform is
// fully unrolled into registers.
template <int N>
struct DigitReversal {
  int v[N];
  NF_HD constexpr DigitReversal() : v() {
    const Factors f = factorize(N);
    for (int p = 0; p < N; ++p) {
      int rem = p, m = N, s = 1, idx = 0;
      for (int l = 0; l < f.count; ++l) {
        m /= f.r[l];
        const int j = rem / m;
        rem -= j * m;
        idx += j * s;
        s *= f.r[l];
      }
      v[p] = idx;
    }
  }
};

template <bool FORWARD, int R>
NF_HD void butterfly_ct(cf* t, const cf* table, int n_top) {
  if constexpr (R == 2) {
    bfly2(t[0], t[1]);
  } else if constexpr (R == 3) {
    radix3<FORWARD>(t);
  } else if constexpr (R == 4) {
    radix4<FORWARD>(t);
  } else if constexpr (R == 5) {
    radix5<FORWARD>(t);
  } else {
    cf scratch[R];
    const int stride = n_top / R;
#pragma unroll
    for (int q = 0; q < R; ++q) {
      cf acc = t[0];
#pragma unroll
      for (int j = 1; j < R; ++j) {
        cf w = table[((j * q) % R) * stride];
        if (!FORWARD) w.i = -w.i;
        acc = cadd(acc, cmul_plain(t[j], w));
      }
      scratch[q] = acc;
    }
#pragma unroll
    for (int q = 0; q < R; ++q) t[q] = scratch[q];
  }
}

template <bool FORWARD, int N, int LEV, int INNER>
NF_HD void ct_level(cf* a, const cf* table) {
  constexpr Factors F = factorize(N);
  constexpr int R = F.r[LEV];
  constexpr int LEN = R * INNER;
  constexpr int STEP = N / LEN;
#pragma unroll
  for (int base = 0; base < N; base += LEN) {
#pragma unroll
    for (int k1 = 0; k1 < INNER; ++k1) {
      cf t[R];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        cf v = a[base + j * INNER + k1];
        if (j * k1 != 0) {
          cf w = table[j * k1 * STEP];
          if (!FORWARD) w.i = -w.i;
          v = cmul_plain(v, w);
        }
        t[j] = v;
      }
      butterfly_ct<FORWARD, R>(t, table, N);
#pragma unroll
      for (int q = 0; q < R; ++q) a[base + k1 + INNER * q] = t[q];
    }
  }
  if constexpr (LEV > 0) ct_level<FORWARD, N, LEV - 1, LEN>(a, table);
}

template <bool FORWARD, int N>
NF_HD void fft_ct(cf* a, const cf* table) {
  if constexpr (N > 1) {
    constexpr DigitReversal<N> perm{};
    constexpr Factors F = factorize(N);
    cf src[N];
#pragma unroll
    for (int p = 0; p < N; ++p) src[p] = a[p];
#pragma unroll
    for (int p = 0; p < N; ++p) a[p] = src[perm.v[p]];
    ct_level<FORWARD, N, F.count - 1, 1>(a, table);
  }
}

// ---------------------------------------------------------------------------
// Team form of fft_ct<N>: the transform shared by T = F.r[0] lanes (the outermost
// radix), each holding M = N / T elements in registers instead of N.
//
// After the digit-reversed load, every level but the outermost combines elements inside
// one run of M consecutive positions (its groups have LEN <= M elements and start at
// multiples of LEN), so lane t runs those levels on positions [t*M, t*M + M) with the
// same butterflies, twiddles and operation order as fft_ct. The digit-reversed input of
// position t*M + i is element t + off(i) (the outermost digit is the lowest one of the
// input index), so each lane gathers its run directly. The outermost level's butterfly
// k1 takes run position k1 of every lane and writes positions k1 + M*q; lane t computes
// the butterflies k1 = t, t + T, ... after the runs have been exchanged through memory
// the caller provides. Results are bit-identical to fft_ct<N>.
// ---------------------------------------------------------------------------
template <bool FORWARD, int N, int LEV, int INNER, int EXTENT>
NF_HD void ct_level_run(cf* a, const cf* table) {
  constexpr Factors F = factorize(N);
  constexpr int R = F.r[LEV];
  constexpr int LEN = R * INNER;
  constexpr int STEP = N / LEN;
  static_assert(EXTENT % LEN == 0, "inner levels must stay inside a run");
#pragma unroll
  for (int base = 0; base < EXTENT; base += LEN) {
#pragma unroll
    for (int k1 = 0; k1 < INNER; ++k1) {
      cf t[R];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        cf v = a[base + j * INNER + k1];
        if (j * k1 != 0) {
          cf w = table[j * k1 * STEP];
          if (!FORWARD) w.i = -w.i;
          v = cmul_plain(v, w);
        }
        t[j] = v;
      }
      butterfly_ct<FORWARD, R>(t, table, N);
#pragma unroll
      for (int q = 0; q < R; ++q) a[base + k1 + INNER * q] = t[q];
    }
  }
  if constexpr (LEV > 1) ct_level_run<FORWARD, N, LEV - 1, LEN, EXTENT>(a, table);
}

template <bool FORWARD, int N>
struct TeamFFT {
  static constexpr Factors F = factorize(N);
  static constexpr int T = F.r[0];  // lanes of a team
  static constexpr int M = N / T;   // elements per lane
  static_assert(F.count >= 2 && M % T == 0, "team transforms need M = N/T divisible by T");

  // The lane's run after every level but the outermost: local[i] = position t*M + i, whose
  // digit-reversed input is element t + perm[i].
  template <class Load>
  NF_HD static void run(int t, cf* local, const cf* table, Load&& load) {
    constexpr DigitReversal<N> perm{};
#pragma unroll
    for (int i = 0; i < M; ++i) local[i] = load(t + perm.v[i]);
    ct_level_run<FORWARD, N, F.count - 1, 1, M>(local, table);
  }
  // Outermost level: butterflies k1 = t + T*m; read(j, i) returns element i of lane j's
  // run (position j*M + i of the exchanged runs), write(x, v) receives output element x.
  template <class Read, class Write>
  NF_HD static void outer(int t, const cf* table, Read&& read, Write&& write) {
#pragma unroll
    for (int m = 0; m < M / T; ++m) {
      const int k1 = t + T * m;
      cf v[T];
#pragma unroll
      for (int j = 0; j < T; ++j) {
        v[j] = read(j, k1);
        if (j * k1 != 0) {
          cf w = table[j * k1];
          if (!FORWARD) w.i = -w.i;
          v[j] = cmul_plain(v[j], w);
        }
      }
      butterfly_ct<FORWARD, T>(v, table, N);
#pragma unroll
      for (int q = 0; q < T; ++q) write(k1 + M * q, v[q]);
    }
  }
};

// In-place project transform of a[0..n-1]; `table` holds w_n^m, m < n.
// NC > 0: compile-time length (fft_ct above). NC == 0: the same butterflies in a
// runtime loop nest for lengths n <= RCAP.
constexpr int kMaxProject = 128;
// The runtime loop nest keeps one radix's values in buffers of kMaxRadix: a length whose
// largest factor exceeds it (a prime side of 67..127) has no runtime transform, and plans
// reject such block sides (largest_radix below).
constexpr int kMaxRadix = kMaxProject < 64 ? kMaxProject : 64;
NF_HD constexpr int largest_radix(int n) {
  const Factors f = factorize(n);
  int m = 1;
  for (int l = 0; l < f.count; ++l) m = f.r[l] > m ? f.r[l] : m;
  return m;
}
template <bool FORWARD, int NC, int RCAP = kMaxProject>
NF_HD void fft_project(cf* a, int n_rt, const cf* table) {
  if constexpr (NC > 0) {
    fft_ct<FORWARD, NC>(a, table);
  } else {
    const int n = n_rt;
    if (n <= 1) return;
    const Factors f = factorize(n);
    cf src[RCAP];
    for (int p = 0; p < n; ++p) src[p] = a[p];
    for (int p = 0; p < n; ++p) {
      int rem = p, m = n, s = 1, idx = 0;
      for (int l = 0; l < f.count; ++l) {
        m /= f.r[l];
        const int j = rem / m;
        rem -= j * m;
        idx += j * s;
        s *= f.r[l];
      }
      a[p] = src[idx];
    }
    int inner = 1;
    for (int lev = f.count - 1; lev >= 0; --lev) {
      const int r = f.r[lev];
      const int len = r * inner;
      const int tw_step = n / len;
      for (int base = 0; base < n; base += len) {
        for (int k1 = 0; k1 < inner; ++k1) {
          cf t[kMaxRadix];
          cf scratch[kMaxRadix];
          for (int j = 0; j < r; ++j) {
            cf v = a[base + j * inner + k1];
            const int e = j * k1;
            if (e != 0) {
              cf w = table[e * tw_step];
              if (!FORWARD) w.i = -w.i;
              v = cmul_plain(v, w);
            }
            t[j] = v;
          }
          butterfly<FORWARD>(t, r, table, n, scratch);
          for (int q = 0; q < r; ++q) a[base + k1 + inner * q] = t[q];
        }
      }
      inner = len;
    }
  }
}

// 1-D transform dispatch. The reference uses its codelets only for square 8x8,
// 16x16 and 32x32 blocks (fft_backend.cpp:262-273); every other shape goes to
// PocketFFT, which the project transform stands in for. The caller passes
// `codelet` = (block is square and its side is 8, 16 or 32).
template <bool FORWARD, int NC>
NF_HD void fft_1d(cf* a, int n_rt, const cf* table, bool codelet) {
  const int n = NC > 0 ? NC : n_rt;
  if (codelet && n == 8) {
    fft8<FORWARD>(a);
  } else if (codelet && n == 16) {
    fft16<FORWARD>(a);
  } else if (codelet && n == 32) {
    fft32<FORWARD>(a);
  } else {
    fft_project<FORWARD, NC>(a, n, table);
  }
}
NF_HD bool is_codelet_length(int n) { return n == 8 || n == 16 || n == 32; }

// ---------------------------------------------------------------------------
// Real 2-D building blocks (half spectrum [H][W/2+1], x fastest).
// ---------------------------------------------------------------------------

// Forward transform of one real row of W samples into K = W/2+1 bins: the row is
// transformed as complex data with zero imaginary parts (the codelets' method,
// fft16x16_avx2.cpp:239-262). The 16- and 32-point codelets store the Nyquist
// bin's imaginary part as exactly 0 (fft16x16_avx2.cpp:268-271,
// fft32x32_avx2.cpp:329-335); the project transform does the same for every even W.
template <int WC>
NF_HD void row_forward(const float* x, int w_rt, cf* bins, const cf* table, bool codelet, int bin_stride = 1) {
  if constexpr (WC == 16 || WC == 32) {
    if (codelet) {  // the real-row forms of the 16- and 32-point codelet transforms
      if constexpr (WC == 16) fft16_real_forward(x, bins, bin_stride);
      else fft32_real_forward(x, bins, bin_stride);
      return;
    }
  }
  const int w = WC > 0 ? WC : w_rt;
  constexpr int CAP = WC > 0 ? WC : kMaxProject;
  constexpr int U = WC > 0 ? CAP : 1;
  cf a[CAP];
#pragma unroll U
  for (int k = 0; k < CAP; ++k)
    if (k < w) a[k] = cf{x[k], 0.0f};
  fft_1d<true, WC>(a, w, table, codelet);
  const int K = w / 2 + 1;
#pragma unroll U
  for (int k = 0; k < CAP / 2 + 1; ++k)
    if (k < K) bins[k * bin_stride] = a[k];
  if (w % 2 == 0 && !(codelet && w == 8)) bins[(w / 2) * bin_stride].i = 0.0f;
}

// Inverse of one row: K bins -> W real samples scaled by fct. Bins 1..(W-1)/2 are
// mirrored as conjugates (imaginary part negated as 0-x, fft16x16_avx2.cpp:420-423).
// The codelets keep the DC and Nyquist bins as given; for the project transform
// their imaginary parts are cleared, because a half-complex inverse defines the
// row from their real parts only.
template <int WC>
NF_HD void row_inverse(const cf* bins, int w_rt, float fct, float* out, const cf* table, bool codelet,
                       int bin_stride = 1) {
  if constexpr (WC == 16 || WC == 32) {
    if (codelet) {  // the real-row forms of the 16- and 32-point codelet transforms
      if constexpr (WC == 16) fft16_real_inverse(bins, bin_stride, fct, out);
      else fft32_real_inverse(bins, bin_stride, fct, out);
      return;
    }
  }
  const int w = WC > 0 ? WC : w_rt;
  constexpr int CAP = WC > 0 ? WC : kMaxProject;
  constexpr int U = WC > 0 ? CAP : 1;
  const int K = w / 2 + 1;
  cf a[CAP];
#pragma unroll U
  for (int k = 0; k < CAP / 2 + 1; ++k)
    if (k < K) a[k] = bins[k * bin_stride];
#pragma unroll U
  for (int k = 1; k < CAP; ++k)
    if (k < (w + 1) / 2) a[w - k] = cf{a[k].r, fsub(0.0f, a[k].i)};
  if (!codelet) {
    a[0].i = 0.0f;
    if (w % 2 == 0) a[w / 2].i = 0.0f;
  }
  fft_1d<false, WC>(a, w, table, codelet);
#pragma unroll U
  for (int k = 0; k < CAP; ++k)
    if (k < w) out[k] = fmul(a[k].r, fct);
}

// Serial reference drivers for whole blocks (host builders and CPU checks). The
// tile kernels distribute the same row/column steps over threads.
NF_HD void block_r2c(const float* in, int in_stride, cf* out, int out_stride, int h, int w, const cf* tw_h,
                     const cf* tw_w) {
  const bool codelet = (h == w) && (w == 8 || w == 16 || w == 32);
  const int K = w / 2 + 1;
  for (int y = 0; y < h; ++y) row_forward<0>(in + y * in_stride, w, out + y * out_stride, tw_w, codelet);
  cf col[kMaxProject];
  for (int k = 0; k < K; ++k) {
    for (int y = 0; y < h; ++y) col[y] = out[y * out_stride + k];
    fft_1d<true, 0>(col, h, tw_h, codelet);
    for (int y = 0; y < h; ++y) out[y * out_stride + k] = col[y];
  }
}
NF_HD void block_c2r(const cf* in, int in_stride, float* out, int out_stride, int h, int w, float fct,
                     const cf* tw_h, const cf* tw_w) {
  const bool codelet = (h == w) && (w == 8 || w == 16 || w == 32);
  const int K = w / 2 + 1;
  cf tmp[kMaxProject * (kMaxProject / 2 + 1)];
  cf col[kMaxProject];
  for (int k = 0; k < K; ++k) {
    for (int y = 0; y < h; ++y) col[y] = in[y * in_stride + k];
    fft_1d<false, 0>(col, h, tw_h, codelet);
    for (int y = 0; y < h; ++y) tmp[y * K + k] = col[y];
  }
  for (int y = 0; y < h; ++y) row_inverse<0>(tmp + y * K, w, fct, out + y * out_stride, tw_w, codelet);
}

} // namespace nf
