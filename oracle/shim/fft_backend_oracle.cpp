// Test infrastructure (oracle only): the FFT backend table that the compiled
// neo-fft core links against, in place of src/spectral/fft_backend.cpp.
//
// The reference's backend wraps PocketFFT (commit c90e55b3, fetched by
// cmake/Dependencies.cmake:15-18), which is absent from this machine, so
// fft_backend.cpp cannot be compiled. This file provides the same interface
// (src/spectral/fft_backend.hpp:8-30, symbol neo_fft::detail::scalar_fft()):
//
//   * square 8x8, 16x16 and 32x32 blocks call the reference's own AVX2 codelets,
//     compiled unchanged from src/spectral/codelets/*.cpp (as the reference's
//     avx2/avx512 backends do, fft_backend.cpp:262-273);
//   * every other shape uses the project transform (fft_core.cuh), which stands in
//     for PocketFFT. Parity with PocketFFT's own rounding is therefore unpinned for
//     those shapes; the project transform is checked against binary64 DFTs instead.
//   * 3-D volumes: spatial 2-D transform per temporal slice, then the temporal
//     axis (forward); temporal axis first, then spatial (inverse) — the order of
//     the reference's dense codelet path (fft_backend.cpp:636-652, 668-676).
//   * try_c2r_3d_slice returns false, so the core takes its full-inverse path.
#include "spectral/fft_backend.hpp"
#include "spectral/codelets/fft16x16.hpp"
#include "spectral/codelets/fft32x32.hpp"
#include "spectral/codelets/fft8x8.hpp"

#include "fft_core.cuh"

#include <cmath>
#include <map>
#include <mutex>
#include <stdexcept>
#include <vector>

namespace {
using cfloat = std::complex<float>;

const nf::cf* table(int n) {
  static std::mutex mu;
  static std::map<int, std::vector<nf::cf>> tables;
  std::lock_guard<std::mutex> lock(mu);
  auto& t = tables[n];
  if (t.empty()) {
    t.resize(std::size_t(n));
    for (int m = 0; m < n; ++m) {
      const double a = 2.0 * 3.14159265358979323846264338327950288 * double(m) / double(n);
      t[std::size_t(m)] = {float(std::cos(a)), float(-std::sin(a))};
    }
  }
  return t.data();
}

bool codelet_shape(int h, int w) { return h == w && (w == 8 || w == 16 || w == 32); }

// The stand-in transform covers lengths up to 128 whose factors are at most 64 (the
// product's limits); other lengths are refused rather than transformed wrongly.
void stand_in_length(int n) {
  if (n < 1 || n > nf::kMaxProject || nf::largest_radix(n) > nf::kMaxRadix)
    throw std::invalid_argument("transform length outside the oracle's stand-in transform");
}

void r2c_one(int h, int w, const float* in, std::size_t in_rs, cfloat* out, std::size_t out_rs) {
  if (codelet_shape(h, w)) {
    if (w == 8) neo_fft::codelet::fft8x8_r2c(in, in_rs, out, out_rs);
    else if (w == 16) neo_fft::codelet::fft16x16_r2c(in, in_rs, out, out_rs);
    else neo_fft::codelet::fft32x32_r2c(in, in_rs, out, out_rs);
    return;
  }
  stand_in_length(h);
  stand_in_length(w);
  nf::block_r2c(in, int(in_rs), reinterpret_cast<nf::cf*>(out), int(out_rs), h, w, table(h), table(w));
}
void c2r_one(int h, int w, const cfloat* in, std::size_t in_rs, float* out, std::size_t out_rs, float fct) {
  if (codelet_shape(h, w)) {
    if (w == 8) neo_fft::codelet::fft8x8_c2r(in, in_rs, out, out_rs, fct);
    else if (w == 16) neo_fft::codelet::fft16x16_c2r(in, in_rs, out, out_rs, fct);
    else neo_fft::codelet::fft32x32_c2r(in, in_rs, out, out_rs, fct);
    return;
  }
  stand_in_length(h);
  stand_in_length(w);
  nf::block_c2r(reinterpret_cast<const nf::cf*>(in), int(in_rs), out, int(out_rs), h, w, fct, table(h),
                table(w));
}

void r2c(int h, int w, const float* in, std::size_t in_rs, cfloat* out, std::size_t out_rs) {
  r2c_one(h, w, in, in_rs, out, out_rs);
}
void c2r(int h, int w, const cfloat* in, std::size_t in_rs, float* out, std::size_t out_rs, float fct) {
  c2r_one(h, w, in, in_rs, out, out_rs, fct);
}
void batch_r2c(std::size_t batch, int h, int w, const float* in, std::size_t in_dist, std::size_t in_rs,
               cfloat* out, std::size_t out_dist, std::size_t out_rs) {
  for (std::size_t b = 0; b < batch; ++b) r2c_one(h, w, in + b * in_dist, in_rs, out + b * out_dist, out_rs);
}
void batch_c2r(std::size_t batch, int h, int w, const cfloat* in, std::size_t in_dist, std::size_t in_rs,
               float* out, std::size_t out_dist, std::size_t out_rs, float fct) {
  for (std::size_t b = 0; b < batch; ++b)
    c2r_one(h, w, in + b * in_dist, in_rs, out + b * out_dist, out_rs, fct);
}

// Temporal axis over T slices of `bins` complex values each (in place).
void temporal_axis(int t, std::size_t bins, cfloat* v, bool forward) {
  stand_in_length(t);
  std::vector<nf::cf> line(static_cast<std::size_t>(t));
  const nf::cf* tw = table(t);
  for (std::size_t k = 0; k < bins; ++k) {
    for (int z = 0; z < t; ++z) line[std::size_t(z)] = reinterpret_cast<nf::cf&>(v[std::size_t(z) * bins + k]);
    if (forward) nf::fft_project<true, 0>(line.data(), t, tw);
    else nf::fft_project<false, 0>(line.data(), t, tw);
    for (int z = 0; z < t; ++z) v[std::size_t(z) * bins + k] = {line[std::size_t(z)].r, line[std::size_t(z)].i};
  }
}
void r2c_3d(int d, int h, int w, const float* in, cfloat* out) {
  const int k = w / 2 + 1;
  const std::size_t samples = std::size_t(h) * w, bins = std::size_t(h) * k;
  for (int z = 0; z < d; ++z) r2c_one(h, w, in + z * samples, std::size_t(w), out + z * bins, std::size_t(k));
  if (d > 1) temporal_axis(d, bins, out, true);
}
void c2r_3d(int d, int h, int w, const cfloat* in, float* out, float fct) {
  const int k = w / 2 + 1;
  const std::size_t samples = std::size_t(h) * w, bins = std::size_t(h) * k;
  std::vector<cfloat> tmp(in, in + std::size_t(d) * bins);
  if (d > 1) temporal_axis(d, bins, tmp.data(), false);
  for (int z = 0; z < d; ++z)
    c2r_one(h, w, tmp.data() + z * bins, std::size_t(k), out + z * samples, std::size_t(w), fct);
}
void batch_r2c_3d(std::size_t batch, int d, int h, int w, const float* in, std::size_t in_dist, cfloat* out,
                  std::size_t out_dist) {
  for (std::size_t b = 0; b < batch; ++b) r2c_3d(d, h, w, in + b * in_dist, out + b * out_dist);
}
void batch_c2r_3d(std::size_t batch, int d, int h, int w, const cfloat* in, std::size_t in_dist, float* out,
                  std::size_t out_dist, float fct) {
  for (std::size_t b = 0; b < batch; ++b) c2r_3d(d, h, w, in + b * in_dist, out + b * out_dist, fct);
}
bool try_c2r_3d_slice(std::size_t, int, int, int, int, const cfloat*, std::size_t, float*, std::size_t, float) {
  return false;
}
} // namespace

namespace neo_fft::detail {
const FftBackend& scalar_fft() noexcept {
  static const FftBackend backend{1,        "oracle-codelet+project", r2c,          c2r,
                                  batch_r2c, batch_c2r,                r2c_3d,       c2r_3d,
                                  batch_r2c_3d, batch_c2r_3d,          try_c2r_3d_slice};
  return backend;
}
} // namespace neo_fft::detail
