// Test-only: the per-bin arithmetic of the sm_100a kernels (neo_fft_b200/csrc/device_plan.cuh,
// compiled here as host code, where its fadd/fmul/fdiv/fsqrt are the plain IEEE operations the
// device intrinsics round the same way) against the reference core's own scalar kernels, linked
// from the oracle library built from the reference sources:
//   spectral_bin     vs detail::spectral_prevalidated (src/kernels/scalar/spectral.cpp:5-53)
//   ratio_bin        vs the same, ftype 0 with exponent 1
//   enhancement_gain vs enhancement_gain (src/algorithms/fft3d_profile.cpp:69-81)
//   kalman_bin       vs kalman_scalar (src/kernels/scalar/kalman.cpp:3-24)
// over seeded random bins spanning many decades, exact zeros, subnormals and values at the
// thresholds. Every result must be equal bit for bit, and a bin the reference rejects as
// non-finite must be flagged, except where only a denominator overflows (counted apart).
// Prints one line per function with its count of mismatches.
#include "kernels/kalman.hpp"
#include "kernels/spectral.hpp"

#include "device_plan.cuh"

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include <stdexcept>
#include <vector>

namespace {
using C = std::complex<float>;

std::uint32_t bits(float v) {
  std::uint32_t u;
  std::memcpy(&u, &v, 4);
  return u;
}
bool same(float a, float b) { return bits(a) == bits(b); }

// A value drawn over 1e-20 .. 1e12 in magnitude, either sign, with exact zeros, subnormals,
// small integers and a few values up to 1e17 (powers up to 1e34, still finite, where the
// sharpen and ftype 4 denominators overflow) mixed in.
float draw(std::mt19937& g) {
  std::uniform_real_distribution<double> u(0.0, 1.0);
  const double pick = u(g);
  const double sign = u(g) < 0.5 ? -1.0 : 1.0;
  if (pick < 0.04) return 0.0f;
  if (pick < 0.06) return float(sign * 1e-41);  // subnormal
  if (pick < 0.12) return float(sign * std::floor(u(g) * 64));
  if (pick < 0.17) return float(sign * std::pow(10.0, 12.0 + 5.0 * u(g)));
  return float(sign * std::pow(10.0, -20.0 + 32.0 * u(g)));
}
float positive(std::mt19937& g, double lo_exp, double hi_exp) {
  std::uniform_real_distribution<double> u(0.0, 1.0);
  return float(std::pow(10.0, lo_exp + (hi_exp - lo_exp) * u(g)));
}

struct Tables {
  std::vector<float> primary, sharpen_w, halo_w;
  std::vector<C> grid;
  std::vector<nf::cf> dgrid;
};

int overflow_only = 0;  // bins the reference rejects for an overflowing denominator alone

int check_spectral(std::mt19937& g, int type, bool table, bool use_grid, bool enh, float exponent, int trials) {
  const int n = 64;
  Tables t;
  t.primary.resize(n);
  t.sharpen_w.resize(n);
  t.halo_w.resize(n);
  t.grid.resize(n);
  t.dgrid.resize(n);
  for (int k = 0; k < n; ++k) {
    t.primary[k] = positive(g, -6, 6);
    t.sharpen_w[k] = positive(g, -2, 0);
    t.halo_w[k] = positive(g, -2, 0);
    t.grid[k] = {draw(g), draw(g)};
    t.dgrid[k] = {t.grid[k].real(), t.grid[k].imag()};
  }
  neo_fft::SpectralParams rp;
  rp.type = type;
  rp.a = positive(g, -4, 4);
  rp.b = positive(g, -1, 1);
  rp.low = positive(g, -2, 2);
  rp.high = positive(g, 2, 6);
  rp.exponent = exponent;
  rp.floor = type == -1 ? 0.3f : 0.0f;
  if (table) {
    rp.primary_mode = neo_fft::PrimaryMode::Table;
    rp.primary = {t.primary.data(), t.primary.size()};
  }
  if (enh) {
    rp.enhancement.sharpen = 0.4f;
    rp.enhancement.dehalo = 0.3f;
    rp.enhancement.a = positive(g, -2, 2);
    rp.enhancement.b = positive(g, 0, 4);
    rp.enhancement.c = positive(g, -2, 2);
    rp.enhancement.sharpen_window = {t.sharpen_w.data(), t.sharpen_w.size()};
    rp.enhancement.halo_window = {t.halo_w.data(), t.halo_w.size()};
  }
  nfd::DevSpectral dp{};
  dp.type = type;
  dp.a = rp.a;
  dp.b = rp.b;
  dp.low = rp.low;
  dp.high = rp.high;
  dp.exponent = rp.exponent;
  dp.floor = rp.floor;
  dp.primary = table ? t.primary.data() : nullptr;
  dp.enh = enh ? 1 : 0;
  dp.sharpen = rp.enhancement.sharpen;
  dp.dehalo = rp.enhancement.dehalo;
  dp.ea = rp.enhancement.a;
  dp.eb = rp.enhancement.b;
  dp.ec = rp.enhancement.c;
  dp.sharpen_w = t.sharpen_w.data();
  dp.halo_w = t.halo_w.data();
  dp.emode = std::fabs(exponent - 1.0f) < 0.00005f ? 0 : std::fabs(exponent - 0.5f) < 0.00005f ? 1 : 2;
  const float scale = use_grid ? positive(g, -3, 0) : 0.0f;
  int bad_count = 0;
  for (int trial = 0; trial < trials; ++trial) {
    const int k = int(g() % n);
    C x = {draw(g), draw(g)};
    if (trial % 16 == 0) {  // a bin whose power sits on the threshold or the range ends
      const float target = type == 3 ? (trial % 32 ? rp.low : rp.high) : (table ? t.primary[k] : rp.a);
      x = {std::sqrt(target), 0.0f};
    }
    // reference: one bin
    C rx = x;
    bool ref_threw = false;
    try {
      neo_fft::detail::spectral_prevalidated(&rx, use_grid ? &t.grid[k] : nullptr, 1, scale,
                                              [&] {
                                                neo_fft::SpectralParams q = rp;  // the bin's own table entries
                                                if (table) q.primary = {&t.primary[k], 1};
                                                if (enh) {
                                                  q.enhancement.sharpen_window = {&t.sharpen_w[k], 1};
                                                  q.enhancement.halo_window = {&t.halo_w[k], 1};
                                                }
                                                return q;
                                              }());
    } catch (const std::runtime_error&) {
      ref_threw = true;
    }
    bool bad = false;
    const nf::cf out = nfd::spectral_bin<>({x.real(), x.imag()}, use_grid ? t.dgrid.data() : nullptr, k, scale, dp,
                                           bad);
    if (ref_threw) {
      // The reference also rejects an intermediate that overflows while the bin's value
      // stays finite: ftype 4's and the sharpen term's denominators (q + low)(q + high) and
      // (q + a)(q + b) pass FLT_MAX once the power q exceeds about 1.8e19, where their
      // quotient rounds to 0. The kernels report only non-finite powers and outputs, so
      // those bins come out finite and unflagged; any other unflagged rejection is a mismatch.
      if (!bad) {
        const double mr = use_grid ? double(scale) * t.grid[k].real() : 0.0;
        const double mi = use_grid ? double(scale) * t.grid[k].imag() : 0.0;
        const double q = (x.real() - mr) * (x.real() - mr) + (x.imag() - mi) * (x.imag() - mi);
        if (q >= 1e19 && (type == 4 || enh)) ++overflow_only;
        else ++bad_count;
      }
      continue;
    }
    if (bad || !same(out.r, rx.real()) || !same(out.i, rx.imag())) ++bad_count;
    if (type == 0 && dp.emode == 0 && !enh) {  // the ratio form of the ftype 0 strips
      float guard = 0.0f;
      const nf::cf r2 = nfd::ratio_bin({x.real(), x.imag()}, use_grid ? t.dgrid.data() : nullptr, k, scale, dp,
                                       guard);
      if (!same(r2.r, rx.real()) || !same(r2.i, rx.imag()) || guard != 0.0f) ++bad_count;
    }
  }
  return bad_count;
}

int check_kalman(std::mt19937& g, bool pattern, int trials) {
  const int n = 64;
  std::vector<float> pat(n);
  for (auto& v : pat) v = (g() % 8 == 0) ? 0.0f : positive(g, -6, 4);
  const float uniform = (g() % 8 == 0) ? 0.0f : positive(g, -4, 4);
  const float ratio2 = positive(g, -1, 1);
  int bad_count = 0;
  for (int trial = 0; trial < trials; ++trial) {
    const int k = int(g() % n);
    C x = {draw(g), draw(g)}, last = {draw(g), draw(g)};
    if (trial % 4 == 0) last = {x.real() + float(std::ldexp(draw(g), -30)), x.imag()};  // blend, not reset
    float cov = positive(g, -8, 6), proc = positive(g, -8, 6);
    C rl = last;
    float rc = cov, rq = proc;
    bool ref_threw = false;
    try {
      neo_fft::kalman_scalar(&x, &rl, &rc, &rq, pattern ? &pat[k] : nullptr, uniform, ratio2, 1);
    } catch (const std::runtime_error&) {
      ref_threw = true;
    }
    nf::cf dl = {last.real(), last.imag()};
    float dc = cov, dq = proc;
    const bool ok = nfd::kalman_bin({x.real(), x.imag()}, dl, dc, dq, pattern ? pat.data() : nullptr, k, uniform,
                                    ratio2);
    if (ref_threw) {
      if (ok) ++bad_count;
      continue;
    }
    if (!ok || !same(dl.r, rl.real()) || !same(dl.i, rl.imag()) || !same(dc, rc) || !same(dq, rq)) ++bad_count;
  }
  return bad_count;
}

int check_enhancement(std::mt19937& g, int trials) {
  const int n = 64;
  std::vector<float> sw(n), hw(n);
  for (int k = 0; k < n; ++k) {
    sw[k] = positive(g, -2, 0);
    hw[k] = positive(g, -2, 0);
  }
  int bad_count = 0;
  for (int trial = 0; trial < trials; ++trial) {
    neo_fft::Enhancement e;
    e.sharpen = (trial % 3 == 0) ? 0.0f : positive(g, -1, 0);
    e.dehalo = (trial % 5 == 0) ? 0.0f : positive(g, -1, 0);
    e.a = positive(g, -2, 2);
    e.b = (trial % 7 == 0) ? 0.0f : positive(g, 0, 4);
    e.c = positive(g, -2, 2);
    e.sharpen_window = {sw.data(), sw.size()};
    e.halo_window = {hw.data(), hw.size()};
    nfd::DevSpectral d{};
    d.sharpen = e.sharpen;
    d.dehalo = e.dehalo;
    d.ea = e.a;
    d.eb = e.b;
    d.ec = e.c;
    d.sharpen_w = sw.data();
    d.halo_w = hw.data();
    const int k = int(g() % n);
    const float q = positive(g, -15, 12);
    float want;
    try {
      want = neo_fft::enhancement_gain(q, std::size_t(k), e);
    } catch (const std::runtime_error&) {
      continue;  // the spectral bin flags it through its output
    }
    if (!same(nfd::enhancement_gain(q, k, d), want)) ++bad_count;
  }
  return bad_count;
}
} // namespace

int main() {
  std::mt19937 g(20240611);
  const int trials = 40000;
  int total = 0;
  struct Case {
    const char* name;
    int type;
    bool table, grid, enh;
    float exponent;
  };
  const Case cases[] = {
      {"fft3d_wiener", -1, false, false, false, 1.0f},
      {"fft3d_wiener_table_grid", -1, true, true, false, 1.0f},
      {"fft3d_wiener_enhanced", -1, false, true, true, 1.0f},
      {"fft3d_enhance_only", -2, false, true, true, 1.0f},
      {"dft_ftype0_ratio", 0, true, true, false, 1.0f},
      {"dft_ftype0_sqrt", 0, true, false, false, 0.5f},
      {"dft_ftype0_pow", 0, false, true, false, 1.7f},
      {"dft_ftype1", 1, true, true, false, 1.0f},
      {"dft_ftype2", 2, true, false, false, 1.0f},
      {"dft_ftype3", 3, true, true, false, 1.0f},
      {"dft_ftype4", 4, true, true, false, 1.0f},
  };
  for (const Case& c : cases) {
    const int m = check_spectral(g, c.type, c.table, c.grid, c.enh, c.exponent, trials);
    std::printf("%s %d\n", c.name, m);
    total += m;
  }
  for (int pattern = 0; pattern < 2; ++pattern) {
    const int m = check_kalman(g, pattern != 0, trials);
    std::printf("kalman%s %d\n", pattern ? "_pattern" : "_uniform", m);
    total += m;
  }
  const int m = check_enhancement(g, trials);
  std::printf("enhancement_gain %d\n", m);
  total += m;
  std::printf("overflow_only %d\n", overflow_only);
  return total == 0 ? 0 : 1;
}
