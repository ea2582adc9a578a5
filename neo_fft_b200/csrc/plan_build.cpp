// Creation-time tables; see plan_build.hpp. Compiled with -fno-fast-math
// -ffp-contract=off so binary32 expressions round exactly as in the reference.
#include "plan_build.hpp"

#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <limits>
#include <utility>

namespace nfb {
namespace {

int dimension(long long n) {
  require(n > 0 && n <= INT32_MAX, "dimension outside int32 domain");
  return int(n);
}
long long ceil_div(long long n, long long d) {
  require(n >= 0 && d > 0, "invalid ceiling division");
  return n / d + (n % d != 0);
}
void nonnegative(float v, const char* name) {
  if (!(std::isfinite(v) && v >= 0)) throw std::invalid_argument(std::string("invalid ") + name);
}
// Single-reflection admission (src/spectral/geometry.hpp:9-14).
Axis admit(Axis a) {
  require(a.offset >= 0 && a.cover >= (long long)a.offset + a.length && a.offset < a.length &&
              (long long)a.cover - a.offset - a.length < a.length,
          "selected-plane padding exceeds one-reflection domain");
  return a;
}
void valid_format(nf_format f) {
  require(f.floating ? f.bits == 32 : (f.bits == 8 || f.bits == 10 || f.bits == 12 || f.bits == 14 || f.bits == 16),
          "unsupported sample format");
}
// Cover-plane size check of the Geometry constructor (geometry.hpp:51-54).
void check_geometry(const Axis& x, const Axis& y) {
  const long long row = (long long)x.cover * 4;
  require(row / 4 <= INT32_MAX, "invalid plane byte stride");
  (void)y;
}

// --- DFTTest curves (src/algorithms/profile.cpp:8-45) ---
using Curve = std::vector<std::pair<float, float>>;
Curve sorted(const std::vector<float>& values) {
  require(values.size() % 2 == 0, "DFTTest curve requires frequency/value pairs");
  Curve knots;
  for (std::size_t i = 0; i < values.size(); i += 2) {
    require(std::isfinite(values[i]) && values[i] >= 0 && values[i] <= 1, "DFTTest curve position outside 0..1");
    require(std::isfinite(values[i + 1]) && values[i + 1] >= 0, "DFTTest invalid curve value");
    knots.emplace_back(values[i], values[i + 1]);
  }
  std::sort(knots.begin(), knots.end());
  if (!knots.empty()) {
    require(knots.front().first == 0 && knots.back().first == 1, "DFTTest curve requires endpoints 0 and 1");
    for (std::size_t i = 1; i < knots.size(); ++i)
      require(knots[i - 1].first < knots[i].first, "DFTTest duplicate curve position after binary32 conversion");
  }
  return knots;
}
Curve prepare(const std::vector<float>& values, float sigma, float exponent) {
  auto knots = sorted(values);
  if (knots.empty()) knots = {{0.0f, sigma}, {1.0f, sigma}};
  for (auto& knot : knots) knot.second = finite(std::pow(knot.second, exponent));
  return knots;
}
float interpolate(const Curve& curve, float f) {
  auto hi = std::lower_bound(curve.begin(), curve.end(), f, [](const auto& knot, float v) { return knot.first < v; });
  require(hi != curve.end(), "DFTTest frequency outside curve");
  if (hi->first == f) return hi->second;
  require(hi != curve.begin(), "DFTTest frequency outside curve");
  const auto lo = hi - 1;
  const float t = finite((f - lo->first) / (hi->first - lo->first));
  return finite(finite(lo->second * (1 - t)) + finite(hi->second * t));
}
float frequency(int i, int length) { return length == 1 ? 0 : float(std::min(i, length - i)) / float(length / 2); }
void validate_curves(const Curves& c) {
  require(c.system == 0 || c.system == 1, "DFTTest ssystem outside 0..1");
  for (const auto* v : {&c.shared, &c.x, &c.y, &c.time}) sorted(*v);
}

// --- FFT3D and DFTTest configuration checks (src/algorithms/plan.cpp:45-90) ---
void validate_enhancement(const nf_fft3d_config& c) {
  for (float v : {c.sharpen, c.svr, c.smin, c.smax, c.dehalo, c.ht})
    require(std::isfinite(v) && v >= 0, "FFT3D invalid enhancement parameter");
  require(c.smin <= c.smax, "FFT3D smin exceeds smax");
  for (float v : {c.scutoff, c.hr}) require(std::isfinite(v) && v > 0, "FFT3D cutoff/radius must be positive");
}
void validate_fft3d(const nf_fft3d_config& c) {
  require(c.kalman_warmup >= 0, "FFT3D kalman_warmup must be nonnegative");
  require(c.cache_frames >= -1 && c.cache_mb >= -1, "FFT3D cache limits must be >= -1");
  require(c.left >= 0 && c.top >= 0 && c.right >= 0 && c.bottom >= 0, "ROI margins must be nonnegative");
  require(c.bw >= 2 && c.bh >= 2, "FFT3D bw/bh must be >=2");
  require(c.ow <= c.bw / 2 && c.oh <= c.bh / 2, "FFT3D ow/oh exceeds half block");
  require(c.wintype >= 0 && c.wintype <= 2, "FFT3D wintype outside 0..2");
  require(c.bt >= -1 && c.bt <= 5, "FFT3D bt outside -1..5");
  nonnegative(c.kratio, "kratio");
  validate_enhancement(c);
  nonnegative(c.pfactor, "FFT3D pfactor");
  require(std::isfinite(c.pcutoff) && c.pcutoff > 0, "FFT3D pcutoff must be positive");
  require(c.px >= 0 && c.py >= 0, "FFT3D px/py must be nonnegative");
  for (int i = 0; i < 3; ++i) {
    const int has = i == 0 ? c.has_sigma2 : i == 1 ? c.has_sigma3 : c.has_sigma4;
    const float v = i == 0 ? c.sigma2 : i == 1 ? c.sigma3 : c.sigma4;
    nonnegative(has ? v : c.sigma, "FFT3D sigma2..4");
  }
  nonnegative(c.sigma, "FFT3D sigma");
  nonnegative(c.degrid, "FFT3D degrid");
  require(std::isfinite(c.beta) && c.beta >= 1, "FFT3D beta must be >=1");
}
Curves curves_of(const nf_dft_config& c) {
  auto v = [](const float* p, int n) { return p && n > 0 ? std::vector<float>(p, p + n) : std::vector<float>{}; };
  Curves r;
  r.shared = v(c.slocation, c.n_slocation);
  r.x = v(c.ssx, c.n_ssx);
  r.y = v(c.ssy, c.n_ssy);
  r.time = v(c.sst, c.n_sst);
  r.system = c.ssystem;
  return r;
}
void validate_dft(const nf_dft_config& c) {
  require(c.opt == 0 || c.opt == 1 || c.opt == 2 || c.opt == 3 || c.opt == 8, "DFTTest opt outside 0,1,2,3,8");
  require(c.dither >= 0 && c.dither_seed >= 0, "dither and dither_seed must be nonnegative");
  validate_curves(curves_of(c));
  require(c.n_nlocation <= 500, "DFTTest nlocation exceeds 500 tuples");
  const float alpha = c.has_alpha ? c.alpha : (c.ftype == 0 ? 5.0f : 7.0f);
  require(std::isfinite(alpha) && alpha > 0, "DFTTest alpha must be positive");
  for (int i = 0; i < c.n_nlocation; ++i)
    require(c.nlocation[4 * i] >= 0 && c.nlocation[4 * i + 1] >= 0 && c.nlocation[4 * i + 2] >= 0 &&
                c.nlocation[4 * i + 3] >= 0,
            "DFTTest negative sample coordinate");
  require(c.block > 0 && (c.mode == 0 || c.mode == 1), "DFTTest invalid sbsize/smode");
  require(c.mode != 0 || c.block % 2 == 1, "DFTTest center mode requires odd sbsize");
  require(c.mode == 0 || (c.overlap >= 0 && c.overlap < c.block), "DFTTest invalid sosize");
  validate_temporal(c.tbsize, c.temporal_mode, c.temporal_overlap);
  if (c.mode == 1 && c.overlap > c.block / 2)
    require(c.block % (c.block - c.overlap) == 0, "DFTTest heavy overlap requires divisible step");
  require(c.swin >= 0 && c.swin <= 11 && c.twin >= 0 && c.twin <= 11, "DFTTest invalid swin/twin");
  require(c.ftype >= 0 && c.ftype <= 4, "DFTTest ftype outside 0..4");
  nonnegative(c.sbeta, "DFTTest sbeta");
  nonnegative(c.tbeta, "DFTTest tbeta");
  nonnegative(c.sigma, "DFTTest sigma");
  nonnegative(c.sigma2, "DFTTest sigma2");
  nonnegative(c.pmin, "DFTTest pmin");
  nonnegative(c.pmax, "DFTTest pmax");
  require(c.pmin <= c.pmax, "DFTTest pmin exceeds pmax");
  require(std::isfinite(c.f0beta) && c.f0beta > 0, "DFTTest f0beta must be positive");
}

// The block transform must fit the tile kernels' register/shared budgets.
void gpu_block_limits(int bh, int bw, int t) {
  require(bh <= nf::kMaxProject && bw <= nf::kMaxProject,
          "block size exceeds the GPU tile limit of 128 samples per side");
  require(nf::largest_radix(bh) <= nf::kMaxRadix && nf::largest_radix(bw) <= nf::kMaxRadix,
          "block side has a prime factor above 64, beyond the GPU transform's radix limit");
  require((long long)bh * (bw / 2 + 1) * t <= 16384, "block volume exceeds the GPU tile limit");
}

double i0a(double arg) {
  double num = 1, den = 1, total = 1;
  for (int k = 1; k <= 14; ++k) {
    num *= arg / 2;
    den *= k;
    const double v = num / den;
    total += v * v;
    require(std::isfinite(total), "DFTTest Kaiser window overflow");
    if (v <= 1e-8) break;
  }
  return total;
}
} // namespace

// --- geometry (src/spectral/geometry.hpp:15-48) ---
Axis fft3d_axis(int length, int block, int overlap) {
  dimension(length);
  require(block >= 2 && length >= block, "FFT3D block must be >=2 and fit selected plane");
  if (overlap < 0) overlap = block / 3;
  require(overlap <= block / 2, "FFT3D overlap exceeds half block");
  const int step = block - overlap;
  const int count = dimension(ceil_div((long long)length - overlap, step) + 2);
  const int cover = dimension((long long)count * step + overlap);
  return admit({length, block, overlap, step, count, cover, step});
}
Axis dft_axis(int length, int block, int mode, int overlap) {
  dimension(length);
  dimension(block);
  require(mode == 0 || mode == 1, "DFTTest smode must be 0 or 1");
  if (mode == 0) {
    require(block % 2 == 1, "DFTTest center mode requires odd sbsize");
    const int c = block / 2;
    return admit({length, block, 0, 1, length, dimension((long long)length + 2LL * c), c});
  }
  require(overlap >= 0 && overlap < block, "DFTTest sosize outside block");
  const int step = block - overlap;
  require(overlap <= block / 2 || block % step == 0, "DFTTest heavy overlap requires divisible step");
  const int cover = dimension((long long)block * ceil_div(length, block) + 2LL * std::max(step, overlap));
  Axis a = admit({length, block, overlap, step, (cover - block) / step + 1, cover, (cover - length) / 2});
  require(a.offset >= block - step && (long long)a.offset + length <= (long long)a.count * step,
          "DFTTest visible crop lacks complete phase coverage");
  return a;
}
int reflect(int c, const Axis& a) {
  const long long j = (long long)c - a.offset;
  return int(j < 0 ? -j : j < a.length ? j : 2LL * a.length - 2 - j);
}

// --- windows (src/algorithms/windows.cpp:6-152) ---
AxisWindow fft3d_window(int block, int overlap, int type) {
  require(block >= 2 && overlap >= 0 && overlap <= block / 2, "FFT3D window geometry invalid");
  require(type >= 0 && type <= 2, "FFT3D wintype outside 0..2");
  AxisWindow win{std::vector<float>(block, 1.0f), std::vector<float>(block, 1.0f)};
  constexpr float pi = 3.14159265358979323846f;
  for (int j = 0; j < overlap; ++j) {
    const float left = std::cos(pi * (float(j - overlap) + 0.5f) / (2.0f * float(overlap)));
    const float right = std::cos(pi * (float(j) + 0.5f) / (2.0f * float(overlap)));
    for (int side = 0; side < 2; ++side) {
      const float c = side ? right : left;
      const int pos = side ? block - overlap + j : j;
      const float a = type == 0 ? c : type == 1 ? std::sqrt(c) : 1.0f;
      win.analysis[pos] = a;
      win.synthesis[pos] = type == 0 ? c : type == 1 ? (a * a) * a : c * c;
    }
  }
  return win;
}
double dft_raw_window(int id, int j, int length, float beta) {
  require(id >= 0 && id <= 11 && length > 0 && j >= 0 && j < length && std::isfinite(beta) && beta >= 0,
          "DFTTest window parameter invalid");
  constexpr double pi = 3.1415926535897932384626433832795;
  const double n = j + 0.5, r = n / length, theta = 2 * pi * r;
  auto c = [&](int m) { return std::cos(m * theta); };
  double value = 0;
  switch (id) {
    case 0: value = 0.5 - 0.5 * c(1); break;
    case 1: value = 0.53836 - 0.46164 * c(1); break;
    case 2: value = 0.42 - 0.5 * c(1) + 0.08 * c(2); break;
    case 3: value = 0.35875 - 0.48829 * c(1) + 0.14128 * c(2) - 0.01168 * c(3); break;
    case 4: value = i0a(pi * beta * std::sqrt(1 - (2 * r - 1) * (2 * r - 1))) / i0a(pi * beta); break;
    case 5: {
      constexpr std::array<double, 7> a{0.27105140069342415,   -0.433297939234486060, 0.218122999543110620,
                                        -0.065925446388030898, 0.010811742098372268,  -7.7658482522509342e-4,
                                        1.3887217350903198e-5};
      value = a[0];
      for (int m = 1; m < 7; ++m) value += a[m] * c(m);
      break;
    }
    case 6: value = 0.2810639 - 0.5208972 * c(1) + 0.1980399 * c(2); break;
    case 7: value = 1; break;
    case 8: value = (2.0 / length) * (length / 2.0 - std::abs(n - length / 2.0)); break;
    case 9: value = 0.62 - 0.48 * (r - 0.5) - 0.38 * c(1); break;
    case 10: value = 0.355768 - 0.487396 * c(1) + 0.144232 * c(2) - 0.012604 * c(3); break;
    case 11: value = 0.3635819 - 0.4891775 * c(1) + 0.1365995 * c(2) - 0.0106411 * c(3); break;
  }
  require(std::isfinite(value), "DFTTest non-finite window");
  return value;
}
DftWindow dft_window_3d(int tbsize, int block, int overlap, int mode, int spatial, int temporal, float sbeta,
                        float tbeta, int temporal_mode, int temporal_overlap) {
  dimension(tbsize);
  dimension(block);
  require(tbsize > 0 && tbsize <= 15, "DFTTest tbsize outside 1..15");
  require(temporal_mode == 0 || temporal_mode == 1, "DFTTest temporal window mode invalid");
  require(temporal_mode == 0 || (temporal_overlap >= 0 && temporal_overlap < tbsize),
          "DFTTest temporal overlap invalid");
  require(mode == 0 || mode == 1, "DFTTest window mode invalid");
  require(overlap >= 0 && overlap < block, "DFTTest window overlap invalid");
  std::vector<double> raw(block), sw(block);
  for (int j = 0; j < block; ++j) raw[j] = dft_raw_window(spatial, j, block, sbeta);
  sw = raw;
  if (mode == 1) {
    const int step = block - overlap;
    for (int j = 0; j < block; ++j) {
      double d = 0;
      for (int k = j; k >= 0; k -= step) d += raw[k] * raw[k];
      for (long long k = (long long)j + step; k < block; k += step) d += raw[k] * raw[k];
      require(std::isfinite(d) && d > 0, "DFTTest zero or invalid window denominator");
      sw[j] = raw[j] / std::sqrt(d);
    }
  }
  std::vector<double> tw(tbsize);
  for (int z = 0; z < tbsize; ++z) tw[z] = dft_raw_window(temporal, z, tbsize, tbeta);
  if (temporal_mode == 1) {
    const auto raw_time = tw;
    const int step = tbsize - temporal_overlap;
    for (int z = 0; z < tbsize; ++z) {
      double energy = 0;
      for (int h = z; h >= 0; h -= step) energy += raw_time[h] * raw_time[h];
      for (int h = z + step; h < tbsize; h += step) energy += raw_time[h] * raw_time[h];
      require(std::isfinite(energy) && energy > 0, "DFTTest temporal phase energy invalid");
      tw[z] = raw_time[z] / std::sqrt(energy);
      require(std::isfinite(tw[z]), "DFTTest temporal window invalid");
    }
  }
  const double volume = double(tbsize) * double(block) * double(block);
  const double inv_sqrt_v = 1.0 / std::sqrt(volume);
  DftWindow w{std::vector<float>(std::size_t(tbsize) * block * block), 0};
  float energy = 0.0f;
  for (int z = 0; z < tbsize; ++z)
    for (int y = 0; y < block; ++y) {
      const double factor = tw[z] * sw[y];
      float* out = w.h.data() + (std::size_t(z) * block + y) * block;
      for (int x = 0; x < block; ++x) {
        const double v = factor * sw[x] * inv_sqrt_v;
        require(std::isfinite(v) && std::abs(v) <= std::numeric_limits<float>::max(), "DFTTest window overflow");
        const float hv = float(v);
        out[x] = hv;
        energy += hv * hv;
      }
    }
  require(std::isfinite(energy) && energy > 0, "DFTTest zero or invalid window energy");
  w.wscale = 1.0f / energy;
  require(std::isfinite(w.wscale) && w.wscale > 0, "DFTTest invalid wscale");
  return w;
}

// --- DFTTest sigma curves (src/algorithms/profile.cpp:52-100) ---
std::vector<float> dft_profile(const Curves& c, int T, int S, float sigma, float divisor) {
  validate_curves(c);
  require(T > 0 && S > 0 && std::isfinite(sigma) && sigma >= 0 && std::isfinite(divisor) && divisor > 0,
          "DFTTest invalid profile shape or scale");
  const int K = S / 2 + 1;
  std::vector<float> result(std::size_t(T) * S * K);
  if (c.empty()) {
    std::fill(result.begin(), result.end(), finite(sigma / divisor));
    return result;
  }
  const int dims = (T > 1 ? 1 : 0) + (S > 1 ? 2 : 0);
  const bool shared = !c.shared.empty();
  const float exponent = dims == 0 || (shared && c.system == 1) ? 1.0f : 1.0f / float(dims);
  const auto time = prepare(shared ? c.shared : c.time, sigma, exponent);
  if (dims == 0) {
    result[0] = finite(interpolate(time, 0) / divisor);
    return result;
  }
  const auto y = prepare(shared ? c.shared : c.y, sigma, exponent);
  const auto x = prepare(shared ? c.shared : c.x, sigma, exponent);
  std::vector<float> ft(T), fy(S), fx(K);
  for (int z = 0; z < T; ++z) ft[z] = frequency(z, T);
  for (int j = 0; j < S; ++j) fy[j] = frequency(j, S);
  for (int i = 0; i < K; ++i) fx[i] = frequency(i, S);
  // TableKernels::curve (kernels/scalar/table.cpp:17-30): exact knots return their
  // value, otherwise linear interpolation, then division by `div`.
  auto curve = [](float* out, const float* freq, std::size_t n, const Curve& knots, float div) {
    for (std::size_t i = 0; i < n; ++i) {
      auto hi = std::lower_bound(knots.begin(), knots.end(), freq[i],
                                 [](const auto& knot, float v) { return knot.first < v; });
      require(hi != knots.end(), "DFTTest frequency outside curve");
      float value;
      if (hi->first == freq[i]) value = hi->second;
      else {
        require(hi != knots.begin(), "DFTTest frequency outside curve");
        const auto lo = hi - 1;
        const float t = finite((freq[i] - lo->first) / (hi->first - lo->first));
        value = finite(finite(lo->second * (1 - t)) + finite(hi->second * t));
      }
      out[i] = finite(value / div);
    }
  };
  if (c.system == 1) {
    std::vector<float> radius(K);
    for (int z = 0; z < T; ++z)
      for (int j = 0; j < S; ++j) {
        const float other = ft[z] * ft[z] + fy[j] * fy[j];
        for (int i = 0; i < K; ++i)
          radius[i] = finite(std::sqrt(finite(finite(other + finite(fx[i] * fx[i])) / float(dims))));
        curve(result.data() + (std::size_t(z) * S + j) * K, radius.data(), radius.size(), time, divisor);
      }
  } else {
    std::vector<float> vt(T), vy(S), vx(K);
    if (T == 1) vt[0] = 1;
    else curve(vt.data(), ft.data(), ft.size(), time, 1);
    if (S == 1) {
      vy[0] = 1;
      vx[0] = 1;
    } else {
      curve(vy.data(), fy.data(), fy.size(), y, 1);
      curve(vx.data(), fx.data(), fx.size(), x, 1);
    }
    for (int z = 0; z < T; ++z)
      for (int j = 0; j < S; ++j) {
        const float factor = finite(vt[z] * vy[j]);
        float* out = result.data() + (std::size_t(z) * S + j) * K;
        for (int i = 0; i < K; ++i) out[i] = finite(finite(factor * vx[i]) / divisor);
      }
  }
  return result;
}

// --- FFT3D analytic profile and enhancement (src/algorithms/fft3d_profile.cpp:13-68) ---
std::vector<float> fft3d_profile(int W, int H, const float s[4]) {
  require(W >= 2 && H >= 2, "FFT3D profile shape invalid");
  for (int i = 0; i < 4; ++i) require(std::isfinite(s[i]) && s[i] >= 0, "FFT3D invalid scaled sigma");
  const int K = W / 2 + 1;
  const float norm = 1 / (float(W) * float(H));
  std::vector<float> p(std::size_t(H) * K), fx(K);
  for (int x = 0; x < K; ++x) fx[x] = float(x) / float(K);
  const float a = std::sqrt(.5f) / 4, b = std::sqrt(.5f) / 2;
  for (int y = 0; y < H; ++y) {
    const float fy = float(H - 2 * std::abs(y - H / 2)) / float(H);
    const float other = fy * fy;
    for (int x = 0; x < K; ++x) {
      // TableKernels::radius then ::analytic (kernels/scalar/table.cpp:5-16).
      const float f = finite(std::sqrt(finite(finite(other + finite(fx[x] * fx[x])) / 2.0f)));
      const float v = f < a ? finite(s[3] + finite(finite((s[2] - s[3]) * f) / a))
                      : f < b ? finite(s[2] + finite(finite((s[1] - s[2]) * (f - a)) / (b - a)))
                              : finite(s[0] + finite(finite((s[1] - s[0]) * (1 - f)) / (1 - b)));
      p[std::size_t(y) * K + x] = finite(finite(v * v) / norm);
    }
  }
  return p;
}
Enhancement enhancement_tables(int W, int H, float factor, const nf_fft3d_config& c) {
  validate_enhancement(c);
  require(W >= 2 && H >= 2 && std::isfinite(factor) && factor > 0, "FFT3D invalid enhancement geometry");
  Enhancement r;
  r.sharpen = c.sharpen;
  r.dehalo = c.dehalo;
  if (c.sharpen == 0 && c.dehalo == 0) return r;
  const float norm = 1 / (float(W) * float(H));
  float cutoff = 1;
  if (c.sharpen != 0) {
    const float lo = finite(c.smin * factor), hi = finite(c.smax * factor);
    r.a = finite(finite(lo * lo) / norm);
    r.b = finite(finite(hi * hi) / norm);
    cutoff = finite(finite(2 * c.scutoff) * c.scutoff);
    require(cutoff > 0, "FFT3D sharpen cutoff underflow");
  }
  if (c.dehalo != 0) r.c = finite(finite(c.ht * c.ht) / norm);
  const std::size_t count = std::size_t(H) * (W / 2 + 1);
  if (c.sharpen != 0) r.sharpen_window.resize(count);
  if (c.dehalo != 0) r.halo_window.resize(count);
  const int K = W / 2 + 1;
  std::vector<float> x2(K);
  for (int x = 0; x < K; ++x) x2[x] = float(x) * float(x) / (float(W / 2) * float(W / 2));
  for (int y = 0; y < H; ++y) {
    const float dy = float(y < H / 2 ? y : H - y);
    const float y2 = finite(finite(finite(dy * dy) * c.svr) * c.svr) / (float(H / 2) * float(H / 2));
    const std::size_t off = std::size_t(y) * K;
    // TableKernels::enhancement (kernels/scalar/table.cpp:39-49).
    for (int i = 0; i < K; ++i) {
      const float d2 = finite(y2 + x2[i]);
      if (c.sharpen != 0) r.sharpen_window[off + i] = finite(1 - std::exp(finite(-d2 / cutoff)));
      if (c.dehalo != 0) {
        const float first = finite(finite(finite(-.7f * d2) * c.hr) * c.hr);
        const float second = finite(finite(-d2 * c.hr) * c.hr);
        r.halo_window[off + i] = finite(std::exp(first) - std::exp(second));
      }
    }
  }
  float maximum = 0;
  for (float v : r.halo_window) maximum = std::max(maximum, v);
  if (c.dehalo != 0) {
    require(std::isfinite(maximum) && maximum > 0, "FFT3D degenerate dehalo window");
    for (float& v : r.halo_window) v = finite(v / maximum);
  }
  return r;
}

// --- temporal lattice (src/algorithms/temporal_grid.hpp:5-40) ---
void validate_temporal(int size, int mode, int overlap) {
  require(mode == 0 || mode == 1, "DFTTest tmode outside 0..1");
  require(size >= 1 && size <= 15, "DFTTest tbsize outside 1..15");
  require(mode != 0 || size % 2 == 1, "DFTTest centered tbsize must be odd");
  if (mode == 1) {
    require(overlap >= 0 && overlap < size, "DFTTest invalid tosize");
    require(overlap <= size / 2 || size % (size - overlap) == 0,
            "DFTTest temporal heavy overlap requires divisible step");
  }
}
static long long floor_div(long long v, int d) {
  require(d > 0, "invalid temporal divisor");
  return v / d - (v % d < 0);
}
std::vector<TemporalBlock> temporal_blocks(int frame, int length, int size, int overlap) {
  validate_temporal(size, 1, overlap);
  require(length >= size && frame >= 0 && frame < length, "invalid temporal clip/index");
  const int step = size - overlap;
  const long long anchor = -std::max(step, overlap), n = frame;
  const long long first = std::max(0LL, floor_div(n - size - anchor, step) + 1);
  const long long last = floor_div(n - anchor, step);
  std::vector<TemporalBlock> blocks;
  for (long long j = first; j <= last; ++j) {
    const long long start = anchor + j * step;
    TemporalBlock b{start, int(n - start), {}};
    for (int z = 0; z < size; ++z) b.slots[z] = int(std::clamp(start + z, 0LL, (long long)length - 1));
    blocks.push_back(b);
  }
  return blocks;
}

std::vector<cf> twiddle_table(int n) {
  std::vector<cf> t(std::size_t(std::max(n, 1)));
  for (int m = 0; m < n; ++m) {
    const double a = 2.0 * 3.14159265358979323846264338327950288 * double(m) / double(n);
    t[std::size_t(m)] = {float(std::cos(a)), float(-std::sin(a))};
  }
  return t;
}
void host_r2c_2d(const float* in, cf* out, int h, int w) {
  const auto th = twiddle_table(h), tw = twiddle_table(w);
  nf::block_r2c(in, w, out, w / 2 + 1, h, w, th.data(), tw.data());
}
void host_r2c_3d(const float* in, cf* out, int t, int h, int w) {
  const int K = w / 2 + 1;
  const std::size_t samples = std::size_t(h) * w, bins = std::size_t(h) * K;
  for (int z = 0; z < t; ++z) host_r2c_2d(in + z * samples, out + z * bins, h, w);
  if (t > 1) {
    const auto tt = twiddle_table(t);
    std::vector<cf> line(static_cast<std::size_t>(t));
    for (std::size_t k = 0; k < bins; ++k) {
      for (int z = 0; z < t; ++z) line[std::size_t(z)] = out[std::size_t(z) * bins + k];
      nf::fft_project<true, 0>(line.data(), t, tt.data());
      for (int z = 0; z < t; ++z) out[std::size_t(z) * bins + k] = line[std::size_t(z)];
    }
  }
}

// --- Plan(FFT3D) (src/algorithms/plan.cpp:91-169) ---
PlanTables build_fft3d(int w, int h, nf_format f, const nf_fft3d_config& c) {
  validate_fft3d(c);
  PlanTables p;
  p.algo = Algo::FFT3D;
  p.format = f;
  p.gx = fft3d_axis(w, c.bw, c.ow);
  p.gy = fft3d_axis(h, c.bh, c.oh);
  check_geometry(p.gx, p.gy);
  p.temporal_size = std::max(1, c.bt);
  p.bh = dimension(c.bh);
  p.bw = dimension(c.bw);
  p.bins = c.bh * (c.bw / 2 + 1);
  gpu_block_limits(c.bh, c.bw, 1);
  p.denoise = c.bt != -1;
  p.wx = fft3d_window(c.bw, p.gx.overlap, c.wintype);
  p.wy = fft3d_window(c.bh, p.gy.overlap, c.wintype);
  p.mean_scale = c.degrid;
  valid_format(f);
  const float factor = f.floating ? 1.0f / 255 : float(1 << (f.bits - 8));
  p.sampled = c.pfactor > 0;
  p.sigma_eff = p.sampled ? 0 : finite(c.sigma * factor);
  p.norm = 1.0f / (float(c.bw) * float(c.bh));
  p.beta = c.beta;
  float sigmas[4] = {0, 0, 0, 0};
  if (!p.sampled) {
    sigmas[0] = p.sigma_eff;
    sigmas[1] = finite((c.has_sigma2 ? c.sigma2 : c.sigma) * factor);
    sigmas[2] = finite((c.has_sigma3 ? c.sigma3 : c.sigma) * factor);
    sigmas[3] = finite((c.has_sigma4 ? c.sigma4 : c.sigma) * factor);
  }
  p.varying = sigmas[1] != sigmas[0] || sigmas[2] != sigmas[0] || sigmas[3] != sigmas[0];
  p.preview = c.pshow && (p.sampled || p.varying);
  p.denoise = p.denoise && !p.preview;
  p.kalman = c.bt == 0 && !p.preview;
  if (p.kalman) {
    p.sigma_eff = finite(c.sigma * factor);
    p.kalman_r0 = finite((p.sigma_eff * p.sigma_eff) / p.norm);
    p.kalman_ratio2 = finite(c.kratio * c.kratio);
  }
  p.spectral.type = -1;
  p.spectral.floor = (c.beta - 1) / c.beta;
  if (p.denoise && !p.sampled) {
    if (p.varying) {
      p.spectral.primary = fft3d_profile(c.bw, c.bh, sigmas);
      for (float v : p.spectral.primary) finite(float(p.temporal_size) * v);
    } else {
      p.spectral.a = finite((p.sigma_eff * p.sigma_eff) / p.norm);
      for (int T = 1; T <= p.temporal_size; ++T) finite(((float(T) * p.sigma_eff) * p.sigma_eff) / p.norm);
    }
  }
  if (p.kalman && !p.sampled) {
    if (p.spectral.primary.empty()) finite(p.kalman_r0 * p.kalman_ratio2);
    else
      for (float r : p.spectral.primary) finite(std::max(r, 1e-15f) * p.kalman_ratio2);
  }
  if (!p.preview) p.enhancement = enhancement_tables(c.bw, c.bh, factor, c);
  if (!p.preview && !p.enhancement.active()) p.enhancement = Enhancement{};
  p.spectral.fused_enhancement = !p.varying && !p.sampled && p.denoise && p.enhancement.active();
  p.pfactor = c.pfactor;
  p.px = c.px;
  p.py = c.py;
  p.pframe = c.pframe;
  p.kalman_warmup = c.kalman_warmup;
  p.needs_pattern = p.sampled && p.denoise;
  if (p.preview || p.needs_pattern) {
    // plan.cpp:142-158: candidate grid and the scoring weights q/(q+cutoff^2) with
    // q = fx^2 + fy^2 on normalised frequencies.
    if (c.px == 0 && c.py == 0)
      require(p.gx.count >= 5 && p.gy.count >= 5, "FFT3D automatic pattern search requires a 5x5 grid");
    else
      require(c.px < p.gx.count && c.py < p.gy.count, "FFT3D pattern coordinates outside grid");
    const float cutoff2 = finite(c.pcutoff * c.pcutoff);
    require(cutoff2 > 0, "FFT3D pattern cutoff underflow");
    const int K = c.bw / 2 + 1;
    std::vector<float> fx(static_cast<std::size_t>(K));
    for (int x = 0; x <= c.bw / 2; ++x) fx[std::size_t(x)] = 2 * float(x) / float(c.bw);
    p.sample_weights.resize(std::size_t(c.bh) * K);
    for (int y = 0; y < c.bh; ++y) {
      const float fy = 2 * float(std::min(y, c.bh - y)) / float(c.bh);
      const float other = fy * fy;
      for (int x = 0; x < K; ++x) {
        const float q = finite(other + finite(fx[std::size_t(x)] * fx[std::size_t(x)]));
        p.sample_weights[std::size_t(y) * K + x] = finite(q / finite(q + cutoff2));
      }
    }
  }
  if (c.degrid != 0) {
    std::vector<float> block(std::size_t(c.bh) * c.bw);
    const float peak = f.floating ? 1.0f : float((1 << f.bits) - 1);
    for (int y = 0; y < c.bh; ++y)
      for (int x = 0; x < c.bw; ++x) block[std::size_t(y) * c.bw + x] = (peak * p.wy.analysis[y]) * p.wx.analysis[x];
    p.grid.resize(std::size_t(p.bins));
    host_r2c_2d(block.data(), p.grid.data(), c.bh, c.bw);
    require(p.grid[0].r != 0, "FFT3D unusable grid DC");
  }
  return p;
}

// --- Plan(DFTTest) (src/algorithms/plan.cpp:170-226) ---
PlanTables build_dft(int w, int h, nf_format f, const nf_dft_config& c) {
  validate_dft(c);
  PlanTables p;
  p.algo = Algo::DFTTest;
  p.format = f;
  p.gx = dft_axis(w, c.block, c.mode, c.overlap);
  p.gy = dft_axis(h, c.block, c.mode, c.overlap);
  check_geometry(p.gx, p.gy);
  p.temporal_size = c.tbsize;
  p.bh = p.bw = dimension(c.block);
  p.bins = c.block * (c.block / 2 + 1);
  gpu_block_limits(c.block, c.block, c.tbsize);
  p.mean_scale = c.zmean ? 1.0f : 0.0f;
  p.center = c.mode == 0;
  valid_format(f);
  p.temporal_ola = c.temporal_mode == 1;
  p.temporal_overlap = c.temporal_overlap;
  p.dither = c.dither;
  p.dither_seed = c.dither_seed;
  auto win = dft_window_3d(c.tbsize, c.block, c.mode == 0 ? 0 : c.overlap, c.mode, c.swin, c.twin, c.sbeta, c.tbeta,
                           c.temporal_mode, c.temporal_overlap);
  p.h = std::move(win.h);
  p.wscale = win.wscale;
  p.h_synthesis.resize(p.h.size());
  const float volume = float(c.tbsize) * float(c.block) * float(c.block);
  for (std::size_t i = 0; i < p.h.size(); ++i) p.h_synthesis[i] = p.h[i] * volume;
  const bool sampled = c.ftype < 2 && c.n_nlocation > 0;
  if (sampled) {
    (void)dft_noise_setup(c);  // the reference builds its DFTNoise inside Plan (plan.cpp:193-198)
    p.noise_model = true;
  }
  const Curves curves = curves_of(c);
  const float scale = c.ftype < 2 ? p.wscale : 1.0f;
  p.spectral.type = c.ftype;
  p.spectral.a = !sampled && curves.empty() ? finite(c.sigma / scale) : 0;
  p.spectral.b = finite(c.sigma2 / scale);
  p.spectral.low = finite(c.pmin / p.wscale);
  p.spectral.high = finite(c.pmax / p.wscale);
  p.spectral.exponent = c.f0beta;
  p.spectral.floor = 0;
  if (!sampled && !curves.empty()) p.spectral.primary = dft_profile(curves, c.tbsize, c.block, c.sigma, scale);
  if (c.zmean) {
    auto block = p.h;
    for (float& v : block) v = finite(255.0f * v);
    p.grid.resize(std::size_t(c.tbsize) * p.bins);
    host_r2c_3d(block.data(), p.grid.data(), c.tbsize, c.block, c.block);
    require(p.grid[0].r != 0, "DFTTest zmean requires nonzero template DC");
  }
  return p;
}

} // namespace nfb

namespace nfb {

// --- DFTNoise (src/algorithms/dft_noise.cpp:5-41) ---
DftNoiseSetup dft_noise_setup(const nf_dft_config& c) {
  validate_dft(c);
  require(c.ftype < 2 && c.n_nlocation > 0, "inactive DFTTest sample model");
  DftNoiseSetup s;
  s.temporal_size = c.tbsize;
  s.block = c.block;
  s.bins3 = c.tbsize * c.block * (c.block / 2 + 1);
  s.zmean = c.zmean != 0;
  const DftWindow sample = dft_window_3d(c.tbsize, c.block, 0, 0, c.swin, c.twin, c.sbeta, c.tbeta, 0, 0);
  const DftWindow output = dft_window_3d(c.tbsize, c.block, c.mode == 0 ? 0 : c.overlap, c.mode, c.swin, c.twin,
                                         c.sbeta, c.tbeta, c.temporal_mode, c.temporal_overlap);
  const float alpha = c.has_alpha ? c.alpha : (c.ftype == 0 ? 5.0f : 7.0f);
  s.calibration = finite(finite((1.0f / float(c.n_nlocation)) * finite(sample.wscale / output.wscale)) * alpha);
  s.window = sample.h;
  std::vector<float> input(s.window.size());
  for (std::size_t i = 0; i < input.size(); ++i) input[i] = 255.0f * s.window[i];
  s.grid.resize(std::size_t(s.bins3));
  host_r2c_3d(input.data(), s.grid.data(), c.tbsize, c.block, c.block);
  for (const cf& g : s.grid) {
    finite(g.r);
    finite(g.i);
  }
  require(!s.zmean || s.grid[0].r != 0, "DFTTest sample template DC must be nonzero");
  return s;
}

std::vector<float> dft_noise_power(const nf_dft_config& c, const float* slices, int nlocations) {
  const DftNoiseSetup s = dft_noise_setup(c);
  require(slices != nullptr && nlocations == c.n_nlocation, "DFTTest noise slices differ from nlocation");
  const std::size_t samples = s.window.size();
  std::vector<float> input(samples), sum(std::size_t(s.bins3), 0.0f);
  std::vector<cf> spectrum(std::size_t(s.bins3));
  for (int l = 0; l < nlocations; ++l) {
    const float* in = slices + std::size_t(l) * samples;
    for (std::size_t i = 0; i < samples; ++i) input[i] = finite((in[i] * 1.0f) * s.window[i]);
    host_r2c_3d(input.data(), spectrum.data(), s.temporal_size, s.block, s.block);
    const float ratio = s.zmean ? finite(spectrum[0].r / s.grid[0].r) : 0.0f;
    for (int k = 0; k < s.bins3; ++k) {
      const float re = spectrum[k].r - (s.zmean ? ratio * s.grid[k].r : 0.0f);
      const float im = spectrum[k].i - (s.zmean ? ratio * s.grid[k].i : 0.0f);
      const float q = finite((re * re) + (im * im));
      sum[k] = finite(sum[k] + q);
    }
  }
  for (float& v : sum) {
    v = s.calibration * v;
    finite(1.0f * v);
  }
  return sum;
}

} // namespace nfb
