// Test-only: the compile-time (fft_ct) and runtime forms of the project transform
// in neo_fft_b200/csrc/fft_core.cuh must be bit-identical, since kernels use the
// former and the host table builders (and the oracle backend) the latter.
#include "fft_core.cuh"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

namespace {
std::vector<nf::cf> table(int n) {
  std::vector<nf::cf> t(n);
  for (int m = 0; m < n; ++m) {
    const double a = 2.0 * 3.14159265358979323846264338327950288 * double(m) / double(n);
    t[m] = {float(std::cos(a)), float(-std::sin(a))};
  }
  return t;
}
template <int N>
int check(std::mt19937& rng) {
  const auto tw = table(N);
  std::normal_distribution<float> d(0.f, 1.f);
  int bad = 0;
  for (int trial = 0; trial < 20; ++trial) {
    nf::cf a[N], b[N];
    for (int i = 0; i < N; ++i) a[i] = b[i] = {d(rng), d(rng)};
    nf::fft_project<true, N>(a, N, tw.data());
    nf::fft_project<true, 0>(b, N, tw.data());
    if (std::memcmp(a, b, sizeof(a))) ++bad;
    nf::fft_project<false, N>(a, N, tw.data());
    nf::fft_project<false, 0>(b, N, tw.data());
    if (std::memcmp(a, b, sizeof(a))) ++bad;
  }
  return bad;
}
// The team form (lanes run one after another, the runs exchanged through a buffer)
// against the single-thread transform.
template <bool FWD, int N>
int check_team(std::mt19937& rng) {
  using Team = nf::TeamFFT<FWD, N>;
  const auto tw = table(N);
  std::normal_distribution<float> d(0.f, 1.f);
  int bad = 0;
  for (int trial = 0; trial < 20; ++trial) {
    nf::cf in[N], ref[N], buf[N], out[N];
    for (int i = 0; i < N; ++i) in[i] = ref[i] = {d(rng), d(rng)};
    nf::fft_project<FWD, N>(ref, N, tw.data());
    for (int t = 0; t < Team::T; ++t) {
      nf::cf local[Team::M];
      Team::run(t, local, tw.data(), [&](int k) { return in[k]; });
      for (int i = 0; i < Team::M; ++i) buf[t * Team::M + i] = local[i];
    }
    for (int t = 0; t < Team::T; ++t)
      Team::outer(t, tw.data(), [&](int j, int i) { return buf[j * Team::M + i]; },
                  [&](int x, nf::cf v) { out[x] = v; });
    if (std::memcmp(out, ref, sizeof(out))) ++bad;
  }
  return bad;
}
} // namespace

extern "C" int fft_team_mismatches() {
  std::mt19937 rng(11);
  return check_team<true, 48>(rng) + check_team<false, 48>(rng) + check_team<true, 64>(rng) +
         check_team<false, 64>(rng) + check_team<true, 32>(rng) + check_team<false, 96>(rng);
}

extern "C" int fft_forms_mismatches() {
  std::mt19937 rng(7);
  return check<2>(rng) + check<3>(rng) + check<4>(rng) + check<5>(rng) + check<6>(rng) + check<7>(rng) +
         check<8>(rng) + check<9>(rng) + check<12>(rng) + check<15>(rng) + check<16>(rng) + check<20>(rng) +
         check<24>(rng) + check<32>(rng) + check<48>(rng) + check<64>(rng) + check<11>(rng) + check<13>(rng);
}

namespace {
// Equal as numbers: +0 == -0 and NaN == NaN (the real-row forms may give an exact zero
// the other sign and nothing else).
bool same_value(float a, float b) { return (a != a && b != b) || a == b; }
bool same_bits(float a, float b) { return std::memcmp(&a, &b, sizeof a) == 0; }

float draw(std::mt19937& rng, bool structured) {
  std::normal_distribution<float> d(0.f, 1.f);
  if (!structured) return d(rng) * 300.0f;
  const float pool[] = {0.0f, -0.0f, 1.0f, -1.0f, 2.5f, 2.5f, 1e-38f, -3e-39f, 1e38f, -1e38f,
                        INFINITY, -INFINITY, NAN, 7.0f, 7.0f, 7.0f};
  const unsigned pick = rng() % 24u;
  return pick < 16 ? pool[pick] : d(rng);
}
} // namespace

// The real-row forms of the 16-point codelet transform (row_forward<16>,
// row_inverse<16>) against fft16 on complex data with zero imaginary parts and on the
// mirrored half spectrum: identical bits on generic data, identical values (zero signs
// aside, NaN where the other has NaN) on rows of zeros, repeats, infinities and NaNs.
extern "C" int fft16_real_mismatches(int structured) {
  std::mt19937 rng(structured ? 29 : 17);
  int bad = 0;
  auto same = [&](float a, float b) { return structured ? same_value(a, b) : same_bits(a, b); };
  for (int trial = 0; trial < 4000; ++trial) {
    float x[16];
    // structured rows: a flat row, a row of one repeated pair, or draws from the pool
    const int kind = structured ? trial % 3 : 2;
    for (int k = 0; k < 16; ++k) x[k] = kind == 0 ? 5.0f : kind == 1 ? (k & 1 ? -2.0f : 2.0f) : draw(rng, structured);
    if (structured && trial % 7 == 0) x[trial % 16] = -0.0f;
    nf::cf got[9], ref[16];
    nf::row_forward<16>(x, 16, got, nullptr, true);
    for (int k = 0; k < 16; ++k) ref[k] = {x[k], 0.0f};
    nf::fft16<true>(ref);
    ref[8].i = 0.0f;
    for (int k = 0; k < 9; ++k)
      if (!same(got[k].r, ref[k].r) || !same(got[k].i, ref[k].i)) ++bad;
    nf::cf bins[9];
    for (int k = 0; k < 9; ++k) bins[k] = {draw(rng, structured), draw(rng, structured)};
    if (structured && trial % 5 == 0)
      for (int k = 0; k < 9; ++k) bins[k] = bins[trial % 9];
    float out[16];
    const float fct = 1.0f / 256.0f;
    nf::row_inverse<16>(bins, 16, fct, out, nullptr, true);
    nf::cf a[16];
    for (int k = 0; k <= 8; ++k) a[k] = bins[k];
    for (int k = 1; k < 8; ++k) a[16 - k] = {bins[k].r, 0.0f - bins[k].i};
    nf::fft16<false>(a);
    for (int k = 0; k < 16; ++k)
      if (!same(out[k], a[k].r * fct)) ++bad;
  }
  return bad;
}

// The same check for the 32-point real-row forms against fft32.
extern "C" int fft32_real_mismatches(int structured) {
  std::mt19937 rng(structured ? 31 : 19);
  int bad = 0;
  auto same = [&](float a, float b) { return structured ? same_value(a, b) : same_bits(a, b); };
  for (int trial = 0; trial < 3000; ++trial) {
    float x[32];
    const int kind = structured ? trial % 3 : 2;
    for (int k = 0; k < 32; ++k) x[k] = kind == 0 ? 5.0f : kind == 1 ? (k & 1 ? -2.0f : 2.0f) : draw(rng, structured);
    if (structured && trial % 7 == 0) x[trial % 32] = -0.0f;
    nf::cf got[17], ref[32];
    nf::row_forward<32>(x, 32, got, nullptr, true);
    for (int k = 0; k < 32; ++k) ref[k] = {x[k], 0.0f};
    nf::fft32<true>(ref);
    ref[16].i = 0.0f;
    for (int k = 0; k < 17; ++k)
      if (!same(got[k].r, ref[k].r) || !same(got[k].i, ref[k].i)) ++bad;
    nf::cf bins[17];
    for (int k = 0; k < 17; ++k) bins[k] = {draw(rng, structured), draw(rng, structured)};
    if (structured && trial % 5 == 0)
      for (int k = 0; k < 17; ++k) bins[k] = bins[trial % 17];
    float out[32];
    const float fct = 1.0f / 1024.0f;
    nf::row_inverse<32>(bins, 32, fct, out, nullptr, true);
    nf::cf a[32];
    for (int k = 0; k <= 16; ++k) a[k] = bins[k];
    for (int k = 1; k < 16; ++k) a[32 - k] = {bins[k].r, 0.0f - bins[k].i};
    nf::fft32<false>(a);
    for (int k = 0; k < 32; ++k)
      if (!same(out[k], a[k].r * fct)) ++bad;
  }
  return bad;
}

// The runtime project transform of length n (1..kMaxProject, factors at most kMaxRadix; 1 is
// returned for other lengths) on interleaved complex data, forward or inverse (unnormalised),
// with the plan builders' binary32 twiddle table: the Python side compares it with a binary64
// DFT for every length.
extern "C" int project_fft(int n, int forward, const float* in, float* out) {
  if (n < 1 || n > nf::kMaxProject || nf::largest_radix(n) > nf::kMaxRadix) return 1;
  const auto tw = table(n);
  std::vector<nf::cf> a(static_cast<size_t>(n));
  for (int i = 0; i < n; ++i) a[size_t(i)] = {in[2 * i], in[2 * i + 1]};
  if (forward) nf::fft_project<true, 0>(a.data(), n, tw.data());
  else nf::fft_project<false, 0>(a.data(), n, tw.data());
  for (int i = 0; i < n; ++i) {
    out[2 * i] = a[size_t(i)].r;
    out[2 * i + 1] = a[size_t(i)].i;
  }
  return 0;
}
