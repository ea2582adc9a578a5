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
