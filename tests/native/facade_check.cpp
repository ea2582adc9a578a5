// Test-only: exercises include/neo_fft_b200/plan.hpp the way the reference's host
// layer does (src/plugin/filter.hpp:349-360: process_at with sources, frame, plane,
// targets and cache arguments; Kalman initial/advance/render with copied states).
// Prints FNV-1a checksums of the outputs for comparison with the Python path.
#include "neo_fft_b200/checkpoints.hpp"
#include "neo_fft_b200/plan.hpp"

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <vector>

static std::uint64_t fnv(const void* p, std::size_t n) {
  std::uint64_t h = 1469598103934665603ull;
  const auto* b = static_cast<const unsigned char*>(p);
  for (std::size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
  return h;
}

int main() {
  using namespace neo_fft;
  const int w = 96, h = 64;
  std::vector<std::uint16_t> src(std::size_t(w) * h), dst(src.size());
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) src[std::size_t(y) * w + x] = std::uint16_t((x * 37 + y * 101 + (x * y) % 17) * 29 % 60000);
  DFTConfig c;
  c.block = 16; c.overlap = 12; c.sigma = 8; c.curves.shared = {0, 8, 1, 8};
  Plan plan(w, h, SampleFormat{16, false, false}, c);
  span2d::Plane<const std::uint16_t> s(src.data(), w, h, w * 2);
  span2d::Plane<std::uint16_t> d(dst.data(), w, h, w * 2);
  plan.process_at<std::uint16_t>({&s, 1}, d, 0, 0, {}, static_cast<runtime::SpectraCache*>(nullptr));
  std::printf("dft %llu\n", (unsigned long long)fnv(dst.data(), dst.size() * 2));
  // the Workspace& overloads and the plan's pool (plan.hpp:62-75, 98): two leases at once,
  // one idle workspace kept afterwards (tests/unit/execution.cpp:15-18 checks the same)
  {
    auto& pool = plan.workspace_pool();
    std::printf("pool_capacity %zu\n", pool.max_capacity());
    {
      auto one = pool.acquire(), two = pool.acquire();
      std::printf("pool_active %zu\n", pool.active_count());
      std::fill(dst.begin(), dst.end(), std::uint16_t(0));
      plan.process<std::uint16_t>(s, d, *one);
      std::printf("dft_ws %llu\n", (unsigned long long)fnv(dst.data(), dst.size() * 2));
      std::fill(dst.begin(), dst.end(), std::uint16_t(0));
      plan.process<std::uint16_t>({&s, 1}, d, *two);
      std::printf("dft_ws_span %llu\n", (unsigned long long)fnv(dst.data(), dst.size() * 2));
    }
    std::printf("pool_idle %zu pool_budget %zu\n", pool.idle_count(), pool.budget().total_bytes);
    // copy_row() copies a host row (filter.hpp passes it to PackedROI)
    std::vector<std::uint16_t> row(static_cast<std::size_t>(w));
    plan.copy_row()(src.data() + std::size_t(w) * 5, row.data(), std::size_t(w) * 2);
    std::printf("copy_row %d\n", int(std::equal(row.begin(), row.end(), src.begin() + std::size_t(w) * 5)));
  }

  FFT3DConfig k;
  k.bt = 0; k.sigma = 2.5f; k.kratio = 2.0f; k.bw = k.bh = 16;
  std::vector<float> fsrc(std::size_t(w) * h), fdst(fsrc.size());
  for (std::size_t i = 0; i < fsrc.size(); ++i) fsrc[i] = float((i * 7919) % 1000) / 1000.0f;
  Plan kp(w, h, SampleFormat{32, true, false}, k);
  span2d::Plane<const float> fs(fsrc.data(), w, h, w * 4);
  span2d::Plane<float> fd(fdst.data(), w, h, w * 4);
  KalmanState st = kp.initial_kalman();
  for (int f = 0; f < 3; ++f) kp.advance_kalman<float>(fs, st);
  KalmanState copy = st;  // checkpoint copy (filter.hpp:171)
  kp.render_kalman<float>(fs, fd, copy);
  std::printf("kalman %llu\n", (unsigned long long)fnv(fdst.data(), fdst.size() * 4));
  // random-access Kalman frames through the checkpoint policy (filter.hpp:152-250)
  std::vector<std::vector<float>> frames(24, std::vector<float>(fsrc.size()));
  for (int f = 0; f < 24; ++f)
    for (std::size_t i = 0; i < fsrc.size(); ++i) frames[f][i] = float((i * 7919 + std::size_t(f) * 104729) % 1000) / 1000.0f;
  KalmanSeek seek({&kp, nullptr, nullptr, nullptr}, 4);
  for (int n : {5, 6, 7, 20, 3, 21}) {
    auto source = [&](int f) { return span2d::Plane<const float>(frames[f].data(), w, h, w * 4); };
    seek.frame(
        n, [&](const Plan& p, int, int f, KalmanState& s) { p.advance_kalman<float>(source(f), s); },
        [&](const Plan* p, int, const KalmanState* s) {
          if (p && s) p->render_kalman<float>(source(n), fd, *s);
        });
    std::printf("seek%d %llu\n", n, (unsigned long long)fnv(fdst.data(), fdst.size() * 4));
  }
  // sampled FFT3D model: prepare_pattern on a frame, then filter another
  {
    FFT3DConfig pc;
    pc.bw = pc.bh = 16; pc.ow = pc.oh = 8; pc.pfactor = 1.0f;
    std::vector<std::uint8_t> a(std::size_t(w) * h), b(a.size()), o(a.size());
    for (std::size_t i = 0; i < a.size(); ++i) {
      a[i] = std::uint8_t((i * 131 + (i / w) * 7) % 200 + 20);
      b[i] = std::uint8_t((i * 97 + (i / w) * 13) % 180 + 30);
    }
    Plan pp(w, h, SampleFormat{8, false, false}, pc);
    std::printf("pattern_needed %d\n", int(pp.needs_pattern_frame() && !pp.pattern_ready()));
    pp.prepare_pattern<std::uint8_t>({a.data(), w, h, w});
    span2d::Plane<const std::uint8_t> bs(b.data(), w, h, w);
    pp.process_at<std::uint8_t>({&bs, 1}, span2d::Plane<std::uint8_t>(o.data(), w, h, w), 0, 0);
    std::printf("pattern %llu\n", (unsigned long long)fnv(o.data(), o.size()));
  }
  try {
    FFT3DConfig bad;
    bad.bt = 7;
    Plan p2(w, h, SampleFormat{8, false, false}, bad);
  } catch (const std::invalid_argument& e) {
    std::printf("error %s\n", e.what());
  }
  return 0;
}
