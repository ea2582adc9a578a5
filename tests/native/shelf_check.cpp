// Test-only: the snapshot shelf's policy (include/neo_fft_b200/snapshot_shelf.hpp) on
// integer payloads, the same cases tests/test_checkpoints.py runs on the Python mirror.
// Prints one line per check; exits non-zero on the first failure.
#include "neo_fft_b200/snapshot_shelf.hpp"

#include <cstdio>
#include <vector>

using Shelf = neo_fft::SnapshotShelf<int>;

static int failures = 0;
static void expect(bool ok, const char* what) {
  std::printf("%s %s\n", ok ? "ok" : "FAIL", what);
  if (!ok) ++failures;
}
static std::vector<int> frames(const Shelf& s) {
  std::vector<int> f;
  for (int i = 0; i < Shelf::kSlots; ++i)
    if (s.frame_at(i) >= 1) f.push_back(s.frame_at(i));
  std::vector<int> sorted;
  for (int lo = 1 << 30; !f.empty();) {
    lo = f[0];
    size_t at = 0;
    for (size_t i = 1; i < f.size(); ++i)
      if (f[i] < lo) lo = f[i], at = i;
    sorted.push_back(lo);
    f.erase(f.begin() + long(at));
  }
  return sorted;
}

int main() {
  auto none = [](int&) {};
  {
    Shelf s(64 << 20, true);
    for (int f : {3, 9, 6}) s.offer(f, f * 10, 1000, none);
    int found = 0;
    int* p = s.latest(8, 0, &found);
    expect(p && *p == 60 && found == 6, "latest snapshot inside [0, 8] is frame 6");
    expect(s.latest(20, 0) && *s.latest(20, 0) == 90, "latest inside [0, 20] is frame 9");
    expect(!s.latest(8, 7), "nothing inside [7, 8]");
    expect(!s.latest(2, 0), "nothing inside [0, 2]");
  }
  {
    Shelf s(64 << 20, true);
    expect(!s.offer(0, 1, 1000, none) && s.held() == 0, "frame 0 is never stored");
    s.offer(4, 41, 1000, none);
    expect(!s.offer(4, 42, 1000, none) && *s.latest(4, 0) == 41, "the first snapshot of a frame stays");
  }
  {
    Shelf s(64 << 20, true);
    std::vector<int> evicted;
    for (int f : {1, 2, 3, 4}) s.offer(f, int(f), 1000, none);
    s.latest(1, 0);  // frame 1 becomes the most recently used
    s.offer(5, 5, 1000, [&](int& v) { evicted.push_back(v); });
    expect(frames(s) == std::vector<int>({1, 3, 4, 5}) && evicted == std::vector<int>({2}),
           "four slots, least recently used evicted");
  }
  {
    const size_t big = size_t(40) << 20;
    Shelf s(2 * big + (1 << 20), false);
    for (int f : {1, 2, 3}) s.offer(f, int(f), big, none);
    expect(frames(s) == std::vector<int>({2, 3}), "explicit budget evicts to fit");
    Shelf hard(1 << 20, false);
    expect(!hard.offer(1, 1, big, none) && hard.held() == 0, "explicit budget is hard");
    Shelf def(64 << 20, true);
    def.offer(1, 1, size_t(100) << 20, none);
    def.offer(2, 2, size_t(100) << 20, none);
    expect(frames(def) == std::vector<int>({2}), "default budget keeps one oversized snapshot");
  }
  return failures ? 1 : 0;
}
