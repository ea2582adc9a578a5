// Kalman checkpoints and bounded-warmup seeks over device-resident states.
//
// neo_fft::KalmanCheckpoints keeps up to four snapshots of the per-plane Kalman states
// (each a device allocation, copied device to device) with the reference's policy
// (src/runtime/checkpoints.hpp:32-79): acquire(frame, earliest) leases the latest
// snapshot in [earliest, frame]; publish() ignores frame < 1 and frames already held,
// then evicts least-recently used snapshots until the new one fits the budget. The
// default budget is 64 MiB and always retains one snapshot even when a single one is
// larger (large geometries keep continuing sequentially); an explicit budget is hard.
//
// neo_fft::KalmanSeek reproduces the host layer's random-access rule
// (src/plugin/filter.hpp:152-250): frame 0 is passed through; for frame n > 0 the
// latest snapshot not older than n - warmup - 1 is continued, or the initial state is
// advanced over the warmup frames n - warmup .. n (frames 1 .. n when n <= warmup);
// the frame is rendered from that state and the new state is published.
#pragma once
#include "neo_fft_b200/plan.hpp"

#include <array>
#include <cstddef>
#include <functional>
#include <memory>
#include <mutex>

namespace neo_fft {

struct KalmanCheckpoint {
  int frame = 0;
  std::array<KalmanState, 4> planes;
  std::size_t bytes() const {
    std::size_t n = sizeof(*this);
    for (const auto& p : planes) n += p.bytes() - sizeof(p);
    return n;
  }
};

class KalmanCheckpoints {
 public:
  using Lease = std::shared_ptr<const KalmanCheckpoint>;
  KalmanCheckpoints() : budget_(64u << 20), retain_one_(true) {}
  explicit KalmanCheckpoints(std::size_t budget) : budget_(budget), retain_one_(false) {}

  Lease acquire(int frame, int earliest = 0) {
    std::lock_guard<std::mutex> lock(mutex_);
    Slot* best = nullptr;
    for (auto& s : slots_)
      if (s.value && s.value->frame >= earliest && s.value->frame <= frame && (!best || s.value->frame > best->value->frame))
        best = &s;
    if (!best) return {};
    touch(*best);
    return best->value;
  }

  void publish(std::unique_ptr<KalmanCheckpoint> owned) {
    if (!owned || owned->frame < 1) return;
    Lease value(owned.release());
    const std::size_t need = sizeof(*this) + value->bytes();
    const std::size_t limit = retain_one_ && need > budget_ ? need : budget_;
    if (need > limit) return;
    std::lock_guard<std::mutex> lock(mutex_);
    for (auto& s : slots_)
      if (s.value && s.value->frame == value->frame) {  // first snapshot of a frame wins
        touch(s);
        return;
      }
    while (used_ > limit - need || held() == slots_.size()) {
      Slot* oldest = nullptr;
      for (auto& s : slots_)
        if (s.value && (!oldest || s.age > oldest->age)) oldest = &s;
      used_ -= oldest->value->bytes();
      oldest->value.reset();
    }
    for (auto& s : slots_)
      if (!s.value) {
        used_ += value->bytes();
        s.value = std::move(value);
        s.age = 4;
        touch(s);
        break;
      }
  }

  std::size_t bytes() const {
    std::lock_guard<std::mutex> lock(mutex_);
    return used_ + sizeof(*this);
  }

 private:
  struct Slot {
    Lease value;
    unsigned age = 0;
  };
  void touch(Slot& selected) {
    for (auto& s : slots_)
      if (s.value && &s != &selected && s.age < selected.age) ++s.age;
    selected.age = 0;
  }
  std::size_t held() const {
    std::size_t n = 0;
    for (const auto& s : slots_) n += s.value ? 1 : 0;
    return n;
  }
  std::array<Slot, 4> slots_{};
  const std::size_t budget_;
  const bool retain_one_;
  std::size_t used_ = 0;
  mutable std::mutex mutex_;
};

// One plane set's Kalman filter with random-access frame requests.
class KalmanSeek {
 public:
  // plans[p] may be null (plane not filtered); warmup is the host layer's kalman_warmup.
  KalmanSeek(std::array<const Plan*, 4> plans, int warmup, std::shared_ptr<KalmanCheckpoints> checkpoints =
                                                                  std::make_shared<KalmanCheckpoints>())
      : plans_(plans), warmup_(warmup), checkpoints_(std::move(checkpoints)) {}

  // advance(plan, plane, frame, state) consumes source frame `frame` of plane `plane`;
  // render(plan, plane, state) writes output frame n (state == nullptr: pass-through).
  using Advance = std::function<void(const Plan&, int, int, KalmanState&)>;
  using Render = std::function<void(const Plan*, int, const KalmanState*)>;

  void frame(int n, const Advance& advance, const Render& render) {
    if (n == 0) {
      for (int p = 0; p < 4; ++p) render(plans_[p], p, nullptr);
      return;
    }
    const int earliest = n > warmup_ ? n - warmup_ - 1 : 0;
    KalmanCheckpoints::Lease start = checkpoints_->acquire(n, earliest);
    const int replay_start = start ? start->frame : earliest;
    std::unique_ptr<KalmanCheckpoint> current;
    if (replay_start < n) {
      current = start ? std::make_unique<KalmanCheckpoint>(*start) : std::make_unique<KalmanCheckpoint>();
      if (!start)
        for (int p = 0; p < 4; ++p)
          if (plans_[p]) current->planes[p] = plans_[p]->initial_kalman();
      for (int f = replay_start + 1; f <= n; ++f) {
        for (int p = 0; p < 4; ++p)
          if (plans_[p]) advance(*plans_[p], p, f, current->planes[p]);
        current->frame = f;
      }
    }
    const KalmanCheckpoint* state = current ? current.get() : start.get();
    for (int p = 0; p < 4; ++p) render(plans_[p], p, state && plans_[p] ? &state->planes[p] : nullptr);
    if (current) checkpoints_->publish(std::move(current));
  }

  KalmanCheckpoints& checkpoints() { return *checkpoints_; }

 private:
  std::array<const Plan*, 4> plans_;
  int warmup_;
  std::shared_ptr<KalmanCheckpoints> checkpoints_;
};

} // namespace neo_fft
