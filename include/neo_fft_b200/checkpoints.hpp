// Kalman checkpoints and bounded-warmup seeks over device-resident states.
//
// neo_fft::KalmanCheckpoints keeps up to four snapshots of the per-plane Kalman states
// (each a device allocation, copied device to device) with the observable policy of the
// reference's runtime::Checkpoints (src/runtime/checkpoints.hpp:32-79), implemented by
// SnapshotShelf: acquire(frame, earliest) leases the latest snapshot in [earliest, frame];
// publish() ignores frame < 1 and frames already held, then evicts least-recently used
// snapshots until the new one fits the budget. The default budget is 64 MiB and always
// retains one snapshot even when a single one is larger (large geometries keep
// continuing sequentially); an explicit budget is hard.
//
// neo_fft::KalmanSeek reproduces the host layer's random-access rule
// (src/plugin/filter.hpp:152-250): frame 0 is passed through; for frame n > 0 the
// latest snapshot not older than n - warmup - 1 is continued, or the initial state is
// advanced over the warmup frames n - warmup .. n (frames 1 .. n when n <= warmup);
// the frame is rendered from that state and the new state is published.
#pragma once
#include "neo_fft_b200/plan.hpp"
#include "neo_fft_b200/snapshot_shelf.hpp"

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

// The snapshots of one plane set, held on a SnapshotShelf (snapshot_shelf.hpp): leases
// are shared, so a snapshot evicted while a request still continues from it stays alive
// until that request drops it.
class KalmanCheckpoints {
 public:
  using Lease = std::shared_ptr<const KalmanCheckpoint>;
  KalmanCheckpoints() : shelf_(std::size_t(64) << 20, true) {}
  explicit KalmanCheckpoints(std::size_t budget) : shelf_(budget, false) {}

  Lease acquire(int frame, int earliest = 0) {
    std::lock_guard<std::mutex> lock(mutex_);
    Lease* hit = shelf_.latest(frame, earliest);
    return hit ? *hit : Lease{};
  }

  void publish(std::unique_ptr<KalmanCheckpoint> owned) {
    if (!owned) return;
    const int frame = owned->frame;
    const std::size_t size = owned->bytes();
    Lease lease(owned.release());
    std::lock_guard<std::mutex> lock(mutex_);
    shelf_.offer(frame, std::move(lease), size, [](Lease&) {});
  }

  std::size_t bytes() const {
    std::lock_guard<std::mutex> lock(mutex_);
    return shelf_.used_bytes() + sizeof(*this);
  }

 private:
  SnapshotShelf<Lease> shelf_;
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
