// A bounded shelf of Kalman state snapshots keyed by frame number.
//
// Observable policy (the one the host layer's random-access replay depends on,
// src/runtime/checkpoints.hpp:32-79): at most four snapshots; a lookup returns the
// snapshot with the highest frame inside [earliest, frame]; frames below 1 are never
// stored; while a snapshot of a frame is held, a newer snapshot of the same frame is
// dropped (histories can differ after a seek, and the held one may be in use); a new
// snapshot evicts least-recently-used ones until it fits the byte budget and a slot is
// free. With `keep_oversized`, a snapshot larger than the whole budget is still kept
// (alone), so large geometries can continue sequentially.
//
// Mechanism: every lookup hit and every store stamps the slot with the next value of a
// use counter; the slot with the smallest stamp is the least recently used.
#pragma once
#include <array>
#include <cstddef>
#include <cstdint>
#include <utility>

namespace neo_fft {

template <class Payload>
class SnapshotShelf {
 public:
  static constexpr int kSlots = 4;

  SnapshotShelf(std::size_t budget, bool keep_oversized) : budget_(budget), keep_oversized_(keep_oversized) {}

  // The held payload with the highest frame in [earliest, frame], marked as used, and
  // its frame in *found; nullptr when there is none.
  Payload* latest(int frame, int earliest, int* found = nullptr) {
    Slot* hit = nullptr;
    for (Slot& s : slots_)
      if (s.frame >= earliest && s.frame >= 1 && s.frame <= frame && (!hit || s.frame > hit->frame)) hit = &s;
    if (!hit) return nullptr;
    hit->stamp = ++clock_;
    if (found) *found = hit->frame;
    return &hit->payload;
  }

  // Offers a snapshot of `frame` occupying `bytes`. Returns true when it was stored;
  // otherwise the caller keeps (and disposes of) the payload. `evict(payload&)` is
  // called for each snapshot removed to make room, before it is overwritten.
  template <class Evict>
  bool offer(int frame, Payload&& payload, std::size_t bytes, Evict&& evict) {
    if (frame < 1) return false;
    const std::size_t cap = keep_oversized_ && bytes > budget_ ? bytes : budget_;
    if (bytes > cap) return false;
    for (Slot& s : slots_)
      if (s.frame == frame) {  // the snapshot already held for this frame stays
        s.stamp = ++clock_;
        return false;
      }
    for (;;) {
      int held = 0;
      Slot* lru = nullptr;
      for (Slot& s : slots_)
        if (s.frame >= 1) {
          ++held;
          if (!lru || s.stamp < lru->stamp) lru = &s;
        }
      if (held < kSlots && used_ + bytes <= cap) break;
      evict(lru->payload);
      used_ -= lru->bytes;
      lru->frame = -1;
      lru->bytes = 0;
      lru->payload = Payload{};
    }
    for (Slot& s : slots_)
      if (s.frame < 1) {
        s.frame = frame;
        s.payload = std::move(payload);
        s.bytes = bytes;
        s.stamp = ++clock_;
        used_ += bytes;
        return true;
      }
    return false;  // unreachable: the loop above left a free slot
  }

  // Removes every snapshot (evict(payload&) for each).
  template <class Evict>
  void clear(Evict&& evict) {
    for (Slot& s : slots_)
      if (s.frame >= 1) {
        evict(s.payload);
        s.frame = -1;
        s.bytes = 0;
        s.payload = Payload{};
      }
    used_ = 0;
  }

  std::size_t used_bytes() const { return used_; }
  int held() const {
    int n = 0;
    for (const Slot& s : slots_) n += s.frame >= 1 ? 1 : 0;
    return n;
  }
  // Frame of slot i (-1 when empty), for inspection.
  int frame_at(int i) const { return slots_[std::size_t(i)].frame; }

 private:
  struct Slot {
    int frame = -1;
    Payload payload{};
    std::size_t bytes = 0;
    std::uint64_t stamp = 0;
  };
  std::array<Slot, kSlots> slots_{};
  std::uint64_t clock_ = 0;
  std::size_t used_ = 0;
  const std::size_t budget_;
  const bool keep_oversized_;
};

}  // namespace neo_fft
