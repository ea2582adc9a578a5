// Host request layer: the reference host layer's request/process pair
// (src/plugin/filter.hpp:253-528) over the batched forms of this library. Output frames
// are produced in ranges of consecutive frames; each range is one batched launch over
// device-resident source frames, and the next two ranges are fetched and computed in
// further banks of device buffers while the current one is read out.
//
// Frame selection per output frame n (clip of N frames) follows filter.hpp:
//   FFT3D bt 2..5       frames n - bt/2 .. n + (bt-1)/2, or n alone where that window
//                       leaves the clip (filter.hpp:267-279)
//   DFTTest tmode 0     slots clamp(n - T/2 + j, 0, N - 1) (filter.hpp:289-296)
//   DFTTest tmode 1     the covering temporal blocks (temporal_grid.hpp:5-40)
//   single-frame plans  frame n
#include "neo_fft_b200.h"
#include "plan_build.hpp"
#include "plan_info.hpp"
#include "neo_fft_b200/snapshot_shelf.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

enum class Kind { Copy, Single, ClipFFT3D, ClipDFT, PerFrame, Kalman };

struct Range {
  int n0 = 0, n1 = 0;  // outputs delivered: [n0, n1)
  int s0 = 0, s1 = 0;  // source frames fetched: [s0, s1) -> source slots 0 .. s1-s0-1
  int o0 = 0;          // clip frame of output slot 0
};

struct Failure {
  nf_status code;
  std::string msg;
};
[[noreturn]] void raise(nf_status code, const std::string& msg) { throw Failure{code, msg}; }
void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) raise(NF_DEVICE_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
}
void check(nf_status s, const char* err) {
  if (s != NF_OK) raise(s, err);
}

}  // namespace

struct nf_frame_server {
  struct Bank {
    unsigned char* src = nullptr;
    unsigned char* out = nullptr;
    int src_cap = 0, out_cap = 0;  // frames
    Range r;
    bool valid = false;
    bool checked = false;  // plan status read after the range's filtering
    unsigned long long used = 0;
    cudaStream_t stream = nullptr;
    std::map<int, nf_batch*> batches;       // keyed by frame count
    std::map<int, nf_clip_batch*> clips;    // keyed by sub-clip length
    void drop_forms() {
      for (auto& b : batches) nf_batch_destroy(b.second);
      for (auto& c : clips) nf_clip_batch_destroy(c.second);
      batches.clear();
      clips.clear();
    }
  };

  // FFT3D bt=0: snapshots of the per-plane Kalman states (device states, one per plane)
  // on a SnapshotShelf with the host layer's policy (runtime/checkpoints.hpp:32-79): up to
  // four, least recently used evicted first, a 64 MiB budget that always keeps one; the
  // first snapshot of a frame wins.
  using PlaneStates = std::vector<nf_kalman_state*>;
  static void release_states(PlaneStates& v) {
    for (nf_kalman_state*& k : v)
      if (k) {
        nf_kalman_state_destroy(k);
        k = nullptr;
      }
  }
  struct Snapshot {  // a state being advanced by a request, not yet on the shelf
    int frame = -1;
    PlaneStates planes;
    size_t bytes = 0;
  };
  static constexpr size_t kSnapshotBudget = size_t(64) << 20;
  neo_fft::SnapshotShelf<PlaneStates> snaps{kSnapshotBudget, true};
  int warmup = 8;

  std::vector<const nf_plan*> plans;  // per plane; nullptr: copied
  std::vector<nfi::PlanInfo> info;
  std::vector<size_t> pitch, offset;  // processed planes in a device frame slot
  size_t frame_bytes = 0;
  int planes = 0, N = 0, R = 1, T = 1, left = 0, right = 0, overlap = 0;
  Kind kind = Kind::Copy;
  bool preview = false;
  nf_frame_source source = nullptr;
  void* user = nullptr;
  static constexpr int kBanks = 3;  // the range being read out and two ranges ahead
  Bank banks[kBanks];
  unsigned long long tick = 0;
  long long computed = 0, fetched = 0;
  bool patterns_done = false;
  mutable std::mutex mu;

  ~nf_frame_server() {
    for (auto& b : banks)
      if (b.stream) cudaStreamSynchronize(b.stream);
    snaps.clear(release_states);
    for (auto& b : banks) {
      if (b.stream) cudaStreamSynchronize(b.stream);
      b.drop_forms();
      if (b.src) cudaFree(b.src);
      if (b.out) cudaFree(b.out);
      if (b.stream) cudaStreamDestroy(b.stream);
    }
  }

  // Source frames of output n, in slot order, with the temporal targets of DFTTest tmode 1.
  std::vector<int> slots(int n, std::vector<int>* targets = nullptr) const {
    std::vector<int> s;
    if (kind == Kind::Kalman) {  // at most the warm-up window before n (none at frame 0)
      for (int f = n > warmup ? n - warmup : std::min(n, 1); f <= n; ++f) s.push_back(f);
      return s;
    }
    if (kind == Kind::Copy || kind == Kind::Single || preview) return {n};
    if (info_of_processed().fft3d) {
      if (n < left || N - 1 - n < right) return {n};
      for (int f = n - left; f <= n + right; ++f) s.push_back(f);
      return s;
    }
    if (info_of_processed().tmode1) {
      for (const auto& b : nfb::temporal_blocks(n, N, T, overlap)) {
        if (targets) targets->push_back(b.target);
        for (int z = 0; z < T; ++z) s.push_back(b.slots[size_t(z)]);
      }
      return s;
    }
    const int c = T / 2;
    for (int j = 0; j < T; ++j) s.push_back(std::min(std::max(n - c + j, 0), N - 1));
    return s;
  }

  const nfi::PlanInfo& info_of_processed() const {
    for (size_t p = 0; p < plans.size(); ++p)
      if (plans[p]) return info[p];
    return info[0];
  }

  Range range_of(int n) const {
    Range r;
    switch (kind) {
      case Kind::ClipDFT: {
        const int rt = ((R + T - 1) / T) * T;  // whole temporal blocks per range
        const int last = ((N - T) / rt) * rt;  // the last range absorbs a tail shorter than T
        r.n0 = std::min((n / rt) * rt, last);
        r.n1 = r.n0 == last ? N : r.n0 + rt;
        r.s0 = r.o0 = r.n0;
        r.s1 = r.n1;
        return r;
      }
      case Kind::ClipFFT3D:
        r.n0 = (n / R) * R;
        r.n1 = std::min(N, r.n0 + R);
        // Margins of the window on both sides; their own outputs are not delivered (at
        // the sub-clip edge they take the single-frame fallback).
        r.s0 = r.o0 = std::max(0, r.n0 - left);
        r.s1 = std::min(N, r.n1 + right);
        return r;
      default:
        r.n0 = (n / R) * R;
        r.n1 = std::min(N, r.n0 + R);
        r.o0 = r.n0;
        r.s0 = N;
        r.s1 = 0;
        for (int m = r.n0; m < r.n1; ++m)
          for (int f : slots(m)) {
            r.s0 = std::min(r.s0, f);
            r.s1 = std::max(r.s1, f + 1);
          }
        return r;
    }
  }

  unsigned char* slot(unsigned char* base, int f, int p) const {
    return base + size_t(f) * frame_bytes + offset[size_t(p)];
  }

  void ensure(Bank& b, int src_frames, int out_frames) {
    if (src_frames <= b.src_cap && out_frames <= b.out_cap) return;
    check(cudaStreamSynchronize(b.stream), "stream synchronisation failed");
    b.drop_forms();  // their tables point into the old buffers
    b.valid = false;
    if (src_frames > b.src_cap) {
      if (b.src) cudaFree(b.src);
      b.src = nullptr;
      b.src_cap = 0;
      check(cudaMalloc(reinterpret_cast<void**>(&b.src), size_t(src_frames) * frame_bytes), "device allocation failed");
      b.src_cap = src_frames;
    }
    if (out_frames > b.out_cap) {
      if (b.out) cudaFree(b.out);
      b.out = nullptr;
      b.out_cap = 0;
      check(cudaMalloc(reinterpret_cast<void**>(&b.out), size_t(out_frames) * frame_bytes), "device allocation failed");
      b.out_cap = out_frames;
    }
  }

  nf_const_plane fetch(int frame, int p) const {
    nf_const_plane v{};
    if (source(user, frame, p, &v) != 0 || !v.data)
      raise(NF_INVALID_ARGUMENT, "frame source failed for frame " + std::to_string(frame) + " plane " + std::to_string(p));
    if (plans[size_t(p)] && (v.width != info[size_t(p)].width || v.height != info[size_t(p)].height))
      raise(NF_INVALID_ARGUMENT, "frame plane dimensions differ from plan");
    return v;
  }

  // FFT3D sampled noise models from the pattern frame (filter.hpp:455-471), once.
  void prepare_patterns(cudaStream_t st) {
    if (patterns_done) return;
    char err[512] = {0};
    for (int p = 0; p < planes; ++p) {
      const nf_plan* plan = plans[size_t(p)];
      if (!plan || !info[size_t(p)].fft3d || nf_plan_model_state(plan) != 1) continue;
      const nf_const_plane v = fetch(std::min(std::max(info[size_t(p)].pframe, 0), N - 1), p);
      check(nf_plan_prepare_pattern_host(const_cast<nf_plan*>(plan), v, st, err, sizeof err), err);
    }
    patterns_done = true;
  }

  // Fetches the range's sources into bank b and enqueues its filtering on b's stream.
  // Returns once the source copies are complete (the views may be released after).
  void compute(Bank& b, const Range& r) {
    try {
      compute_range(b, r);
    } catch (...) {
      b.valid = false;
      cudaStreamSynchronize(b.stream);  // no copy from the host's views stays in flight
      throw;
    }
  }

  void compute_range(Bank& b, const Range& r) {
    char err[512] = {0};
    const int ns = r.s1 - r.s0, no = kind == Kind::ClipFFT3D ? ns : r.n1 - r.n0;
    ensure(b, ns, no);
    b.valid = false;
    for (int f = 0; f < ns; ++f)
      for (int p = 0; p < planes; ++p) {
        if (!plans[size_t(p)]) continue;
        const nf_const_plane v = fetch(r.s0 + f, p);
        const auto& in = info[size_t(p)];
        check(cudaMemcpy2DAsync(slot(b.src, f, p), pitch[size_t(p)], v.data, size_t(v.stride_bytes),
                                size_t(in.width) * size_t(in.elem), size_t(in.height), cudaMemcpyDefault, b.stream),
              "source copy failed");
      }
    fetched += ns;
    // The host may release the source views once the copies are complete.
    cudaEvent_t copied;
    check(cudaEventCreateWithFlags(&copied, cudaEventDisableTiming), "event creation failed");
    std::unique_ptr<CUevent_st, decltype(&cudaEventDestroy)> copied_guard(copied, &cudaEventDestroy);
    check(cudaEventRecord(copied, b.stream), "event record failed");
    switch (kind) {
      case Kind::Single: {
        nf_batch*& bt = b.batches[ns];
        if (!bt) {
          std::vector<nf_batch_item> items;
          for (int f = 0; f < ns; ++f)
            for (int p = 0; p < planes; ++p)
              if (plans[size_t(p)]) items.push_back({plans[size_t(p)], device_plane(b.src, f, p), out_plane(b.out, f, p)});
          check(nf_batch_create(items.data(), int(items.size()), &bt, err, sizeof err), err);
        }
        check(nf_batch_graph_launch(bt, b.stream, err, sizeof err), err);
        break;
      }
      case Kind::ClipFFT3D:
      case Kind::ClipDFT: {
        nf_clip_batch*& cb = b.clips[ns];
        if (!cb) {
          std::vector<std::vector<nf_const_plane>> frames;
          std::vector<std::vector<nf_plane>> dsts;
          std::vector<nf_clip_item> items;
          for (int p = 0; p < planes; ++p) {
            if (!plans[size_t(p)]) continue;
            frames.emplace_back();
            dsts.emplace_back();
            for (int f = 0; f < ns; ++f) {
              frames.back().push_back(device_plane(b.src, f, p));
              dsts.back().push_back(out_plane(b.out, f, p));
            }
          }
          size_t k = 0;
          for (int p = 0; p < planes; ++p)
            if (plans[size_t(p)]) {
              items.push_back({plans[size_t(p)], frames[k].data(), dsts[k].data(), ns});
              ++k;
            }
          check(nf_clip_batch_create(items.data(), int(items.size()), &cb, err, sizeof err), err);
        }
        check(nf_clip_batch_graph_launch(cb, b.stream, err, sizeof err), err);
        break;
      }
      default: {
        for (int n = r.n0; n < r.n1; ++n) {
          std::vector<int> targets;
          const std::vector<int> s = slots(n, &targets);
          for (int p = 0; p < planes; ++p) {
            if (!plans[size_t(p)]) continue;
            std::vector<nf_const_plane> srcs;
            for (int f : s) srcs.push_back(device_plane(b.src, f - r.s0, p));
            check(nf_plan_process_device(plans[size_t(p)], srcs.data(), int(srcs.size()),
                                         targets.empty() ? nullptr : targets.data(), int(targets.size()),
                                         out_plane(b.out, n - r.o0, p), n, p, b.stream, err, sizeof err),
                  err);
          }
        }
        break;
      }
    }
    computed += r.n1 - r.n0;
    check(cudaEventSynchronize(copied), "source copy failed");
    b.r = r;
    b.valid = true;
    b.checked = false;
  }

  nf_const_plane device_plane(unsigned char* base, int f, int p) const {
    return {slot(base, f, p), info[size_t(p)].width, info[size_t(p)].height, (long long)pitch[size_t(p)]};
  }
  nf_plane out_plane(unsigned char* base, int f, int p) const {
    return {slot(base, f, p), info[size_t(p)].width, info[size_t(p)].height, (long long)pitch[size_t(p)]};
  }

  Bank* holding(int n) {
    for (auto& b : banks)
      if (b.valid && b.r.n0 <= n && n < b.r.n1) return &b;
    return nullptr;
  }

  // ---- FFT3D bt=0 (Kalman) ------------------------------------------------------
  // The snapshot's states go onto the shelf, or are destroyed when the shelf declines
  // them (frame already held, or over the budget).
  void publish(Snapshot& s) {
    if (!snaps.offer(s.frame, std::move(s.planes), s.bytes, release_states)) release_states(s.planes);
    s.planes.clear();
    s.frame = -1;
    s.bytes = 0;
  }

  void upload(Bank& b, int frame) {
    for (int p = 0; p < planes; ++p) {
      if (!plans[size_t(p)]) continue;
      const nf_const_plane v = fetch(frame, p);
      const auto& in = info[size_t(p)];
      check(cudaMemcpy2DAsync(slot(b.src, 0, p), pitch[size_t(p)], v.data, size_t(v.stride_bytes),
                              size_t(in.width) * size_t(in.elem), size_t(in.height), cudaMemcpyDefault, b.stream),
            "source copy failed");
    }
    ++fetched;
  }

  // The host layer's random-access rule for Kalman plans (filter.hpp:152-250): frame 0
  // passes through; frame n continues the latest snapshot not older than n - warmup - 1
  // (or the initial state from there) over the frames up to n, renders n from that state
  // and publishes it.
  void get_kalman(int n, const nf_plane* dsts) {
    Bank& b = banks[0];
    cudaStream_t st = b.stream;
    prepare_patterns(st);
    ensure(b, 1, 1);
    b.valid = false;  // slot 0 holds Kalman sources, not a range
    char err[512] = {0};
    Snapshot cur;
    const PlaneStates* state = nullptr;
    bool have_n = false;
    try {
      if (n > 0) {
        const int earliest = n > warmup ? n - warmup - 1 : 0;
        int start_frame = 0;
        PlaneStates* start = snaps.latest(n, earliest, &start_frame);
        const int replay_start = start ? start_frame : earliest;
        if (replay_start < n) {
          cur.planes.assign(size_t(planes), nullptr);
          for (int p = 0; p < planes; ++p) {
            if (!plans[size_t(p)]) continue;
            if (start) check(nf_kalman_state_clone((*start)[size_t(p)], &cur.planes[size_t(p)], st, err, sizeof err), err);
            else check(nf_kalman_state_create(plans[size_t(p)], 0, &cur.planes[size_t(p)], err, sizeof err), err);
            cur.bytes += nf_kalman_state_bytes(cur.planes[size_t(p)]);
          }
          // frames before n are advanced; frame n is advanced and rendered together below
          // (nf_kalman_step_device: the same results as advance then render)
          for (int f = replay_start + 1; f <= n; ++f) {
            upload(b, f);
            if (f == n) break;
            for (int p = 0; p < planes; ++p)
              if (plans[size_t(p)])
                check(nf_kalman_advance_device(plans[size_t(p)], device_plane(b.src, 0, p), cur.planes[size_t(p)], st,
                                               err, sizeof err),
                      err);
          }
          cur.frame = n;
          have_n = true;
          state = &cur.planes;
        } else {
          state = start;
        }
      }
      if (state && !have_n) upload(b, n);
      for (int p = 0; p < planes; ++p) {
        const nf_plane& d = dsts[p];
        if (!d.data) raise(NF_INVALID_ARGUMENT, "null destination plane");
        if (plans[size_t(p)] && state) {
          const auto& in = info[size_t(p)];
          if (d.width != in.width || d.height != in.height) raise(NF_INVALID_ARGUMENT, "frame dimensions differ from plan");
          if (have_n)
            check(nf_kalman_step_device(plans[size_t(p)], device_plane(b.src, 0, p), out_plane(b.out, 0, p),
                                        cur.planes[size_t(p)], st, err, sizeof err),
                  err);
          else
            check(nf_kalman_render_device(plans[size_t(p)], device_plane(b.src, 0, p), out_plane(b.out, 0, p),
                                          (*state)[size_t(p)], st, err, sizeof err),
                  err);
          check(cudaMemcpy2DAsync(d.data, size_t(d.stride_bytes), slot(b.out, 0, p), pitch[size_t(p)],
                                  size_t(in.width) * size_t(in.elem), size_t(in.height), cudaMemcpyDefault, st),
                "output copy failed");
        } else {
          // Frame 0 and planes that are not processed: the source plane (filter.hpp:216-218).
          const nf_const_plane v = fetch(n, p);
          if (d.width != v.width || d.height != v.height) raise(NF_INVALID_ARGUMENT, "frame dimensions differ from source");
          check(cudaMemcpy2DAsync(d.data, size_t(d.stride_bytes), v.data, size_t(v.stride_bytes),
                                  size_t(v.width) * size_t(elem_of(p)), size_t(v.height), cudaMemcpyDefault, st),
                "plane copy failed");
        }
      }
      check(cudaStreamSynchronize(st), "Kalman filtering failed");
      for (const nf_plan* plan : plans)
        if (plan) check(nf_plan_sync_status(plan, st, err, sizeof err), err);
    } catch (...) {
      cudaStreamSynchronize(st);
      release_states(cur.planes);
      throw;
    }
    ++computed;
    if (have_n) publish(cur);
  }

  void get(int n, const nf_plane* dsts) {
    if (n < 0 || n >= N) raise(NF_INVALID_ARGUMENT, "frame outside clip");
    if (kind == Kind::Kalman) {
      get_kalman(n, dsts);
      return;
    }
    Bank* b = nullptr;
    if (kind != Kind::Copy) {
      prepare_patterns(banks[0].stream);
      b = holding(n);
      if (!b) {
        b = &banks[0];
        for (auto& c : banks)
          if (c.used < b->used) b = &c;
        compute(*b, range_of(n));
      }
      b->used = ++tick;
    }
    cudaStream_t st = b ? b->stream : banks[0].stream;
    for (int p = 0; p < planes; ++p) {
      const nf_plane& d = dsts[p];
      if (!d.data) raise(NF_INVALID_ARGUMENT, "null destination plane");
      if (plans[size_t(p)]) {
        const auto& in = info[size_t(p)];
        if (d.width != in.width || d.height != in.height) raise(NF_INVALID_ARGUMENT, "frame dimensions differ from plan");
        check(cudaMemcpy2DAsync(d.data, size_t(d.stride_bytes), slot(b->out, n - b->r.o0, p), pitch[size_t(p)],
                                size_t(in.width) * size_t(in.elem), size_t(in.height), cudaMemcpyDefault, st),
              "output copy failed");
      } else {
        // Plane not processed: the source frame's plane (filter.hpp:362-371).
        const nf_const_plane v = fetch(n, p);
        if (d.width != v.width || d.height != v.height) raise(NF_INVALID_ARGUMENT, "frame dimensions differ from source");
        const size_t row = size_t(v.width) * size_t(elem_of(p));
        check(cudaMemcpy2DAsync(d.data, size_t(d.stride_bytes), v.data, size_t(v.stride_bytes), row,
                                size_t(v.height), cudaMemcpyDefault, st),
              "plane copy failed");
      }
    }
    check(cudaStreamSynchronize(st), "output copy failed");
    if (b && !b->checked) {
      // Non-finite input or output of the range's filtering (Plan::run's checks).
      char err[512] = {0};
      for (const nf_plan* plan : plans)
        if (plan) {
          const nf_status ps = nf_plan_sync_status(plan, st, err, sizeof err);
          if (ps != NF_OK) {
            b->valid = false;
            raise(ps, err);
          }
        }
      b->checked = true;
    }
    // Sequential readers: the ranges after this one go into the other banks, so the
    // next range's source copies overlap the filtering of the one before it.
    if (b) {
      std::vector<const Bank*> keep{b};
      int next = b->r.n1;
      while (next < N && int(keep.size()) < kBanks) {
        Bank* h = holding(next);
        if (!h) {
          for (auto& c : banks)
            if (std::find(keep.begin(), keep.end(), &c) == keep.end() && (!h || c.used < h->used)) h = &c;
          try {
            compute(*h, range_of(next));
            h->used = ++tick;
          } catch (const std::exception&) {
            break;  // reported when one of its frames is requested
          } catch (const Failure&) {
            break;
          }
        }
        keep.push_back(h);
        next = h->r.n1;
      }
    }
  }

  int elem_default = 1;
  int elem_of(int p) const { return plans[size_t(p)] ? info[size_t(p)].elem : elem_default; }
};

extern "C" {

nf_status nf_frame_server_create(const nf_plan* const* plans, int planes, int num_frames, int range_frames,
                                 nf_frame_source source, void* user, nf_frame_server** out, char* err,
                                 size_t len) {
  auto fail = [&](nf_status code, const std::string& msg) {
    if (err && len) {
      std::strncpy(err, msg.c_str(), len - 1);
      err[len - 1] = 0;
    }
    return code;
  };
  try {
    if (!out || !plans || !source) return fail(NF_INVALID_ARGUMENT, "null server output, plans or source");
    if (planes < 1 || planes > 4) return fail(NF_INVALID_ARGUMENT, "frames hold 1..4 planes");
    if (num_frames < 1) return fail(NF_INVALID_ARGUMENT, "clip frame count must be positive");
    if (range_frames < 1 || range_frames > 1024) return fail(NF_INVALID_ARGUMENT, "range_frames must be 1..1024");
    auto s = std::make_unique<nf_frame_server>();
    s->planes = planes;
    s->N = num_frames;
    s->R = range_frames;
    s->source = source;
    s->user = user;
    bool first = true;
    nfi::PlanInfo ref{};
    for (int p = 0; p < planes; ++p) {
      s->plans.push_back(plans[p]);
      s->info.push_back(plans[p] ? nfi::plan_info(plans[p]) : nfi::PlanInfo{});
      if (!plans[p]) {
        s->offset.push_back(0);
        s->pitch.push_back(0);
        continue;
      }
      const nfi::PlanInfo& i = s->info.back();
      if (first) {
        ref = i;
        first = false;
      } else if (i.fft3d != ref.fft3d || i.temporal_size != ref.temporal_size || i.tmode1 != ref.tmode1 ||
                 i.temporal_overlap != ref.temporal_overlap || i.preview != ref.preview || i.single != ref.single ||
                 i.clip != ref.clip || i.kalman != ref.kalman) {
        return fail(NF_INVALID_ARGUMENT, "planes of a frame server must share the temporal configuration");
      }
      const size_t pitch = ((size_t(i.width) * size_t(i.elem) + 255) / 256) * 256;
      s->pitch.push_back(pitch);
      s->offset.push_back(s->frame_bytes);
      s->frame_bytes += pitch * size_t(i.height);
      s->elem_default = i.elem;
    }
    if (first) return fail(NF_INVALID_ARGUMENT, "a frame server needs at least one processed plane");
    {
      s->T = ref.temporal_size;
      s->preview = ref.preview;
      s->overlap = ref.temporal_overlap;
      if (!ref.fft3d && s->T > num_frames)
        return fail(NF_INVALID_ARGUMENT, "tbsize must be less than or equal to the number of frames");
      if (ref.fft3d && !ref.preview && s->T >= 2) {
        s->left = s->T / 2;
        s->right = (s->T - 1) / 2;
      }
      if (ref.kalman) {
        s->kind = Kind::Kalman;
        s->warmup = ref.kalman_warmup;
        s->left = s->right = 0;
      } else if (ref.preview) s->kind = Kind::PerFrame;
      else if (ref.clip) s->kind = ref.fft3d ? Kind::ClipFFT3D : Kind::ClipDFT;
      else if (ref.single && s->T == 1) s->kind = Kind::Single;
      else s->kind = Kind::PerFrame;
    }
    for (auto& b : s->banks) {
      const cudaError_t e = cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking);
      if (e != cudaSuccess) return fail(NF_DEVICE_ERROR, std::string("stream creation failed: ") + cudaGetErrorString(e));
    }
    *out = s.release();
    return NF_OK;
  } catch (const Failure& f) {
    return fail(f.code, f.msg);
  } catch (const std::exception& e) {
    return fail(NF_INVALID_ARGUMENT, e.what());
  }
}

nf_status nf_frame_server_request(const nf_frame_server* s, int n, int* frames, int capacity, int* count,
                                  char* err, size_t len) {
  auto fail = [&](nf_status code, const std::string& msg) {
    if (err && len) {
      std::strncpy(err, msg.c_str(), len - 1);
      err[len - 1] = 0;
    }
    return code;
  };
  if (!s || !count) return fail(NF_INVALID_ARGUMENT, "null server or count");
  if (n < 0 || n >= s->N) return fail(NF_INVALID_ARGUMENT, "frame outside clip");
  try {
    std::vector<int> r = s->slots(n);
    for (int p = 0; p < s->planes; ++p)  // sampled FFT3D models read the pattern frame (filter.hpp:268)
      if (s->plans[size_t(p)] && s->info[size_t(p)].fft3d && nf_plan_model_state(s->plans[size_t(p)]) != 0)
        r.push_back(std::min(std::max(s->info[size_t(p)].pframe, 0), s->N - 1));
    std::sort(r.begin(), r.end());
    r.erase(std::unique(r.begin(), r.end()), r.end());
    *count = int(r.size());
    for (int i = 0; i < std::min(capacity, int(r.size())); ++i)
      if (frames) frames[i] = r[size_t(i)];
    return NF_OK;
  } catch (const std::exception& e) {
    return fail(NF_INVALID_ARGUMENT, e.what());
  }
}

nf_status nf_frame_server_get(nf_frame_server* s, int n, const nf_plane* dsts, char* err, size_t len) {
  auto fail = [&](nf_status code, const std::string& msg) {
    if (err && len) {
      std::strncpy(err, msg.c_str(), len - 1);
      err[len - 1] = 0;
    }
    return code;
  };
  if (!s || !dsts) return fail(NF_INVALID_ARGUMENT, "null server or destinations");
  std::lock_guard<std::mutex> lock(s->mu);
  try {
    s->get(n, dsts);
    return NF_OK;
  } catch (const Failure& f) {
    for (auto& b : s->banks) b.valid = false;
    return fail(f.code, f.msg);
  } catch (const std::exception& e) {
    for (auto& b : s->banks) b.valid = false;
    return fail(NF_INVALID_ARGUMENT, e.what());
  }
}

void nf_frame_server_counters(const nf_frame_server* s, long long* computed, long long* fetched) {
  if (!s) return;
  std::lock_guard<std::mutex> lock(s->mu);
  if (computed) *computed = s->computed;
  if (fetched) *fetched = s->fetched;
}

void nf_frame_server_destroy(nf_frame_server* s) { delete s; }

}  // extern "C"
