// C++ drop-in facade: the class signature of neo-fft's core `Plan`
// (src/algorithms/plan.hpp:18-140 in the reference) implemented over the C ABI in
// neo_fft_b200.h, so the VapourSynth/AviSynth host layer (src/plugin/filter.hpp,
// src/plugin/descriptors.hpp) can call the B200 path unchanged.
//
// Planes are the host's DualSynth2 `span2d` views in host memory; each call stages
// them through the plan's device buffers (nf_plan_process_host). Errors are
// rethrown with the reference's exception types and texts: std::invalid_argument
// for configuration/geometry, std::runtime_error("non-finite sample or
// intermediate") for data (src/base/checked.hpp:13-41).
//
// The sampled noise models (pfactor, nlocation) are not implemented on the B200
// path; plans requesting them fail at creation with std::invalid_argument, so the
// pattern-model members below report an inactive model.
#pragma once
#include "neo_fft_b200.h"

#include <dualsynth/span2d.hpp>

#include <array>
#include <complex>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <optional>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

namespace neo_fft {

// Row copy used by the host layer's ROI packing (kernels/rows.hpp:4-7). Plan::copy_row()
// returns nf_copy_row, which also copies rows that live in device memory.
using CopyRow = void (*)(const void*, void*, std::size_t);
inline void copy_row_scalar(const void* source, void* dst, std::size_t bytes) {
  if (bytes) std::memcpy(dst, source, bytes);
}

namespace runtime {
class SpectraCache;     // host-side raw-spectrum cache: not used by the B200 path
class Retention;

// Per-request working state (src/runtime/workspace.hpp, workspace_pool.hpp:12-75). On the
// B200 path a request's working set is device staging taken from the library's memory pool
// per call; the workspace carries the CUDA stream the request's calls are ordered on, so
// requests served by different host threads overlap on the GPU.
struct WorkspaceBudget {
  std::size_t total_bytes = 0;  // device staging of one request (its source slots and output)
  int temporal_slots = 1;
};

class Workspace {
 public:
  explicit Workspace(const WorkspaceBudget& budget) : budget_(budget) {
    char err[256] = {0};
    if (nf_stream_create(&stream_, err, sizeof(err)) != NF_OK) throw std::runtime_error(err);
  }
  Workspace(const Workspace&) = delete;
  Workspace& operator=(const Workspace&) = delete;
  ~Workspace() { nf_stream_destroy(stream_); }
  const WorkspaceBudget& budget() const noexcept { return budget_; }
  void* stream() const noexcept { return stream_; }

 private:
  WorkspaceBudget budget_;
  void* stream_ = nullptr;
};

class WorkspacePool;

// A leased workspace; returned to its pool when the lease ends.
class WorkspaceLease {
 public:
  WorkspaceLease() noexcept = default;
  WorkspaceLease(WorkspacePool* pool, std::unique_ptr<Workspace> ws) noexcept : pool_(pool), ws_(std::move(ws)) {}
  WorkspaceLease(WorkspaceLease&& o) noexcept : pool_(o.pool_), ws_(std::move(o.ws_)) { o.pool_ = nullptr; }
  WorkspaceLease& operator=(WorkspaceLease&& o) noexcept {
    if (this != &o) {
      reset();
      pool_ = o.pool_;
      ws_ = std::move(o.ws_);
      o.pool_ = nullptr;
    }
    return *this;
  }
  WorkspaceLease(const WorkspaceLease&) = delete;
  WorkspaceLease& operator=(const WorkspaceLease&) = delete;
  ~WorkspaceLease() { reset(); }
  Workspace* get() const noexcept { return ws_.get(); }
  Workspace* operator->() const noexcept { return ws_.get(); }
  Workspace& operator*() const noexcept { return *ws_; }
  explicit operator bool() const noexcept { return ws_ != nullptr; }
  inline void reset() noexcept;

 private:
  WorkspacePool* pool_ = nullptr;
  std::unique_ptr<Workspace> ws_;
};

// Any number of workspaces may be leased at once; at most max_capacity idle ones are kept
// for reuse, the rest are released when their lease ends.
class WorkspacePool {
 public:
  explicit WorkspacePool(WorkspaceBudget budget, std::size_t max_capacity = 1)
      : budget_(budget), max_capacity_(max_capacity) {}
  WorkspacePool(const WorkspacePool&) = delete;
  WorkspacePool& operator=(const WorkspacePool&) = delete;
  WorkspaceLease acquire() {
    std::unique_ptr<Workspace> ws;
    {
      std::lock_guard<std::mutex> lock(mu_);
      ++active_;
      if (!idle_.empty()) {
        ws = std::move(idle_.back());
        idle_.pop_back();
      }
    }
    if (!ws) {
      try {
        ws = std::make_unique<Workspace>(budget_);
      } catch (...) {
        std::lock_guard<std::mutex> lock(mu_);
        --active_;
        throw;
      }
    }
    return WorkspaceLease(this, std::move(ws));
  }
  const WorkspaceBudget& budget() const noexcept { return budget_; }
  std::size_t max_capacity() const noexcept { return max_capacity_; }
  std::size_t active_count() const {
    std::lock_guard<std::mutex> lock(mu_);
    return active_;
  }
  std::size_t idle_count() const {
    std::lock_guard<std::mutex> lock(mu_);
    return idle_.size();
  }

 private:
  friend class WorkspaceLease;
  void give_back(std::unique_ptr<Workspace> ws) noexcept {
    std::unique_ptr<Workspace> drop;
    std::lock_guard<std::mutex> lock(mu_);
    --active_;
    if (idle_.size() < max_capacity_) idle_.push_back(std::move(ws));
    else drop = std::move(ws);
  }
  WorkspaceBudget budget_;
  std::size_t max_capacity_;
  std::size_t active_ = 0;
  std::vector<std::unique_ptr<Workspace>> idle_;
  mutable std::mutex mu_;
};

inline void WorkspaceLease::reset() noexcept {
  if (pool_ && ws_) pool_->give_back(std::move(ws_));
  pool_ = nullptr;
  ws_.reset();
}
}  // namespace runtime

enum class Algorithm { FFT3D, DFTTest };
struct SampleFormat {
  int bits = 8;
  bool floating = false, chroma = false;
};
struct EnhancementConfig {
  float sharpen = 0, scutoff = .3f, svr = 1, smin = 4, smax = 20;
  float dehalo = 0, hr = 2, ht = 50;
};
struct DFTCurves {
  std::vector<float> shared, x, y, time;
  int system = 0;
  bool empty() const { return shared.empty() && x.empty() && y.empty() && time.empty(); }
};
struct NoiseLocation {
  int frame, plane, y, x;
};
struct FFT3DConfig {
  int bw = 32, bh = 32, ow = -1, oh = -1, wintype = 0, opt = 0, bt = 1;
  float sigma = 2, beta = 1, degrid = 1, kratio = 2;
  std::optional<float> sigma2, sigma3, sigma4;
  EnhancementConfig enhancement;
  float pfactor = 0, pcutoff = .1f;
  int pframe = 0, px = 0, py = 0;
  bool pshow = false;
  int left = 0, top = 0, right = 0, bottom = 0;
  bool interlaced = false;
  int cache_frames = -1, cache_mb = 128;
  int kalman_warmup = 8;
};
struct DFTConfig {
  int block = 16, overlap = 12, mode = 1, swin = 0, twin = 7, ftype = 0, opt = 0, tbsize = 1;
  float sbeta = 2.5f, tbeta = 2.5f, sigma = 8, sigma2 = 8, pmin = 0, pmax = 500, f0beta = 1;
  bool zmean = true;
  int temporal_mode = 0, temporal_overlap = 0;
  int dither = 0, dither_seed = 0;
  DFTCurves curves;
  std::vector<NoiseLocation> locations;
  std::optional<float> alpha;
};
struct Axis {
  int length = 0, block = 0, overlap = 0, step = 0, count = 0, cover = 0, offset = 0;
};
struct Geometry {
  Axis x, y;
};

namespace detail {
inline nf_dft_config to_c(const DFTConfig& c, std::vector<int>& loc) {
  nf_dft_config n{};
  n.block = c.block; n.overlap = c.overlap; n.mode = c.mode; n.swin = c.swin; n.twin = c.twin;
  n.ftype = c.ftype; n.opt = c.opt; n.tbsize = c.tbsize; n.sbeta = c.sbeta; n.tbeta = c.tbeta;
  n.sigma = c.sigma; n.sigma2 = c.sigma2; n.pmin = c.pmin; n.pmax = c.pmax; n.f0beta = c.f0beta;
  n.zmean = c.zmean; n.temporal_mode = c.temporal_mode; n.temporal_overlap = c.temporal_overlap;
  n.dither = c.dither; n.dither_seed = c.dither_seed;
  n.slocation = c.curves.shared.data(); n.n_slocation = int(c.curves.shared.size());
  n.ssx = c.curves.x.data(); n.n_ssx = int(c.curves.x.size());
  n.ssy = c.curves.y.data(); n.n_ssy = int(c.curves.y.size());
  n.sst = c.curves.time.data(); n.n_sst = int(c.curves.time.size());
  n.ssystem = c.curves.system;
  loc.clear();
  for (const auto& l : c.locations) loc.insert(loc.end(), {l.frame, l.plane, l.y, l.x});
  n.nlocation = loc.data(); n.n_nlocation = int(c.locations.size());
  n.has_alpha = c.alpha.has_value(); n.alpha = c.alpha.value_or(0);
  return n;
}
inline void check(nf_status s, const char* err) {
  if (s == NF_OK) return;
  if (s == NF_INVALID_ARGUMENT) throw std::invalid_argument(err);
  throw std::runtime_error(err);
}
template <class T>
nf_const_plane cplane(const span2d::Plane<const T>& p) {
  return {p.data(), p.width(), p.height(), p.stride_bytes()};
}
template <class T>
nf_plane mplane(const span2d::Plane<T>& p) {
  return {p.data(), p.width(), p.height(), p.stride_bytes()};
}
}  // namespace detail

// Kalman state (kernels/kalman.hpp:5-14) held in device memory. Copies are deep
// (the host layer copies checkpoints before replay, filter.hpp:171).
class KalmanState {
 public:
  KalmanState() = default;
  KalmanState(const KalmanState& o) { *this = o; }
  KalmanState& operator=(const KalmanState& o) {
    if (this == &o) return *this;
    reset();
    if (o.state_) {
      char err[256] = {0};
      nf_kalman_state* s = nullptr;
      detail::check(nf_kalman_state_clone(o.state_, &s, nullptr, err, sizeof(err)), err);
      state_ = s;
      plan_ = o.plan_;
    }
    return *this;
  }
  KalmanState(KalmanState&& o) noexcept : plan_(o.plan_), state_(o.state_) { o.state_ = nullptr; }
  KalmanState& operator=(KalmanState&& o) noexcept {
    std::swap(plan_, o.plan_);
    std::swap(state_, o.state_);
    return *this;
  }
  ~KalmanState() { reset(); }
  nf_kalman_state* handle() const { return state_; }
  // KalmanState::bytes (runtime/checkpoints.hpp:13-14 sums them per checkpoint).
  std::size_t bytes() const { return sizeof(*this) + (state_ ? nf_kalman_state_bytes(state_) : 0); }

 private:
  friend class Plan;
  void reset() {
    if (state_) nf_kalman_state_destroy(state_);
    state_ = nullptr;
  }
  const nf_plan* plan_ = nullptr;
  nf_kalman_state* state_ = nullptr;
};

// DFTNoise (src/algorithms/dft_noise.hpp:9-30): the sampled noise model shared by the
// DFTTest plans of one filter. prepare() gathers tbsize slices per location through the
// host layer's callback and builds the per-bin table once; plans upload the published
// table before their next call.
class DFTNoise {
 public:
  explicit DFTNoise(const DFTConfig& c)
      : locations(c.locations), temporal_size(c.tbsize), block_size(c.block), config_(c) {}
  using Gather = std::function<void(const NoiseLocation&, int, span2d::Span<float>)>;
  void prepare(const Gather& gather) const {
    std::lock_guard<std::mutex> lock(mu_);
    if (power_) return;
    const std::size_t slice = std::size_t(block_size) * block_size;
    std::vector<float> slices(locations.size() * std::size_t(temporal_size) * slice);
    for (std::size_t l = 0; l < locations.size(); ++l)
      for (int z = 0; z < temporal_size; ++z)
        gather(locations[l], z, span2d::Span<float>(slices.data() + (l * temporal_size + std::size_t(z)) * slice, slice));
    auto out = std::make_shared<std::vector<float>>(std::size_t(temporal_size) * block_size * (block_size / 2 + 1));
    std::vector<int> loc;
    nf_dft_config n = detail::to_c(config_, loc);
    char err[512] = {0};
    detail::check(nf_dft_noise_power(&n, slices.data(), int(locations.size()), out->data(), int(out->size()), err,
                                     sizeof(err)),
                  err);
    power_ = std::move(out);
  }
  std::shared_ptr<const std::vector<float>> power() const {
    std::lock_guard<std::mutex> lock(mu_);
    return power_;
  }
  const std::vector<NoiseLocation> locations;
  const int temporal_size, block_size;

 private:
  DFTConfig config_;
  mutable std::mutex mu_;
  mutable std::shared_ptr<const std::vector<float>> power_;
};

class Plan {
 public:
  // Plan(int, int, SampleFormat, const FFT3DConfig&) — plan.hpp:51.
  Plan(int width, int height, SampleFormat format, const FFT3DConfig& c,
       std::shared_ptr<runtime::Retention> = {})
      : format(format), algorithm(Algorithm::FFT3D) {
    nf_fft3d_config n{};
    n.bw = c.bw; n.bh = c.bh; n.ow = c.ow; n.oh = c.oh; n.wintype = c.wintype; n.opt = c.opt; n.bt = c.bt;
    n.sigma = c.sigma; n.beta = c.beta; n.degrid = c.degrid; n.kratio = c.kratio;
    n.has_sigma2 = c.sigma2.has_value(); n.sigma2 = c.sigma2.value_or(0);
    n.has_sigma3 = c.sigma3.has_value(); n.sigma3 = c.sigma3.value_or(0);
    n.has_sigma4 = c.sigma4.has_value(); n.sigma4 = c.sigma4.value_or(0);
    const auto& e = c.enhancement;
    n.sharpen = e.sharpen; n.scutoff = e.scutoff; n.svr = e.svr; n.smin = e.smin; n.smax = e.smax;
    n.dehalo = e.dehalo; n.hr = e.hr; n.ht = e.ht;
    n.pfactor = c.pfactor; n.pcutoff = c.pcutoff; n.pframe = c.pframe; n.px = c.px; n.py = c.py;
    n.pshow = c.pshow; n.left = c.left; n.top = c.top; n.right = c.right; n.bottom = c.bottom;
    n.interlaced = c.interlaced; n.cache_frames = c.cache_frames; n.cache_mb = c.cache_mb;
    n.kalman_warmup = c.kalman_warmup;
    char err[512] = {0};
    detail::check(nf_plan_create_fft3d(width, height, to_c(format), &n, &plan_, err, sizeof(err)), err);
    // plan.cpp:110-115: preview when pshow samples a pattern or shows a varying-sigma plan
    const auto differs = [&](const std::optional<float>& v) { return v.has_value() && *v != c.sigma; };
    preview_ = c.pshow && (c.pfactor > 0 || differs(c.sigma2) || differs(c.sigma3) || differs(c.sigma4));
    kalman_ = c.bt == 0 && !preview_;
    init();
  }
  // Plan(int, int, SampleFormat, const DFTConfig&, noise) — plan.hpp:52; plans of one
  // filter share the sampled noise model (filter.hpp:81-82).
  Plan(int width, int height, SampleFormat format, const DFTConfig& c, std::shared_ptr<const DFTNoise> noise = {},
       std::shared_ptr<runtime::Retention> = {})
      : format(format), algorithm(Algorithm::DFTTest) {
    std::vector<int> loc;
    nf_dft_config n = detail::to_c(c, loc);
    char err[512] = {0};
    detail::check(nf_plan_create_dft(width, height, to_c(format), &n, &plan_, err, sizeof(err)), err);
    init();
    if (nf_plan_model_state(plan_) != 0) noise_ = noise ? std::move(noise) : std::make_shared<DFTNoise>(c);
  }
  std::shared_ptr<const DFTNoise> dft_noise() const { return noise_; }
  Plan(const Plan&) = delete;
  Plan& operator=(const Plan&) = delete;
  ~Plan() { nf_plan_destroy(plan_); }

  Geometry geometry;
  const SampleFormat format;
  const Algorithm algorithm;
  int temporal_size = 1;
  struct Fft {
    std::size_t bins_ = 0;
    std::size_t bins() const { return bins_; }
  } fft;

  // process (plan.hpp:58-75): one plane or temporal slots, with the plan's pooled
  // workspace or the caller's.
  template <class T>
  void process(span2d::Plane<const T> src, span2d::Plane<T> dst) const {
    process_at<T>({&src, 1}, dst, 0, 0);
  }
  template <class T>
  void process(span2d::Plane<const T> src, span2d::Plane<T> dst, runtime::Workspace& ws) const {
    run<T>({&src, 1}, dst, 0, 0, {}, ws.stream());
  }
  template <class T>
  void process(span2d::Span<const span2d::Plane<const T>> sources, span2d::Plane<T> dst) const {
    process_at<T>(sources, dst, 0, 0);
  }
  template <class T>
  void process(span2d::Span<const span2d::Plane<const T>> sources, span2d::Plane<T> dst,
               runtime::Workspace& ws) const {
    run<T>(sources, dst, 0, 0, {}, ws.stream());
  }
  // process_at (plan.hpp:77-80): a workspace leased from the plan's pool for the call; the
  // SpectraCache arguments are accepted and ignored.
  template <class T, class Cache = runtime::SpectraCache, class Request = void>
  void process_at(span2d::Span<const span2d::Plane<const T>> sources, span2d::Plane<T> dst, int frame, int plane,
                  span2d::Span<const int> targets = {}, Cache* = nullptr, Request* = nullptr) const {
    auto lease = pool_->acquire();
    run<T>(sources, dst, frame, plane, targets, lease->stream());
  }
  CopyRow copy_row() const { return &nf_copy_row; }
  runtime::WorkspacePool& workspace_pool() const noexcept { return *pool_; }

  bool kalman() const { return kalman_; }
  bool preview() const { return preview_; }
  // FFT3D sampled model (plan.hpp:90-97): the pattern candidate of a host plane, its
  // publication, and prepare_pattern (search + publish unless already published).
  bool needs_pattern_frame() const { return algorithm == Algorithm::FFT3D && nf_plan_model_state(plan_) != 0; }
  bool pattern_ready() const { return nf_plan_model_state(plan_) == 2; }
  template <class T>
  std::shared_ptr<const std::vector<float>> pattern_candidate(span2d::Plane<const T> source) const {
    auto out = std::make_shared<std::vector<float>>(fft.bins());
    char err[512] = {0};
    detail::check(nf_plan_pattern_candidate_host(plan_, detail::cplane(source), out->data(), int(out->size()), nullptr,
                                                 err, sizeof(err)),
                  err);
    return out;
  }
  void publish_pattern(std::shared_ptr<const std::vector<float>> model) const {
    char err[512] = {0};
    detail::check(nf_plan_set_noise_model(plan_, model->data(), int(model->size()), err, sizeof(err)), err);
  }
  template <class T>
  void prepare_pattern(span2d::Plane<const T> source) const {
    char err[512] = {0};
    detail::check(nf_plan_prepare_pattern_host(plan_, detail::cplane(source), nullptr, err, sizeof(err)), err);
  }
  KalmanState initial_kalman() const {
    KalmanState s;
    char err[512] = {0};
    detail::check(nf_kalman_state_create(plan_, 0, &s.state_, err, sizeof(err)), err);
    s.plan_ = plan_;
    return s;
  }
  template <class T>
  void advance_kalman(span2d::Plane<const T> source, KalmanState& state) const {
    char err[512] = {0};
    detail::check(nf_kalman_advance_host(plan_, detail::cplane(source), state.state_, nullptr, err, sizeof(err)),
                  err);
  }
  template <class T>
  void render_kalman(span2d::Plane<const T> source, span2d::Plane<T> dst, const KalmanState& state) const {
    char err[512] = {0};
    detail::check(nf_kalman_render_host(plan_, detail::cplane(source), detail::mplane(dst), state.state_, nullptr,
                                        err, sizeof(err)),
                  err);
  }
  const nf_plan* handle() const { return plan_; }

 private:
  template <class T>
  void run(span2d::Span<const span2d::Plane<const T>> sources, span2d::Plane<T> dst, int frame, int plane,
           span2d::Span<const int> targets, void* stream) const {
    if (noise_) upload_noise();
    std::vector<nf_const_plane> s;
    s.reserve(sources.size());
    for (const auto& p : sources) s.push_back(detail::cplane(p));
    char err[512] = {0};
    detail::check(nf_plan_process_host(plan_, s.data(), int(s.size()), targets.data(), int(targets.size()),
                                       detail::mplane(dst), frame, plane, stream, err, sizeof(err)),
                  err);
  }
  // Publishes the shared noise model's table to this plan once it exists.
  void upload_noise() const {
    auto power = noise_->power();
    std::lock_guard<std::mutex> lock(noise_mu_);
    if (!power || power.get() == uploaded_) return;
    char err[512] = {0};
    detail::check(nf_plan_set_noise_model(plan_, power->data(), int(power->size()), err, sizeof(err)), err);
    uploaded_ = power.get();
  }
  std::shared_ptr<const DFTNoise> noise_;
  mutable std::mutex noise_mu_;
  mutable const std::vector<float>* uploaded_ = nullptr;
  static nf_format to_c(SampleFormat f) { return {f.bits, f.floating ? 1 : 0, f.chroma ? 1 : 0}; }
  void init() {
    nf_axis x{}, y{};
    int t = 1, b = 0;
    nf_plan_geometry(plan_, &x, &y, &t, &b);
    geometry.x = {x.length, x.block, x.overlap, x.step, x.count, x.cover, x.offset};
    geometry.y = {y.length, y.block, y.overlap, y.step, y.count, y.cover, y.offset};
    temporal_size = t;
    fft.bins_ = std::size_t(b);
    const std::size_t sample = format.floating ? 4 : (format.bits > 8 ? 2 : 1);
    const std::size_t plane_bytes = std::size_t(x.length) * std::size_t(y.length) * sample;
    pool_ = std::make_unique<runtime::WorkspacePool>(
        runtime::WorkspaceBudget{plane_bytes * std::size_t(t + 1), t});
  }
  nf_plan* plan_ = nullptr;
  std::unique_ptr<runtime::WorkspacePool> pool_;
  bool kalman_ = false;
  bool preview_ = false;
};

}  // namespace neo_fft
