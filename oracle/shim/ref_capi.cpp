// Test infrastructure (oracle only): extern "C" entry points over the neo-fft
// reference core (`neo_fft::Plan`, src/algorithms/plan.hpp:49-140) compiled from
// its own sources, so Python tests and the CPU baseline can drive it through
// ctypes. Configuration structs are the product's public ones
// (include/neo_fft_b200.h) so both sides receive identical parameters.
//
// Nothing here is linked into the product library.
#include "algorithms/plan.hpp"
#include "algorithms/dft_noise.hpp"
#include "algorithms/temporal_grid.hpp"
#include "kernels/dither.hpp"
#include "neo_fft_b200.h"
#include "fft_core.cuh"

#include <cmath>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

using namespace neo_fft;

namespace {
int fail(char* err, size_t len, const char* msg, int code) {
  if (err && len) {
    std::strncpy(err, msg, len - 1);
    err[len - 1] = 0;
  }
  return code;
}
template <class F>
int guarded(char* err, size_t len, F&& f) {
  try {
    f();
    return 0;
  } catch (const std::invalid_argument& e) {
    return fail(err, len, e.what(), 1);
  } catch (const std::runtime_error& e) {
    return fail(err, len, e.what(), 2);
  } catch (const std::exception& e) {
    return fail(err, len, e.what(), 3);
  }
}
FFT3DConfig to_ref(const nf_fft3d_config& c) {
  FFT3DConfig r;
  r.bw = c.bw; r.bh = c.bh; r.ow = c.ow; r.oh = c.oh; r.wintype = c.wintype; r.opt = c.opt; r.bt = c.bt;
  r.sigma = c.sigma; r.beta = c.beta; r.degrid = c.degrid; r.kratio = c.kratio;
  if (c.has_sigma2) r.sigma2 = c.sigma2;
  if (c.has_sigma3) r.sigma3 = c.sigma3;
  if (c.has_sigma4) r.sigma4 = c.sigma4;
  r.enhancement.sharpen = c.sharpen; r.enhancement.scutoff = c.scutoff; r.enhancement.svr = c.svr;
  r.enhancement.smin = c.smin; r.enhancement.smax = c.smax; r.enhancement.dehalo = c.dehalo;
  r.enhancement.hr = c.hr; r.enhancement.ht = c.ht;
  r.pfactor = c.pfactor; r.pcutoff = c.pcutoff; r.pframe = c.pframe; r.px = c.px; r.py = c.py;
  r.pshow = c.pshow != 0;
  r.left = c.left; r.top = c.top; r.right = c.right; r.bottom = c.bottom; r.interlaced = c.interlaced != 0;
  r.cache_frames = c.cache_frames; r.cache_mb = c.cache_mb; r.kalman_warmup = c.kalman_warmup;
  return r;
}
std::vector<float> vec(const float* p, int n) { return p && n > 0 ? std::vector<float>(p, p + n) : std::vector<float>{}; }
DFTConfig to_ref(const nf_dft_config& c) {
  DFTConfig r;
  r.block = c.block; r.overlap = c.overlap; r.mode = c.mode; r.swin = c.swin; r.twin = c.twin;
  r.ftype = c.ftype; r.opt = c.opt; r.tbsize = c.tbsize;
  r.sbeta = c.sbeta; r.tbeta = c.tbeta; r.sigma = c.sigma; r.sigma2 = c.sigma2; r.pmin = c.pmin; r.pmax = c.pmax;
  r.f0beta = c.f0beta; r.zmean = c.zmean != 0; r.temporal_mode = c.temporal_mode;
  r.temporal_overlap = c.temporal_overlap; r.dither = c.dither; r.dither_seed = c.dither_seed;
  r.curves.shared = vec(c.slocation, c.n_slocation);
  r.curves.x = vec(c.ssx, c.n_ssx);
  r.curves.y = vec(c.ssy, c.n_ssy);
  r.curves.time = vec(c.sst, c.n_sst);
  r.curves.system = c.ssystem;
  for (int i = 0; i < c.n_nlocation; ++i)
    r.locations.push_back({c.nlocation[4 * i], c.nlocation[4 * i + 1], c.nlocation[4 * i + 2], c.nlocation[4 * i + 3]});
  if (c.has_alpha) r.alpha = c.alpha;
  return r;
}
struct RefPlan {
  std::unique_ptr<Plan> plan;
};

template <class T>
void run_process(const Plan& p, const nf_const_plane* src, int n, const int* targets, int nt, nf_plane dst,
                 int frame, int plane) {
  std::vector<span2d::Plane<const T>> s;
  for (int i = 0; i < n; ++i)
    s.push_back({static_cast<const T*>(src[i].data), src[i].width, src[i].height, src[i].stride_bytes});
  span2d::Plane<T> d{static_cast<T*>(dst.data), dst.width, dst.height, dst.stride_bytes};
  p.process_at<T>({s.data(), s.size()}, d, frame, plane, {targets, std::size_t(nt)});
}
} // namespace

extern "C" {

int ref_plan_create_fft3d(int w, int h, nf_format f, const nf_fft3d_config* c, void** out, char* err, size_t len) {
  return guarded(err, len, [&] {
    auto r = std::make_unique<RefPlan>();
    r->plan = std::make_unique<Plan>(w, h, SampleFormat{f.bits, f.floating != 0, f.chroma != 0}, to_ref(*c));
    *out = r.release();
  });
}
int ref_plan_create_dft(int w, int h, nf_format f, const nf_dft_config* c, void** out, char* err, size_t len) {
  return guarded(err, len, [&] {
    auto r = std::make_unique<RefPlan>();
    r->plan = std::make_unique<Plan>(w, h, SampleFormat{f.bits, f.floating != 0, f.chroma != 0}, to_ref(*c));
    *out = r.release();
  });
}
void ref_plan_destroy(void* p) { delete static_cast<RefPlan*>(p); }

// DFTNoise::prepare (dft_noise.cpp:26-41) of the plan's shared model, fed from
// `slices` ([location][tbsize][sbsize][sbsize], 8-bit amplitude units), then the
// published model copied to `power`.
int ref_plan_prepare_noise(void* p, const float* slices, int nloc, float* power, int count, char* err, size_t len) {
  return guarded(err, len, [&] {
    const Plan& pl = *static_cast<RefPlan*>(p)->plan;
    auto noise = pl.dft_noise();
    if (!noise) throw std::invalid_argument("plan has no sampled noise model");
    if (nloc != int(noise->locations.size())) throw std::invalid_argument("slice count differs from nlocation");
    const std::size_t slice = std::size_t(noise->block_size) * noise->block_size;
    noise->prepare([&](const NoiseLocation& location, int z, span2d::Span<float> out) {
      std::size_t l = 0;
      while (l < noise->locations.size() && &noise->locations[l] != &location) ++l;
      const float* src = slices + (l * std::size_t(noise->temporal_size) + std::size_t(z)) * slice;
      std::memcpy(out.data(), src, slice * sizeof(float));
    });
    auto model = noise->power();
    if (!model || int(model->size()) != count) throw std::invalid_argument("noise model size mismatch");
    std::memcpy(power, model->data(), model->size() * sizeof(float));
  });
}

int ref_plan_geometry(void* p, nf_axis* x, nf_axis* y, int* temporal, int* bins) {
  const Plan& pl = *static_cast<RefPlan*>(p)->plan;
  auto cp = [](const Axis& a, nf_axis* o) {
    o->length = a.length; o->block = a.block; o->overlap = a.overlap; o->step = a.step;
    o->count = a.count; o->cover = a.cover; o->offset = a.offset;
  };
  cp(pl.geometry.x, x);
  cp(pl.geometry.y, y);
  *temporal = pl.temporal_size;
  *bins = int(pl.fft.bins());
  return 0;
}

// storage: 1 = u8, 2 = u16, 4 = f32.
int ref_plan_process(void* p, int storage, const nf_const_plane* src, int n, const int* targets, int nt,
                     nf_plane dst, int frame, int plane, char* err, size_t len) {
  const Plan& pl = *static_cast<RefPlan*>(p)->plan;
  return guarded(err, len, [&] {
    if (storage == 1) run_process<std::uint8_t>(pl, src, n, targets, nt, dst, frame, plane);
    else if (storage == 2) run_process<std::uint16_t>(pl, src, n, targets, nt, dst, frame, plane);
    else run_process<float>(pl, src, n, targets, nt, dst, frame, plane);
  });
}

// Frames run concurrently: `threads` workers pull frame indices from a shared
// counter (the reference's concurrency model: one shared Plan, one workspace per
// request). Frame f uses sources[f*nslots .. f*nslots+nslots-1] and dsts[f].
int ref_plan_process_many(void* p, int storage, const nf_const_plane* sources, int nslots, nf_plane* dsts,
                          int nframes, int threads, char* err, size_t len) {
  const Plan& pl = *static_cast<RefPlan*>(p)->plan;
  std::atomic<int> next{0};
  std::atomic<int> status{0};
  std::string message;
  std::mutex mu;
  auto worker = [&] {
    for (;;) {
      const int f = next.fetch_add(1);
      if (f >= nframes || status.load()) return;
      char local[256] = {0};
      const int rc = ref_plan_process(p, storage, sources + std::size_t(f) * nslots, nslots, nullptr, 0, dsts[f], f,
                                      0, local, sizeof(local));
      if (rc) {
        std::lock_guard<std::mutex> lock(mu);
        status = rc;
        message = local;
      }
    }
  };
  (void)pl;
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
  for (auto& t : pool) t.join();
  if (status) return fail(err, len, message.c_str(), status);
  return 0;
}

// Kalman: state = complex L, float C, float Q per bin (kernels/kalman.hpp:5-14).
int ref_kalman_create(void* p, void** out, char* err, size_t len) {
  const Plan& pl = *static_cast<RefPlan*>(p)->plan;
  return guarded(err, len, [&] { *out = new KalmanState(pl.initial_kalman()); });
}
void ref_kalman_destroy(void* s) { delete static_cast<KalmanState*>(s); }
size_t ref_kalman_bins(void* s) { return static_cast<KalmanState*>(s)->last.size(); }
int ref_kalman_read(void* s, float* last, float* cov, float* proc) {
  const auto& st = *static_cast<KalmanState*>(s);
  std::memcpy(last, st.last.data(), st.last.size() * sizeof(std::complex<float>));
  std::memcpy(cov, st.covariance.data(), st.covariance.size() * sizeof(float));
  std::memcpy(proc, st.process.data(), st.process.size() * sizeof(float));
  return 0;
}
// Plan::pattern_candidate<T> (plan.cpp:271-277) copied to `power`, and publish_pattern.
int ref_plan_pattern_candidate(void* p, int storage, nf_const_plane src, float* power, int count, char* err,
                               size_t len) {
  const Plan& pl = *static_cast<RefPlan*>(p)->plan;
  return guarded(err, len, [&] {
    runtime::PublishedModel::Model m;
    if (storage == 1)
      m = pl.pattern_candidate<std::uint8_t>({static_cast<const std::uint8_t*>(src.data), src.width, src.height, src.stride_bytes});
    else if (storage == 2)
      m = pl.pattern_candidate<std::uint16_t>({static_cast<const std::uint16_t*>(src.data), src.width, src.height, src.stride_bytes});
    else
      m = pl.pattern_candidate<float>({static_cast<const float*>(src.data), src.width, src.height, src.stride_bytes});
    if (!m || int(m->size()) != count) throw std::invalid_argument("pattern size mismatch");
    std::memcpy(power, m->data(), m->size() * sizeof(float));
  });
}
int ref_plan_publish_pattern(void* p, const float* power, int count, char* err, size_t len) {
  const Plan& pl = *static_cast<RefPlan*>(p)->plan;
  return guarded(err, len, [&] {
    pl.publish_pattern(std::make_shared<const std::vector<float>>(power, power + count));
  });
}
int ref_kalman_advance(void* p, int storage, nf_const_plane src, void* s, char* err, size_t len) {
  const Plan& pl = *static_cast<RefPlan*>(p)->plan;
  auto& st = *static_cast<KalmanState*>(s);
  return guarded(err, len, [&] {
    if (storage == 1)
      pl.advance_kalman<std::uint8_t>({static_cast<const std::uint8_t*>(src.data), src.width, src.height, src.stride_bytes}, st);
    else if (storage == 2)
      pl.advance_kalman<std::uint16_t>({static_cast<const std::uint16_t*>(src.data), src.width, src.height, src.stride_bytes}, st);
    else
      pl.advance_kalman<float>({static_cast<const float*>(src.data), src.width, src.height, src.stride_bytes}, st);
  });
}
int ref_kalman_render(void* p, int storage, nf_const_plane src, nf_plane dst, void* s, char* err, size_t len) {
  const Plan& pl = *static_cast<RefPlan*>(p)->plan;
  const auto& st = *static_cast<KalmanState*>(s);
  return guarded(err, len, [&] {
    if (storage == 1)
      pl.render_kalman<std::uint8_t>({static_cast<const std::uint8_t*>(src.data), src.width, src.height, src.stride_bytes},
                                     {static_cast<std::uint8_t*>(dst.data), dst.width, dst.height, dst.stride_bytes}, st);
    else if (storage == 2)
      pl.render_kalman<std::uint16_t>({static_cast<const std::uint16_t*>(src.data), src.width, src.height, src.stride_bytes},
                                      {static_cast<std::uint16_t*>(dst.data), dst.width, dst.height, dst.stride_bytes}, st);
    else
      pl.render_kalman<float>({static_cast<const float*>(src.data), src.width, src.height, src.stride_bytes},
                              {static_cast<float*>(dst.data), dst.width, dst.height, dst.stride_bytes}, st);
  });
}

// FFT entry points (RealFFT / RealFFT3D, src/spectral/fft.hpp:11-62).
int ref_fft_r2c(int h, int w, const float* in, float* out) {
  RealFFT f(h, w);
  f.forward(in, reinterpret_cast<std::complex<float>*>(out));
  return 0;
}
int ref_fft_c2r(int h, int w, const float* in, float* out) {
  RealFFT f(h, w);
  f.inverse(reinterpret_cast<const std::complex<float>*>(in), out);
  return 0;
}
int ref_fft_r2c_3d(int d, int h, int w, const float* in, float* out) {
  RealFFT3D f(d, h, w);
  f.forward(in, reinterpret_cast<std::complex<float>*>(out));
  return 0;
}
int ref_fft_c2r_3d(int d, int h, int w, const float* in, float* out) {
  RealFFT3D f(d, h, w);
  f.inverse(reinterpret_cast<const std::complex<float>*>(in), out);
  return 0;
}

// Creation-time tables (windows.cpp, profile.cpp, fft3d_profile.cpp).
int ref_fft3d_window(int block, int overlap, int type, float* analysis, float* synthesis, char* err, size_t len) {
  return guarded(err, len, [&] {
    auto w = fft3d_window(block, overlap, type);
    std::memcpy(analysis, w.analysis.data(), w.analysis.size() * sizeof(float));
    std::memcpy(synthesis, w.synthesis.data(), w.synthesis.size() * sizeof(float));
  });
}
int ref_dft_window_3d(int tbsize, int block, int overlap, int mode, int swin, int twin, float sbeta, float tbeta,
                      int tmode, int tov, float* h, float* wscale, char* err, size_t len) {
  return guarded(err, len, [&] {
    auto w = dft_window_3d(tbsize, block, overlap, mode, swin, twin, sbeta, tbeta, 0, tmode, tov);
    std::memcpy(h, w.h.data(), w.h.size() * sizeof(float));
    *wscale = w.wscale;
  });
}
int ref_dft_profile(const nf_dft_config* c, float divisor, float* out, char* err, size_t len) {
  return guarded(err, len, [&] {
    const auto r = to_ref(*c);
    auto p = dft_profile(r.curves, r.tbsize, r.block, r.sigma, divisor, 0);
    std::memcpy(out, p.data(), p.size() * sizeof(float));
  });
}
int ref_fft3d_profile(int w, int h, const float* sigmas, float* out, char* err, size_t len) {
  return guarded(err, len, [&] {
    auto p = fft3d_profile(w, h, {sigmas[0], sigmas[1], sigmas[2], sigmas[3]}, 0);
    std::memcpy(out, p.data(), p.size() * sizeof(float));
  });
}
int ref_dither(const float* src, int w, int h, int src_stride, unsigned char* dst, int dst_stride, int mode, int seed,
               int frame, int plane, char* err, size_t len) {
  return guarded(err, len, [&] {
    dither_scalar({src, w, h, std::ptrdiff_t(src_stride) * 4}, {dst, w, h, dst_stride}, mode, seed, frame, plane);
  });
}
unsigned ref_dither_hash(unsigned seed, unsigned n, unsigned p, unsigned y, unsigned x) {
  return dither_hash(seed, n, p, y, x);
}
// The covering temporal blocks of an output frame (temporal_grid.hpp): up to `cap`
// blocks, each with its start, target slice and `size` clamped slots.
int ref_temporal_blocks(int frame, int length, int size, int overlap, long long* starts, int* targets, int* slots,
                        int cap, int* count, char* err, size_t len) {
  return guarded(err, len, [&] {
    const auto blocks = temporal_blocks(frame, length, size, overlap);
    *count = int(blocks.size());
    for (int i = 0; i < std::min(cap, *count); ++i) {
      starts[i] = blocks[size_t(i)].start;
      targets[i] = blocks[size_t(i)].target;
      for (int z = 0; z < size; ++z) slots[i * size + z] = blocks[size_t(i)].slots[size_t(z)];
    }
  });
}
} // extern "C"

// The product's transform arithmetic (fft_core.cuh) evaluated on the host, for
// bit-exact comparison against the reference codelets reached through RealFFT.
extern "C" int ref_replica_r2c(int h, int w, const float* in, float* out) {
  std::vector<nf::cf> th(static_cast<std::size_t>(h)), tw(static_cast<std::size_t>(w));
  for (int pass = 0; pass < 2; ++pass) {
    auto& t = pass ? tw : th;
    const int n = pass ? w : h;
    for (int m = 0; m < n; ++m) {
      const double a = 2.0 * 3.14159265358979323846264338327950288 * double(m) / double(n);
      t[std::size_t(m)] = {float(std::cos(a)), float(-std::sin(a))};
    }
  }
  nf::block_r2c(in, w, reinterpret_cast<nf::cf*>(out), w / 2 + 1, h, w, th.data(), tw.data());
  return 0;
}
extern "C" int ref_replica_c2r(int h, int w, const float* in, float* out) {
  std::vector<nf::cf> th(static_cast<std::size_t>(h)), tw(static_cast<std::size_t>(w));
  for (int pass = 0; pass < 2; ++pass) {
    auto& t = pass ? tw : th;
    const int n = pass ? w : h;
    for (int m = 0; m < n; ++m) {
      const double a = 2.0 * 3.14159265358979323846264338327950288 * double(m) / double(n);
      t[std::size_t(m)] = {float(std::cos(a)), float(-std::sin(a))};
    }
  }
  nf::block_c2r(reinterpret_cast<const nf::cf*>(in), w / 2 + 1, out, w, h, w, 1.0f / (float(w) * float(h)), th.data(),
                tw.data());
  return 0;
}
