// C ABI of the B200 pipeline (include/neo_fft_b200.h): plan creation, validation
// and kernel launches. Host-side checks mirror neo-fft's Plan::run
// (src/algorithms/plan.cpp:331-375) with the same error texts.
#include "neo_fft_b200.h"
#include "plan_build.hpp"
#include "tile_spatial.cuh"
#include "tile_volume.cuh"
#include "launch.hpp"
#include "kalman.cuh"
#define NF_ADJOINT_AUX_KERNELS
#include "adjoint.cuh"
#include "tile_temporal.cuh"
#include "pattern.cuh"
#include "dither.cuh"
#include "plan_info.hpp"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <atomic>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <queue>
#include <tuple>
#include <string>
#include <vector>

using nf::cf;

struct nf_plan {
  nfb::PlanTables t;
  nfd::DevPlan dev{};
  void* tables = nullptr;  // one device allocation holding every table
  int* err = nullptr;      // device error word
  int device = 0;
  float* learn = nullptr;  // FFT3D bt=1: replaceable per-bin noise table (inside `tables`)
  mutable std::mutex staging_mu;
  mutable void* staging = nullptr;  // device staging for the host-memory path
  mutable size_t staging_bytes = 0;
  std::atomic<bool> model_ready{false};  // sampled noise model published (primary table filled)
  // FFT3D pattern search (pfactor / pshow): device scratch for the plane's block spectra,
  // candidate scores, the chosen block's power and the preview block.
  struct Pattern {
    void* dev = nullptr;
    nfd::DevPlan* plan = nullptr;
    nfd::SpectraJob* job = nullptr;
    int* item_base = nullptr;
    float* weights = nullptr;
    cf* spectra = nullptr;
    float* scores = nullptr;
    float* power = nullptr;
    float* block = nullptr;
    cf* work = nullptr;  // preview block spectrum
    int nbc = 1, items = 0, cand_x0 = 0, cand_y0 = 0, cand_nx = 0, cand_ny = 0;
    size_t smem = 0;
  };
  mutable Pattern pattern;
  mutable std::mutex pattern_mu;
  // Page-locked host slots for the per-call work tables of the two-pass temporal path:
  // a copy from pageable memory would first wait for all earlier work on the stream.
  static constexpr int kUploadSlots = 8;
  mutable std::mutex upload_mu;
  mutable unsigned char* upload = nullptr;  // kUploadSlots x upload_slot bytes
  mutable size_t upload_slot = 0;
  mutable cudaEvent_t upload_done[kUploadSlots] = {};
  mutable int upload_next = 0;
  ~nf_plan() {
    for (cudaEvent_t& e : upload_done)
      if (e) {
        cudaEventSynchronize(e);
        cudaEventDestroy(e);
      }
    if (upload) cudaFreeHost(upload);
    if (pattern.dev) cudaFree(pattern.dev);
    if (tables) cudaFree(tables);
    if (err) cudaFree(err);
    if (staging) cudaFree(staging);
  }
};

struct nf_kalman_state {
  const nf_plan* plan = nullptr;
  size_t count = 0;
  int fp64 = 0;
  cf* last = nullptr;       // [count]
  void* covariance = nullptr;  // float or double [count]
  void* process = nullptr;
  ~nf_kalman_state() {
    if (last) cudaFree(last);
    if (covariance) cudaFree(covariance);
    if (process) cudaFree(process);
  }
};

// One persistent launch group: planes of one block shape and storage.
struct BatchGroup {
  int bh = 0, bw = 0, storage = 0, algo = 0, ctas = 0;
  int mapped = 0;  // planes staged through tensor maps
  size_t smem = 0;
  void* dev = nullptr;  // plans | shapes | jobs | tile_base | tiles_x
  nfd::BatchWork work{};
};

struct nf_batch {
  // Dithered 8-bit DFTTest items (nf_batch_create_indexed): the batch filters them into a
  // float accumulator plane, then the dither pass writes the item's output (plan.cpp:617-623),
  // as nf_plan_process_device does.
  struct DitherJob {
    const nf_plan* plan;
    float* acc;
    size_t pitch;  // bytes per accumulator row
    float* boundary;
    unsigned char* dst;
    long long dst_stride;
    int width, height, frame, plane;
  };
  std::vector<DitherJob> dithers;
  void* dither_mem = nullptr;
  std::vector<BatchGroup> groups;                 // the strip geometry in use (one of `variants`)
  std::vector<std::vector<BatchGroup>> variants;  // candidate geometries, timed on the first launch
  bool tuned = false;
  int chosen = -1;  // index into `variants` once tuned or selected
  std::vector<const nf_plan*> plans;  // distinct plans (sampled noise models are checked per launch)
  int* counters = nullptr;  // one queue head per group
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t capture_stream = nullptr;
  ~nf_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (capture_stream) cudaStreamDestroy(capture_stream);
    for (auto& v : variants)
      for (auto& g : v)
        if (g.dev) cudaFree(g.dev);
    if (counters) cudaFree(counters);
    if (dither_mem) cudaFree(dither_mem);
  }
};

// FFT3D temporal clips: per frame step, pass 1 (spectra of the newest frame of every
// clip into its ring of T frame spectra) then pass 2 (the outputs whose windows are
// complete). Work lists of every step are built and uploaded once at creation.
struct nf_clip_batch {
  std::vector<const nf_plan*> plans;  // distinct plans (sampled noise models are checked per launch)
  int bh = 0, bw = 0, storage = 0;
  int slice = 0;  // 0: FFT3D temporal clips; 1: DFTTest tmode 1 slice form
  size_t smem1 = 0, smem2 = 0, smem2p = 0;
  int nbc = 1, ctas2 = 1, ctas2p = 1;
  struct Step {
    nfd::SpectraWork w1{};
    nfd::VolumeSpectraWork w1v{};
    int items1 = 0;
    nfd::BatchWork w2{};   // frames filtered across time (slot or slice spectra)
    int tiles2 = 0;
    nfd::BatchWork w2p{};  // FFT3D clip-edge frames: single-frame pixel strips
    int tiles2p = 0;
  };
  std::vector<Step> steps;
  // DFTTest clips whose output frames share no transform (tmode 0: a frame's slot weight
  // depends on its place in each output's window; tmode 1 with tosize > 0: an output adds
  // several temporal blocks in temporal-block order over the whole tile; smode 0): one
  // filter call per output frame with the host layer's frame selection, in the batch's
  // launch and its graph.
  struct FrameCall {
    const nf_plan* plan;
    std::vector<nf_const_plane> sources;
    std::vector<int> targets;
    nf_plane dst;
  };
  std::vector<FrameCall> calls;
  void* dev = nullptr;      // plans | shapes | per-step job tables
  void* rings = nullptr;    // frame spectra, T per clip plane
  void* tspec = nullptr;    // slot pointer arrays of the temporal jobs
  int* counters = nullptr;  // two work-queue heads per step (temporal, clip-edge pixel)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t capture_stream = nullptr;
  ~nf_clip_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (capture_stream) cudaStreamDestroy(capture_stream);
    for (void* q : {dev, rings, tspec, static_cast<void*>(counters)})
      if (q) cudaFree(q);
  }
};

// Streamed host form: frames in host memory through a ring of device slots; chunk c
// uses slot c % depth. Host->device copies, device->host copies and each slot's
// batched launch run on their own streams ordered by per-slot events (ready: inputs
// staged; done: outputs written; free: outputs copied back), so the copies of
// neighbouring chunks overlap the launch of this one, and the next chunk's CTAs take
// the SMs that this launch's tail leaves idle.
struct nf_host_batch {
  std::vector<const nf_plan*> plans;
  std::vector<size_t> pitch, offset;  // per plane of a frame: device row pitch, offset in the frame
  size_t frame_bytes = 0;             // device bytes of one frame (all planes)
  int chunk = 1, depth = 2;
  void* dev = nullptr;                // depth slots x (chunk input frames | chunk output frames)
  struct Slot {
    std::vector<nf_batch*> batches;   // [n - 1]: the slot's first n frames, built on first use
    cudaEvent_t ready = nullptr, done = nullptr, free = nullptr;
    cudaStream_t run = nullptr;       // the slot's launches
  };
  std::vector<Slot> slots;
  cudaStream_t h2d = nullptr, d2h = nullptr;
  cudaEvent_t start = nullptr, end = nullptr;
  unsigned char* frame_ptr(int slot, int f, bool out) const {
    return static_cast<unsigned char*>(dev) + (size_t(slot) * 2 + (out ? 1 : 0)) * size_t(chunk) * frame_bytes +
           size_t(f) * frame_bytes;
  }
  ~nf_host_batch() {
    for (cudaStream_t s : {h2d, d2h})
      if (s) cudaStreamSynchronize(s);
    for (auto& s : slots)
      if (s.run) cudaStreamSynchronize(s.run);
    for (auto& s : slots) {
      for (nf_batch* b : s.batches) delete b;
      for (cudaEvent_t e : {s.ready, s.done, s.free})
        if (e) cudaEventDestroy(e);
      if (s.run) cudaStreamDestroy(s.run);
    }
    for (cudaEvent_t e : {start, end})
      if (e) cudaEventDestroy(e);
    for (cudaStream_t s : {h2d, d2h})
      if (s) cudaStreamDestroy(s);
    if (dev) cudaFree(dev);
  }
};

namespace {

nf_status fail(char* err, size_t len, const std::string& msg, nf_status code) {
  if (err && len) {
    std::strncpy(err, msg.c_str(), len - 1);
    err[len - 1] = 0;
  }
  return code;
}
nf_status cuda_fail(char* err, size_t len, cudaError_t e, const char* what) {
  return fail(err, len, std::string(what) + ": " + cudaGetErrorString(e), NF_DEVICE_ERROR);
}
// A failed CUDA call inside a guarded body (reported as NF_DEVICE_ERROR).
struct CudaFailure {
  cudaError_t e;
  const char* what;
};
inline void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaFailure{e, what};
}
template <class F>
nf_status guarded(char* err, size_t len, F&& f) {
  try {
    return f();
  } catch (const CudaFailure& c) {
    return cuda_fail(err, len, c.e, c.what);
  } catch (const std::invalid_argument& e) {
    return fail(err, len, e.what(), NF_INVALID_ARGUMENT);
  } catch (const std::runtime_error& e) {
    return fail(err, len, e.what(), NF_NON_FINITE);
  } catch (const std::bad_alloc&) {
    return fail(err, len, "host allocation failed", NF_DEVICE_ERROR);
  }
}

int storage_of(nf_format f) { return f.floating ? nfd::kStoreF32 : (f.bits == 8 ? nfd::kStoreU8 : nfd::kStoreU16); }

// Stream-ordered scratch of the per-call paths comes from a pool per device that this
// library owns and that keeps freed memory for reuse. The device's default pool hands
// memory back to the system at every synchronisation, so the next call would map its
// scratch (hundreds of MB for the temporal paths at 1080p) afresh, and the mapping
// stalls the stream. The pools live until the process exits and hold their high-water
// mark of scratch.
cudaError_t scratch_alloc(void** ptr, size_t bytes, cudaStream_t st) {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = pools.find(dev);
    if (it == pools.end()) {
      cudaMemPoolProps props{};
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      if ((e = cudaMemPoolCreate(&pool, &props)) != cudaSuccess) return e;
      unsigned long long keep = ~0ull;
      if ((e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) return e;
      it = pools.emplace(dev, pool).first;
    }
    pool = it->second;
  }
  return cudaMallocFromPoolAsync(ptr, bytes, pool, st);
}

// Batched forms read each plan's primary table when they run, so a sampled noise model
// (DFTTest nlocation, FFT3D pfactor) must be published before every launch, as for
// nf_plan_process_device.
nf_status check_models(const std::vector<const nf_plan*>& plans, char* err, size_t len);

// Packs host tables into one aligned blob and records each table's offset.
struct Blob {
  std::vector<unsigned char> bytes;
  size_t add(const void* p, size_t n) {
    if (!n) return SIZE_MAX;
    const size_t off = (bytes.size() + 255) & ~size_t(255);
    bytes.resize(off + n);
    std::memcpy(bytes.data() + off, p, n);
    return off;
  }
  template <class T>
  size_t add(const std::vector<T>& v) {
    return add(v.data(), v.size() * sizeof(T));
  }
};

// Bulk-tensor staging of batched pixel strips. The driver's tensor-map encoder is
// reached through the runtime's entry-point query (no link against the driver library).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  return fn;
}

// Staged width of a strip shape in samples: the window rounded up to whole 4-sample
// groups, plus the remainder of the start column's 16-byte rounding, in whole boxes of
// 256 bytes (nfd::kStagingBoxBytes). 0 beyond eight boxes.
int tma_box_width(const nfd::StripShape& S, int storage) {
  const int align = 16 / storage, box = nfd::kStagingBoxBytes / storage;
  const int w = (((S.win_max + 3) & ~3) + align - 1 + box - 1) / box * box;
  return w <= 8 * box ? w : 0;
}

// The 2-D tensor map of a source plane with boxes of box_w x box_h samples, or false
// when the plane breaks a tensor-map rule (16-byte aligned base and row stride).
bool encode_plane_map(CUtensorMap* m, const void* base, int width, int height, long long stride, int storage, int box_w,
                      int box_h) {
  const auto fn = tensor_map_encoder();
  if (!fn || box_w <= 0 || box_h <= 0 || box_h > 256 || stride <= 0 || (stride & 15) != 0 ||
      (reinterpret_cast<uintptr_t>(base) & 15) != 0 || stride < (long long)width * storage)
    return false;
  const CUtensorMapDataType type = storage == nfd::kStoreU8    ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                                   : storage == nfd::kStoreU16 ? CU_TENSOR_MAP_DATA_TYPE_UINT16
                                                                : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const cuuint64_t dims[2] = {cuuint64_t(width), cuuint64_t(height)};
  const cuuint64_t strides[1] = {cuuint64_t(stride)};
  const cuuint32_t box[2] = {cuuint32_t(box_w), cuuint32_t(box_h)};
  const cuuint32_t elem_strides[2] = {1, 1};
  return fn(m, type, 2, const_cast<void*>(base), dims, strides, box, elem_strides, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

nfd::DevAxis dev_axis(const nfb::Axis& a) {
  return {a.length, a.block, a.overlap, a.step, a.count, a.cover, a.offset};
}

// Temporal twiddles of the FFT3D temporal kernel (get_fft3d_twiddles,
// src/kernels/scalar/spectral.cpp:67-88): binary64 angles, binary32 values.
void temporal_twiddles(int T, int c, std::vector<cf>& fwd, std::vector<cf>& inv) {
  constexpr double kPi = 3.1415926535897932384626433832795;
  fwd.assign(size_t(T) * T, cf{0, 0});
  inv.assign(size_t(T), cf{0, 0});
  for (int m = 0; m < T; ++m)
    for (int j = 0; j < T; ++j) {
      const double angle = -2.0 * kPi * double(j * m) / double(T);
      fwd[size_t(m) * T + j] = {float(std::cos(angle)), float(std::sin(angle))};
    }
  for (int m = 0; m < T; ++m) {
    const double a = +2.0 * kPi * double(c * m) / double(T);
    inv[size_t(m)] = {float(std::cos(a)), float(std::sin(a))};
  }
}

// DFTTest plans always carry a device primary table so it can be replaced
// (nf_plan_set_primary); without sigma curves it holds the uniform value a, which
// gives the same per-bin arithmetic as the uniform path.
// FFT3D bt=1 denoising plans (no Kalman, no sampled pattern, no preview) keep a per-bin
// noise table that nf_plan_set_primary can replace (the learnable table of the
// differentiable FFT3D): the profile table of varying sigmas, or the uniform value a.
// Until it is replaced the plan filters with its own table or uniform value.
bool fft3d_learnable(const nfb::PlanTables& t) {
  return t.algo == nfb::Algo::FFT3D && t.temporal_size == 1 && t.denoise && !t.kalman && !t.needs_pattern &&
         !t.preview;
}
std::vector<float> learn_table(const nfb::PlanTables& t) {
  if (!fft3d_learnable(t)) return {};
  if (!t.spectral.primary.empty()) return t.spectral.primary;
  return std::vector<float>(size_t(t.bins), t.spectral.a);
}

std::vector<float> primary_table(const nfb::PlanTables& t) {
  if (t.algo == nfb::Algo::FFT3D && t.needs_pattern) return std::vector<float>(size_t(t.bins), 0.0f);
  if (t.algo != nfb::Algo::DFTTest || !t.spectral.primary.empty()) return t.spectral.primary;
  return std::vector<float>(size_t(t.temporal_size) * size_t(t.bins), t.spectral.a);
}

nf_status finalize_plan(std::unique_ptr<nf_plan>& p, char* err, size_t len) {
  const nfb::PlanTables& t = p->t;
  cudaError_t e = cudaGetDevice(&p->device);
  if (e != cudaSuccess) return cuda_fail(err, len, e, "no CUDA device");
  Blob blob;
  const auto twh = nfb::twiddle_table(t.bh), tww = nfb::twiddle_table(t.bw), twt = nfb::twiddle_table(t.temporal_size);
  std::vector<cf> tfwd, tinv;
  temporal_twiddles(std::max(1, t.temporal_size), t.temporal_size / 2, tfwd, tinv);
  const size_t o_wxa = blob.add(t.wx.analysis), o_wya = blob.add(t.wy.analysis), o_wxs = blob.add(t.wx.synthesis),
               o_wys = blob.add(t.wy.synthesis), o_h = blob.add(t.h), o_hs = blob.add(t.h_synthesis),
               o_grid = blob.add(t.grid), o_prim = blob.add(primary_table(t)), o_learn = blob.add(learn_table(t)),
               o_sw = blob.add(t.enhancement.sharpen_window), o_hw = blob.add(t.enhancement.halo_window),
               o_twh = blob.add(twh), o_tww = blob.add(tww), o_twt = blob.add(twt), o_tf = blob.add(tfwd),
               o_ti = blob.add(tinv);
  if ((e = cudaMalloc(&p->tables, std::max<size_t>(blob.bytes.size(), 256))) != cudaSuccess)
    return cuda_fail(err, len, e, "device allocation failed");
  if ((e = cudaMemcpy(p->tables, blob.bytes.data(), blob.bytes.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
    return cuda_fail(err, len, e, "table upload failed");
  if ((e = cudaMalloc(&p->err, sizeof(int))) != cudaSuccess) return cuda_fail(err, len, e, "device allocation failed");
  if ((e = cudaMemset(p->err, 0, sizeof(int))) != cudaSuccess) return cuda_fail(err, len, e, "device memset failed");
  auto* base = static_cast<unsigned char*>(p->tables);
  auto ptr = [&](size_t off) -> const void* { return off == SIZE_MAX ? nullptr : base + off; };

  nfd::DevPlan& d = p->dev;
  d.algo = t.algo == nfb::Algo::FFT3D ? 0 : 1;
  d.gx = dev_axis(t.gx);
  d.gy = dev_axis(t.gy);
  d.bh = t.bh;
  d.bw = t.bw;
  d.K = t.bw / 2 + 1;
  d.bins = t.bins;
  d.T = t.temporal_size;
  d.storage = storage_of(t.format);
  const bool int_chroma = !t.format.floating && t.format.chroma;
  if (d.algo == 0) {
    d.dec_base = int_chroma ? float(1 << (t.format.bits - 1)) : 0.0f;
    d.dec_scale = 1.0f;
    d.out_base = d.dec_base;
    d.out_scale = 1.0f;
  } else {
    d.dec_base = 0.0f;
    d.dec_scale = t.format.floating ? 255.0f : 1.0f / float(1 << (t.format.bits - 8));
    d.out_base = 0.0f;
    d.out_scale = t.format.floating ? 1.0f / 255.0f : float(1 << (t.format.bits - 8));
  }
  d.out_peak = t.format.floating ? 1.0f : float((1 << t.format.bits) - 1);
  d.wxa = static_cast<const float*>(ptr(o_wxa));
  d.wya = static_cast<const float*>(ptr(o_wya));
  d.wxs = static_cast<const float*>(ptr(o_wxs));
  d.wys = static_cast<const float*>(ptr(o_wys));
  d.h = static_cast<const float*>(ptr(o_h));
  d.hsyn = static_cast<const float*>(ptr(o_hs));
  d.grid = static_cast<const cf*>(ptr(o_grid));
  d.mean_scale = t.mean_scale;
  const auto& s = t.spectral;
  const auto& en = t.enhancement;
  d.filt = {s.type,  s.a, s.b, s.low, s.high, s.exponent, s.floor, static_cast<const float*>(ptr(o_prim)),
            s.fused_enhancement ? 1 : 0,
            en.sharpen, en.dehalo, en.a, en.b, en.c,
            static_cast<const float*>(ptr(o_sw)), static_cast<const float*>(ptr(o_hw))};
  d.enh = {-2, 0, 0, 0, 0, 1, 0, nullptr, en.active() ? 1 : 0, en.sharpen, en.dehalo, en.a, en.b, en.c,
           static_cast<const float*>(ptr(o_sw)), static_cast<const float*>(ptr(o_hw))};
  {  // ftype 0 exponent tests of spectral.cpp:25-27, once per plan instead of per bin
    const float e1 = s.exponent - 1.0f, e5 = s.exponent - 0.5f;
    d.filt.emode = std::fabs(e1) < 0.00005f ? 0 : std::fabs(e5) < 0.00005f ? 1 : 2;
  }
  if (d.algo == 0)
    d.fft3d_mode = !t.denoise ? nfd::kEnhanceOnly
                              : (!s.primary.empty() || t.needs_pattern ? nfd::kWienerThenEnh : nfd::kWienerFused);
  d.codelet = (t.bh == t.bw && (t.bw == 8 || t.bw == 16 || t.bw == 32)) ? 1 : 0;
  d.twh = static_cast<const cf*>(ptr(o_twh));
  d.tww = static_cast<const cf*>(ptr(o_tww));
  d.twt = static_cast<const cf*>(ptr(o_twt));
  d.tfwd = static_cast<const cf*>(ptr(o_tf));
  d.tinv = static_cast<const cf*>(ptr(o_ti));
  d.center = t.center ? 1 : 0;
  d.err = p->err;
  d.lower = (t.beta - 1.0f) / t.beta;
  // NoisePower of the temporal path (plan.cpp:421-425): T*sigma^2/norm or table*T.
  d.noise_uniform = ((float(t.temporal_size) * t.sigma_eff) * t.sigma_eff) / t.norm;
  d.noise_mult = float(t.temporal_size);
  d.kalman_r0 = t.kalman_r0;
  d.kalman_ratio2 = t.kalman_ratio2;
  p->learn = static_cast<float*>(const_cast<void*>(ptr(o_learn)));
  return NF_OK;
}

// --- plane validation (checked_plane / plane_extent, src/base/checked.hpp:43-79) ---
size_t plane_extent(long long w, long long h, ptrdiff_t stride, size_t elem) {
  nfb::require(w > 0 && w <= INT32_MAX && h > 0 && h <= INT32_MAX, "dimension outside int32 domain");
  nfb::require(stride > 0 && stride % ptrdiff_t(elem) == 0 && stride / ptrdiff_t(elem) <= INT32_MAX,
               "invalid plane byte stride");
  const size_t row = size_t(w) * elem;
  nfb::require(size_t(stride) >= row, "stride shorter than active row");
  return size_t(h - 1) * size_t(stride) + row;
}
void check_pointer(const void* data, size_t elem) {
  nfb::require(data && reinterpret_cast<uintptr_t>(data) % elem == 0, "invalid plane pointer alignment");
}
void disjoint(const void* a, size_t an, const void* b, size_t bn) {
  const auto ap = reinterpret_cast<uintptr_t>(a), bp = reinterpret_cast<uintptr_t>(b);
  nfb::require(ap + an <= bp || bp + bn <= ap, "partially overlapping or aliased buffers");
}

struct Checked {
  int tslots = 1;
  int unique = 0;
};

Checked validate_call(const nf_plan& p, const nf_const_plane* sources, int n, const int* targets, int nt,
                      const nf_plane& dst) {
  const auto& t = p.t;
  nfb::require(n > 0 && sources, "sources must not be empty");
  nfb::require(n <= 225, "too many temporal slots");
  Checked c;
  c.tslots = t.temporal_ola ? t.temporal_size : n;
  if (t.temporal_ola) {
    nfb::require(nt > 0 && nt <= 15 && n == nt * t.temporal_size, "invalid temporal block inputs");
    for (int i = 0; i < nt; ++i) nfb::require(targets[i] >= 0 && targets[i] < c.tslots, "invalid target temporal slice");
  }
  if (t.algo == nfb::Algo::DFTTest)
    nfb::require(c.tslots == t.temporal_size, "DFTTest sources size must match plan temporal_size");
  else
    nfb::require(c.tslots == t.temporal_size || c.tslots == 1,
                 "FFT3D sources size must match plan temporal_size or single-frame fallback");
  nfb::require(dst.width == t.gx.length && dst.height == t.gy.length, "frame dimensions differ from plan");
  const size_t elem = size_t(storage_of(t.format));
  const size_t de = plane_extent(dst.width, dst.height, dst.stride_bytes, elem);
  check_pointer(dst.data, elem);
  for (int j = 0; j < n; ++j) {
    const auto& s = sources[j];
    nfb::require(s.width == t.gx.length && s.height == t.gy.length, "frame dimensions differ from plan");
    bool seen = false;
    for (int i = 0; i < j; ++i)
      if (sources[i].data == s.data && sources[i].stride_bytes == s.stride_bytes) seen = true;
    if (seen) continue;
    const size_t se = plane_extent(s.width, s.height, s.stride_bytes, elem);
    check_pointer(s.data, elem);
    disjoint(s.data, se, dst.data, de);
    ++c.unique;
  }
  return c;
}

// Resident CTAs of the plain launch: two per SM for blocks up to 16x16, else one.

// What the tiles of a strip launch compute: pixels staged and transformed forward and
// back (all phases), or spectra that are already in memory (FFT3D temporal pass 2,
// DFTTest slices, Kalman render), whose tiles skip the staging ring and the forward rows.
// Pixels: pixel tiles of plain launches; Staged: pixel tiles of batches, whose shared
// memory also holds the two raw boxes of the bulk-tensor staging.
enum class StripWork { Pixels, Temporal, Slice, Kalman, Staged };

// Resident CTAs of a plain strip launch: two per SM up to 16x16 blocks, and for Kalman
// renders up to 32x32 (kalman_render_kernel); one otherwise.
bool two_per_sm(const nfd::DevPlan& d, StripWork w) {
  return d.bh * d.bw <= 256 || (w == StripWork::Kalman && d.bh * d.bw <= 1024 && d.bh == d.bw &&
                                (d.bw == 8 || d.bw == 12 || d.bw == 16 || d.bw == 32));
}
int plain_ctas(const nfd::DevPlan& d, StripWork w) { return (two_per_sm(d, w) ? 2 : 1) * 148; }

// Modelled duration of one strip tile of `cols` x `rows` output samples: per block row,
// rounds of 256 threads over the row phases (nb*bh real rows forward and inverse, weight
// 1 each) and the column phase (nb*(bw/2+1) complex columns: forward, filter and
// inverse, weight 3; temporal filter or Kalman gain and inverse, 2; inverse only, 1),
// times the block rows plus a setup of two.
double tile_cost(const nfd::DevPlan& d, int cols, int rows, StripWork w) {
  const int K = d.bw / 2 + 1;
  const int nb = (cols + d.bw - d.gx.step + d.gx.step - 1) / d.gx.step;
  const int br = (rows + d.bh - d.gy.step + d.gy.step - 1) / d.gy.step + 2;
  const bool px = w == StripWork::Pixels || w == StripWork::Staged;
  const double wrows = px ? 2.0 : 1.0;
  const double wcols = px ? 3.0 : w == StripWork::Slice ? 1.0 : 2.0;
  return (wrows * ((nb * d.bh + 255) / 256) + wcols * ((nb * K + 255) / 256)) * br;
}

// Strip geometry. plain_planes > 0: one plain launch over that many planes (grid of
// strips x segments x planes); the segment height aims the grid at one wave of resident
// CTAs and the strip width minimises the modelled launch time (the tiles' greedy
// schedule over the resident CTAs). plain_planes == 0: batched forms, whose callers set
// the segment height; the width minimises the modelled work per owned column. Both keep
// the shared-memory budget of the occupancy target (two CTAs per SM up to 16x16 blocks,
// one above). Returns every feasible width, best modelled first (batched forms time the
// first few on their first launch). Results are cached per geometry: plain launches ask on
// every call.
std::vector<nfd::StripShape> strip_candidates(const nfd::DevPlan& d, int plain_planes, StripWork work) {
  struct Key {
    int len_x, len_y, bh, bw, sx, sy, tab, planes, work;
    bool operator<(const Key& o) const {
      return std::tie(len_x, len_y, bh, bw, sx, sy, tab, planes, work) <
             std::tie(o.len_x, o.len_y, o.bh, o.bw, o.sx, o.sy, o.tab, o.planes, o.work);
    }
  };
  static std::mutex memo_mu;
  static std::map<Key, std::vector<nfd::StripShape>> memo;
  const Key key{d.gx.length, d.gy.length, d.bh, d.bw, d.gx.step, d.gy.step, nfd::strip_table_floats(d), plain_planes,
                int(work)};
  {
    std::lock_guard<std::mutex> lock(memo_mu);
    const auto it = memo.find(key);
    if (it != memo.end()) return it->second;
  }
  const int edge = (d.bw + d.gx.step - 1) / d.gx.step - 1;  // blocks beyond the owned columns
  auto shape = [&](int nbx) {
    nfd::StripShape c;
    c.tab_floats = nfd::strip_table_floats(d);
    c.tma_box_w = 0;
    c.raw_bytes = 0;
    c.tw = std::min(std::max(d.gx.step, (nbx - edge) * d.gx.step), d.gx.length);
    c.nbx_max = (c.tw + d.bw - 1) / d.gx.step + 2;
    c.win_max = (c.nbx_max - 1) * d.gx.step + d.bw;
    int q = (c.win_max + 3) / 4;
    if (q % 2 == 0) ++q;  // odd float4 count: consecutive staged rows start in different banks
    // Staging ring: pixel tiles only (DFTTest slices, Kalman renders and FFT3D temporal
    // tiles have no pixel input). Temporal tiles of 48x48 blocks use it as the scratch
    // through which their teams of four lanes exchange row-transform runs.
    if (work == StripWork::Pixels || work == StripWork::Staged) {
      c.ring_pitch = 4 * q;
      if (work == StripWork::Staged) {  // raw boxes: staged width x step samples, two buffers
        c.tma_box_w = tma_box_width(c, d.storage);
        c.raw_bytes = int((size_t(c.tma_box_w) * d.gy.step * size_t(d.storage) + 127) & ~size_t(127));
        if (c.tma_box_w == 0) c.raw_bytes = 0;
      }
    } else if (work == StripWork::Temporal && d.bh == 48 && d.bw == 48) {  // 512-thread CTAs
      int t = (nfd::team_scratch_floats(d.bw, 512) + d.bh - 1) / d.bh;
      t = (t + 3) / 4;
      c.ring_pitch = 4 * t;
    } else {
      c.ring_pitch = 0;
    }
    c.th = d.gy.length;
    return c;
  };
  const size_t budget = size_t(two_per_sm(d, work) ? 110 : 200) * 1024;
  const int slots = plain_ctas(d, work);
  std::vector<std::pair<double, nfd::StripShape>> ranked;
  std::vector<double> costs;
  for (int nbx = edge + 2; nbx <= 128; ++nbx) {
    nfd::StripShape c = shape(nbx);
    if (nfd::strip_smem_bytes(d.bh, d.bw, c) > budget) continue;
    double cost;
    if (plain_planes > 0) {
      // Segment count: the shortest simulated schedule of the grid over the resident
      // CTAs (taller segments recompute fewer overlapping block rows; more segments fill
      // more SMs on small planes).
      const int strips = (d.gx.length + c.tw - 1) / c.tw;
      const int max_segs = std::max(1, std::min(d.gy.length / std::max(8, d.gy.step),
                                                (4 * slots + strips * plain_planes - 1) / (strips * plain_planes)));
      double best_span = -1.0;
      int best_th = d.gy.length;
      for (int segs = 1; segs <= max_segs; ++segs) {
        const int th = std::max(1, (d.gy.length + segs - 1) / segs);
        if (segs > 1 && th == (d.gy.length + segs - 2) / (segs - 1)) continue;  // same height as segs - 1
        costs.clear();
        for (int z = 0; z < plain_planes; ++z)
          for (int y0 = 0; y0 < d.gy.length; y0 += th)
            for (int x0 = 0; x0 < d.gx.length; x0 += c.tw)
              costs.push_back(tile_cost(d, std::min(c.tw, d.gx.length - x0), std::min(th, d.gy.length - y0), work));
        std::priority_queue<double, std::vector<double>, std::greater<double>> free_at;
        double span = 0;
        for (double t : costs) {
          double t0 = 0;
          if (int(free_at.size()) >= slots) {
            t0 = free_at.top();
            free_at.pop();
          }
          free_at.push(t0 + t);
          span = std::max(span, t0 + t);
        }
        if (best_span < 0 || span < best_span) {
          best_span = span;
          best_th = th;
        }
      }
      c.th = best_th;
      cost = best_span;
    } else {
      cost = tile_cost(d, c.tw, 0, work) / double(c.tw);
    }
    ranked.emplace_back(cost, c);
    if (c.tw >= d.gx.length) break;  // wider strips own no more columns
  }
  std::stable_sort(ranked.begin(), ranked.end(),
                   [](const auto& a, const auto& b) { return a.first < b.first; });
  std::vector<nfd::StripShape> out;
  for (const auto& r : ranked) out.push_back(r.second);
  if (out.empty()) {  // over the budget even at its narrowest
    nfd::StripShape c = shape(edge + 2);
    if (nfd::strip_smem_bytes(d.bh, d.bw, c) > size_t(227) * 1024) c.tma_box_w = c.raw_bytes = 0;
    out.push_back(c);
  }
  std::lock_guard<std::mutex> lock(memo_mu);
  return memo.emplace(key, out).first->second;
}

nfd::StripShape pick_strip(const nfd::DevPlan& d, int plain_planes, StripWork work) {
  return strip_candidates(d, plain_planes, work).front();
}

// Segment height of the strips of a batch group. The device queue hands tiles to the
// resident CTAs in list order, so a launch lasts about as long as the greedy list
// schedule of its tiles (tile_cost) over those CTAs; the candidate height with the
// shortest schedule wins. `queue` lists each job's plan and strip width in queue order.
int batch_segment_height(const std::vector<std::pair<const nfd::DevPlan*, int>>& queue, int bh, long long slots,
                         StripWork work) {
  int seg_h = 256;
  double best = -1;
  std::vector<double> costs;
  for (int h : {64, 96, 128, 160, 192, 224, 256, 320, 384, 448, 512, 640, 768, 1024}) {
    if (h < 2 * bh) continue;
    costs.clear();
    for (const auto& q : queue) {
      const nfd::DevPlan& d = *q.first;
      const int len = d.gy.length, segs = std::max(1, (len + h - 1) / h), th = (len + segs - 1) / segs;
      for (int y0 = 0; y0 < len; y0 += th)
        for (int x0 = 0; x0 < d.gx.length; x0 += q.second)
          costs.push_back(tile_cost(d, std::min(q.second, d.gx.length - x0), std::min(th, len - y0), work));
    }
    std::priority_queue<double, std::vector<double>, std::greater<double>> free_at;
    double span = 0;
    for (double c : costs) {
      double t0 = 0;
      if ((long long)free_at.size() >= slots) {
        t0 = free_at.top();
        free_at.pop();
      }
      free_at.push(t0 + c);
      span = std::max(span, t0 + c);
    }
    if (best < 0 || span < best) {
      best = span;
      seg_h = h;
    }
  }
  return seg_h;
}


cudaError_t launch_spatial_shape(const nfd::DevPlan& d, const nfd::StripShape& S, dim3 grid, size_t smem,
                                 const nfd::PlaneJobs& job, cudaStream_t st) {
  if (d.bh == d.bw) {
    switch (d.bw) {
      case 8: return nfd::launch_spatial_8x8(d, S, grid, smem, job, st);
      case 16: return nfd::launch_spatial_16x16(d, S, grid, smem, job, st);
      case 32: return nfd::launch_spatial_32x32(d, S, grid, smem, job, st);
      case 12: return nfd::launch_spatial_12x12(d, S, grid, smem, job, st);
      case 48: return nfd::launch_spatial_48x48(d, S, grid, smem, job, st);
      default: break;
    }
  }
  return nfd::launch_spatial_0x0(d, S, grid, smem, job, st);
}

// One launch over J.n planes of one plan; the strip shape aims the whole grid at one
// wave of resident CTAs.
cudaError_t run_spatial_planes(const nfd::DevPlan& d, const nfd::PlaneJobs& J, cudaStream_t st) {
  bool render = true;  // every plane renders a Kalman state: no pixel tiles
  for (int i = 0; i < J.n; ++i) render = render && J.job[i].kalman_L != nullptr;
  const nfd::StripShape S = pick_strip(d, J.n, render ? StripWork::Kalman : StripWork::Pixels);
  const size_t smem = nfd::strip_smem_bytes(d.bh, d.bw, S);
  const dim3 grid((d.gx.length + S.tw - 1) / S.tw, (d.gy.length + S.th - 1) / S.th, J.n);
  if (render) {
    if (d.bh == d.bw) {
      switch (d.bw) {
        case 8: return nfd::launch_kalman_render_8x8(d, S, grid, smem, J, st);
        case 16: return nfd::launch_kalman_render_16x16(d, S, grid, smem, J, st);
        case 32: return nfd::launch_kalman_render_32x32(d, S, grid, smem, J, st);
        case 12: return nfd::launch_kalman_render_12x12(d, S, grid, smem, J, st);
        case 48: return nfd::launch_kalman_render_48x48(d, S, grid, smem, J, st);
        default: break;
      }
    }
    return nfd::launch_kalman_render_0x0(d, S, grid, smem, J, st);
  }
  return launch_spatial_shape(d, S, grid, smem, J, st);
}

cudaError_t run_spatial(const nfd::DevPlan& d, const void* src, ptrdiff_t ss, void* dst, ptrdiff_t ds, const cf* L,
                        cudaStream_t st) {
  nfd::PlaneJobs J{};
  J.n = 1;
  J.job[0] = {static_cast<const unsigned char*>(src), (long long)ss, static_cast<unsigned char*>(dst), (long long)ds,
              L, 0};
  return run_spatial_planes(d, J, st);
}

cudaError_t run_volume(const nfd::DevPlan& d, const nfd::VolumeSources& v, void* dst, ptrdiff_t ds, cudaStream_t st) {
  nfd::VolumeShape S;
  S.threads = 256;
  const int b = std::max(d.bh, d.bw);
  const size_t per_block = size_t(d.T) * d.bh * (d.bw / 2 + 1) * sizeof(cf);
  int tile = b <= 16 ? 64 : b <= 32 ? 64 : 48;
  S.tw = std::min(tile, d.gx.length);
  S.th = std::min(b <= 16 ? tile / 2 : tile, d.gy.length);
  S.nbc = int(std::max<size_t>(1, std::min<size_t>((96 * 1024) / per_block, (S.tw + d.bw - 1) / d.gx.step + 2)));
  while (nfd::volume_smem_bytes(d.bh, d.bw, d.T, S) > 200 * 1024 && S.nbc > 1) --S.nbc;
  while (nfd::volume_smem_bytes(d.bh, d.bw, d.T, S) > 200 * 1024 && S.tw > 8) {
    S.tw /= 2;
    S.th = std::max(1, S.th / 2);
  }
  const size_t smem = nfd::volume_smem_bytes(d.bh, d.bw, d.T, S);
  const dim3 grid((d.gx.length + S.tw - 1) / S.tw, (d.gy.length + S.th - 1) / S.th);
  if (d.bh == d.bw) {
    switch (d.bw) {
      case 8: return nfd::launch_volume_8x8(d, S, grid, smem, v, dst, ds, st);
      case 16: return nfd::launch_volume_16x16(d, S, grid, smem, v, dst, ds, st);
      case 32: return nfd::launch_volume_32x32(d, S, grid, smem, v, dst, ds, st);
      case 12: return nfd::launch_volume_12x12(d, S, grid, smem, v, dst, ds, st);
      case 48: return nfd::launch_volume_48x48(d, S, grid, smem, v, dst, ds, st);
      default: break;
    }
  }
  return nfd::launch_volume_0x0(d, S, grid, smem, v, dst, ds, st);
}

nf_status read_error_word(const nf_plan& p, cudaStream_t st, char* err, size_t len) {
  int h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, p.err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(err, len, e, "device synchronisation failed");
  if (h) {
    cudaMemsetAsync(p.err, 0, sizeof(int), st);
    cudaStreamSynchronize(st);
    if (h & nfd::kErrStaging) return fail(err, len, "a source staging copy did not complete", NF_DEVICE_ERROR);
    return fail(err, len, "non-finite sample or intermediate", NF_NON_FINITE);
  }
  return NF_OK;
}

// --- FFT3D pattern search (plan.cpp:227-288) ---
cudaError_t launch_spectra_shape(int bh, int bw, int storage, const nfd::SpectraWork& w, int items, size_t smem,
                                 cudaStream_t st);
nf_status alloc_pattern(nf_plan& p, char* err, size_t len) {
  const auto& t = p.t;
  auto& pt = p.pattern;
  int nbc = 1;
  for (int n = 2; n <= std::min(16, t.gx.count); ++n)
    if (nfd::spectra_smem_bytes(t.bh, t.bw, t.gx.step, n) <= 100 * 1024) nbc = n;
  pt.nbc = nbc;
  pt.smem = nfd::spectra_smem_bytes(t.bh, t.bw, t.gx.step, nbc);
  const int chunks = (t.gx.count + nbc - 1) / nbc;
  pt.items = chunks * t.gy.count;
  const bool automatic = t.px == 0 && t.py == 0;
  pt.cand_x0 = automatic ? 2 : t.px;
  pt.cand_y0 = automatic ? 2 : t.py;
  pt.cand_nx = automatic ? t.gx.count - 4 : 1;
  pt.cand_ny = automatic ? t.gy.count - 4 : 1;
  const size_t nblocks = size_t(t.gx.count) * t.gy.count;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off = (off + bytes + 255) & ~size_t(255);
    return o;
  };
  const size_t o_plan = take(sizeof(nfd::DevPlan)), o_job = take(sizeof(nfd::SpectraJob)), o_base = take(2 * sizeof(int)),
               o_w = take(t.sample_weights.size() * sizeof(float)), o_spec = take(nblocks * t.bins * sizeof(cf)),
               o_sc = take(size_t(pt.cand_nx) * pt.cand_ny * sizeof(float)), o_pw = take(size_t(t.bins) * sizeof(float)),
               o_blk = take(size_t(t.bh) * t.bw * sizeof(float)), o_work = take(size_t(t.bins) * sizeof(cf));
  cudaError_t e = cudaMalloc(&pt.dev, off);
  if (e != cudaSuccess) return cuda_fail(err, len, e, "device allocation failed");
  auto* b = static_cast<unsigned char*>(pt.dev);
  pt.plan = reinterpret_cast<nfd::DevPlan*>(b + o_plan);
  pt.job = reinterpret_cast<nfd::SpectraJob*>(b + o_job);
  pt.item_base = reinterpret_cast<int*>(b + o_base);
  pt.weights = reinterpret_cast<float*>(b + o_w);
  pt.spectra = reinterpret_cast<cf*>(b + o_spec);
  pt.scores = reinterpret_cast<float*>(b + o_sc);
  pt.power = reinterpret_cast<float*>(b + o_pw);
  pt.block = reinterpret_cast<float*>(b + o_blk);
  pt.work = reinterpret_cast<cf*>(b + o_work);
  const int base[2] = {0, pt.items};
  if ((e = cudaMemcpy(pt.plan, &p.dev, sizeof(nfd::DevPlan), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(pt.item_base, base, sizeof(base), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(pt.weights, t.sample_weights.data(), t.sample_weights.size() * sizeof(float),
                      cudaMemcpyHostToDevice)) != cudaSuccess)
    return cuda_fail(err, len, e, "pattern upload failed");
  return NF_OK;
}

void check_pattern_source(const nf_plan& p, const nf_const_plane& s) {
  nfb::require(s.width == p.t.gx.length && s.height == p.t.gy.length, "pattern plane dimensions differ from plan");
  const size_t elem = size_t(storage_of(p.t.format));
  plane_extent(s.width, s.height, s.stride_bytes, elem);
  check_pointer(s.data, elem);
}

// Scores every candidate block of `src` and returns the first minimum (row-major order);
// with `power`, also the chosen block's unscaled power. Synchronises `st`.
nf_status select_pattern(const nf_plan& p, const nf_const_plane& src, cudaStream_t st, int& bx, int& by,
                         std::vector<float>* power, char* err, size_t len) {
  check_pattern_source(p, src);
  auto& pt = p.pattern;
  const auto& t = p.t;
  const nfd::SpectraJob job{static_cast<const unsigned char*>(src.data), (long long)src.stride_bytes, pt.spectra, 0,
                            (t.gx.count + pt.nbc - 1) / pt.nbc};
  cudaError_t e = cudaMemcpyAsync(pt.job, &job, sizeof(job), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_fail(err, len, e, "pattern upload failed");
  const nfd::SpectraWork w{pt.plan, pt.job, pt.item_base, 1, pt.nbc};
  if ((e = launch_spectra_shape(t.bh, t.bw, storage_of(t.format), w, pt.items, pt.smem, st)) != cudaSuccess)
    return cuda_fail(err, len, e, "kernel launch failed");
  const int ncand = pt.cand_nx * pt.cand_ny;
  nfd::pattern_score_kernel<<<(ncand + 127) / 128, 128, 0, st>>>(pt.plan, pt.spectra, pt.weights, pt.cand_x0,
                                                                 pt.cand_y0, pt.cand_nx, pt.cand_ny, pt.scores);
  std::vector<float> scores(static_cast<size_t>(ncand));
  if ((e = cudaGetLastError()) != cudaSuccess ||
      (e = cudaMemcpyAsync(scores.data(), pt.scores, scores.size() * sizeof(float), cudaMemcpyDeviceToHost, st)) !=
          cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return cuda_fail(err, len, e, "pattern search failed");
  const nf_status s = read_error_word(p, st, err, len);
  if (s != NF_OK) return s;
  int best = -1;
  for (int c = 0; c < ncand; ++c) {
    if (!std::isfinite(scores[size_t(c)])) return fail(err, len, "non-finite sample or intermediate", NF_NON_FINITE);
    if (best < 0 || scores[size_t(c)] < scores[size_t(best)]) best = c;
  }
  nfb::require(best >= 0, "FFT3D no pattern candidate");
  bx = pt.cand_x0 + best % pt.cand_nx;
  by = pt.cand_y0 + best / pt.cand_nx;
  if (power) {
    nfd::pattern_power_kernel<<<1, 256, 0, st>>>(pt.plan, pt.spectra, bx, by, pt.power);
    power->resize(size_t(t.bins));
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(power->data(), pt.power, power->size() * sizeof(float), cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
      return cuda_fail(err, len, e, "pattern search failed");
  }
  return NF_OK;
}

// pattern_candidate (plan.cpp:271-277): the chosen block's power scaled by pfactor (1 for
// Kalman) and the sampling weights; the scaled table must survive the temporal multiplier.
nf_status pattern_candidate(const nf_plan& p, const nf_const_plane& src, cudaStream_t st, std::vector<float>& power,
                            char* err, size_t len) {
  int bx = 0, by = 0;
  const nf_status s = select_pattern(p, src, st, bx, by, &power, err, len);
  if (s != NF_OK) return s;
  const auto& t = p.t;
  const float factor = t.kalman ? 1.0f : t.pfactor, maximum = float(t.temporal_size);
  for (size_t k = 0; k < power.size(); ++k) {
    float v = factor * power[k];
    v = v * t.sample_weights[k];
    nfb::finite(maximum * v);
    power[k] = v;
  }
  if (t.kalman)
    for (float r : power) nfb::finite(std::max(r, 1e-15f) * t.kalman_ratio2);
  return NF_OK;
}

template <int ST>
cudaError_t preview_launch(const nf_plan& p, const nf_const_plane& src, const nf_plane& dst, int ox, int oy,
                           cudaStream_t st) {
  auto& pt = p.pattern;
  nfd::pattern_block_kernel<ST><<<1, 32, 0, st>>>(pt.plan, static_cast<const unsigned char*>(src.data),
                                                  (long long)src.stride_bytes, ox, oy, pt.work, pt.block);
  const dim3 b(32, 8), g((p.t.gx.length + 31) / 32, (p.t.gy.length + 7) / 8);
  nfd::pattern_fill_kernel<ST><<<g, b, 0, st>>>(pt.plan, static_cast<unsigned char*>(dst.data),
                                                (long long)dst.stride_bytes, ox, oy, pt.block);
  return cudaGetLastError();
}

// pshow: the chosen pattern block of the first source, everything else zero (plan.cpp:409-418).
nf_status preview_pattern(const nf_plan& p, const nf_const_plane& src, const nf_plane& dst, cudaStream_t st,
                          char* err, size_t len) {
  std::lock_guard<std::mutex> lock(p.pattern_mu);
  int bx = 0, by = 0;
  const nf_status s = select_pattern(p, src, st, bx, by, nullptr, err, len);
  if (s != NF_OK) return s;
  const int ox = bx * p.t.gx.step, oy = by * p.t.gy.step;
  const int storage = storage_of(p.t.format);
  const cudaError_t e = storage == nfd::kStoreU8    ? preview_launch<nfd::kStoreU8>(p, src, dst, ox, oy, st)
                        : storage == nfd::kStoreU16 ? preview_launch<nfd::kStoreU16>(p, src, dst, ox, oy, st)
                                                    : preview_launch<nfd::kStoreF32>(p, src, dst, ox, oy, st);
  if (e != cudaSuccess) return cuda_fail(err, len, e, "kernel launch failed");
  return NF_OK;
}

// DFTTest 8-bit output with dither > 0 goes through the error-diffusion pass
// (plan.cpp:617-623); other formats ignore dither.
bool dithers(const nfb::PlanTables& t) {
  return t.algo == nfb::Algo::DFTTest && t.dither > 0 && !t.format.floating && t.format.bits == 8;
}

nf_status filter_device(const nf_plan& p, const nfd::DevPlan& d, const nf_const_plane* sources, int n,
                        const int* targets, int nt, nf_plane dst, cudaStream_t st, char* err, size_t len);

// Filters into a float accumulator plane (stream-ordered scratch), then dithers it into dst.
nf_status process_dithered(const nf_plan& p, const nf_const_plane* sources, int n, const int* targets, int nt,
                           nf_plane dst, int frame, int plane, cudaStream_t st, char* err, size_t len,
                           int* err_word = nullptr) {
  nfb::require(frame >= 0 && plane >= 0, "invalid dither coordinates or mode");
  const int W = p.t.gx.length, H = p.t.gy.length;
  const size_t pitch = ((size_t(W) * sizeof(float) + 255) / 256) * 256;
  void* scratch = nullptr;
  cudaError_t e = scratch_alloc(&scratch, pitch * size_t(H) + size_t(W) * sizeof(float), st);
  if (e != cudaSuccess) return cuda_fail(err, len, e, "device allocation failed");
  auto* acc = static_cast<float*>(scratch);
  float* boundary = reinterpret_cast<float*>(static_cast<unsigned char*>(scratch) + pitch * size_t(H));
  nfd::DevPlan d = p.dev;
  d.raw_out = 1;
  if (err_word) d.err = err_word;
  const nf_plane raw{acc, W, H, ptrdiff_t(pitch)};
  const nf_status s = filter_device(p, d, sources, n, targets, nt, raw, st, err, len);
  if (s == NF_OK) {
    nfd::dither_kernel<<<1, std::min(nfd::kDitherRows, H), 0, st>>>(
        acc, (long long)(pitch / sizeof(float)), static_cast<unsigned char*>(dst.data), (long long)dst.stride_bytes, W,
        H, p.t.dither, unsigned(p.t.dither_seed), unsigned(frame), unsigned(plane), boundary, d.err);
    e = cudaGetLastError();
  }
  cudaFreeAsync(scratch, st);
  if (s != NF_OK) return s;
  if (e != cudaSuccess) return cuda_fail(err, len, e, "kernel launch failed");
  return NF_OK;
}

// err_word: a per-call error flag in place of the plan's (host-memory calls from several
// threads then report their own non-finite data).
nf_status process_device(const nf_plan& p, const nf_const_plane* sources, int n, const int* targets, int nt,
                          nf_plane dst, int frame, int plane, cudaStream_t st, char* err, size_t len,
                          int* err_word = nullptr) {
  if (dithers(p.t)) {
    validate_call(p, sources, n, targets, nt, dst);
    return process_dithered(p, sources, n, targets, nt, dst, frame, plane, st, err, len, err_word);
  }
  if (!err_word) return filter_device(p, p.dev, sources, n, targets, nt, dst, st, err, len);
  nfd::DevPlan d = p.dev;
  d.err = err_word;
  return filter_device(p, d, sources, n, targets, nt, dst, st, err, len);
}

cudaError_t launch_temporal_shape(int bh, int bw, int storage, int slice, const nfd::BatchWork& w, int ctas,
                                  size_t smem, cudaStream_t st);
cudaError_t launch_volume_spectra_shape(int bh, int bw, int storage, const nfd::VolumeSpectraWork& w, int items,
                                        size_t smem, cudaStream_t st);

// Block columns per chunk of the spectra passes. FFT3D frames: the least modelled work per
// block column (rounds of 256 threads over the n·bh rows and n·(bw/2+1) columns of the
// chunk) within the shared-memory budget of the occupancy the kernel's registers allow (two
// CTAs per SM up to 16x16 blocks, one above); ties go to the wider chunk. DFTTest volumes:
// the widest chunk within 100 KB. smem(n) is the pass's shared memory for n columns.
template <class SmemFn>
int pass1_chunk(int bh, int bw, int T, bool slice, int max_count, SmemFn smem) {
  const int K = bw / 2 + 1, tt = slice ? T : 1;
  const size_t budget = size_t(100) * 1024;  // two CTAs per SM (spectra_batch_kernel)
  int best_n = 1;
  double best = -1.0;
  if (slice) {  // DFTTest volumes: the widest chunk within 100 KB measured fastest
    for (int n = 2; n <= std::min(32, max_count); ++n)
      if (smem(n) <= size_t(100) * 1024) best_n = n;
    return best_n;
  }
  for (int n = 1; n <= std::min(16, max_count); ++n) {
    if (n > 1 && smem(n) > budget) break;  // shared memory grows with n
    const double c = (double((tt * n * bh + 255) / 256) + double((tt * n * K + 255) / 256) +
                      (slice ? double((bh * K * n + 255) / 256) : 0.0)) / double(n);
    if (best < 0 || c <= best) {
      best = c;
      best_n = n;
    }
  }
  return best_n;
}

// Per-call temporal filtering in two passes over stream-ordered scratch (the clip form's
// kernels for a single output): FFT3D bt 2..5 — the T slots' spatial spectra, then the
// temporal strip; DFTTest tmode 1 with one covering block — the volume's filtered slice
// spectra, then the slice strip of the target. The work tables travel in the same
// allocation (uploaded from host memory, which the copy stages before returning).
struct TwoPassHeader {
  nfd::DevPlan plan;
  nfd::StripShape shape;
  nfd::PlaneJob job;
  int base[2];
  int tiles_x;
  int counter;
};

nf_status run_two_pass(const nf_plan& p, const nfd::DevPlan& d, const nf_const_plane* sources, int T, int target,
                       const nf_plane& dst, cudaStream_t st, char* err, size_t len) {
  const auto& t = p.t;
  const bool slice = t.algo == nfb::Algo::DFTTest;
  const int storage = storage_of(t.format);
  const size_t frame = size_t(t.gy.count) * t.bins * t.gx.count;  // complex per slot spectrum
  const int nbc = pass1_chunk(t.bh, t.bw, T, slice, t.gx.count, [&](int n) {
    return slice ? nfd::volume_spectra_smem_bytes(t.bh, t.bw, T, t.gx.step, n)
                 : nfd::spectra_smem_bytes(t.bh, t.bw, t.gx.step, n);
  });
  const size_t smem1 = slice ? nfd::volume_spectra_smem_bytes(t.bh, t.bw, T, t.gx.step, nbc)
                             : nfd::spectra_smem_bytes(t.bh, t.bw, t.gx.step, nbc);
  const int chunks = (t.gx.count + nbc - 1) / nbc, items = chunks * t.gy.count;
  nfd::StripShape S = pick_strip(d, 1, slice ? StripWork::Slice : StripWork::Temporal);
  const size_t smem2 = nfd::strip_smem_bytes(t.bh, t.bw, S);
  const int tx = (t.gx.length + S.tw - 1) / S.tw, ty = (t.gy.length + S.th - 1) / S.th;

  auto al = [](size_t n) { return (n + 255) & ~size_t(255); };
  const size_t o_hdr = 0, o_slots = al(sizeof(TwoPassHeader)), o_jobs = o_slots + al(sizeof(cf*) * 16),
               o_base = o_jobs + al(std::max(sizeof(nfd::VolumeSpectraJob), sizeof(nfd::SpectraJob) * size_t(T))),
               o_spec = o_base + al(sizeof(int) * size_t(T + 1));
  const size_t bytes = o_spec + size_t(T) * al(frame * sizeof(cf));
  void* scratch = nullptr;
  cudaError_t e = scratch_alloc(&scratch, bytes, st);
  if (e != cudaSuccess) return cuda_fail(err, len, e, "device allocation failed");
  auto* b = static_cast<unsigned char*>(scratch);
  auto spec = [&](int z) { return reinterpret_cast<cf*>(b + o_spec + size_t(z) * al(frame * sizeof(cf))); };

  std::lock_guard<std::mutex> upload_lock(p.upload_mu);
  if (!p.upload || p.upload_slot < o_spec) {
    for (cudaEvent_t& ev : p.upload_done) {
      if (ev) cudaEventSynchronize(ev);
      else if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) break;
    }
    if (p.upload) cudaFreeHost(p.upload);
    p.upload = nullptr;
    p.upload_slot = 0;
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&p.upload), nf_plan::kUploadSlots * al(o_spec));
    if (e != cudaSuccess) {
      p.upload = nullptr;
      cudaFreeAsync(scratch, st);
      return cuda_fail(err, len, e, "host allocation failed");
    }
    p.upload_slot = al(o_spec);
  }
  const int us = p.upload_next;
  p.upload_next = (us + 1) % nf_plan::kUploadSlots;
  cudaEventSynchronize(p.upload_done[us]);  // the slot's previous copy has been read
  unsigned char* host = p.upload + size_t(us) * p.upload_slot;
  std::memset(host, 0, o_spec);
  auto* hdr = reinterpret_cast<TwoPassHeader*>(host + o_hdr);
  hdr->plan = d;
  hdr->shape = S;
  const int zt = slice ? target : 0;
  hdr->job = {nullptr, 0, static_cast<unsigned char*>(dst.data), (long long)dst.stride_bytes, nullptr, 0, zt,
              reinterpret_cast<const cf* const*>(b + o_slots + (slice ? sizeof(cf*) * size_t(zt) : 0))};
  hdr->base[0] = 0;
  hdr->base[1] = tx * ty;
  hdr->tiles_x = tx;
  hdr->counter = 0;
  auto* slots = reinterpret_cast<const cf**>(host + o_slots);
  for (int z = 0; z < T; ++z) slots[z] = spec(z);
  auto* base = reinterpret_cast<int*>(host + o_base);
  if (slice) {
    auto* vj = reinterpret_cast<nfd::VolumeSpectraJob*>(host + o_jobs);
    for (int z = 0; z < T; ++z) {
      vj->src[z] = static_cast<const unsigned char*>(sources[z].data);
      vj->src_stride[z] = sources[z].stride_bytes;
      vj->out[z] = spec(z);
    }
    vj->plan = 0;
    vj->chunks_x = chunks;
    base[0] = 0;
    base[1] = items;
  } else {
    auto* sj = reinterpret_cast<nfd::SpectraJob*>(host + o_jobs);
    for (int z = 0; z < T; ++z) {
      sj[z] = {static_cast<const unsigned char*>(sources[z].data), (long long)sources[z].stride_bytes, spec(z), 0,
               chunks};
      base[z] = z * items;
    }
    base[T] = T * items;
  }
  e = cudaMemcpyAsync(scratch, host, o_spec, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaEventRecord(p.upload_done[us], st);
  const auto* dplan = reinterpret_cast<const nfd::DevPlan*>(b + o_hdr + offsetof(TwoPassHeader, plan));
  if (e == cudaSuccess) {
    if (slice) {
      const nfd::VolumeSpectraWork w{dplan, reinterpret_cast<const nfd::VolumeSpectraJob*>(b + o_jobs),
                                     reinterpret_cast<const int*>(b + o_base), 1, nbc};
      e = launch_volume_spectra_shape(t.bh, t.bw, storage, w, items, smem1, st);
    } else {
      const nfd::SpectraWork w{dplan, reinterpret_cast<const nfd::SpectraJob*>(b + o_jobs),
                               reinterpret_cast<const int*>(b + o_base), T, nbc};
      e = launch_spectra_shape(t.bh, t.bw, storage, w, T * items, smem1, st);
    }
  }
  if (e == cudaSuccess) {
    nfd::BatchWork w{};
    w.plans = dplan;
    w.shapes = reinterpret_cast<const nfd::StripShape*>(b + o_hdr + offsetof(TwoPassHeader, shape));
    w.jobs = reinterpret_cast<const nfd::PlaneJob*>(b + o_hdr + offsetof(TwoPassHeader, job));
    w.job_tile_base = reinterpret_cast<const int*>(b + o_hdr + offsetof(TwoPassHeader, base));
    w.job_tiles_x = reinterpret_cast<const int*>(b + o_hdr + offsetof(TwoPassHeader, tiles_x));
    w.njobs = 1;
    w.counter = reinterpret_cast<int*>(b + o_hdr + offsetof(TwoPassHeader, counter));
    const int ctas2 = std::min(tx * ty, plain_ctas(d, slice ? StripWork::Slice : StripWork::Temporal));
    e = launch_temporal_shape(t.bh, t.bw, storage, slice ? 1 : 0, w, ctas2, smem2, st);
  }
  cudaFreeAsync(scratch, st);
  if (e != cudaSuccess) return cuda_fail(err, len, e, "kernel launch failed");
  return NF_OK;
}

nf_status check_models(const std::vector<const nf_plan*>& plans, char* err, size_t len) {
  for (const nf_plan* p : plans) {
    if (p->t.noise_model && !p->model_ready.load(std::memory_order_acquire))
      return fail(err, len, "DFTTest sample model not initialized", NF_INVALID_ARGUMENT);
    if (p->t.needs_pattern && !p->model_ready.load(std::memory_order_acquire))
      return fail(err, len, "FFT3D sampled model not initialized", NF_INVALID_ARGUMENT);
  }
  return NF_OK;
}

// The filter proper with the device plan `d` (the plan's own, or a copy that keeps the
// raw accumulator for the dither pass).
nf_status filter_device(const nf_plan& p, const nfd::DevPlan& d, const nf_const_plane* sources, int n,
                        const int* targets, int nt, nf_plane dst, cudaStream_t st, char* err, size_t len) {
  const Checked c = validate_call(p, sources, n, targets, nt, dst);
  cudaError_t e;
  if (p.t.algo == nfb::Algo::FFT3D && p.t.kalman)
    return fail(err, len, "Kalman plans render through nf_kalman_render_device", NF_INVALID_ARGUMENT);
  if (p.t.noise_model && !p.model_ready.load(std::memory_order_acquire))
    return fail(err, len, "DFTTest sample model not initialized", NF_INVALID_ARGUMENT);
  if (p.t.needs_pattern && !p.model_ready.load(std::memory_order_acquire))
    return fail(err, len, "FFT3D sampled model not initialized", NF_INVALID_ARGUMENT);
  if (p.t.preview) return preview_pattern(p, sources[0], dst, st, err, len);
  if (c.tslots == 1 && !p.t.temporal_ola) {
    e = run_spatial(d, sources[0].data, sources[0].stride_bytes, dst.data, dst.stride_bytes, nullptr, st);
  } else if (p.t.algo == nfb::Algo::FFT3D && c.tslots == p.t.temporal_size && !p.t.preview) {
    return run_two_pass(p, d, sources, c.tslots, 0, dst, st, err, len);
  } else if (p.t.algo == nfb::Algo::DFTTest && p.t.temporal_ola && nt == 1 && !p.t.center &&
             p.t.temporal_size <= nfd::kMaxVolumeSlots) {
    return run_two_pass(p, d, sources, p.t.temporal_size, targets[0], dst, st, err, len);
  } else {
    nfd::VolumeSources v{};
    for (int j = 0; j < n; ++j) {
      v.ptr[j] = static_cast<const unsigned char*>(sources[j].data);
      v.stride[j] = sources[j].stride_bytes;
    }
    v.ola = p.t.temporal_ola ? 1 : 0;
    v.nblocks = p.t.temporal_ola ? nt : 1;
    for (int i = 0; p.t.temporal_ola && i < nt; ++i) v.target[i] = targets[i];
    e = run_volume(d, v, dst.data, dst.stride_bytes, st);
  }
  if (e != cudaSuccess) return cuda_fail(err, len, e, "kernel launch failed");
  return NF_OK;
}

template <class T>
__global__ void fill_kernel(T* p, size_t n, T v) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) p[i] = v;
}

cudaError_t run_kalman_advance(const nfd::DevPlan& d, const void* src, ptrdiff_t ss, const nfd::KalmanArgs& a,
                               cudaStream_t st) {
  if (d.bh == d.bw) {
    switch (d.bw) {
      case 8: return nfd::launch_kalman_8x8(d, src, ss, a, st);
      case 16: return nfd::launch_kalman_16x16(d, src, ss, a, st);
      case 32: return nfd::launch_kalman_32x32(d, src, ss, a, st);
      case 12: return nfd::launch_kalman_12x12(d, src, ss, a, st);
      case 48: return nfd::launch_kalman_48x48(d, src, ss, a, st);
      default: break;
    }
  }
  return nfd::launch_kalman_0x0(d, src, ss, a, st);
}

void check_kalman_source(const nf_plan& p, const nf_const_plane& s) {
  nfb::require(p.t.kalman, "not a Kalman plan");
  nfb::require(s.width == p.t.gx.length && s.height == p.t.gy.length, "Kalman source shape differs");
  const size_t elem = size_t(storage_of(p.t.format));
  plane_extent(s.width, s.height, s.stride_bytes, elem);
  check_pointer(s.data, elem);
}

cudaError_t launch_batch_group(const BatchGroup& g, cudaStream_t st) {
  if (g.bh == g.bw) {
    switch (g.bw) {
      case 8: return nfd::launch_spatial_batch_8x8(g.storage, g.algo, g.work, g.ctas, g.smem, st);
      case 16: return nfd::launch_spatial_batch_16x16(g.storage, g.algo, g.work, g.ctas, g.smem, st);
      case 32: return nfd::launch_spatial_batch_32x32(g.storage, g.algo, g.work, g.ctas, g.smem, st);
      case 12: return nfd::launch_spatial_batch_12x12(g.storage, g.algo, g.work, g.ctas, g.smem, st);
      case 48: return nfd::launch_spatial_batch_48x48(g.storage, g.algo, g.work, g.ctas, g.smem, st);
      default: break;
    }
  }
  return nfd::launch_spatial_batch_0x0(g.storage, g.algo, g.work, g.ctas, g.smem, st);
}

cudaError_t launch_spectra_shape(int bh, int bw, int storage, const nfd::SpectraWork& w, int items, size_t smem,
                                 cudaStream_t st) {
  if (bh == bw) {
    switch (bw) {
      case 8: return nfd::launch_spectra_batch_8x8(storage, w, items, smem, st);
      case 16: return nfd::launch_spectra_batch_16x16(storage, w, items, smem, st);
      case 32: return nfd::launch_spectra_batch_32x32(storage, w, items, smem, st);
      case 12: return nfd::launch_spectra_batch_12x12(storage, w, items, smem, st);
      case 48: return nfd::launch_spectra_batch_48x48(storage, w, items, smem, st);
      default: break;
    }
  }
  return nfd::launch_spectra_batch_0x0(storage, w, items, smem, st);
}

cudaError_t launch_volume_spectra_shape(int bh, int bw, int storage, const nfd::VolumeSpectraWork& w, int items,
                                        size_t smem, cudaStream_t st) {
  if (bh == bw) {
    switch (bw) {
      case 8: return nfd::launch_volume_spectra_batch_8x8(storage, w, items, smem, st);
      case 16: return nfd::launch_volume_spectra_batch_16x16(storage, w, items, smem, st);
      case 32: return nfd::launch_volume_spectra_batch_32x32(storage, w, items, smem, st);
      case 12: return nfd::launch_volume_spectra_batch_12x12(storage, w, items, smem, st);
      case 48: return nfd::launch_volume_spectra_batch_48x48(storage, w, items, smem, st);
      default: break;
    }
  }
  return nfd::launch_volume_spectra_batch_0x0(storage, w, items, smem, st);
}

cudaError_t launch_temporal_shape(int bh, int bw, int storage, int slice, const nfd::BatchWork& w, int ctas,
                                  size_t smem, cudaStream_t st) {
  if (bh == bw) {
    switch (bw) {
      case 8: return nfd::launch_temporal_batch_8x8(storage, slice, w, ctas, smem, st);
      case 16: return nfd::launch_temporal_batch_16x16(storage, slice, w, ctas, smem, st);
      case 32: return nfd::launch_temporal_batch_32x32(storage, slice, w, ctas, smem, st);
      case 12: return nfd::launch_temporal_batch_12x12(storage, slice, w, ctas, smem, st);
      case 48: return nfd::launch_temporal_batch_48x48(storage, slice, w, ctas, smem, st);
      default: break;
    }
  }
  return nfd::launch_temporal_batch_0x0(storage, slice, w, ctas, smem, st);
}

} // namespace

extern "C" {

int nf_abi_version(void) { return NF_ABI_VERSION; }

void nf_copy_row(const void* source, void* dst, size_t bytes) {
  if (!bytes) return;
  // Pageable host memory the runtime has never seen reports cudaMemoryTypeUnregistered.
  cudaPointerAttributes a{}, b{};
  const bool src_host = cudaPointerGetAttributes(&a, source) == cudaSuccess && a.type == cudaMemoryTypeUnregistered;
  const bool dst_host = cudaPointerGetAttributes(&b, dst) == cudaSuccess && b.type == cudaMemoryTypeUnregistered;
  if (src_host && dst_host) std::memcpy(dst, source, bytes);
  else cudaMemcpy(dst, source, bytes, cudaMemcpyDefault);
}

nf_status nf_stream_create(void** stream, char* err, size_t len) {
  if (!stream) return NF_INVALID_ARGUMENT;
  cudaStream_t s = nullptr;
  const cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e != cudaSuccess) return cuda_fail(err, len, e, "stream creation failed");
  *stream = s;
  return NF_OK;
}

void nf_stream_destroy(void* stream) {
  if (stream) {
    cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    cudaStreamDestroy(static_cast<cudaStream_t>(stream));
  }
}

void nf_fft3d_config_default(nf_fft3d_config* c) {
  *c = nf_fft3d_config{};
  c->bw = 32; c->bh = 32; c->ow = -1; c->oh = -1; c->wintype = 0; c->opt = 0; c->bt = 1;
  c->sigma = 2; c->beta = 1; c->degrid = 1; c->kratio = 2;
  c->sharpen = 0; c->scutoff = .3f; c->svr = 1; c->smin = 4; c->smax = 20; c->dehalo = 0; c->hr = 2; c->ht = 50;
  c->pfactor = 0; c->pcutoff = .1f;
  c->cache_frames = -1; c->cache_mb = 128; c->kalman_warmup = 8;
}
void nf_dft_config_default(nf_dft_config* c) {
  *c = nf_dft_config{};
  c->block = 16; c->overlap = 12; c->mode = 1; c->swin = 0; c->twin = 7; c->ftype = 0; c->opt = 0; c->tbsize = 1;
  c->sbeta = 2.5f; c->tbeta = 2.5f; c->sigma = 8; c->sigma2 = 8; c->pmin = 0; c->pmax = 500; c->f0beta = 1;
  c->zmean = 1;
}

nf_status nf_plan_create_fft3d(int width, int height, nf_format format, const nf_fft3d_config* config,
                               nf_plan** plan, char* err, size_t err_len) {
  return guarded(err, err_len, [&]() -> nf_status {
    nfb::require(config && plan, "missing configuration or output pointer");
    auto p = std::make_unique<nf_plan>();
    p->t = nfb::build_fft3d(width, height, format, *config);
    nf_status s = finalize_plan(p, err, err_len);
    if (s != NF_OK) return s;
    if ((p->t.preview || p->t.needs_pattern) && (s = alloc_pattern(*p, err, err_len)) != NF_OK) return s;
    *plan = p.release();
    return NF_OK;
  });
}
nf_status nf_plan_create_dft(int width, int height, nf_format format, const nf_dft_config* config, nf_plan** plan,
                             char* err, size_t err_len) {
  return guarded(err, err_len, [&]() -> nf_status {
    nfb::require(config && plan, "missing configuration or output pointer");
    auto p = std::make_unique<nf_plan>();
    p->t = nfb::build_dft(width, height, format, *config);
    const nf_status s = finalize_plan(p, err, err_len);
    if (s != NF_OK) return s;
    *plan = p.release();
    return NF_OK;
  });
}
void nf_plan_destroy(nf_plan* plan) { delete plan; }

nf_status nf_plan_geometry(const nf_plan* p, nf_axis* x, nf_axis* y, int* temporal_size, int* bins) {
  if (!p) return NF_INVALID_ARGUMENT;
  auto cp = [](const nfb::Axis& a, nf_axis* o) {
    if (o) *o = {a.length, a.block, a.overlap, a.step, a.count, a.cover, a.offset};
  };
  cp(p->t.gx, x);
  cp(p->t.gy, y);
  if (temporal_size) *temporal_size = p->t.temporal_size;
  if (bins) *bins = p->t.bins;
  return NF_OK;
}

nf_status nf_plan_process_device(const nf_plan* p, const nf_const_plane* sources, int nsources, const int* targets,
                                 int ntargets, nf_plane dst, int frame, int plane, void* stream, char* err,
                                 size_t err_len) {
  return guarded(err, err_len, [&]() -> nf_status {
    nfb::require(p != nullptr, "null plan");
    return process_device(*p, sources, nsources, targets, ntargets, dst, frame, plane,
                          static_cast<cudaStream_t>(stream), err, err_len);
  });
}

nf_status nf_plan_process_planes_device(const nf_plan* p, const nf_const_plane* sources, const nf_plane* dsts,
                                        int nplanes, void* stream, char* err, size_t err_len) {
  return guarded(err, err_len, [&]() -> nf_status {
    nfb::require(p && sources && dsts, "null argument");
    nfb::require(nplanes > 0 && nplanes <= nfd::kMaxPlaneJobs, "multi-plane calls take 1..32 planes");
    nfb::require(!(p->t.algo == nfb::Algo::FFT3D && p->t.kalman), "Kalman plans render through nf_kalman_render_device");
    nfb::require(p->t.temporal_size == 1 && !p->t.temporal_ola,
                 "multi-plane calls take single-frame plans (FFT3D bt=1, DFTTest tbsize=1)");
    nfb::require(!dithers(p->t), "dithered 8-bit DFTTest output runs through nf_plan_process_device");
    nfd::PlaneJobs J{};
    J.n = nplanes;
    for (int i = 0; i < nplanes; ++i) {
      validate_call(*p, &sources[i], 1, nullptr, 0, dsts[i]);
      J.job[i] = {static_cast<const unsigned char*>(sources[i].data), (long long)sources[i].stride_bytes,
                  static_cast<unsigned char*>(dsts[i].data), (long long)dsts[i].stride_bytes, nullptr, 0};
    }
    const cudaError_t e = run_spatial_planes(p->dev, J, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(err, err_len, e, "kernel launch failed");
    return NF_OK;
  });
}

nf_status nf_plan_sync_status(const nf_plan* p, void* stream, char* err, size_t err_len) {
  if (!p) return fail(err, err_len, "null plan", NF_INVALID_ARGUMENT);
  return read_error_word(*p, static_cast<cudaStream_t>(stream), err, err_len);
}

nf_status nf_plan_process_host(const nf_plan* p, const nf_const_plane* sources, int nsources, const int* targets,
                               int ntargets, nf_plane dst, int frame, int plane, void* stream, char* err,
                               size_t err_len) {
  return guarded(err, err_len, [&]() -> nf_status {
    nfb::require(p != nullptr, "null plan");
    const Checked c = validate_call(*p, sources, nsources, targets, ntargets, dst);
    (void)c;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : cudaStreamPerThread;
    const size_t elem = size_t(storage_of(p->t.format));
    const size_t pitch = ((size_t(p->t.gx.length) * elem + 255) / 256) * 256;
    const size_t plane_bytes = pitch * size_t(p->t.gy.length);
    // Unique sources are staged once; repeated slots reuse the staged copy.
    std::vector<int> slot_of(static_cast<size_t>(nsources), -1);
    std::vector<int> uniq;
    for (int j = 0; j < nsources; ++j) {
      for (int i = 0; i < j; ++i)
        if (sources[i].data == sources[j].data && sources[i].stride_bytes == sources[j].stride_bytes) {
          slot_of[size_t(j)] = slot_of[size_t(i)];
          break;
        }
      if (slot_of[size_t(j)] < 0) {
        slot_of[size_t(j)] = int(uniq.size());
        uniq.push_back(j);
      }
    }
    // Per-call device staging from the library's pool on the caller's stream (the
    // calling thread's default stream when none is given), so calls from several host
    // threads overlap their copies and kernels; a per-call error flag keeps each call's
    // non-finite report its own.
    const size_t need = plane_bytes * (uniq.size() + 1) + 256;
    void* scratch = nullptr;
    cudaError_t e = scratch_alloc(&scratch, need, st);
    if (e != cudaSuccess) return cuda_fail(err, err_len, e, "device allocation failed");
    auto* base = static_cast<unsigned char*>(scratch);
    int* err_word = reinterpret_cast<int*>(base + plane_bytes * (uniq.size() + 1));
    auto finish = [&](nf_status s) {
      cudaFreeAsync(scratch, st);
      return s;
    };
    if ((e = cudaMemsetAsync(err_word, 0, sizeof(int), st)) != cudaSuccess)
      return finish(cuda_fail(err, err_len, e, "device memset failed"));
    std::vector<nf_const_plane> dsrc(static_cast<size_t>(nsources));
    for (size_t u = 0; u < uniq.size(); ++u) {
      const auto& s = sources[uniq[u]];
      e = cudaMemcpy2DAsync(base + u * plane_bytes, pitch, s.data, size_t(s.stride_bytes), size_t(s.width) * elem,
                            size_t(s.height), cudaMemcpyHostToDevice, st);
      if (e != cudaSuccess) return finish(cuda_fail(err, err_len, e, "host to device copy failed"));
    }
    for (int j = 0; j < nsources; ++j)
      dsrc[size_t(j)] = {base + size_t(slot_of[size_t(j)]) * plane_bytes, sources[j].width, sources[j].height,
                         ptrdiff_t(pitch)};
    nf_plane ddst{base + uniq.size() * plane_bytes, dst.width, dst.height, ptrdiff_t(pitch)};
    nf_status s = process_device(*p, dsrc.data(), nsources, targets, ntargets, ddst, frame, plane, st, err, err_len,
                                 err_word);
    if (s != NF_OK) {
      cudaStreamSynchronize(st);  // no copy from the caller's host memory stays in flight
      return finish(s);
    }
    e = cudaMemcpy2DAsync(dst.data, size_t(dst.stride_bytes), ddst.data, pitch, size_t(dst.width) * elem,
                          size_t(dst.height), cudaMemcpyDeviceToHost, st);
    int flag = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, err_word, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(scratch, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(err, err_len, e, "device to host copy failed");
    if (flag) return fail(err, err_len, "non-finite sample or intermediate", NF_NON_FINITE);
    return NF_OK;
  });
}

nf_status nf_kalman_state_create(const nf_plan* p, int fp64, nf_kalman_state** out, char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(p && out, "null plan or output pointer");
    nfb::require(p->t.kalman, "not a Kalman plan");
    auto s = std::make_unique<nf_kalman_state>();
    s->plan = p;
    s->fp64 = fp64 ? 1 : 0;
    s->count = size_t(p->t.gx.count) * size_t(p->t.gy.count) * size_t(p->t.bins);
    const size_t var = s->fp64 ? sizeof(double) : sizeof(float);
    cudaError_t e;
    if ((e = cudaMalloc(&s->last, s->count * sizeof(cf))) != cudaSuccess ||
        (e = cudaMalloc(&s->covariance, s->count * var)) != cudaSuccess ||
        (e = cudaMalloc(&s->process, s->count * var)) != cudaSuccess)
      return cuda_fail(err, len, e, "device allocation failed");
    // initial_kalman (plan.cpp:293-300): L = 0, C = Q = R0.
    cudaMemset(s->last, 0, s->count * sizeof(cf));
    const int blocks = int(std::min<size_t>(4096, (s->count + 255) / 256));
    if (s->fp64) {
      fill_kernel<double><<<blocks, 256>>>(static_cast<double*>(s->covariance), s->count, double(p->t.kalman_r0));
      fill_kernel<double><<<blocks, 256>>>(static_cast<double*>(s->process), s->count, double(p->t.kalman_r0));
    } else {
      fill_kernel<float><<<blocks, 256>>>(static_cast<float*>(s->covariance), s->count, p->t.kalman_r0);
      fill_kernel<float><<<blocks, 256>>>(static_cast<float*>(s->process), s->count, p->t.kalman_r0);
    }
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return cuda_fail(err, len, e, "state initialisation failed");
    *out = s.release();
    return NF_OK;
  });
}
void nf_kalman_state_destroy(nf_kalman_state* s) { delete s; }
nf_status nf_kalman_state_copy(nf_kalman_state* dst, const nf_kalman_state* src, void* stream) {
  if (!dst || !src || dst->count != src->count || dst->fp64 != src->fp64) return NF_INVALID_ARGUMENT;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t var = src->fp64 ? sizeof(double) : sizeof(float);
  cudaError_t e = cudaMemcpyAsync(dst->last, src->last, src->count * sizeof(cf), cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dst->covariance, src->covariance, src->count * var, cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dst->process, src->process, src->count * var, cudaMemcpyDeviceToDevice, st);
  return e == cudaSuccess ? NF_OK : NF_DEVICE_ERROR;
}
nf_status nf_kalman_state_clone(const nf_kalman_state* src, nf_kalman_state** out, void* stream, char* err,
                                size_t len) {
  if (!src || !out) return fail(err, len, "null state or output pointer", NF_INVALID_ARGUMENT);
  nf_kalman_state* s = nullptr;
  nf_status st = nf_kalman_state_create(src->plan, src->fp64, &s, err, len);
  if (st != NF_OK) return st;
  if ((st = nf_kalman_state_copy(s, src, stream)) != NF_OK) {
    nf_kalman_state_destroy(s);
    return fail(err, len, "state copy failed", st);
  }
  *out = s;
  return NF_OK;
}
size_t nf_kalman_state_bytes(const nf_kalman_state* s) {
  if (!s) return 0;
  return s->count * (sizeof(cf) + 2 * (s->fp64 ? sizeof(double) : sizeof(float)));
}
nf_status nf_kalman_advance_device(const nf_plan* p, nf_const_plane source, nf_kalman_state* state, void* stream,
                                   char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(p && state, "null plan or state");
    check_kalman_source(*p, source);
    nfb::require(state->count == size_t(p->t.gx.count) * p->t.gy.count * p->t.bins, "Kalman state shape differs");
    nfb::require(!p->t.needs_pattern || p->model_ready.load(std::memory_order_acquire),
                 "Kalman sampled model not initialized");
    nfd::KalmanArgs a{state->last,
                      state->fp64 ? nullptr : static_cast<float*>(state->covariance),
                      state->fp64 ? nullptr : static_cast<float*>(state->process),
                      state->fp64 ? static_cast<double*>(state->covariance) : nullptr,
                      state->fp64 ? static_cast<double*>(state->process) : nullptr,
                      p->t.spectral.primary.empty() && !p->t.needs_pattern ? nullptr : p->dev.filt.primary,
                      state->fp64};
    const cudaError_t e = run_kalman_advance(p->dev, source.data, source.stride_bytes, a, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(err, len, e, "kernel launch failed");
    return NF_OK;
  });
}
nf_status nf_kalman_render_device(const nf_plan* p, nf_const_plane source, nf_plane dst, const nf_kalman_state* state,
                                  void* stream, char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(p && state, "null plan or state");
    check_kalman_source(*p, source);
    nfb::require(state->count == size_t(p->t.gx.count) * p->t.gy.count * p->t.bins, "Kalman checkpoint shape differs");
    nfb::require(dst.width == p->t.gx.length && dst.height == p->t.gy.length, "frame dimensions differ from plan");
    const size_t elem = size_t(storage_of(p->t.format));
    const size_t de = plane_extent(dst.width, dst.height, dst.stride_bytes, elem);
    check_pointer(dst.data, elem);
    disjoint(source.data, plane_extent(source.width, source.height, source.stride_bytes, elem), dst.data, de);
    nfd::DevPlan d = p->dev;
    d.fft3d_mode = nfd::kEnhanceOnly;  // render copies L, then enhances (plan.cpp:471-477)
    const cudaError_t e = run_spatial(d, source.data, source.stride_bytes, dst.data, dst.stride_bytes, state->last,
                                      static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(err, len, e, "kernel launch failed");
    return NF_OK;
  });
}
// Kalman step: nf_kalman_advance_device followed by nf_kalman_render_device of the same
// frame, in two launches (the advance kernel renders each run of blocks it advanced into
// a buffer of synthesised blocks, then kalman_ola_kernel adds them per pixel). The buffer
// is stream-ordered scratch of the library's pool: bh * bw floats per block.
nf_status nf_kalman_step_device(const nf_plan* p, nf_const_plane source, nf_plane dst, nf_kalman_state* state,
                                void* stream, char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(p && state, "null plan or state");
    check_kalman_source(*p, source);
    nfb::require(state->count == size_t(p->t.gx.count) * p->t.gy.count * p->t.bins, "Kalman state shape differs");
    nfb::require(!p->t.needs_pattern || p->model_ready.load(std::memory_order_acquire),
                 "Kalman sampled model not initialized");
    nfb::require(dst.width == p->t.gx.length && dst.height == p->t.gy.length, "frame dimensions differ from plan");
    const size_t elem = size_t(storage_of(p->t.format));
    const size_t de = plane_extent(dst.width, dst.height, dst.stride_bytes, elem);
    check_pointer(dst.data, elem);
    disjoint(source.data, plane_extent(source.width, source.height, source.stride_bytes, elem), dst.data, de);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t synth_bytes = size_t(p->t.gx.count) * p->t.gy.count * size_t(p->t.bh) * p->t.bw * sizeof(float);
    void* synth = nullptr;
    cudaError_t e = scratch_alloc(&synth, synth_bytes, st);
    if (e != cudaSuccess) return cuda_fail(err, len, e, "device allocation failed");
    nfd::KalmanArgs a{state->last,
                      state->fp64 ? nullptr : static_cast<float*>(state->covariance),
                      state->fp64 ? nullptr : static_cast<float*>(state->process),
                      state->fp64 ? static_cast<double*>(state->covariance) : nullptr,
                      state->fp64 ? static_cast<double*>(state->process) : nullptr,
                      p->t.spectral.primary.empty() && !p->t.needs_pattern ? nullptr : p->dev.filt.primary,
                      state->fp64,
                      static_cast<float*>(synth)};
    nfd::DevPlan d = p->dev;
    d.fft3d_mode = nfd::kEnhanceOnly;  // the render enhances the estimate (plan.cpp:471-477)
    e = run_kalman_advance(d, source.data, source.stride_bytes, a, st);
    if (e == cudaSuccess) {
      // four (two) pixels per thread when they share their covering blocks: 16 (8)-byte loads
      const int per = ((d.gx.step | d.bw | d.gx.offset) & 3) == 0 ? 4 : ((d.gx.step | d.bw | d.gx.offset) & 1) == 0 ? 2 : 1;
      const dim3 grid((unsigned((dst.width + per - 1) / per) + 255) / 256, unsigned(dst.height));
      auto* out = static_cast<unsigned char*>(dst.data);
      const long long ds = (long long)dst.stride_bytes;
      const float* sy = static_cast<const float*>(synth);
      auto ola = [&](auto storage, auto v) {
        nfd::kalman_ola_kernel<decltype(storage)::value, decltype(v)::value><<<grid, 256, 0, st>>>(d, sy, out, ds);
      };
      using U8 = std::integral_constant<int, nfd::kStoreU8>;
      using U16 = std::integral_constant<int, nfd::kStoreU16>;
      using F32 = std::integral_constant<int, nfd::kStoreF32>;
      auto by_width = [&](auto storage) {
        if (per == 4) ola(storage, std::integral_constant<int, 4>{});
        else if (per == 2) ola(storage, std::integral_constant<int, 2>{});
        else ola(storage, std::integral_constant<int, 1>{});
      };
      if (d.storage == nfd::kStoreU8) by_width(U8{});
      else if (d.storage == nfd::kStoreU16) by_width(U16{});
      else by_width(F32{});
      e = cudaGetLastError();
    }
    cudaFreeAsync(synth, st);
    if (e != cudaSuccess) return cuda_fail(err, len, e, "kernel launch failed");
    return NF_OK;
  });
}
namespace {
// Copies a host plane into the plan's staging buffer (slot `slot` of `nslots`).
nf_status stage_host_plane(const nf_plan& p, const nf_const_plane& s, int slot, int nslots, cudaStream_t st,
                           nf_const_plane* out, nf_plane* dst_out, char* err, size_t len) {
  const size_t elem = size_t(storage_of(p.t.format));
  const size_t pitch = ((size_t(p.t.gx.length) * elem + 255) / 256) * 256;
  const size_t plane_bytes = pitch * size_t(p.t.gy.length);
  const size_t need = plane_bytes * size_t(nslots);
  cudaError_t e;
  if (p.staging_bytes < need) {
    if (p.staging) cudaFree(p.staging);
    p.staging = nullptr;
    p.staging_bytes = 0;
    if ((e = cudaMalloc(&p.staging, need)) != cudaSuccess) return cuda_fail(err, len, e, "device allocation failed");
    p.staging_bytes = need;
  }
  auto* base = static_cast<unsigned char*>(p.staging) + size_t(slot) * plane_bytes;
  if (s.data) {
    e = cudaMemcpy2DAsync(base, pitch, s.data, size_t(s.stride_bytes), size_t(s.width) * elem, size_t(s.height),
                          cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail(err, len, e, "host to device copy failed");
  }
  if (out) *out = {base, s.width, s.height, ptrdiff_t(pitch)};
  if (dst_out) *dst_out = {base, s.width, s.height, ptrdiff_t(pitch)};
  return NF_OK;
}
} // namespace

nf_status nf_plan_pattern_candidate_host(const nf_plan* p, nf_const_plane source, float* power, int count,
                                         void* stream, char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(p != nullptr, "null plan");
    check_pattern_source(*p, source);
    std::lock_guard<std::mutex> lock(p->staging_mu);
    nf_const_plane staged{};
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    nf_status s = stage_host_plane(*p, source, 0, 1, st, &staged, nullptr, err, len);
    if (s != NF_OK) return s;
    return nf_plan_pattern_candidate(p, staged, power, count, stream, err, len);
  });
}

nf_status nf_plan_prepare_pattern_host(nf_plan* p, nf_const_plane source, void* stream, char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(p != nullptr, "null plan");
    nfb::require(p->t.needs_pattern, "FFT3D sampling is inactive");
    if (p->model_ready.load(std::memory_order_acquire)) return NF_OK;
    std::vector<float> v(size_t(p->t.bins));
    nf_status s = nf_plan_pattern_candidate_host(p, source, v.data(), int(v.size()), stream, err, len);
    if (s != NF_OK) return s;
    return nf_plan_set_noise_model(p, v.data(), int(v.size()), err, len);
  });
}

nf_status nf_kalman_advance_host(const nf_plan* p, nf_const_plane source, nf_kalman_state* state, void* stream,
                                 char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(p && state, "null plan or state");
    check_kalman_source(*p, source);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lock(p->staging_mu);
    nf_const_plane d{};
    nf_status s = stage_host_plane(*p, source, 0, 1, st, &d, nullptr, err, len);
    if (s != NF_OK) return s;
    s = nf_kalman_advance_device(p, d, state, stream, err, len);
    if (s != NF_OK) return s;
    return read_error_word(*p, st, err, len);
  });
}

nf_status nf_kalman_render_host(const nf_plan* p, nf_const_plane source, nf_plane dst, const nf_kalman_state* state,
                                void* stream, char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(p && state, "null plan or state");
    check_kalman_source(*p, source);
    nfb::require(dst.width == p->t.gx.length && dst.height == p->t.gy.length, "frame dimensions differ from plan");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lock(p->staging_mu);
    nf_const_plane d{};
    nf_plane o{};
    nf_status s = stage_host_plane(*p, source, 0, 2, st, &d, nullptr, err, len);
    if (s == NF_OK) s = stage_host_plane(*p, nf_const_plane{nullptr, dst.width, dst.height, dst.stride_bytes}, 1, 2, st,
                                         nullptr, &o, err, len);
    if (s != NF_OK) return s;
    s = nf_kalman_render_device(p, d, o, state, stream, err, len);
    if (s != NF_OK) return s;
    const size_t elem = size_t(storage_of(p->t.format));
    const cudaError_t e = cudaMemcpy2DAsync(dst.data, size_t(dst.stride_bytes), o.data, size_t(o.stride_bytes),
                                            size_t(dst.width) * elem, size_t(dst.height), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return cuda_fail(err, len, e, "device to host copy failed");
    return read_error_word(*p, st, err, len);
  });
}

nf_status nf_kalman_state_read(const nf_kalman_state* s, float* last, float* cov, float* proc, size_t count) {
  if (!s || count != s->count) return NF_INVALID_ARGUMENT;
  if (cudaMemcpy(last, s->last, count * sizeof(cf), cudaMemcpyDeviceToHost) != cudaSuccess) return NF_DEVICE_ERROR;
  if (!s->fp64) {
    if (cudaMemcpy(cov, s->covariance, count * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return NF_DEVICE_ERROR;
    if (cudaMemcpy(proc, s->process, count * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return NF_DEVICE_ERROR;
    return NF_OK;
  }
  std::vector<double> tmp(count);
  if (cudaMemcpy(tmp.data(), s->covariance, count * 8, cudaMemcpyDeviceToHost) != cudaSuccess) return NF_DEVICE_ERROR;
  for (size_t i = 0; i < count; ++i) cov[i] = float(tmp[i]);
  if (cudaMemcpy(tmp.data(), s->process, count * 8, cudaMemcpyDeviceToHost) != cudaSuccess) return NF_DEVICE_ERROR;
  for (size_t i = 0; i < count; ++i) proc[i] = float(tmp[i]);
  return NF_OK;
}

namespace {
// frames / plane_ids: each item's frame and plane numbers (nf_plan_process_device's `frame`
// and `plane`), or null: they seed the noise of dithered 8-bit DFTTest output, which only
// the indexed form accepts.
nf_status batch_create(const nf_batch_item* items, const int* frames, const int* plane_ids, int count, bool indexed,
                       nf_batch** out, char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(out && (count == 0 || items), "null batch output or items");
    auto b = std::make_unique<nf_batch>();
    std::vector<std::pair<size_t, int>> dithered;  // (entry, item) of dithered items
    struct Entry {
      int group, plan;
      nfd::PlaneJob job;
      int tiles_x, tiles;
      long long cost;
    };
    std::vector<Entry> entries;
    std::vector<std::vector<const nf_plan*>> group_plans;
    std::vector<std::vector<char>> group_raw;  // per group plan: filters into a dither accumulator
    for (int i = 0; i < count; ++i) {
      const nf_batch_item& it = items[i];
      nfb::require(it.plan != nullptr, "null plan in batch");
      const nf_plan& p = *it.plan;
      nfb::require(!p.t.kalman && (p.t.temporal_size == 1 || p.t.algo == nfb::Algo::FFT3D) && !p.t.temporal_ola,
                   "batch items must be single-frame plans");
      const bool dith = dithers(p.t);
      nfb::require(!dith || indexed,
                   "dithered 8-bit DFTTest output runs through nf_plan_process_device or nf_batch_create_indexed");
      nfb::require(!p.t.preview, "pshow previews run through nf_plan_process_device");
      validate_call(p, &it.source, 1, nullptr, 0, it.dst);
      nfb::require(!dith || ((!frames || frames[i] >= 0) && (!plane_ids || plane_ids[i] >= 0)),
                   "invalid dither coordinates or mode");
      if (std::find(b->plans.begin(), b->plans.end(), &p) == b->plans.end()) b->plans.push_back(&p);
      const int storage = storage_of(p.t.format), algo = p.t.algo == nfb::Algo::FFT3D ? 0 : 1;
      int gi = -1;
      for (size_t g = 0; g < b->groups.size(); ++g)
        if (b->groups[g].bh == p.t.bh && b->groups[g].bw == p.t.bw && b->groups[g].storage == storage &&
            b->groups[g].algo == algo)
          gi = int(g);
      if (gi < 0) {
        gi = int(b->groups.size());
        BatchGroup g;
        g.bh = p.t.bh;
        g.bw = p.t.bw;
        g.storage = storage;
        g.algo = algo;
        b->groups.push_back(g);
        group_plans.emplace_back();
        group_raw.emplace_back();
      }
      // a dithered item's plan enters its group a second time, keeping the raw accumulator
      auto& plans = group_plans[size_t(gi)];
      auto& raws = group_raw[size_t(gi)];
      int pi = -1;
      for (size_t j = 0; j < plans.size(); ++j)
        if (plans[j] == &p && raws[j] == char(dith)) pi = int(j);
      if (pi < 0) {
        pi = int(plans.size());
        plans.push_back(&p);
        raws.push_back(char(dith));
      }
      Entry e{gi, pi,
              {static_cast<const unsigned char*>(it.source.data), (long long)it.source.stride_bytes,
               static_cast<unsigned char*>(it.dst.data), (long long)it.dst.stride_bytes, nullptr, pi},
              0, 0, (long long)p.t.gx.count * p.t.gy.count};
      if (dith) dithered.emplace_back(entries.size(), i);
      entries.push_back(e);
    }
    cudaError_t ce;
    if (!dithered.empty()) {  // accumulator planes and dither boundary rows, 256-byte aligned
      auto up = [](size_t v) { return (v + 255) & ~size_t(255); };
      size_t bytes = 0;
      for (const auto& d : dithered) {
        const nf_plan& p = *items[d.second].plan;
        bytes += up(size_t(p.t.gx.length) * sizeof(float)) * size_t(p.t.gy.length) + up(size_t(p.t.gx.length) * sizeof(float));
      }
      if ((ce = cudaMalloc(&b->dither_mem, bytes)) != cudaSuccess) return cuda_fail(err, len, ce, "device allocation failed");
      auto* at = static_cast<unsigned char*>(b->dither_mem);
      for (const auto& d : dithered) {
        const nf_batch_item& it = items[d.second];
        const nf_plan& p = *it.plan;
        const int W = p.t.gx.length, H = p.t.gy.length;
        const size_t pitch = up(size_t(W) * sizeof(float));
        nf_batch::DitherJob j{&p, reinterpret_cast<float*>(at), pitch, reinterpret_cast<float*>(at + pitch * size_t(H)),
                              static_cast<unsigned char*>(it.dst.data), (long long)it.dst.stride_bytes, W, H,
                              frames ? frames[d.second] : 0, plane_ids ? plane_ids[d.second] : 0};
        at += pitch * size_t(H) + up(size_t(W) * sizeof(float));
        entries[d.first].job.dst = reinterpret_cast<unsigned char*>(j.acc);
        entries[d.first].job.dst_stride = (long long)pitch;
        b->dithers.push_back(j);
      }
    }
    if (!b->groups.empty() &&
        (ce = cudaMalloc(&b->counters, sizeof(int) * b->groups.size())) != cudaSuccess)
      return cuda_fail(err, len, ce, "device allocation failed");
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    // Candidate geometries: variant v gives every plan its v-th best strip width by the
    // tile-cost model (or its last one); the first launch times them (nf_batch_launch).
    constexpr int kVariants = 3;
    int nvar = 1;
    for (const auto& plans : group_plans)
      for (const nf_plan* p : plans)
        nvar = std::max(nvar, std::min(kVariants, int(strip_candidates(p->dev, 0, StripWork::Staged).size())));
    const std::vector<BatchGroup> proto = b->groups;
    for (int v = 0; v < nvar; ++v) {
      std::vector<BatchGroup> groups = proto;
      for (size_t gi = 0; gi < groups.size(); ++gi) {
        BatchGroup& g = groups[gi];
        const auto& plans = group_plans[gi];
        std::vector<nfd::DevPlan> dplans;
        std::vector<nfd::StripShape> shapes;
        for (size_t j = 0; j < plans.size(); ++j) {
          const nf_plan* p = plans[j];
          dplans.push_back(p->dev);
          if (group_raw[gi][j]) dplans.back().raw_out = 1;  // the dither pass converts
          const auto& cand = strip_candidates(p->dev, 0, StripWork::Staged);
          shapes.push_back(cand[std::min(size_t(v), cand.size() - 1)]);
        }
        std::vector<Entry> mine;
        for (auto& e : entries)
          if (e.group == int(gi)) mine.push_back(e);
        // Largest planes first: shortens the tail of the dynamic queue.
        std::stable_sort(mine.begin(), mine.end(), [](const Entry& a, const Entry& c) { return a.cost > c.cost; });
        // Tall strips (the batch already supplies parallelism), one segment height for
        // the group, chosen by the queue's schedule over the resident CTAs.
        std::vector<std::pair<const nfd::DevPlan*, int>> queue;
        for (auto& e : mine) queue.emplace_back(&plans[size_t(e.plan)]->dev, shapes[size_t(e.plan)].tw);
        const int seg_h =
            batch_segment_height(queue, g.bh, (long long)(g.bh * g.bw <= 256 ? 2 : 1) * sms, StripWork::Staged);
        for (size_t j = 0; j < plans.size(); ++j) {
          const int segs = std::max(1, (plans[j]->t.gy.length + seg_h - 1) / seg_h);
          shapes[j].th = (plans[j]->t.gy.length + segs - 1) / segs;
          g.smem = std::max(g.smem, nfd::strip_smem_bytes(g.bh, g.bw, shapes[j]));
        }
        std::vector<nfd::PlaneJob> jobs;
        std::vector<CUtensorMap> maps;
        std::vector<int> base(1, 0), tiles_x, map_of;
        for (auto& e : mine) {
          const nfd::StripShape& S = shapes[size_t(e.plan)];
          const nf_plan* p = plans[size_t(e.plan)];
          const int tx = (p->t.gx.length + S.tw - 1) / S.tw, ty = (p->t.gy.length + S.th - 1) / S.th;
          jobs.push_back(e.job);
          CUtensorMap m;
          const bool mapped = S.tma_box_w > 0 && encode_plane_map(&m, e.job.src, p->t.gx.length, p->t.gy.length,
                                                                   e.job.src_stride, g.storage,
                                                                   nfd::kStagingBoxBytes / g.storage, p->t.gy.step);
          map_of.push_back(mapped ? int(maps.size()) : -1);
          if (mapped) maps.push_back(m);
          g.mapped += mapped ? 1 : 0;
          tiles_x.push_back(tx);
          base.push_back(base.back() + tx * ty);
        }
        Blob blob;
        const size_t o_p = blob.add(dplans), o_s = blob.add(shapes), o_j = blob.add(jobs), o_b = blob.add(base),
                     o_t = blob.add(tiles_x), o_m = blob.add(maps);  // tensor maps: 256-byte aligned
        if ((ce = cudaMalloc(&g.dev, blob.bytes.size())) != cudaSuccess) {
          b->variants.push_back(groups);  // freed with the batch
          return cuda_fail(err, len, ce, "device allocation failed");
        }
        for (size_t i = 0; i < jobs.size(); ++i)  // jobs point at their maps in device memory
          if (map_of[i] >= 0) {
            jobs[i].tmap = static_cast<unsigned char*>(g.dev) + o_m + size_t(map_of[i]) * sizeof(CUtensorMap);
            std::memcpy(blob.bytes.data() + o_j + i * sizeof(nfd::PlaneJob), &jobs[i], sizeof(nfd::PlaneJob));
          }
        if ((ce = cudaMemcpy(g.dev, blob.bytes.data(), blob.bytes.size(), cudaMemcpyHostToDevice)) != cudaSuccess) {
          b->variants.push_back(groups);
          return cuda_fail(err, len, ce, "batch upload failed");
        }
        auto* base_ptr = static_cast<unsigned char*>(g.dev);
        g.work.plans = reinterpret_cast<const nfd::DevPlan*>(base_ptr + o_p);
        g.work.shapes = reinterpret_cast<const nfd::StripShape*>(base_ptr + o_s);
        g.work.jobs = reinterpret_cast<const nfd::PlaneJob*>(base_ptr + o_j);
        g.work.job_tile_base = reinterpret_cast<const int*>(base_ptr + o_b);
        g.work.job_tiles_x = reinterpret_cast<const int*>(base_ptr + o_t);
        g.work.njobs = int(jobs.size());
        g.work.counter = b->counters + gi;
        g.ctas = std::max(1, std::min(base.back(), 2 * sms));
      }
      b->variants.push_back(groups);
    }
    b->groups = b->variants.empty() ? std::vector<BatchGroup>{} : b->variants.front();
    b->tuned = b->variants.size() <= 1;
    if (b->tuned) b->chosen = 0;
    *out = b.release();
    return NF_OK;
  });
}
} // namespace

nf_status nf_batch_create(const nf_batch_item* items, int count, nf_batch** out, char* err, size_t len) {
  return batch_create(items, nullptr, nullptr, count, false, out, err, len);
}
nf_status nf_batch_create_indexed(const nf_batch_item* items, const int* frames, const int* planes, int count,
                                  nf_batch** out, char* err, size_t len) {
  return batch_create(items, frames, planes, count, true, out, err, len);
}

namespace {
cudaError_t launch_groups(nf_batch& b, const std::vector<BatchGroup>& groups, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(b.counters, 0, sizeof(int) * groups.size(), st);
  for (const auto& g : groups)
    if (e == cudaSuccess) e = launch_batch_group(g, st);
  return e;
}

// Autotuning on the first launch outside a stream capture: every candidate geometry
// writes the same outputs bit for bit, so each is launched and timed once on `st` (after
// one warm-up launch) and the fastest is kept. The host waits for these launches once.
cudaError_t tune_batch(nf_batch& b, cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(st, &cs);
  if (e != cudaSuccess || cs != cudaStreamCaptureStatusNone) return e;  // keep the modelled choice
  const size_t n = b.variants.size();
  std::vector<cudaEvent_t> ev(n + 1, nullptr);
  for (auto& x : ev)
    if (e == cudaSuccess) e = cudaEventCreate(&x);
  if (e == cudaSuccess) e = launch_groups(b, b.variants[0], st);  // warm-up
  for (size_t v = 0; v < n && e == cudaSuccess; ++v) {
    e = cudaEventRecord(ev[v], st);
    if (e == cudaSuccess) e = launch_groups(b, b.variants[v], st);
  }
  if (e == cudaSuccess) e = cudaEventRecord(ev[n], st);
  if (e == cudaSuccess) e = cudaEventSynchronize(ev[n]);
  size_t best = 0;
  float best_ms = -1.0f;
  for (size_t v = 0; v < n && e == cudaSuccess; ++v) {
    float ms = 0.0f;
    e = cudaEventElapsedTime(&ms, ev[v], ev[v + 1]);
    if (e == cudaSuccess && (best_ms < 0 || ms < best_ms)) {
      best_ms = ms;
      best = v;
    }
  }
  for (auto& x : ev)
    if (x) cudaEventDestroy(x);
  if (e == cudaSuccess) {
    b.groups = b.variants[best];
    b.tuned = true;
    b.chosen = int(best);
  }
  return e;
}
}  // namespace

nf_status nf_batch_launch(nf_batch* b, void* stream, char* err, size_t len) {
  if (!b) return fail(err, len, "null batch", NF_INVALID_ARGUMENT);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (b->groups.empty()) return NF_OK;
  if (const nf_status ms = check_models(b->plans, err, len)) return ms;
  cudaError_t e = cudaSuccess;
  if (!b->tuned && (e = tune_batch(*b, st)) != cudaSuccess) return cuda_fail(err, len, e, "batch tuning failed");
  if ((e = launch_groups(*b, b->groups, st)) != cudaSuccess) return cuda_fail(err, len, e, "kernel launch failed");
  for (const auto& d : b->dithers) {  // the dither pass of each dithered item (as process_dithered)
    nfd::dither_kernel<<<1, std::min(nfd::kDitherRows, d.height), 0, st>>>(
        d.acc, (long long)(d.pitch / sizeof(float)), d.dst, d.dst_stride, d.width, d.height, d.plan->t.dither,
        unsigned(d.plan->t.dither_seed), unsigned(d.frame), unsigned(d.plane), d.boundary, d.plan->dev.err);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(err, len, e, "kernel launch failed");
  }
  return NF_OK;
}

nf_status nf_batch_graph_launch(nf_batch* b, void* stream, char* err, size_t len) {
  if (!b) return fail(err, len, "null batch", NF_INVALID_ARGUMENT);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (const nf_status ms = check_models(b->plans, err, len)) return ms;
  cudaError_t e;
  if (!b->tuned && !b->groups.empty() && (e = tune_batch(*b, st)) != cudaSuccess)
    return cuda_fail(err, len, e, "batch tuning failed");
  if (!b->exec) {
    // Capture needs a non-legacy stream; capture on a private one and replay on `st`.
    if (!b->capture_stream && (e = cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking)) != cudaSuccess)
      return cuda_fail(err, len, e, "stream creation failed");
    if ((e = cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
      return cuda_fail(err, len, e, "graph capture failed");
    const nf_status s = nf_batch_launch(b, b->capture_stream, err, len);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(b->capture_stream, &g);
    if (s != NF_OK) {
      if (g) cudaGraphDestroy(g);
      return s;
    }
    if (e != cudaSuccess) return cuda_fail(err, len, e, "graph capture failed");
    b->graph = g;
    if ((e = cudaGraphInstantiate(&b->exec, b->graph, 0)) != cudaSuccess)
      return cuda_fail(err, len, e, "graph instantiation failed");
  }
  if ((e = cudaGraphLaunch(b->exec, st)) != cudaSuccess) return cuda_fail(err, len, e, "graph launch failed");
  return NF_OK;
}

int nf_batch_geometry_count(const nf_batch* b) { return b ? int(b->variants.size()) : 0; }
int nf_batch_geometry(const nf_batch* b) { return b ? b->chosen : -1; }
int nf_batch_mapped_planes(const nf_batch* b) {
  int n = 0;
  if (b)
    for (const auto& g : b->groups) n += g.mapped;
  return n;
}

nf_status nf_batch_select_geometry(nf_batch* b, int index, char* err, size_t len) {
  if (!b) return fail(err, len, "null batch", NF_INVALID_ARGUMENT);
  if (index < 0 || index >= int(b->variants.size()))
    return fail(err, len, "geometry index outside the batch's candidates", NF_INVALID_ARGUMENT);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->groups = b->variants[size_t(index)];
  b->chosen = index;
  b->tuned = true;
  return NF_OK;
}

void nf_batch_destroy(nf_batch* b) { delete b; }

nf_status nf_clip_batch_create(const nf_clip_item* items, int count, nf_clip_batch** out, char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(out && count > 0 && items, "null clip batch output or items");
    auto b = std::make_unique<nf_clip_batch>();
    // DFTTest temporal clips outside the two-pass slice form become per-frame calls; the
    // rest are grouped into the two passes below.
    std::vector<nf_clip_item> grouped;
    for (int i = 0; i < count; ++i) {
      const nf_clip_item& it = items[i];
      nfb::require(it.plan != nullptr && it.frames && it.dsts && it.nframes > 0, "invalid clip item");
      const nf_plan& p = *it.plan;
      const bool per_frame = p.t.algo == nfb::Algo::DFTTest && p.t.temporal_size >= 2 &&
                             !(p.t.temporal_ola && p.t.temporal_overlap == 0 && !p.t.center &&
                               p.t.temporal_size <= nfd::kMaxVolumeSlots);
      if (!per_frame) {
        grouped.push_back(it);
        continue;
      }
      nfb::require(!dithers(p.t), "dithered 8-bit DFTTest output runs through nf_plan_process_device");
      nfb::require(!p.t.preview, "pshow previews run through nf_plan_process_device");
      nfb::require(it.nframes >= p.t.temporal_size || !p.t.temporal_ola, "DFTTest clips must hold at least tbsize frames");
      const int N = it.nframes, T = p.t.temporal_size;
      const size_t elem = size_t(storage_of(p.t.format));
      for (int n = 0; n < N; ++n) {
        nf_clip_batch::FrameCall c{&p, {}, {}, it.dsts[n]};
        if (p.t.temporal_ola) {  // the covering temporal blocks (temporal_grid.hpp:5-40)
          for (const auto& blk : nfb::temporal_blocks(n, N, T, p.t.temporal_overlap)) {
            c.targets.push_back(blk.target);
            for (int z = 0; z < T; ++z) c.sources.push_back(it.frames[blk.slots[size_t(z)]]);
          }
        } else {  // slots clamp(n - T/2 + j, 0, N - 1) (filter.hpp:289-296)
          for (int j = 0; j < T; ++j) c.sources.push_back(it.frames[std::min(std::max(n - T / 2 + j, 0), N - 1)]);
        }
        validate_call(p, c.sources.data(), int(c.sources.size()), c.targets.empty() ? nullptr : c.targets.data(),
                      int(c.targets.size()), c.dst);
        const size_t de = plane_extent(c.dst.width, c.dst.height, c.dst.stride_bytes, elem);
        for (int g = 0; g < N; ++g)  // outputs are written while other outputs still read the clip
          disjoint(it.frames[g].data,
                   plane_extent(it.frames[g].width, it.frames[g].height, it.frames[g].stride_bytes, elem),
                   c.dst.data, de);
        b->calls.push_back(std::move(c));
      }
      if (std::find(b->plans.begin(), b->plans.end(), &p) == b->plans.end()) b->plans.push_back(&p);
    }
    if (grouped.empty()) {
      *out = b.release();
      return NF_OK;
    }
    items = grouped.data();
    count = int(grouped.size());
    std::vector<const nf_plan*> plans;
    std::vector<int> plan_of(static_cast<size_t>(count));
    for (int i = 0; i < count; ++i) {
      const nf_clip_item& it = items[i];
      nfb::require(it.plan != nullptr && it.frames && it.dsts && it.nframes > 0, "invalid clip item");
      const nf_plan& p = *it.plan;
      const bool fft3d = p.t.algo == nfb::Algo::FFT3D && !p.t.kalman && p.t.temporal_size >= 2 &&
                         p.t.temporal_size <= 5;
      const bool dft = p.t.algo == nfb::Algo::DFTTest && p.t.temporal_ola && p.t.temporal_overlap == 0 &&
                       !p.t.center && p.t.temporal_size >= 2 && p.t.temporal_size <= nfd::kMaxVolumeSlots;
      nfb::require(fft3d || dft, "clip batches take FFT3D plans with bt 2..5 or DFTTest plans with tbsize >= 2");
      const int storage = storage_of(p.t.format);
      if (i == 0) {
        b->bh = p.t.bh;
        b->bw = p.t.bw;
        b->storage = storage;
        b->slice = dft ? 1 : 0;
      }
      nfb::require(p.t.bh == b->bh && p.t.bw == b->bw && storage == b->storage && (dft ? 1 : 0) == b->slice,
                   "clip batch items must share algorithm, block shape and sample storage");
      nfb::require(!dft || it.nframes >= p.t.temporal_size, "DFTTest clips must hold at least tbsize frames");
      nfb::require(!dithers(p.t), "dithered 8-bit DFTTest output runs through nf_plan_process_device");
      nfb::require(!p.t.preview, "pshow previews run through nf_plan_process_device");
      const size_t elem = size_t(storage);
      for (int f = 0; f < it.nframes; ++f) {
        if (dft) {
          std::vector<nf_const_plane> block(size_t(p.t.temporal_size), it.frames[f]);
          const int target = 0;
          validate_call(p, block.data(), p.t.temporal_size, &target, 1, it.dsts[f]);
        } else {
          validate_call(p, &it.frames[f], 1, nullptr, 0, it.dsts[f]);
        }
        // outputs are written while other outputs still read the clip's frames
        const size_t de = plane_extent(it.dsts[f].width, it.dsts[f].height, it.dsts[f].stride_bytes, elem);
        for (int g = 0; g < it.nframes; ++g)
          disjoint(it.frames[g].data,
                   plane_extent(it.frames[g].width, it.frames[g].height, it.frames[g].stride_bytes, elem),
                   it.dsts[f].data, de);
      }
      int pi = -1;
      for (size_t j = 0; j < plans.size(); ++j)
        if (plans[j] == &p) pi = int(j);
      if (pi < 0) {
        pi = int(plans.size());
        plans.push_back(&p);
      }
      plan_of[size_t(i)] = pi;
    }
    const std::vector<const nf_plan*> call_plans = b->plans;  // plans of the per-frame calls
    b->plans = plans;
    for (const nf_plan* q : call_plans)
      if (std::find(b->plans.begin(), b->plans.end(), q) == b->plans.end()) b->plans.push_back(q);
    // strips of pass 2 (tall segments: the batch supplies the parallelism) and the
    // block-column chunk of pass 1
    std::vector<nfd::DevPlan> dplans;
    std::vector<nfd::StripShape> shapes;
    // Segment height of the pass-2 strips: one value for the batch, chosen so that the
    // items of one frame step (every clip's output) fill whole waves of resident CTAs;
    // each item costs its rows plus the block-row halo above it.
    int sms_ = 148;
    cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, 0);
    const long long slots = (long long)(b->bh * b->bw <= 256 ? 2 : 1) * sms_;
    std::vector<int> strips_x(plans.size());
    for (size_t j = 0; j < plans.size(); ++j) {
      const nfd::StripShape S = pick_strip(plans[j]->dev, 0, b->slice ? StripWork::Slice : StripWork::Temporal);
      strips_x[j] = (plans[j]->t.gx.length + S.tw - 1) / S.tw;
    }
    int seg_h = 256;
    long long best = -1;
    for (int h : {64, 96, 128, 160, 192, 224, 256, 320, 384, 448, 512, 640, 768, 1024}) {
      if (h < 2 * b->bh) continue;
      long long items = 0;
      for (int i = 0; i < count; ++i) {
        const int j = plan_of[size_t(i)];
        const int outputs = b->slice ? plans[size_t(j)]->t.temporal_size : 1;  // outputs per step
        items += (long long)outputs * strips_x[size_t(j)] * ((plans[size_t(j)]->t.gy.length + h - 1) / h);
      }
      const long long cost = ((items + slots - 1) / slots) * (h + b->bh);
      if (best < 0 || cost < best) {
        best = cost;
        seg_h = h;
      }
    }
    std::vector<nfd::StripShape> shapes_p;  // clip-edge pixel strips (FFT3D)
    for (const nf_plan* p : plans) {
      dplans.push_back(p->dev);
      nfd::StripShape S = pick_strip(p->dev, 0, b->slice ? StripWork::Slice : StripWork::Temporal);
      const int segs = std::max(1, (p->t.gy.length + seg_h - 1) / seg_h);
      S.th = (p->t.gy.length + segs - 1) / segs;
      shapes.push_back(S);
      b->smem2 = std::max(b->smem2, nfd::strip_smem_bytes(b->bh, b->bw, S));
      nfd::StripShape Sp = pick_strip(p->dev, 0, StripWork::Pixels);
      Sp.th = S.th;
      shapes_p.push_back(Sp);
      if (!b->slice) b->smem2p = std::max(b->smem2p, nfd::strip_smem_bytes(b->bh, b->bw, Sp));
    }
    int max_count = 1, step = plans[0]->t.gx.step;
    for (const nf_plan* p : plans) max_count = std::max(max_count, p->t.gx.count);
    for (const nf_plan* p : plans) step = std::min(step, p->t.gx.step);
    int tmax = 1;
    for (const nf_plan* p : plans) tmax = std::max(tmax, p->t.temporal_size);
    auto pass1_smem = [&](int st, int n) {
      return b->slice ? nfd::volume_spectra_smem_bytes(b->bh, b->bw, tmax, st, n)
                      : nfd::spectra_smem_bytes(b->bh, b->bw, st, n);
    };
    b->nbc = pass1_chunk(b->bh, b->bw, tmax, b->slice != 0, max_count, [&](int n) {
      size_t m = 0;  // the largest over the plans' steps (wider windows need more)
      for (const nf_plan* p : plans) m = std::max(m, pass1_smem(p->t.gx.step, n));
      return m;
    });
    b->smem1 = 0;
    for (const nf_plan* p : plans) b->smem1 = std::max(b->smem1, pass1_smem(p->t.gx.step, b->nbc));
    nfb::require(b->smem1 <= 200 * 1024, "block size too large for the spectra pass");
    // rings: FFT3D, T frame spectra per clip plane that has interior outputs; DFTTest,
    // the T filtered slice spectra of one temporal block
    std::vector<size_t> ring_off(static_cast<size_t>(count), SIZE_MAX);
    size_t ring_bytes = 0;
    for (int i = 0; i < count; ++i) {
      const nf_plan& p = *items[i].plan;
      if (!b->slice && items[i].nframes < p.t.temporal_size) continue;
      ring_off[size_t(i)] = ring_bytes;
      const size_t frame = size_t(p.t.gy.count) * p.t.bins * p.t.gx.count * sizeof(cf);
      ring_bytes += ((frame * p.t.temporal_size) + 255) & ~size_t(255);
    }
    cudaError_t ce;
    if (ring_bytes && (ce = cudaMalloc(&b->rings, ring_bytes)) != cudaSuccess)
      return cuda_fail(err, len, ce, "device allocation failed");
    auto frame_spec = [&](int i, int f) {
      const nf_plan& p = *items[i].plan;
      const size_t frame = size_t(p.t.gy.count) * p.t.bins * p.t.gx.count;
      return reinterpret_cast<cf*>(static_cast<unsigned char*>(b->rings) + ring_off[size_t(i)]) +
             size_t(f % p.t.temporal_size) * frame;
    };
    int nsteps = 0;
    for (int i = 0; i < count; ++i) {
      const int T = items[i].plan->t.temporal_size;
      nsteps = std::max(nsteps, b->slice ? (items[i].nframes + T - 1) / T : items[i].nframes + (T - 1) / 2);
    }
    // slot pointer arrays of all temporal jobs
    std::vector<const cf*> slot_ptrs;
    struct Pass2 {
      std::vector<nfd::PlaneJob> jobs;
      std::vector<size_t> tspec_index;  // SIZE_MAX for pixel jobs
      std::vector<int> base{0}, tiles_x;
    };
    std::vector<std::vector<nfd::SpectraJob>> pass1(static_cast<size_t>(nsteps));
    std::vector<std::vector<nfd::VolumeSpectraJob>> pass1v(static_cast<size_t>(nsteps));
    std::vector<std::vector<int>> pass1_base(static_cast<size_t>(nsteps), std::vector<int>(1, 0));
    std::vector<Pass2> pass2(static_cast<size_t>(nsteps)), pass2p(static_cast<size_t>(nsteps));
    for (int s = 0; s < nsteps; ++s) {
      for (int i = 0; b->slice && i < count; ++i) {
        // DFTTest: step s is temporal block s, frames T*s .. T*s+T-1 clamped to the clip
        // (temporal_grid.hpp:5-40 with tosize 0); its outputs are the frames it starts.
        const nf_clip_item& it = items[i];
        const nf_plan& p = *it.plan;
        const int T = p.t.temporal_size, start = T * s;
        if (start >= it.nframes) continue;
        const int pi = plan_of[size_t(i)];
        nfd::VolumeSpectraJob vj{};
        for (int z = 0; z < T; ++z) {
          const int f = std::min(std::max(start + z, 0), it.nframes - 1);
          vj.src[z] = static_cast<const unsigned char*>(it.frames[f].data);
          vj.src_stride[z] = it.frames[f].stride_bytes;
          vj.out[z] = frame_spec(i, z);
        }
        vj.plan = pi;
        vj.chunks_x = (p.t.gx.count + b->nbc - 1) / b->nbc;
        pass1v[size_t(s)].push_back(vj);
        pass1_base[size_t(s)].push_back(pass1_base[size_t(s)].back() + vj.chunks_x * p.t.gy.count);
        Pass2& q = pass2[size_t(s)];
        const nfd::StripShape& S = shapes[size_t(pi)];
        const int tx = (p.t.gx.length + S.tw - 1) / S.tw, ty = (p.t.gy.length + S.th - 1) / S.th;
        for (int z = 0; z < T && start + z < it.nframes; ++z) {
          const int n = start + z;
          q.jobs.push_back({nullptr, 0, static_cast<unsigned char*>(it.dsts[n].data),
                            (long long)it.dsts[n].stride_bytes, nullptr, pi, z, nullptr});
          q.tspec_index.push_back(slot_ptrs.size());
          slot_ptrs.push_back(frame_spec(i, z));
          q.tiles_x.push_back(tx);
          q.base.push_back(q.base.back() + tx * ty);
        }
      }
      for (int i = 0; !b->slice && i < count; ++i) {
        const nf_clip_item& it = items[i];
        const nf_plan& p = *it.plan;
        const int bt = p.t.temporal_size, left = bt / 2, right = (bt - 1) / 2;
        const int pi = plan_of[size_t(i)];
        if (ring_off[size_t(i)] != SIZE_MAX && s < it.nframes) {
          const int chunks = (p.t.gx.count + b->nbc - 1) / b->nbc;
          pass1[size_t(s)].push_back({static_cast<const unsigned char*>(it.frames[s].data),
                                      (long long)it.frames[s].stride_bytes, frame_spec(i, s), pi, chunks});
          pass1_base[size_t(s)].push_back(pass1_base[size_t(s)].back() + chunks * p.t.gy.count);
        }
        const int t = s - right;
        if (t < 0 || t >= it.nframes) continue;
        const bool fallback = it.nframes < bt || t < left || it.nframes - 1 - t < right;
        nfd::PlaneJob job{fallback ? static_cast<const unsigned char*>(it.frames[t].data) : nullptr,
                          (long long)it.frames[t].stride_bytes, static_cast<unsigned char*>(it.dsts[t].data),
                          (long long)it.dsts[t].stride_bytes, nullptr, pi, 0, nullptr};
        Pass2& q = fallback ? pass2p[size_t(s)] : pass2[size_t(s)];
        q.jobs.push_back(job);
        if (fallback) {
          q.tspec_index.push_back(SIZE_MAX);
        } else {
          q.tspec_index.push_back(slot_ptrs.size());
          for (int j = 0; j < bt; ++j) slot_ptrs.push_back(frame_spec(i, t - left + j));
        }
        const nfd::StripShape& S = fallback ? shapes_p[size_t(pi)] : shapes[size_t(pi)];
        const int tx = (p.t.gx.length + S.tw - 1) / S.tw, ty = (p.t.gy.length + S.th - 1) / S.th;
        q.tiles_x.push_back(tx);
        q.base.push_back(q.base.back() + tx * ty);
      }
    }
    if (!slot_ptrs.empty()) {
      if ((ce = cudaMalloc(&b->tspec, slot_ptrs.size() * sizeof(cf*))) != cudaSuccess)
        return cuda_fail(err, len, ce, "device allocation failed");
      if ((ce = cudaMemcpy(b->tspec, slot_ptrs.data(), slot_ptrs.size() * sizeof(cf*), cudaMemcpyHostToDevice)) !=
          cudaSuccess)
        return cuda_fail(err, len, ce, "clip batch upload failed");
    }
    const auto* slots_dev = static_cast<const cf* const*>(b->tspec);
    Blob blob;
    const size_t o_p = blob.add(dplans), o_s = blob.add(shapes), o_sp = blob.add(shapes_p);
    struct Offsets {
      size_t j1 = SIZE_MAX, b1 = SIZE_MAX, j2 = SIZE_MAX, b2 = SIZE_MAX, t2 = SIZE_MAX;
      size_t j2p = SIZE_MAX, b2p = SIZE_MAX, t2p = SIZE_MAX;
    };
    std::vector<Offsets> offs(static_cast<size_t>(nsteps));
    for (int s = 0; s < nsteps; ++s) {
      Offsets& o = offs[size_t(s)];
      if (!pass1[size_t(s)].empty()) {
        o.j1 = blob.add(pass1[size_t(s)]);
        o.b1 = blob.add(pass1_base[size_t(s)]);
      } else if (!pass1v[size_t(s)].empty()) {
        o.j1 = blob.add(pass1v[size_t(s)]);
        o.b1 = blob.add(pass1_base[size_t(s)]);
      }
      Pass2& q = pass2[size_t(s)];
      for (size_t j = 0; j < q.jobs.size(); ++j)
        if (q.tspec_index[j] != SIZE_MAX) q.jobs[j].tspec = slots_dev + q.tspec_index[j];
      if (!q.jobs.empty()) {
        o.j2 = blob.add(q.jobs);
        o.b2 = blob.add(q.base);
        o.t2 = blob.add(q.tiles_x);
      }
      const Pass2& qp = pass2p[size_t(s)];
      if (!qp.jobs.empty()) {
        o.j2p = blob.add(qp.jobs);
        o.b2p = blob.add(qp.base);
        o.t2p = blob.add(qp.tiles_x);
      }
    }
    if ((ce = cudaMalloc(&b->dev, blob.bytes.size())) != cudaSuccess)
      return cuda_fail(err, len, ce, "device allocation failed");
    if ((ce = cudaMemcpy(b->dev, blob.bytes.data(), blob.bytes.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
      return cuda_fail(err, len, ce, "clip batch upload failed");
    if ((ce = cudaMalloc(&b->counters, 2 * sizeof(int) * size_t(nsteps))) != cudaSuccess)
      return cuda_fail(err, len, ce, "device allocation failed");
    auto* base = static_cast<unsigned char*>(b->dev);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    const int per_sm = b->bh * b->bw <= 256 ? 2 : 1;
    b->steps.resize(size_t(nsteps));
    for (int s = 0; s < nsteps; ++s) {
      auto& st = b->steps[size_t(s)];
      const Offsets& o = offs[size_t(s)];
      if (o.j1 != SIZE_MAX && !b->slice) {
        st.w1.plans = reinterpret_cast<const nfd::DevPlan*>(base + o_p);
        st.w1.jobs = reinterpret_cast<const nfd::SpectraJob*>(base + o.j1);
        st.w1.item_base = reinterpret_cast<const int*>(base + o.b1);
        st.w1.njobs = int(pass1[size_t(s)].size());
        st.w1.nbc = b->nbc;
        st.items1 = pass1_base[size_t(s)].back();
      } else if (o.j1 != SIZE_MAX) {
        st.w1v.plans = reinterpret_cast<const nfd::DevPlan*>(base + o_p);
        st.w1v.jobs = reinterpret_cast<const nfd::VolumeSpectraJob*>(base + o.j1);
        st.w1v.item_base = reinterpret_cast<const int*>(base + o.b1);
        st.w1v.njobs = int(pass1v[size_t(s)].size());
        st.w1v.nbc = b->nbc;
        st.items1 = pass1_base[size_t(s)].back();
      }
      if (o.j2 != SIZE_MAX) {
        st.w2.plans = reinterpret_cast<const nfd::DevPlan*>(base + o_p);
        st.w2.shapes = reinterpret_cast<const nfd::StripShape*>(base + o_s);
        st.w2.jobs = reinterpret_cast<const nfd::PlaneJob*>(base + o.j2);
        st.w2.job_tile_base = reinterpret_cast<const int*>(base + o.b2);
        st.w2.job_tiles_x = reinterpret_cast<const int*>(base + o.t2);
        st.w2.njobs = int(pass2[size_t(s)].jobs.size());
        st.w2.counter = b->counters + 2 * s;
        st.tiles2 = pass2[size_t(s)].base.back();
      }
      if (o.j2p != SIZE_MAX) {
        st.w2p.plans = reinterpret_cast<const nfd::DevPlan*>(base + o_p);
        st.w2p.shapes = reinterpret_cast<const nfd::StripShape*>(base + o_sp);
        st.w2p.jobs = reinterpret_cast<const nfd::PlaneJob*>(base + o.j2p);
        st.w2p.job_tile_base = reinterpret_cast<const int*>(base + o.b2p);
        st.w2p.job_tiles_x = reinterpret_cast<const int*>(base + o.t2p);
        st.w2p.njobs = int(pass2p[size_t(s)].jobs.size());
        st.w2p.counter = b->counters + 2 * s + 1;
        st.tiles2p = pass2p[size_t(s)].base.back();
      }
    }
    b->ctas2 = per_sm * sms;
    b->ctas2p = per_sm * sms;
    *out = b.release();
    return NF_OK;
  });
}

nf_status nf_clip_batch_launch(nf_clip_batch* b, void* stream, char* err, size_t len) {
  if (!b) return fail(err, len, "null clip batch", NF_INVALID_ARGUMENT);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (const nf_status ms = check_models(b->plans, err, len)) return ms;
  for (const auto& c : b->calls) {
    const nf_status s = filter_device(*c.plan, c.plan->dev, c.sources.data(), int(c.sources.size()),
                                      c.targets.empty() ? nullptr : c.targets.data(), int(c.targets.size()), c.dst, st,
                                      err, len);
    if (s != NF_OK) return s;
  }
  if (b->steps.empty()) return NF_OK;
  cudaError_t e = cudaMemsetAsync(b->counters, 0, 2 * sizeof(int) * b->steps.size(), st);
  if (e != cudaSuccess) return cuda_fail(err, len, e, "queue reset failed");
  for (const auto& s : b->steps) {
    if (s.items1 > 0) {
      e = b->slice ? launch_volume_spectra_shape(b->bh, b->bw, b->storage, s.w1v, s.items1, b->smem1, st)
                   : launch_spectra_shape(b->bh, b->bw, b->storage, s.w1, s.items1, b->smem1, st);
      if (e != cudaSuccess) return cuda_fail(err, len, e, "kernel launch failed");
    }
    if (s.w2.njobs > 0) {
      const int ctas = std::max(1, std::min(b->ctas2, s.tiles2));
      if ((e = launch_temporal_shape(b->bh, b->bw, b->storage, b->slice, s.w2, ctas, b->smem2, st)) != cudaSuccess)
        return cuda_fail(err, len, e, "kernel launch failed");
    }
    if (s.w2p.njobs > 0) {  // clip-edge frames: single-frame pixel strips (FFT3D)
      BatchGroup g;
      g.bh = b->bh;
      g.bw = b->bw;
      g.storage = b->storage;
      g.algo = 0;
      g.ctas = std::max(1, std::min(b->ctas2p, s.tiles2p));
      g.smem = b->smem2p;
      g.work = s.w2p;
      if ((e = launch_batch_group(g, st)) != cudaSuccess) return cuda_fail(err, len, e, "kernel launch failed");
    }
  }
  return NF_OK;
}

nf_status nf_clip_batch_graph_launch(nf_clip_batch* b, void* stream, char* err, size_t len) {
  if (!b) return fail(err, len, "null clip batch", NF_INVALID_ARGUMENT);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (const nf_status ms = check_models(b->plans, err, len)) return ms;
  cudaError_t e;
  if (!b->exec) {
    if (!b->capture_stream && (e = cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking)) != cudaSuccess)
      return cuda_fail(err, len, e, "stream creation failed");
    if ((e = cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
      return cuda_fail(err, len, e, "graph capture failed");
    const nf_status s = nf_clip_batch_launch(b, b->capture_stream, err, len);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(b->capture_stream, &g);
    if (s != NF_OK) {
      if (g) cudaGraphDestroy(g);
      return s;
    }
    if (e != cudaSuccess) return cuda_fail(err, len, e, "graph capture failed");
    b->graph = g;
    if ((e = cudaGraphInstantiate(&b->exec, b->graph, 0)) != cudaSuccess)
      return cuda_fail(err, len, e, "graph instantiation failed");
  }
  if ((e = cudaGraphLaunch(b->exec, st)) != cudaSuccess) return cuda_fail(err, len, e, "graph launch failed");
  return NF_OK;
}

void nf_clip_batch_destroy(nf_clip_batch* b) { delete b; }

nf_status nf_host_batch_create(const nf_plan* const* plans, int planes, int frames_per_chunk, int depth,
                               nf_host_batch** out, char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(out && plans, "null host batch output or plans");
    nfb::require(planes > 0 && planes <= 16, "host batches take 1..16 planes per frame");
    nfb::require(frames_per_chunk > 0 && frames_per_chunk <= 256, "frames_per_chunk must be 1..256");
    nfb::require(depth >= 2 && depth <= 8, "depth must be 2..8 slots");
    auto h = std::make_unique<nf_host_batch>();
    h->chunk = frames_per_chunk;
    h->depth = depth;
    for (int p = 0; p < planes; ++p) {
      nfb::require(plans[p] != nullptr, "null plan in host batch");
      const auto& t = plans[p]->t;
      nfb::require(!t.kalman && (t.temporal_size == 1 || t.algo == nfb::Algo::FFT3D) && !t.temporal_ola,
                   "host batch planes must use single-frame plans");
      nfb::require(!dithers(t), "dithered 8-bit DFTTest output runs through nf_plan_process_device");
      const size_t elem = size_t(storage_of(t.format));
      const size_t pitch = ((size_t(t.gx.length) * elem + 255) / 256) * 256;
      h->plans.push_back(plans[p]);
      h->pitch.push_back(pitch);
      h->offset.push_back(h->frame_bytes);
      h->frame_bytes += pitch * size_t(t.gy.length);
    }
    cudaError_t e;
    const size_t total = size_t(depth) * 2 * size_t(frames_per_chunk) * h->frame_bytes;
    if ((e = cudaMalloc(&h->dev, total)) != cudaSuccess) return cuda_fail(err, len, e, "device allocation failed");
    for (cudaStream_t* s : {&h->h2d, &h->d2h})
      if ((e = cudaStreamCreateWithFlags(s, cudaStreamNonBlocking)) != cudaSuccess)
        return cuda_fail(err, len, e, "stream creation failed");
    for (cudaEvent_t* ev : {&h->start, &h->end})
      if ((e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming)) != cudaSuccess)
        return cuda_fail(err, len, e, "event creation failed");
    h->slots.resize(size_t(depth));
    for (auto& s : h->slots) {
      s.batches.assign(size_t(frames_per_chunk), nullptr);
      for (cudaEvent_t* ev : {&s.ready, &s.done, &s.free})
        if ((e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming)) != cudaSuccess)
          return cuda_fail(err, len, e, "event creation failed");
      if ((e = cudaStreamCreateWithFlags(&s.run, cudaStreamNonBlocking)) != cudaSuccess)
        return cuda_fail(err, len, e, "stream creation failed");
    }
    *out = h.release();
    return NF_OK;
  });
}

namespace {
// The batch over the first n frames of a slot, built on first use.
nf_status host_slot_batch(nf_host_batch& h, int slot, int n, nf_batch** b, char* err, size_t len) {
  nf_batch*& cached = h.slots[size_t(slot)].batches[size_t(n - 1)];
  if (!cached) {
    const int planes = int(h.plans.size());
    std::vector<nf_batch_item> items;
    for (int f = 0; f < n; ++f)
      for (int p = 0; p < planes; ++p) {
        const auto& t = h.plans[size_t(p)]->t;
        const long long stride = (long long)h.pitch[size_t(p)];
        items.push_back({h.plans[size_t(p)],
                         {h.frame_ptr(slot, f, false) + h.offset[size_t(p)], t.gx.length, t.gy.length, stride},
                         {h.frame_ptr(slot, f, true) + h.offset[size_t(p)], t.gx.length, t.gy.length, stride}});
      }
    const nf_status s = nf_batch_create(items.data(), int(items.size()), &cached, err, len);
    if (s != NF_OK) return s;
  }
  *b = cached;
  return NF_OK;
}
}  // namespace

nf_status nf_host_batch_process(nf_host_batch* h, const nf_const_plane* sources, const nf_plane* dsts, int frames,
                                void* stream, char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(h != nullptr, "null host batch");
    nfb::require(frames >= 0, "negative frame count");
    if (frames == 0) return NF_OK;
    nfb::require(sources && dsts, "null sources or destinations");
    const int planes = int(h->plans.size());
    for (int f = 0; f < frames; ++f)
      for (int p = 0; p < planes; ++p) {
        const auto& t = h->plans[size_t(p)]->t;
        const nf_const_plane& s = sources[size_t(f) * planes + p];
        const nf_plane& d = dsts[size_t(f) * planes + p];
        const size_t elem = size_t(storage_of(t.format));
        nfb::require(s.width == t.gx.length && s.height == t.gy.length && d.width == t.gx.length &&
                         d.height == t.gy.length,
                     "frame dimensions differ from plan");
        plane_extent(s.width, s.height, s.stride_bytes, elem);
        plane_extent(d.width, d.height, d.stride_bytes, elem);
        check_pointer(s.data, elem);
        check_pointer(d.data, elem);
      }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    auto ck = cuda_check;
    ck(cudaEventRecord(h->start, st), "event record failed");
    ck(cudaStreamWaitEvent(h->h2d, h->start, 0), "stream wait failed");
    const int nchunks = (frames + h->chunk - 1) / h->chunk;
    for (int c = 0; c < nchunks; ++c) {
      const int slot = c % h->depth, f0 = c * h->chunk, n = std::min(h->chunk, frames - f0);
      auto& S = h->slots[size_t(slot)];
      nf_batch* b = nullptr;
      const nf_status bs = host_slot_batch(*h, slot, n, &b, err, len);
      if (bs != NF_OK) return bs;
      ck(cudaStreamWaitEvent(h->h2d, S.free, 0), "stream wait failed");
      for (int f = 0; f < n; ++f)
        for (int p = 0; p < planes; ++p) {
          const auto& t = h->plans[size_t(p)]->t;
          const nf_const_plane& s = sources[size_t(f0 + f) * planes + p];
          ck(cudaMemcpy2DAsync(h->frame_ptr(slot, f, false) + h->offset[size_t(p)], h->pitch[size_t(p)], s.data,
                               size_t(s.stride_bytes), size_t(t.gx.length) * size_t(storage_of(t.format)),
                               size_t(t.gy.length), cudaMemcpyHostToDevice, h->h2d),
             "host to device copy failed");
        }
      ck(cudaEventRecord(S.ready, h->h2d), "event record failed");
      ck(cudaStreamWaitEvent(S.run, S.ready, 0), "stream wait failed");
      const nf_status ls = nf_batch_graph_launch(b, S.run, err, len);
      if (ls != NF_OK) return ls;
      ck(cudaEventRecord(S.done, S.run), "event record failed");
      ck(cudaStreamWaitEvent(h->d2h, S.done, 0), "stream wait failed");
      for (int f = 0; f < n; ++f)
        for (int p = 0; p < planes; ++p) {
          const auto& t = h->plans[size_t(p)]->t;
          const nf_plane& d = dsts[size_t(f0 + f) * planes + p];
          ck(cudaMemcpy2DAsync(d.data, size_t(d.stride_bytes), h->frame_ptr(slot, f, true) + h->offset[size_t(p)],
                               h->pitch[size_t(p)], size_t(t.gx.length) * size_t(storage_of(t.format)),
                               size_t(t.gy.length), cudaMemcpyDeviceToHost, h->d2h),
             "device to host copy failed");
        }
      ck(cudaEventRecord(S.free, h->d2h), "event record failed");
    }
    ck(cudaEventRecord(h->end, h->d2h), "event record failed");
    ck(cudaStreamWaitEvent(st, h->end, 0), "stream wait failed");
    return NF_OK;
  });
}

size_t nf_host_batch_device_bytes(const nf_host_batch* h) {
  return h ? size_t(h->depth) * 2 * size_t(h->chunk) * h->frame_bytes : 0;
}

void nf_host_batch_destroy(nf_host_batch* h) { delete h; }

nf_status nf_dft_noise_power(const nf_dft_config* c, const float* slices, int nlocations, float* power, int count,
                             char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(c && power, "null config or output");
    const std::vector<float> v = nfb::dft_noise_power(*c, slices, nlocations);
    nfb::require(count == int(v.size()), "noise model size mismatch");
    std::memcpy(power, v.data(), v.size() * sizeof(float));
    return NF_OK;
  });
}

nf_status nf_plan_set_noise_model(nf_plan* p, const float* power, int count, char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(p && power, "null plan or model");
    nfb::require(p->t.noise_model || p->t.needs_pattern, "plan has no sampled noise model");
    nfb::require(count == (p->t.noise_model ? p->t.temporal_size : 1) * p->t.bins, "noise model size mismatch");
    for (int i = 0; i < count; ++i) nfb::finite(power[i]);
    cudaError_t e = cudaMemcpy(const_cast<float*>(p->dev.filt.primary), power, size_t(count) * sizeof(float),
                               cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(err, len, e, "model upload failed");
    p->model_ready.store(true, std::memory_order_release);
    return NF_OK;
  });
}

nf_status nf_plan_pattern_candidate(const nf_plan* p, nf_const_plane source, float* power, int count, void* stream,
                                    char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(p && power, "null plan or output");
    nfb::require(p->t.needs_pattern, "FFT3D sampling is inactive");
    nfb::require(count == p->t.bins, "noise model size mismatch");
    std::lock_guard<std::mutex> lock(p->pattern_mu);
    std::vector<float> v;
    const nf_status s = pattern_candidate(*p, source, static_cast<cudaStream_t>(stream), v, err, len);
    if (s != NF_OK) return s;
    std::memcpy(power, v.data(), v.size() * sizeof(float));
    return NF_OK;
  });
}

nf_status nf_plan_prepare_pattern(nf_plan* p, nf_const_plane source, void* stream, char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(p != nullptr, "null plan");
    nfb::require(p->t.needs_pattern, "FFT3D sampling is inactive");
    if (p->model_ready.load(std::memory_order_acquire)) return NF_OK;
    std::vector<float> v(size_t(p->t.bins));
    nf_status s = nf_plan_pattern_candidate(p, source, v.data(), int(v.size()), stream, err, len);
    if (s != NF_OK) return s;
    return nf_plan_set_noise_model(p, v.data(), int(v.size()), err, len);
  });
}

int nf_plan_model_state(const nf_plan* p) {
  if (!p) return -1;
  const bool needs = p->t.noise_model || p->t.needs_pattern;
  return needs ? (p->model_ready.load(std::memory_order_acquire) ? 2 : 1) : 0;
}

nf_status nf_roi_make(int width, int height, int sub_w, int sub_h, int left, int top, int right, int bottom,
                      int interlaced, nf_roi* roi, char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(roi != nullptr, "null ROI output");
    nfb::require(sub_w >= 0 && sub_w < 8 && sub_h >= 0 && sub_h < 8 && left >= 0 && top >= 0 && right >= 0 &&
                     bottom >= 0,
                 "ROI margins and subsampling must be nonnegative");
    const int ax = 1 << sub_w, ay = 1 << sub_h;
    nfb::require(left % ax == 0 && right % ax == 0 && top % ay == 0 && bottom % ay == 0,
                 "selected chroma ROI margins must align to subsampling");
    const int l = left / ax, r = right / ax, t = top / ay, b = bottom / ay;
    nfb::require(l < width && r < width - l && t < height && b < height - t, "ROI must be nonempty");
    *roi = {l, t, width - l - r, height - t - b, interlaced ? 1 : 0};
    nfb::require(!interlaced || roi->height % 2 == 0, "interlaced ROI height must be even");
    return NF_OK;
  });
}

extern "C++" {
namespace {
// Packed row y of the ROI <- plane row top + roi_row(y) (ROI::row, roi.hpp:8-10).
__device__ __forceinline__ int roi_row(const nf_roi& r, int y) {
  return r.interlaced ? (y < r.height / 2 ? 2 * y : 2 * (r.height - 1 - y) + 1) : y;
}
template <class T>
__global__ void roi_copy_kernel(nf_roi r, const unsigned char* src, long long ss, unsigned char* dst, long long ds,
                                int unpack) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= r.width) return;
  const int py = r.top + roi_row(r, y);
  if (!unpack) {
    reinterpret_cast<T*>(dst + ptrdiff_t(y) * ds)[x] = reinterpret_cast<const T*>(src + ptrdiff_t(py) * ss)[r.left + x];
  } else {
    reinterpret_cast<T*>(dst + ptrdiff_t(py) * ds)[r.left + x] = reinterpret_cast<const T*>(src + ptrdiff_t(y) * ss)[x];
  }
}
nf_status roi_copy(const nf_roi* roi, const void* src, int sw, int sh, ptrdiff_t ss, void* dst, int dw, int dh,
                   ptrdiff_t ds, int elem, bool unpack, void* stream, char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(roi && src && dst, "null ROI or plane");
    nfb::require(elem == 1 || elem == 2 || elem == 4, "element size must be 1, 2 or 4 bytes");
    const nf_roi& r = *roi;
    nfb::require(r.width > 0 && r.height > 0 && r.left >= 0 && r.top >= 0 && (!r.interlaced || r.height % 2 == 0),
                 "invalid ROI");
    const int fw = unpack ? dw : sw, fh = unpack ? dh : sh, pw = unpack ? sw : dw, ph = unpack ? sh : dh;
    nfb::require(r.left + r.width <= fw && r.top + r.height <= fh, "ROI outside the plane");
    nfb::require(pw == r.width && ph == r.height, "packed plane dimensions differ from ROI");
    plane_extent(sw, sh, ss, size_t(elem));
    plane_extent(dw, dh, ds, size_t(elem));
    check_pointer(src, size_t(elem));
    check_pointer(dst, size_t(elem));
    disjoint(src, plane_extent(sw, sh, ss, size_t(elem)), dst, plane_extent(dw, dh, ds, size_t(elem)));
    const dim3 b(256), g((r.width + 255) / 256, r.height);
    auto* s = static_cast<const unsigned char*>(src);
    auto* d = static_cast<unsigned char*>(dst);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (elem == 1) roi_copy_kernel<unsigned char><<<g, b, 0, st>>>(r, s, ss, d, ds, unpack ? 1 : 0);
    else if (elem == 2) roi_copy_kernel<unsigned short><<<g, b, 0, st>>>(r, s, ss, d, ds, unpack ? 1 : 0);
    else roi_copy_kernel<float><<<g, b, 0, st>>>(r, s, ss, d, ds, unpack ? 1 : 0);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(err, len, e, "kernel launch failed");
    return NF_OK;
  });
}
} // namespace
} // extern "C++"

nf_status nf_roi_pack_device(const nf_roi* roi, nf_const_plane source, nf_plane packed, int elem, void* stream,
                             char* err, size_t len) {
  return roi_copy(roi, source.data, source.width, source.height, source.stride_bytes, packed.data, packed.width,
                  packed.height, packed.stride_bytes, elem, false, stream, err, len);
}
nf_status nf_roi_unpack_device(const nf_roi* roi, nf_const_plane packed, nf_plane dst, int elem, void* stream,
                               char* err, size_t len) {
  return roi_copy(roi, packed.data, packed.width, packed.height, packed.stride_bytes, dst.data, dst.width, dst.height,
                  dst.stride_bytes, elem, true, stream, err, len);
}

nf_status nf_plan_set_primary(nf_plan* p, const float* table, int count, void* stream, char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(p && table, "null plan or table");
    const bool fft3d = p->t.algo == nfb::Algo::FFT3D;
    nfb::require(!fft3d || p->learn,
                 "primary tables are replaceable on DFTTest plans and FFT3D bt=1 plans without Kalman or pattern");
    nfb::require(count == (fft3d ? p->t.bins : p->t.temporal_size * p->t.bins), "primary table shape mismatch");
    float* dst = fft3d ? p->learn : const_cast<float*>(p->dev.filt.primary);
    const cudaError_t e = cudaMemcpyAsync(dst, table, size_t(count) * sizeof(float), cudaMemcpyDeviceToDevice,
                                          static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(err, len, e, "table copy failed");
    // FFT3D: calls launched from now on read the per-bin table (batches built earlier
    // keep the plan's previous filter).
    if (fft3d) p->dev.filt.primary = p->learn;
    return NF_OK;
  });
}

nf_status nf_plan_get_primary(const nf_plan* p, float* table, int count, void* stream, char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(p && table, "null plan or table");
    const bool fft3d = p->t.algo == nfb::Algo::FFT3D;
    nfb::require(!fft3d || p->learn,
                 "primary tables are replaceable on DFTTest plans and FFT3D bt=1 plans without Kalman or pattern");
    nfb::require(count == (fft3d ? p->t.bins : p->t.temporal_size * p->t.bins), "primary table shape mismatch");
    const float* src = fft3d ? p->learn : p->dev.filt.primary;
    const cudaError_t e = cudaMemcpyAsync(table, src, size_t(count) * sizeof(float), cudaMemcpyDeviceToDevice,
                                          static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(err, len, e, "table copy failed");
    return NF_OK;
  });
}

namespace {
void check_adjoint_plan(const nf_plan& p) {
  const auto& t = p.t;
  nfb::require(t.algo == nfb::Algo::DFTTest && t.temporal_size == 1 && !t.center && t.format.floating &&
                   (t.spectral.type >= 0 && t.spectral.type <= 2),
               "backward requires a float DFTTest plan with tbsize=1, smode=1 and ftype 0, 1 or 2");
}
void check_fft3d_adjoint_plan(const nf_plan& p) {
  const auto& t = p.t;
  nfb::require(fft3d_learnable(t) && t.format.floating &&
                   (p.dev.fft3d_mode == nfd::kWienerFused || !t.enhancement.active()),
               "FFT3D backward requires a float plan with bt=1, no Kalman or pattern, and sharpen/dehalo fused "
               "into the Wiener gain (uniform sigma)");
}
// Cover tiles of the backward: 64-pixel-wide strips (a whole number of block steps);
// the tile height is chosen for the whole call so that the CTAs of all planes fill
// whole waves of resident CTAs (two per SM), weighing each CTA by the rows it
// transforms (tile height plus the block-height halo).
nfd::AdjointShape adjoint_shape(const nfd::DevPlan& d, int nplanes) {
  // Cover tiles: width and height by a modelled schedule. Per block row a tile runs the
  // two forward row passes (pixels and upstream gradient, 2·nb·bh rows), the column pass
  // (two forward columns and the per-bin adjoint, nb·(bw/2+1) columns, weight 3), the
  // inverse columns (weight 1.5) and the inverse rows, each in rounds of 256 threads; the
  // launch lasts about ceil(tiles / resident CTAs) tiles. Two CTAs per SM must fit.
  const int K = d.bw / 2 + 1;
  const long long slots = 2LL * 148;
  const int edge = (d.bw + d.gx.step - 1) / d.gx.step - 1;
  nfd::AdjointShape best_s{};
  double best = -1.0;
  for (int nbx = edge + 2; nbx <= 64; ++nbx) {
    nfd::AdjointShape S{};
    // tables staged per tile: DFTTest h and h*V; FFT3D its four windows and the fused
    // enhancement windows; both the template and the primary table
    S.tab_floats = (d.algo == 0 ? 2 * (d.bh + d.bw) + (d.filt.enh ? 2 * d.bins : 0) : 2 * d.bh * d.bw) +
                   (d.grid ? 2 * d.bins : 0) + d.bins;
    S.tab_floats = (S.tab_floats + 3) & ~3;
    S.tw = std::min(d.gx.cover, std::max(d.gx.step, (nbx - edge) * d.gx.step));
    S.nbx_max = (S.tw + d.bw - 1) / d.gx.step + 2;
    S.win_max = (S.nbx_max - 1) * d.gx.step + d.bw;
    int q = (S.win_max + 3) / 4;
    if (q % 2 == 0) ++q;
    S.ring_pitch = 4 * q;
    S.tiles_x = (d.gx.cover + S.tw - 1) / S.tw;
    if (nbx > edge + 2 && nfd::adjoint_smem_bytes(d.bh, d.bw, S) > size_t(110) * 1024) break;
    const int nb = (S.tw + d.bw - d.gx.step + d.gx.step - 1) / d.gx.step;
    const double per_row = double((2 * nb * d.bh + 255) / 256) + 4.5 * double((nb * K + 255) / 256) +
                           double((nb * d.bh + 255) / 256);
    const int lo = std::min(d.gy.cover, std::max(2 * d.bh, 32));
    for (int th = lo; th <= d.gy.cover; th += std::max(1, d.gy.step)) {
      const long long tiles_y = (d.gy.cover + th - 1) / th;
      const long long ctas = (long long)std::max(1, nplanes) * S.tiles_x * tiles_y;
      const double rows = double(th + d.bh) / d.gy.step + 2.0;
      const double cost = double((ctas + slots - 1) / slots) * rows * per_row;
      if (best < 0 || cost < best) {
        best = cost;
        best_s = S;
        best_s.th = th;
      }
      if (tiles_y == 1) break;
    }
    if (S.tw >= d.gx.cover) break;
  }
  best_s.tiles_y = (d.gy.cover + best_s.th - 1) / best_s.th;
  return best_s;
}
size_t align256(size_t n) { return (n + 255) & ~size_t(255); }
} // namespace

nf_status nf_dft_backward_scratch_bytes(const nf_plan* p, int nplanes, size_t* bytes) {
  if (!p || !bytes || nplanes < 0) return NF_INVALID_ARGUMENT;
  const nfd::AdjointShape S = adjoint_shape(p->dev, nplanes);
  const size_t tiles = size_t(S.tiles_x) * S.tiles_y;
  *bytes = size_t(nplanes) * align256(size_t(p->t.gx.cover) * p->t.gy.cover * 4) +
           align256(size_t(nplanes) * tiles * p->t.bins * 4);
  return NF_OK;
}

namespace {
// The backward launch shared by both algorithms (checked by the caller): the adjoint
// tiles, the fold onto the source and the ordered table-gradient reduction.
nf_status run_backward(const nf_plan* p, const nf_const_plane* sources, const nf_const_plane* outputs,
                       const nf_const_plane* grad_out, const nf_plane* grad_src, int nplanes, float* grad_primary,
                       void* scratch, size_t scratch_bytes, void* stream, char* err, size_t len) {
  nfb::require(nplanes > 0 && nplanes <= nfd::kAdjointMaxPlanes, "backward takes 1..32 planes per call");
  size_t need = 0;
  nf_dft_backward_scratch_bytes(p, nplanes, &need);
  nfb::require(scratch && scratch_bytes >= need, "backward scratch too small");
  auto check_plane = [&](const nf_const_plane& v) {
    nfb::require(v.width == p->t.gx.length && v.height == p->t.gy.length, "frame dimensions differ from plan");
    plane_extent(v.width, v.height, v.stride_bytes, 4);
    check_pointer(v.data, 4);
  };
  for (int i = 0; i < nplanes; ++i) {
    nf_plane gs = grad_src[i];
    validate_call(*p, &sources[i], 1, nullptr, 0, gs);
    check_plane(grad_out[i]);
    if (outputs) check_plane(outputs[i]);
  }
  const nfd::DevPlan& d = p->dev;
  const nfd::AdjointShape S = adjoint_shape(d, nplanes);
  const size_t tiles = size_t(S.tiles_x) * S.tiles_y;
  const size_t cov = align256(size_t(p->t.gx.cover) * p->t.gy.cover * 4), part = tiles * p->t.bins * 4;
  auto* base = static_cast<unsigned char*>(scratch);
  nfd::AdjointBatch B{};
  B.n = nplanes;
  for (int i = 0; i < nplanes; ++i) {
    B.job[i] = {static_cast<const float*>(sources[i].data), (long long)sources[i].stride_bytes,
                static_cast<const float*>(grad_out[i].data), (long long)grad_out[i].stride_bytes,
                reinterpret_cast<float*>(base + size_t(i) * cov),
                reinterpret_cast<float*>(base + size_t(nplanes) * cov + size_t(i) * part),
                outputs ? static_cast<const float*>(outputs[i].data) : nullptr,
                outputs ? (long long)outputs[i].stride_bytes : 0};
    B.gsrc[i] = static_cast<float*>(grad_src[i].data);
    B.gsrc_stride[i] = grad_src[i].stride_bytes;
  }
  const size_t smem = nfd::adjoint_smem_bytes(d.bh, d.bw, S);
  nfb::require(smem <= 227 * 1024, "block size too large for the backward tile");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = (d.bh == 16 && d.bw == 16) ? nfd::launch_adjoint_16x16(d, S, B, smem, st)
                                              : nfd::launch_adjoint_0x0(d, S, B, smem, st);
  if (e != cudaSuccess) return cuda_fail(err, len, e, "kernel launch failed");
  const dim3 fb(32, 8), fg((p->t.gx.length + 31) / 32, (p->t.gy.length + 7) / 8, nplanes);
  nfd::dft_adjoint_fold_kernel<<<fg, fb, 0, st>>>(d, B);
  // partials of all planes are contiguous: tiles*nplanes rows of `bins`
  nfd::dft_adjoint_reduce_kernel<<<(p->t.bins + 31) / 32, dim3(32, 32), 0, st>>>(
      reinterpret_cast<const float*>(base + size_t(nplanes) * cov), int(tiles) * nplanes, p->t.bins, grad_primary);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(err, len, e, "kernel launch failed");
  return NF_OK;
}
}  // namespace

nf_status nf_dft_backward_device(const nf_plan* p, const nf_const_plane* sources, const nf_const_plane* grad_out,
                                 const nf_plane* grad_src, int nplanes, float* grad_primary, void* scratch,
                                 size_t scratch_bytes, void* stream, char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(p && sources && grad_out && grad_src && grad_primary, "null argument");
    check_adjoint_plan(*p);
    return run_backward(p, sources, nullptr, grad_out, grad_src, nplanes, grad_primary, scratch, scratch_bytes,
                        stream, err, len);
  });
}

nf_status nf_fft3d_backward_device(const nf_plan* p, const nf_const_plane* sources, const nf_const_plane* outputs,
                                   const nf_const_plane* grad_out, const nf_plane* grad_src, int nplanes,
                                   float* grad_primary, void* scratch, size_t scratch_bytes, void* stream, char* err,
                                   size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(p && sources && outputs && grad_out && grad_src && grad_primary, "null argument");
    check_fft3d_adjoint_plan(*p);
    return run_backward(p, sources, outputs, grad_out, grad_src, nplanes, grad_primary, scratch, scratch_bytes,
                        stream, err, len);
  });
}

nf_status nf_kernel_info(char* fft_backend, size_t fb_len, char* target, size_t t_len, char* fft, size_t f_len,
                         int* lanes) {
  auto put = [](char* dst, size_t n, const char* s) {
    if (dst && n) {
      std::strncpy(dst, s, n - 1);
      dst[n - 1] = 0;
    }
  };
  put(fft_backend, fb_len, "cuda-sm100a");
  put(target, t_len, "sm_100a");
  put(fft, f_len, "codelet8/16/32+project-mixed-radix");
  if (lanes) *lanes = 32;
  return NF_OK;
}

} // extern "C"

namespace nfi {
PlanInfo plan_info(const nf_plan* p) {
  const auto& t = p->t;
  PlanInfo i;
  i.fft3d = t.algo == nfb::Algo::FFT3D;
  i.width = t.gx.length;
  i.height = t.gy.length;
  i.elem = storage_of(t.format);
  i.temporal_size = t.temporal_size;
  i.tmode1 = t.temporal_ola;
  i.temporal_overlap = t.temporal_overlap;
  i.kalman = t.kalman;
  i.preview = t.preview;
  i.single = !t.kalman && !t.preview && !dithers(t) && (t.temporal_size == 1 || i.fft3d) && !t.temporal_ola;
  i.clip = !t.preview && !dithers(t) &&
           ((i.fft3d && !t.kalman && t.temporal_size >= 2 && t.temporal_size <= 5) ||
            (!i.fft3d && t.temporal_ola && t.temporal_overlap == 0 && !t.center && t.temporal_size >= 2 &&
             t.temporal_size <= nfd::kMaxVolumeSlots));
  i.pframe = t.pframe;
  i.kalman_warmup = t.kalman_warmup;
  i.device = p->device;
  return i;
}
nf_status check_backward_call(const nf_plan* p, int nplanes, char* err, size_t len) {
  return guarded(err, len, [&]() -> nf_status {
    nfb::require(p, "null plan");
    check_adjoint_plan(*p);
    nfb::require(nplanes > 0 && nplanes <= nfd::kAdjointMaxPlanes, "backward takes 1..32 planes per call");
    return NF_OK;
  });
}
}  // namespace nfi
