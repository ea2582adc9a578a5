/* neo_fft_b200 — C ABI of the B200 (sm_100a) per-plane spectral pipeline.
 *
 * This header is the drop-in boundary for neo-fft's core `Plan`
 * (src/algorithms/plan.hpp:49-140 in the reference). Everything below is plain C:
 * pointers, sizes and status codes, no C++ or CUDA types. A C++ facade with the
 * reference's class signature (include/neo_fft_b200/plan.hpp) is built on it.
 *
 * Memory: plane pointers passed to the *_device entry points are CUDA device
 * pointers; the *_host entry points take host memory and stage it through the
 * plan's device buffers. `stream` is a cudaStream_t passed as void* (NULL = the
 * legacy default stream).
 *
 * Errors: every call returns nf_status and, when `err` is non-NULL, writes a
 * NUL-terminated message of at most err_len bytes. NF_INVALID_ARGUMENT mirrors the
 * reference's std::invalid_argument (src/base/checked.hpp:13-20) with the same
 * message texts; NF_NON_FINITE mirrors std::runtime_error("non-finite sample or
 * intermediate") (checked.hpp:37-41). On any error the destination contents are
 * unspecified; no Kalman state or model is published by a failed call.
 */
#ifndef NEO_FFT_B200_H
#define NEO_FFT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NF_ABI_VERSION 1

typedef enum nf_status {
  NF_OK = 0,
  NF_INVALID_ARGUMENT = 1, /* configuration, geometry, shape or aliasing error */
  NF_NON_FINITE = 2,       /* non-finite sample or intermediate */
  NF_DEVICE_ERROR = 3      /* CUDA launch/allocation failure or device unavailable */
} nf_status;

/* SampleFormat (plan.hpp:20-23): integer bits 8..16, or floating with bits 32. */
typedef struct nf_format {
  int bits;
  int floating;
  int chroma;
} nf_format;

/* FFT3DConfig (plan.hpp:24-36) with EnhancementConfig (fft3d_profile.hpp:6-9).
 * Optional sigma2..4 are "unset" when the has_* flag is 0. */
typedef struct nf_fft3d_config {
  int bw, bh, ow, oh, wintype, opt, bt;
  float sigma, beta, degrid, kratio;
  int has_sigma2, has_sigma3, has_sigma4;
  float sigma2, sigma3, sigma4;
  float sharpen, scutoff, svr, smin, smax, dehalo, hr, ht;
  float pfactor, pcutoff;
  int pframe, px, py, pshow;
  int left, top, right, bottom, interlaced;
  int cache_frames, cache_mb, kalman_warmup;
} nf_fft3d_config;

/* DFTConfig (plan.hpp:37-46) with DFTCurves (profile.hpp:7-12). Curves are
 * frequency/value pairs; NULL/0 means empty. nlocation holds (frame, plane, y, x)
 * tuples (dft_noise.hpp:10). */
typedef struct nf_dft_config {
  int block, overlap, mode, swin, twin, ftype, opt, tbsize;
  float sbeta, tbeta, sigma, sigma2, pmin, pmax, f0beta;
  int zmean, temporal_mode, temporal_overlap, dither, dither_seed;
  const float* slocation; int n_slocation;
  const float* ssx; int n_ssx;
  const float* ssy; int n_ssy;
  const float* sst; int n_sst;
  int ssystem;
  const int* nlocation; int n_nlocation;
  int has_alpha; float alpha;
} nf_dft_config;

/* Axis (src/spectral/geometry.hpp:6-8). */
typedef struct nf_axis {
  int length, block, overlap, step, count, cover, offset;
} nf_axis;

/* span2d::Plane equivalent: signed byte stride (bottom-up planes allowed). */
typedef struct nf_const_plane {
  const void* data;
  int width, height;
  ptrdiff_t stride_bytes;
} nf_const_plane;
typedef struct nf_plane {
  void* data;
  int width, height;
  ptrdiff_t stride_bytes;
} nf_plane;

typedef struct nf_plan nf_plan;
typedef struct nf_kalman_state nf_kalman_state;

/* Defaults of FFT3DConfig{} / DFTConfig{} (plan.hpp:24-46). */
void nf_fft3d_config_default(nf_fft3d_config* c);
void nf_dft_config_default(nf_dft_config* c);

/* Plan(int w, int h, SampleFormat, const FFT3DConfig&) — plan.hpp:51, plan.cpp:91-169. */
nf_status nf_plan_create_fft3d(int width, int height, nf_format format, const nf_fft3d_config* config,
                               nf_plan** plan, char* err, size_t err_len);
/* Plan(int w, int h, SampleFormat, const DFTConfig&) — plan.hpp:52, plan.cpp:170-226. */
nf_status nf_plan_create_dft(int width, int height, nf_format format, const nf_dft_config* config,
                             nf_plan** plan, char* err, size_t err_len);
void nf_plan_destroy(nf_plan* plan);

/* Public members geometry/temporal_size/fft.bins() (plan.hpp:53-57; read by
 * filter.hpp:97-98). `bins` is the spatial half-spectrum bin count. */
nf_status nf_plan_geometry(const nf_plan* plan, nf_axis* x, nf_axis* y, int* temporal_size, int* bins);

/* Plan::process_at<T>(sources, dst, frame, plane, targets) — plan.hpp:77-80, run()
 * plan.cpp:331-640. `sources` holds nsources logical temporal slots (they may alias
 * each other, never dst). For DFTTest tmode=1, sources holds ntargets blocks of
 * tbsize slots and targets the slice of each block (temporal_grid.hpp:24-40).
 * Device pointers; asynchronous on `stream`. The non-finite check of this call is
 * accumulated on the plan and reported by nf_plan_sync_status. */
nf_status nf_plan_process_device(const nf_plan* plan, const nf_const_plane* sources, int nsources,
                                 const int* targets, int ntargets, nf_plane dst, int frame, int plane,
                                 void* stream, char* err, size_t err_len);
/* Same as above with host planes: copies in, launches, copies out and synchronises;
 * returns NF_NON_FINITE like the reference's frame evaluation, for this call's planes
 * only. A null stream means the calling thread's default stream, so host threads that
 * each filter their own frames (the host layer's frame threads) overlap on the GPU.
 * Page-locked host planes let the copies run asynchronously. */
nf_status nf_plan_process_host(const nf_plan* plan, const nf_const_plane* sources, int nsources,
                               const int* targets, int ntargets, nf_plane dst, int frame, int plane,
                               void* stream, char* err, size_t err_len);
/* Several planes of one single-frame plan (FFT3D bt=1, DFTTest tbsize=1) in one launch,
 * for callers that hold many small planes at once (patch batches). Same results as one
 * nf_plan_process_device call per plane; at most 32 planes per call. The reference has
 * no counterpart: its host calls Plan::process_at once per plane (filter.hpp:349-360). */
nf_status nf_plan_process_planes_device(const nf_plan* plan, const nf_const_plane* sources, const nf_plane* dsts,
                                        int nplanes, void* stream, char* err, size_t err_len);
/* Synchronises `stream` and returns NF_NON_FINITE if any launch since the last call
 * met a non-finite sample or intermediate (then clears the flag). */
nf_status nf_plan_sync_status(const nf_plan* plan, void* stream, char* err, size_t err_len);

/* Kalman (bt=0): initial_kalman / advance_kalman / render_kalman — plan.hpp:84-88,
 * plan.cpp:293-321, kernels/scalar/kalman.cpp:3-24. The state (complex L, float C,
 * float Q per bin; kernels/kalman.hpp:5-14) lives in device memory. `fp64_variance`
 * = 1 keeps C and Q in binary64 (state then holds 24 bytes per bin). */
nf_status nf_kalman_state_create(const nf_plan* plan, int fp64_variance, nf_kalman_state** state, char* err,
                                 size_t err_len);
void nf_kalman_state_destroy(nf_kalman_state* state);
nf_status nf_kalman_state_copy(nf_kalman_state* dst, const nf_kalman_state* src, void* stream);
/* A new state of the same plan and variance precision holding a copy of `src`
 * (KalmanState's copy constructor, kernels/kalman.hpp:5-14; checkpoints copy states,
 * filter.hpp:171). */
nf_status nf_kalman_state_clone(const nf_kalman_state* src, nf_kalman_state** out, void* stream, char* err,
                                size_t err_len);
/* Device bytes held by a state (KalmanState::bytes, used by the checkpoint budget,
 * runtime/checkpoints.hpp:10-16). */
size_t nf_kalman_state_bytes(const nf_kalman_state* state);
nf_status nf_kalman_advance_device(const nf_plan* plan, nf_const_plane source, nf_kalman_state* state, void* stream,
                                   char* err, size_t err_len);
nf_status nf_kalman_render_device(const nf_plan* plan, nf_const_plane source, nf_plane dst,
                                  const nf_kalman_state* state, void* stream, char* err, size_t err_len);
/* Kalman step: advance_kalman(source, state) then render_kalman(source, dst, state) of
 * the same frame (the sequence filter.hpp:198 and :225 run for each output frame), in one
 * pass over the blocks: each block is transformed forward once and back once and its
 * state read and written once. Results and error reporting equal the two calls above.
 * Takes stream-ordered scratch of bh*bw floats per block from the library's pool. */
nf_status nf_kalman_step_device(const nf_plan* plan, nf_const_plane source, nf_plane dst, nf_kalman_state* state,
                                void* stream, char* err, size_t err_len);
/* Host-memory variants: the plane is staged through the plan's device buffers and
 * the call synchronises `stream` (NF_NON_FINITE like the reference). */
nf_status nf_kalman_advance_host(const nf_plan* plan, nf_const_plane source, nf_kalman_state* state, void* stream,
                                 char* err, size_t err_len);
nf_status nf_kalman_render_host(const nf_plan* plan, nf_const_plane source, nf_plane dst,
                                const nf_kalman_state* state, void* stream, char* err, size_t err_len);
/* Read back the state (host arrays of `count` bins; C/Q as float). */
nf_status nf_kalman_state_read(const nf_kalman_state* state, float* last_interleaved, float* covariance,
                               float* process, size_t count);

/* Batched / persistent form (no reference counterpart: the reference filters one
 * plane per call, plan.cpp:331). A batch holds many single-frame planes (FFT3D
 * bt=1/-1 and DFTTest tbsize=1 plans) of possibly different sizes and plans —
 * luma and chroma, clips of mixed resolutions — and filters them with one
 * persistent launch per block shape, driven by a device work queue. Planes are
 * device memory and must stay valid while the batch is in use. Results are
 * identical to nf_plan_process_device on each plane. Non-finite values are
 * reported through each plan's nf_plan_sync_status. */
typedef struct nf_batch nf_batch;
typedef struct nf_batch_item {
  const nf_plan* plan;
  nf_const_plane source;
  nf_plane dst;
} nf_batch_item;
nf_status nf_batch_create(const nf_batch_item* items, int count, nf_batch** batch, char* err, size_t err_len);
/* The same with each item's frame and plane numbers (the `frame` and `plane` arguments of
 * nf_plan_process_device; NULL arrays mean 0). They seed the noise of dithered 8-bit DFTTest
 * output (dither.cpp:4-41, plan.cpp:617-623), so this form also takes dithered items: the
 * batch filters them into a float accumulator of its own and runs the dither pass per item,
 * with outputs equal to nf_plan_process_device(..., frame, plane, ...). */
nf_status nf_batch_create_indexed(const nf_batch_item* items, const int* frames, const int* planes, int count,
                                  nf_batch** batch, char* err, size_t err_len);
/* Enqueues the batch on `stream`: no allocation. The first call outside a stream
 * capture also tunes the strip geometry: it launches each of up to three candidate
 * geometries once (after a warm-up launch; all write the same outputs) and waits for
 * them, keeping the fastest. Later calls do not synchronise and may be captured in a
 * CUDA graph; a first call inside a capture keeps the modelled geometry. */
nf_status nf_batch_launch(nf_batch* batch, void* stream, char* err, size_t err_len);
/* Captures nf_batch_launch into a CUDA graph on first use, then replays the graph. */
nf_status nf_batch_graph_launch(nf_batch* batch, void* stream, char* err, size_t err_len);
/* Candidate strip geometries the batch holds (1..3; 0 = the tile-cost model's choice), the
 * one in use (-1 until the first launch has tuned), and a fixed choice: selecting one skips
 * the tuning and drops a captured graph. Every candidate writes the same outputs. */
int nf_batch_geometry_count(const nf_batch* batch);
int nf_batch_geometry(const nf_batch* batch);
nf_status nf_batch_select_geometry(nf_batch* batch, int index, char* err, size_t err_len);
/* Planes of the geometry in use whose interior block rows are staged by bulk-tensor
 * copies prefetched one block row ahead (a 2-D tensor map per plane; planes whose base
 * address or row stride is not a multiple of 16 bytes, or whose strips are wider than a
 * tensor-map box, are staged by direct loads). A copy that does not arrive within about
 * a second is reported by nf_batch_sync_status / nf_plan_sync_status as NF_DEVICE_ERROR
 * "a source staging copy did not complete"; the outputs are still written. */
int nf_batch_mapped_planes(const nf_batch* batch);
void nf_batch_destroy(nf_batch* batch);

/* Temporal clips in batched form: every output frame of every clip, with the host
 * layer's frame selection, equal bit for bit to one nf_plan_process_device call per
 * output frame. No reference counterpart: the reference filters one frame per call.
 *  - FFT3D bt 2..5: frame n from frames n-bt/2 .. n+(bt-1)/2, or from frame n alone
 *    where that window leaves the clip (filter.hpp:407-421). Each frame's spatial
 *    spectra are computed once into a device ring of bt frame spectra per clip plane
 *    (the reference caches them in SpectraCache, plan.cpp:437-447).
 *  - DFTTest tmode 1 with tosize 0 and smode 1 (clips of at least tbsize frames): the
 *    temporal blocks of temporal_grid.hpp:5-40 each serve tbsize output frames, so each
 *    block's volume is transformed and filtered once for all of them.
 *  - Other DFTTest temporal plans (tmode 0 with the clamped centred window of
 *    filter.hpp:289-296; tmode 1 with tosize > 0, whose outputs add their covering
 *    temporal blocks; smode 0): one filter call per output frame inside the batch's
 *    launch and graph, since their frames share no transform between outputs.
 * The grouped items (the first two kinds) must share the algorithm, block shape and sample
 * storage; planes must stay allocated while the batch is used, and outputs must not
 * overlap any frame of their clip. */
typedef struct nf_clip_batch nf_clip_batch;
typedef struct nf_clip_item {
  const nf_plan* plan;
  const nf_const_plane* frames; /* nframes source planes (device memory) */
  const nf_plane* dsts;         /* nframes output planes (device memory) */
  int nframes;
} nf_clip_item;
nf_status nf_clip_batch_create(const nf_clip_item* items, int count, nf_clip_batch** batch, char* err,
                               size_t err_len);
/* Enqueues all frame steps on `stream` (no allocation or synchronisation). */
nf_status nf_clip_batch_launch(nf_clip_batch* batch, void* stream, char* err, size_t err_len);
/* Captures nf_clip_batch_launch into a CUDA graph on first use, then replays it. */
nf_status nf_clip_batch_graph_launch(nf_clip_batch* batch, void* stream, char* err, size_t err_len);
void nf_clip_batch_destroy(nf_clip_batch* batch);

/* Streamed host form (the reference host layer filters frames concurrently on its
 * frame threads, src/plugin/descriptors.hpp:58; its Plan::process call itself takes
 * host planes, plan.hpp:58-75). Frames of single-frame planes in HOST memory pass
 * through a ring of `depth` device slots of `frames_per_chunk` frames each: the
 * host->device copies, the device->host copies and each slot's batched launch run on
 * their own streams, ordered by per-slot events, so the copies hide behind the
 * filtering and the next chunk's launch fills the SMs that the tail of the current
 * one leaves idle. plans[p] filters plane p of every
 * frame (the same plan may serve several planes). Overlap needs page-locked host
 * buffers; pageable ones give the same results without it. Results equal
 * nf_plan_process_host on every plane; non-finite values are reported through each plan's
 * nf_plan_sync_status. One nf_host_batch serves one caller at a time. */
typedef struct nf_host_batch nf_host_batch;
nf_status nf_host_batch_create(const nf_plan* const* plans, int planes, int frames_per_chunk, int depth,
                               nf_host_batch** batch, char* err, size_t err_len);
/* sources[f * planes + p] and dsts[f * planes + p] are host planes of frame f. The
 * copies start after the work queued on `stream` before the call, and `stream` waits
 * for the last copy back: the outputs are complete once `stream` is synchronised. A
 * source may be its own destination. */
nf_status nf_host_batch_process(nf_host_batch* batch, const nf_const_plane* sources, const nf_plane* dsts,
                                int frames, void* stream, char* err, size_t err_len);
/* Device bytes held by the slot ring (inputs and outputs of depth x frames_per_chunk frames). */
size_t nf_host_batch_device_bytes(const nf_host_batch* batch);
void nf_host_batch_destroy(nf_host_batch* batch);

/* Host request layer (the reference host layer's request/process pair over its frame
 * server, src/plugin/filter.hpp:253-528): output frames of a clip of `num_frames`
 * frames with `planes` planes each, filtered in ranges of about `range_frames`
 * consecutive output frames per batched launch, with the host layer's frame selection.
 * FFT3D bt 2..5 and DFTTest tmode 1 with tosize 0 run the clip form (each source
 * frame's spectra computed once per range: the device ring in place of SpectraCache);
 * single-frame plans run the batched form; other DFTTest temporal modes and pshow
 * previews run one nf_plan_process_device call per frame over device-resident
 * sources. Three banks of device buffers hold consecutive ranges: the next two
 * ranges are fetched and computed while the current one is read out. plans[p] NULL
 * copies plane p from the source frame (a plane that is not processed). FFT3D bt=0
 * (Kalman) plans follow the host layer's random-access rule (filter.hpp:152-250): frame
 * 0 passes through, frame n continues the latest of up to four device-resident state
 * snapshots not older than n - kalman_warmup - 1 (or the initial state), renders n and
 * publishes its state (64 MiB budget, one snapshot always kept); request(n) then lists
 * the frames a cold request reads. FFT3D sampled noise models (pfactor) are prepared from
 * the pattern frame on first use; DFTTest sampled models (nlocation) must be
 * published before the first request. Calls are serialised internally. */
typedef struct nf_frame_server nf_frame_server;
/* Returns the view of plane `plane` of source frame `frame` (host or device memory)
 * in *view; 0 on success. The view must stay valid until the call that asked for it
 * returns. */
typedef int (*nf_frame_source)(void* user, int frame, int plane, nf_const_plane* view);
nf_status nf_frame_server_create(const nf_plan* const* plans, int planes, int num_frames, int range_frames,
                                 nf_frame_source source, void* user, nf_frame_server** server, char* err,
                                 size_t err_len);
/* Filter::request: the source frames output frame n reads, ascending and unique
 * (*count of them; at most `capacity` written). */
nf_status nf_frame_server_request(const nf_frame_server* server, int n, int* frames, int capacity, int* count,
                                  char* err, size_t err_len);
/* Filter::process: output frame n into dsts[planes] (host or device memory); returns
 * once the planes are written. */
nf_status nf_frame_server_get(nf_frame_server* server, int n, const nf_plane* dsts, char* err, size_t err_len);
/* Output frames computed so far and source frames fetched so far (for hosts that
 * size their caches). */
void nf_frame_server_counters(const nf_frame_server* server, long long* computed, long long* fetched);
void nf_frame_server_destroy(nf_frame_server* server);

/* Sampled noise models (the published table is the plan's per-bin primary table:
 * tbsize*bins floats for DFTTest, bins for FFT3D). DFTTest with nlocation (ftype 0/1): DFTNoise
 * (src/algorithms/dft_noise.cpp:5-41) builds the per-bin primary table from windowed
 * 3-D power spectra of sample volumes the host layer gathers (filter.hpp:476-490):
 * `slices` holds nlocations x tbsize x sbsize x sbsize floats in 8-bit amplitude units.
 * nf_dft_noise_power computes the table (tbsize * bins floats) on the host, as the
 * reference does once per filter; nf_plan_set_noise_model publishes it to a plan (every
 * plan of the filter shares one model). Processing before publication fails with the
 * reference's "DFTTest sample model not initialized".
 * nf_plan_model_state: 0 = plan has no sampled model, 1 = waiting for it, 2 = ready. */
nf_status nf_dft_noise_power(const nf_dft_config* config, const float* slices, int nlocations, float* power,
                             int count, char* err, size_t err_len);
nf_status nf_plan_set_noise_model(nf_plan* plan, const float* power, int count, char* err, size_t err_len);
int nf_plan_model_state(const nf_plan* plan);
/* FFT3D with pfactor > 0: the pattern search of plan.cpp:227-288 on a device plane of
 * the pattern frame (filter.hpp:175-194, 455-471). nf_plan_pattern_candidate scores
 * every candidate block (the px/py block, or all blocks two or more inside the grid),
 * takes the first minimum and returns its power scaled by pfactor (1 for Kalman) and
 * the sampling weights (`count` = bins floats, host memory; synchronises `stream`);
 * publish it with nf_plan_set_noise_model (pattern_candidate + publish_pattern,
 * plan.hpp:93-94). nf_plan_prepare_pattern does both unless a model is already
 * published (prepare_pattern, plan.hpp:95-97). Processing before publication fails
 * with "FFT3D sampled model not initialized". With pshow, nf_plan_process_device
 * renders the chosen block of the first source on a zero plane instead of filtering. */
nf_status nf_plan_pattern_candidate(const nf_plan* plan, nf_const_plane source, float* power, int count, void* stream,
                                    char* err, size_t err_len);
nf_status nf_plan_prepare_pattern(nf_plan* plan, nf_const_plane source, void* stream, char* err, size_t err_len);
/* The same with the source plane in host memory (staged through the plan). */
nf_status nf_plan_pattern_candidate_host(const nf_plan* plan, nf_const_plane source, float* power, int count,
                                         void* stream, char* err, size_t err_len);
nf_status nf_plan_prepare_pattern_host(nf_plan* plan, nf_const_plane source, void* stream, char* err,
                                       size_t err_len);

/* Region of interest and interlaced packing (src/plugin/roi.hpp:6-40). The host layer
 * filters the ROI of a plane as its own image; with `interlaced`, the packed image holds
 * the top field's rows in order followed by the bottom field's rows in reverse order, so
 * reflection at the packed image's edges stays within one field. nf_roi_make validates
 * the margins like make_roi (chroma margins must align to the subsampling, the ROI must be
 * nonempty, interlaced heights even); nf_roi_pack_device / nf_roi_unpack_device copy
 * between a full device plane and its packed image (elem_bytes 1, 2 or 4). */
typedef struct nf_roi {
  int left, top, width, height, interlaced;
} nf_roi;
nf_status nf_roi_make(int width, int height, int sub_w, int sub_h, int left, int top, int right, int bottom,
                      int interlaced, nf_roi* roi, char* err, size_t err_len);
nf_status nf_roi_pack_device(const nf_roi* roi, nf_const_plane source, nf_plane packed, int elem_bytes, void* stream,
                             char* err, size_t err_len);
nf_status nf_roi_unpack_device(const nf_roi* roi, nf_const_plane packed, nf_plane dst, int elem_bytes, void* stream,
                               char* err, size_t err_len);

/* Differentiable form (no reference counterpart; the reference has no gradients).
 * DFTTest plans keep their per-bin primary table A ([tbsize][sbsize][sbsize/2+1],
 * already calibrated: the threshold the Wiener gain compares with) in device memory.
 * nf_plan_set_primary replaces it from device memory on `stream`, so a training loop
 * can learn it; a plan without sigma curves starts from its uniform value, which
 * nf_plan_get_primary copies out. FFT3D plans with bt=1 (no Kalman, no sampled pattern,
 * no preview) keep a per-bin noise table a ([bh][bw/2+1]: sigma^2/norm when sigma is
 * uniform, else the sigma profile) the same way; once replaced, per-call launches
 * filter with it (batches built earlier keep the previous filter). Replacing the table
 * changes the plan: calls on other streams that use the plan must be ordered with the
 * replacement. */
nf_status nf_plan_set_primary(nf_plan* plan, const float* table_device, int count, void* stream, char* err,
                              size_t err_len);
nf_status nf_plan_get_primary(const nf_plan* plan, float* table_device, int count, void* stream, char* err,
                              size_t err_len);
/* Backward of nf_plan_process_device for float DFTTest plans (tbsize=1, smode=1,
 * ftype 0, 1 or 2): given the forward inputs and the gradient of the outputs,
 * writes the gradient of the inputs and the summed gradient of the primary table
 * over all planes. Forward spectra are recomputed, not stored. `scratch` is caller-
 * provided device memory of nf_dft_backward_scratch_bytes bytes. Sums run in a fixed
 * order, so gradients are deterministic. At most 32 planes per call. */
nf_status nf_dft_backward_scratch_bytes(const nf_plan* plan, int nplanes, size_t* bytes);
nf_status nf_dft_backward_device(const nf_plan* plan, const nf_const_plane* sources, const nf_const_plane* grad_out,
                                 const nf_plane* grad_sources, int nplanes, float* grad_primary, void* scratch,
                                 size_t scratch_bytes, void* stream, char* err, size_t err_len);

/* Backward of nf_plan_process_device for float FFT3D plans with bt=1 (no Kalman, no
 * sampled pattern, no preview) whose sharpen/dehalo factors are fused into the Wiener
 * gain (uniform sigma, or no enhancement): gradients of sum(grad_out * output) for the
 * source pixels and the per-bin noise table a of the gain max((q - a)/q, floor)
 * (kernels/scalar/spectral.cpp:18-22; enhancement fft3d_profile.cpp:69-81). The noise
 * table is read and replaced with nf_plan_get_primary/nf_plan_set_primary (bins values).
 * `outputs` are the forward outputs (the float output is clamped to [0, 1], and the
 * gradient passes only where it lies strictly inside). Scratch as nf_dft_backward_device
 * (nf_dft_backward_scratch_bytes bytes); at most 32 planes per call. No counterpart in
 * the reference (it has no gradients). */
nf_status nf_fft3d_backward_device(const nf_plan* plan, const nf_const_plane* sources, const nf_const_plane* outputs,
                                   const nf_const_plane* grad_out, const nf_plane* grad_sources, int nplanes,
                                   float* grad_primary, void* scratch, size_t scratch_bytes, void* stream, char* err,
                                   size_t err_len);

/* Allocation-free backward: nf_dft_backward_device with its scratch in a fixed
 * 16 MiB device buffer inside the library (one per device) instead of a caller
 * buffer. No counterpart in the reference (it has no gradients). For hosts that
 * must not allocate device memory per call: a plain C host has no caching
 * allocator to borrow from, and cudaMalloc/cudaFree synchronise the device, which
 * stalls every other stream such a host keeps busy. Calls whose scratch need
 * (nf_dft_backward_scratch_bytes) exceeds nf_dft_backward_static_capacity() fail
 * with NF_INVALID_ARGUMENT, and so do calls made while a device other than the
 * plan's is current (the buffer is per device). The first call on each device looks the buffer's
 * address up (cudaGetSymbolAddress) and should come before any stream capture;
 * later calls only launch kernels. The buffer is shared: calls that overlap in
 * time (other threads or unordered streams) race on it and must be serialised. */
size_t nf_dft_backward_static_capacity(void);
nf_status nf_dft_backward_device_static(const nf_plan* plan, const nf_const_plane* sources,
                                        const nf_const_plane* grad_out, const nf_plane* grad_sources, int nplanes,
                                        float* grad_primary, void* stream, char* err, size_t err_len);

/* KernelInfo (docs/api/en/kernel-info.md; vapoursynth.cpp:64-69): labels of the
 * active implementation. Each string buffer receives at most len bytes. */
nf_status nf_kernel_info(char* fft_backend, size_t fft_backend_len, char* target, size_t target_len, char* fft,
                         size_t fft_len, int* fft_lanes);

/* Library/ABI version for loaders. */
int nf_abi_version(void);

/* Row copy of the host layer's ROI packing (Plan::copy_row, src/algorithms/plan.hpp:82;
 * CopyRow and copy_row_scalar, src/kernels/rows.hpp:4-7): `bytes` bytes from source to
 * dst, each in host or device memory (device rows are copied with cudaMemcpy, host rows
 * with memcpy). Signature-compatible with neo_fft::CopyRow. */
void nf_copy_row(const void* source, void* dst, size_t bytes);

/* A non-blocking CUDA stream for one request's workspace (the facade's
 * runtime::Workspace, in place of the reference's per-request host workspace,
 * src/runtime/workspace_pool.hpp:12-75). Destroying waits for the stream's work. */
nf_status nf_stream_create(void** stream, char* err, size_t err_len);
void nf_stream_destroy(void* stream);

#ifdef __cplusplus
}
#endif
#endif /* NEO_FFT_B200_H */
