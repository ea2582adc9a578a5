// Test-only host shim: exposes the product's creation-time table builders
// (neo_fft_b200/csrc/plan_build.cpp) so CPU tests can compare them with the
// reference core's tables without a GPU.
#include "plan_build.hpp"

#include <cstring>
#include <stdexcept>

extern "C" {
int tb_fft3d_window(int block, int overlap, int type, float* a, float* s) {
  try {
    auto w = nfb::fft3d_window(block, overlap, type);
    std::memcpy(a, w.analysis.data(), w.analysis.size() * 4);
    std::memcpy(s, w.synthesis.data(), w.synthesis.size() * 4);
    return 0;
  } catch (...) { return 1; }
}
int tb_dft_window_3d(int tb, int b, int o, int mode, int sw, int tw, float sbeta, float tbeta, int tmode, int tov,
                     float* h, float* wscale) {
  try {
    auto w = nfb::dft_window_3d(tb, b, o, mode, sw, tw, sbeta, tbeta, tmode, tov);
    std::memcpy(h, w.h.data(), w.h.size() * 4);
    *wscale = w.wscale;
    return 0;
  } catch (...) { return 1; }
}
// Full plan tables: writes sizes into `sizes` and copies tables into caller buffers
// (grid as interleaved floats). Returns 1 on invalid_argument, 2 on runtime_error.
int tb_plan(int algo, int w, int h, nf_format f, const void* cfg, int* sizes, float* grid, float* primary,
            float* sharpen, float* halo, float* hwin, float* scalars, char* err, size_t len) {
  try {
    nfb::PlanTables t = algo == 0 ? nfb::build_fft3d(w, h, f, *static_cast<const nf_fft3d_config*>(cfg))
                                  : nfb::build_dft(w, h, f, *static_cast<const nf_dft_config*>(cfg));
    sizes[0] = int(t.grid.size());
    sizes[1] = int(t.spectral.primary.size());
    sizes[2] = int(t.enhancement.sharpen_window.size());
    sizes[3] = int(t.enhancement.halo_window.size());
    sizes[4] = int(t.h.size());
    if (grid) std::memcpy(grid, t.grid.data(), t.grid.size() * 8);
    if (primary) std::memcpy(primary, t.spectral.primary.data(), t.spectral.primary.size() * 4);
    if (sharpen) std::memcpy(sharpen, t.enhancement.sharpen_window.data(), t.enhancement.sharpen_window.size() * 4);
    if (halo) std::memcpy(halo, t.enhancement.halo_window.data(), t.enhancement.halo_window.size() * 4);
    if (hwin) std::memcpy(hwin, t.h.data(), t.h.size() * 4);
    scalars[0] = t.spectral.a; scalars[1] = t.spectral.b; scalars[2] = t.spectral.low; scalars[3] = t.spectral.high;
    scalars[4] = t.spectral.floor; scalars[5] = t.wscale; scalars[6] = t.enhancement.a; scalars[7] = t.enhancement.b;
    scalars[8] = t.enhancement.c; scalars[9] = t.kalman_r0; scalars[10] = t.kalman_ratio2;
    sizes[5] = t.gx.count; sizes[6] = t.gy.count; sizes[7] = t.gx.cover; sizes[8] = t.gy.cover;
    sizes[9] = t.gx.offset; sizes[10] = t.gy.offset;
    return 0;
  } catch (const std::invalid_argument& e) {
    std::strncpy(err, e.what(), len - 1);
    return 1;
  } catch (const std::runtime_error& e) {
    std::strncpy(err, e.what(), len - 1);
    return 2;
  }
}
// The product's C++ temporal lattice (plan_build.cpp, used by the clip batches and the frame
// server): up to `cap` blocks with start, target and `size` slots; 1 with the text on error.
int tb_temporal_blocks(int frame, int length, int size, int overlap, long long* starts, int* targets, int* slots,
                       int cap, int* count, char* err, size_t len) {
  try {
    const auto blocks = nfb::temporal_blocks(frame, length, size, overlap);
    *count = int(blocks.size());
    for (int i = 0; i < cap && i < *count; ++i) {
      starts[i] = blocks[size_t(i)].start;
      targets[i] = blocks[size_t(i)].target;
      for (int z = 0; z < size; ++z) slots[i * size + z] = blocks[size_t(i)].slots[z];
    }
    return 0;
  } catch (const std::exception& e) {
    std::strncpy(err, e.what(), len - 1);
    err[len - 1] = 0;
    return 1;
  }
}
}
