// Creation-time plan tables for the B200 pipeline (host side).
//
// Everything a neo-fft `Plan` computes in its constructors
// (src/algorithms/plan.cpp:45-226) is computed here once on the host: validation
// with the reference's error texts, block geometry, analysis/synthesis windows,
// noise and enhancement tables and the degrid/zmean template. The tables are then
// uploaded to device memory and stay immutable for the plan's lifetime.
//
// The arithmetic follows the reference operation by operation (binary32 with no
// contraction, binary64 where the reference uses double), so the tables are
// bit-identical to the reference's; tests compare them against the reference core.
#pragma once
#include "neo_fft_b200.h"
#include "fft_core.cuh"

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace nfb {

using nf::cf;

struct Axis {
  int length = 0, block = 0, overlap = 0, step = 0, count = 0, cover = 0, offset = 0;
};

// Errors carry the reference's texts; invalid_argument for configuration and
// geometry (src/base/checked.hpp:13-20), runtime_error for non-finite values
// (checked.hpp:37-41).
inline void require(bool ok, const char* message) {
  if (!ok) throw std::invalid_argument(message);
}
inline float finite(float v) {
  if (!(v - v == 0.0f)) throw std::runtime_error("non-finite sample or intermediate");
  return v;
}

Axis fft3d_axis(int length, int block, int overlap);
Axis dft_axis(int length, int block, int mode, int overlap);
int reflect(int cover_coordinate, const Axis& a);

struct AxisWindow {
  std::vector<float> analysis, synthesis;
};
AxisWindow fft3d_window(int block, int overlap, int type);
double dft_raw_window(int id, int j, int length, float beta);
struct DftWindow {
  std::vector<float> h;
  float wscale = 0;
};
DftWindow dft_window_3d(int tbsize, int block, int overlap, int mode, int spatial, int temporal, float sbeta,
                        float tbeta, int temporal_mode, int temporal_overlap);

struct Curves {
  std::vector<float> shared, x, y, time;
  int system = 0;
  bool empty() const { return shared.empty() && x.empty() && y.empty() && time.empty(); }
};
std::vector<float> dft_profile(const Curves& c, int T, int S, float sigma, float divisor);
std::vector<float> fft3d_profile(int W, int H, const float s[4]);

struct Enhancement {
  float sharpen = 0, dehalo = 0, a = 0, b = 0, c = 0;
  std::vector<float> sharpen_window, halo_window;
  bool active() const { return sharpen != 0 || dehalo != 0; }
};
Enhancement enhancement_tables(int W, int H, float factor, const nf_fft3d_config& c);

// Temporal lattice of DFTTest tmode=1 (src/algorithms/temporal_grid.hpp:5-40).
void validate_temporal(int size, int mode, int overlap);
struct TemporalBlock {
  long long start;
  int target;
  int slots[15];
};
std::vector<TemporalBlock> temporal_blocks(int frame, int length, int size, int overlap);

// Project twiddle table w_n^m = exp(-2*pi*i*m/n), binary64 rounded once.
std::vector<cf> twiddle_table(int n);

// Host transforms with the device's arithmetic (fft_core.cuh).
void host_r2c_2d(const float* in, cf* out, int h, int w);
void host_r2c_3d(const float* in, cf* out, int t, int h, int w);

enum class Algo { FFT3D, DFTTest };

// Per-bin spectral parameters (kernels/spectral.hpp:75-83): type -2 enhancement
// only, -1 FFT3D Wiener, 0..4 DFTTest ftypes. `primary` empty means uniform `a`.
struct Spectral {
  int type = -1;
  float a = 0, b = 0, low = 0, high = 0, exponent = 1, floor = 0;
  std::vector<float> primary;
  bool fused_enhancement = false;
};

struct PlanTables {
  Algo algo = Algo::FFT3D;
  nf_format format{};
  Axis gx, gy;
  int temporal_size = 1;
  int bh = 0, bw = 0, bins = 0;  // spatial block, half-spectrum bins
  // FFT3D
  AxisWindow wx, wy;
  bool denoise = true, kalman = false, preview = false, sampled = false, varying = false;
  bool needs_pattern = false;          // sampled && denoise: primary table from the pattern block
  float pfactor = 0;
  int px = 0, py = 0;                  // pattern block (0, 0: automatic search)
  int pframe = 0;                      // frame the pattern is sampled from (before clamping)
  int kalman_warmup = 8;               // host layer's bounded Kalman warm-up on random access
  std::vector<float> sample_weights;   // [bh][bw/2+1] pattern scoring weights (plan.cpp:142-158)
  float sigma_eff = 0, norm = 0, beta = 1, kalman_r0 = 0, kalman_ratio2 = 0;
  Enhancement enhancement;
  // DFTTest
  std::vector<float> h, h_synthesis;
  float wscale = 0;
  bool center = false, temporal_ola = false;
  bool noise_model = false;  // primary table comes from the sampled noise model (nlocation)
  int temporal_overlap = 0, dither = 0, dither_seed = 0;
  // both
  Spectral spectral;
  float mean_scale = 0;
  std::vector<cf> grid;  // empty: no degrid / zmean
};

PlanTables build_fft3d(int width, int height, nf_format format, const nf_fft3d_config& c);

// DFTTest sampled noise model (DFTNoise, src/algorithms/dft_noise.cpp:5-41): sample
// window, template spectrum of 255*window and calibration, checked at plan creation;
// dft_noise_power averages the windowed 3-D power spectra of the gathered slices
// ([location][tbsize][sbsize][sbsize], 8-bit amplitude units) into the primary table.
struct DftNoiseSetup {
  std::vector<float> window;
  std::vector<cf> grid;
  float calibration = 0;
  int temporal_size = 1, block = 0, bins3 = 0;
  bool zmean = false;
};
DftNoiseSetup dft_noise_setup(const nf_dft_config& c);
std::vector<float> dft_noise_power(const nf_dft_config& c, const float* slices, int nlocations);
PlanTables build_dft(int width, int height, nf_format format, const nf_dft_config& c);

} // namespace nfb
