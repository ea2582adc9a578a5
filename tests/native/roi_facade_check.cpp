// Test-only: the reference host layer's ROI/interlaced code, compiled unchanged from its own
// source (src/plugin/roi.hpp, reached through -I <reference>/src), against the B200 facade
// (include/neo_fft_b200/plan.hpp), making the calls src/plugin/filter.hpp makes:
//   * plane<T>, FFT3D with an interlaced ROI (filter.hpp:354-365): PackedROI per source with
//     plan->copy_row(), process_at over the packed views, output.write(d, roi);
//   * render_plane<T> (filter.hpp:217-230): render_kalman through PackedROI;
//   * prepare_pattern<T> (filter.hpp:372-380): prepare_pattern on the packed view;
//   * with_roi<T> (filter.hpp:138-143): the packed view handed to a callable.
// Usage: roi_facade_check <in.u8> <out_fft3d.u8> <out_kalman.f32> <out_pattern.u8>
// (raw planes of the sizes below). Exits non-zero on an exception.
#include "plugin/roi.hpp"

#include <cstdio>
#include <cstdint>
#include <fstream>
#include <vector>

using namespace neo_fft;
using neo_fft::plugin::PackedROI;
using neo_fft::plugin::ROI;

namespace {
constexpr int W = 160, H = 120;

template <class T>
std::vector<T> read_raw(const char* path, std::size_t n) {
  std::vector<T> v(n);
  std::ifstream f(path, std::ios::binary);
  f.read(reinterpret_cast<char*>(v.data()), std::streamsize(n * sizeof(T)));
  if (!f) throw std::runtime_error(std::string("cannot read ") + path);
  return v;
}
template <class T>
void write_raw(const char* path, const std::vector<T>& v) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), std::streamsize(v.size() * sizeof(T)));
}

// filter.hpp:354-365, the interlaced branch of plane<T> for FFT3D (temporal slots of
// one frame here: the same source three times, as the host layer's edge clamps do).
template <class T>
void plane_interlaced(const std::vector<span2d::Plane<const T>>& checked_srcs, span2d::Plane<T> d, const Plan* plan,
                      const ROI& roi, int frame, int plane_index) {
  const auto& original = checked_srcs[checked_srcs.size() / 2];
  for (int y = 0; y < d.height(); ++y) std::memcpy(d.row_ptr(y), original.row_ptr(y), std::size_t(d.width()) * sizeof(T));
  std::vector<PackedROI<T>> packed;
  packed.reserve(checked_srcs.size());
  for (auto source : checked_srcs) packed.emplace_back(source, roi, plan->copy_row());
  std::vector<span2d::Plane<const T>> views;
  for (auto& image : packed) views.push_back(image.view);
  PackedROI<T> output(original, roi, plan->copy_row());
  plan->process_at<T>({views.data(), views.size()}, output.view, frame, plane_index, {},
                      static_cast<runtime::SpectraCache*>(nullptr));
  output.write(d, roi);
}

// filter.hpp:138-143
template <class T, class Function>
void with_roi(span2d::Plane<const T> s, const ROI& roi, CopyRow copy, Function&& fn) {
  if (!roi.interlaced) fn(checked_subplane(s, roi.left, roi.top, roi.width, roi.height));
  else {
    PackedROI<T> packed(s, roi, copy);
    fn(span2d::Plane<const T>(packed.view));
  }
}
}  // namespace

int main(int argc, char** argv) {
  if (argc < 5) return 2;
  try {
    FFT3DConfig c;
    c.bw = c.bh = 16; c.ow = c.oh = 8; c.sigma = 3.0f; c.bt = 3;
    c.left = 8; c.top = 4; c.right = 16; c.bottom = 12; c.interlaced = true;
    const ROI roi = plugin::make_roi(W, H, 0, 0, c);
    const auto src = read_raw<std::uint8_t>(argv[1], std::size_t(W) * H);
    span2d::Plane<const std::uint8_t> s(src.data(), W, H, W);
    // FFT3D bt=3 over an interlaced ROI
    Plan plan(roi.width, roi.height, SampleFormat{8, false, false}, c);
    std::vector<std::uint8_t> out(src.size());
    span2d::Plane<std::uint8_t> d(out.data(), W, H, W);
    plane_interlaced<std::uint8_t>({s, s, s}, d, &plan, roi, 0, 0);
    write_raw(argv[2], out);
    // Kalman render through PackedROI (filter.hpp:227-229) after two advances via with_roi
    FFT3DConfig k = c;
    k.bt = 0; k.kratio = 2.0f;
    Plan kp(roi.width, roi.height, SampleFormat{32, true, false}, k);
    std::vector<float> fsrc(src.size()), fout(src.size());
    for (std::size_t i = 0; i < src.size(); ++i) fsrc[i] = float(src[i]) / 255.0f;
    span2d::Plane<const float> fs(fsrc.data(), W, H, W * 4);
    KalmanState st = kp.initial_kalman();
    for (int f = 0; f < 2; ++f)
      with_roi<float>(fs, roi, kp.copy_row(), [&](auto view) { kp.advance_kalman(view, st); });
    span2d::Plane<float> fd(fout.data(), W, H, W * 4);
    for (int y = 0; y < H; ++y) std::memcpy(fd.row_ptr(y), fs.row_ptr(y), std::size_t(W) * 4);
    {
      PackedROI<float> input(fs, roi, kp.copy_row()), output(fs, roi, kp.copy_row());
      kp.render_kalman(span2d::Plane<const float>(input.view), output.view, st);
      output.write(fd, roi);
    }
    write_raw(argv[3], fout);
    // prepare_pattern on the packed view (filter.hpp:372-380), then filter the frame
    FFT3DConfig pc = c;
    pc.bt = 1; pc.pfactor = 1.0f;
    Plan pp(roi.width, roi.height, SampleFormat{8, false, false}, pc);
    {
      PackedROI<std::uint8_t> packed(s, roi, pp.copy_row());
      pp.prepare_pattern(span2d::Plane<const std::uint8_t>(packed.view));
    }
    std::vector<std::uint8_t> pout(src.size());
    plane_interlaced<std::uint8_t>({s}, span2d::Plane<std::uint8_t>(pout.data(), W, H, W), &pp, roi, 0, 0);
    write_raw(argv[4], pout);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "exception: %s\n", e.what());
    return 1;
  }
  std::printf("ok\n");
  return 0;
}
