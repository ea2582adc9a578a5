// Test infrastructure (oracle only): a minimal project-written stand-in for the
// DualSynth2 `span2d` header that the neo-fft core includes. DualSynth2 is fetched
// by the reference's CMake at configure time (cmake/Dependencies.cmake:11-19) and
// is absent here, so the oracle build supplies this header instead.
//
// Semantics follow what the core and its tests rely on:
//   * Plane<T>: data pointer, width, height and a SIGNED byte stride (bottom-up
//     planes are legal, tests/unit/foundation.cpp:22-29), row_ptr/row/subplane,
//     element access (y, x), implicit Plane<T> -> Plane<const T>.
//   * Span<T>: pointer + count, brace-constructible, implicit Span<T> -> Span<const T>.
//   * RestrictPlane/RestrictSpan are plain aliases (the restrict qualifier is an
//     optimisation hint only).
#pragma once
#include <cstddef>
#include <cstdint>
#include <type_traits>

namespace span2d {

template <class T>
class Span {
public:
  using element_type = T;
  constexpr Span() noexcept = default;
  constexpr Span(T* data, std::size_t size) noexcept : data_(data), size_(size) {}
  template <class U, class = std::enable_if_t<std::is_same_v<const U, T> && !std::is_same_v<U, T>>>
  constexpr Span(const Span<U>& other) noexcept : data_(other.data()), size_(other.size()) {}
  constexpr T* data() const noexcept { return data_; }
  constexpr std::size_t size() const noexcept { return size_; }
  constexpr bool empty() const noexcept { return size_ == 0; }
  constexpr T& operator[](std::size_t i) const noexcept { return data_[i]; }
  constexpr T* begin() const noexcept { return data_; }
  constexpr T* end() const noexcept { return data_ + size_; }
  constexpr Span as_restrict() const noexcept { return *this; }

private:
  T* data_ = nullptr;
  std::size_t size_ = 0;
};

template <class T>
class Plane {
public:
  using element_type = T;
  constexpr Plane() noexcept = default;
  constexpr Plane(T* data, int width, int height, std::ptrdiff_t stride_bytes) noexcept
      : data_(data), width_(width), height_(height), stride_bytes_(stride_bytes) {}
  template <class U, class = std::enable_if_t<std::is_same_v<const U, T> && !std::is_same_v<U, T>>>
  constexpr Plane(const Plane<U>& other) noexcept
      : data_(other.data()), width_(other.width()), height_(other.height()), stride_bytes_(other.stride_bytes()) {}

  constexpr T* data() const noexcept { return data_; }
  constexpr int width() const noexcept { return width_; }
  constexpr int height() const noexcept { return height_; }
  constexpr std::ptrdiff_t stride_bytes() const noexcept { return stride_bytes_; }
  constexpr std::ptrdiff_t stride() const noexcept { return stride_bytes_ / std::ptrdiff_t(sizeof(T)); }
  constexpr bool empty() const noexcept { return data_ == nullptr || width_ <= 0 || height_ <= 0; }

  template <class I>
  T* row_ptr(I y) const noexcept {
    using byte = std::conditional_t<std::is_const_v<T>, const unsigned char, unsigned char>;
    return reinterpret_cast<T*>(reinterpret_cast<byte*>(data_) + std::ptrdiff_t(y) * stride_bytes_);
  }
  template <class I>
  Span<T> row(I y) const noexcept { return Span<T>(row_ptr(y), std::size_t(width_)); }
  template <class I, class J>
  T& operator()(I y, J x) const noexcept { return row_ptr(y)[std::ptrdiff_t(x)]; }
  Plane subplane(int x, int y, int w, int h) const noexcept { return Plane(row_ptr(y) + x, w, h, stride_bytes_); }
  constexpr Plane as_restrict() const noexcept { return *this; }

private:
  T* data_ = nullptr;
  int width_ = 0, height_ = 0;
  std::ptrdiff_t stride_bytes_ = 0;
};

template <class T> using RestrictPlane = Plane<T>;
template <class T> using RestrictSpan = Span<T>;

} // namespace span2d
