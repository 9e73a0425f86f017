// Project-written stand-in for the point header of the `numericaltoolbox`
// dependency (empty submodule in the reference checkout). Test infrastructure
// only: lets the reference's headers compile for the CPU reference build.
#pragma once
#include <array>
#include <cmath>
#include <cstddef>
#include <span>
#include <type_traits>

namespace MATH::GEOMETRY {

/// fixed-size point: contiguous coordinates, converts to a raw pointer
template <class T, int ndim>
struct Point {
  static constexpr std::size_t N = ndim > 0 ? (std::size_t)ndim : 0;
  std::array<T, N> x{};

  constexpr Point() = default;
  constexpr Point(std::initializer_list<T> il) {
    std::size_t i = 0;
    for (const T& v : il) { if (i < N) x[i++] = v; }
  }
  template <class I>
    requires std::is_integral_v<I>
  constexpr T& operator[](I i) { return x[i]; }
  template <class I>
    requires std::is_integral_v<I>
  constexpr const T& operator[](I i) const { return x[i]; }
  constexpr T* data() { return x.data(); }
  constexpr const T* data() const { return x.data(); }
  constexpr operator T*() { return x.data(); }
  constexpr operator const T*() const { return x.data(); }
  constexpr operator std::span<T, N>() { return std::span<T, N>(x.data(), N); }
  constexpr operator std::span<const T, N>() const { return std::span<const T, N>(x.data(), N); }
  constexpr auto begin() { return x.begin(); }
  constexpr auto end() { return x.end(); }
  constexpr auto begin() const { return x.begin(); }
  constexpr auto end() const { return x.end(); }
  static constexpr std::size_t size() { return N; }
};

/// non-owning view of ndim coordinates
template <class T, int ndim>
struct PointView {
  T* p;
  constexpr PointView(T* ptr) : p(ptr) {}
  constexpr PointView(Point<T, ndim>& pt) : p(pt.data()) {}
  template <class I>
    requires std::is_integral_v<I>
  constexpr T& operator[](I i) const { return p[i]; }
  constexpr T* data() const { return p; }
  constexpr operator T*() const { return p; }
  static constexpr std::size_t size() { return ndim; }
};

/// Euclidean distance between two points
template <class T, int ndim>
constexpr T distance(const Point<T, ndim>& a, const Point<T, ndim>& b) {
  T s = 0;
  for (int i = 0; i < ndim; ++i) { T d = a[i] - b[i]; s += d * d; }
  return std::sqrt(s);
}

}  // namespace MATH::GEOMETRY
