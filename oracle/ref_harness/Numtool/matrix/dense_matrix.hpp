// Project-written stand-in for the dense matrix header of the
// `numericaltoolbox` dependency. Test infrastructure only.
#pragma once
#include <vector>
#include <cstddef>

namespace MATH::MATRIX {
template <class T>
class DenseMatrix {
  std::size_t m_ = 0, n_ = 0;
  std::vector<T> a_;
 public:
  DenseMatrix() = default;
  DenseMatrix(std::size_t m, std::size_t n) : m_(m), n_(n), a_(m * n, T(0)) {}
  T* operator[](std::size_t i) { return a_.data() + i * n_; }
  const T* operator[](std::size_t i) const { return a_.data() + i * n_; }
  DenseMatrix& operator=(const T& v) { for (auto& x : a_) x = v; return *this; }
  std::size_t m() const { return m_; }
  std::size_t n() const { return n_; }
  T* data() { return a_.data(); }
};
}  // namespace MATH::MATRIX
