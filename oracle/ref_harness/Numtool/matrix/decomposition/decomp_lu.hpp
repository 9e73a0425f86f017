// Project-written stand-in for the LU decomposition of the `numericaltoolbox`
// dependency: partial-pivoting Doolittle LU in place, and the matching
// forward/back substitution. Test infrastructure only.
#pragma once
#include <cmath>
#include <exception>
#include <utility>
#include "../dense_matrix.hpp"
#include "../permutation_matrix.hpp"
namespace MATH::MATRIX::SOLVERS {
struct SingularMatrixException : std::exception {
  const char* what() const noexcept override { return "singular matrix"; }
};
template <class T>
PermutationMatrix<unsigned int> decompose_lu(DenseMatrix<T>& a) {
  unsigned int n = (unsigned int)a.m();
  PermutationMatrix<unsigned int> pi{n};
  for (unsigned int k = 0; k < n; ++k) {
    unsigned int piv = k;
    T best = std::abs(a[k][k]);
    for (unsigned int i = k + 1; i < n; ++i)
      if (std::abs(a[i][k]) > best) { best = std::abs(a[i][k]); piv = i; }
    if (best == T(0)) throw SingularMatrixException{};
    if (piv != k) {
      for (unsigned int j = 0; j < n; ++j) std::swap(a[k][j], a[piv][j]);
      std::swap(pi.p[k], pi.p[piv]);
    }
    for (unsigned int i = k + 1; i < n; ++i) {
      a[i][k] /= a[k][k];
      for (unsigned int j = k + 1; j < n; ++j) a[i][j] -= a[i][k] * a[k][j];
    }
  }
  return pi;
}
template <class T>
void sub_lu(const DenseMatrix<T>& a, const PermutationMatrix<unsigned int>& pi, const T* b, T* x) {
  std::size_t n = a.m();
  for (std::size_t i = 0; i < n; ++i) {
    T s = b[pi[i]];
    for (std::size_t j = 0; j < i; ++j) s -= a[i][j] * x[j];
    x[i] = s;
  }
  for (std::size_t ii = n; ii-- > 0;) {
    T s = x[ii];
    for (std::size_t j = ii + 1; j < n; ++j) s -= a[ii][j] * x[j];
    x[ii] = s / a[ii][ii];
  }
}
}  // namespace MATH::MATRIX::SOLVERS
