// Project-written stand-in for the Lagrange polynomial helpers of the
// `numericaltoolbox` dependency. dNlagrange1d<T, Pn>(j, k, x) is the k-th
// derivative of the j-th Lagrange polynomial through the Pn+1 equispaced nodes
// x_m = -1 + 2m/Pn on [-1, 1], evaluated by differentiating the product form
// term by term. Test infrastructure only.
#pragma once
#include "LegendrePoly.hpp"

namespace POLYNOMIAL {
namespace detail {
/// sum over all ways to drop `k` distinct factors (m != j) of prod (x - x_m)
template <class T, int Pn>
constexpr T drop_sum(int j, int k, T x, const T* nodes, int start, const bool* dropped) {
  if (k == 0) {
    T p = 1;
    for (int m = 0; m <= Pn; ++m)
      if (m != j && !dropped[m]) p *= (x - nodes[m]);
    return p;
  }
  T s = 0;
  bool d2[Pn + 1];
  for (int m = 0; m <= Pn; ++m) d2[m] = dropped[m];
  for (int m = start; m <= Pn; ++m) {
    if (m == j || dropped[m]) continue;
    d2[m] = true;
    s += drop_sum<T, Pn>(j, k - 1, x, nodes, m + 1, d2);
    d2[m] = false;
  }
  return s;
}
}  // namespace detail

template <class T, int Pn>
constexpr T dNlagrange1d(int j, int k, T x) {
  T nodes[Pn + 1];
  for (int m = 0; m <= Pn; ++m) nodes[m] = (Pn == 0) ? T(0) : T(-1) + T(2) * m / Pn;
  T denom = 1;
  for (int m = 0; m <= Pn; ++m) if (m != j) denom *= (nodes[j] - nodes[m]);
  bool dropped[Pn + 1] = {};
  // k-th derivative of a product of linear factors: k! * sum over unordered
  // k-subsets of dropped factors of the product of the rest
  T fact = 1;
  for (int i = 2; i <= k; ++i) fact *= i;
  return fact * detail::drop_sum<T, Pn>(j, k, x, nodes, 0, dropped) / denom;
}
}  // namespace POLYNOMIAL
namespace MATH { namespace POLYNOMIAL = ::POLYNOMIAL; }
