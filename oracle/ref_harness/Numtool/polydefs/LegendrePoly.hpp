// Project-written stand-in for the Legendre polynomial helpers of the
// `numericaltoolbox` dependency. Restates the three-term recurrence
//   (k+1) P_{k+1}(x) = (2k+1) x P_k(x) - k P_{k-1}(x)
// and P_n'(x) = n (x P_n(x) - P_{n-1}(x)) / (x^2 - 1). Test infrastructure only.
#pragma once
#include <cmath>

namespace POLYNOMIAL {
template <class T, int n>
constexpr T legendre1d(T x) {
  if constexpr (n == 0) return 1;
  T pkm1 = 1, pk = x;
  for (int k = 1; k < n; ++k) {
    T pkp1 = ((2 * k + 1) * x * pk - k * pkm1) / (k + 1);
    pkm1 = pk;
    pk = pkp1;
  }
  return pk;
}
template <class T, int n>
constexpr T dlegendre1d(T x) {
  if constexpr (n == 0) return 0;
  // derivative recurrence P'_{k+1} = P'_{k-1} + (2k+1) P_k, robust at |x| = 1
  T pkm1 = 1, pk = x;       // P_0, P_1
  T dkm1 = 0, dk = 1;       // P_0', P_1'
  for (int k = 1; k < n; ++k) {
    T pkp1 = ((2 * k + 1) * x * pk - k * pkm1) / (k + 1);
    T dkp1 = dkm1 + (2 * k + 1) * pk;
    pkm1 = pk; pk = pkp1;
    dkm1 = dk; dk = dkp1;
  }
  return dk;
}
/// Legendre polynomial of runtime degree n
template <class T>
constexpr T legendre(int n, T x) {
  if (n == 0) return 1;
  T pkm1 = 1, pk = x;
  for (int k = 1; k < n; ++k) {
    T pkp1 = ((2 * k + 1) * x * pk - k * pkm1) / (k + 1);
    pkm1 = pk; pk = pkp1;
  }
  return pk;
}
template <class T>
constexpr T dlegendre(int n, T x) {
  if (n == 0) return 0;
  T pkm1 = 1, pk = x, dkm1 = 0, dk = 1;
  for (int k = 1; k < n; ++k) {
    T pkp1 = ((2 * k + 1) * x * pk - k * pkm1) / (k + 1);
    T dkp1 = dkm1 + (2 * k + 1) * pk;
    pkm1 = pk; pk = pkp1; dkm1 = dk; dk = dkp1;
  }
  return dk;
}
}  // namespace POLYNOMIAL
namespace MATH { namespace POLYNOMIAL = ::POLYNOMIAL; }
