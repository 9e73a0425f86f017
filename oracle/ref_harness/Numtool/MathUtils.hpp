// Project-written stand-in for the integer/math utility header of the
// `numericaltoolbox` dependency. Test infrastructure only.
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdint>

#ifndef SQUARED
#define SQUARED(x) ((x) * (x))
#endif

namespace MATH {

/// compile-time integer power base^exp
template <int base, int exp>
struct power_T {
  static constexpr int value = base * power_T<base, exp - 1>::value;
};
template <int base>
struct power_T<base, 0> {
  static constexpr int value = 1;
};

template <int n>
constexpr long long factorial() {
  long long r = 1;
  for (int i = 2; i <= n; ++i) r *= i;
  return r;
}

template <int n, int k>
constexpr long long binomial() {
  if (k < 0 || k > n) return 0;
  long long r = 1;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

constexpr long long factorial(int n) {
  long long r = 1;
  for (int i = 2; i <= n; ++i) r *= i;
  return r;
}

constexpr long long binomial(int n, int k) {
  if (k < 0 || k > n) return 0;
  long long r = 1;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

template <class T>
constexpr T integer_pow(T base, int exp) {
  T r = 1;
  for (int i = 0; i < exp; ++i) r *= base;
  return r;
}

/// floor(log2(n)) for positive integers
template <class I>
constexpr int log2(I n) {
  int r = 0;
  while (n > 1) { n >>= 1; ++r; }
  return r;
}

}  // namespace MATH
