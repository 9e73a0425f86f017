// Project-written stand-in for the fixed-size tensor header of the
// `numericaltoolbox` dependency (gitlab.com/gabsillis/numericaltoolbox), which is
// an empty git submodule in the reference checkout (pinned commit unknown: the
// gitlink lives in git metadata that is not available).
//
// Test infrastructure only: it lets the reference's own, unmodified headers
// compile so that they can be run as the CPU reference for parity checks.
// Every function restates the published mathematics that the reference's call
// sites rely on (determinant, adjugate, generalised cross product, norms).
#pragma once
#include <array>
#include <cmath>
#include <cstddef>
#include <concepts>
#include <type_traits>
#include <algorithm>

#ifndef SQUARED
#define SQUARED(x) ((x) * (x))
#endif

namespace NUMTOOL::TENSOR::FIXED_SIZE {

template <class T, std::size_t... sizes>
struct Tensor;

namespace detail {
template <std::size_t... s> struct prod_t { static constexpr std::size_t value = 1; };
template <std::size_t a, std::size_t... s> struct prod_t<a, s...> {
  static constexpr std::size_t value = a * prod_t<s...>::value;
};
}  // namespace detail

// rank-1
template <class T, std::size_t n>
struct Tensor<T, n> {
  using value_type = T;
  static constexpr std::size_t rank_v = 1;
  static constexpr std::size_t total = n;
  T _data[n == 0 ? 1 : n];

  constexpr T& operator[](std::size_t i) { return _data[i]; }
  constexpr const T& operator[](std::size_t i) const { return _data[i]; }
  constexpr T* data() { return _data; }
  constexpr const T* data() const { return _data; }
  constexpr T* ptr() { return _data; }
  constexpr const T* ptr() const { return _data; }
  static constexpr std::size_t size() { return n; }
  static constexpr std::size_t rank() { return 1; }
  static constexpr std::size_t extent(std::size_t) { return n; }
  constexpr T* begin() { return _data; }
  constexpr T* end() { return _data + n; }
  constexpr const T* begin() const { return _data; }
  constexpr const T* end() const { return _data + n; }

  constexpr Tensor& operator=(const T& v) {
    for (std::size_t i = 0; i < n; ++i) _data[i] = v;
    return *this;
  }
  constexpr Tensor& operator+=(const Tensor& o) {
    for (std::size_t i = 0; i < n; ++i) _data[i] += o._data[i];
    return *this;
  }
  constexpr Tensor& operator-=(const Tensor& o) {
    for (std::size_t i = 0; i < n; ++i) _data[i] -= o._data[i];
    return *this;
  }
  constexpr Tensor& operator+=(const T& v) {
    for (std::size_t i = 0; i < n; ++i) _data[i] += v;
    return *this;
  }
  constexpr Tensor& operator*=(const T& v) {
    for (std::size_t i = 0; i < n; ++i) _data[i] *= v;
    return *this;
  }
  constexpr Tensor& operator/=(const T& v) {
    for (std::size_t i = 0; i < n; ++i) _data[i] /= v;
    return *this;
  }

  /// value of the tensor at a list of indices (rank-1: first entry)
  template <class I>
  constexpr T list_index(const I* idx) const { return _data[idx[0]]; }
};

// rank >= 2
template <class T, std::size_t n, std::size_t m, std::size_t... rest>
struct Tensor<T, n, m, rest...> {
  using value_type = T;
  using sub_t = Tensor<T, m, rest...>;
  static constexpr std::size_t total = n * detail::prod_t<m, rest...>::value;
  sub_t _data[n];

  constexpr sub_t& operator[](std::size_t i) { return _data[i]; }
  constexpr const sub_t& operator[](std::size_t i) const { return _data[i]; }

  // C++23 multidimensional subscript
  template <class I0, class... Is>
    requires(sizeof...(Is) >= 1 && std::is_integral_v<I0>)
  constexpr T& operator[](I0 i0, Is... is) { return _data[i0][is...]; }
  template <class I0, class... Is>
    requires(sizeof...(Is) >= 1 && std::is_integral_v<I0>)
  constexpr const T& operator[](I0 i0, Is... is) const { return _data[i0][is...]; }

  constexpr T* data() { return reinterpret_cast<T*>(this); }
  constexpr const T* data() const { return reinterpret_cast<const T*>(this); }
  constexpr T* ptr() { return data(); }
  constexpr const T* ptr() const { return data(); }
  static constexpr std::size_t size() { return total; }
  static constexpr std::size_t rank() { return 2 + sizeof...(rest); }

  constexpr Tensor& operator=(const T& v) {
    for (std::size_t i = 0; i < n; ++i) _data[i] = v;
    return *this;
  }
  constexpr Tensor& operator+=(const Tensor& o) {
    for (std::size_t i = 0; i < n; ++i) _data[i] += o._data[i];
    return *this;
  }
  constexpr Tensor& operator*=(const T& v) {
    for (std::size_t i = 0; i < n; ++i) _data[i] *= v;
    return *this;
  }
  constexpr Tensor& operator/=(const T& v) {
    for (std::size_t i = 0; i < n; ++i) _data[i] /= v;
    return *this;
  }

  /// value at a list of indices, e.g. levi_civita.list_index({i, j, k})
  template <class I>
  constexpr T list_index(const I* idx) const { return _data[idx[0]].list_index(idx + 1); }
};

// elementwise arithmetic (recursive over the nested storage so that it stays
// usable in constant expressions)
template <class T, std::size_t n>
constexpr void ew_binary(Tensor<T, n>& r, const Tensor<T, n>& a, const Tensor<T, n>& b, int op) {
  for (std::size_t i = 0; i < n; ++i) r[i] = (op == 0) ? a[i] - b[i] : a[i] + b[i];
}
template <class T, std::size_t n, std::size_t m, std::size_t... rest>
constexpr void ew_binary(Tensor<T, n, m, rest...>& r, const Tensor<T, n, m, rest...>& a,
                         const Tensor<T, n, m, rest...>& b, int op) {
  for (std::size_t i = 0; i < n; ++i) ew_binary(r[i], a[i], b[i], op);
}
template <class T, std::size_t n>
constexpr void ew_scale(Tensor<T, n>& r, const Tensor<T, n>& a, const T& v, int op) {
  for (std::size_t i = 0; i < n; ++i) r[i] = (op == 0) ? a[i] / v : a[i] * v;
}
template <class T, std::size_t n, std::size_t m, std::size_t... rest>
constexpr void ew_scale(Tensor<T, n, m, rest...>& r, const Tensor<T, n, m, rest...>& a, const T& v, int op) {
  for (std::size_t i = 0; i < n; ++i) ew_scale(r[i], a[i], v, op);
}
template <class T, std::size_t n>
constexpr T sum_sq(const Tensor<T, n>& a) {
  T s = 0;
  for (std::size_t i = 0; i < n; ++i) s += a[i] * a[i];
  return s;
}
template <class T, std::size_t n, std::size_t m, std::size_t... rest>
constexpr T sum_sq(const Tensor<T, n, m, rest...>& a) {
  T s = 0;
  for (std::size_t i = 0; i < n; ++i) s += sum_sq(a[i]);
  return s;
}

template <class T, std::size_t... s>
constexpr Tensor<T, s...> operator-(const Tensor<T, s...>& a, const Tensor<T, s...>& b) {
  Tensor<T, s...> r{};
  ew_binary(r, a, b, 0);
  return r;
}
template <class T, std::size_t... s>
constexpr Tensor<T, s...> operator+(const Tensor<T, s...>& a, const Tensor<T, s...>& b) {
  Tensor<T, s...> r{};
  ew_binary(r, a, b, 1);
  return r;
}
template <class T, std::size_t... s>
constexpr Tensor<T, s...> operator/(const Tensor<T, s...>& a, const T& v) {
  Tensor<T, s...> r{};
  ew_scale(r, a, v, 0);
  return r;
}
template <class T, std::size_t... s>
constexpr Tensor<T, s...> operator*(const T& v, const Tensor<T, s...>& a) {
  Tensor<T, s...> r{};
  ew_scale(r, a, v, 1);
  return r;
}
template <class T, std::size_t... s>
constexpr Tensor<T, s...> operator*(const Tensor<T, s...>& a, const T& v) { return v * a; }

/// y += alpha * x
template <class T, std::size_t n>
constexpr void axpy(T alpha, const Tensor<T, n>& x, Tensor<T, n>& y) {
  for (std::size_t i = 0; i < n; ++i) y[i] += alpha * x[i];
}

/// dot product of two vectors
template <class T, std::size_t n>
constexpr T dot(const Tensor<T, n>& a, const Tensor<T, n>& b) {
  T s = 0;
  for (std::size_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

/// Frobenius norm sqrt(sum a_ij^2)
template <class T, std::size_t... s>
constexpr T frobenius(const Tensor<T, s...>& a) {
  return std::sqrt(sum_sq(a));
}

/// Euclidean norm of a vector
template <class T, std::size_t n>
constexpr T norml2(const Tensor<T, n>& a) { return std::sqrt(dot(a, a)); }

/// unit vector a / |a|
template <class T, std::size_t n>
constexpr Tensor<T, n> normalize(const Tensor<T, n>& a) {
  T nrm = std::sqrt(dot(a, a));
  Tensor<T, n> r{};
  for (std::size_t i = 0; i < n; ++i) r[i] = a[i] / nrm;
  return r;
}

/// determinant by cofactor expansion (sizes used by the reference: 1, 2, 3)
template <class T, std::size_t n>
constexpr T determinant(const Tensor<T, n, n>& a) {
  if constexpr (n == 1) {
    return a[0][0];
  } else if constexpr (n == 2) {
    return a[0][0] * a[1][1] - a[0][1] * a[1][0];
  } else if constexpr (n == 3) {
    return a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1])
         - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0])
         + a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
  } else {
    // Laplace expansion along the first row
    T det = 0;
    for (std::size_t j = 0; j < n; ++j) {
      Tensor<T, n - 1, n - 1> minor{};
      for (std::size_t r = 1; r < n; ++r) {
        std::size_t cc = 0;
        for (std::size_t c = 0; c < n; ++c) {
          if (c == j) continue;
          minor[r - 1][cc++] = a[r][c];
        }
      }
      T sgn = (j % 2 == 0) ? 1 : -1;
      det += sgn * a[0][j] * determinant(minor);
    }
    return det;
  }
}

/// adjugate (transpose of the cofactor matrix): inverse(a) = adjugate(a) / det(a)
template <class T, std::size_t n>
constexpr Tensor<T, n, n> adjugate(const Tensor<T, n, n>& a) {
  Tensor<T, n, n> adj{};
  if constexpr (n == 1) {
    adj[0][0] = 1;
  } else if constexpr (n == 2) {
    adj[0][0] = a[1][1];
    adj[0][1] = -a[0][1];
    adj[1][0] = -a[1][0];
    adj[1][1] = a[0][0];
  } else {
    for (std::size_t i = 0; i < n; ++i) {
      for (std::size_t j = 0; j < n; ++j) {
        Tensor<T, n - 1, n - 1> minor{};
        std::size_t rr = 0;
        for (std::size_t r = 0; r < n; ++r) {
          if (r == j) continue;
          std::size_t cc = 0;
          for (std::size_t c = 0; c < n; ++c) {
            if (c == i) continue;
            minor[rr][cc++] = a[r][c];
          }
          ++rr;
        }
        T sgn = ((i + j) % 2 == 0) ? 1 : -1;
        adj[i][j] = sgn * determinant(minor);
      }
    }
  }
  return adj;
}

/// Levi-Civita symbol of rank n as a fixed-size tensor
template <class T, std::size_t... s> struct lc_builder;
template <class T, std::size_t n>
constexpr T& flat_ref(Tensor<T, n>& t, std::size_t flat) { return t[flat]; }
template <class T, std::size_t n, std::size_t m, std::size_t... rest>
constexpr T& flat_ref(Tensor<T, n, m, rest...>& t, std::size_t flat) {
  constexpr std::size_t sub = Tensor<T, m, rest...>::total;
  return flat_ref(t[flat / sub], flat % sub);
}
template <class T, std::size_t n, std::size_t... idx>
constexpr auto make_levi_civita(std::index_sequence<idx...>) {
  Tensor<T, ((void)idx, n)...> t{};
  std::size_t total = 1;
  for (std::size_t k = 0; k < n; ++k) total *= n;
  for (std::size_t flat = 0; flat < total; ++flat) {
    std::size_t ind[n];
    std::size_t rem = flat;
    for (std::size_t k = 0; k < n; ++k) {
      ind[n - 1 - k] = rem % n;
      rem /= n;
    }
    // sign of the permutation (0 if an index repeats)
    T sgn = 1;
    for (std::size_t a = 0; a < n; ++a)
      for (std::size_t b = a + 1; b < n; ++b) {
        if (ind[a] == ind[b]) sgn = 0;
        else if (ind[a] > ind[b]) sgn = -sgn;
      }
    flat_ref(t, flat) = sgn;
  }
  return t;
}
template <class T, int n>
inline constexpr auto levi_civita = make_levi_civita<T, (std::size_t)n>(std::make_index_sequence<(std::size_t)n>{});

/// Vector orthogonal to the n-1 columns of the n x (n-1) matrix J: the
/// generalised cross product (Hodge star of the columns),
///   v_i = eps_{i j1 ... j_{n-1}} J_{j1,0} ... J_{j_{n-1},n-2}.
/// In 2D this is (J_10, -J_00): the tangent rotated clockwise, which is the
/// outward normal for counter-clockwise traversal.
template <class T, std::size_t n, std::size_t m>
constexpr Tensor<T, n> calc_ortho(const Tensor<T, n, m>& J) {
  static_assert(m + 1 == n, "calc_ortho expects an n x (n-1) matrix");
  Tensor<T, n> v{};
  if constexpr (n == 1) {
    v[0] = 1;
  } else if constexpr (n == 2) {
    v[0] = J[1][0];
    v[1] = -J[0][0];
  } else if constexpr (n == 3) {
    v[0] = J[1][0] * J[2][1] - J[2][0] * J[1][1];
    v[1] = J[2][0] * J[0][1] - J[0][0] * J[2][1];
    v[2] = J[0][0] * J[1][1] - J[1][0] * J[0][1];
  }
  return v;
}

}  // namespace NUMTOOL::TENSOR::FIXED_SIZE
