// Project-written stand-in (test infrastructure only).
#pragma once
#include <vector>
namespace MATH::MATRIX {
template <class I>
struct PermutationMatrix {
  std::vector<I> p;
  PermutationMatrix() = default;
  explicit PermutationMatrix(I n) : p(n) { for (I i = 0; i < n; ++i) p[i] = i; }
  I operator[](std::size_t i) const { return p[i]; }
};
}  // namespace MATH::MATRIX
