// Project-written stand-in for the template-metaprogramming helpers of the
// `numericaltoolbox` dependency. Test infrastructure only.
#pragma once
#include <utility>
#include <type_traits>

namespace NUMTOOL::TMP {

/// call f.template operator()<i>(args...) for i in [begin, end)
template <int begin, int end, class F, class... Args>
constexpr void constexpr_for_range(F&& f, Args&&... args) {
  if constexpr (begin < end) {
    f.template operator()<begin>(args...);
    constexpr_for_range<begin + 1, end>(std::forward<F>(f), args...);
  }
}

/// integer sequence of [first, last] inclusive
template <class I, I first, I last>
struct make_range_sequence {};

/// run f.template operator()<value>() where value == index and value is
/// a member of the inclusive range sequence; returns f's result
template <class I, I first, I last, class F>
constexpr auto invoke_at_index(make_range_sequence<I, first, last>, I index, F&& f) {
  if constexpr (first == last) {
    return f.template operator()<first>();
  } else {
    if (index == first) return f.template operator()<first>();
    return invoke_at_index(make_range_sequence<I, first + 1, last>{}, index, std::forward<F>(f));
  }
}

constexpr int pow(int base, int exp) {
  int r = 1;
  for (int i = 0; i < exp; ++i) r *= base;
  return r;
}

}  // namespace NUMTOOL::TMP
