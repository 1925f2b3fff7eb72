// Compatibility name of the reference header include/FloatUtils.h: the float
// comparison helpers its tests use (FloatUtils.h:40-61).
#ifndef BBKDE_COMPAT_FLOATUTILS_H
#define BBKDE_COMPAT_FLOATUTILS_H
#include <algorithm>
#include <cmath>
#include <limits>
#include <type_traits>

namespace bbrcit {

// True iff |lhs - rhs| <= abs_err or |lhs - rhs| <= rel_err * max(|lhs|, |rhs|).
template <typename T>
typename std::enable_if<!std::numeric_limits<T>::is_integer, bool>::type
approximately_equal(T lhs, T rhs, T rel_err, T abs_err = std::numeric_limits<T>::min()) {
  T diff = std::abs(lhs - rhs);
  if (diff <= abs_err) return true;
  return diff <= rel_err * std::max(std::abs(lhs), std::abs(rhs));
}

template <typename T>
typename std::enable_if<!std::numeric_limits<T>::is_integer, bool>::type
almost_equal(T lhs, T rhs) {
  return std::abs(lhs - rhs) <= std::numeric_limits<T>::epsilon() *
                                    std::max(std::abs(lhs), std::abs(rhs));
}

}  // namespace bbrcit
#endif
