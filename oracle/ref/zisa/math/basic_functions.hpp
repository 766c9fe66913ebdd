// Stand-in for ZisaCore's zisa/math/basic_functions.hpp: the scalar helpers
// the reference's pointwise headers call, as the C++ standard library gives
// them; pow<n> is the integer power by repeated multiplication.  TEST
// INFRASTRUCTURE (oracle/_ref only).
#ifndef AZ_ORACLE_ZISA_BASIC_FUNCTIONS_HPP_
#define AZ_ORACLE_ZISA_BASIC_FUNCTIONS_HPP_

#include <algorithm>
#include <cmath>

namespace zisa {

constexpr double pi = 3.14159265358979323846;

template <class T> inline T sqrt(const T &x) { return std::sqrt(x); }
template <class T> inline T abs(const T &x) { return std::abs(x); }
template <class T> inline T exp(const T &x) { return std::exp(x); }
template <class T, class U> inline auto pow(const T &x, const U &y) { return std::pow(x, y); }
template <int n, class T> inline T pow(const T &x) {
  if constexpr (n == 0) {
    return T(1);
  } else {
    return x * pow<n - 1>(x);
  }
}
template <class T> inline T atan2(const T &y, const T &x) { return std::atan2(y, x); }
template <class T> inline T max(const T &a, const T &b) { return std::max(a, b); }
template <class T> inline T min(const T &a, const T &b) { return std::min(a, b); }

}

#endif
