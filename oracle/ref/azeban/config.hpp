// What the reference's CMake writes from include/azeban/config.hpp.in for a
// double-precision build (FP_PRECISION = double, the CMake default,
// CMakeLists.txt:19,35-39).  The reference's own headers are included from
// the reference tree, unmodified.  TEST INFRASTRUCTURE (oracle/_ref only).
#ifndef AZ_ORACLE_AZEBAN_CONFIG_HPP_
#define AZ_ORACLE_AZEBAN_CONFIG_HPP_

#include <azeban/complex.hpp>
#include <zisa/config.hpp>

namespace azeban {

using zisa::int_t;
using real_t = double;
using complex_t = Complex<real_t>;

}

#endif
