// Stand-in for ZisaCore's zisa/config.hpp (ZisaCore is fetched by the
// reference's CMake at a pinned commit, CMakeLists.txt:239-261, and is not
// part of the reference tree).  Only what the reference's pointwise headers
// use: the function qualifier and the index type.  TEST INFRASTRUCTURE: used
// only to compile those headers into oracle/_ref.
#ifndef AZ_ORACLE_ZISA_CONFIG_HPP_
#define AZ_ORACLE_ZISA_CONFIG_HPP_

#include <cstddef>

#define ANY_DEVICE_INLINE inline
#define ANY_DEVICE

namespace zisa {
using int_t = std::size_t;
}

#endif
