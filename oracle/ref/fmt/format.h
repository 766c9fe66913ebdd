// Stand-in for the declarations of the fmt library that the reference's
// include/azeban/complex.hpp names when it is not compiled by nvcc (a
// formatter specialisation, never instantiated here).  TEST INFRASTRUCTURE
// (oracle/_ref only).
#ifndef AZ_ORACLE_FMT_FORMAT_H_
#define AZ_ORACLE_FMT_FORMAT_H_

namespace fmt {
template <typename T, typename Char = char, typename Enable = void>
struct formatter;
template <typename OutputIt, typename... Args>
OutputIt format_to(OutputIt out, const char *, const Args &...) {
  return out;
}
}

#endif
