// Stand-in for ZisaMemory's zisa/memory/array_view.hpp: a non-owning view
// with element access, all the reference's padding helpers
// (include/azeban/operations/copy_to_padded_functions.hpp) need.  TEST
// INFRASTRUCTURE (oracle/_ref only).
#ifndef AZ_ORACLE_ZISA_ARRAY_VIEW_HPP_
#define AZ_ORACLE_ZISA_ARRAY_VIEW_HPP_

#include <cstddef>

namespace zisa {

template <class T, int n_dims>
struct array_view {
  T *ptr = nullptr;
  T &operator[](std::size_t i) const { return ptr[i]; }
  T *raw() const { return ptr; }
};

}

#endif
