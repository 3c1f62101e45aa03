// Minimal stand-in for LvArray::memcpy as the reference calls it: a whole-array copy (no index prefix
// on either side) between two 2-D views of the same shape, element by element so that the two layouts
// may differ (oracle reference build, test infrastructure).
#pragma once

#include <array>

#include "Array.hpp"

namespace LvArray {

template <int N_DST_INDICES, int N_SRC_INDICES, typename DST, typename SRC>
void memcpy(DST const & dst, std::array<std::ptrdiff_t, N_DST_INDICES> const &, SRC const & src,
            std::array<std::ptrdiff_t, N_SRC_INDICES> const &)
{
  static_assert(N_DST_INDICES == 0 && N_SRC_INDICES == 0, "only whole-array copies");
  LVARRAY_ERROR_IF_NE(dst.size(), src.size());
  for (std::ptrdiff_t i = 0; i < dst.size(0); ++i)
    for (std::ptrdiff_t j = 0; j < dst.size(1); ++j) dst(i, j) = src(i, j);
}

}  // namespace LvArray
