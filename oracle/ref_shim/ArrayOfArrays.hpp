// Minimal stand-in for LvArray's ArrayOfArrays (a list of variable-length arrays), as the reference's
// QMC point cache uses it (oracle reference build, test infrastructure).
#pragma once

#include <vector>

#include "Array.hpp"

namespace LvArray {

template <typename T, typename INDEX, template <typename> class BUFFER>
class ArrayOfArrays {
 public:
  ArrayOfArrays(INDEX nArrays = 0, INDEX capacity = 0) : m_arrays(size_t(nArrays))
  {
    for (auto & a : m_arrays) a.reserve(size_t(capacity));
  }
  INDEX size() const { return INDEX(m_arrays.size()); }
  INDEX sizeOfArray(INDEX i) const { return INDEX(m_arrays[size_t(i)].size()); }
  template <typename ATOMIC, typename... ARGS>
  void emplaceBackAtomic(INDEX i, ARGS &&... args)
  {
    m_arrays[size_t(i)].emplace_back(std::forward<ARGS>(args)...);
  }
  template <typename... ARGS>
  void emplaceBack(INDEX i, ARGS &&... args)
  {
    m_arrays[size_t(i)].emplace_back(std::forward<ARGS>(args)...);
  }
  T const & operator()(INDEX i, INDEX j) const { return m_arrays[size_t(i)][size_t(j)]; }
  T & operator()(INDEX i, INDEX j) { return m_arrays[size_t(i)][size_t(j)]; }

 private:
  std::vector<std::vector<T>> m_arrays;
};

template <typename T, typename INDEX, bool CONST_SIZES, template <typename> class BUFFER>
class ArrayOfArraysView;

}  // namespace LvArray
