// Minimal stand-in for LvArray's multi-dimensional Array / ArrayView / ArraySlice, written for the
// oracle's reference build (test infrastructure): it lets the reference's own hot-path templates
// (HartreeFock.hpp, HartreeFock.cpp, integration/*.hpp) compile and run on the host unchanged.
//
// The semantics kept are the ones those sources rely on:
//   * a view is a shallow handle: copies (for example a lambda's [=] capture) share the data, and its
//     element access and zero() are const members that return / write mutable elements;
//   * Array<T, N, PERM> owns its data, is a view of itself (derived from ArrayView<T, N, USD>), and lays
//     dimensions out in the order of the permutation PERM, the last one with unit stride (USD);
//   * operator[] drops the leading dimension and gives ArraySlice<T, N - 1, USD - 1> (so the unit-stride
//     index deduced by the reference's templates is LvArray's); a 1-D slice or view gives T &;
//   * T -> T const conversions of views and slices, and view -> slice conversions, are implicit.
// Storage is value-initialised (zeros), as LvArray's is for arithmetic and complex types.
#pragma once

#include <algorithm>
#include <array>
#include <complex>
#include <iterator>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#include "Macros.hpp"
#include "RAJA/RAJA.hpp"

namespace LvArray {

enum class MemorySpace { undefined, host, cuda, hip };

template <typename T>
class ChaiBuffer {};

namespace typeManipulation {

// std::array-like fixed-size array
template <typename T, camp::idx_t N>
struct CArray {
  using value_type = T;
  constexpr T & operator[](camp::idx_t i) { return data[i]; }
  constexpr T const & operator[](camp::idx_t i) const { return data[i]; }
  static constexpr camp::idx_t size() { return N; }
  T data[N > 0 ? N : 1] {};
};

// f applied to each element of a tuple, in order
template <typename F, typename TUPLE>
void forEachInTuple(F && f, TUPLE && t)
{
  std::apply([&](auto &&... x) { (f(x), ...); }, std::forward<TUPLE>(t));
}

}  // namespace typeManipulation

namespace internal {
template <typename PERM>
struct PermInfo;
template <camp::idx_t... I>
struct PermInfo<camp::idx_seq<I...>> {
  static constexpr int ndim = sizeof...(I);
  static constexpr std::array<camp::idx_t, sizeof...(I)> order {I...};
  static constexpr int usd = int(order[sizeof...(I) - 1]);
};
}  // namespace internal

template <typename T, int NDIM, int USD, typename INDEX>
class ArraySlice {
 public:
  using ValueType = T;
  ArraySlice(T * data, INDEX const * dims, INDEX const * strides) : m_data(data), m_dims(dims), m_strides(strides) {}

  template <typename U = T, std::enable_if_t<!std::is_const<U>::value, int> = 0>
  operator ArraySlice<T const, NDIM, USD, INDEX>() const
  {
    return ArraySlice<T const, NDIM, USD, INDEX>(m_data, m_dims, m_strides);
  }
  ArraySlice<T const, NDIM, USD, INDEX> toSliceConst() const { return ArraySlice<T const, NDIM, USD, INDEX>(m_data, m_dims, m_strides); }
  ArraySlice toSlice() const { return *this; }

  INDEX size() const
  {
    INDEX n = 1;
    for (int d = 0; d < NDIM; ++d) n *= m_dims[d];
    return n;
  }
  INDEX size(int d) const { return m_dims[d]; }
  bool empty() const { return size() == 0; }
  T * data() const { return m_data; }

  // iteration over a 1-D slice, in index order
  struct Iterator {
    T * p;
    INDEX stride;
    T & operator*() const { return *p; }
    Iterator & operator++()
    {
      p += stride;
      return *this;
    }
    Iterator operator++(int)
    {
      Iterator const r = *this;
      p += stride;
      return r;
    }
    Iterator & operator--()
    {
      p -= stride;
      return *this;
    }
    Iterator operator+(std::ptrdiff_t k) const { return Iterator {p + k * stride, stride}; }
    Iterator operator-(std::ptrdiff_t k) const { return Iterator {p - k * stride, stride}; }
    std::ptrdiff_t operator-(Iterator const & o) const { return (p - o.p) / stride; }
    Iterator & operator+=(std::ptrdiff_t k)
    {
      p += k * stride;
      return *this;
    }
    Iterator & operator-=(std::ptrdiff_t k)
    {
      p -= k * stride;
      return *this;
    }
    T & operator[](std::ptrdiff_t k) const { return p[k * stride]; }
    bool operator==(Iterator const & o) const { return p == o.p; }
    bool operator!=(Iterator const & o) const { return p != o.p; }
    bool operator<(Iterator const & o) const { return p < o.p; }
    bool operator>(Iterator const & o) const { return p > o.p; }
    bool operator<=(Iterator const & o) const { return p <= o.p; }
    bool operator>=(Iterator const & o) const { return p >= o.p; }
    using iterator_category = std::random_access_iterator_tag;
    using value_type = std::remove_const_t<T>;
    using difference_type = std::ptrdiff_t;
    using pointer = T *;
    using reference = T &;
  };
  Iterator begin() const
  {
    static_assert(NDIM == 1, "iteration over 1-D slices");
    return Iterator {m_data, m_strides[0]};
  }
  Iterator end() const
  {
    static_assert(NDIM == 1, "iteration over 1-D slices");
    return Iterator {m_data + m_dims[0] * m_strides[0], m_strides[0]};
  }

  decltype(auto) operator[](INDEX i) const
  {
    if constexpr (NDIM == 1) {
      return (m_data[i * m_strides[0]]);
    } else {
      return ArraySlice<T, NDIM - 1, USD - 1, INDEX>(m_data + i * m_strides[0], m_dims + 1, m_strides + 1);
    }
  }

  template <typename... I>
  T & operator()(I... idx) const
  {
    static_assert(sizeof...(I) == NDIM, "wrong number of indices");
    INDEX const ii[] = {INDEX(idx)...};
    INDEX off = 0;
    for (int d = 0; d < NDIM; ++d) off += ii[d] * m_strides[d];
    return m_data[off];
  }

 private:
  T * m_data;
  INDEX const * m_dims;
  INDEX const * m_strides;
};

template <typename T, int NDIM, int USD, typename INDEX, template <typename> class BUFFER>
class ArrayView {
 public:
  using ValueType = T;
  using NonConst = std::remove_const_t<T>;

  ArrayView() = default;

  template <typename U = T, std::enable_if_t<!std::is_const<U>::value, int> = 0>
  operator ArrayView<T const, NDIM, USD, INDEX, BUFFER>() const
  {
    return toViewConst();
  }
  operator ArraySlice<T, NDIM, USD, INDEX>() const { return toSlice(); }
  template <typename U = T, std::enable_if_t<!std::is_const<U>::value, int> = 0>
  operator ArraySlice<T const, NDIM, USD, INDEX>() const
  {
    return toSliceConst();
  }

  ArrayView<T, NDIM, USD, INDEX, BUFFER> toView() const { return ArrayView<T, NDIM, USD, INDEX, BUFFER>(*this, 0); }
  ArrayView<T const, NDIM, USD, INDEX, BUFFER> toViewConst() const
  {
    ArrayView<T const, NDIM, USD, INDEX, BUFFER> v;
    v.assignFrom(m_store, m_data, m_dims, m_strides);
    return v;
  }
  ArraySlice<T, NDIM, USD, INDEX> toSlice() const { return ArraySlice<T, NDIM, USD, INDEX>(m_data, m_dims, m_strides); }
  ArraySlice<T const, NDIM, USD, INDEX> toSliceConst() const { return ArraySlice<T const, NDIM, USD, INDEX>(m_data, m_dims, m_strides); }

  INDEX size() const
  {
    INDEX n = 1;
    for (int d = 0; d < NDIM; ++d) n *= m_dims[d];
    return n;
  }
  INDEX size(int d) const { return m_dims[d]; }
  bool empty() const { return size() == 0; }
  T * data() const { return m_data; }
  T * begin() const { return m_data; }
  T * end() const { return m_data + size(); }

  decltype(auto) operator[](INDEX i) const
  {
    if constexpr (NDIM == 1) {
      return (m_data[i * m_strides[0]]);
    } else {
      return ArraySlice<T, NDIM - 1, USD - 1, INDEX>(m_data + i * m_strides[0], m_dims + 1, m_strides + 1);
    }
  }

  template <typename... I>
  T & operator()(I... idx) const
  {
    static_assert(sizeof...(I) == NDIM, "wrong number of indices");
    INDEX const ii[] = {INDEX(idx)...};
    INDEX off = 0;
    for (int d = 0; d < NDIM; ++d) off += ii[d] * m_strides[d];
    return m_data[off];
  }

  // every element (the storage is contiguous whatever the permutation)
  void zero() const
  {
    static_assert(!std::is_const<T>::value, "zero() of a const view");
    std::fill(m_data, m_data + size(), T {});
  }
  template <typename POLICY>
  void setValues(T const & v) const
  {
    std::fill(m_data, m_data + size(), v);
  }
  void move(MemorySpace, bool = true) const {}
  void registerTouch(MemorySpace) const {}

  // the raw state (for the const conversion and Array)
  void assignFrom(std::shared_ptr<std::vector<NonConst>> const & store, T * data, INDEX const * dims, INDEX const * strides)
  {
    m_store = store;
    m_data = data;
    std::copy(dims, dims + NDIM, m_dims);
    std::copy(strides, strides + NDIM, m_strides);
  }

 protected:
  ArrayView(ArrayView const & o, int) : m_store(o.m_store), m_data(o.m_data)
  {
    std::copy(o.m_dims, o.m_dims + NDIM, m_dims);
    std::copy(o.m_strides, o.m_strides + NDIM, m_strides);
  }

  std::shared_ptr<std::vector<NonConst>> m_store;
  T * m_data = nullptr;
  INDEX m_dims[NDIM] = {};
  INDEX m_strides[NDIM] = {};

  template <typename, int, int, typename, template <typename> class>
  friend class ArrayView;
};

template <typename T, int NDIM, typename PERM, typename INDEX, template <typename> class BUFFER>
class Array : public ArrayView<T, NDIM, internal::PermInfo<PERM>::usd, INDEX, BUFFER> {
  using Base = ArrayView<T, NDIM, internal::PermInfo<PERM>::usd, INDEX, BUFFER>;
  static_assert(internal::PermInfo<PERM>::ndim == NDIM, "permutation rank");

 public:
  Array() { allocate(std::array<INDEX, NDIM> {}); }
  template <typename... D, std::enable_if_t<sizeof...(D) == NDIM && (std::is_integral<D>::value && ...), int> = 0>
  explicit Array(D... dims)
  {
    allocate(std::array<INDEX, NDIM> {INDEX(dims)...});
  }
  Array(Array const & o) : Base()
  {
    allocate(dimsOf(o));
    std::copy(o.m_data, o.m_data + o.size(), this->m_data);
  }
  Array(Array && o) noexcept = default;
  Array & operator=(Array const & o)
  {
    if (this != &o) {
      allocate(dimsOf(o));
      std::copy(o.m_data, o.m_data + o.size(), this->m_data);
    }
    return *this;
  }
  Array & operator=(Array && o) noexcept = default;

  template <typename... D>
  void resize(D... dims)
  {
    static_assert(sizeof...(D) == NDIM, "resize takes every dimension");
    allocate(std::array<INDEX, NDIM> {INDEX(dims)...});
  }

 private:
  static std::array<INDEX, NDIM> dimsOf(Array const & o)
  {
    std::array<INDEX, NDIM> d;
    for (int i = 0; i < NDIM; ++i) d[i] = o.size(i);
    return d;
  }
  void allocate(std::array<INDEX, NDIM> const & dims)
  {
    INDEX n = 1;
    for (int d = 0; d < NDIM; ++d) n *= dims[d];
    auto store = std::make_shared<std::vector<std::remove_const_t<T>>>(size_t(n));
    // strides: the permutation's last dimension has unit stride, the one before it the next, ...
    INDEX strides[NDIM];
    INDEX s = 1;
    for (int k = NDIM - 1; k >= 0; --k) {
      int const d = int(internal::PermInfo<PERM>::order[k]);
      strides[d] = s;
      s *= dims[d];
    }
    this->assignFrom(store, store->data(), dims.data(), strides);
  }
};

}  // namespace LvArray
