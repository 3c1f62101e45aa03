// Minimal stand-in for RAJA as the reference's hot-path sources use it: execution-policy tags, forall
// over a typed range (OpenMP parallel for the omp_parallel_for_exec policy, as RAJA runs it, and in
// index order otherwise), atomics, and reducers that the copies captured by value in a loop body share
// (thread-safe), and the permutation tags of LvArray arrays.
#pragma once

#include <cstddef>
#include <memory>
#include <mutex>
#include <type_traits>
#include <utility>

namespace camp {
using idx_t = std::ptrdiff_t;
template <idx_t... I>
struct idx_seq {
  static constexpr int size = sizeof...(I);
};
namespace detail {
template <idx_t N, idx_t... I>
struct makeSeq : makeSeq<N - 1, N - 1, I...> {};
template <idx_t... I>
struct makeSeq<0, I...> {
  using type = idx_seq<I...>;
};
}  // namespace detail
template <idx_t N>
using make_idx_seq_t = typename detail::makeSeq<N>::type;
}  // namespace camp

namespace RAJA {
using PERM_I = camp::idx_seq<0>;
using PERM_IJ = camp::idx_seq<0, 1>;
using PERM_JI = camp::idx_seq<1, 0>;
using PERM_IJK = camp::idx_seq<0, 1, 2>;
using PERM_IKJ = camp::idx_seq<0, 2, 1>;
using PERM_JIK = camp::idx_seq<1, 0, 2>;
using PERM_JKI = camp::idx_seq<1, 2, 0>;
using PERM_KIJ = camp::idx_seq<2, 0, 1>;
using PERM_KJI = camp::idx_seq<2, 1, 0>;
using PERM_IJKL = camp::idx_seq<0, 1, 2, 3>;

struct loop_exec {};
struct seq_exec {};
struct omp_parallel_for_exec {};
template <int BLOCK = 256>
struct cuda_exec {};
template <int BLOCK = 256>
struct cuda_exec_async {};
struct seq_atomic {};
struct builtin_atomic {};
struct cuda_atomic {};
struct seq_reduce {};
struct omp_reduce {};
struct cuda_reduce {};
namespace resources {
struct Host {};
struct Cuda {};
}  // namespace resources

template <typename INDEX>
struct TypedRangeSegment {
  TypedRangeSegment(INDEX b, INDEX e) : begin(b), end(e) {}
  INDEX begin, end;
};

template <typename POLICY, typename INDEX, typename BODY>
void forall(TypedRangeSegment<INDEX> const & seg, BODY && body)
{
  if constexpr (std::is_same_v<POLICY, omp_parallel_for_exec>) {
#pragma omp parallel for schedule(dynamic, 1)
    for (INDEX i = seg.begin; i < seg.end; ++i) body(i);
  } else {
    for (INDEX i = seg.begin; i < seg.end; ++i) body(i);
  }
}

template <typename POLICY, typename T, typename U>
T atomicAdd(T * ptr, U const & value)
{
  T old;
#pragma omp atomic capture
  {
    old = *ptr;
    *ptr += value;
  }
  return old;
}

namespace detail {
template <typename T>
struct Shared {
  explicit Shared(T v) : value(v) {}
  T value;
  std::mutex lock;
};
}  // namespace detail

template <typename REDUCE, typename T>
class ReduceSum {
 public:
  explicit ReduceSum(T init) : m_s(std::make_shared<detail::Shared<T>>(init)) {}
  ReduceSum const & operator+=(T const & v) const
  {
    std::lock_guard<std::mutex> g(m_s->lock);
    m_s->value += v;
    return *this;
  }
  T get() const { return m_s->value; }
  operator T() const { return m_s->value; }

 private:
  std::shared_ptr<detail::Shared<T>> m_s;
};

template <typename REDUCE, typename T>
class ReduceMax {
 public:
  explicit ReduceMax(T init) : m_s(std::make_shared<detail::Shared<T>>(init)) {}
  ReduceMax const & max(T const & v) const
  {
    std::lock_guard<std::mutex> g(m_s->lock);
    if (v > m_s->value) m_s->value = v;
    return *this;
  }
  T get() const { return m_s->value; }

 private:
  std::shared_ptr<detail::Shared<T>> m_s;
};

template <typename REDUCE, typename T>
class ReduceMin {
 public:
  explicit ReduceMin(T init) : m_s(std::make_shared<detail::Shared<T>>(init)) {}
  ReduceMin const & min(T const & v) const
  {
    std::lock_guard<std::mutex> g(m_s->lock);
    if (v < m_s->value) m_s->value = v;
    return *this;
  }
  T get() const { return m_s->value; }

 private:
  std::shared_ptr<detail::Shared<T>> m_s;
};
}  // namespace RAJA
