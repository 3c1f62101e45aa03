// Minimal stand-ins for the LvArray math and tensorOps routines the reference's hot-path sources call
// (oracle reference build, test infrastructure).
#pragma once

#include <cmath>

#include "Array.hpp"

namespace LvArray {
namespace math {
template <typename T>
inline void sincos(T const x, T & s, T & c)
{
  s = std::sin(x);
  c = std::cos(x);
}
template <typename T>
inline T invSqrt(T const x)
{
  return T(1) / std::sqrt(x);
}
}  // namespace math

namespace tensorOps {
// v[i] *= s for i < M
template <int M, typename V, typename S>
inline void scale(V && v, S const s)
{
  for (int i = 0; i < M; ++i) v[i] *= s;
}
// v[i] += s * w[i] for i < M
template <int M, typename V, typename W, typename S>
inline void scaledAdd(V && v, W const & w, S const s)
{
  for (int i = 0; i < M; ++i) v[i] += s * w[i];
}
// sum_i a[i] b[i] for i < M
template <int M, typename A, typename B>
inline auto AiBi(A const & a, B const & b)
{
  auto r = a[0] * b[0];
  for (int i = 1; i < M; ++i) r += a[i] * b[i];
  return r;
}
}  // namespace tensorOps
}  // namespace LvArray
