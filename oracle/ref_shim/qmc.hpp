// Stand-in for the interface of the mppmu/qmc integrator (an un-vendored submodule of the reference)
// as the reference's QMC point cache drives it.  The points it hands out are the caller's unit-cube
// points when the oracle's reference build has provided some (providedPoints(), one vector of M
// coordinates per point, each handed out once), so that the reference's QMCGrid maps exactly the
// oracle's inputs; otherwise a plain centred lattice (grids whose points, weights and basis values
// the build then replaces with the oracle's).
#pragma once

#include <cstdint>
#include <vector>

namespace integrators {
inline std::vector<std::vector<double>> & providedPoints()
{
  static std::vector<std::vector<double>> points;
  return points;
}

namespace transforms {
struct None {
  template <typename I, typename D, unsigned long long M>
  struct type {};
};
}  // namespace transforms

template <typename T, typename D, unsigned int M, template <typename, typename, unsigned long long> class P>
class Qmc {
 public:
  using U = unsigned long long;
  struct result {
    T integral;
    T error;
    U n;
    U m;
    U iterations;
    U evaluations;
  };
  U maxeval = 1;
  U minn = 1;
  U minm = 1;
  U get_next_n(U n) const { return n; }
  template <typename F>
  result integrate(F & f) const
  {
    T sum {};
    D x[M];
    std::vector<std::vector<double>> const & given = providedPoints();
    if (!given.empty()) {
      for (auto const & q : given) {
        for (unsigned int d = 0; d < M; ++d) x[d] = D(q[d]);
        sum += f(x);
      }
      U const k = U(given.size());
      return result {sum / T(k), T {}, k, 1, 1, k};
    }
    U const n = get_next_n(minn);
    for (U s = 0; s < minm; ++s)
      for (U i = 0; i < n; ++i) {
        for (unsigned int d = 0; d < M; ++d) x[d] = (D(i) + D(0.5)) / D(n);
        sum += f(x);
      }
    return result {sum / T(n * minm), T {}, n, minm, 1, n * minm};
  }
};
}  // namespace integrators
