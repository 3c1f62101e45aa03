// Atomic basis functions shared by the device evaluator (tcscf_gpu.cu) and the host one-electron
// matrices (host_grids.cpp): the per-function record and the radial parts of the three families.
#pragma once

#include <cuda_runtime.h>
#include <cmath>

#include "../../include/tcscf_gpu.h"

namespace tcscf {

struct DevSto {
  double alpha, norm;   // radial exponent (STO, Ochi: alpha; hydrogen-like: beta = Z / n) and normalisation
  int n, l, m;
  int rtype;    // 0: m == 0, 1: cos-type (m > 0), 2: sin-type (m < 0)
  int partner;  // index of the -m function (-1 for m == 0)
  int family;   // tcscf_basis_family
};

// generalised Laguerre polynomial L_k^(a)(x) by its three-term recurrence
// (k + 1) L_(k+1) = (2k + 1 + a - x) L_k - (k + a) L_(k-1), L_0 = 1, L_1 = 1 + a - x
__host__ __device__ inline double genLaguerre(int k, double a, double x)
{
  if (k <= 0) return 1.0;
  double lm1 = 1.0, lk = 1.0 + a - x;
  for (int i = 1; i < k; ++i) {
    double const ln = ((2 * i + 1 + a - x) * lk - (i + a) * lm1) / (i + 1);
    lm1 = lk;
    lk = ln;
  }
  return lk;
}

// radial part R(r) of a basis function and dR/dr (the latter for the STO and Ochi families)
__host__ __device__ inline void basisRadial(DevSto const & s, double r, double & R, double & dR)
{
  double pw = 1.0;
  if (s.family == TCSCF_BASIS_STO) {
    for (int i = 0; i < s.n - 1; ++i) pw *= r;
    R = s.norm * pw * exp(-s.alpha * r);
    dR = ((s.n - 1) / r - s.alpha) * R;                     // SlaterTypeOrbital.hpp:71
    return;
  }
  for (int i = 0; i < s.l; ++i) pw *= r;
  double const e = exp(-s.alpha * r);
  if (s.family == TCSCF_BASIS_OCHI) {
    double const x = 2 * s.alpha * r;
    R = s.norm * pw * genLaguerre(s.n, 2 * s.l + 2, x) * e;   // OchiBasis.hpp:51-53
    // OchiBasis.hpp:64-72: (l / r - alpha) R + [n > 0] (-2 alpha) N r^l e^(-alpha r) L_(n-1)^(2l+3)(2 alpha r)
    double const dL = s.n > 0 ? -2 * s.alpha * s.norm * pw * e * genLaguerre(s.n - 1, 2 * s.l + 3, x) : 0.0;
    dR = (s.l / r - s.alpha) * R + dL;
    return;
  }
  R = s.norm * pw * genLaguerre(s.n - s.l - 1, 2 * s.l + 1, 2 * s.alpha * r) * e;   // HydrogenLikeBasis.hpp:44-47
  dR = 0.0;
}

// normalisation constant of a basis function (SlaterTypeOrbital.hpp:27-37, OchiBasis.hpp:25-32,
// HydrogenLikeBasis.hpp:22-30 with truncatedFactorial, mathFunctions.hpp:101-110)
inline double basisNormalization(tcscf_sto const & b)
{
  auto truncFact = [](int mx, int mn) { double r = 1; for (int i = mn + 1; i <= mx; ++i) r *= i; return r; };
  if (b.family == TCSCF_BASIS_OCHI) return std::pow(2 * b.alpha, b.l + 1.5) / std::sqrt(truncFact(b.n + 2 * b.l + 2, b.n));
  if (b.family == TCSCF_BASIS_HYDROGEN) {
    double const beta = b.alpha / b.n;
    return -std::pow(2 * beta, b.l + 1.5) / std::sqrt(2 * b.n * truncFact(b.n + b.l, b.n - b.l - 1));
  }
  return std::pow(2 * b.alpha, b.n) * std::sqrt(2 * b.alpha / truncFact(2 * b.n, 1));
}

}  // namespace tcscf
