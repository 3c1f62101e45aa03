// Host-side grid generation of libtcscf_gpu.so (negligible work, no device involvement):
// Chebyshev-Gauss radial rules with the reference's changes of variables, radial x angular product
// grids, the QMCGrid point mapping and a seeded scrambled Sobol point source.
#include <algorithm>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <string>
#include <unordered_set>
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/tcscf_gpu.h"
#include "basis.cuh"

namespace {
constexpr double kPi = 3.141592653589793238462643383279502884;

uint64_t splitmix64(uint64_t & s)
{
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Sobol direction numbers (32 bits) for the first three dimensions: dimension 1 is the van der
// Corput sequence; dimensions 2 and 3 use the primitive polynomials x+1 (m1 = 1) and x^2+x+1
// (m1 = 1, m2 = 3) with the Bratley-Fox recurrence.
void directionNumbers(int dim, uint32_t v[32])
{
  if (dim == 0) { for (int k = 0; k < 32; ++k) v[k] = 1u << (31 - k); return; }
  uint32_t m[33];
  int s;
  if (dim == 1) { s = 1; m[1] = 1; }
  else { s = 2; m[1] = 1; m[2] = 3; }
  for (int k = s + 1; k <= 32; ++k) {
    if (s == 1) m[k] = (2u * m[k - 1]) ^ m[k - 1];
    else m[k] = (2u * m[k - 1]) ^ (4u * m[k - 2]) ^ m[k - 2];
  }
  for (int k = 1; k <= 32; ++k) v[k - 1] = m[k] << (32 - k);
}
// Ochi and hydrogen-like one-electron matrices (tcscf_overlap_core_analytic).  Radial integrals use
// the reference driver's core grid: 1000-point Chebyshev-Gauss with the Treutler-Ahlrichs M4 map,
// a = 1, eps = 0.9 (HartreeFockTest.cpp:364-367).
int overlapCoreLaguerre(const tcscf_sto * basis, int nb, int Z, double * S, double * H)
{
  int const nr = 1000;
  std::vector<double> r(nr), w(nr);
  tcscf_grid_radial(nr, TCSCF_MAP_TREUTLER_AHLRICHS_M4, 1.0, 0.9, r.data(), w.data());
  std::vector<tcscf::DevSto> d(nb);
  std::vector<double> R(size_t(nb) * nr);
  for (int b = 0; b < nb; ++b) {
    tcscf_sto const & s = basis[b];
    if (s.n < (s.family == TCSCF_BASIS_OCHI ? 0 : 1) || s.l < std::abs(s.m) || !(s.alpha > 0)) return TCSCF_ERR_INVALID_ARGUMENT;
    if (s.family == TCSCF_BASIS_HYDROGEN && s.l >= s.n) return TCSCF_ERR_INVALID_ARGUMENT;
    d[b].alpha = s.family == TCSCF_BASIS_HYDROGEN ? s.alpha / s.n : s.alpha;
    d[b].norm = tcscf::basisNormalization(s);
    d[b].n = s.n; d[b].l = s.l; d[b].m = s.m; d[b].family = s.family;
    for (int k = 0; k < nr; ++k) {
      double dR = 0;
      tcscf::basisRadial(d[b], r[k], R[size_t(b) * nr + k], dR);
    }
  }
  for (int i = 0; i < nb; ++i)
    for (int j = 0; j < nb; ++j) {
      tcscf_sto const & b1 = basis[i];
      tcscf_sto const & b2 = basis[j];
      bool const lm = b1.l == b2.l && b1.m == b2.m;
      double s = 0, h = 0;
      if (b1.family == TCSCF_BASIS_OCHI) {
        // OchiBasis.hpp:118-125: orthonormal by construction, whatever the exponents
        s = (b1.n == b2.n && lm) ? 1.0 : 0.0;
        if (H) {
          // OchiBasis.hpp:130-155
          if (b1.alpha != b2.alpha) return TCSCF_ERR_INVALID_ARGUMENT;
          if (lm) {
            double integral = 0;   // sum_k w fnl1 fnl2 / r with fnl = R r
            for (int k = 0; k < nr; ++k) integral += w[k] * R[size_t(i) * nr + k] * r[k] * R[size_t(j) * nr + k];
            double const a = b1.alpha;
            double const coeff = a * (b1.l + 1) * (1 + 2 * std::min(b1.n, b2.n) / double(2 * b1.l + 3)) - Z;
            h = coeff * integral - (b1.n == b2.n) * a * a / 2;
          }
        }
      } else {
        // the generic overlap (AtomicBasis.hpp:19-31) reduces to the radial integral of R1 R2 r^2
        if (lm) {
          double integral = 0;
          for (int k = 0; k < nr; ++k) integral += w[k] * R[size_t(i) * nr + k] * R[size_t(j) * nr + k] * r[k] * r[k];
          s = integral;
        }
        // HydrogenLikeBasis.hpp:70-82
        if (b1.n == b2.n && lm) h = -double(Z) * Z / (2.0 * b1.n * b1.n);
      }
      if (S) S[i * nb + j] = s;
      if (H) H[i * nb + j] = h;
    }
  return TCSCF_OK;
}

}  // namespace

extern "C" {

int tcscf_grid_radial(int n, int map, double p0, double p1, double * u, double * w)
{
  if (n <= 0 || !u || !w || map < 0 || map > 4) return TCSCF_ERR_INVALID_ARGUMENT;
  // ChebyshevGauss (ChebyshevGauss.hpp:9-49): x_i = cos(theta_i), weight sin(theta_i),
  // theta_i = (i+1) pi/(n+1), global weight pi/(n+1); createGrid (quadrature.hpp:75-102) folds
  // point weight * jacobian * global weight.
  double const freq = kPi / (n + 1);
  for (int i = 0; i < n; ++i) {
    double const th = (i + 1) * freq;
    double const x = std::cos(th), wt = std::sin(th);
    double uu = x, jac = 1;
    switch (map) {
      case TCSCF_MAP_LINEAR: uu = p0 * x; jac = p0; break;
      case TCSCF_MAP_X_OVER_1MX: uu = x / (1 - x); jac = std::pow(1 - x, -2); break;
      case TCSCF_MAP_TREUTLER_AHLRICHS_M4: {
        // changeOfVariables.hpp:266-303
        double const eol = p1 / std::log(2.0), alpha = 0.6;
        double const logPart = std::log((1 + p0) / (1 - x));
        double const xa1 = std::pow(x + p0, alpha - 1), xa = xa1 * (x + p0);
        uu = eol * std::pow(x + p0, alpha) * logPart;
        jac = eol * (alpha * xa1 * logPart + xa / (1 - x));
        break;
      }
      case TCSCF_MAP_ONE_PLUS_X: uu = (1 + x) / (1 - x); jac = 2 / ((1 - x) * (1 - x)); break;
      default: break;
    }
    u[i] = uu;
    w[i] = wt * jac * freq;
  }
  return TCSCF_OK;
}

int tcscf_grid_product(int nrad, const double * r, const double * wr, int nang, const double * ang, double * pts, double * w)
{
  if (nrad <= 0 || nang <= 0 || !r || !wr || !ang || !pts || !w) return TCSCF_ERR_INVALID_ARGUMENT;
  int64_t const N = int64_t(nrad) * nang;
  for (int ir = 0; ir < nrad; ++ir)
    for (int ia = 0; ia < nang; ++ia) {
      int64_t const i = int64_t(ir) * nang + ia;
      double const th = ang[3 * ia], ph = ang[3 * ia + 1];
      double const st = std::sin(th), ct = std::cos(th), sp = std::sin(ph), cp = std::cos(ph);
      pts[i] = r[ir] * cp * st;  // Spherical::toCartesian (mathFunctions.hpp:202-211)
      pts[N + i] = r[ir] * sp * st;
      pts[2 * N + i] = r[ir] * ct;
      w[i] = wr[ir] * r[ir] * r[ir] * ang[3 * ia + 2];
    }
  return TCSCF_OK;
}

int tcscf_grid_qmc(int ndim, int64_t n, const double * u, double * pts, double * w)
{
  if ((ndim != 2 && ndim != 3) || n <= 0 || !u || !pts || !w) return TCSCF_ERR_INVALID_ARGUMENT;
  double const eol = 0.9 / std::log(2.0), alpha = 0.6;
  for (int64_t i = 0; i < n; ++i) {
    double const x0 = u[i], x1 = u[n + i];
    double const logPart = std::log(1.0 / (1 - x0));
    double const xa1 = std::pow(x0, alpha - 1), xa = xa1 * x0;
    double const r = eol * std::pow(x0, alpha) * logPart;
    double jac = eol * (alpha * xa1 * logPart + xa / (1 - x0));
    double const th = std::acos(1 - 2 * x1);
    jac *= 1 / std::sqrt(x1 * (1 - x1));
    double ph = 0;
    if (ndim == 3) { ph = 2 * kPi * u[2 * n + i]; jac *= 2 * kPi; }
    double const st = std::sin(th), ct = std::cos(th);
    if (ndim == 2) { pts[i] = r * std::cos(ph) * st; pts[n + i] = r * ct; }
    else { pts[i] = r * std::cos(ph) * st; pts[n + i] = r * std::sin(ph) * st; pts[2 * n + i] = r * ct; }
    w[i] = jac * (1.0 / double(n)) * r * r * st;
  }
  return TCSCF_OK;
}

int tcscf_sobol(int ndim, int64_t n, uint64_t seed, double * u)
{
  if (ndim < 1 || ndim > 3 || n <= 0 || n > (int64_t(1) << 32) || !u) return TCSCF_ERR_INVALID_ARGUMENT;
  uint64_t st = seed;
  for (int d = 0; d < ndim; ++d) {
    uint32_t v[32];
    directionNumbers(d, v);
    // linear matrix scrambling: random lower-triangular binary matrix (digits ordered from the most
    // significant) with unit diagonal applied to every direction number, then a random digital
    // shift.  Output digit r depends on input digits 0..r only, which keeps the net property.
    uint32_t L[32];
    for (int r = 0; r < 32; ++r) {
      uint32_t const bits = uint32_t(splitmix64(st));
      uint32_t const above = r == 0 ? 0u : (bits & ~((1u << (32 - r)) - 1u));
      L[r] = (1u << (31 - r)) | above;  // row r: diagonal bit (31-r) plus random more-significant bits
    }
    uint32_t sv[32];
    for (int k = 0; k < 32; ++k) {
      uint32_t out = 0;
      for (int r = 0; r < 32; ++r) {
        // output bit (31-r) = parity(L[r] & v[k])
        uint32_t const x = L[r] & v[k];
        out |= uint32_t(__builtin_parity(x)) << (31 - r);
      }
      sv[k] = out;
    }
    uint32_t const shift = uint32_t(splitmix64(st));
    for (int64_t i = 0; i < n; ++i) {
      uint64_t const g = uint64_t(i) ^ (uint64_t(i) >> 1);
      uint32_t x = 0;
      for (int k = 0; k < 32; ++k) if ((g >> k) & 1u) x ^= sv[k];
      x ^= shift;
      u[int64_t(d) * n + i] = (double(x) + 0.5) * (1.0 / 4294967296.0);
    }
  }
  return TCSCF_OK;
}

int tcscf_overlap_core_analytic(const tcscf_sto * basis, int nb, int Z, double * S, double * H)
{
  if (!basis || nb <= 0 || (!S && !H)) return TCSCF_ERR_INVALID_ARGUMENT;
  int const family = basis[0].family;
  for (int i = 0; i < nb; ++i)
    if (basis[i].family != family || family < TCSCF_BASIS_STO || family > TCSCF_BASIS_HYDROGEN) return TCSCF_ERR_INVALID_ARGUMENT;
  if (family != TCSCF_BASIS_STO) return overlapCoreLaguerre(basis, nb, Z, S, H);
  auto fact = [](int k) { double r = 1; for (int i = 2; i <= k; ++i) r *= i; return r; };
  auto nrm = [&](tcscf_sto const & b) { return std::pow(2 * b.alpha, b.n) * std::sqrt(2 * b.alpha / fact(2 * b.n)); };
  auto ovl = [](int sn, double sa) { return std::tgamma(sn + 1) / std::pow(sa, sn + 1); };
  for (int i = 0; i < nb; ++i)
    for (int j = 0; j < nb; ++j) {
      tcscf_sto const & b1 = basis[i];
      tcscf_sto const & b2 = basis[j];
      double s = 0, h = 0;
      if (b1.l == b2.l && b1.m == b2.m) {
        double const n1 = nrm(b1), n2 = nrm(b2);
        // SlaterTypeOrbital.hpp:134-145 and :149-171
        s = n1 * n2 * ovl(b1.n + b2.n, b1.alpha + b2.alpha);
        int const nn = b2.n, l = b2.l, ns = b1.n + b2.n;
        double const a = b2.alpha, as = b1.alpha + b2.alpha;
        h = 0.5 * n1 * n2 * ((l * (l + 1) - nn * (nn - 1)) * ovl(ns - 2, as) + 2 * (nn * a - Z) * ovl(ns - 1, as)
                             - std::pow(a, 2) * ovl(ns, as));
      }
      if (S) S[i * nb + j] = s;
      if (H) H[i * nb + j] = h;
    }
  return TCSCF_OK;
}

// loadSTO (SlaterTypeOrbital.cpp:24-75): the BASIS block of <directory>/<basisSet>/<element>, one
// "<n><S|P|D|F> <alpha>" entry per line up to END, each expanded over m = -l..l, entries above maxL
// skipped.  out may be null (count only); otherwise at most capacity functions are written and
// *count is the total.  The reference aborts on an unknown basis set, a missing basis-set directory or
// an unparsable line: those return TCSCF_ERR_INVALID_ARGUMENT here.  A missing element file gives
// an empty basis, as the reference's (its existence check is disabled).
int tcscf_load_sto(const char * directory, const char * basisSet, const char * element, int maxL, tcscf_sto * out, int capacity,
                   int * count)
{
  if (!directory || !basisSet || !element || !count || capacity < 0) return TCSCF_ERR_INVALID_ARGUMENT;
  static std::unordered_set<std::string> const valid = {"TZ3P", "QZ6P", "ATZ3P", "AQZ6P"};
  if (!valid.count(basisSet)) return TCSCF_ERR_INVALID_ARGUMENT;
  std::filesystem::path const dir = std::filesystem::path(directory) / basisSet;
  std::error_code ec;
  if (!std::filesystem::is_directory(dir, ec)) return TCSCF_ERR_INVALID_ARGUMENT;
  std::ifstream contents(dir / element);
  int total = 0;
  for (std::string line; std::getline(contents, line);) {
    if (line.rfind("BASIS", 0) != 0) continue;
    while (std::getline(contents, line) && line.rfind("END", 0) != 0) {
      int n;
      char type;
      double alpha;
      std::istringstream ls(line);
      if (ls >> n >> type >> alpha) {
        int const l = type == 'S' ? 0 : type == 'P' ? 1 : type == 'D' ? 2 : type == 'F' ? 3 : -1;
        if (l < 0) return TCSCF_ERR_INVALID_ARGUMENT;   // spdfToL, SlaterTypeOrbital.cpp:11-21
        if (l > maxL) continue;
        for (int m = -l; m <= l; ++m) {
          if (out && total < capacity) out[total] = tcscf_sto{alpha, n, l, m, TCSCF_BASIS_STO};
          ++total;
        }
      } else if (!line.empty()) {
        return TCSCF_ERR_INVALID_ARGUMENT;
      }
    }
    break;
  }
  *count = total;
  return TCSCF_OK;
}

}  // extern "C"
