// ORACLE — TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement (C++17 + OpenMP, FP64) of corbett5/tcscf's grid-quadrature Fock build, used
// only as the parity reference by tests/, __graft_entry__.smoke() and the cpu_baseline / reference arm of
// bench.py.  It is never linked into, loaded by or called from the product library
// (tcscf_b200/libtcscf_gpu.so).  Every routine cites the reference file:line it follows; loop
// orders are the reference's except where noted (a transposed basis table is used for the r2
// inner products so that the CPU baseline is not memory-latency bound; the arithmetic per term is
// unchanged).
//
// Pinned by: Chebyshev-Gauss, radial-map and Lebedev/Y_lm known answers
// (src/unitTests/IntegrationTest.cpp:19-197), STO quadrature overlap == analytic overlap to 1e-14
// (src/unitTests/SlaterTypeOrbitalTest.cpp:14-47), Ochi gradient == central finite difference to
// 1e-8 (src/unitTests/gradientsTest.cpp:59-93) and MGS orthogonality
// (src/unitTests/orthogonalizationTest.cpp:48-62); see tests/test_oracle_known_answers.py.
// The r12 contraction and SCF energies have no golden values in the reference: for those this
// restatement *is* the parity reference.
//
// Deviation (documented): every r12 kernel returns 0 for an exactly coincident pair r1 == r2
// (the reference's own r12Inv convention, src/unitTests/IntegrationTest.cpp:298-309); the
// reference's HartreeFockTest.cpp:248-253 kernel has no guard because its grids never coincide.

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <limits>
#include <dlfcn.h>
#include <omp.h>

using cplx = std::complex<double>;

namespace {

constexpr double PI = 3.141592653589793238462643383279502884;

struct Sto { double alpha; int32_t n, l, m; int32_t family; };       // == tcscf_sto (family 0 STO, 1 Ochi, 2 hydrogen-like)
struct Ochi { double a, a12; int32_t nterms, pad; int32_t S[8][3]; double c[8][2]; };  // == tcscf_ochi

struct Vec3 { double x, y, z; };
struct CVec3 { cplx x, y, z; };

// mathFunctions.hpp:88-97
double factorial(int n) { double r = 1; for (int i = 2; i <= n; ++i) r *= i; return r; }

// mathFunctions.hpp:115-139  (std::sph_legendre includes the Condon-Shortley phase)
cplx cExp(double t) { return {std::cos(t), std::sin(t)}; }
cplx sphericalHarmonic(int l, int m, double theta, double phi)
{ return std::sph_legendre(l, std::abs(m), theta) * cExp(m * phi); }

// SlaterTypeOrbital.hpp:27-37
double stoNormalization(double alpha, int n)
{ return std::pow(2 * alpha, n) * std::sqrt(2 * alpha / factorial(2 * n)); }

// mathFunctions.hpp:101-110
double truncatedFactorial(int max, int min) { double r = 1; for (int i = min + 1; i <= max; ++i) r *= i; return r; }

// OchiBasis.hpp:25-32 and HydrogenLikeBasis.hpp:22-30 (beta = Z / n)
double ochiNormalization(double alpha, int n, int l) { return std::pow(2 * alpha, l + 1.5) / std::sqrt(truncatedFactorial(n + 2 * l + 2, n)); }
double hydrogenNormalization(double Z, int n, int l)
{ return -std::pow(2 * (Z / n), l + 1.5) / std::sqrt(2 * n * truncatedFactorial(n + l, n - l - 1)); }
double basisNormalization(Sto const & b)
{
  if (b.family == 1) return ochiNormalization(b.alpha, b.n, b.l);
  if (b.family == 2) return hydrogenNormalization(b.alpha, b.n, b.l);
  return stoNormalization(b.alpha, b.n);
}

// SlaterTypeOrbital.hpp:57-58; OchiBasis.hpp:51-53; HydrogenLikeBasis.hpp:44-47 (assocLaguerre is
// std::assoc_laguerre, mathFunctions.hpp:144-148)
double radialComponent(Sto const & b, double nrm, double r)
{
  if (b.family == 1) return nrm * std::pow(r, b.l) * std::assoc_laguerre(b.n, 2 * b.l + 2, 2 * b.alpha * r) * std::exp(-b.alpha * r);
  if (b.family == 2) {
    double const beta = b.alpha / b.n;
    return nrm * std::pow(r, b.l) * std::assoc_laguerre(b.n - b.l - 1, 2 * b.l + 1, 2 * beta * r) * std::exp(-beta * r);
  }
  return nrm * std::pow(r, b.n - 1) * std::exp(-b.alpha * r);
}

// mathFunctions.hpp:240-261 (Cartesian::toSpherical)
void toSpherical(double x, double y, double z, double & r, double & th, double & ph)
{ r = std::hypot(x, y, z); th = std::acos(z / r); ph = std::atan2(y, x); }

// SlaterTypeOrbital.hpp:51-52
cplx stoValue(Sto const & b, double nrm, double r, double th, double ph)
{ return radialComponent(b, nrm, r) * sphericalHarmonic(b.l, b.m, th, ph); }

// SlaterTypeOrbital.hpp:63-106 (kept verbatim in arithmetic, including the m<0 and pole quirks)
CVec3 stoGradient(Sto const & b, double nrm, double r, double th, double ph)
{
  int const n = b.n, l = b.l, m = b.m;
  double const radial = radialComponent(b, nrm, r);
  cplx const Ylm = sphericalHarmonic(l, m, th, ph);
  double dRadialPart = ((n - 1) / r - b.alpha) * radial;
  if (b.family == 1) {
    // OchiBasis.hpp:64-72
    double const dLaguerrePart = (n > 0) * -2 * b.alpha * nrm * std::pow(r, l) * std::exp(-b.alpha * r) *
                                 (n > 0 ? std::assoc_laguerre(n - 1, 2 * l + 3, 2 * b.alpha * r) : 0.0);
    dRadialPart = (l / r - b.alpha) * radial + dLaguerrePart;
  }
  cplx const Ylmp1 = double(l != m) * std::sqrt(double((l - m) * (l + m + 1))) * cExp(-ph) * sphericalHarmonic(l, m + 1, th, ph);
  cplx const rHat = dRadialPart * Ylm;
  cplx const thetaHat = (double(m) * Ylm / std::tan(th) + Ylmp1) * radial / r;
  cplx const phiHat = cplx(0, 1) * double(m) * Ylm * radial / (r * std::sin(th));
  CVec3 a{};
  double const rx = std::cos(ph) * std::sin(th), ry = std::sin(ph) * std::sin(th), rz = std::cos(th);
  a.x += rHat * rx; a.y += rHat * ry; a.z += rHat * rz;
  double const tx = std::cos(ph) * std::cos(th), ty = std::sin(ph) * std::cos(th), tz = -std::sin(th);
  a.x += thetaHat * tx; a.y += thetaHat * ty; a.z += thetaHat * tz;
  double const px = -std::sin(ph), py = std::cos(ph), pz = 0;
  a.x += phiHat * px; a.y += phiHat * py; a.z += phiHat * pz;
  return a;
}

// SlaterTypeOrbital.hpp:125-128
double overlapNonNormalized(int sumOfN, double sumOfAlpha)
{ return std::tgamma(sumOfN + 1) / std::pow(sumOfAlpha, sumOfN + 1); }

// jastrowFunctions.hpp:14-32
double ochiValue(Ochi const & u, double r1, double r2, double r12, bool same)
{
  double const r12T = r12 / (r12 + u.a12), r1T = r1 / (r1 + u.a), r2T = r2 / (r2 + u.a);
  double res = 0;
  for (int k = 0; k < u.nterms; ++k)
    res = res + u.c[k][same] * std::pow(r12T, u.S[k][0]) * std::pow(r1T, u.S[k][1]) * std::pow(r2T, u.S[k][2]);
  return res;
}

// jastrowFunctions.hpp:72-108
Vec3 ochiGradient(Ochi const & u, Vec3 const & p1, Vec3 const & p2, bool same)
{
  Vec3 const d{p1.x - p2.x, p1.y - p2.y, p1.z - p2.z};
  double const r1 = std::hypot(p1.x, p1.y, p1.z), r2 = std::hypot(p2.x, p2.y, p2.z), r12 = std::hypot(d.x, d.y, d.z);
  double const r1T = r1 / (r1 + u.a), r2T = r2 / (r2 + u.a), r12T = r12 / (r12 + u.a12);
  double const r1Scale = u.a / (std::pow(r1, 2) * (r1 + u.a));
  double const r12Scale = u.a12 / (std::pow(r12, 2) * (r12 + u.a12));
  double r1Length = 0, r12Length = 0;
  for (int k = 0; k < u.nterms; ++k) {
    int const i = u.S[k][0], j = u.S[k][1], kk = u.S[k][2];
    double const factor = u.c[k][same] * std::pow(r12T, i) * std::pow(r1T, j) * std::pow(r2T, kk);
    r1Length += factor * j * r1Scale;
    r12Length += factor * i * r12Scale;
  }
  return {r12Length * d.x + r1Length * p1.x, r12Length * d.y + r1Length * p1.y, r12Length * d.z + r1Length * p1.z};
}

// jastrowFunctions.hpp:34-70
double ochiLaplacian(Ochi const & u, Vec3 const & p1, Vec3 const & p2, bool same)
{
  Vec3 const d{p1.x - p2.x, p1.y - p2.y, p1.z - p2.z};
  double const r1 = std::hypot(p1.x, p1.y, p1.z), r2 = std::hypot(p2.x, p2.y, p2.z), r12 = std::hypot(d.x, d.y, d.z);
  double const r1T = r1 / (r1 + u.a), r2T = r2 / (r2 + u.a), r12T = r12 / (r12 + u.a12);
  double const r1Scale = std::pow(u.a / (r1 * (r1 + u.a)), 2);
  double const r12Scale = std::pow(u.a12 / (r12 * (r12 + u.a12)), 2);
  double const dot = p1.x * d.x + p1.y * d.y + p1.z * d.z;
  double const r1DotR12Scale = 2 * dot * u.a12 * u.a / (std::pow(r1 * r12, 2) * (r1 + u.a) * (r12 + u.a12));
  double res = 0;
  for (int k = 0; k < u.nterms; ++k) {
    int const i = u.S[k][0], j = u.S[k][1], kk = u.S[k][2];
    double const factor = u.c[k][same] * std::pow(r12T, i) * std::pow(r1T, j) * std::pow(r2T, kk);
    res = res + factor * ((j + 1) * j * r1Scale + (i + 1) * i * r12Scale + i * j * r1DotR12Scale);
  }
  return res;
}

// Kernel functors of HartreeFockTest.cpp:248-253 (1/r12), :276-296 (TC scalar), :300-318 (grad u).
enum Kernel { K_INV_R12 = 0, K_TC_SCALAR_SAME = 1, K_TC_SCALAR_OPPO = 2, K_GRAD_U_SAME = 3, K_GRAD_U_OPPO = 4 };

double scalarKernel(int kernel, Ochi const * u, Vec3 const & p1, Vec3 const & p2)
{
  double const dx = p1.x - p2.x, dy = p1.y - p2.y, dz = p1.z - p2.z;
  if (dx == 0 && dy == 0 && dz == 0) return 0;
  double const r12 = std::hypot(dx, dy, dz);
  if (kernel == K_INV_R12) return 1 / r12;
  bool const same = kernel == K_TC_SCALAR_SAME;
  Vec3 const g12 = ochiGradient(*u, p1, p2, same);
  Vec3 const g21 = ochiGradient(*u, p2, p1, same);
  return 2 / r12 - (g12.x * g12.x + g12.y * g12.y + g12.z * g12.z) - (g21.x * g21.x + g21.y * g21.y + g21.z * g21.z);
}

Vec3 vectorKernel(int kernel, Ochi const * u, Vec3 const & p1, Vec3 const & p2)
{
  if (p1.x == p2.x && p1.y == p2.y && p1.z == p2.z) return {0, 0, 0};
  return ochiGradient(*u, p1, p2, kernel == K_GRAD_U_SAME);
}

Vec3 point(double const * pts, int ndim, int64_t n, int64_t i)
{
  if (ndim == 2) return {pts[i], 0, pts[n + i]};
  return {pts[i], pts[n + i], pts[2 * n + i]};
}

// --- LAPACK through scipy's bundled OpenBLAS (dlopen; path supplied by the caller) -------------
using zhegvd_t = void (*)(int const *, char const *, char const *, int const *, cplx *, int const *, cplx *, int const *,
                          double *, cplx *, int const *, double *, int const *, int *, int const *, int *, size_t, size_t);
using zggev_t = void (*)(char const *, char const *, int const *, cplx *, int const *, cplx *, int const *, cplx *, cplx *,
                         cplx *, int const *, cplx *, int const *, cplx *, int const *, double *, int *, size_t, size_t);
zhegvd_t g_zhegvd = nullptr;
zggev_t g_zggev = nullptr;

// Generalized Hermitian eigensolve A x = lambda B x on column-major A (overwritten by the
// eigenvectors) and B (destroyed): LvArray::dense::hegvd, UPPER_TRIANGULAR (HartreeFock.cpp:869-876).
int hegvd(int n, cplx * A, cplx * B, double * w)
{
  if (!g_zhegvd) return -100;
  int itype = 1, info = 0, lwork = -1, lrwork = -1, liwork = -1;
  cplx wq; double rq; int iq;
  g_zhegvd(&itype, "V", "U", &n, A, &n, B, &n, w, &wq, &lwork, &rq, &lrwork, &iq, &liwork, &info, 1, 1);
  lwork = int(wq.real()) + 1; lrwork = int(rq) + 1; liwork = iq + 1;
  std::vector<cplx> work(lwork); std::vector<double> rwork(lrwork); std::vector<int> iwork(liwork);
  g_zhegvd(&itype, "V", "U", &n, A, &n, B, &n, w, work.data(), &lwork, rwork.data(), &lrwork, iwork.data(), &liwork, &info, 1, 1);
  return info;
}

// LvArray::dense::ggev, right eigenvectors only (HartreeFock.cpp:1277-1286).
int ggev(int n, cplx * A, cplx * B, cplx * alpha, cplx * beta, cplx * VR)
{
  if (!g_zggev) return -100;
  int info = 0, lwork = -1, one = 1;
  cplx wq; cplx vl;
  std::vector<double> rwork(8 * n);
  g_zggev("N", "V", &n, A, &n, B, &n, alpha, beta, &vl, &one, VR, &n, &wq, &lwork, rwork.data(), &info, 1, 1);
  lwork = int(wq.real()) + 1;
  std::vector<cplx> work(lwork);
  g_zggev("N", "V", &n, A, &n, B, &n, alpha, beta, &vl, &one, VR, &n, work.data(), &lwork, rwork.data(), &info, 1, 1);
  return info;
}

// HartreeFock.cpp:183-213 (calculateIaa), Iji element type U, density complex
template <typename U>
void calculateIaa(cplx * Iaa, U const * Iji, int64_t N1, int nb, cplx const * D)
{
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < N1; ++r) {
    cplx result{};
    U const * F = Iji + r * nb * nb;
    for (int j = 0; j < nb; ++j)
      for (int i = 0; i < nb; ++i)
        result += F[j * nb + i] * D[i * nb + j];
    Iaa[r] += result;
  }
}

// HartreeFock.cpp:144-179 (calculateFai)
template <typename U>
void calculateFai(cplx * Fai, U const * Fji, cplx const * vals, int64_t N1, int nb, cplx const * D)
{
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < N1; ++r) {
    U const * F = Fji + r * nb * nb;
    for (int j = 0; j < nb; ++j) {
      cplx kSum = 0;
      for (int k = 0; k < nb; ++k) kSum += D[k * nb + j] * vals[r * nb + k];
      for (int i = 0; i < nb; ++i) Fai[r * nb + i] += kSum * F[j * nb + i];
    }
  }
}

// HartreeFock.cpp:758-780
void enforceOneElectronSymmetry(cplx * op, int nspin, int nb, double const * h)
{
  for (int idx = 0; idx < nb * nb; ++idx)
    for (int s = 0; s < nspin; ++s)
      op[s * nb * nb + idx] *= double(std::abs(h[idx]) > 0);
}

// HartreeFock.cpp:48-98; scfOperator written row-major (spin, j, i); G3 may be null.
cplx constructSCFOperator(cplx * scf, double const * h, cplx const * G2, cplx const * G3, cplx const * D, int nspin, int nb)
{
  cplx energy = 0;
  for (int ji = 0; ji < nb * nb; ++ji) {
    int const j = ji / nb, i = ji % nb;
    for (int s = 0; s < nspin; ++s) {
      int64_t const o = int64_t(s) * nb * nb;
      scf[o + j * nb + i] = h[j * nb + i] + G2[o + j * nb + i];
      cplx e = h[j * nb + i] + G2[o + j * nb + i] / 2.0;
      if (G3) { scf[o + j * nb + i] -= G3[o + j * nb + i]; e -= G3[o + j * nb + i] / 3.0; }
      energy += D[o + i * nb + j] * e;
    }
  }
  return energy;
}

// HartreeFock.cpp:20-44 ; C column-major (u, a) with leading dimension ldc
void getNewDensity(int nocc, cplx * D, cplx const * C, int nb, int ldc)
{
  for (int u = 0; u < nb; ++u)
    for (int v = 0; v < nb; ++v) {
      cplx t = 0;
      for (int a = 0; a < nocc; ++a) t += C[a * ldc + u] * std::conj(C[a * ldc + v]);
      D[u * nb + v] = t;
    }
}

// One RCS/UOS Fock build (HartreeFock.cpp:817-855 RCS, :925-968 UOS).
// F type U: double (2-D r2 grid) or cplx (3-D r2 grid).  D: [nspin][nb][nb] row-major.
// Outputs G [nspin][nb][nb] (after the symmetry mask), Fock [nspin][nb][nb] row-major (j,i), E.
template <typename U>
double fockBuild(int nspin, U const * Fji, int64_t N1, int nb, cplx const * vals, double const * w1, cplx const * D,
                 double const * h, int respectSym, cplx * G, cplx * Fock)
{
  std::vector<cplx> Faa(size_t(nspin) * N1, 0.0), Fai(size_t(nspin) * N1 * nb, 0.0);
  for (int s = 0; s < nspin; ++s) {
    calculateIaa(Faa.data() + s * N1, Fji, N1, nb, D + s * nb * nb);
    calculateFai(Fai.data() + s * N1 * nb, Fji, vals, N1, nb, D + s * nb * nb);
  }
  for (int s = 0; s < nspin; ++s) {
    cplx const * Fs = Faa.data() + s * N1;
    cplx const * Fo = Faa.data() + (nspin == 2 ? (1 - s) : s) * N1;
    cplx const * Fi = Fai.data() + s * N1 * nb;
#pragma omp parallel for schedule(static)
    for (int ji = 0; ji < nb * nb; ++ji) {
      int const j = ji / nb, i = ji % nb;
      cplx c = 0;
      for (int64_t r = 0; r < N1; ++r) {
        if (nspin == 1)
          c += w1[r] * std::conj(vals[r * nb + j]) * (2.0 * vals[r * nb + i] * Fs[r] - Fi[r * nb + i]);
        else
          c += w1[r] * std::conj(vals[r * nb + j]) * (vals[r * nb + i] * (Fs[r] + Fo[r]) - Fi[r * nb + i]);
      }
      G[int64_t(s) * nb * nb + ji] = c;
    }
  }
  if (respectSym) enforceOneElectronSymmetry(G, nspin, nb, h);
  cplx const e = constructSCFOperator(Fock, h, G, nullptr, D, nspin, nb);
  return (nspin == 1 ? 2.0 : 1.0) * e.real();
}

// orthogonalization.hpp:14-83 and :136-154 (metric MGS, including the :152 Euclidean-norm quirk)
// vectors: nvec rows of length n; metric column-major (metric(i,j) = M[j*n+i]).
void modifiedGramSchmidtMetric(cplx * vecs, int nvec, int n, cplx const * M)
{
  auto ip = [&](cplx const * a, cplx const * b) {
    cplx d = 0;
    for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) d = d + std::conj(a[i]) * M[j * n + i] * b[j];
    return d;
  };
  auto normM = [&](cplx const * v) { return std::sqrt(ip(v, v).real()); };
  auto normE = [&](cplx const * v) { double d = 0; for (int i = 0; i < n; ++i) d = d + std::norm(v[i]); return std::sqrt(d); };
  { double const s = 1 / normM(vecs); for (int i = 0; i < n; ++i) vecs[i] *= s; }
  for (int i = 1; i < nvec; ++i) {
    for (int j = i; j < nvec; ++j) {
      cplx const sc = ip(vecs + (i - 1) * n, vecs + j * n);
      for (int k = 0; k < n; ++k) vecs[j * n + k] = vecs[j * n + k] + (-sc) * vecs[(i - 1) * n + k];
    }
    double const s = 1 / normE(vecs + i * n);
    for (int k = 0; k < n; ++k) vecs[i * n + k] *= s;
  }
}

// orthogonalization.hpp:116-132 (Euclidean MGS)
void modifiedGramSchmidt(cplx * vecs, int nvec, int n)
{
  auto ip = [&](cplx const * a, cplx const * b) { cplx d = 0; for (int i = 0; i < n; ++i) d = d + std::conj(a[i]) * b[i]; return d; };
  auto normE = [&](cplx const * v) { double d = 0; for (int i = 0; i < n; ++i) d = d + std::norm(v[i]); return std::sqrt(d); };
  { double const s = 1 / normE(vecs); for (int i = 0; i < n; ++i) vecs[i] *= s; }
  for (int i = 1; i < nvec; ++i) {
    for (int j = i; j < nvec; ++j) {
      cplx const sc = ip(vecs + (i - 1) * n, vecs + j * n);
      for (int k = 0; k < n; ++k) vecs[j * n + k] = vecs[j * n + k] + (-sc) * vecs[(i - 1) * n + k];
    }
    double const s = 1 / normE(vecs + i * n);
    for (int k = 0; k < n; ++k) vecs[i * n + k] *= s;
  }
}

cplx dot3(CVec3 const & a, CVec3 const & b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
CVec3 conj3(CVec3 const & a) { return {std::conj(a.x), std::conj(a.y), std::conj(a.z)}; }
void scaledAdd3(CVec3 & a, cplx s, CVec3 const & b) { a.x = a.x + s * b.x; a.y = a.y + s * b.y; a.z = a.z + s * b.z; }
double norm3(CVec3 const & a) { return std::norm(a.x) + std::norm(a.y) + std::norm(a.z); }

} // namespace

extern "C" {

int oracle_abi_version() { return 1; }

int oracle_set_lapack(char const * path)
{
  void * h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!h) return -1;
  g_zhegvd = reinterpret_cast<zhegvd_t>(dlsym(h, "scipy_zhegvd_"));
  if (!g_zhegvd) g_zhegvd = reinterpret_cast<zhegvd_t>(dlsym(h, "zhegvd_"));
  g_zggev = reinterpret_cast<zggev_t>(dlsym(h, "scipy_zggev_"));
  if (!g_zggev) g_zggev = reinterpret_cast<zggev_t>(dlsym(h, "zggev_"));
  return (g_zhegvd && g_zggev) ? 0 : -2;
}

void oracle_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }
int oracle_get_threads() { return omp_get_max_threads(); }

// ---- grids: ChebyshevGauss.hpp:9-49, changeOfVariables.hpp:8-232, quadrature.hpp:75-102 ----------
// map: 0 None, 1 Linear(scale=p0), 2 XOver1mX, 3 TreutlerAhlrichsM4(a=p0, eps=p1), 4 (1+x)/(1-x)
// (map 4 is not in the reference; it is the radial map the product-grid workloads name,
//  u = (1+x)/(1-x), jacobian 2/(1-x)^2).
void oracle_radial_grid(int n, int map, double p0, double p1, double * u, double * w)
{
  double const freq = PI / (n + 1);
  for (int i = 0; i < n; ++i) {
    double const theta = (i + 1) * freq;
    double const x = std::cos(theta), wt = std::sin(theta);
    double uu = x, jac = 1;
    if (map == 1) { uu = p0 * x; jac = p0; }
    else if (map == 2) { uu = x / (1 - x); jac = std::pow(1 - x, -2); }
    else if (map == 3) {
      double const eOverL2 = p1 / std::log(2.0), alpha = 0.6;
      uu = eOverL2 * std::pow(x + p0, alpha) * std::log((1 + p0) / (1 - x));
      double const logPart = std::log((1 + p0) / (1 - x));
      double const xa1 = std::pow(x + p0, alpha - 1), xa = xa1 * (x + p0);
      jac = eOverL2 * (alpha * xa1 * logPart + xa / (1 - x));
    } else if (map == 4) { uu = (1 + x) / (1 - x); jac = 2 / ((1 - x) * (1 - x)); }
    u[i] = uu;
    w[i] = wt * jac * freq;
  }
}

// Product radial x angular grid (TreutlerAhlrichsLebedev.hpp:18-74 with the caller's r^2,
// SlaterTypeOrbitalTest.cpp:36): point (ir, ia) -> index ir*nang + ia, Cartesian through
// Spherical::toCartesian (mathFunctions.hpp:202-211), weight = w_r * r^2 * w_ang.
// ang: nang x {theta, phi, w}.  pts out: [3][N] (QuadratureGrid layout, quadrature.hpp:25-35).
void oracle_product_grid(int nrad, double const * r, double const * wr, int nang, double const * ang, double * pts, double * w)
{
  int64_t const N = int64_t(nrad) * nang;
  for (int ir = 0; ir < nrad; ++ir)
    for (int ia = 0; ia < nang; ++ia) {
      int64_t const i = int64_t(ir) * nang + ia;
      double const th = ang[3 * ia], ph = ang[3 * ia + 1];
      pts[i] = r[ir] * std::cos(ph) * std::sin(th);
      pts[N + i] = r[ir] * std::sin(ph) * std::sin(th);
      pts[2 * N + i] = r[ir] * std::cos(th);
      w[i] = wr[ir] * r[ir] * r[ir] * ang[3 * ia + 2];
    }
}

// QMC point mapping of QMCGrid::QMCGrid (integrateAll.hpp:21-65) with QMCCache's weights
// (qmcWrapper.hpp:128-136): unit-cube points u [ndim][N] -> Cartesian pts [ndim][N] and weights.
void oracle_qmc_grid(int ndim, int64_t N, double const * u, double * pts, double * w)
{
  double const a = 0, eOverL2 = 0.9 / std::log(2.0), alpha = 0.6;
  for (int64_t i = 0; i < N; ++i) {
    double const x0 = u[i], x1 = u[N + i];
    double const r = eOverL2 * std::pow(x0 + a, alpha) * std::log((1 + a) / (1 - x0));
    double const logPart = std::log((1 + a) / (1 - x0));
    double const xa1 = std::pow(x0 + a, alpha - 1), xa = xa1 * (x0 + a);
    double jac = eOverL2 * (alpha * xa1 * logPart + xa / (1 - x0));
    double const th = std::acos(1 - 2 * x1);
    jac *= 1 / std::sqrt(x1 * (1 - x1));
    double ph = 0;
    if (ndim == 3) { ph = 2 * PI * u[2 * N + i]; jac *= 2 * PI; }
    double const weight = 1.0 * jac * (1.0 / double(N));
    if (ndim == 2) { pts[i] = r * std::cos(ph) * std::sin(th); pts[N + i] = r * std::cos(th); }
    else {
      pts[i] = r * std::cos(ph) * std::sin(th);
      pts[N + i] = r * std::sin(ph) * std::sin(th);
      pts[2 * N + i] = r * std::cos(th);
    }
    w[i] = weight * std::pow(r, 2) * std::sin(th);
  }
}

// ---- basis: QMCGrid::setBasisFunctions (integrateAll.hpp:88-137) --------------------------------
// vals: ndim==3 -> complex [N][nb] interleaved; ndim==2 -> real [N][nb] (std::real).
// grads (optional, complex Cartesian [N][nb][3] interleaved).
void oracle_basis_values(double const * pts, int64_t N, int ndim, Sto const * basis, int nb, double * vals, double * grads)
{
  std::vector<double> nrm(nb);
  for (int b = 0; b < nb; ++b) nrm[b] = basisNormalization(basis[b]);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < N; ++i) {
    Vec3 const p = point(pts, ndim, N, i);
    double r, th, ph;
    toSpherical(p.x, p.y, p.z, r, th, ph);
    for (int b = 0; b < nb; ++b) {
      cplx const v = stoValue(basis[b], nrm[b], r, th, ph);
      if (ndim == 2) vals[i * nb + b] = v.real();
      else { vals[2 * (i * nb + b)] = v.real(); vals[2 * (i * nb + b) + 1] = v.imag(); }
      if (grads) {
        CVec3 const g = stoGradient(basis[b], nrm[b], r, th, ph);
        double * o = grads + 6 * (i * nb + b);
        o[0] = g.x.real(); o[1] = g.x.imag(); o[2] = g.y.real(); o[3] = g.y.imag(); o[4] = g.z.real(); o[5] = g.z.imag();
      }
    }
  }
}

void oracle_sph_harmonic(int l, int m, double theta, double phi, double * out)
{ cplx const v = sphericalHarmonic(l, m, theta, phi); out[0] = v.real(); out[1] = v.imag(); }

double oracle_sto_normalization(double alpha, int n) { return stoNormalization(alpha, n); }

// Analytic overlap and core Hamiltonian (SlaterTypeOrbital.hpp:134-181), filled as in
// HartreeFockTest.cpp:370-381.  S, H row-major [nb][nb] (S(i,j) symmetric, real).
void oracle_overlap_core(Sto const * basis, int nb, int Z, double * S, double * H)
{
  if (basis[0].family != 0) {
    // Ochi (OchiBasis.hpp:118-155) and hydrogen-like (HydrogenLikeBasis.hpp:70-82; the generic overlap
    // of AtomicBasis.hpp:19-31 reduced to its radial integral) on the reference driver's core grid:
    // ChebyshevGauss(1000) with TreutlerAhlrichsM4(1, 0.9) (HartreeFockTest.cpp:364-367)
    int const nr = 1000;
    std::vector<double> r(nr), w(nr);
    oracle_radial_grid(nr, 3, 1.0, 0.9, r.data(), w.data());
    for (int i = 0; i < nb; ++i)
      for (int j = 0; j < nb; ++j) {
        Sto const & b1 = basis[i];
        Sto const & b2 = basis[j];
        double const n1 = basisNormalization(b1), n2 = basisNormalization(b2);
        bool const lm = b1.l == b2.l && b1.m == b2.m;
        double sv = 0, hv = 0;
        if (b1.family == 1) {
          sv = (b1.n == b2.n) && lm;
          if (lm) {
            double integral = 0;   // integrate<1>(grid, fnl1(r) / r * fnl2(r)), fnl = radial * r
            for (int k = 0; k < nr; ++k)
              integral += w[k] * (radialComponent(b1, n1, r[k]) * r[k]) * (1 / r[k]) * (radialComponent(b2, n2, r[k]) * r[k]);
            double const coeff = b1.alpha * (b1.l + 1) * (1 + 2 * std::min(b1.n, b2.n) / double(2 * b1.l + 3)) - Z;
            hv = coeff * integral - (b1.n == b2.n) * std::pow(b1.alpha, 2) / 2;
          }
        } else {
          if (lm)
            for (int k = 0; k < nr; ++k) sv += w[k] * radialComponent(b1, n1, r[k]) * radialComponent(b2, n2, r[k]) * r[k] * r[k];
          if (b1.n == b2.n && lm) hv = -std::pow(Z, 2) / (2.0 * std::pow(b1.n, 2));
        }
        S[i * nb + j] = sv;
        H[i * nb + j] = hv;
      }
    return;
  }
  for (int i = 0; i < nb; ++i)
    for (int j = 0; j < nb; ++j) {
      Sto const & b1 = basis[i];
      Sto const & b2 = basis[j];
      double const n1 = stoNormalization(b1.alpha, b1.n), n2 = stoNormalization(b2.alpha, b2.n);
      if (b1.l != b2.l || b1.m != b2.m) { S[i * nb + j] = 0; H[i * nb + j] = 0; continue; }
      S[i * nb + j] = n1 * n2 * overlapNonNormalized(b1.n + b2.n, b1.alpha + b2.alpha);
      int const n = b2.n, l = b2.l, nSum = b1.n + b2.n;
      double const alpha = b2.alpha, aSum = b1.alpha + b2.alpha;
      H[i * nb + j] = 0.5 * n1 * n2 * ((l * (l + 1) - n * (n - 1)) * overlapNonNormalized(nSum - 2, aSum)
                                        + 2 * (n * alpha - Z) * overlapNonNormalized(nSum - 1, aSum)
                                        - std::pow(alpha, 2) * overlapNonNormalized(nSum, aSum));
    }
}

// Quadrature overlap / core Hamiltonian on a 3-D grid (the integrand of SlaterTypeOrbitalTest.cpp:30-38
// for S; 0.5 grad(phi_i)* . grad(phi_j) - Z phi_i* phi_j / r for H).  S, H complex row-major.
void oracle_quadrature_overlap_core(double const * pts, double const * w, int64_t N, double const * vals, double const * grads,
                                    int nb, int Z, double * S, double * H)
{
  cplx const * v = reinterpret_cast<cplx const *>(vals);
  cplx const * g = reinterpret_cast<cplx const *>(grads);
#pragma omp parallel for schedule(dynamic)
  for (int ij = 0; ij < nb * nb; ++ij) {
    int const i = ij / nb, j = ij % nb;
    cplx s = 0, hsum = 0;
    for (int64_t p = 0; p < N; ++p) {
      double const r = std::hypot(pts[p], pts[N + p], pts[2 * N + p]);
      cplx const ov = std::conj(v[p * nb + i]) * v[p * nb + j];
      s += w[p] * ov;
      if (g) {
        cplx const * gi = g + 3 * (p * nb + i);
        cplx const * gj = g + 3 * (p * nb + j);
        cplx const kin = std::conj(gi[0]) * gj[0] + std::conj(gi[1]) * gj[1] + std::conj(gi[2]) * gj[2];
        hsum += w[p] * (0.5 * kin - double(Z) * ov / r);
      }
    }
    S[2 * ij] = s.real(); S[2 * ij + 1] = s.imag();
    if (H) { H[2 * ij] = hsum.real(); H[2 * ij + 1] = hsum.imag(); }
  }
}

// Jastrow (jastrowFunctions.hpp:9-115)
double oracle_ochi_value(Ochi const * u, double r1, double r2, double r12, int same) { return ochiValue(*u, r1, r2, r12, same != 0); }
void oracle_ochi_gradient(Ochi const * u, double const * p1, double const * p2, int same, double * out)
{
  Vec3 const g = ochiGradient(*u, {p1[0], p1[1], p1[2]}, {p2[0], p2[1], p2[2]}, same != 0);
  out[0] = g.x; out[1] = g.y; out[2] = g.z;
}
double oracle_ochi_laplacian(Ochi const * u, double const * p1, double const * p2, int same)
{ return ochiLaplacian(*u, {p1[0], p1[1], p1[2]}, {p2[0], p2[1], p2[2]}, same != 0); }

// Kernel values g(r1,r2) (no weight) for the vectorised checks of the device generator.
void oracle_kernel_values(int kernel, Ochi const * u, double const * p1, int64_t N1, double const * p2, int64_t N2, int ndim2, double * out)
{
#pragma omp parallel for schedule(static)
  for (int64_t a = 0; a < N1; ++a) {
    Vec3 const q1{p1[a], p1[N1 + a], p1[2 * N1 + a]};
    for (int64_t b = 0; b < N2; ++b) {
      Vec3 const q2 = point(p2, ndim2, N2, b);
      if (kernel >= K_GRAD_U_SAME) {
        Vec3 const g = vectorKernel(kernel, u, q1, q2);
        out[3 * (a * N2 + b)] = g.x; out[3 * (a * N2 + b) + 1] = g.y; out[3 * (a * N2 + b) + 2] = g.z;
      } else out[a * N2 + b] = scalarKernel(kernel, u, q1, q2);
    }
  }
}

// precomputeIntegrand + computeF (HartreeFock.hpp:23-51 / :55-83 and :88-131 / :136-180), kernel rows
// generated per r1 point instead of stored as N1 x N2 (identical values: f(r1,r2) * w2).
// ndim2 == 2: r2 basis values real [N2][nb], F real [N1][nb][nb] scaled by 2*pi.
// ndim2 == 3: r2 basis values complex [N2][nb], F complex [N1][nb][nb].
void oracle_compute_F(double const * p1, int64_t N1, double const * p2, double const * w2, int64_t N2, int ndim2,
                      double const * vals2, int nb, int kernel, Ochi const * u, double * F)
{
  bool const cx = ndim2 == 3;
  // transposed basis table [nb][N2] for unit-stride r2 inner products
  std::vector<cplx> bt(size_t(nb) * N2);
  for (int64_t r = 0; r < N2; ++r)
    for (int b = 0; b < nb; ++b)
      bt[size_t(b) * N2 + r] = cx ? cplx(vals2[2 * (r * nb + b)], vals2[2 * (r * nb + b) + 1]) : cplx(vals2[r * nb + b], 0);
#pragma omp parallel
  {
    std::vector<double> values(N2);
    std::vector<cplx> left(N2);
#pragma omp for schedule(dynamic, 1)
    for (int64_t a = 0; a < N1; ++a) {
      Vec3 const q1{p1[a], p1[N1 + a], p1[2 * N1 + a]};
      for (int64_t b = 0; b < N2; ++b) values[b] = scalarKernel(kernel, u, q1, point(p2, ndim2, N2, b)) * w2[b];
      for (int j = 0; j < nb; ++j) {
        cplx const * bj = bt.data() + size_t(j) * N2;
        for (int64_t b = 0; b < N2; ++b) left[b] = std::conj(bj[b]) * values[b];
        for (int i = j; i < nb; ++i) {
          cplx const * bi = bt.data() + size_t(i) * N2;
          cplx ans = 0;
          if (cx) {
            for (int64_t b = 0; b < N2; ++b) ans += left[b] * bi[b];
            double * o = F + 2 * (a * nb * nb + j * nb + i);
            o[0] = ans.real(); o[1] = ans.imag();
            double * o2 = F + 2 * (a * nb * nb + i * nb + j);
            o2[0] = ans.real(); o2[1] = -ans.imag();
          } else {
            double s = 0;
            for (int64_t b = 0; b < N2; ++b) s += left[b].real() * bi[b].real();
            F[a * nb * nb + j * nb + i] = 2 * PI * s;
            F[a * nb * nb + i * nb + j] = 2 * PI * s;
          }
        }
      }
    }
  }
}

// computeV (HartreeFock.hpp:185-229): V [N1][nb][nb][3] complex, vector kernel * w2.
void oracle_compute_V(double const * p1, int64_t N1, double const * p2, double const * w2, int64_t N2,
                      double const * vals2, int nb, int kernel, Ochi const * u, double * V)
{
  cplx const * v2 = reinterpret_cast<cplx const *>(vals2);
#pragma omp parallel
  {
    std::vector<Vec3> vf(N2);
#pragma omp for schedule(dynamic, 1)
    for (int64_t a = 0; a < N1; ++a) {
      Vec3 const q1{p1[a], p1[N1 + a], p1[2 * N1 + a]};
      for (int64_t b = 0; b < N2; ++b) {
        Vec3 g = vectorKernel(kernel, u, q1, point(p2, 3, N2, b));
        vf[b] = {g.x * w2[b], g.y * w2[b], g.z * w2[b]};
      }
      for (int j = 0; j < nb; ++j)
        for (int i = j; i < nb; ++i) {
          CVec3 ans{};
          for (int64_t b = 0; b < N2; ++b) {
            cplx const sc = std::conj(v2[b * nb + j]) * v2[b * nb + i];
            ans.x = ans.x + sc * vf[b].x; ans.y = ans.y + sc * vf[b].y; ans.z = ans.z + sc * vf[b].z;
          }
          cplx * o = reinterpret_cast<cplx *>(V) + 3 * (a * nb * nb + j * nb + i);
          o[0] = ans.x; o[1] = ans.y; o[2] = ans.z;
          cplx * o2 = reinterpret_cast<cplx *>(V) + 3 * (a * nb * nb + i * nb + j);
          o2[0] = std::conj(ans.x); o2[1] = std::conj(ans.y); o2[2] = std::conj(ans.z);
        }
    }
  }
}

// One Fock build from a precomputed F (RCS nspin=1 / UOS nspin=2).  fcomplex: F complex (3-D r2).
double oracle_fock_build(int nspin, int fcomplex, double const * F, int64_t N1, int nb, double const * vals1, double const * w1,
                         double const * D, double const * h, int respectSym, double * G, double * Fock)
{
  cplx const * v = reinterpret_cast<cplx const *>(vals1);
  cplx const * Dc = reinterpret_cast<cplx const *>(D);
  cplx * Gc = reinterpret_cast<cplx *>(G);
  cplx * Fc = reinterpret_cast<cplx *>(Fock);
  if (fcomplex) return fockBuild<cplx>(nspin, reinterpret_cast<cplx const *>(F), N1, nb, v, w1, Dc, h, respectSym, Gc, Fc);
  return fockBuild<double>(nspin, F, N1, nb, v, w1, Dc, h, respectSym, Gc, Fc);
}

// Full RCS (HartreeFock.cpp:785-886) or UOS (:890-1003) SCF on a precomputed F.
// S row-major real [nb][nb] (copied into the column-major complex BMatrix), h row-major real.
// Outputs: energy, iterations, density [nspin][nb][nb], eigenvalues [nspin][nb].
// Returns 0 on convergence, 1 on non-convergence, <0 on LAPACK error.
int oracle_scf(int nspin, int nup, int ndown, int fcomplex, double const * F, int64_t N1, int nb, double const * vals1,
               double const * w1, double const * S, double const * h, int respectSym, double tol, int maxIter,
               double * energyOut, int * itersOut, double * densityOut, double * eigOut)
{
  int const nn = nb * nb;
  std::vector<cplx> D(size_t(nspin) * nn, 0.0), G(size_t(nspin) * nn), Fock(size_t(nspin) * nn), A(nn), B(nn);
  std::vector<double> w(nb);
  double energy = std::numeric_limits<double>::max();
  int const nocc[2] = {nspin == 1 ? (nup + ndown) / 2 : nup, ndown};
  for (int it = 0; it < maxIter; ++it) {
    double const e = oracle_fock_build(nspin, fcomplex, F, N1, nb, vals1, w1, reinterpret_cast<double const *>(D.data()), h,
                                       respectSym, reinterpret_cast<double *>(G.data()), reinterpret_cast<double *>(Fock.data()));
    *itersOut = it + 1;
    if (std::abs(e - energy) < tol) {
      *energyOut = e;
      std::memcpy(densityOut, D.data(), sizeof(cplx) * D.size());
      return 0;
    }
    energy = e;
    for (int s = 0; s < nspin; ++s) {
      // fockOperator is PERM_IKJ: element (j,i) of spin s at column-major [i*nb + j]
      for (int j = 0; j < nb; ++j)
        for (int i = 0; i < nb; ++i) A[i * nb + j] = Fock[s * nn + j * nb + i];
      for (int i = 0; i < nb; ++i)
        for (int j = 0; j < nb; ++j) B[j * nb + i] = S[i * nb + j];
      int const info = hegvd(nb, A.data(), B.data(), w.data());
      if (info != 0) return info < 0 ? info : -1000 - info;
      for (int i = 0; i < nb; ++i) eigOut[s * nb + i] = w[i];
      getNewDensity(nocc[s], D.data() + s * nn, A.data(), nb, nb);
    }
  }
  *energyOut = energy;
  std::memcpy(densityOut, D.data(), sizeof(cplx) * D.size());
  return 1;
}

// ---- transcorrelated terms (HartreeFock.cpp:102-609 and :1105-1261) ------------------------------
// Inputs (complex unless noted): vals1 [N1][nb], grads1 [N1][nb][3], w1 real, FjiSame/Oppo [N1][nb][nb]
// (real when fcomplex==0), VjiSame/Oppo [N1][nb][nb][3], D [2][nb][nb], occ[s] column-major
// (nb x nocc[s], PERM_JI).  Outputs G2, G3 [2][nb][nb] (after the symmetry mask), Fock, energy.
double oracle_tc_fock_build(int fcomplex, double const * FjiSame_, double const * FjiOppo_, double const * VjiSame_,
                            double const * VjiOppo_, int64_t N1, int nb, double const * vals1_, double const * grads1_,
                            double const * w1, double const * D_, int nup, int ndown, double const * occUp_,
                            double const * occDown_, double const * h, int respectSym, double * G2_, double * G3_, double * Fock_)
{
  using C3 = CVec3;
  cplx const * vals = reinterpret_cast<cplx const *>(vals1_);
  C3 const * grads = reinterpret_cast<C3 const *>(grads1_);
  C3 const * VjiSame = reinterpret_cast<C3 const *>(VjiSame_);
  C3 const * VjiOppo = reinterpret_cast<C3 const *>(VjiOppo_);
  cplx const * D = reinterpret_cast<cplx const *>(D_);
  cplx const * occ[2] = {reinterpret_cast<cplx const *>(occUp_), reinterpret_cast<cplx const *>(occDown_)};
  int const nel[2] = {nup, ndown};
  int64_t const nn = int64_t(nb) * nb;
  auto Dat = [&](int s, int i, int j) { return D[s * nn + i * nb + j]; };
  auto val = [&](int64_t r, int b) { return vals[r * nb + b]; };
  auto grad = [&](int64_t r, int b) { return grads[r * nb + b]; };
  auto Vs = [&](int64_t r, int j, int i) { return VjiSame[r * nn + j * nb + i]; };
  auto Vo = [&](int64_t r, int j, int i) { return VjiOppo[r * nn + j * nb + i]; };

  std::vector<cplx> FaaSPO(2 * N1, 0.0), FaiSame(2 * N1 * nb, 0.0), Vai(2 * N1 * nb, 0.0);
  std::vector<C3> VaaSPO(2 * N1, C3{}), Vja(2 * N1 * nb, C3{}), scaledGradients(2 * N1, C3{});
  std::vector<C3> VjbSame[2], VjbOppo[2], VabSame[2], VabOppo[2];
  std::vector<double> sumNormsSame[2], sumNormsOppo[2];
  for (int s = 0; s < 2; ++s) {
    VjbSame[s].assign(N1 * nb * nel[s], C3{}); VjbOppo[s].assign(N1 * nb * nel[s], C3{});
    VabSame[s].assign(N1 * nel[s] * nel[s], C3{}); VabOppo[s].assign(N1 * nel[s] * nel[s], C3{});
    sumNormsSame[s].assign(N1, 0.0); sumNormsOppo[s].assign(N1, 0.0);
  }

  for (int s = 0; s < 2; ++s) {
    cplx const * Ds = D + s * nn;
    cplx const * Do = D + (1 - s) * nn;
    if (fcomplex) {
      calculateIaa(FaaSPO.data() + s * N1, reinterpret_cast<cplx const *>(FjiSame_), N1, nb, Ds);
      calculateIaa(FaaSPO.data() + s * N1, reinterpret_cast<cplx const *>(FjiOppo_), N1, nb, Do);
      calculateFai(FaiSame.data() + s * N1 * nb, reinterpret_cast<cplx const *>(FjiSame_), vals, N1, nb, Ds);
    } else {
      calculateIaa(FaaSPO.data() + s * N1, FjiSame_, N1, nb, Ds);
      calculateIaa(FaaSPO.data() + s * N1, FjiOppo_, N1, nb, Do);
      calculateFai(FaiSame.data() + s * N1 * nb, FjiSame_, vals, N1, nb, Ds);
    }
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < N1; ++r) {
      // calculateIaa on Vji (:1125-1126)
      C3 res{};
      for (int j = 0; j < nb; ++j)
        for (int i = 0; i < nb; ++i) { C3 const v = Vs(r, j, i); cplx const d = Ds[i * nb + j]; res.x += v.x * d; res.y += v.y * d; res.z += v.z * d; }
      C3 res2{};
      for (int j = 0; j < nb; ++j)
        for (int i = 0; i < nb; ++i) { C3 const v = Vo(r, j, i); cplx const d = Do[i * nb + j]; res2.x += v.x * d; res2.y += v.y * d; res2.z += v.z * d; }
      C3 & vaa = VaaSPO[s * N1 + r];
      vaa.x += res.x; vaa.y += res.y; vaa.z += res.z;
      vaa.x += res2.x; vaa.y += res2.y; vaa.z += res2.z;
      // calculateVai (:217-252)
      for (int j = 0; j < nb; ++j) {
        C3 kSum{};
        for (int k = 0; k < nb; ++k) scaledAdd3(kSum, Ds[k * nb + j], grad(r, k));
        for (int i = 0; i < nb; ++i) Vai[(s * N1 + r) * nb + i] += dot3(Vs(r, j, i), kSum);
      }
      // calculateVja (:256-291)
      for (int i = 0; i < nb; ++i) {
        cplx kSum = 0;
        for (int k = 0; k < nb; ++k) kSum += Ds[i * nb + k] * std::conj(val(r, k));
        for (int j = 0; j < nb; ++j) scaledAdd3(Vja[(s * N1 + r) * nb + j], kSum, Vs(r, j, i));
      }
    }
    // calculateScaledGradients (:102-140), both spins
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < N1; ++r) {
      C3 ans[2]{};
      for (int j = 0; j < nb; ++j)
        for (int i = 0; i < nb; ++i)
          for (int sp = 0; sp < 2; ++sp) scaledAdd3(ans[sp], Dat(sp, i, j) * std::conj(val(r, j)), grad(r, i));
      scaledGradients[r] = ans[0]; scaledGradients[N1 + r] = ans[1];
    }
    // calculateVjb (:295-337) and calculateVab (:341-393) with occupiedOrbitals[s] (nb x nel, column-major)
    int const no = nel[s];
    cplx const * C = occ[s];
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < N1; ++r) {
      for (int j = 0; j < nb; ++j)
        for (int b = 0; b < no; ++b) {
          C3 rs{}, ro{};
          for (int i = 0; i < nb; ++i) { scaledAdd3(rs, C[b * nb + i], Vs(r, j, i)); scaledAdd3(ro, C[b * nb + i], Vo(r, j, i)); }
          VjbSame[s][(r * nb + j) * no + b] = rs; VjbOppo[s][(r * nb + j) * no + b] = ro;
        }
      for (int a = 0; a < no; ++a)
        for (int b = 0; b < no; ++b) {
          C3 rs{}, ro{};
          for (int j = 0; j < nb; ++j) {
            cplx const cc = std::conj(C[a * nb + j]);
            scaledAdd3(rs, cc, VjbSame[s][(r * nb + j) * no + b]);
            scaledAdd3(ro, cc, VjbOppo[s][(r * nb + j) * no + b]);
          }
          VabSame[s][(r * no + a) * no + b] = rs; VabOppo[s][(r * no + a) * no + b] = ro;
          sumNormsSame[s][r] += norm3(rs); sumNormsOppo[s][r] += norm3(ro);
        }
    }
  }

  // three-electron precomputation (:1140-1148)
  std::vector<C3> VTilde(2 * N1), VTildeSubI(2 * N1 * nb, C3{}), SumConjVTOcc(2 * N1);
  std::vector<cplx> SumVbiDotVTb(2 * N1 * nb, 0.0);
  std::vector<double> occDensity(2 * N1);
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < N1; ++r) {
    // calculateVTilde (:397-434)
    C3 res[2]{};
    for (int j = 0; j < nb; ++j)
      for (int i = 0; i < nb; ++i)
        for (int sp = 0; sp < 2; ++sp) { scaledAdd3(res[sp], Dat(sp, i, j), Vs(r, j, i)); scaledAdd3(res[sp], Dat(1 - sp, i, j), Vo(r, j, i)); }
    VTilde[r] = res[0]; VTilde[N1 + r] = res[1];
    // calculateVTildeSubI (:438-480)
    for (int k = 0; k < nb; ++k) {
      cplx ell[2]{};
      for (int l = 0; l < nb; ++l) for (int sp = 0; sp < 2; ++sp) ell[sp] += Dat(sp, l, k) * val(r, l);
      for (int i = 0; i < nb; ++i) for (int sp = 0; sp < 2; ++sp) scaledAdd3(VTildeSubI[(sp * N1 + r) * nb + i], ell[sp], Vs(r, k, i));
    }
  }
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < N1; ++r) {
    // calculateSumOverb_Vbi_dot_VTildeb (:484-526)
    for (int k = 0; k < nb; ++k) {
      C3 ell[2]{};
      for (int l = 0; l < nb; ++l) for (int sp = 0; sp < 2; ++sp) scaledAdd3(ell[sp], Dat(sp, l, k), VTildeSubI[(sp * N1 + r) * nb + l]);
      for (int i = 0; i < nb; ++i) for (int sp = 0; sp < 2; ++sp) SumVbiDotVTb[(sp * N1 + r) * nb + i] += dot3(Vs(r, k, i), ell[sp]);
    }
    // calculateOccupiedElectronDensity (:530-567)
    cplx cur[2]{};
    for (int k = 0; k < nb; ++k)
      for (int l = 0; l < nb; ++l)
        for (int sp = 0; sp < 2; ++sp) cur[sp] += Dat(sp, l, k) * std::conj(val(r, k)) * val(r, l);
    occDensity[r] = cur[0].real(); occDensity[N1 + r] = cur[1].real();
    // calculateSumOverb_conjVTildeb_occb (:571-609)
    C3 cs[2]{};
    for (int k = 0; k < nb; ++k)
      for (int l = 0; l < nb; ++l)
        for (int sp = 0; sp < 2; ++sp) scaledAdd3(cs[sp], Dat(sp, l, k) * val(r, l), conj3(VTildeSubI[(sp * N1 + r) * nb + k]));
    SumConjVTOcc[r] = cs[0]; SumConjVTOcc[N1 + r] = cs[1];
  }

  cplx * G2 = reinterpret_cast<cplx *>(G2_);
  cplx * G3 = reinterpret_cast<cplx *>(G3_);
  std::vector<cplx> vecComp(2 * nn);
  for (int s = 0; s < 2; ++s) {
    int const so = 1 - s;
#pragma omp parallel for schedule(dynamic)
    for (int ji = 0; ji < nb * nb; ++ji) {
      int const j = ji / nb, i = ji % nb;
      cplx scalar = 0, vector = 0, scalar3 = 0;
      for (int64_t r = 0; r < N1; ++r) {
        cplx const cvj = std::conj(val(r, j));
        scalar += w1[r] * (cvj * (FaaSPO[s * N1 + r] * val(r, i) - FaiSame[(s * N1 + r) * nb + i]));
        cplx va = 0;
        va += cvj * (dot3(VaaSPO[s * N1 + r], grad(r, i)) - Vai[(s * N1 + r) * nb + i]);
        va += dot3(Vs(r, j, i), scaledGradients[s * N1 + r]);
        va += dot3(Vo(r, j, i), scaledGradients[so * N1 + r]);
        va -= dot3(Vja[(s * N1 + r) * nb + j], grad(r, i));
        vector += w1[r] * va;
        C3 const & VT = VTilde[s * N1 + r];
        C3 const & VTsubI = VTildeSubI[(s * N1 + r) * nb + i];
        C3 const & VTsubJ = VTildeSubI[(s * N1 + r) * nb + j];
        cplx s3 = 0;
        s3 += cvj * (norm3(VT) - sumNormsSame[s][r] - sumNormsOppo[so][r]) * val(r, i);
        s3 += 2.0 * cvj * (SumVbiDotVTb[(s * N1 + r) * nb + i] - dot3(VT, VTsubI));
        s3 += 2.0 * (std::conj(SumVbiDotVTb[(s * N1 + r) * nb + j]) - dot3(conj3(VTsubJ), VT)) * val(r, i);
        cplx sbS = 0, sbO = 0;
        for (int b = 0; b < nel[s]; ++b) {
          sbS += dot3(VjbSame[s][(r * nb + j) * nel[s] + b], conj3(VjbSame[s][(r * nb + i) * nel[s] + b]));
          sbO += dot3(VjbOppo[s][(r * nb + j) * nel[s] + b], conj3(VjbOppo[s][(r * nb + i) * nel[s] + b]));
        }
        s3 += 2.0 * occDensity[s * N1 + r] * (dot3(Vs(r, j, i), VT) - sbS);
        s3 += 2.0 * (dot3(VTsubI, conj3(VTsubJ)) - dot3(Vs(r, j, i), SumConjVTOcc[s * N1 + r]));
        s3 += 2.0 * occDensity[so * N1 + r] * (dot3(Vo(r, j, i), VTilde[so * N1 + r]) - sbO);
        s3 -= 2.0 * dot3(Vo(r, j, i), SumConjVTOcc[so * N1 + r]);
        scalar3 += w1[r] * s3;
      }
      G2[s * nn + ji] = scalar / 2.0;
      vecComp[s * nn + ji] = vector / 2.0;
      G3[s * nn + ji] = scalar3 / 2.0;
    }
    for (int ji = 0; ji < nb * nb; ++ji) {
      int const j = ji / nb, i = ji % nb;
      G2[s * nn + ji] += vecComp[s * nn + ji] - std::conj(vecComp[s * nn + i * nb + j]);
    }
  }
  if (respectSym) { enforceOneElectronSymmetry(G2, 2, nb, h); enforceOneElectronSymmetry(G3, 2, nb, h); }
  cplx const e = constructSCFOperator(reinterpret_cast<cplx *>(Fock_), h, G2, G3, D, 2, nb);
  return e.real();
}

// Full TC SCF (HartreeFock.cpp:1007-1362).  Returns 0 on convergence, 1 otherwise, <0 LAPACK error.
int oracle_tc_scf(int fcomplex, double const * FjiSame, double const * FjiOppo, double const * VjiSame, double const * VjiOppo,
                  int64_t N1, int nb, double const * vals1, double const * grads1, double const * w1, double const * S,
                  double const * h, int nup, int ndown, int respectSym, double tol, int maxIter, double * energyOut,
                  int * itersOut, double * densityOut, double * pseudoEnergyOut)
{
  int const nn = nb * nb;
  int const nel[2] = {nup, ndown};
  std::vector<cplx> D(2 * nn, 0.0), G2(2 * nn), G3(2 * nn), Fock(2 * nn), A(nn), B(nn), VR(nn), alpha(nb), beta(nb);
  std::vector<cplx> occ[2] = {std::vector<cplx>(size_t(nb) * nup, 0.0), std::vector<cplx>(size_t(nb) * ndown, 0.0)};
  std::vector<cplx> eig(2 * nb), evec(2 * nn);
  std::vector<int> sorted(2 * nb);
  for (int i = 0; i < nb; ++i) { sorted[i] = i; sorted[nb + i] = i; }
  double energy = std::numeric_limits<double>::max();
  for (int it = 0; it < maxIter; ++it) {
    double const e = oracle_tc_fock_build(fcomplex, FjiSame, FjiOppo, VjiSame, VjiOppo, N1, nb, vals1, grads1, w1,
                                          reinterpret_cast<double const *>(D.data()), nup, ndown,
                                          reinterpret_cast<double const *>(occ[0].data()), reinterpret_cast<double const *>(occ[1].data()),
                                          h, respectSym, reinterpret_cast<double *>(G2.data()), reinterpret_cast<double *>(G3.data()),
                                          reinterpret_cast<double *>(Fock.data()));
    *itersOut = it + 1;
    if (std::abs(e - energy) < tol) {
      *energyOut = e;
      std::memcpy(densityOut, D.data(), sizeof(cplx) * D.size());
      return 0;
    }
    energy = e;
    for (int s = 0; s < 2; ++s) {
      for (int j = 0; j < nb; ++j)
        for (int i = 0; i < nb; ++i) A[i * nb + j] = Fock[s * nn + j * nb + i];
      for (int i = 0; i < nb; ++i)
        for (int j = 0; j < nb; ++j) B[j * nb + i] = S[i * nb + j];
      int const info = ggev(nb, A.data(), B.data(), alpha.data(), beta.data(), VR.data());
      if (info != 0) return info < 0 ? info : -1000 - info;
      for (int i = 0; i < nb; ++i) eig[s * nb + i] = alpha[i] / beta[i];
      std::memcpy(evec.data() + s * nn, VR.data(), sizeof(cplx) * nn);
    }
    for (int s = 0; s < 2; ++s) {
      int * si = sorted.data() + s * nb;
      std::sort(si, si + nb, [&](int a, int b) { return std::real(eig[s * nb + a]) < std::real(eig[s * nb + b]); });
      std::vector<cplx> occT(size_t(nel[s]) * nb);
      for (int i = 0; i < nel[s]; ++i) {
        pseudoEnergyOut[s * nb + i] = std::real(eig[s * nb + si[i]]);
        for (int j = 0; j < nb; ++j) occT[i * nb + j] = evec[s * nn + si[i] * nb + j];
      }
      std::vector<cplx> Mc(nn);
      for (int i = 0; i < nb; ++i) for (int j = 0; j < nb; ++j) Mc[j * nb + i] = S[i * nb + j];
      if (nel[s] > 0) modifiedGramSchmidtMetric(occT.data(), nel[s], nb, Mc.data());
      for (int i = 0; i < nel[s]; ++i)
        for (int j = 0; j < nb; ++j) occ[s][i * nb + j] = occT[i * nb + j];
      getNewDensity(nel[s], D.data() + s * nn, occ[s].data(), nb, nb);
    }
  }
  *energyOut = energy;
  std::memcpy(densityOut, D.data(), sizeof(cplx) * D.size());
  return 1;
}

// MGS entry points for the orthogonalisation known-answer test (vectors as rows).
void oracle_mgs(double * vecs, int nvec, int n, double const * metricColMajor)
{
  if (metricColMajor) modifiedGramSchmidtMetric(reinterpret_cast<cplx *>(vecs), nvec, n, reinterpret_cast<cplx const *>(metricColMajor));
  else modifiedGramSchmidt(reinterpret_cast<cplx *>(vecs), nvec, n);
}

// ---- 4- and 6-index tensors (integrateAll.hpp:152-317, :328-442) -------------------------------
// integrateAllR1R2: r1 3-D (complex values), r2 2-D (real values, gradients complex [N2][nb][3]);
// answer [nb]^4 complex.  use_gradient selects evaluateR2GradientIntegral and the (b2,b1,b4,b3) store.
void oracle_integrate_all_r1r2(int use_gradient, double const * p1, double const * w1, int64_t N1, double const * vals1,
                               double const * p2, double const * w2, int64_t N2, double const * vals2, double const * grads2,
                               int nb, int kernel, Ochi const * u, double * answer_)
{
  cplx const * v1 = reinterpret_cast<cplx const *>(vals1);
  CVec3 const * g2 = reinterpret_cast<CVec3 const *>(grads2);
  int64_t const nb2 = int64_t(nb) * nb, nb3 = nb2 * nb;
  int const nthreads = omp_get_max_threads();
  std::vector<std::vector<cplx>> partial(nthreads, std::vector<cplx>(nb3 * nb, 0.0));
#pragma omp parallel
  {
    std::vector<cplx> & acc = partial[omp_get_thread_num()];
    std::vector<double> fval(N2);
    std::vector<Vec3> fvec(N2);
#pragma omp for schedule(dynamic, 1)
    for (int64_t a = 0; a < N1; ++a) {
      Vec3 const q1{p1[a], p1[N1 + a], p1[2 * N1 + a]};
      for (int64_t b = 0; b < N2; ++b) {
        Vec3 const q2 = point(p2, 2, N2, b);
        if (use_gradient) fvec[b] = vectorKernel(kernel, u, q1, q2); else fval[b] = scalarKernel(kernel, u, q1, q2);
      }
      for (int b4 = 0; b4 < nb; ++b4)
        for (int b2 = 0; b2 < nb; ++b2) {
          cplx inner = 0;
          for (int64_t b = 0; b < N2; ++b) {
            cplx integrand;
            if (use_gradient) {
              CVec3 const g = g2[b * nb + b4];
              integrand = w2[b] * (fvec[b].x * g.x + fvec[b].y * g.y + fvec[b].z * g.z);
            } else integrand = w2[b] * fval[b] * vals2[b * nb + b4];
            inner += vals2[b * nb + b2] * integrand;
          }
          inner *= 2 * PI;
          inner *= w1[a];
          for (int b1 = 0; b1 < nb; ++b1)
            for (int b3 = 0; b3 < nb; ++b3) {
              cplx const r1c = std::conj(v1[a * nb + b1]) * v1[a * nb + b3];
              cplx const add = inner * r1c;
              if (use_gradient) acc[b2 * nb3 + b1 * nb2 + b4 * nb + b3] += add;
              else acc[b1 * nb3 + b2 * nb2 + b3 * nb + b4] += add;
            }
        }
    }
  }
  cplx * answer = reinterpret_cast<cplx *>(answer_);
  for (int64_t k = 0; k < nb3 * nb; ++k) { cplx s = 0; for (int t = 0; t < nthreads; ++t) s += partial[t][k]; answer[k] = s; }
}

// threeElectronIntegrals (integrateAll.hpp:361-442): answer [nb]^6 complex, V with grad u (same spin).
void oracle_three_electron_integrals(double const * p1, double const * w1, int64_t N1, double const * vals1, double const * p2,
                                     double const * w2, int64_t N2, double const * vals2, int nb, Ochi const * u, double * answer_)
{
  cplx const * v1 = reinterpret_cast<cplx const *>(vals1);
  cplx const * v2 = reinterpret_cast<cplx const *>(vals2);
  int64_t const nn = int64_t(nb) * nb;
  std::vector<CVec3> V(N1 * nn);
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t a = 0; a < N1; ++a) {
    Vec3 const q1{p1[a], p1[N1 + a], p1[2 * N1 + a]};
    for (int q = 0; q < nb; ++q)
      for (int t = 0; t < nb; ++t) {
        CVec3 ans{};
        for (int64_t b = 0; b < N2; ++b) {
          Vec3 const q2 = point(p2, 3, N2, b);
          cplx const sc = w2[b] * std::conj(v2[b * nb + q]) * v2[b * nb + t];
          Vec3 const g = vectorKernel(K_GRAD_U_SAME, u, q1, q2);
          ans.x += sc * g.x; ans.y += sc * g.y; ans.z += sc * g.z;
        }
        V[a * nn + q * nb + t] = ans;
      }
  }
  int64_t const n6 = nn * nn * nn;
  cplx * answer = reinterpret_cast<cplx *>(answer_);
  std::fill(answer, answer + n6, cplx(0));
  // reduction over r1 per output element (p,q,r,s,t,u) in r1 order (the reference's atomics have no fixed order)
#pragma omp parallel for schedule(static)
  for (int64_t idx = 0; idx < n6; ++idx) {
    int64_t k = idx;
    int const uu = k % nb; k /= nb; int const t = k % nb; k /= nb; int const s = k % nb; k /= nb;
    int const r = k % nb; k /= nb; int const q = k % nb; k /= nb; int const p = int(k);
    cplx acc = 0;
    for (int64_t a = 0; a < N1; ++a) {
      CVec3 const & A = V[a * nn + q * nb + t];
      CVec3 const & B = V[a * nn + r * nb + uu];
      cplx const d = A.x * B.x + A.y * B.y + A.z * B.z;
      acc += w1[a] * std::conj(v1[a * nb + p]) * d * v1[a * nb + s];
    }
    answer[idx] = acc;
  }
}

// computeQ (HartreeFock.cpp:613-683): the 6-index verification tensors of the TC 3-body term,
// Q[j][p][r][i][q][s] = sum_r1 w (conj(b_j) (V_pq . V_rs) b_i + conj(b_p) (V_ji . V_rs) b_q
//                                 + conj(b_r) (V_ji . V_pq) b_s)
// for the same-same (Vs, Vs), same-opposite (Vs, Vo) and opposite-opposite (Vo, Vo) pairs.  vals1
// complex [N1][nb]; V complex Cartesian [N1][nb][nb][3]; outputs complex [nb]^6 row-major.
void oracle_compute_q(int64_t N1, int nb, double const * w1, double const * vals1, double const * Vs, double const * Vo, double * Qss,
                      double * Qso, double * Qoo)
{
  cplx const * b = reinterpret_cast<cplx const *>(vals1);
  cplx const * vs = reinterpret_cast<cplx const *>(Vs);
  cplx const * vo = reinterpret_cast<cplx const *>(Vo);
  int64_t const n6 = int64_t(nb) * nb * nb * nb * nb * nb;
  cplx * ss = reinterpret_cast<cplx *>(Qss);
  cplx * so = reinterpret_cast<cplx *>(Qso);
  cplx * oo = reinterpret_cast<cplx *>(Qoo);
  for (int64_t o = 0; o < n6; ++o) ss[o] = so[o] = oo[o] = 0.0;
  auto V = [&](cplx const * v, int64_t a, int x, int y, int d) { return v[((a * nb + x) * nb + y) * 3 + d]; };
  auto dot = [&](cplx const * v1, cplx const * v2, int64_t a, int x1, int y1, int x2, int y2) {
    return V(v1, a, x1, y1, 0) * V(v2, a, x2, y2, 0) + V(v1, a, x1, y1, 1) * V(v2, a, x2, y2, 1) + V(v1, a, x1, y1, 2) * V(v2, a, x2, y2, 2);
  };
  // r1 outermost per j slab (each thread owns the outputs of its j; the reference adds atomically)
#pragma omp parallel for schedule(dynamic)
  for (int j = 0; j < nb; ++j)
    for (int64_t a = 0; a < N1; ++a) {
      double const w = w1[a];
      for (int p = 0; p < nb; ++p)
        for (int r = 0; r < nb; ++r)
          for (int i = 0; i < nb; ++i)
            for (int q = 0; q < nb; ++q)
              for (int s2 = 0; s2 < nb; ++s2) {
                cplx const bj = std::conj(b[a * nb + j]), bp = std::conj(b[a * nb + p]), br = std::conj(b[a * nb + r]);
                cplx const bi = b[a * nb + i], bq = b[a * nb + q], bs = b[a * nb + s2];
                cplx const ss123 = bj * dot(vs, vs, a, p, q, r, s2) * bi, so123 = bj * dot(vs, vo, a, p, q, r, s2) * bi,
                           oo123 = bj * dot(vo, vo, a, p, q, r, s2) * bi;
                cplx const ss213 = bp * dot(vs, vs, a, j, i, r, s2) * bq, so213 = bp * dot(vs, vo, a, j, i, r, s2) * bq,
                           oo213 = bp * dot(vo, vo, a, j, i, r, s2) * bq;
                cplx const ss312 = br * dot(vs, vs, a, j, i, p, q) * bs, so312 = br * dot(vs, vo, a, j, i, p, q) * bs,
                           oo312 = br * dot(vo, vo, a, j, i, p, q) * bs;
                int64_t const o = ((((int64_t(j) * nb + p) * nb + r) * nb + i) * nb + q) * nb + s2;
                ss[o] += w * (ss123 + ss213 + ss312);
                so[o] += w * (so123 + so213 + so312);
                oo[o] += w * (oo123 + oo213 + oo312);
              }
    }
}

// assembleG (HartreeFock.cpp:687-752) without its debugging checks: G3[spin][j][i] from the Q
// tensors and the spin densities D [2][nb][nb] (element (q, p) at [q][p]).
void oracle_assemble_g(int nb, double const * Qss, double const * Qso, double const * Qoo, double const * density, double * G3)
{
  cplx const * SS = reinterpret_cast<cplx const *>(Qss);
  cplx const * SO = reinterpret_cast<cplx const *>(Qso);
  cplx const * OO = reinterpret_cast<cplx const *>(Qoo);
  cplx const * D = reinterpret_cast<cplx const *>(density);
  cplx * G = reinterpret_cast<cplx *>(G3);
  int64_t const nn = int64_t(nb) * nb;
  auto Q = [&](cplx const * T, int j, int p, int r, int x, int y, int z) {
    return T[((((int64_t(j) * nb + p) * nb + r) * nb + x) * nb + y) * nb + z];
  };
  auto Dm = [&](int spin, int x, int y) { return D[spin * nn + int64_t(x) * nb + y]; };
  for (int j = 0; j < nb; ++j)
    for (int i = 0; i < nb; ++i) {
      cplx value[2] = {0.0, 0.0};
      for (int p = 0; p < nb; ++p)
        for (int q = 0; q < nb; ++q)
          for (int r = 0; r < nb; ++r)
            for (int s2 = 0; s2 < nb; ++s2)
              for (int spin = 0; spin < 2; ++spin) {
                value[spin] += Dm(spin, q, p) * Dm(spin, s2, r) *
                               (Q(SS, j, p, r, i, q, s2) - Q(SS, j, p, r, i, s2, q) + 2.0 * Q(SS, j, p, r, q, s2, i) - 2.0 * Q(SS, j, p, r, s2, q, i));
                value[spin] += 2.0 * Dm(spin, q, p) * Dm(!spin, s2, r) * (Q(SO, j, p, r, i, q, s2) - Q(SO, j, p, r, q, i, s2));
                value[spin] += Dm(!spin, q, p) * Dm(!spin, s2, r) * (Q(OO, j, p, r, i, q, s2) - Q(OO, j, p, r, i, s2, q));
              }
      G[0 * nn + int64_t(j) * nb + i] = value[0] / 2.0;
      G[1 * nn + int64_t(j) * nb + i] = value[1] / 2.0;
    }
}

} // extern "C"
