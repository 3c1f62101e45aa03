// The reference's own hot-path code, compiled from its sources where they lie (src/HartreeFock.cpp,
// which includes src/HartreeFock.hpp and the src/integration headers) over the LvArray / RAJA /
// Caliper / qmc stand-ins in oracle/ref_shim/, with C entry points that take the oracle's array
// layouts.  Test infrastructure only: the tests pin the oracle's restatement (tcscf_oracle.cpp) to
// these functions.  Built by `make ref` into oracle/_ref/ where the reference sources are present.
//
// Each entry point builds the reference's QMCGrid objects and then replaces their points, weights,
// basis values and gradients with the caller's, so the reference's templates run on exactly the
// oracle's inputs:
//   tcscf_ref_compute_F  precomputeIntegrand + computeF (HartreeFock.hpp:23-180) with the kernels of
//                        the reference's tests (1/r12: HartreeFockTest.cpp:248-253; the TC scalar
//                        kernels: :274-295), 2-D real or 3-D complex r2 grids
//   tcscf_ref_compute_V  precomputeIntegrand + computeV (HartreeFock.hpp:185-229) with grad u
//                        (HartreeFockTest.cpp:299-317)
//   tcscf_ref_scf        RCSHartreeFock / UOSHartreeFock::compute (HartreeFock.cpp:785-1003): the SCF
//                        loop with calculateIaa / calculateFai, the Fock assembly, constructSCFOperator
//                        and zhegvd
//   tcscf_ref_tc_scf     TCHartreeFock::compute (HartreeFock.cpp:1007-1362) with zggev
//   tcscf_ref_qmc_grid   the QMCGrid constructor (integrateAll.hpp:21-63: createGrid with the
//                        TreutlerAhlrichsM4 / azimuthal / linear maps, then the r^2 sin(theta) jacobian)
//                        on the caller's unit-cube points
//   tcscf_ref_sto_values QMCGrid::setBasisFunctions (integrateAll.hpp:88-137) with SlaterTypeOrbital
//                        values and gradients (SlaterTypeOrbital.hpp:16-112) on the caller's points
//   tcscf_ref_overlap_core  the analytic STO overlap and core-Hamiltonian elements
//                        (SlaterTypeOrbital.hpp:118-176)
//   tcscf_ref_family_values / tcscf_ref_family_overlap_core  the same for the Ochi and hydrogen-like
//                        families (OchiBasis.hpp, HydrogenLikeBasis.hpp), the core elements on the
//                        grid of the reference's driver (ChebyshevGauss(1000) with TreutlerAhlrichsM4(1,
//                        0.9), HartreeFockTest.cpp:363-365)
//   tcscf_ref_integrate_all_r1r2, tcscf_ref_three_electron_integrals  the 4- and 6-index tensors
//                        (integrateAll.hpp:152-442)
//   tcscf_ref_compute_q, tcscf_ref_assemble_g  the 3-body verification route (HartreeFock.cpp:613-752)
//   tcscf_ref_radial_grid  createGrid(ChebyshevGauss(n), map) (quadrature.hpp:75-104, ChebyshevGauss.hpp)
//                        with the None, Linear, XOver1mX or TreutlerAhlrichsM4 change of variables
//   tcscf_ref_load_sto   loadSTO (SlaterTypeOrbital.cpp:24-75), and tcscf_ref_basis_library the
//                        reference's basis-set library directory the build was given
// Array layouts (row-major, complex as interleaved doubles): points [ndim][N]; weights [N]; basis
// values [N][nb] (complex for 3-D grids, real for 2-D); gradients [N][nb][3] complex; F [N1][nb][nb]
// (real for 2-D r2, complex for 3-D); V [N1][nb][nb][3] complex; S, h [nb][nb] real; density
// [nspin][nb][nb] complex.
#include <dlfcn.h>

#include "HartreeFock.cpp"
#include "SlaterTypeOrbital.cpp"
#include "SlaterTypeOrbital.hpp"
#include "OchiBasis.hpp"
#include "HydrogenLikeBasis.hpp"
#include "integration/ChebyshevGauss.hpp"
#include "jastrowFunctions.hpp"

namespace {

using namespace tcscf;
using cplx = std::complex<double>;

// the oracle's basis-function record (tcscf_oracle.cpp; family 0 = STO)
struct StoParams {
  double alpha;
  int32_t n, l, m, family;
};

std::vector<SlaterTypeOrbital<double>> makeStos(StoParams const * b, int nb)
{
  std::vector<SlaterTypeOrbital<double>> out;
  for (int i = 0; i < nb; ++i) out.emplace_back(b[i].alpha, b[i].n, b[i].l, b[i].m);
  return out;
}

// the oracle's Ochi parameter block (tcscf_oracle.cpp)
struct OchiParams {
  double a, a12;
  int32_t nterms, pad;
  int32_t S[8][3];
  double c[8][2];   // [term][0 = opposite spin, 1 = same spin]
};

jastrowFunctions::Ochi<double> makeOchi(OchiParams const & p)
{
  Array2d<double> c(p.nterms, 2);
  Array2d<int> S(p.nterms, 3);
  for (int t = 0; t < p.nterms; ++t) {
    c(t, 0) = p.c[t][0];
    c(t, 1) = p.c[t][1];
    for (int d = 0; d < 3; ++d) S(t, d) = p.S[t][d];
  }
  return jastrowFunctions::Ochi<double> {p.a, p.a12, c, S};
}

template <int NDIM>
integration::QMCGrid<double, NDIM> makeGrid(double const * pts, double const * w, int64_t n, double const * vals, double const * grads, int nb)
{
  integration::QMCGrid<double, NDIM> g(1);
  g.quadratureGrid = integration::QuadratureGrid<double>(NDIM, int(n));
  for (int d = 0; d < NDIM; ++d)
    for (int64_t i = 0; i < n; ++i) g.quadratureGrid.points(d, i) = pts[d * n + i];
  for (int64_t i = 0; i < n; ++i) g.quadratureGrid.weights(i) = w[i];
  g.basisValues.resize(n, nb);
  for (int64_t i = 0; i < n; ++i)
    for (int b = 0; b < nb; ++b) {
      if constexpr (NDIM == 3)
        g.basisValues(i, b) = cplx(vals[2 * (i * nb + b)], vals[2 * (i * nb + b) + 1]);
      else
        g.basisValues(i, b) = vals[i * nb + b];
    }
  if (grads) {
    g.basisGradients.resize(n, nb);
    for (int64_t i = 0; i < n; ++i)
      for (int b = 0; b < nb; ++b) {
        double const * q = grads + 6 * (i * nb + b);
        g.basisGradients(i, b) = Cartesian<cplx> {cplx(q[0], q[1]), cplx(q[2], q[3]), cplx(q[4], q[5])};
      }
  }
  return g;
}

// The kernels of the reference's tests: 1/r12 (kernel 0) and the TC scalar kernels 2/r12 - |grad_12 u|^2
// - |grad_21 u|^2 for same (1) and opposite (2) spins.
template <typename GRID2>
Array2d<double> scalarIntegrand(integration::QMCGrid<double, 3> const & g1, GRID2 const & g2, int kernel, OchiParams const * up)
{
  Array2d<double> values(g1.nGrid(), g2.nGrid());
  if (kernel == 0) {
    precomputeIntegrand(values.toView(), g1, g2, [](Cartesian<double> const & r1, Cartesian<double> const & r2) { return 1 / (r1 - r2).r(); });
  } else {
    jastrowFunctions::Ochi<double> const u = makeOchi(*up);
    bool const same = kernel == 1;
    precomputeIntegrand(values.toView(), g1, g2, [&u, same](Cartesian<double> const & r1, Cartesian<double> const & r2) {
      Cartesian<double> const grad12 = u.gradient(r1, r2, same);
      Cartesian<double> const grad21 = u.gradient(r2, r1, same);
      return 2 / (r1 - r2).r() - dot(grad12, grad12) - dot(grad21, grad21);
    });
  }
  return values;
}

// Calls body with the reference test's kernel as a lambda of (r1, r2): 1/r12 (0), the TC scalar kernels
// (1 same spin, 2 opposite) or grad u (3 same, 4 opposite)
template <typename BODY>
void withKernel(int kernel, OchiParams const * up, BODY && body)
{
  if (kernel == 0) {
    body([](Cartesian<double> const & r1, Cartesian<double> const & r2) { return 1 / (r1 - r2).r(); });
    return;
  }
  jastrowFunctions::Ochi<double> const u = makeOchi(*up);
  if (kernel <= 2) {
    bool const same = kernel == 1;
    body([&u, same](Cartesian<double> const & r1, Cartesian<double> const & r2) {
      Cartesian<double> const grad12 = u.gradient(r1, r2, same);
      Cartesian<double> const grad21 = u.gradient(r2, r1, same);
      return 2 / (r1 - r2).r() - dot(grad12, grad12) - dot(grad21, grad21);
    });
  } else {
    bool const same = kernel == 3;
    body([&u, same](Cartesian<double> const & r1, Cartesian<double> const & r2) { return u.gradient(r1, r2, same); });
  }
}

template <typename T, int N, typename A>
void copyOut(A const & a, int64_t count, double * out)
{
  T const * d = a.data();
  for (int64_t k = 0; k < count; ++k) {
    out[2 * k] = d[k].real();
    out[2 * k + 1] = d[k].imag();
  }
}

template <typename F>
int guarded(F && f)
{
  try {
    return f();
  } catch (std::exception const & e) {
    std::fprintf(stderr, "tcscf_ref: %s\n", e.what());
    return -1;
  }
}

}  // namespace

extern "C" {

// LAPACK (zhegvd, zggev) from a shared library, e.g. scipy's bundled OpenBLAS; 0 on success
int tcscf_ref_set_lapack(char const * path)
{
  void * h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!h) return -1;
  using namespace LvArray::dense::lapack;
  zhegvd() = reinterpret_cast<zhegvd_t>(dlsym(h, "scipy_zhegvd_"));
  if (!zhegvd()) zhegvd() = reinterpret_cast<zhegvd_t>(dlsym(h, "zhegvd_"));
  zggev() = reinterpret_cast<zggev_t>(dlsym(h, "scipy_zggev_"));
  if (!zggev()) zggev() = reinterpret_cast<zggev_t>(dlsym(h, "zggev_"));
  return (zhegvd() && zggev()) ? 0 : -2;
}

int tcscf_ref_compute_F(double const * p1, double const * w1, int64_t N1, double const * vals1, double const * p2, double const * w2,
                        int64_t N2, int ndim2, double const * vals2, int nb, int kernel, OchiParams const * u, double * F)
{
  return guarded([&] {
    auto const g1 = makeGrid<3>(p1, w1, N1, vals1, nullptr, nb);
    if (ndim2 == 2) {
      auto const g2 = makeGrid<2>(p2, w2, N2, vals2, nullptr, nb);
      Array2d<double> const values = scalarIntegrand(g1, g2, kernel, u);
      Array3d<double> const out = computeF(g1, g2, values.toViewConst());
      for (int64_t a = 0; a < N1; ++a)
        for (int j = 0; j < nb; ++j)
          for (int i = 0; i < nb; ++i) F[(a * nb + j) * nb + i] = out(a, j, i);
    } else {
      auto const g2 = makeGrid<3>(p2, w2, N2, vals2, nullptr, nb);
      Array2d<double> const values = scalarIntegrand(g1, g2, kernel, u);
      Array3d<cplx> const out = computeF(g1, g2, values.toViewConst());
      for (int64_t a = 0; a < N1; ++a)
        for (int j = 0; j < nb; ++j)
          for (int i = 0; i < nb; ++i) {
            cplx const v = out(a, j, i);
            F[2 * ((a * nb + j) * nb + i)] = v.real();
            F[2 * ((a * nb + j) * nb + i) + 1] = v.imag();
          }
    }
    return 0;
  });
}

// kernel 3: grad u same spin, 4: opposite spin
int tcscf_ref_compute_V(double const * p1, double const * w1, int64_t N1, double const * vals1, double const * p2, double const * w2,
                        int64_t N2, double const * vals2, int nb, int kernel, OchiParams const * up, double * V)
{
  return guarded([&] {
    auto const g1 = makeGrid<3>(p1, w1, N1, vals1, nullptr, nb);
    auto const g2 = makeGrid<3>(p2, w2, N2, vals2, nullptr, nb);
    jastrowFunctions::Ochi<double> const u = makeOchi(*up);
    bool const same = kernel == 3;
    Array2d<Cartesian<double>> values(N1, N2);
    precomputeIntegrand(values.toView(), g1, g2,
                        [&u, same](Cartesian<double> const & r1, Cartesian<double> const & r2) { return u.gradient(r1, r2, same); });
    Array3d<Cartesian<cplx>> const out = computeV(g1, g2, values.toViewConst());
    for (int64_t a = 0; a < N1; ++a)
      for (int j = 0; j < nb; ++j)
        for (int i = 0; i < nb; ++i) {
          Cartesian<cplx> const v = out(a, j, i);
          double * o = V + 6 * ((a * nb + j) * nb + i);
          cplx const c[3] = {v.x(), v.y(), v.z()};
          for (int d = 0; d < 3; ++d) {
            o[2 * d] = c[d].real();
            o[2 * d + 1] = c[d].imag();
          }
        }
    return 0;
  });
}

// RCS (nspin 1) or UOS (nspin 2) SCF on a real F [N1][nb][nb]; returns the driver's convergence-loop
// count, or -1 when it threw (non-convergence included)
int tcscf_ref_scf(int nspin, int nup, int ndown, double const * F, double const * p1, double const * w1, int64_t N1, int nb,
                  double const * vals1, double const * S, double const * h, int respectSym, double * energy, double * density)
{
  return guarded([&] {
    auto const g1 = makeGrid<3>(p1, w1, N1, vals1, nullptr, nb);
    Array3d<double> Fji(N1, nb, nb);
    for (int64_t a = 0; a < N1; ++a)
      for (int j = 0; j < nb; ++j)
        for (int i = 0; i < nb; ++i) Fji(a, j, i) = F[(a * nb + j) * nb + i];
    Array2d<cplx, RAJA::PERM_JI> overlap(nb, nb);
    Array2d<double> H(nb, nb);
    for (int j = 0; j < nb; ++j)
      for (int i = 0; i < nb; ++i) {
        overlap(j, i) = S[j * nb + i];
        H(j, i) = h[j * nb + i];
      }
    auto copyDensity = [&](auto const & D) {
      for (int s = 0; s < nspin; ++s)
        for (int j = 0; j < nb; ++j)
          for (int i = 0; i < nb; ++i) {
            cplx const v = D(s, j, i);
            density[2 * ((s * nb + j) * nb + i)] = v.real();
            density[2 * ((s * nb + j) * nb + i) + 1] = v.imag();
          }
    };
    if (nspin == 1) {
      RCSHartreeFock<cplx> hf(nup + ndown, nb);
      *energy = hf.compute(overlap.toViewConst(), H.toViewConst(), g1, Fji.toViewConst(), respectSym != 0);
      copyDensity(hf.density);
      return hf.numberOfConvergenceLoops();
    }
    UOSHartreeFock<cplx> hf(nup, ndown, nb);
    *energy = hf.compute(overlap.toViewConst(), H.toViewConst(), g1, Fji.toViewConst(), respectSym != 0);
    copyDensity(hf.density);
    return hf.numberOfConvergenceLoops();
  });
}

// TC SCF on real FjiSame / FjiOppo [N1][nb][nb] and complex VjiSame / VjiOppo [N1][nb][nb][3]
int tcscf_ref_tc_scf(double const * FjiSame, double const * FjiOppo, double const * VjiSame, double const * VjiOppo, double const * p1,
                     double const * w1, int64_t N1, int nb, double const * vals1, double const * grads1, double const * S,
                     double const * h, int nup, int ndown, int respectSym, double * energy, double * density)
{
  return guarded([&] {
    auto const g1 = makeGrid<3>(p1, w1, N1, vals1, grads1, nb);
    Array3d<double> Fs(N1, nb, nb), Fo(N1, nb, nb);
    Array3d<Cartesian<cplx>> Vs(N1, nb, nb), Vo(N1, nb, nb);
    for (int64_t a = 0; a < N1; ++a)
      for (int j = 0; j < nb; ++j)
        for (int i = 0; i < nb; ++i) {
          int64_t const k = (a * nb + j) * nb + i;
          Fs(a, j, i) = FjiSame[k];
          Fo(a, j, i) = FjiOppo[k];
          double const * s = VjiSame + 6 * k;
          double const * o = VjiOppo + 6 * k;
          Vs(a, j, i) = Cartesian<cplx> {cplx(s[0], s[1]), cplx(s[2], s[3]), cplx(s[4], s[5])};
          Vo(a, j, i) = Cartesian<cplx> {cplx(o[0], o[1]), cplx(o[2], o[3]), cplx(o[4], o[5])};
        }
    Array2d<cplx, RAJA::PERM_JI> overlap(nb, nb);
    Array2d<double> H(nb, nb);
    for (int j = 0; j < nb; ++j)
      for (int i = 0; i < nb; ++i) {
        overlap(j, i) = S[j * nb + i];
        H(j, i) = h[j * nb + i];
      }
    TCHartreeFock<cplx> hf(nup, ndown, nb);
    *energy = hf.compute(overlap.toViewConst(), H.toViewConst(), g1, Fs.toViewConst(), Fo.toViewConst(), Vs.toViewConst(), Vo.toViewConst(),
                         respectSym != 0);
    for (int s = 0; s < 2; ++s)
      for (int j = 0; j < nb; ++j)
        for (int i = 0; i < nb; ++i) {
          cplx const v = hf.density(s, j, i);
          density[2 * ((s * nb + j) * nb + i)] = v.real();
          density[2 * ((s * nb + j) * nb + i) + 1] = v.imag();
        }
    return hf.numberOfConvergenceLoops();
  });
}

// points [ndim][N] and weights [N] of the reference's QMC grid built from the unit-cube points u [ndim][N]
int tcscf_ref_qmc_grid(int ndim, int64_t N, double const * u, double * pts, double * w)
{
  return guarded([&] {
    auto & given = integrators::providedPoints();
    given.assign(size_t(N), std::vector<double>(size_t(ndim)));
    for (int64_t i = 0; i < N; ++i)
      for (int d = 0; d < ndim; ++d) given[size_t(i)][size_t(d)] = u[d * N + i];
    auto readBack = [&](auto const & g) {
      LVARRAY_ERROR_IF_NE(g.quadratureGrid.weights.size(), N);
      for (int d = 0; d < ndim; ++d)
        for (int64_t i = 0; i < N; ++i) pts[d * N + i] = g.quadratureGrid.points(d, i);
      for (int64_t i = 0; i < N; ++i) w[i] = g.quadratureGrid.weights(i);
    };
    if (ndim == 2)
      readBack(integration::QMCGrid<double, 2>(N));
    else
      readBack(integration::QMCGrid<double, 3>(N));
    given.clear();
    return 0;
  });
}

// STO values [N][nb] (complex for ndim 3, real for ndim 2) and, when grads is not null, gradients
// [N][nb][3] complex on the points [ndim][N]
int tcscf_ref_sto_values(int ndim, int64_t N, double const * pts, StoParams const * basis, int nb, double * vals, double * grads)
{
  return guarded([&] {
    std::vector<SlaterTypeOrbital<double>> const stos = makeStos(basis, nb);
    std::vector<double> const zeros(size_t(N), 0.0);
    auto run = [&](auto & g) {
      for (int d = 0; d < ndim; ++d)
        for (int64_t i = 0; i < N; ++i) g.quadratureGrid.points(d, i) = pts[d * N + i];
      g.setBasisFunctions(stos, grads != nullptr);
      for (int64_t i = 0; i < N; ++i)
        for (int b = 0; b < nb; ++b) {
          auto const v = g.basisValues(i, b);
          if constexpr (std::is_same_v<std::decay_t<decltype(v)>, cplx>) {
            vals[2 * (i * nb + b)] = v.real();
            vals[2 * (i * nb + b) + 1] = v.imag();
          } else {
            vals[i * nb + b] = v;
          }
          if (grads) {
            Cartesian<cplx> const q = g.basisGradients(i, b);
            cplx const c[3] = {q.x(), q.y(), q.z()};
            for (int d = 0; d < 3; ++d) {
              grads[6 * (i * nb + b) + 2 * d] = c[d].real();
              grads[6 * (i * nb + b) + 2 * d + 1] = c[d].imag();
            }
          }
        }
    };
    if (ndim == 2) {
      auto g = makeGrid<2>(pts, zeros.data(), N, nullptr, nullptr, 0);
      run(g);
    } else {
      auto g = makeGrid<3>(pts, zeros.data(), N, nullptr, nullptr, 0);
      run(g);
    }
    return 0;
  });
}

// analytic S and core H [nb][nb] (row j, column i) for nuclear charge Z
int tcscf_ref_overlap_core(StoParams const * basis, int nb, int Z, double * S, double * H)
{
  return guarded([&] {
    std::vector<SlaterTypeOrbital<double>> const stos = makeStos(basis, nb);
    for (int j = 0; j < nb; ++j)
      for (int i = 0; i < nb; ++i) {
        S[j * nb + i] = overlap(stos[size_t(j)], stos[size_t(i)]);
        H[j * nb + i] = coreMatrixElement(Z, stos[size_t(j)], stos[size_t(i)]);
      }
    return 0;
  });
}

// values [N][nb] (complex for ndim 3, real for ndim 2) and, for the Ochi family when grads is not null,
// gradients [N][nb][3] of Ochi (family 1, alpha the exponent) or hydrogen-like (family 2, alpha the
// nuclear charge) functions
int tcscf_ref_family_values(int ndim, int64_t N, double const * pts, StoParams const * basis, int nb, double * vals, double * grads)
{
  return guarded([&] {
    std::vector<double> const zeros(size_t(N), 0.0);
    auto run = [&](auto & g, auto const & fns) {
      for (int d = 0; d < ndim; ++d)
        for (int64_t i = 0; i < N; ++i) g.quadratureGrid.points(d, i) = pts[d * N + i];
      g.setBasisFunctions(fns, grads != nullptr);
      for (int64_t i = 0; i < N; ++i)
        for (int b = 0; b < nb; ++b) {
          auto const v = g.basisValues(i, b);
          if constexpr (std::is_same_v<std::decay_t<decltype(v)>, cplx>) {
            vals[2 * (i * nb + b)] = v.real();
            vals[2 * (i * nb + b) + 1] = v.imag();
          } else {
            vals[i * nb + b] = v;
          }
          if (grads) {
            Cartesian<cplx> const q = g.basisGradients(i, b);
            cplx const c[3] = {q.x(), q.y(), q.z()};
            for (int d = 0; d < 3; ++d) {
              grads[6 * (i * nb + b) + 2 * d] = c[d].real();
              grads[6 * (i * nb + b) + 2 * d + 1] = c[d].imag();
            }
          }
        }
    };
    auto byFamily = [&](auto & g) {
      if (basis[0].family == 1) {
        std::vector<OchiBasisFunction<double>> fns;
        for (int i = 0; i < nb; ++i) fns.emplace_back(basis[i].alpha, basis[i].n, basis[i].l, basis[i].m);
        run(g, fns);
      } else {
        std::vector<HydrogenLikeBasisFunction<double>> fns;
        for (int i = 0; i < nb; ++i) fns.emplace_back(int(basis[i].alpha), basis[i].n, basis[i].l, basis[i].m);
        run(g, fns);
      }
    };
    if (ndim == 2) {
      auto g = makeGrid<2>(pts, zeros.data(), N, nullptr, nullptr, 0);
      byFamily(g);
    } else {
      auto g = makeGrid<3>(pts, zeros.data(), N, nullptr, nullptr, 0);
      byFamily(g);
    }
    return 0;
  });
}

// S and core H [nb][nb] of an Ochi (family 1) or hydrogen-like (family 2) basis as the reference's driver
// fills them; S of the hydrogen-like family is the generic numerical overlap and is not computed (NaN)
int tcscf_ref_family_overlap_core(StoParams const * basis, int nb, int Z, double * S, double * H)
{
  return guarded([&] {
    integration::QuadratureGrid<double> const coreGrid =
        integration::createGrid(integration::ChebyshevGauss<double>(1000), integration::changeOfVariables::TreutlerAhlrichsM4<double>(1, 0.9));
    if (basis[0].family == 1) {
      std::vector<OchiBasisFunction<double>> fns;
      for (int i = 0; i < nb; ++i) fns.emplace_back(basis[i].alpha, basis[i].n, basis[i].l, basis[i].m);
      for (int i = 0; i < nb; ++i)
        for (int j = 0; j < nb; ++j) {
          S[i * nb + j] = overlap(fns[size_t(i)], fns[size_t(j)]);
          H[i * nb + j] = coreMatrixElement(coreGrid, Z, fns[size_t(i)], fns[size_t(j)]);
        }
    } else {
      std::vector<HydrogenLikeBasisFunction<double>> fns;
      for (int i = 0; i < nb; ++i) fns.emplace_back(int(basis[i].alpha), basis[i].n, basis[i].l, basis[i].m);
      for (int i = 0; i < nb; ++i)
        for (int j = 0; j < nb; ++j) {
          S[i * nb + j] = std::numeric_limits<double>::quiet_NaN();
          H[i * nb + j] = coreMatrixElement(coreGrid, Z, fns[size_t(i)], fns[size_t(j)]);
        }
    }
    return 0;
  });
}

// integrateAllR1R2<use_gradient>: r1 3-D (complex values), r2 2-D (real values; complex gradients
// [N2][nb][3] for use_gradient), the kernel of withKernel (scalar kernels 0-2 without, grad u 3-4 with
// gradients); answer [nb]^4 complex
int tcscf_ref_integrate_all_r1r2(int useGradient, double const * p1, double const * w1, int64_t N1, double const * vals1, double const * p2,
                                 double const * w2, int64_t N2, double const * vals2, double const * grads2, int nb, int kernel,
                                 OchiParams const * u, double * out)
{
  return guarded([&] {
    auto const g1 = makeGrid<3>(p1, w1, N1, vals1, nullptr, nb);
    auto const g2 = makeGrid<2>(p2, w2, N2, vals2, useGradient ? grads2 : nullptr, nb);
    int64_t const n4 = int64_t(nb) * nb * nb * nb;
    withKernel(kernel, u, [&](auto && f) {
      using R = decltype(f(Cartesian<double> {}, Cartesian<double> {}));
      if constexpr (std::is_same_v<R, double>) {
        LVARRAY_ERROR_IF(useGradient, "integrateAllR1R2: a scalar kernel takes the value form");
        Array4d<cplx> const a = integration::integrateAllR1R2<false>(g1, g2, f);
        copyOut<cplx, 4>(a, n4, out);
      } else {
        LVARRAY_ERROR_IF(!useGradient, "integrateAllR1R2: a vector kernel takes the gradient form");
        Array4d<cplx> const a = integration::integrateAllR1R2<true>(g1, g2, f);
        copyOut<cplx, 4>(a, n4, out);
      }
    });
    return 0;
  });
}

// threeElectronIntegrals with the Ochi Jastrow factor: r1, r2 3-D grids; answer [nb]^6 complex
int tcscf_ref_three_electron_integrals(double const * p1, double const * w1, int64_t N1, double const * vals1, double const * p2,
                                       double const * w2, int64_t N2, double const * vals2, int nb, OchiParams const * up, double * out)
{
  return guarded([&] {
    auto const g1 = makeGrid<3>(p1, w1, N1, vals1, nullptr, nb);
    auto const g2 = makeGrid<3>(p2, w2, N2, vals2, nullptr, nb);
    jastrowFunctions::Ochi<double> const u = makeOchi(*up);
    Array6d<cplx> const a = integration::threeElectronIntegrals(g1, g2, u);
    int64_t const n6 = int64_t(nb) * nb * nb * nb * nb * nb;
    copyOut<cplx, 6>(a, n6, out);
    return 0;
  });
}

// internal::computeQ: Q same-same, same-opposite, opposite-opposite [nb]^6 complex from the grad-u
// tensors Vs, Vo [N1][nb][nb][3] complex, the r1 weights and basis values [N1][nb] complex
int tcscf_ref_compute_q(int64_t N1, int nb, double const * w1, double const * vals1, double const * Vs, double const * Vo, double * Qss,
                        double * Qso, double * Qoo)
{
  return guarded([&] {
    Array1d<double> W(N1);
    Array2d<cplx> B(N1, nb);
    Array3d<Cartesian<cplx>> S3(N1, nb, nb), O3(N1, nb, nb);
    for (int64_t a = 0; a < N1; ++a) {
      W(a) = w1[a];
      for (int b = 0; b < nb; ++b) B(a, b) = cplx(vals1[2 * (a * nb + b)], vals1[2 * (a * nb + b) + 1]);
      for (int j = 0; j < nb; ++j)
        for (int i = 0; i < nb; ++i) {
          int64_t const k = (a * nb + j) * nb + i;
          double const * s = Vs + 6 * k;
          double const * o = Vo + 6 * k;
          S3(a, j, i) = Cartesian<cplx> {cplx(s[0], s[1]), cplx(s[2], s[3]), cplx(s[4], s[5])};
          O3(a, j, i) = Cartesian<cplx> {cplx(o[0], o[1]), cplx(o[2], o[3]), cplx(o[4], o[5])};
        }
    }
    Array6d<cplx> qss(nb, nb, nb, nb, nb, nb), qso(nb, nb, nb, nb, nb, nb), qoo(nb, nb, nb, nb, nb, nb);
    internal::computeQ(qss.toView(), qso.toView(), qoo.toView(), S3.toViewConst(), O3.toViewConst(), W.toViewConst(), B.toViewConst());
    int64_t const n6 = int64_t(nb) * nb * nb * nb * nb * nb;
    copyOut<cplx, 6>(qss, n6, Qss);
    copyOut<cplx, 6>(qso, n6, Qso);
    copyOut<cplx, 6>(qoo, n6, Qoo);
    return 0;
  });
}

// internal::assembleG: G3 [2][nb][nb] complex from the Q tensors and the spin densities [2][nb][nb]
int tcscf_ref_assemble_g(int nb, double const * Qss, double const * Qso, double const * Qoo, double const * density, double * G3)
{
  return guarded([&] {
    int64_t const n6 = int64_t(nb) * nb * nb * nb * nb * nb;
    Array6d<cplx> qss(nb, nb, nb, nb, nb, nb), qso(nb, nb, nb, nb, nb, nb), qoo(nb, nb, nb, nb, nb, nb);
    for (int64_t k = 0; k < n6; ++k) {
      qss.data()[k] = cplx(Qss[2 * k], Qss[2 * k + 1]);
      qso.data()[k] = cplx(Qso[2 * k], Qso[2 * k + 1]);
      qoo.data()[k] = cplx(Qoo[2 * k], Qoo[2 * k + 1]);
    }
    Array3d<cplx> D(2, nb, nb), G(2, nb, nb);
    for (int64_t k = 0; k < 2 * int64_t(nb) * nb; ++k) D.data()[k] = cplx(density[2 * k], density[2 * k + 1]);
    internal::assembleG(G.toView(), qss.toViewConst(), qso.toViewConst(), qoo.toViewConst(), D.toViewConst());
    copyOut<cplx, 3>(G, 2 * int64_t(nb) * nb, G3);
    return 0;
  });
}

// points u [n] and weights w [n] of createGrid(ChebyshevGauss(n), map), map 0 None, 1 Linear(p0),
// 2 XOver1mX, 3 TreutlerAhlrichsM4(p0, p1)
int tcscf_ref_radial_grid(int n, int map, double p0, double p1, double * u, double * w)
{
  return guarded([&] {
    using namespace integration;
    auto store = [&](QuadratureGrid<double> const & g) {
      LVARRAY_ERROR_IF_NE(g.weights.size(), n);
      for (int i = 0; i < n; ++i) {
        u[i] = g.points(0, i);
        w[i] = g.weights(i);
      }
    };
    ChebyshevGauss<double> const cg(n);
    if (map == 0) store(createGrid(cg, changeOfVariables::None<double, 1> {}));
    else if (map == 1) store(createGrid(cg, changeOfVariables::Linear<double> {p0}));
    else if (map == 2) store(createGrid(cg, changeOfVariables::XOver1mX<double> {}));
    else if (map == 3) store(createGrid(cg, changeOfVariables::TreutlerAhlrichsM4<double>(p0, p1)));
    else throw std::runtime_error("radial map not in the reference");
    return 0;
  });
}

// loadSTO(directory, basisSet, element, maxL): the number of functions (at most maxOut written to out,
// family 0), or -1 when the reference's loader rejected the arguments
int tcscf_ref_load_sto(char const * directory, char const * basisSet, char const * element, int maxL, StoParams * out, int maxOut)
{
  try {
    std::vector<SlaterTypeOrbital<double>> const b = loadSTO(directory, basisSet, element, maxL);
    for (size_t i = 0; i < b.size() && int(i) < maxOut; ++i) out[i] = StoParams {b[i].alpha, b[i].n, b[i].l, b[i].m, 0};
    return int(b.size());
  } catch (std::exception const &) {
    return -1;
  }
}

// the reference's basis-set library directory (basisFunctions/ beside its src/), or "" when the build was
// not told
char const * tcscf_ref_basis_library()
{
#ifdef TCSCF_REF_BASIS_DIR
  return TCSCF_REF_BASIS_DIR;
#else
  return "";
#endif
}

}  // extern "C"
