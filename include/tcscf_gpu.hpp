/*
 * tcscf_gpu.hpp — header-only C++17 host layer over the C ABI of libtcscf_gpu.so (tcscf_gpu.h),
 * with the names of corbett5/tcscf's integration and SCF interface:
 *   QMCGrid / setBasisFunctions / basisValues        src/integration/integrateAll.hpp:12-142
 *   computeF / computeV (precomputeIntegrand)         src/HartreeFock.hpp:23-229
 *   integrateAllR1R2 / threeElectronIntegrals         src/integration/integrateAll.hpp:147-442
 *   RCSHartreeFock / UOSHartreeFock::compute          src/HartreeFock.hpp:233-349, HartreeFock.cpp:785-1003
 *   TCHartreeFock::compute                            src/HartreeFock.hpp:353-394, HartreeFock.cpp:1007-1362
 *   loadSTO                                           src/SlaterTypeOrbital.cpp:24-75
 *   overlap / coreMatrixElement                       src/SlaterTypeOrbital.hpp:134-181
 *
 * Inputs are contiguous arrays passed as any type with data() and size() (std::vector, std::span, or
 * an LvArray view); the layouts are those of tcscf_gpu.h.  Complex arrays are std::complex<double>.
 * Failures throw, as the reference throws or aborts: ConvergenceError for an SCF that did not
 * converge (HartreeFock.hpp:13-19), LinearAlgebraError for an eigen-solver failure (LvArray's
 * dense::Error), Error with the status code for everything else.  One Context per host thread; the
 * calls on a context are not reentrant.
 */
#ifndef TCSCF_GPU_HPP
#define TCSCF_GPU_HPP

#include <complex>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "tcscf_gpu.h"

namespace tcscf::gpu {

using cplx = std::complex<double>;

class Error : public std::runtime_error {
 public:
  Error(int code, std::string const & msg) : std::runtime_error("tcscf error " + std::to_string(code) + ": " + msg), code_(code) {}
  int code() const noexcept { return code_; }

 private:
  int code_;
};

class ConvergenceError : public Error {
 public:
  using Error::Error;
};

class LinearAlgebraError : public Error {
 public:
  using Error::Error;
};

inline void check(int code, tcscf_ctx * ctx)
{
  if (code == TCSCF_OK) return;
  std::string const msg = ctx ? tcscf_last_error(ctx) : "";
  if (code == TCSCF_ERR_NOT_CONVERGED) throw ConvergenceError(code, msg);
  if (code == TCSCF_ERR_LINALG) throw LinearAlgebraError(code, msg);
  throw Error(code, msg);
}

namespace detail {

inline double const * real(cplx const * p) { return reinterpret_cast<double const *>(p); }
inline double * real(cplx * p) { return reinterpret_cast<double *>(p); }

template <class V> void requireSize(V const & v, std::size_t n, char const * what)
{
  if (static_cast<std::size_t>(v.size()) != n) throw Error(TCSCF_ERR_INVALID_ARGUMENT, std::string(what) + " has the wrong size");
}

}  // namespace detail

// ---- host-side grids and basis sets ----------------------------------------------------------

// integration::QuadratureGrid (quadrature.hpp:25-35): points [ndim][N] and weights [N]
struct QuadratureGrid {
  int ndim = 3;
  std::vector<double> points;
  std::vector<double> weights;
  std::int64_t size() const { return static_cast<std::int64_t>(weights.size()); }
};

// createGrid(ChebyshevGauss(n), map) (quadrature.hpp:75-102): abscissae and weights
inline std::pair<std::vector<double>, std::vector<double>> radialGrid(int n, tcscf_map map, double p0 = 0.0, double p1 = 0.0)
{
  std::vector<double> u(n > 0 ? n : 0), w(n > 0 ? n : 0);
  check(tcscf_grid_radial(n, map, p0, p1, u.data(), w.data()), nullptr);
  return {std::move(u), std::move(w)};
}

// radial x angular product rule (TreutlerAhlrichsLebedev.hpp:18-74 with the caller's r^2); angular
// table nang x {theta, phi, weight}
template <class R, class A> QuadratureGrid productGrid(R const & r, R const & wr, A const & angular)
{
  detail::requireSize(wr, r.size(), "radial weights");
  if (angular.size() % 3 != 0) throw Error(TCSCF_ERR_INVALID_ARGUMENT, "angular table is not nang x 3");
  int const nrad = static_cast<int>(r.size()), nang = static_cast<int>(angular.size() / 3);
  QuadratureGrid g;
  g.points.resize(3 * std::size_t(nrad) * nang);
  g.weights.resize(std::size_t(nrad) * nang);
  check(tcscf_grid_product(nrad, r.data(), wr.data(), nang, angular.data(), g.points.data(), g.weights.data()), nullptr);
  return g;
}

// QMCGrid's point mapping of unit-cube points u [ndim][N] (integrateAll.hpp:21-65)
template <class U> QuadratureGrid qmcGrid(int ndim, U const & u)
{
  if (ndim <= 0 || u.size() % ndim != 0) throw Error(TCSCF_ERR_INVALID_ARGUMENT, "u is not [ndim][N]");
  std::int64_t const n = static_cast<std::int64_t>(u.size() / ndim);
  QuadratureGrid g;
  g.ndim = ndim;
  g.points.resize(std::size_t(ndim) * n);
  g.weights.resize(n);
  check(tcscf_grid_qmc(ndim, n, u.data(), g.points.data(), g.weights.data()), nullptr);
  return g;
}

// seeded scrambled Sobol points [ndim][n] in [0, 1)
inline std::vector<double> sobol(int ndim, std::int64_t n, std::uint64_t seed)
{
  std::vector<double> u(std::size_t(ndim > 0 ? ndim : 0) * std::size_t(n > 0 ? n : 0));
  check(tcscf_sobol(ndim, n, seed, u.data()), nullptr);
  return u;
}

// loadSTO (SlaterTypeOrbital.cpp:24-75): size query, then fill
inline std::vector<tcscf_sto> loadSTO(std::string const & directory, std::string const & basisSet, std::string const & element, int maxL)
{
  int n = 0;
  check(tcscf_load_sto(directory.c_str(), basisSet.c_str(), element.c_str(), maxL, nullptr, 0, &n), nullptr);
  std::vector<tcscf_sto> basis(n);
  check(tcscf_load_sto(directory.c_str(), basisSet.c_str(), element.c_str(), maxL, basis.data(), n, &n), nullptr);
  basis.resize(n);
  return basis;
}

// overlap and coreMatrixElement (SlaterTypeOrbital.hpp:134-181 and the Ochi / hydrogen-like forms):
// S and H real [nb][nb]
inline std::pair<std::vector<double>, std::vector<double>> overlapCore(std::vector<tcscf_sto> const & basis, int Z)
{
  std::size_t const nn = basis.size() * basis.size();
  std::vector<double> S(nn), H(nn);
  check(tcscf_overlap_core_analytic(basis.data(), static_cast<int>(basis.size()), Z, S.data(), H.data()), nullptr);
  return {std::move(S), std::move(H)};
}

// ---- device context, grids and tensors -------------------------------------------------------

class Context {
 public:
  explicit Context(int device = 0) { check(tcscf_ctx_create(device, &ctx_), nullptr); }
  ~Context() { tcscf_ctx_destroy(ctx_); }
  Context(Context const &) = delete;
  Context & operator=(Context const &) = delete;

  tcscf_ctx * handle() const { return ctx_; }
  void synchronize() { check(tcscf_synchronize(ctx_), ctx_); }
  // measured launch schedule of the tensor-core builds (off by default)
  void setAutotune(bool on) { check(tcscf_set_autotune(ctx_, on ? 1 : 0), ctx_); }
  // device ms of the last build's r12 contraction and of the whole call, kernels launched
  void lastTiming(double & contractionMs, double & totalMs, int & launches)
  {
    check(tcscf_last_timing(ctx_, &contractionMs, &totalMs, &launches), ctx_);
  }

 private:
  tcscf_ctx * ctx_ = nullptr;
};

// integration::QMCGrid<REAL, NDIM> with its basis values on the device
class QMCGrid {
 public:
  QMCGrid(Context & c, QuadratureGrid const & g) : ctx_(c.handle()), n_(g.size()), ndim_(g.ndim)
  {
    detail::requireSize(g.points, std::size_t(g.ndim) * g.weights.size(), "points");
    check(tcscf_grid_create(ctx_, g.points.data(), g.weights.data(), n_, g.ndim, &id_), ctx_);
  }
  ~QMCGrid()
  {
    if (id_) tcscf_grid_destroy(ctx_, id_);
  }
  // ownership of the device grid moves (grid ids start at 1; a moved-from grid holds 0)
  QMCGrid(QMCGrid && o) noexcept : ctx_(o.ctx_), n_(o.n_), ndim_(o.ndim_), id_(o.id_), nb_(o.nb_), gradients_(o.gradients_) { o.id_ = 0; }
  QMCGrid(QMCGrid const &) = delete;
  QMCGrid & operator=(QMCGrid const &) = delete;
  QMCGrid & operator=(QMCGrid &&) = delete;

  int id() const { return id_; }
  tcscf_ctx * context() const { return ctx_; }
  std::int64_t nGrid() const { return n_; }
  int ndim() const { return ndim_; }
  int nBasis() const { return nb_; }
  bool hasGradients() const { return gradients_; }

  // setBasisFunctions (integrateAll.hpp:88-137): values (and gradients) evaluated on the device
  void setBasisFunctions(std::vector<tcscf_sto> const & basis, bool storeGradients = false)
  {
    check(tcscf_grid_set_basis(ctx_, id_, basis.data(), static_cast<int>(basis.size()), storeGradients ? 1 : 0), ctx_);
    nb_ = static_cast<int>(basis.size());
    gradients_ = storeGradients;
  }

  // basisValues [N][nb]: complex on a 3-D grid; on a 2-D grid the real values (imaginary parts 0)
  std::vector<cplx> basisValues() const
  {
    std::size_t const count = std::size_t(n_) * nb_;
    if (ndim_ == 3) {
      std::vector<cplx> v(count);
      check(tcscf_grid_basis_values(ctx_, id_, detail::real(v.data()), nullptr), ctx_);
      return v;
    }
    std::vector<double> r(count);
    check(tcscf_grid_basis_values(ctx_, id_, r.data(), nullptr), ctx_);
    return std::vector<cplx>(r.begin(), r.end());
  }

 private:
  tcscf_ctx * ctx_;
  std::int64_t n_;
  int ndim_;
  int id_ = 0;
  int nb_ = 0;
  bool gradients_ = false;
};

// a device-resident Fji / Vji tensor of the precompute form (released with the object)
class DeviceTensor {
 public:
  DeviceTensor(tcscf_ctx * ctx, int handle) : ctx_(ctx), handle_(handle) {}
  ~DeviceTensor()
  {
    if (handle_) tcscf_tensor_destroy(ctx_, handle_);
  }
  DeviceTensor(DeviceTensor && o) noexcept : ctx_(o.ctx_), handle_(o.handle_) { o.handle_ = 0; }
  DeviceTensor(DeviceTensor const &) = delete;
  DeviceTensor & operator=(DeviceTensor const &) = delete;
  int handle() const { return handle_; }

 private:
  tcscf_ctx * ctx_;
  int handle_;
};

// quadrature S and H on a 3-D grid whose basis has gradients (SlaterTypeOrbitalTest.cpp:14-47): complex [nb][nb]
inline std::pair<std::vector<cplx>, std::vector<cplx>> overlapCoreQuadrature(QMCGrid const & g, int Z)
{
  std::size_t const nn = std::size_t(g.nBasis()) * g.nBasis();
  std::vector<cplx> S(nn), H(nn);
  check(tcscf_overlap_core_quadrature(g.context(), g.id(), Z, detail::real(S.data()), detail::real(H.data())), g.context());
  return {std::move(S), std::move(H)};
}

// precomputeIntegrand + computeF (HartreeFock.hpp:23-180): scalar kernels; kept on the device for
// the precompute-form Fock build and the TC SCF
inline DeviceTensor computeF(QMCGrid const & r1Grid, QMCGrid const & r2Grid, tcscf_kernel kernel = TCSCF_K_INV_R12,
                             tcscf_ochi const * jastrow = nullptr, tcscf_precision precision = TCSCF_PREC_FP64)
{
  int h = 0;
  check(tcscf_compute_F(r1Grid.context(), r1Grid.id(), r2Grid.id(), kernel, jastrow, precision, nullptr, 1, &h), r1Grid.context());
  return DeviceTensor(r1Grid.context(), h);
}

// precomputeIntegrand + computeV (HartreeFock.hpp:55-83, 185-229): vector kernels, on the device
inline DeviceTensor computeV(QMCGrid const & r1Grid, QMCGrid const & r2Grid, tcscf_kernel kernel, tcscf_ochi const & jastrow,
                             tcscf_precision precision = TCSCF_PREC_FP64)
{
  int h = 0;
  check(tcscf_compute_V(r1Grid.context(), r1Grid.id(), r2Grid.id(), kernel, &jastrow, precision, nullptr, 1, &h), r1Grid.context());
  return DeviceTensor(r1Grid.context(), h);
}

// integrateAllR1R2 (integrateAll.hpp:221-317): [nb]^4 complex; r1 3-D, r2 2-D grid
inline std::vector<cplx> integrateAllR1R2(QMCGrid const & r1Grid, QMCGrid const & r2Grid, bool useGradient, tcscf_kernel kernel,
                                          tcscf_ochi const * jastrow = nullptr)
{
  std::size_t const nb = std::size_t(r1Grid.nBasis());
  std::vector<cplx> answer(nb * nb * nb * nb);
  check(tcscf_integrate_all_r1r2(r1Grid.context(), r1Grid.id(), r2Grid.id(), useGradient ? 1 : 0, kernel, jastrow,
                                 detail::real(answer.data())),
        r1Grid.context());
  return answer;
}

// threeElectronIntegrals (integrateAll.hpp:361-442): [nb]^6 complex
inline std::vector<cplx> threeElectronIntegrals(QMCGrid const & r1Grid, QMCGrid const & r2Grid, tcscf_ochi const & jastrow)
{
  std::size_t const nb = std::size_t(r1Grid.nBasis());
  std::vector<cplx> answer(nb * nb * nb * nb * nb * nb);
  check(tcscf_three_electron_integrals(r1Grid.context(), r1Grid.id(), r2Grid.id(), &jastrow, detail::real(answer.data())),
        r1Grid.context());
  return answer;
}

// ---- Fock builds and SCF drivers ------------------------------------------------------------

struct FockBuild {
  std::vector<cplx> G;      // [nspin][nb][nb], element (j, i) at [s][j][i]
  std::vector<cplx> fock;   // F = h + G, same layout
  double energy = 0.0;
};

// per-iteration direct-form Fock build (calculateIaa / calculateFai / assembly, HartreeFock.cpp:144-213,
// 822-850 and 933-956) at the requested precision; density [nspin][nb][nb] complex, h real [nb][nb]
template <class D, class H>
FockBuild fockBuild(QMCGrid const & r1Grid, QMCGrid const & r2Grid, D const & density, H const & h, bool respectSymmetry = true,
                    tcscf_precision precision = TCSCF_PREC_FP64)
{
  std::size_t const nn = std::size_t(r1Grid.nBasis()) * r1Grid.nBasis();
  detail::requireSize(h, nn, "h");
  if (nn == 0 || density.size() % nn != 0 || (density.size() / nn != 1 && density.size() / nn != 2))
    throw Error(TCSCF_ERR_INVALID_ARGUMENT, "density is not [nspin][nb][nb]");
  int const nspin = static_cast<int>(density.size() / nn);
  FockBuild out;
  out.G.resize(nspin * nn);
  out.fock.resize(nspin * nn);
  check(tcscf_fock_build(r1Grid.context(), r1Grid.id(), r2Grid.id(), nspin, detail::real(density.data()), h.data(),
                         respectSymmetry ? 1 : 0, precision, detail::real(out.G.data()), detail::real(out.fock.data()), &out.energy),
        r1Grid.context());
  return out;
}

// RCSHartreeFock / UOSHartreeFock (HartreeFock.hpp:233-349): zero initial density, the direct-form
// Fock build at `precision`, the FP64 generalized Hermitian eigen-solve; stop when |dE| < tol
class HartreeFockBase {
 public:
  HartreeFockBase(int nspin, int numSpinUp, int numSpinDown, int numBasisFunctions, int maxIter)
    : nspin_(nspin), nUp_(numSpinUp), nDown_(numSpinDown), nb_(numBasisFunctions), maxIter_(maxIter),
      density_(std::size_t(nspin) * numBasisFunctions * numBasisFunctions), eigenvalues_(std::size_t(nspin) * numBasisFunctions)
  {}

  // overlap real [nb][nb] (symmetric, so its row- and column-major forms agree), oneElectronTerms real [nb][nb]
  template <class S, class H>
  double compute(S const & overlap, H const & oneElectronTerms, QMCGrid const & r1Grid, QMCGrid const & r2Grid,
                 bool respectOneElectronSymmetry = true, tcscf_precision precision = TCSCF_PREC_FP64, double tol = 1e-5,
                 int maxIter = 0, int diis = 0, bool realEigensolve = false)
  {
    std::size_t const nn = std::size_t(nb_) * nb_;
    if (r1Grid.nBasis() != nb_) throw Error(TCSCF_ERR_INVALID_ARGUMENT, "grid basis size differs from numBasisFunctions");
    detail::requireSize(overlap, nn, "overlap");
    detail::requireSize(oneElectronTerms, nn, "oneElectronTerms");
    tcscf_ctx * ctx = r1Grid.context();
    check(tcscf_set_scf_options(ctx, diis, realEigensolve ? 1 : 0), ctx);
    double energy = 0.0;
    int const st = tcscf_scf(ctx, r1Grid.id(), r2Grid.id(), nspin_, nUp_, nDown_, overlap.data(), oneElectronTerms.data(),
                             respectOneElectronSymmetry ? 1 : 0, precision, tol, maxIter > 0 ? maxIter : maxIter_, &energy,
                             &iterations_, detail::real(density_.data()), eigenvalues_.data());
    tcscf_set_scf_options(ctx, 0, 0);
    check(st, ctx);
    return energy;
  }

  int numberOfConvergenceLoops() const { return iterations_; }
  std::vector<cplx> const & density() const { return density_; }        // [nspin][nb][nb]
  std::vector<double> const & eigenvalues() const { return eigenvalues_; }  // [nspin][nb], ascending

 protected:
  int nspin_, nUp_, nDown_, nb_, maxIter_;
  int iterations_ = 0;
  std::vector<cplx> density_;
  std::vector<double> eigenvalues_;
};

// restricted closed shell, at most 50 iterations (HartreeFock.cpp:815)
class RCSHartreeFock : public HartreeFockBase {
 public:
  RCSHartreeFock(int numSpinUp, int numSpinDown, int numBasisFunctions)
    : HartreeFockBase(1, numSpinUp, numSpinDown, numBasisFunctions, 50)
  {}
  double highestOccupiedOrbitalEnergy() const { return eigenvalues_[(nUp_ + nDown_) / 2 - 1]; }

  // compute() with the whole loop on the device (tcscf_scf_graph): with capture, the iterations after
  // the first two are one CUDA graph launch whose device-side WHILE node ends the loop
  template <class S, class H>
  double computeOnDevice(S const & overlap, H const & oneElectronTerms, QMCGrid const & r1Grid, QMCGrid const & r2Grid,
                         bool respectOneElectronSymmetry = true, tcscf_precision precision = TCSCF_PREC_FP64, double tol = 1e-5,
                         int maxIter = 0, bool capture = true)
  {
    std::size_t const nn = std::size_t(nb_) * nb_;
    if (r1Grid.nBasis() != nb_) throw Error(TCSCF_ERR_INVALID_ARGUMENT, "grid basis size differs from numBasisFunctions");
    detail::requireSize(overlap, nn, "overlap");
    detail::requireSize(oneElectronTerms, nn, "oneElectronTerms");
    tcscf_ctx * ctx = r1Grid.context();
    double energy = 0.0;
    check(tcscf_scf_graph(ctx, r1Grid.id(), r2Grid.id(), nUp_, nDown_, overlap.data(), oneElectronTerms.data(),
                          respectOneElectronSymmetry ? 1 : 0, precision, tol, maxIter > 0 ? maxIter : maxIter_, capture ? 1 : 0, &energy,
                          &iterations_, detail::real(density_.data()), eigenvalues_.data(), &graphLaunches_),
          ctx);
    return energy;
  }
  int graphLaunches() const { return graphLaunches_; }

 private:
  int graphLaunches_ = 0;
};

// unrestricted open shell, at most 100 iterations (HartreeFock.cpp:923)
class UOSHartreeFock : public HartreeFockBase {
 public:
  UOSHartreeFock(int numSpinUp, int numSpinDown, int numBasisFunctions)
    : HartreeFockBase(2, numSpinUp, numSpinDown, numBasisFunctions, 100)
  {}
  double highestOccupiedOrbitalEnergy() const
  {
    double const up = nUp_ > 0 ? eigenvalues_[nUp_ - 1] : -1e300;
    double const down = nDown_ > 0 ? eigenvalues_[nb_ + nDown_ - 1] : -1e300;
    return up > down ? up : down;
  }
};

// TCHartreeFock (HartreeFock.hpp:353-394, HartreeFock.cpp:1007-1362): transcorrelated SCF from the
// device-resident TC scalar kernels (same / opposite spin) and grad u tensors, at most 200 iterations
class TCHartreeFock {
 public:
  TCHartreeFock(int numSpinUp, int numSpinDown, int numBasisFunctions)
    : nUp_(numSpinUp), nDown_(numSpinDown), nb_(numBasisFunctions), density_(2 * std::size_t(numBasisFunctions) * numBasisFunctions),
      pseudoEnergies_(2 * std::size_t(numBasisFunctions))
  {}

  template <class S, class H>
  double compute(S const & overlap, H const & oneElectronTerms, QMCGrid const & r1Grid, DeviceTensor const & fjiSame,
                 DeviceTensor const & fjiOppo, DeviceTensor const & vjiSame, DeviceTensor const & vjiOppo,
                 bool respectOneElectronSymmetry = true, double tol = 1e-5, int maxIter = 200)
  {
    std::size_t const nn = std::size_t(nb_) * nb_;
    detail::requireSize(overlap, nn, "overlap");
    detail::requireSize(oneElectronTerms, nn, "oneElectronTerms");
    double energy = 0.0;
    check(tcscf_tc_scf(r1Grid.context(), r1Grid.id(), fjiSame.handle(), fjiOppo.handle(), vjiSame.handle(), vjiOppo.handle(),
                       overlap.data(), oneElectronTerms.data(), nUp_, nDown_, respectOneElectronSymmetry ? 1 : 0, tol, maxIter,
                       &energy, &iterations_, detail::real(density_.data()), pseudoEnergies_.data()),
          r1Grid.context());
    return energy;
  }

  int numberOfConvergenceLoops() const { return iterations_; }
  std::vector<cplx> const & density() const { return density_; }
  std::vector<double> const & pseudoEnergies() const { return pseudoEnergies_; }

 private:
  int nUp_, nDown_, nb_;
  int iterations_ = 0;
  std::vector<cplx> density_;
  std::vector<double> pseudoEnergies_;
};

}  // namespace tcscf::gpu

#endif  // TCSCF_GPU_HPP
