// Host-side check of the C++ layer include/tcscf_gpu.hpp, compiled and run by tests/test_cpp_shim.py.
//
// Runs without a device: grids, basis-set loading, analytic overlap / core matrices and the error
// mapping.  The device paths (QMCGrid, fockBuild, the SCF classes, computeF / computeV, the 4- and
// 6-index tensors) are compiled here, so every template of the header is instantiated, and run when a
// context can be created (tests/test_gpu_cpp_shim.py on a B200).
//
//   shim_host <basis-set directory holding TZ3P/He>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "tcscf_gpu.hpp"

namespace {

int failures = 0;

void expect(bool ok, char const * what)
{
  std::printf("%s %s\n", ok ? "ok  " : "FAIL", what);
  if (!ok) ++failures;
}

double const pi = 3.14159265358979323846;

// the 6-point octahedral angular rule: {theta, phi, weight}, weights summing to 4 pi
std::vector<double> octahedron()
{
  double const w = 4 * pi / 6;
  return {pi / 2, 0, w, pi / 2, pi, w, pi / 2, pi / 2, w, pi / 2, 3 * pi / 2, w, 0, 0, w, pi, 0, w};
}

// the pattern of a reference-side adaptor: a device grid built and returned by value
tcscf::gpu::QMCGrid upload(tcscf::gpu::Context & ctx, tcscf::gpu::QuadratureGrid const & g, std::vector<tcscf_sto> const & basis)
{
  tcscf::gpu::QMCGrid d(ctx, g);
  d.setBasisFunctions(basis, false);
  return d;
}

// device paths: He through every class of the header; the energies are printed as "key value" lines
// for tests/test_gpu_cpp_shim.py, which checks them against the oracle
void deviceRun(tcscf::gpu::Context & ctx)
{
  using namespace tcscf::gpu;
  std::vector<tcscf_sto> basis;
  for (int k = 0; k < 6; ++k) basis.push_back({0.9 * std::pow(1.8, k), 1, 0, 0, TCSCF_BASIS_STO});
  auto const [r, wr] = radialGrid(40, TCSCF_MAP_ONE_PLUS_X);
  QuadratureGrid const g = productGrid(r, wr, octahedron());
  QMCGrid G(ctx, g);
  G.setBasisFunctions(basis, true);
  auto const [S, H] = overlapCore(basis, 2);
  RCSHartreeFock hf(1, 1, static_cast<int>(basis.size()));
  double const E = hf.compute(S, H, G, G, true, TCSCF_PREC_FP64, 1e-10);
  std::vector<cplx> D(hf.density());
  FockBuild const f64 = fockBuild(G, G, D, H, true, TCSCF_PREC_FP64);
  FockBuild const fb = fockBuild(G, G, D, H, true, TCSCF_PREC_BF16X3);
  std::printf("E_SCF %.15f\nITER %d\nE_FOCK_FP64 %.15f\nE_FOCK_BF16X3 %.15f\n", E, hf.numberOfConvergenceLoops(), f64.energy, fb.energy);
  expect(std::abs(f64.energy - E) < 1e-10, "FP64 Fock build at the converged density reproduces the SCF energy");
  expect(std::abs(fb.energy - E) < 1e-6, "split-BF16 Fock build at the converged density reproduces the SCF energy");
  RCSHartreeFock dev(1, 1, static_cast<int>(basis.size()));
  double const Eg = dev.computeOnDevice(S, H, G, G, true, TCSCF_PREC_FP64, 1e-10);
  std::printf("E_GRAPH %.15f\n", Eg);
  expect(dev.graphLaunches() == 1 && std::abs(Eg - E) < 1e-8, "device-loop SCF (one graph launch) reproduces the SCF energy");
  UOSHartreeFock uos(1, 1, static_cast<int>(basis.size()));
  double const Eu = uos.compute(S, H, G, G, true, TCSCF_PREC_FP64, 1e-10);
  std::printf("E_UOS %.15f\n", Eu);
  expect(std::abs(Eu - E) < 1e-8, "UOS SCF of the closed-shell atom equals the RCS energy");
  DeviceTensor F = computeF(G, G);
  expect(F.handle() != 0, "computeF keeps a device tensor");
  DeviceTensor Fm = computeF(G, G, TCSCF_K_INV_R12, nullptr, TCSCF_PREC_BF16X3);
  expect(Fm.handle() != 0, "computeF in split BF16 keeps a device tensor");
  std::vector<cplx> const vals = G.basisValues();
  expect(vals.size() == std::size_t(g.size()) * basis.size(), "basisValues is [N][nb]");
  auto const [Sq, Hq] = overlapCoreQuadrature(G, 2);
  double ds = 0;
  for (std::size_t i = 0; i < Sq.size(); ++i) ds = std::max(ds, std::abs(Sq[i] - S[i]));
  std::printf("S_QUAD_ERR %.3e\n", ds);
  tcscf_ochi u{};
  u.a = 1.0; u.a12 = 1.0; u.nterms = 1; u.S[0][0] = 1; u.c[0][0] = -0.5; u.c[0][1] = -0.25;
  DeviceTensor V = computeV(G, G, TCSCF_K_GRAD_U_SAME, u);
  expect(V.handle() != 0, "computeV keeps a device tensor");
  if (false) {  // instantiated, not run: the remaining device entry points of the header
    QMCGrid G2 = upload(ctx, qmcGrid(2, sobol(2, 64, 1)), basis);
    (void)integrateAllR1R2(G, G2, false, TCSCF_K_INV_R12);
    (void)threeElectronIntegrals(G, G, u);
    TCHartreeFock tc(1, 1, 6);
    (void)tc.compute(S, H, G, F, F, V, V);
    double a = 0, b = 0;
    int n = 0;
    ctx.lastTiming(a, b, n);
    ctx.setAutotune(false);
  }
}

}  // namespace

int main(int argc, char ** argv)
{
  using namespace tcscf::gpu;

  // radial maps, the reference's known answers (IntegrationTest.cpp:76-105 with TA-M4 a = 1, eps = 1)
  {
    auto const [r, w] = radialGrid(100, TCSCF_MAP_TREUTLER_AHLRICHS_M4, 1.0, 1.0);
    double s1 = 0, s2 = 0;
    for (std::size_t i = 0; i < r.size(); ++i) {
      s1 += std::exp(-r[i]) * w[i];
      s2 += (r[i] * r[i] - 3 * r[i]) * std::exp(-1.5 * r[i]) * w[i];
    }
    expect(std::abs(s1 - 1.0) < 1e-7, "radialGrid: integral of exp(-r) = 1");
    expect(std::abs(s2 + 20.0 / 27.0) < 1e-10, "radialGrid: integral of (r^2 - 3r) exp(-3r/2) = -20/27");
  }
  // product rule: weights carry r^2 and the angular weights, so sum w exp(-r) = 4 pi * 2
  {
    auto const [r, wr] = radialGrid(80, TCSCF_MAP_ONE_PLUS_X);
    QuadratureGrid const g = productGrid(r, wr, octahedron());
    double s = 0;
    for (std::int64_t i = 0; i < g.size(); ++i) {
      double const x = g.points[i], y = g.points[g.size() + i], z = g.points[2 * g.size() + i];
      s += g.weights[i] * std::exp(-std::sqrt(x * x + y * y + z * z));
    }
    expect(g.size() == 80 * 6 && std::abs(s - 8 * pi) < 1e-8, "productGrid: 4 pi integral of r^2 exp(-r)");
  }
  // QMC mapping of scrambled Sobol points: a normalised density integrates to about 1
  {
    QuadratureGrid const g = qmcGrid(3, sobol(3, 1 << 14, 20261203));
    double s = 0;
    for (std::int64_t i = 0; i < g.size(); ++i) {
      double const x = g.points[i], y = g.points[g.size() + i], z = g.points[2 * g.size() + i];
      s += g.weights[i] * std::exp(-2 * std::sqrt(x * x + y * y + z * z)) / pi;
    }
    expect(g.size() == (1 << 14) && std::abs(s - 1.0) < 2e-2, "qmcGrid: hydrogen 1s density integrates to 1");
  }
  // analytic S and H: normalised STOs, hydrogen 1s (zeta = 1, Z = 1) core element -1/2
  {
    std::vector<tcscf_sto> const basis = {{1.0, 1, 0, 0, TCSCF_BASIS_STO}, {0.7, 2, 1, 0, TCSCF_BASIS_STO}};
    auto const [S, H] = overlapCore(basis, 1);
    expect(std::abs(S[0] - 1) < 1e-12 && std::abs(S[3] - 1) < 1e-12 && S[1] == 0.0, "overlapCore: unit diagonal, l-orthogonal");
    expect(std::abs(H[0] + 0.5) < 1e-12, "overlapCore: hydrogen 1s core element -1/2");
  }
  // loadSTO from the directory given on the command line
  if (argc > 1) {
    std::vector<tcscf_sto> const b = loadSTO(argv[1], "TZ3P", "He", 3);
    expect(b.size() == 3 + 6 + 5 + 7 && b[0].alpha == 2.9 && b[3].l == 1 && b[3].m == -1, "loadSTO: m expansion in file order");
    // a missing element file gives an empty basis, as the reference's loader; a missing basis-set
    // directory is an error
    expect(loadSTO(argv[1], "TZ3P", "Ne", 3).empty(), "loadSTO: missing element file -> empty basis");
    int code = 0;
    try {
      (void)loadSTO(argv[1], "QZ6P", "He", 3);
    } catch (Error const & e) {
      code = e.code();
    }
    expect(code == TCSCF_ERR_INVALID_ARGUMENT, "loadSTO: missing basis-set directory throws Error(TCSCF_ERR_INVALID_ARGUMENT)");
  }
  // error mapping: a bad argument throws Error with its status
  {
    int code = 0;
    try {
      (void)radialGrid(0, TCSCF_MAP_NONE);
    } catch (Error const & e) {
      code = e.code();
    }
    expect(code == TCSCF_ERR_INVALID_ARGUMENT, "radialGrid(0) throws Error(TCSCF_ERR_INVALID_ARGUMENT)");
  }
  // the device: without one, Context throws Error(TCSCF_ERR_NO_DEVICE); with one, the device paths run
  try {
    Context ctx(0);
    deviceRun(ctx);
  } catch (ConvergenceError const &) {
    expect(false, "device SCF converged");
  } catch (Error const & e) {
    std::printf("no device: %s\n", e.what());
    expect(e.code() == TCSCF_ERR_NO_DEVICE || e.code() == TCSCF_ERR_UNSUPPORTED, "Context without a B200 throws Error(NO_DEVICE)");
  }
  std::printf("%d failure(s)\n", failures);
  return failures == 0 ? 0 : 1;
}
