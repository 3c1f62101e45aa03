/*
 * tcscf_gpu.h — C ABI of libtcscf_gpu.so, the B200 (sm_100a) grid-quadrature Fock build.
 *
 * Drop-in boundary for corbett5/tcscf's integral routines (src/integration/integrateAll.hpp,
 * src/HartreeFock.hpp:23-229) and the per-iteration Fock build / SCF drivers of
 * src/HartreeFock.cpp.  Plain pointers and sizes only; complex numbers are interleaved
 * (re, im) doubles exactly like std::complex<double> (src/RAJAInterface.hpp:98-103 relies on that
 * layout too).  Every entry point returns a tcscf_status; the message of the last failure on a
 * context is available from tcscf_last_error().
 *
 * Layouts (reference index orders, last index contiguous):
 *   points      [ndim][N]            (integration::QuadratureGrid::points, quadrature.hpp:25-35)
 *   weights     [N]
 *   basis vals  [N][nb]              (QMCGrid::basisValues, integrateAll.hpp:139-141); complex for
 *                                    3-D grids, real for 2-D grids
 *   basis grads [N][nb][3] complex   (QMCGrid::basisGradients)
 *   Fji         [N1][nb][nb]         (computeF, HartreeFock.hpp:88-180); complex for a 3-D r2 grid,
 *                                    real (with the 2*pi of HartreeFock.hpp:123) for a 2-D r2 grid
 *   Vji         [N1][nb][nb][3] complex (computeV, HartreeFock.hpp:185-229)
 *   density, G, Fock [nspin][nb][nb] complex, element (j,i) at [s][j][i] (row-major; the reference's
 *                                    fockOperator is PERM_IKJ, i.e. its transpose per spin)
 *   S, H        [nb][nb] real row-major
 *
 * Threading: one context per host thread; calls on a context are not reentrant.  All device work
 * of a context runs on its own CUDA stream (tcscf_ctx_stream).
 */
#ifndef TCSCF_GPU_H
#define TCSCF_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum tcscf_status {
  TCSCF_OK = 0,
  TCSCF_ERR_INVALID_ARGUMENT = 1, /* LVARRAY_ERROR_IF_NE / CHECK_BOUNDS_* in the reference */
  TCSCF_ERR_CUDA = 2,
  TCSCF_ERR_TIMEOUT = 3,          /* a bounded device wait gave up */
  TCSCF_ERR_NONFINITE = 4,        /* NaN/Inf in an energy or Fock matrix */
  TCSCF_ERR_NOT_CONVERGED = 5,    /* tcscf::ConvergenceError (HartreeFock.hpp:13-19) */
  TCSCF_ERR_LINALG = 6,           /* LvArray::dense::Error (eigen-solve failure) */
  TCSCF_ERR_UNSUPPORTED = 7,      /* shape or feature outside what this library implements */
  TCSCF_ERR_NO_DEVICE = 8
} tcscf_status;

/* Atomic basis function families; every function is radial(r) * Y_lm(theta, phi) and one basis
 * holds one family (the reference's QMCGrid::setBasisFunctions is a template over the family). */
typedef enum tcscf_basis_family {
  TCSCF_BASIS_STO = 0,      /* SlaterTypeOrbital (SlaterTypeOrbital.hpp:27-106): N r^(n-1) e^(-alpha r), n >= 1 */
  TCSCF_BASIS_OCHI = 1,     /* OchiBasisFunction (OchiBasis.hpp:14-110): N r^l L_n^(2l+2)(2 alpha r) e^(-alpha r), n >= 0 */
  TCSCF_BASIS_HYDROGEN = 2  /* HydrogenLikeBasisFunction (HydrogenLikeBasis.hpp:11-60): alpha = Z, beta = Z / n,
                               N r^l L_(n-l-1)^(2l+1)(2 beta r) e^(-beta r); values only (the reference has no gradient) */
} tcscf_basis_family;

/* One basis function (SlaterTypeOrbital / OchiBasisFunction / HydrogenLikeBasisFunction constructor
 * arguments): alpha = orbital exponent (STO, Ochi) or nuclear charge Z (hydrogen-like); family is a
 * tcscf_basis_family (0 = STO). */
typedef struct tcscf_sto {
  double alpha;
  int32_t n, l, m, family;
} tcscf_sto;

/* Ochi / Boys-Handy Jastrow factor (jastrowFunctions.hpp:9-115):
 * u = sum_k c[k][same] * (r12/(r12+a12))^S[k][0] * (r1/(r1+a))^S[k][1] * (r2/(r2+a))^S[k][2];
 * c[k][0] is the opposite-spin and c[k][1] the same-spin coefficient. */
typedef struct tcscf_ochi {
  double a, a12;
  int32_t nterms, pad;
  int32_t S[8][3];
  double c[8][2];
} tcscf_ochi;

/* r12 kernels: the lambdas of src/unitTests/HartreeFockTest.cpp:248-253 (1/r12), :276-296
 * (TC scalar 2/r12 - |grad_1 u(r1,r2)|^2 - |grad_1 u(r2,r1)|^2) and :300-318 (grad_1 u). An exactly
 * coincident pair r1 == r2 contributes 0 in every kernel. */
typedef enum tcscf_kernel {
  TCSCF_K_INV_R12 = 0,
  TCSCF_K_TC_SCALAR_SAME = 1,
  TCSCF_K_TC_SCALAR_OPPO = 2,
  TCSCF_K_GRAD_U_SAME = 3,
  TCSCF_K_GRAD_U_OPPO = 4
} tcscf_kernel;

/* Precision of the r12 contraction (the direct Fock build; computeF / computeV take FP64 and BF16X3).
 * FP64: CUDA-core FP64 throughout.  BF16X3: tcgen05 tensor cores on fixed-point BF16
 * slices of every operand (24 bits for the orbital factors and the weighted basis, 16 or 24 bits for
 * g * rho; power-of-two scales per row / column / r2 block of 64), so the tensor-core sum of the
 * leading slices is exact; each block is added into double-float (FP32 hi + lo) accumulators.
 * TF32: tcgen05 kind::tf32 on operands rounded to TF32 (10 explicit mantissa bits), FP32
 * accumulation within an r2 block of 64, blocks added into double-float accumulators. */
typedef enum tcscf_precision {
  TCSCF_PREC_FP64 = 0,
  TCSCF_PREC_BF16X3 = 1,
  TCSCF_PREC_TF32 = 2
} tcscf_precision;

/* radial changes of variables (changeOfVariables.hpp:8-232); TCSCF_MAP_ONE_PLUS_X is
 * r = (1+x)/(1-x) (jacobian 2/(1-x)^2), which the reference does not have. */
typedef enum tcscf_map {
  TCSCF_MAP_NONE = 0,
  TCSCF_MAP_LINEAR = 1,             /* p0 = scale */
  TCSCF_MAP_X_OVER_1MX = 2,
  TCSCF_MAP_TREUTLER_AHLRICHS_M4 = 3, /* p0 = a, p1 = epsilon */
  TCSCF_MAP_ONE_PLUS_X = 4
} tcscf_map;

typedef struct tcscf_ctx tcscf_ctx;

/* ---- context -------------------------------------------------------------------------------- */
int tcscf_ctx_create(int device, tcscf_ctx ** ctx);
int tcscf_ctx_destroy(tcscf_ctx * ctx);
const char * tcscf_last_error(tcscf_ctx * ctx);
/* Self-test of the failure path of the library's bounded device waits (no reference counterpart):
 * one warp waits, through the same bounded-wait helper as the tensor-core kernels, on an mbarrier that
 * nothing arrives at, and gives up after limit_ms (1..1000) milliseconds.  Returns TCSCF_ERR_TIMEOUT,
 * the expected outcome; the context stays usable afterwards. */
int tcscf_selftest_bounded_wait(tcscf_ctx * ctx, double limit_ms);
/* the context's cudaStream_t, for callers that time or order work around it */
int tcscf_ctx_stream(tcscf_ctx * ctx, void ** stream);
int tcscf_synchronize(tcscf_ctx * ctx);
/* device time in ms of the dominant r12 contraction kernel(s) of the most recent Fock build /
 * computeF call, measured with CUDA events on the context stream; launches = kernels launched */
int tcscf_last_timing(tcscf_ctx * ctx, double * contraction_ms, double * total_ms, int * launches);
/* diagnostics: the Coulomb potential VH[N1] (both spins) and the first spin's exchange potential
 * T[N1][nb] (real-harmonic basis) of the most recent direct Fock build on this context.  A split-BF16
 * build with one grid as r1 and r2 and a positive semi-definite real density contracts only the pairs
 * on and above each 128-point r1 tile's diagonal (the diagonal tile at half weight): T is then that
 * half, whose r1 quadrature plus its transpose is the exchange matrix; VH is complete either way */
int tcscf_last_potentials(tcscf_ctx * ctx, double * VH, double * T);

/* ---- host-side grid generation (replaces ChebyshevGauss/changeOfVariables/createGrid,
 *      TreutlerAhlrichsLebedev and QMCGrid's point mapping) ---------------------------------- */
/* createGrid(ChebyshevGauss(n), map) (quadrature.hpp:75-102): abscissae u[n], weights w[n] */
int tcscf_grid_radial(int n, int map, double p0, double p1, double * u, double * w);
/* radial x angular product grid, index ir*nang + ia; ang = nang x {theta, phi, weight} (the
 * reference's Lebedev table layout, src/integration/data/LebedevData_*.hpp); weight r^2 w_r w_ang
 * (TreutlerAhlrichsLebedev.hpp:46-74 with the caller's r^2). pts [3][N], w [N]. */
int tcscf_grid_product(int nrad, const double * r, const double * wr, int nang, const double * ang, double * pts, double * w);
/* QMCGrid<REAL,NDIM> point mapping (integrateAll.hpp:21-65, qmcWrapper.hpp:128-136) of unit-cube
 * points u [ndim][N]: TA-M4(a=0, eps=0.9) radius, theta = acos(1-2u), phi = 2 pi u, weight
 * jacobian * r^2 sin(theta) / N.  ndim 2 gives (x, z) rows. */
int tcscf_grid_qmc(int ndim, int64_t n, const double * u, double * pts, double * w);
/* seeded scrambled Sobol points in [0,1)^ndim (ndim <= 3), layout [ndim][n]; replaces the
 * un-vendored mppmu/qmc lattice generator (qmcWrapper.hpp:94-141). */
int tcscf_sobol(int ndim, int64_t n, uint64_t seed, double * u);

/* loadSTO (SlaterTypeOrbital.cpp:24-75): the STO basis of an element from the ADF-style basis-set
 * library <directory>/<basisSet>/<element> (basisSet one of TZ3P, QZ6P, ATZ3P, AQZ6P), functions with
 * l <= maxL expanded over m = -l..l.  out may be NULL to query *count; otherwise at most capacity
 * functions are written.  Host only. */
int tcscf_load_sto(const char * directory, const char * basisSet, const char * element, int maxL, tcscf_sto * out, int capacity,
                   int * count);

/* ---- analytic one-electron matrices -----------------------------------------------------------
 * STO: SlaterTypeOrbital.hpp:134-181.  Ochi: overlap = [n, l, m equal] (OchiBasis.hpp:118-125), core
 * element from the radial integral of fnl fnl / r (OchiBasis.hpp:130-155) on the reference driver's
 * 1000-point Chebyshev-Gauss grid with the Treutler-Ahlrichs M4 map (a = 1, eps = 0.9,
 * HartreeFockTest.cpp:364-367); functions of different exponents have no core element
 * (TCSCF_ERR_INVALID_ARGUMENT).  Hydrogen-like: overlap = [l, m equal] x the radial integral of
 * R1 R2 r^2 on the same grid (the generic AtomicBasis.hpp overlap), core element -Z^2 / (2 n^2) when
 * n, l, m are equal (HydrogenLikeBasis.hpp:70-82).  One family per call. */
int tcscf_overlap_core_analytic(const tcscf_sto * basis, int nb, int Z, double * S, double * H);

/* ---- device-resident grids (QMCGrid, integrateAll.hpp:12-142) ------------------------------- */
/* copies points [ndim][n] and weights [n] from host memory; ndim 2 or 3.  Grid buffers come from a
 * memory pool owned by the context, in the order of its stream: tcscf_grid_destroy returns them to
 * the pool after the context's queued work, without a device-wide synchronisation, and the pool keeps
 * up to 4 GiB of freed grid memory for later grids until the context is destroyed. */
int tcscf_grid_create(tcscf_ctx * ctx, const double * points, const double * weights, int64_t n, int ndim, int * grid);
int tcscf_grid_destroy(tcscf_ctx * ctx, int grid);
/* QMCGrid::setBasisFunctions (integrateAll.hpp:88-137): evaluates the STOs (and gradients) on the
 * device.  The basis must contain the -m partner of every m != 0 function. */
int tcscf_grid_set_basis(tcscf_ctx * ctx, int grid, const tcscf_sto * basis, int nb, int gradients);
/* copies QMCGrid::basisValues / basisGradients to host buffers (either may be NULL) */
int tcscf_grid_basis_values(tcscf_ctx * ctx, int grid, double * values, double * gradients);

/* Near-coincident pairs of two grids (no reference counterpart): the r1 / r2 point pairs that are
 * closer than 2^-16 |r1| (below what FP32 coordinates resolve) without being identical.  The
 * tensor-core paths leave these pairs out of their FP32 kernel generation and add them back evaluated
 * in FP64, so every precision follows the reference's rule that only an exactly coincident pair
 * contributes 0 (IntegrationTest.cpp:298-309).  The list is found on the first use of the grid pair
 * (here or in a tensor-core build) and kept until either grid is destroyed. */
int tcscf_near_coincident_pairs(tcscf_ctx * ctx, int r1, int r2, int * count);

/* quadrature S_ij = sum_g w phi_i^* phi_j and H_ij = sum_g w (1/2 grad phi_i^* . grad phi_j - Z phi_i^* phi_j / r)
 * on a 3-D grid with gradients; S, H complex [nb][nb] */
int tcscf_overlap_core_quadrature(tcscf_ctx * ctx, int grid, int Z, double * S, double * H);
/* Same quadrature with no device allocation: the block results use a fixed 2 MiB device array
 * (nb <= 256, else TCSCF_ERR_UNSUPPORTED), for callers that cannot allocate device memory at that
 * point (device memory already handed to their own pool, or no device-wide synchronisation allowed).
 * tcscf_ctx_create looks up the array's address on its device, so calls do no set-up of their own;
 * overlapping calls on one device share the array and race.  No counterpart in the reference. */
int tcscf_overlap_core_quadrature_static(tcscf_ctx * ctx, int grid, int Z, double * S, double * H);

/* ---- r12 kernel contractions (precompute form) --------------------------------------------- */
/* precomputeIntegrand + computeF (HartreeFock.hpp:23-180): F written to host memory in the Fji
 * layout (complex for a 3-D r2 grid, real x 2 pi for a 2-D r2 grid).  When keep != 0 the result also
 * stays on the device as handle *fji for tcscf_fock_build_precomputed / tcscf_tc_fock_build.
 * precision: TCSCF_PREC_FP64, or TCSCF_PREC_BF16X3 (the r12 kernel-GEMM on the tensor cores in the
 * split-BF16 scheme of the Fock build, kernel values generated in FP32 from FP32 coordinates; the
 * Jastrow factor of a TC kernel must depend on r12 alone, every term S[k] = (i, 0, 0), as the
 * reference's own TC driver uses it, HartreeFockTest.cpp:351-360). */
int tcscf_compute_F(tcscf_ctx * ctx, int r1, int r2, int kernel, const tcscf_ochi * jastrow, int precision, double * F, int keep,
                    int * fji);
/* precomputeIntegrand + computeV (HartreeFock.hpp:55-83, :185-229), vector kernels only; precision as
 * for tcscf_compute_F */
int tcscf_compute_V(tcscf_ctx * ctx, int r1, int r2, int kernel, const tcscf_ochi * jastrow, int precision, double * V, int keep,
                    int * vji);
int tcscf_tensor_destroy(tcscf_ctx * ctx, int handle);

/* ---- 4- and 6-index tensors (integrateAll.hpp:147-442) --------------------------------------- */
/* integrateAllR1R2<USE_GRADIENT> (integrateAll.hpp:221-317): r1 a 3-D grid, r2 a 2-D grid with the
 * same basis; scalar kernel (value form, answer[b1][b2][b3][b4]) or, with use_gradient, a vector
 * kernel dotted into the r2 basis gradients (answer[b2][b1][b4][b3], integrateAll.hpp:302).
 * answer: nb^4 complex in host memory. */
int tcscf_integrate_all_r1r2(tcscf_ctx * ctx, int r1, int r2, int use_gradient, int kernel, const tcscf_ochi * jastrow,
                             double * answer);
/* threeElectronIntegrals (integrateAll.hpp:361-442): r1, r2 3-D grids, same-spin grad u;
 * answer[p][q][r][s][t][u] = sum_r1 w1 conj(phi_p) phi_s V(r1,q,t) . V(r1,r,u), nb^6 complex in host
 * memory (nb <= 32). */
int tcscf_three_electron_integrals(tcscf_ctx * ctx, int r1, int r2, const tcscf_ochi * jastrow, double * answer);

/* ---- per-iteration Fock build ---------------------------------------------------------------- */
/* Direct form: G from the density without any stored Fji.  Same result as calculateIaa /
 * calculateFai / assembly (HartreeFock.cpp:817-843 RCS, :925-956 UOS) on Fji = computeF(r1, r2,
 * 1/r12), followed by enforceOneElectronSymmetry (when respect_symmetry) and constructSCFOperator
 * (HartreeFock.cpp:48-98).  nspin 1 (RCS, energy x2) or 2 (UOS).  h real [nb][nb].
 * Outputs (any may be NULL): G, Fock [nspin][nb][nb] complex, energy. */
int tcscf_fock_build(tcscf_ctx * ctx, int r1, int r2, int nspin, const double * density, const double * h,
                     int respect_symmetry, int precision, double * G, double * fock, double * energy);
/* Same as tcscf_fock_build with density, h, G, fock and energy in device memory (G / fock may be
 * NULL); the work is ordered on the context stream, which is synchronised before returning. */
int tcscf_fock_build_device(tcscf_ctx * ctx, int r1, int r2, int nspin, const double * density, const double * h,
                            int respect_symmetry, int precision, double * G, double * fock, double * energy);
/* Batched RCS Fock builds: instance k uses grids r1[k], r2[k], density[k] ([nb][nb] complex) and
 * h[k]; energy[k] receives its energy and, when fock and fock[k] are not NULL, fock[k] its Fock
 * matrix.  At BF16X3 the r12 contractions of all instances run in one persistent launch per tile
 * class (instances whose density factor is complex in the real-harmonic basis are built on their
 * own); FP64 builds the instances one after another.  Per-instance results are those of
 * tcscf_fock_build_device. */
int tcscf_fock_build_batch(tcscf_ctx * ctx, int count, const int * r1, const int * r2, const double * const * density,
                           const double * const * h, int respect_symmetry, int precision, double * energy, double * const * fock);
/* Same, from a device-resident Fji handle (the reference's precompute form). */
int tcscf_fock_build_precomputed(tcscf_ctx * ctx, int r1, int fji, int nspin, const double * density, const double * h,
                                 int respect_symmetry, double * G, double * fock, double * energy);
/* CUDA-graph use of tcscf_fock_build_batch on this context (no reference counterpart): the batch's
 * persistent tensor launches are captured into a graph the first time a launch sequence (tile
 * classes, grid sizes, work-item counts, device tables) occurs and replayed while it repeats, e.g.
 * over the SCF iterations of one set of instances.  Returns the numbers of captures and replays. */
int tcscf_batch_graph_stats(tcscf_ctx * ctx, int * captures, int * replays);

/* Autotuner of the tensor-core Fock build's schedule (no reference counterpart; off by default).
 * With it on, the first split-BF16 / TF32 direct build of each shape (r1 and r2 points, padded basis
 * size, padded density rank, precision) times every candidate r2 split of its persistent launch with
 * CUDA events on the context stream and keeps the fastest for later builds of that shape; the first
 * tcscf_fock_build_batch of each batch signature (precision, every instance's grid sizes and basis
 * size) times the split policies {default rule, no split, 2x, 4x} over the whole batch and keeps the
 * fastest.  The tile class (NB, RP, X precision) stays the fixed rule: it sets the accuracy.  Results
 * of different splits differ only in the order of the r2 block sums.  Turning it off returns to the
 * default rule and keeps the measurements. */
int tcscf_set_autotune(tcscf_ctx * ctx, int enable);
/* shapes and batch signatures tuned on this context so far, and candidate measurements taken */
int tcscf_autotune_stats(tcscf_ctx * ctx, int * shapes, int * batches, int * measurements);
/* host only: the candidate r2 split counts for a launch over n1 x n2 points on a device with sms SMs,
 * the default rule's first, then 1, 2, 3, 4, 6, 8 while every split keeps at least 16 r2 blocks of 64
 * points (effective counts, no repeats); writes at most capacity of them and their number to count */
int tcscf_autotune_split_candidates(int64_t n1, int64_t n2, int sms, int * splits, int capacity, int * count);
/* host only: the order in which the persistent tensor-core launch over one instance of n1 x n2 points
 * (sym != 0: one grid as r1 and r2, each r1 tile from its diagonal r2 block on) with nsplit r2 splits
 * hands out its work items to grid CTAs, CTA b taking items b, b + grid, ...: the items weighed by their
 * r2 blocks, the most first, in snake order over rounds of grid items.  Writes tile, split and r2 block
 * count (3 ints) of at most capacity items, in that order, and the item count to count.  No reference
 * counterpart (launch scheduling). */
int tcscf_schedule_items(int64_t n1, int64_t n2, int sym, int nsplit, int grid, int * items, int capacity, int * count);

/* ---- SCF drivers (RCSHartreeFock/UOSHartreeFock::compute, HartreeFock.cpp:785-1003) ---------- */
/* Options of tcscf_scf on this context (no reference counterpart; the defaults, 0 and 0, reproduce
 * the reference's plain Roothaan iteration with the complex eigen-solver).  diis in 2..16: the
 * eigen-solve of every iteration after the first takes the combination of the last `diis` Fock
 * matrices that minimises the norm of the combined commutator errors F D S - S D F; the energy and
 * the |dE| < tol test are unchanged.  real_eigensolve != 0: a Fock matrix that is real in the
 * real-harmonic basis is diagonalised there as a real symmetric problem, so the density stays real
 * (half the factor rank, one contraction per build) when the aufbau occupation splits a degenerate
 * shell; in that case the occupied member of the shell differs from the complex solver's arbitrary
 * choice, as it may between LAPACK builds. */
int tcscf_set_scf_options(tcscf_ctx * ctx, int diis, int real_eigensolve);
/* Zero initial density, Fock build (direct form at `precision`), FP64 generalized Hermitian
 * eigen-solve on the device (upper triangle, as LAPACK zhegvd in the reference; see
 * tcscf_set_scf_options for the real-harmonic alternative), new density,
 * until |dE| < tol or max_iter.  S real [nb][nb].  Outputs: energy, iterations, density, eigenvalues
 * [nspin][nb].  Returns TCSCF_ERR_NOT_CONVERGED after max_iter. */
int tcscf_scf(tcscf_ctx * ctx, int r1, int r2, int nspin, int n_up, int n_down, const double * S, const double * h,
              int respect_symmetry, int precision, double tol, int max_iter, double * energy, int * iterations,
              double * density, double * eigenvalues);

/* RCSHartreeFock::compute (HartreeFock.cpp:785-882) with the whole loop on the device (no reference
 * counterpart to the mechanism): from the zero density, every iteration builds the Fock matrix at
 * `precision` from the occupied coefficients (the density's factor D = C C^T, rank n_up), assembles
 * G, F and the energy as tcscf_scf does, tests |dE| < tol on the device, and takes the next C from
 * the Fock matrix in the real-harmonic basis: canonical orthogonalisation of S (eigenvalues of S
 * above 1e-12 of the largest kept; computed once), a device Jacobi eigen-solve, the n_up lowest
 * eigenvectors.  With capture != 0 the iterations after the first two run as one CUDA graph launch whose
 * conditional WHILE node repeats the iteration until the device-side test ends the loop, so the host
 * reads nothing per iteration; with capture == 0 the same launches are issued per iteration and the
 * host reads the loop state after each (results bit-identical to the captured run).  Restricted closed
 * shell (n_up == n_down), nb <= 128, a density that is real in the real-harmonic basis (the real
 * eigen-solve of tcscf_set_scf_options); the tensor-core precisions need n_up within one launch's
 * rank (32 for nb > 64, else 64).  Outputs as tcscf_scf (eigenvalues: the orthogonalised problem's,
 * ascending; NaN beyond their count) and graph_launches (1 when the loop ran as a graph, may be NULL).
 * Returns TCSCF_ERR_NOT_CONVERGED after max_iter. */
int tcscf_scf_graph(tcscf_ctx * ctx, int r1, int r2, int n_up, int n_down, const double * S, const double * h, int respect_symmetry,
                    int precision, double tol, int max_iter, int capture, double * energy, int * iterations, double * density,
                    double * eigenvalues, int * graph_launches);

/* ---- transcorrelated Fock build and SCF (TCHartreeFock, HartreeFock.cpp:102-609, :1007-1362) ---- */
/* One TC Fock build from device-resident tensors: Fji same / opposite spin (computeF with
 * TCSCF_K_TC_SCALAR_SAME / _OPPO) and Vji same / opposite (computeV with TCSCF_K_GRAD_U_SAME / _OPPO),
 * all on the r1 grid, whose basis gradients must be stored.  density [2][nb][nb] complex; occupied
 * orbitals occ_up / occ_down complex, column-major nb x n_up / nb x n_down (occupiedOrbitals,
 * PERM_JI); h real [nb][nb].  Outputs (any may be NULL): G2, G3, Fock [2][nb][nb] complex (after the
 * symmetry mask), energy = sum D(i,j) (h + G2/2 - G3/3)(j,i). */
int tcscf_tc_fock_build(tcscf_ctx * ctx, int r1, int fji_same, int fji_oppo, int vji_same, int vji_oppo, int n_up, int n_down,
                        const double * density, const double * occ_up, const double * occ_down, const double * h,
                        int respect_symmetry, double * G2, double * G3, double * fock, double * energy);
/* computeQ (HartreeFock.cpp:613-683; the reference keeps it, and its comparison with the G_3 of
 * tcscf_tc_fock_build, commented out in TCHartreeFock::compute): the 6-index tensors
 * Q[j][p][r][i][q][s] = sum_r1 w (conj(b_j) (V_pq . V_rs) b_i + conj(b_p) (V_ji . V_rs) b_q
 * + conj(b_r) (V_ji . V_pq) b_s) for the same-same, same-opposite and opposite-opposite pairs of the
 * computeV handles vji_same / vji_oppo on the r1 grid.  Outputs complex [nb]^6 row-major.  Limited by
 * device memory: UNSUPPORTED when its four nb^6 complex buffers (12 GiB at nb = 24) would take more than
 * 3/4 of the device (and for nb > 46). */
int tcscf_tc_compute_q(tcscf_ctx * ctx, int r1, int vji_same, int vji_oppo, double * Qss, double * Qso, double * Qoo);
/* assembleG (HartreeFock.cpp:687-752, without its debugging checks): G3 [2][nb][nb] complex from the
 * three Q tensors and the spin densities [2][nb][nb] complex (element (q, p) at [q][p]).  Limited by
 * device memory like tcscf_tc_compute_q (three nb^6 complex buffers). */
int tcscf_tc_assemble_g(tcscf_ctx * ctx, int nb, const double * Qss, const double * Qso, const double * Qoo, const double * density,
                        double * G3);

/* TCHartreeFock::compute: zero initial density, TC Fock build, the non-Hermitian pencil F C = S C e
 * solved on the device (Cholesky of S, cusolverDnXgeev), eigenvalues sorted by real part, occupied
 * vectors orthogonalised by the S-metric modified Gram-Schmidt of orthogonalization.hpp:136-154,
 * until |dE| < tol.  S real [nb][nb].  Outputs: energy, iterations, density [2][nb][nb], and the
 * occupied pseudo-energies [2][nb] (first n_up / n_down entries; may be NULL).
 * Returns TCSCF_ERR_NOT_CONVERGED after max_iter. */
int tcscf_tc_scf(tcscf_ctx * ctx, int r1, int fji_same, int fji_oppo, int vji_same, int vji_oppo, const double * S, const double * h,
                 int n_up, int n_down, int respect_symmetry, double tol, int max_iter, double * energy, int * iterations,
                 double * density, double * pseudo_energies);

#ifdef __cplusplus
}
#endif

#endif /* TCSCF_GPU_H */
