// Internal launcher interfaces shared by the translation units of libtcscf_gpu.so.
#pragma once

#include <cuda.h>

#include "common.cuh"

namespace tcscf {

// One r12 contraction  T[r1][c] = sum_r2 g(r1,r2) * rho(r1,r2) * V[r2][c]  (+ Coulomb potential
// VH[r1] = sum_r2 g(r1,r2) * coul[r2]) with rho(r1,r2) = sum_b psi1[r1][b] psi2[r2][b].
// With R == 0 rho is 1 (precompute form: V holds weighted basis-pair products).
struct Contraction {
  int64_t n1 = 0, n2 = 0;
  int R = 0;                       // rank of rho (columns of psi1 / psi2)
  int ncol = 0;                    // columns of V / T
  const double * p1 = nullptr;     // [3][n1]
  const double * p2 = nullptr;     // [3][n2]
  const double * psi1 = nullptr;   // [n1][ldpsi]
  const double * psi2 = nullptr;   // [n2][ldpsi]
  int ldpsi = 0;
  const double * coul = nullptr;   // [n2] or null
  const double * V = nullptr;      // [n2][ldv]
  int ldv = 0;
  double * T = nullptr;            // [n1][ldt]
  int ldt = 0;
  double * VH = nullptr;           // [n1] (required when coul != null)
  const void * vtPacked = nullptr; // optional pre-packed Vt of the tensor path (slices and column scales)
  int kernel = TCSCF_K_INV_R12;    // r12 kernel g (vector kernels use `component`)
  int component = 0;
  const tcscf_ochi * jastrow = nullptr;
  int nSplit = 0;                  // r2 split count of the tensor-path launch (0: the default rule)
  int tileNB = 0;                  // T tile width the autotuner asks for (0, or 128 where the rule gives 64)
  int stages = 0;                  // TMA stage count the autotuner asks for (0: the rule)
  // split-BF16 direct form with r1 and r2 the same points (p1 == p2) and psi1 == psi2: compute only the
  // r2 blocks on and above each r1 tile's diagonal (the diagonal tile at half weight); T then holds
  // T' with sum_r1 W T + (sum_r1 W T)^T the full result, and VH is complete (its lower part from
  // the Coulomb row sums over the skipped blocks)
  int sym = 0;
  const NearList * near = nullptr; // tensor paths: pairs dropped in FP32 that the FP64 rule keeps
};

// near-coincident pairs (near_pairs.cu): the list of (g1, g2), found once per grid pair and kept on the
// context; its release when a grid goes away; the FP64 contributions of the listed pairs added to
// c.T (and c.VH) after a tensor contraction of c (direct form when c.R > 0, else the precompute form)
int nearPairsFor(tcscf_ctx * ctx, Grid const & g1, Grid const & g2, NearList const ** out);
void nearPairsForget(tcscf_ctx * ctx, Grid const * g);
int nearCorrect(tcscf_ctx * ctx, Contraction const & c);

int contractFp64(tcscf_ctx * ctx, Contraction const & c);

// one warp waits through the tensor kernels' bounded-wait helper on an mbarrier that nothing arrives
// at, for limitMs; returns TCSCF_ERR_TIMEOUT when the wait gave up (the expected outcome)
int boundedWaitSelfTest(tcscf_ctx * ctx, double limitMs);

// the context's cuBLAS handle (created on first use), bound to the context stream
int blasHandle(tcscf_ctx * ctx, cublasHandle_t * out);

// tensor-core (tcgen05) contraction of the same quantity for g = 1/r12: split-BF16 (flash_tc.cu) or
// TF32 (flash_tf32.cu)
int contractTensor(tcscf_ctx * ctx, Contraction const & c, int precision);
// tensor-core precompute form (flash_pairs.cu): T[r1][p] = sum_r2 g(r1,r2) V[r2][p] with rho == 1
// (c.R == 0) for the kernel c.kernel (component c.component of a vector kernel), g generated in FP32
// and contracted in the split-BF16 scheme of the Fock build; TC kernels need a Jastrow factor of r12
// alone
bool pairsTensorAvailable(Contraction const & c, int precision, std::string * why);
int contractPairsTensor(tcscf_ctx * ctx, Contraction const & c, int precision);
// r2 split counts the autotuner measures for a tensor-path launch over n1 x n2 points on sms SMs:
// the default rule's count first, then 1, 2, 3, 4, 6 and 8 where every split keeps at least 16
// r2 blocks of 64 points (effective counts after rounding the blocks per split, no repeats)
std::vector<int> splitCandidates(int64_t n1, int64_t n2, int sms);
// the split count a batch instance gets under a batch split policy (1: the default rule, 0: no
// split, k > 1: k x the default count, at most the candidates' limit)
int splitForPolicy(Contraction const & c, int precision, int policy);
// one launch of the tensor path (contractTensor splits a larger density factor rank into chunks of
// tensorRankLimit columns)
bool tensorPathAvailable(Contraction const & c, int precision, std::string * why);
int tensorRankLimit(Contraction const & c, int precision);
// packs (once per grid) the transposed operand Vt of the tensor path from V [n2][nb]: BF16 slices
// hi/lo [NB][n2pad] followed by the per-block column scales
int tensorPackedV(tcscf_ctx * ctx, Grid & g2, const double * V, double scale, const void ** packed);

// F = h + G - G3 (G3 may be null), masked where h == 0 when respectSym, and the compensated energy
// factor * sum D(i,j) (h + G/2 - G3/3)(j,i) (constructSCFOperator, HartreeFock.cpp:48-98); G is
// written back masked
int finalizeLaunch(tcscf_ctx * ctx, int nspin, int nb, const double * h, double2 * G, const double2 * G3, const double2 * D, int respectSym,
                   double factor, double2 * fock, double * energy);

// One contraction problem as the tensor kernel sees it (device pointers); a launch covers one or many
// of them (batched builds), all with the same tile shapes NB, RP.
struct TensorInstance {
  int nTiles, nSplit, blocksPerSplit, nBlocks;   // r1 tiles; r2 splits; r2 blocks per split and in total
  int n1;                                          // real r1 rows
  int nb;                                          // real columns of T
  int ldt, pad;
  // symmetric instance: r1 and r2 are the same points and rho(r1, r2) = rho(r2, r1) (psi1 = psi2), so
  // X is symmetric; a tile then takes only the r2 blocks from its own diagonal on, the diagonal
  // tile at half weight, and the caller adds the transpose of the result
  int sym, symPad;
  const float4 * r1xyz;                            // [n1pad] x, y, z, 0
  const float4 * r2pairs;                          // [nBlocks*64] r2 points in pair layout
  const float * a1inv;                             // [n1pad] 1 / psi1 row scale
  const float * a2inv;                             // [nBlocks*64] 1 / psi2 row scale
  const float * cinv;                              // [nBlocks][NB] 1 / Vt column scale
  double * T;                                      // [nSplit][n1][ldt]
  double * VH;                                     // [nSplit][n1]
  int64_t tStride, vhStride;
  const CUtensorMap * maps;                        // device memory, 64-byte aligned: psi1 h/m/l/m/256, psi2 h/m/l, Vt h/m/l
};
constexpr int kTensorMapsPerInstance = 10;

// a contraction whose operands are packed (tensorPrepare) and ready for tensorRun
struct TensorPrep {
  int NB = 0, RP = 0, XS = 2;   // Vt tile columns, rank padding, X slices (2: 16 bits, 3: 24 bits; 0: the TF32 kernel)
  int NS = 0;                   // TMA stages of the split-BF16 kernel
  Contraction c;
  TensorInstance inst{};
  CUtensorMap maps[kTensorMapsPerInstance];
};

// Batched tensor contractions: the operands of one contraction are packed into a caller-provided
// device arena of tensorArenaBytes(c) bytes (tensorPrepare); any number of prepared contractions then
// run in one persistent launch per tile class (tensorRun), which also sums the r2-split partials
// into c.T / c.VH.
size_t tensorArenaBytes(Contraction const & c, int precision = TCSCF_PREC_BF16X3);
int tensorPrepare(tcscf_ctx * ctx, Contraction const & c, int precision, void * arena, size_t arenaBytes, TensorPrep & tp);
int tensorRun(tcscf_ctx * ctx, TensorPrep * const * preps, int count, bool recordStart = true);

// A single prepared contraction whose device tables (instance, tensor maps) and status word are
// uploaded once (tensorPlanUpload, which synchronises); tensorPlanLaunch then issues the persistent
// launch and the split sums with no host synchronisation and no host memory read, so a CUDA graph can
// capture it and replay it while the prepared operands keep their addresses (re-packed in place by
// tensorPrepare on the same arena).  The status word accumulates over launches (0 = every bounded
// wait completed).
struct TensorPlan {
  int NB = 0, RP = 0, XS = 0, NS = 0, grid = 0, nItems = 0;
  const void * inst = nullptr;
  int * status = nullptr;
  const void * items = nullptr;   // the work items (int4) in the order the persistent CTAs take them
  double * lowerPart = nullptr;   // chunk partials of the Coulomb rows below the diagonal tiles (symmetric instances)
  TensorPrep * prep = nullptr;
};
int tensorPlanUpload(tcscf_ctx * ctx, TensorPrep & tp, char const * scratchName, TensorPlan & plan);
int tensorPlanLaunch(tcscf_ctx * ctx, TensorPlan const & plan);

// out[r][c] = sum_s part[s*stride + r*ldPart + c] for r < rows, c < cols (deterministic split sum)
int sumSplitsLaunch(tcscf_ctx * ctx, int64_t n, int nsplit, int64_t stride, const double * part, double * out, int64_t rows, int cols,
                    int ldOut, int ldPart);

// G_s[k][l] (+)= sum_r1 w1 phi[r1][k] * (cJ * phi[r1][l] * VH[r1] - sgnT * T[r1][l]); real, out [nb][nb]
int reduceFockReal(tcscf_ctx * ctx, int64_t n1, int nb, const double * phi, const double * w1, const double * VH, double cJ,
                   const double * T, int ldt, double sgnT, double * out);

// complex reduction G(j,i) = sum_r w[r] conj(A[r][j]) Y[r][i] with Y = cJ * A[r][i] * Faa[r] - Fai[r][i]
int reduceFockComplex(tcscf_ctx * ctx, int64_t n1, int nb, const double * A, const double * w, const double * Faa, double cJ,
                      const double * Fai, double * out);

}  // namespace tcscf
