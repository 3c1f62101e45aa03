// Shared declarations of libtcscf_gpu.so: the context, device-resident grids and tensors, error
// plumbing and small device helpers.  Everything here is product code for sm_100a.
#pragma once

#include <cuda_runtime.h>
#include <cublas_v2.h>
#include <cusolverDn.h>
#include <nvtx3/nvToolsExt.h>
#include <cmath>
#include <cstdint>
#include <array>
#include <map>
#include <string>
#include <vector>

#include "../../include/tcscf_gpu.h"
#include "basis.cuh"

namespace tcscf {

constexpr int kMaxL = 12;            // highest angular momentum the device basis evaluator accepts
constexpr double kPi = 3.141592653589793238462643383279502884;

// Per basis function data the device evaluators read (SlaterTypeOrbital.hpp:27-37 fields plus the
// real-harmonic type used by the tensor paths).


struct Grid {
  int64_t n = 0;
  int ndim = 3;
  double * pts = nullptr;   // [3][n] Cartesian (y row zero for 2-D grids)
  double * w = nullptr;     // [n]
  // basis
  int nb = 0;
  int hasGrad = 0;
  std::vector<tcscf_sto> basis;
  DevSto * dsto = nullptr;  // [nb]
  double * phiR = nullptr;  // real-harmonic basis values [n][nb]
  double * vals = nullptr;  // reference-basis values [n][nb] (complex for ndim 3, real for ndim 2)
  double * grads = nullptr; // [n][nb][3] complex
  // tensor-path cache of the transposed, BF16-split weighted basis values (depends only on the
  // grid and basis, so it is packed once per grid)
  void * vtCache = nullptr;
  int vtNB = 0;
  int64_t vtN2pad = 0;
  double vtScale = 0;
};

struct Tensor {
  double * d = nullptr;
  int64_t n1 = 0;
  int nb = 0;
  int isComplex = 1;
  int vec = 0;  // 3 components (Vji)
};

struct Scratch {
  void * p = nullptr;
  size_t bytes = 0;
};

// pairs (r1 index, r2 index) of two grids that the tensor-core kernels drop for FP32 resolution but
// that are not exactly coincident in FP64 (near_pairs.cu); d is device memory, null when count is 0
struct NearList {
  int2 * d = nullptr;
  int count = 0;
};

}  // namespace tcscf

struct tcscf_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cusolverDnHandle_t solver = nullptr;
  cublasHandle_t blas = nullptr;   // created on first use (4- and 6-index tensors)
  // stream-ordered pool of the grid buffers (points, weights, basis values and gradients, the
  // packed tensor-path operand): grids created and destroyed between SCF runs reuse its memory
  // without driver allocations or the device-wide synchronisation of cudaFree
  cudaMemPool_t gridPool = nullptr;
  std::string err;
  std::map<int, tcscf::Grid> grids;
  std::map<int, tcscf::Tensor> tensors;
  int nextId = 1;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  double lastContractionMs = 0, lastTotalMs = 0;
  int lastLaunches = 0;
  int launchCount = 0;
  int diisSize = 0;   // Pulay DIIS history length of tcscf_scf (0: plain Roothaan iterations)
  // CUDA graph of the most recent batched tensor launch sequence and the launch parameters it was
  // captured with (replayed while a batch repeats them); capture / replay counts
  cudaGraphExec_t tensorGraph = nullptr;
  std::vector<uint64_t> tensorGraphKey;
  int graphCaptures = 0, graphReplays = 0;
  int realEigen = 0;  // tcscf_scf solves a Fock matrix that is real in the real-harmonic basis there
  // set while a conditional graph body is captured: the contraction routines then record no timing
  // events (event nodes are not allowed inside a conditional body)
  int capturing = 0;
  // autotuner (tcscf_set_autotune): the measured schedule (r2 split count, tile class) of the tensor-path launch per shape
  // {n1, n2, padded nb, padded rank, precision}, the split policy per batch signature, the policy
  // the batch build applies (1: the default rule, 0: no split, k > 1: k x the default split),
  // candidate measurements taken, and the two events that time them
  int autotune = 0;
  std::map<std::vector<int64_t>, std::array<int, 3>> tunedSplit;   // {r2 split, T tile width, TMA stages}
  std::map<std::vector<int64_t>, int> tunedBatchPolicy;
  int batchSplitPolicy = 1;
  int tuneMeasurements = 0;
  cudaEvent_t tuneEv[2] = {nullptr, nullptr};
  std::map<std::string, tcscf::Scratch> scratch;
  // near-coincident pair lists per (r1 grid, r2 grid), found on the first tensor-core use of the pair
  std::map<std::pair<const void *, const void *>, tcscf::NearList> nearPairs;
  // device buffers of the most recent direct Fock build (for tcscf_last_potentials)
  const double * lastVH = nullptr;
  const double * lastT = nullptr;
  int64_t lastN1 = 0;
  int lastNb = 0;
};

namespace tcscf {

int fail(tcscf_ctx * ctx, int code, std::string const & msg);

#define TCSCF_CUDA(ctx, call)                                                                 \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return ::tcscf::fail((ctx), TCSCF_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define TCSCF_LAUNCH(ctx)                                                                     \
  do {                                                                                        \
    (ctx)->launchCount++;                                                                     \
    cudaError_t e_ = cudaGetLastError();                                                      \
    if (e_ != cudaSuccess)                                                                    \
      return ::tcscf::fail((ctx), TCSCF_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
  } while (0)

#define TCSCF_CHECK(ctx, cond, code, msg)                                                     \
  do {                                                                                        \
    if (!(cond)) return ::tcscf::fail((ctx), (code), (msg));                                  \
  } while (0)

#define TCSCF_TRY(expr)                                                                       \
  do {                                                                                        \
    int s_ = (expr);                                                                          \
    if (s_ != TCSCF_OK) return s_;                                                            \
  } while (0)

// NVTX range named after the enclosing C-ABI function: profilers that record NVTX show each call
// (and filter kernels by it); without such a tool attached the push and pop do nothing
struct NvtxRange {
  explicit NvtxRange(char const * name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(NvtxRange const &) = delete;
  NvtxRange & operator=(NvtxRange const &) = delete;
};
#define TCSCF_NVTX() ::tcscf::NvtxRange tcscfNvtxRange_(__func__)

// context-owned scratch buffer, grown on demand and kept until the context is destroyed
int scratch(tcscf_ctx * ctx, char const * name, size_t bytes, void ** out);

Grid * findGrid(tcscf_ctx * ctx, int id);

// grid buffers from the context's pool, ordered on ctx->stream; every allocation is checked to be
// 256-byte aligned (vector loads and TMA descriptors rely on it)
int gridAllocBytes(tcscf_ctx * ctx, void ** p, size_t bytes);
template <class T> int gridAlloc(tcscf_ctx * ctx, T ** p, size_t bytes)
{
  void * q = nullptr;
  int const st = gridAllocBytes(ctx, &q, bytes);
  *p = static_cast<T *>(q);
  return st;
}
// returns a grid buffer to the pool in stream order (null is ignored)
void gridRelease(tcscf_ctx * ctx, void * p);
// releases every buffer of a grid and clears its pointers
void gridReleaseAll(tcscf_ctx * ctx, Grid & g);

inline unsigned gridBlocks(int64_t n, int threads)
{
  int64_t b = (n + threads - 1) / threads;
  return unsigned(b < 1 ? 1 : (b > 1048576 ? 1048576 : b));
}

// ---- kernels shared between translation units -------------------------------------------------
// r12 kernel evaluation in FP64 (scalar kernels); returns 0 for an exactly coincident pair.
struct OchiDev {
  double a, a12;
  int nterms;
  int S[8][3];
  double c[8][2];
};

__device__ __forceinline__ double rsqrt_fp64(double x)
{
  // 1/sqrt(x) by two Newton-Raphson steps from the FP32 hardware estimate (quadratic convergence:
  // ~2^-22 -> 2^-44 -> below FP64 rounding): y <- y (3 - x y^2) / 2, then the same step in the
  // residual form y + y (1 - x y^2) / 2 with the residual by FMA, which rounds faithfully
  double y = double(rsqrtf(float(x)));
  double const h = x * y;
  y = y * fma(-0.5 * h, y, 1.5);
  double const r = fma(-x * y, y, 1.0);
  return fma(0.5 * y, r, y);
}

}  // namespace tcscf
