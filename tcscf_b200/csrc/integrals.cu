// 4- and 6-index r12 integral tensors on the GPU (FP64):
//
//   integrateAllR1R2 (integrateAll.hpp:221-317, evaluateR2Integral :152-180, evaluateR2GradientIntegral
//   :187-216): with a 3-D r1 grid and a 2-D r2 grid,
//     (b1 b2|f|b3 b4) = sum_r1 w1 conj(phi_b1) phi_b3 (r1) * 2 pi sum_r2 w2 phi_b2 f(r1,r2) phi_b4 (r2)
//     stored [b1][b2][b3][b4]; the gradient form replaces f phi_b4 by grad1 u(r1,r2) . grad phi_b4(r2)
//     and stores [b2][b1][b4][b3] (integrateAll.hpp:302).
//   threeElectronIntegrals (integrateAll.hpp:361-442, computeV :328-356): with V(r1,q,t) =
//     sum_r2 w2 conj(phi_q) phi_t grad1 u (same spin),
//     answer[p][q][r][s][t][u] = sum_r1 w1 conj(phi_p) phi_s (r1) V(r1,q,t) . V(r1,r,u).
//
// The r2 sums are the library's FP64 r12 contraction (kernel generated on the fly, never stored);
// the r1 sums are one dense GEMM  C[(b1,b3)][(b2,b4)] = sum_r1 A[r1][(b1,b3)] B[r1][(b2,b4)]  on
// cuBLAS (DGEMM when B is real, ZGEMM otherwise; chunked over r1 for the 6-index tensor), followed by
// a permutation into the reference's index order.  The reference's atomics have no fixed summation
// order; here the order is fixed.
#include <cublas_v2.h>

#include "kernels.cuh"

namespace tcscf {
namespace {

constexpr double kTwoPi = 2.0 * 3.141592653589793238462643383279502884;

// A[r1][(b1,b3)] = w1 conj(v1[r1][b1]) v1[r1][b3] for rows [a0, a0 + rows)
__global__ void kR1Pairs(int64_t a0, int64_t rows, int nb, const double2 * __restrict__ vals, const double * __restrict__ w,
                         double2 * __restrict__ A)
{
  int64_t const nn = int64_t(nb) * nb;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < rows * nn; idx += int64_t(gridDim.x) * blockDim.x) {
    int64_t const a = a0 + idx / nn;
    int const k = int(idx % nn);
    double2 const x = vals[a * nb + k / nb], y = vals[a * nb + k % nb];
    double const re = x.x * y.x + x.y * y.y, im = x.x * y.y - x.y * y.x;
    A[idx] = make_double2(w[a] * re, w[a] * im);
  }
}

// r2 operand of the gradient form, component d: V[r2][(b2,b4)] = 2 pi w2 phi_b2(r2) (grad phi_b4(r2))_d as
// interleaved (re, im) columns; 2-D r2 grid (real values, complex gradients [n][nb][3])
__global__ void kGradPairs(int64_t n2, int nb, int d, const double * __restrict__ vals2, const double2 * __restrict__ grads2,
                           const double * __restrict__ w2, double * __restrict__ V)
{
  int64_t const nn = int64_t(nb) * nb;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < n2 * nn; idx += int64_t(gridDim.x) * blockDim.x) {
    int64_t const r = idx / nn;
    int const k = int(idx % nn);
    int const b2 = k / nb, b4 = k % nb;
    double const s = kTwoPi * w2[r] * vals2[r * nb + b2];
    double2 const g = grads2[(r * nb + b4) * 3 + d];
    V[2 * idx] = s * g.x;
    V[2 * idx + 1] = s * g.y;
  }
}

__global__ void kAccumulate(int64_t n, const double * __restrict__ x, double * __restrict__ y, int first)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    y[i] = first ? x[i] : y[i] + x[i];
}

// C column-major [(b1,b3)][(b2,b4)] -> the reference's 4-index layouts
__global__ void kPermute4(int nb, int gradientOrder, const double2 * __restrict__ C, double2 * __restrict__ out)
{
  int64_t const nn = int64_t(nb) * nb, n4 = nn * nn;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < n4; idx += int64_t(gridDim.x) * blockDim.x) {
    int64_t k = idx;
    int const i3 = int(k % nb); k /= nb;
    int const i2 = int(k % nb); k /= nb;
    int const i1 = int(k % nb); k /= nb;
    int const i0 = int(k);
    // non-gradient: out[b1][b2][b3][b4]; gradient: out[b2][b1][b4][b3]
    int const b1 = gradientOrder ? i1 : i0, b2 = gradientOrder ? i0 : i1;
    int const b3 = gradientOrder ? i3 : i2, b4 = gradientOrder ? i2 : i3;
    out[idx] = C[(int64_t(b1) * nb + b3) + (int64_t(b2) * nb + b4) * nn];
  }
}

// Y[r1][(q,t),(r,u)] = sum_d V[r1][q][t][d] V[r1][r][u][d] for rows [a0, a0 + rows)
__global__ void kVDotV(int64_t a0, int64_t rows, int nb, const double2 * __restrict__ V, double2 * __restrict__ Y)
{
  int64_t const nn = int64_t(nb) * nb, n4 = nn * nn;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < rows * n4; idx += int64_t(gridDim.x) * blockDim.x) {
    int64_t const a = a0 + idx / n4;
    int64_t const k = idx % n4;
    int64_t const qt = k / nn, ru = k % nn;
    double2 const * x = V + (a * nn + qt) * 3;
    double2 const * y = V + (a * nn + ru) * 3;
    double re = 0, im = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      re += x[d].x * y[d].x - x[d].y * y[d].y;
      im += x[d].x * y[d].y + x[d].y * y[d].x;
    }
    Y[idx] = make_double2(re, im);
  }
}

// C column-major [(p,s)][(q,t,r,u)] -> answer[p][q][r][s][t][u]
__global__ void kPermute6(int nb, const double2 * __restrict__ C, double2 * __restrict__ out)
{
  int64_t const nn = int64_t(nb) * nb, n6 = nn * nn * nn;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < n6; idx += int64_t(gridDim.x) * blockDim.x) {
    int64_t k = idx;
    int const u = int(k % nb); k /= nb;
    int const t = int(k % nb); k /= nb;
    int const s = int(k % nb); k /= nb;
    int const r = int(k % nb); k /= nb;
    int const q = int(k % nb); k /= nb;
    int const p = int(k);
    int64_t const ps = int64_t(p) * nb + s, qtru = ((int64_t(q) * nb + t) * nb + r) * nb + u;
    out[idx] = C[ps + qtru * nn];
  }
}


int checkPair(tcscf_ctx * ctx, Grid * g1, Grid * g2, int ndim2)
{
  TCSCF_CHECK(ctx, g1 && g2, TCSCF_ERR_INVALID_ARGUMENT, "unknown grid handle");
  TCSCF_CHECK(ctx, g1->nb > 0 && g1->nb == g2->nb, TCSCF_ERR_INVALID_ARGUMENT, "both grids need the same basis");
  TCSCF_CHECK(ctx, g1->ndim == 3, TCSCF_ERR_INVALID_ARGUMENT, "the r1 grid must be three dimensional");
  TCSCF_CHECK(ctx, g2->ndim == ndim2, TCSCF_ERR_INVALID_ARGUMENT,
              ndim2 == 2 ? "integrateAllR1R2 takes a two-dimensional r2 grid" : "threeElectronIntegrals takes a three-dimensional r2 grid");
  return TCSCF_OK;
}

// Y[a][(p,q),(r,s)] = Vx_pq(a) . Vy_rs(a) (complex Cartesian dot, no conjugate) for r1 rows a0..a0+rows
__global__ void kVDotV2(int64_t a0, int64_t rows, int nb, const double2 * __restrict__ Vx, const double2 * __restrict__ Vy,
                        double2 * __restrict__ Y)
{
  int64_t const nn = int64_t(nb) * nb, n4 = nn * nn;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < rows * n4; idx += int64_t(gridDim.x) * blockDim.x) {
    int64_t const a = a0 + idx / n4;
    int64_t const k = idx % n4;
    int64_t const pq = k / nn, rs = k % nn;
    double2 const * x = Vx + (a * nn + pq) * 3;
    double2 const * y = Vy + (a * nn + rs) * 3;
    double re = 0, im = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      re += x[d].x * y[d].x - x[d].y * y[d].y;
      im += x[d].x * y[d].y + x[d].y * y[d].x;
    }
    Y[idx] = make_double2(re, im);
  }
}

// computeQ's three terms from T[(ji)][(pq)][(rs)] = sum_r1 w conj(b_j) b_i (V_pq . V_rs), stored
// column-major as C[(ji) + nn ((pq) nn + (rs))]:
// Q[j][p][r][i][q][s] = T[ji][pq][rs] + T[pq][ji][rs] + T[rs][ji][pq]   (HartreeFock.cpp:655-673)
__global__ void kAssembleQ(int nb, const double2 * __restrict__ C, double2 * __restrict__ Q)
{
  int64_t const nn = int64_t(nb) * nb, n6 = nn * nn * nn;
  auto T = [&](int64_t a, int64_t b, int64_t c) { return C[a + nn * (b * nn + c)]; };
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < n6; idx += int64_t(gridDim.x) * blockDim.x) {
    int64_t k = idx;
    int const s = int(k % nb); k /= nb;
    int const q = int(k % nb); k /= nb;
    int const i = int(k % nb); k /= nb;
    int const r = int(k % nb); k /= nb;
    int const p = int(k % nb); k /= nb;
    int const j = int(k);
    int64_t const ji = int64_t(j) * nb + i, pq = int64_t(p) * nb + q, rs = int64_t(r) * nb + s;
    double2 const a = T(ji, pq, rs), b = T(pq, ji, rs), c = T(rs, ji, pq);
    Q[idx] = make_double2(a.x + b.x + c.x, a.y + b.y + c.y);
  }
}

__device__ __forceinline__ double2 cmulQ(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }

// assembleG (HartreeFock.cpp:687-752, without its debugging checks): one thread per (j, i)
__global__ void kAssembleG(int nb, const double2 * __restrict__ SS, const double2 * __restrict__ SO, const double2 * __restrict__ OO,
                           const double2 * __restrict__ D, double2 * __restrict__ G3)
{
  int64_t const nn = int64_t(nb) * nb;
  for (int64_t ji = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; ji < nn; ji += int64_t(gridDim.x) * blockDim.x) {
    int const j = int(ji / nb), i = int(ji % nb);
    auto Qv = [&](const double2 * T, int p, int r, int x, int y, int z) {
      return T[((((int64_t(j) * nb + p) * nb + r) * nb + x) * nb + y) * nb + z];
    };
    double2 value[2] = {make_double2(0, 0), make_double2(0, 0)};
    for (int p = 0; p < nb; ++p)
      for (int q = 0; q < nb; ++q)
        for (int r = 0; r < nb; ++r)
          for (int s = 0; s < nb; ++s) {
            double2 const ss1 = Qv(SS, p, r, i, q, s), ss2 = Qv(SS, p, r, i, s, q), ss3 = Qv(SS, p, r, q, s, i), ss4 = Qv(SS, p, r, s, q, i);
            double2 const so1 = Qv(SO, p, r, i, q, s), so2 = Qv(SO, p, r, q, i, s);
            double2 const oo1 = Qv(OO, p, r, i, q, s), oo2 = Qv(OO, p, r, i, s, q);
            double2 const tss = make_double2(ss1.x - ss2.x + 2 * ss3.x - 2 * ss4.x, ss1.y - ss2.y + 2 * ss3.y - 2 * ss4.y);
            double2 const tso = make_double2(2 * (so1.x - so2.x), 2 * (so1.y - so2.y));
            double2 const too = make_double2(oo1.x - oo2.x, oo1.y - oo2.y);
            for (int spin = 0; spin < 2; ++spin) {
              double2 const dqp = D[spin * nn + int64_t(q) * nb + p], dsr = D[spin * nn + int64_t(s) * nb + r];
              double2 const oqp = D[(1 - spin) * nn + int64_t(q) * nb + p], osr = D[(1 - spin) * nn + int64_t(s) * nb + r];
              double2 const a = cmulQ(cmulQ(dqp, dsr), tss), b = cmulQ(cmulQ(dqp, osr), tso), c = cmulQ(cmulQ(oqp, osr), too);
              value[spin].x += a.x + b.x + c.x;
              value[spin].y += a.y + b.y + c.y;
            }
          }
    G3[ji] = make_double2(value[0].x / 2, value[0].y / 2);
    G3[nn + ji] = make_double2(value[1].x / 2, value[1].y / 2);
  }
}

}  // namespace
}  // namespace tcscf

using namespace tcscf;

extern "C" {

int tcscf_integrate_all_r1r2(tcscf_ctx * ctx, int r1, int r2, int use_gradient, int kernel, const tcscf_ochi * jastrow, double * answer)
{
  TCSCF_NVTX();
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  Grid * g1 = findGrid(ctx, r1);
  Grid * g2 = findGrid(ctx, r2);
  TCSCF_TRY(checkPair(ctx, g1, g2, 2));
  TCSCF_CHECK(ctx, answer, TCSCF_ERR_INVALID_ARGUMENT, "answer is required");
  if (use_gradient) {
    TCSCF_CHECK(ctx, kernel == TCSCF_K_GRAD_U_SAME || kernel == TCSCF_K_GRAD_U_OPPO, TCSCF_ERR_INVALID_ARGUMENT,
                "the gradient form takes a vector kernel");
    TCSCF_CHECK(ctx, g2->grads, TCSCF_ERR_INVALID_ARGUMENT, "the gradient form needs r2 gradients");
  } else {
    TCSCF_CHECK(ctx, kernel >= TCSCF_K_INV_R12 && kernel <= TCSCF_K_TC_SCALAR_OPPO, TCSCF_ERR_INVALID_ARGUMENT,
                "the value form takes a scalar kernel");
  }
  TCSCF_CHECK(ctx, kernel == TCSCF_K_INV_R12 || (jastrow && jastrow->nterms >= 0 && jastrow->nterms <= 8), TCSCF_ERR_INVALID_ARGUMENT,
              "TC kernels need the Jastrow parameters (at most 8 terms)");
  int const nb = g1->nb;
  int64_t const nn = int64_t(nb) * nb, n1 = g1->n, n2 = g2->n;
  cublasHandle_t h = nullptr;
  TCSCF_TRY(blasHandle(ctx, &h));

  // r2 side B[r1][(b2,b4)]: real (value form, computeF on the 2-D grid, 2 pi included) or complex
  int fid = 0;
  double * B = nullptr;
  if (!use_gradient) {
    TCSCF_TRY(tcscf_compute_F(ctx, r1, r2, kernel, jastrow, TCSCF_PREC_FP64, nullptr, 1, &fid));
    B = ctx->tensors[fid].d;
  }
  size_t const bytesA = sizeof(double2) * size_t(n1) * nn;
  size_t const bytesB = use_gradient ? sizeof(double2) * size_t(n1) * nn * 2 + sizeof(double2) * size_t(n2) * nn : 0;
  size_t const bytesC = sizeof(double2) * size_t(nn) * nn * 2;
  void * p = nullptr;
  int st = scratch(ctx, "integrate_all", bytesA + bytesB + bytesC, &p);
  if (st != TCSCF_OK) { if (fid) tcscf_tensor_destroy(ctx, fid); return st; }
  double2 * A = static_cast<double2 *>(p);
  double2 * C = A + size_t(n1) * nn;
  double2 * out = C + size_t(nn) * nn;
  if (use_gradient) {
    double * Bsum = reinterpret_cast<double *>(out + size_t(nn) * nn);   // [n1][2 nn]
    double * Td = Bsum + size_t(n1) * nn * 2;                            // [n1][2 nn]
    double * Vd = Td + size_t(n1) * nn * 2;                              // [n2][2 nn]
    for (int d = 0; d < 3; ++d) {
      kGradPairs<<<gridBlocks(n2 * nn, 256), 256, 0, ctx->stream>>>(n2, nb, d, g2->vals, reinterpret_cast<const double2 *>(g2->grads),
                                                                      g2->w, Vd);
      TCSCF_LAUNCH(ctx);
      Contraction c;
      c.n1 = n1; c.n2 = n2; c.R = 0; c.ncol = int(2 * nn); c.p1 = g1->pts; c.p2 = g2->pts; c.V = Vd; c.ldv = int(2 * nn);
      c.T = Td; c.ldt = int(2 * nn); c.kernel = kernel; c.component = d; c.jastrow = jastrow;
      TCSCF_TRY(contractFp64(ctx, c));
      kAccumulate<<<gridBlocks(n1 * nn * 2, 256), 256, 0, ctx->stream>>>(n1 * nn * 2, Td, Bsum, d == 0);
      TCSCF_LAUNCH(ctx);
    }
    B = Bsum;
  }
  kR1Pairs<<<gridBlocks(n1 * nn, 256), 256, 0, ctx->stream>>>(0, n1, nb, reinterpret_cast<const double2 *>(g1->vals), g1->w, A);
  TCSCF_LAUNCH(ctx);
  cublasStatus_t bs;
  if (!use_gradient) {
    double const one = 1.0, zero = 0.0;
    // C (as 2 nn x nn real, column-major) = A (2 nn x n1) * B^T, B = F [n1][nn] real
    bs = cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, int(2 * nn), int(nn), int(n1), &one, reinterpret_cast<const double *>(A), int(2 * nn), B,
                     int(nn), &zero, reinterpret_cast<double *>(C), int(2 * nn));
  } else {
    cuDoubleComplex const one = make_cuDoubleComplex(1, 0), zero = make_cuDoubleComplex(0, 0);
    bs = cublasZgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, int(nn), int(nn), int(n1), &one, reinterpret_cast<const cuDoubleComplex *>(A), int(nn),
                     reinterpret_cast<const cuDoubleComplex *>(B), int(nn), &zero, reinterpret_cast<cuDoubleComplex *>(C), int(nn));
  }
  if (fid) tcscf_tensor_destroy(ctx, fid);
  TCSCF_CHECK(ctx, bs == CUBLAS_STATUS_SUCCESS, TCSCF_ERR_CUDA, "cuBLAS GEMM failed");
  kPermute4<<<gridBlocks(nn * nn, 256), 256, 0, ctx->stream>>>(nb, use_gradient ? 1 : 0, C, out);
  TCSCF_LAUNCH(ctx);
  TCSCF_CUDA(ctx, cudaMemcpyAsync(answer, out, sizeof(double2) * size_t(nn) * nn, cudaMemcpyDeviceToHost, ctx->stream));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TCSCF_OK;
}

int tcscf_three_electron_integrals(tcscf_ctx * ctx, int r1, int r2, const tcscf_ochi * jastrow, double * answer)
{
  TCSCF_NVTX();
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  Grid * g1 = findGrid(ctx, r1);
  Grid * g2 = findGrid(ctx, r2);
  TCSCF_TRY(checkPair(ctx, g1, g2, 3));
  TCSCF_CHECK(ctx, answer, TCSCF_ERR_INVALID_ARGUMENT, "answer is required");
  TCSCF_CHECK(ctx, jastrow && jastrow->nterms >= 0 && jastrow->nterms <= 8, TCSCF_ERR_INVALID_ARGUMENT,
              "the Jastrow parameters are required (at most 8 terms)");
  int const nb = g1->nb;
  int64_t const nn = int64_t(nb) * nb, n4 = nn * nn, n6 = n4 * nn, n1 = g1->n;
  TCSCF_CHECK(ctx, nb <= 32, TCSCF_ERR_UNSUPPORTED, "threeElectronIntegrals: nb <= 32 (the nb^6 output exceeds device memory beyond)");
  cublasHandle_t h = nullptr;
  TCSCF_TRY(blasHandle(ctx, &h));
  int vid = 0;
  TCSCF_TRY(tcscf_compute_V(ctx, r1, r2, TCSCF_K_GRAD_U_SAME, jastrow, TCSCF_PREC_FP64, nullptr, 1, &vid));
  const double2 * V = reinterpret_cast<const double2 *>(ctx->tensors[vid].d);
  // r1 chunk so that the (q,t,r,u) operand stays below ~1 GB
  int64_t const chunk = std::max<int64_t>(1, std::min<int64_t>(n1, (int64_t(1) << 26) / n4));
  size_t const bytes = sizeof(double2) * (size_t(chunk) * nn + size_t(chunk) * n4 + 2 * size_t(n6));
  void * p = nullptr;
  int st = scratch(ctx, "three_electron", bytes, &p);
  if (st != TCSCF_OK) { tcscf_tensor_destroy(ctx, vid); return st; }
  double2 * X = static_cast<double2 *>(p);
  double2 * Y = X + size_t(chunk) * nn;
  double2 * C = Y + size_t(chunk) * n4;
  double2 * out = C + size_t(n6);
  cuDoubleComplex const one = make_cuDoubleComplex(1, 0), zero = make_cuDoubleComplex(0, 0);
  for (int64_t a0 = 0; a0 < n1 && st == TCSCF_OK; a0 += chunk) {
    int64_t const rows = std::min(chunk, n1 - a0);
    kR1Pairs<<<gridBlocks(rows * nn, 256), 256, 0, ctx->stream>>>(a0, rows, nb, reinterpret_cast<const double2 *>(g1->vals), g1->w, X);
    ctx->launchCount++;
    kVDotV<<<gridBlocks(rows * n4, 256), 256, 0, ctx->stream>>>(a0, rows, nb, V, Y);
    ctx->launchCount++;
    // C [(p,s)][(q,t,r,u)] (column-major) += X^T Y over this chunk of r1
    cublasStatus_t const bs = cublasZgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, int(nn), int(n4), int(rows), &one,
                                          reinterpret_cast<const cuDoubleComplex *>(X), int(nn), reinterpret_cast<const cuDoubleComplex *>(Y),
                                          int(n4), a0 == 0 ? &zero : &one, reinterpret_cast<cuDoubleComplex *>(C), int(nn));
    if (bs != CUBLAS_STATUS_SUCCESS) st = fail(ctx, TCSCF_ERR_CUDA, "cuBLAS ZGEMM failed");
    cudaError_t const e = cudaGetLastError();
    if (st == TCSCF_OK && e != cudaSuccess) st = fail(ctx, TCSCF_ERR_CUDA, cudaGetErrorString(e));
  }
  tcscf_tensor_destroy(ctx, vid);
  TCSCF_TRY(st);
  kPermute6<<<gridBlocks(n6, 256), 256, 0, ctx->stream>>>(nb, C, out);
  TCSCF_LAUNCH(ctx);
  TCSCF_CUDA(ctx, cudaMemcpyAsync(answer, out, sizeof(double2) * size_t(n6), cudaMemcpyDeviceToHost, ctx->stream));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TCSCF_OK;
}

// The 6-index tensors are limited by device memory, not by a basis size: UNSUPPORTED when their buffers
// (bytes) would take more than 3/4 of the device, so that the grids and tensors already resident keep room
int sixIndexFits(tcscf_ctx * ctx, size_t bytes, char const * what)
{
  size_t freeB = 0, totalB = 0;
  TCSCF_CUDA(ctx, cudaMemGetInfo(&freeB, &totalB));
  TCSCF_CHECK(ctx, bytes <= totalB / 4 * 3, TCSCF_ERR_UNSUPPORTED,
              std::string(what) + ": the nb^6 tensors need " + std::to_string(bytes >> 20) + " MiB of device memory, beyond 3/4 of the " +
                  std::to_string(totalB >> 20) + " MiB on the device");
  return TCSCF_OK;
}

int tcscf_tc_compute_q(tcscf_ctx * ctx, int r1, int vsame, int voppo, double * Qss, double * Qso, double * Qoo)
{
  TCSCF_NVTX();
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  Grid * g1 = findGrid(ctx, r1);
  TCSCF_CHECK(ctx, g1 && g1->nb > 0 && g1->ndim == 3, TCSCF_ERR_INVALID_ARGUMENT, "computeQ: a 3-D r1 grid with basis values is required");
  TCSCF_CHECK(ctx, Qss && Qso && Qoo, TCSCF_ERR_INVALID_ARGUMENT, "computeQ: three outputs are required");
  auto itS = ctx->tensors.find(vsame), itO = ctx->tensors.find(voppo);
  TCSCF_CHECK(ctx, itS != ctx->tensors.end() && itO != ctx->tensors.end() && itS->second.vec && itO->second.vec, TCSCF_ERR_INVALID_ARGUMENT,
              "computeQ: two computeV tensor handles are required");
  int const nb = g1->nb;
  TCSCF_CHECK(ctx, itS->second.nb == nb && itO->second.nb == nb && itS->second.n1 == g1->n && itO->second.n1 == g1->n,
              TCSCF_ERR_INVALID_ARGUMENT, "computeQ: the tensors do not match the r1 grid");
  TCSCF_CHECK(ctx, nb <= 46, TCSCF_ERR_UNSUPPORTED, "computeQ: nb <= 46 (nb^4 stays an int GEMM dimension)");
  int64_t const nn = int64_t(nb) * nb, n4 = nn * nn, n6 = n4 * nn, n1 = g1->n;
  const double2 * Vs = reinterpret_cast<const double2 *>(itS->second.d);
  const double2 * Vo = reinterpret_cast<const double2 *>(itO->second.d);
  cublasHandle_t h = nullptr;
  TCSCF_TRY(blasHandle(ctx, &h));
  int64_t const chunk = std::max<int64_t>(1, std::min<int64_t>(n1, (int64_t(1) << 26) / n4));
  size_t const bytes = sizeof(double2) * (size_t(chunk) * nn + size_t(chunk) * n4 + 4 * size_t(n6));
  TCSCF_TRY(sixIndexFits(ctx, bytes, "computeQ"));
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, "compute_q", bytes, &p));
  double2 * X = static_cast<double2 *>(p);
  double2 * Y = X + size_t(chunk) * nn;
  double2 * C = Y + size_t(chunk) * n4;        // [3][n6]: same-same, same-opposite, opposite-opposite
  double2 * out = C + 3 * size_t(n6);
  const double2 * pairs[3][2] = {{Vs, Vs}, {Vs, Vo}, {Vo, Vo}};
  cuDoubleComplex const one = make_cuDoubleComplex(1, 0), zero = make_cuDoubleComplex(0, 0);
  for (int64_t a0 = 0; a0 < n1; a0 += chunk) {
    int64_t const rows = std::min(chunk, n1 - a0);
    kR1Pairs<<<gridBlocks(rows * nn, 256), 256, 0, ctx->stream>>>(a0, rows, nb, reinterpret_cast<const double2 *>(g1->vals), g1->w, X);
    TCSCF_LAUNCH(ctx);
    for (int t = 0; t < 3; ++t) {
      kVDotV2<<<gridBlocks(rows * n4, 256), 256, 0, ctx->stream>>>(a0, rows, nb, pairs[t][0], pairs[t][1], Y);
      TCSCF_LAUNCH(ctx);
      // C_t [(ji)][(pq,rs)] (column-major) += X^T Y over this chunk of r1
      cublasStatus_t const bs = cublasZgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, int(nn), int(n4), int(rows), &one,
                                            reinterpret_cast<const cuDoubleComplex *>(X), int(nn), reinterpret_cast<const cuDoubleComplex *>(Y),
                                            int(n4), a0 == 0 ? &zero : &one, reinterpret_cast<cuDoubleComplex *>(C + t * n6), int(nn));
      TCSCF_CHECK(ctx, bs == CUBLAS_STATUS_SUCCESS, TCSCF_ERR_CUDA, "cuBLAS ZGEMM failed");
    }
  }
  double * outs[3] = {Qss, Qso, Qoo};
  for (int t = 0; t < 3; ++t) {
    kAssembleQ<<<gridBlocks(n6, 256), 256, 0, ctx->stream>>>(nb, C + t * n6, out);
    TCSCF_LAUNCH(ctx);
    TCSCF_CUDA(ctx, cudaMemcpyAsync(outs[t], out, sizeof(double2) * size_t(n6), cudaMemcpyDeviceToHost, ctx->stream));
    TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return TCSCF_OK;
}

int tcscf_tc_assemble_g(tcscf_ctx * ctx, int nb, const double * Qss, const double * Qso, const double * Qoo, const double * density, double * G3)
{
  TCSCF_NVTX();
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  TCSCF_CHECK(ctx, nb >= 1 && Qss && Qso && Qoo && density && G3, TCSCF_ERR_INVALID_ARGUMENT, "assembleG: nb >= 1 and all arrays are required");
  TCSCF_CHECK(ctx, nb <= 46, TCSCF_ERR_UNSUPPORTED, "assembleG: nb <= 46");
  int64_t const nn = int64_t(nb) * nb, n6 = nn * nn * nn;
  TCSCF_TRY(sixIndexFits(ctx, sizeof(double2) * (3 * size_t(n6) + 4 * size_t(nn)), "assembleG"));
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, "assemble_g", sizeof(double2) * (3 * size_t(n6) + 4 * size_t(nn)), &p));
  double2 * Q = static_cast<double2 *>(p);
  double2 * D = Q + 3 * size_t(n6);
  double2 * G = D + 2 * size_t(nn);
  double const * in[3] = {Qss, Qso, Qoo};
  for (int t = 0; t < 3; ++t)
    TCSCF_CUDA(ctx, cudaMemcpyAsync(Q + t * n6, in[t], sizeof(double2) * size_t(n6), cudaMemcpyHostToDevice, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemcpyAsync(D, density, sizeof(double2) * 2 * size_t(nn), cudaMemcpyHostToDevice, ctx->stream));
  kAssembleG<<<gridBlocks(nn, 64), 64, 0, ctx->stream>>>(nb, Q, Q + n6, Q + 2 * n6, D, G);
  TCSCF_LAUNCH(ctx);
  TCSCF_CUDA(ctx, cudaMemcpyAsync(G3, G, sizeof(double2) * 2 * size_t(nn), cudaMemcpyDeviceToHost, ctx->stream));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TCSCF_OK;
}

}  // extern "C"
