// Near-coincident pairs of the tensor-core paths.
//
// The tensor kernels (kFlashTc, kFlashTf32, kPairTc) generate the r12 kernel from FP32 coordinates and
// drop every pair whose FP32 squared separation is below nearThreshold(r1) (2^-32 |r1|^2): there FP32
// rounding of the coordinates no longer resolves the separation.  The FP64 path drops only exactly
// coincident pairs (the reference's convention, r12Inv in IntegrationTest.cpp:298-309), so two points
// that differ in FP64 but not in FP32 would contribute in one path and not in the other.  This file
// makes the mixed paths follow the FP64 rule:
//   * kFindNearPairs lists, once per (r1 grid, r2 grid), the pairs the tensor kernels drop that are
//     not exactly coincident in FP64, testing the candidate pairs (the r2 points in a narrow band of
//     radii around |r1|, found in the sorted radii) with the kernels' own FP32 arithmetic on the same
//     packed coordinates (so the decisions agree bit for bit);
//   * after each tensor contraction, kNearDirect / kNearPairs add those pairs' contributions evaluated
//     in FP64 (1/r12 with the FP64 density factors for the direct Fock build, the FP64 kernel value for
//     the precompute form).
// Grids whose points do not nearly coincide (product grids of one rule, independent QMC draws) list
// nothing, and the correction then costs nothing.
#include <cub/device/device_radix_sort.cuh>

#include "tc_device.cuh"

namespace tcscf {
namespace {

constexpr int kFindThreads = 256;

// The FP64 radius of every r2 point and its index (the keys and values of the radius sort).
__global__ void kRadii(int64_t n, const double * __restrict__ p, double * rad, int * idx)
{
  for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < n; j += int64_t(gridDim.x) * blockDim.x) {
    double const x = p[j], y = p[n + j], z = p[2 * n + j];
    rad[j] = sqrt(x * x + y * y + z * z);
    idx[j] = int(j);
  }
}

// One thread per r1 row.  A pair the tensor kernels drop has an FP32 squared separation below
// nearThreshold(r1) = max(2^-32 |r1|^2, smallest normal), so (with the coordinates' FP32 rounding,
// 2^-24 |r| each) |r1 - r2| < 2^-15.9 |r1| + 1.1e-19 and the radii differ by less than that: only the
// r2 points whose radius lies within 2^-14 |r1| + 1e-18 of |r1| (a contiguous range of the sorted
// radii) can be dropped.  Each of them is tested with the kernels' own FP32 arithmetic on the same
// packed coordinates; the dropped pairs that are not exactly coincident in FP64 are appended to out
// (count is incremented for every one; at most cap are stored).
__global__ void __launch_bounds__(kFindThreads) kFindNearPairs(int64_t n1, const float4 * __restrict__ r1c, int64_t n2,
                                                               const float4 * __restrict__ r2pairs, const double * __restrict__ rad,
                                                               const int * __restrict__ idx, const double * __restrict__ p1,
                                                               const double * __restrict__ p2, int2 * out, int cap, int * count)
{
  int64_t const i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n1) return;
  double const x = p1[i], y = p1[n1 + i], z = p1[2 * n1 + i];
  double const r = sqrt(x * x + y * y + z * z);
  double const lo = r * (1.0 - 6.103515625e-05) - 1e-18, hi = r * (1.0 + 6.103515625e-05) + 1e-18;   // 2^-14
  int64_t a = 0, b = n2;   // first sorted radius >= lo
  while (a < b) {
    int64_t const m = (a + b) >> 1;
    if (rad[m] < lo) a = m + 1;
    else b = m;
  }
  float4 const q = r1c[i];
  uint64_t const qx = tc::f2pack(q.x, q.x), qy = tc::f2pack(q.y, q.y), qz = tc::f2pack(q.z, q.z);
  for (int64_t k = a; k < n2 && rad[k] <= hi; ++k) {
    int const j = idx[k];
    float4 const pa = r2pairs[2 * (j >> 1)], pb = r2pairs[2 * (j >> 1) + 1];
    bool const odd = j & 1;
    float const ex = odd ? pa.y : pa.x, ey = odd ? pa.w : pa.z, ez = odd ? pb.y : pb.x;
    uint64_t const dx = tc::f2sub(qx, tc::f2pack(ex, ex));
    uint64_t const dy = tc::f2sub(qy, tc::f2pack(ey, ey));
    uint64_t const dz = tc::f2sub(qz, tc::f2pack(ez, ez));
    uint64_t const r2 = tc::f2fma(dx, dx, tc::f2fma(dy, dy, tc::f2mul(dz, dz)));
    float ra, rb;
    tc::f2unpack(r2, ra, rb);
    if (ra >= q.w) continue;
    bool const same = x == p2[j] && y == p2[n2 + j] && z == p2[2 * n2 + j];
    if (same) continue;
    int const c = atomicAdd(count, 1);
    if (c < cap) out[c] = make_int2(int(i), j);
  }
}

// Direct Fock build: T[i][c] += s g rho V[j][c] and VH[i] += g coul[j] for each listed pair, with
// g = 1/r12 and rho = sum_a psi1[i][a] psi2[j][a] in FP64.  s = 1, or for a symmetric contraction
// (T holds the blocks on and above each r1 tile's diagonal, the diagonal tile at half weight) the
// weight the tensor kernel gives the pair's block: 0 below the diagonal tile, 1/2 in it, 1 above.
// One warp per pair.
__global__ void kNearDirect(int count, const int2 * list, int64_t n1, const double * p1, int64_t n2, const double * p2, int R,
                            const double * psi1, const double * psi2, int ldpsi, int ncol, const double * V, int ldv, const double * coul,
                            double * T, int ldt, double * VH, int sym)
{
  int const lane = threadIdx.x & 31;
  for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < count; k += (gridDim.x * blockDim.x) >> 5) {
    int2 const pr = list[k];
    int64_t const i = pr.x, j = pr.y;
    double const dx = p1[i] - p2[j], dy = p1[n1 + i] - p2[n2 + j], dz = p1[2 * n1 + i] - p2[2 * n2 + j];
    double const g = 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
    double rho = 0;
    for (int a = lane; a < R; a += 32) rho += psi1[i * ldpsi + a] * psi2[j * ldpsi + a];
    for (int o = 16; o > 0; o >>= 1) rho += __shfl_xor_sync(0xffffffffu, rho, o);
    if (lane == 0 && coul && VH) atomicAdd(&VH[i], g * coul[j]);
    double s = 1.0;
    if (sym) {
      int64_t const jd = (i / tc::BM) * (tc::BM / tc::BK), jb = j / tc::BK;   // the tile's diagonal block, the pair's block
      s = jb < jd ? 0.0 : (jb < jd + tc::BM / tc::BK ? 0.5 : 1.0);
    }
    if (s != 0.0)
      for (int c = lane; c < ncol; c += 32) atomicAdd(&T[i * ldt + c], s * g * rho * V[j * ldv + c]);
  }
}

// Precompute form: T[i][c] += g(r1_i, r2_j) V[j][c] for each listed pair, g the FP64 value of the kernel
// (kind 0: 1/r12; 1: 2/r12 - 2 u'^2; 2: component comp of u'(r12) (r1 - r2)/r12) for a Jastrow factor
// of r12 alone with u'(r12) = a12 / (r12 + a12)^2 sum_k i_k c_k (r12 / (r12 + a12))^(i_k - 1).
__global__ void kNearPairs(int count, const int2 * list, int64_t n1, const double * p1, int64_t n2, const double * p2, int kind, int comp,
                           int nterms, const int * powers, const double * coef, double a12, int ncol, const double * V, int ldv, double * T,
                           int ldt)
{
  int const lane = threadIdx.x & 31;
  for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < count; k += (gridDim.x * blockDim.x) >> 5) {
    int2 const pr = list[k];
    int64_t const i = pr.x, j = pr.y;
    double const d[3] = {p1[i] - p2[j], p1[n1 + i] - p2[n2 + j], p1[2 * n1 + i] - p2[2 * n2 + j]};
    double const r12 = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double g = 1.0 / r12;
    if (kind != 0) {
      double const t = 1.0 / (r12 + a12), z = r12 * t;
      double up = 0;
      for (int m = 0; m < nterms; ++m) {
        int const e = powers[m];
        if (e < 1) continue;
        double zp = 1;
        for (int q = 1; q < e; ++q) zp *= z;
        up += e * coef[m] * zp;
      }
      up *= a12 * t * t;
      g = kind == 1 ? 2.0 / r12 - 2.0 * up * up : up / r12 * d[comp];
    }
    for (int c = lane; c < ncol; c += 32) atomicAdd(&T[i * ldt + c], g * V[j * ldv + c]);
  }
}

}  // namespace

int nearPairsFor(tcscf_ctx * ctx, Grid const & g1, Grid const & g2, NearList const ** out)
{
  auto const key = std::make_pair(static_cast<const void *>(&g1), static_cast<const void *>(&g2));
  auto it = ctx->nearPairs.find(key);
  if (it != ctx->nearPairs.end()) {
    *out = &it->second;
    return TCSCF_OK;
  }
  TCSCF_CHECK(ctx, g2.n < (int64_t(1) << 31) && g1.n < (int64_t(1) << 31), TCSCF_ERR_UNSUPPORTED, "near-pair search: grid too large");
  int64_t const n1pad = (g1.n + 127) / 128 * 128, n2pad = (g2.n + 63) / 64 * 64;
  int const n2 = int(g2.n);
  size_t sortBytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, sortBytes, static_cast<const double *>(nullptr), static_cast<double *>(nullptr),
                                  static_cast<const int *>(nullptr), static_cast<int *>(nullptr), n2, 0, 64, ctx->stream);
  constexpr int kCap = 1 << 16;
  auto al = [](size_t n) { return (n + 255) & ~size_t(255); };
  size_t const bytes = al(sizeof(float4) * n1pad) + al(sizeof(float4) * n2pad) + 2 * al(sizeof(double) * n2) + 2 * al(sizeof(int) * n2) +
                       al(sortBytes) + al(sizeof(int2) * kCap) + al(sizeof(int)) + 256;
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, "near_find", bytes, &p));
  char * q = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(p) + 255) & ~uintptr_t(255));
  auto take = [&](size_t n) { char * r = q; q += al(n); return r; };
  auto * r1c = reinterpret_cast<float4 *>(take(sizeof(float4) * n1pad));
  auto * r2c = reinterpret_cast<float4 *>(take(sizeof(float4) * n2pad));
  auto * radIn = reinterpret_cast<double *>(take(sizeof(double) * n2));
  auto * radOut = reinterpret_cast<double *>(take(sizeof(double) * n2));
  auto * idxIn = reinterpret_cast<int *>(take(sizeof(int) * n2));
  auto * idxOut = reinterpret_cast<int *>(take(sizeof(int) * n2));
  void * sortTmp = take(sortBytes);
  auto * cand = reinterpret_cast<int2 *>(take(sizeof(int2) * kCap));
  int * dCount = reinterpret_cast<int *>(take(sizeof(int)));
  TCSCF_TRY(packPointsFp32(ctx, g1.n, n1pad, g1.pts, r1c));
  TCSCF_TRY(packPointPairsFp32(ctx, g2.n, n2pad, g2.pts, nullptr, r2c));
  kRadii<<<gridBlocks(n2, 256), 256, 0, ctx->stream>>>(n2, g2.pts, radIn, idxIn);
  TCSCF_LAUNCH(ctx);
  TCSCF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(sortTmp, sortBytes, radIn, radOut, idxIn, idxOut, n2, 0, 64, ctx->stream));
  NearList nl;
  int cap = kCap;
  int2 * list = cand;
  for (int attempt = 0; attempt < 2; ++attempt) {
    TCSCF_CUDA(ctx, cudaMemsetAsync(dCount, 0, sizeof(int), ctx->stream));
    unsigned const blocks = unsigned((g1.n + kFindThreads - 1) / kFindThreads);
    kFindNearPairs<<<blocks, kFindThreads, 0, ctx->stream>>>(g1.n, r1c, n2, r2c, radOut, idxOut, g1.pts, g2.pts, list, cap, dCount);
    TCSCF_LAUNCH(ctx);
    int count = 0;
    TCSCF_CUDA(ctx, cudaMemcpyAsync(&count, dCount, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (count <= cap) {
      if (count > 0) {   // the grid pair keeps its own copy of the list
        TCSCF_CUDA(ctx, cudaMalloc(&nl.d, sizeof(int2) * size_t(count)));
        TCSCF_CUDA(ctx, cudaMemcpyAsync(nl.d, list, sizeof(int2) * size_t(count), cudaMemcpyDeviceToDevice, ctx->stream));
        TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      }
      nl.count = count;
      if (list != cand) cudaFree(list);
      break;
    }
    TCSCF_CHECK(ctx, attempt == 0, TCSCF_ERR_CUDA, "near-pair search: count changed between passes");
    cap = count;
    TCSCF_CUDA(ctx, cudaMalloc(&list, sizeof(int2) * size_t(cap)));
  }
  auto res = ctx->nearPairs.emplace(key, nl);
  *out = &res.first->second;
  return TCSCF_OK;
}

void nearPairsForget(tcscf_ctx * ctx, Grid const * g)
{
  for (auto it = ctx->nearPairs.begin(); it != ctx->nearPairs.end();) {
    if (it->first.first == g || it->first.second == g) {
      if (it->second.d) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(it->second.d);
      }
      it = ctx->nearPairs.erase(it);
    } else {
      ++it;
    }
  }
}

int nearCorrect(tcscf_ctx * ctx, Contraction const & c)
{
  if (!c.near || c.near->count == 0) return TCSCF_OK;
  int const count = c.near->count;
  unsigned const blocks = gridBlocks(int64_t(count) * 32, 256);
  if (c.R > 0) {
    kNearDirect<<<blocks, 256, 0, ctx->stream>>>(count, c.near->d, c.n1, c.p1, c.n2, c.p2, c.R, c.psi1, c.psi2, c.ldpsi, c.ncol, c.V, c.ldv,
                                                 c.coul, c.T, c.ldt, c.VH, c.sym);
    TCSCF_LAUNCH(ctx);
    return TCSCF_OK;
  }
  int const kind = c.kernel == TCSCF_K_INV_R12 ? 0 : (c.kernel <= TCSCF_K_TC_SCALAR_OPPO ? 1 : 2);
  int const same = (c.kernel == TCSCF_K_TC_SCALAR_SAME || c.kernel == TCSCF_K_GRAD_U_SAME) ? 1 : 0;
  // Jastrow powers and coefficients of this spin kind in a small scratch array
  void * q = nullptr;
  TCSCF_TRY(scratch(ctx, "near_jastrow", sizeof(int) * 8 + sizeof(double) * 8, &q));
  int nterms = 0;
  double a12 = 1.0;
  if (kind != 0) {
    int pw[8] = {};
    double cf[8] = {};
    nterms = c.jastrow->nterms;
    for (int k = 0; k < nterms; ++k) { pw[k] = c.jastrow->S[k][0]; cf[k] = c.jastrow->c[k][same]; }
    a12 = c.jastrow->a12;
    TCSCF_CUDA(ctx, cudaMemcpyAsync(q, pw, sizeof(pw), cudaMemcpyHostToDevice, ctx->stream));
    TCSCF_CUDA(ctx, cudaMemcpyAsync(static_cast<char *>(q) + sizeof(pw), cf, sizeof(cf), cudaMemcpyHostToDevice, ctx->stream));
    TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  kNearPairs<<<blocks, 256, 0, ctx->stream>>>(count, c.near->d, c.n1, c.p1, c.n2, c.p2, kind, c.component, nterms, static_cast<const int *>(q),
                                              reinterpret_cast<const double *>(static_cast<char *>(q) + sizeof(int) * 8), a12, c.ncol, c.V, c.ldv,
                                              c.T, c.ldt);
  TCSCF_LAUNCH(ctx);
  return TCSCF_OK;
}

}  // namespace tcscf
