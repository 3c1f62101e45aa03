// FP64 CUDA-core r12 contractions and Fock-matrix reductions.
//
// The r12 contraction is written flash-style: for a tile of r1 points the kernel streams r2 in
// blocks, generates g(r1,r2) from the point coordinates (never stored), forms the density-matrix
// kernel rho(r1,r2) from the occupied-orbital factors, and accumulates  T += (g .* rho) V  in
// registers.  This reassociates the reference's stored-kernel contraction
//   Fai(r1,i) = sum_j (sum_k D(k,j) phi_k(r1)) Fji(r1,j,i),  Fji = computeF(1/r12)
// (HartreeFock.cpp:144-179, HartreeFock.hpp:136-180) into
//   Fai(r1,i) = sum_r2 g(r1,r2) w2 rho(r1,r2) phi_i(r2),  rho(r1,r2) = sum_kj D(k,j) phi_k(r1) phi_j(r2)^*
// and computes the Coulomb potential Faa(r1) (calculateIaa, HartreeFock.cpp:183-213) in the same
// pass.  With R == 0 (rho == 1) and V = weighted basis-pair products the same kernel is the FP64
// precompute form computeF / computeV.
#include "kernels.cuh"

namespace tcscf {
namespace {

constexpr int BK = 32;    // r2 points per block step
constexpr int BN = 128;   // columns per block
constexpr int NT = 256;

struct KArgs {
  int64_t n1, n2, r2PerSplit;
  int R, ncol, ldpsi, ldv, ldt, component, same;
  const double * p1;
  const double * p2;
  const double * psi1;
  const double * psi2;
  const double * coul;
  const double * V;
  double * T;
  double * VH;
  int64_t tStrideSplit;   // elements between split partials of T (0 when not split)
  int64_t vhStrideSplit;
  int sym;                // r1 = r2 points and psi1 = psi2: only r2 >= the block's first row, its own rows at half weight
  OchiDev u;
};

__device__ __forceinline__ double ipow(double x, int k)
{
  double r = 1;
  for (int i = 0; i < k; ++i) r *= x;
  return r;
}

// jastrowFunctions.hpp:72-108 (Ochi::gradient) for points p (first argument) and q.
__device__ __forceinline__ void ochiGrad(OchiDev const & u, double px, double py, double pz, double qx, double qy, double qz,
                                         int same, double & gx, double & gy, double & gz)
{
  double const dx = px - qx, dy = py - qy, dz = pz - qz;
  double const r1 = sqrt(px * px + py * py + pz * pz);
  double const r2 = sqrt(qx * qx + qy * qy + qz * qz);
  double const r12 = sqrt(dx * dx + dy * dy + dz * dz);
  double const r1T = r1 / (r1 + u.a), r2T = r2 / (r2 + u.a), r12T = r12 / (r12 + u.a12);
  double const r1Scale = u.a / (r1 * r1 * (r1 + u.a));
  double const r12Scale = u.a12 / (r12 * r12 * (r12 + u.a12));
  double r1L = 0, r12L = 0;
  for (int k = 0; k < u.nterms; ++k) {
    int const i = u.S[k][0], j = u.S[k][1], kk = u.S[k][2];
    double const f = u.c[k][same] * ipow(r12T, i) * ipow(r1T, j) * ipow(r2T, kk);
    r1L += f * j * r1Scale;
    r12L += f * i * r12Scale;
  }
  gx = r12L * dx + r1L * px;
  gy = r12L * dy + r1L * py;
  gz = r12L * dz + r1L * pz;
}

// g(r1, r2): KIND 0 = 1/r12, 1 = TC scalar, 2 = one component of grad_1 u.  0 for r1 == r2.
template <int KIND>
__device__ __forceinline__ double r12Kernel(KArgs const & a, double x1, double y1, double z1, double x2, double y2, double z2)
{
  double const dx = x1 - x2, dy = y1 - y2, dz = z1 - z2;
  double const rr = fma(dx, dx, fma(dy, dy, dz * dz));
  if (rr == 0.0) return 0.0;
  if (KIND == 0) return rsqrt_fp64(rr);
  if (KIND == 1) {
    double ax, ay, az, bx, by, bz;
    ochiGrad(a.u, x1, y1, z1, x2, y2, z2, a.same, ax, ay, az);
    ochiGrad(a.u, x2, y2, z2, x1, y1, z1, a.same, bx, by, bz);
    return 2.0 / sqrt(rr) - (ax * ax + ay * ay + az * az) - (bx * bx + by * by + bz * bz);
  }
  double gx, gy, gz;
  ochiGrad(a.u, x1, y1, z1, x2, y2, z2, a.same, gx, gy, gz);
  return a.component == 0 ? gx : (a.component == 1 ? gy : gz);
}

__device__ __forceinline__ void cpAsync8(double * dst, const double * src, bool valid)
{
  unsigned const d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  int const n = valid ? 8 : 0;   // src-size 0 zero-fills the destination
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cpAsyncWait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Block: BMT = 16 RPT r1 rows x BN columns, 256 threads.  r2 streamed in BK blocks through a
// two-stage cp.async pipeline (coordinates, Coulomb source, psi2 and V of block i+1 load while block i
// computes).  Phase B: each thread generates VPT kernel values g(r1,r2) (and rho) of one row;
// phase C: register-tiled FP64 GEMM, each thread RPT rows x BN/16 columns, columns interleaved in
// pairs so that a half-warp reads 16 consecutive 16-byte chunks (conflict-free).  RPT = 8 (an 8 x 8
// register tile: 16 shared-memory doubles per 64 FMAs) keeps the FP64 pipe ahead of shared-memory
// bandwidth where RPT = 4 (12 per 32) does not; it holds one block per SM.
template <int KIND, int BN, int RPT>
__global__ void __launch_bounds__(NT, RPT == 8 ? 1 : 2) kContractFp64(KArgs a)
{
  constexpr int CPT = BN / 16;            // columns per thread
  constexpr int BMT = 16 * RPT;           // r1 rows per block
  // the 128 x 128 tile's GEMM on the FP64 tensor cores (mma.m8n8k4): its operands come from registers,
  // so shared memory stops limiting the FP64 rate as it does the 8 x 8 register tile on the CUDA cores
  constexpr bool kDmma = BN == 128;
  // row strides of the X and V tiles: the DMMA fragments read 4 rows (k) x 8 consecutive doubles per
  // warp, which a stride of 8 (mod 16) doubles spreads over all 32 banks (two wavefronts, the minimum)
  constexpr int XLD = kDmma ? BMT + 8 : BMT;
  constexpr int VLD = kDmma ? BN + 8 : BN;
  constexpr int VPT = BMT * BK / NT;      // phase-B values per thread
  constexpr int TPR = BK / VPT;           // phase-B threads per row
  extern __shared__ __align__(16) double sm[];
  int const R = a.R;
  double * sP1 = sm;                              // [R][BMT]
  double * sC1 = sP1 + R * BMT;                   // [3][BMT]
  double * sX = sC1 + 3 * BMT;                    // [BK][XLD]
  double * stage0 = sX + BK * XLD;                // per stage: sV [BK][VLD], sC2 [4][BK], sP2 [R][BK]
  int const stageSize = BK * VLD + 4 * BK + R * BK;

  int const tid = threadIdx.x;
  int64_t const r1base = int64_t(blockIdx.x) * BMT;
  int const cg = blockIdx.z;
  // a symmetric contraction takes the r2 points from this block's own rows on (its own BMT x BMT
  // square at half weight in T); the Coulomb sums over the points before them come from kCoulombLowerFp64
  int64_t const r2split = int64_t(blockIdx.y) * a.r2PerSplit;
  int64_t const r2begin = a.sym ? max(r2split, r1base) : r2split;
  int64_t const r2end = min(a.n2, r2split + a.r2PerSplit);
  int64_t const r2half = a.sym ? r1base + BMT : 0;   // r2 below this (and >= r2begin) at half weight
  bool const doCoul = a.coul != nullptr && cg == 0;

  auto issue = [&](int64_t k0, int st) {
    double * sV = stage0 + st * stageSize;
    double * sC2 = sV + BK * VLD;
    double * sP2 = sC2 + 4 * BK;
    int const kn = int(min(int64_t(BK), r2end - k0));
    for (int idx = tid; idx < BK * BN; idx += NT) {
      int const k = idx / BN, c = idx % BN;
      int const col = cg * BN + c;
      bool const ok = k < kn && col < a.ncol;
      cpAsync8(&sV[k * VLD + c], ok ? &a.V[(k0 + k) * a.ldv + col] : a.V, ok);
    }
    for (int idx = tid; idx < R * BK; idx += NT) {
      int const k = idx / R, b = idx % R;
      bool const ok = k < kn;
      cpAsync8(&sP2[b * BK + k], ok ? &a.psi2[(k0 + k) * a.ldpsi + b] : a.psi2, ok);
    }
    if (tid < 4 * BK) {
      int const d = tid / BK, k = tid % BK;
      bool const ok = k < kn && (d < 3 || doCoul);
      const double * src = d < 3 ? &a.p2[d * a.n2 + k0 + k] : (doCoul ? &a.coul[k0 + k] : a.p2);
      cpAsync8(&sC2[d * BK + k], ok ? src : a.p2, ok);
    }
  };

  int64_t const nsteps = r2end > r2begin ? (r2end - r2begin + BK - 1) / BK : 0;
  if (nsteps > 0) issue(r2begin, 0);
  cpAsyncCommit();

  for (int idx = tid; idx < R * BMT; idx += NT) {
    int const r = idx / R, b = idx % R;
    int64_t const g = r1base + r;
    sP1[b * BMT + r] = g < a.n1 ? a.psi1[g * a.ldpsi + b] : 0.0;
  }
  for (int idx = tid; idx < 3 * BMT; idx += NT) {
    int const d = idx / BMT, r = idx % BMT;
    int64_t const g = r1base + r;
    sC1[idx] = g < a.n1 ? a.p1[d * a.n1 + g] : 1.0e6;
  }
  __syncthreads();

  int const rB = tid / TPR;             // phase-B row
  int const cB = (tid % TPR) * VPT;     // phase-B first column
  double const x1 = sC1[rB], y1 = sC1[BMT + rB], z1 = sC1[2 * BMT + rB];
  int const tr = tid >> 4, tc = tid & 15;
  double acc[RPT][CPT];
#pragma unroll
  for (int i = 0; i < RPT; ++i)
#pragma unroll
    for (int j = 0; j < CPT; ++j) acc[i][j] = 0.0;
  double vh = 0.0;

  for (int64_t step = 0; step < nsteps; ++step) {
    int64_t const k0 = r2begin + step * BK;
    int const st = int(step & 1);
    __syncthreads();   // every thread is done with the stage the next issue overwrites
    if (step + 1 < nsteps) issue(k0 + BK, st ^ 1);
    cpAsyncCommit();
    cpAsyncWait1();
    __syncthreads();
    double const * sV = stage0 + st * stageSize;
    double const * sC2 = sV + BK * VLD;
    double const * sP2 = sC2 + 4 * BK;
    int const kn = int(min(int64_t(BK), r2end - k0));
    double rho[VPT];
#pragma unroll
    for (int j = 0; j < VPT; ++j) rho[j] = R > 0 ? 0.0 : 1.0;
    for (int b = 0; b < R; ++b) {
      // one psi1 value against VPT psi2 values
      double const p = sP1[b * BMT + rB];
#pragma unroll
      for (int j = 0; j < VPT; j += 2) {
        double2 const q = *reinterpret_cast<double2 const *>(&sP2[b * BK + cB + j]);
        rho[j] = fma(p, q.x, rho[j]);
        rho[j + 1] = fma(p, q.y, rho[j + 1]);
      }
    }
#pragma unroll
    for (int j = 0; j < VPT; ++j) {
      int const c = cB + j;
      double g = r12Kernel<KIND>(a, x1, y1, z1, sC2[c], sC2[BK + c], sC2[2 * BK + c]);
      g = c < kn ? g : 0.0;
      vh = fma(g, sC2[3 * BK + c], vh);
      sX[c * XLD + rB] = (k0 + c < r2half ? 0.5 * g : g) * rho[j];
    }
    __syncthreads();
    if constexpr (kDmma) {
      // FP64 tensor cores: warp w owns rows BMT/2 (w & 1) .. + BMT/2 and columns 32 (w >> 1) .. + 32 of
      // the block as RPT x 4 tiles of 8 x 8; mma.m8n8k4 fragments: A[r][k] at lane 4 r + k, B[k][n] at
      // lane 4 n + k, C[r][2 q + e] at lane 4 r + q (element e)
      int const lane = tid & 31, wr = ((tid >> 5) & 1) * (BMT / 2), wc = (tid >> 6) * 32;
      int const fr = lane >> 2, fk = lane & 3;
#pragma unroll 2
      for (int k = 0; k < BK; k += 4) {
        double av[RPT], bv[4];
#pragma unroll
        for (int i = 0; i < RPT; ++i) av[i] = sX[(k + fk) * XLD + wr + 8 * i + fr];
#pragma unroll
        for (int j = 0; j < 4; ++j) bv[j] = sV[(k + fk) * VLD + wc + 8 * j + fr];
#pragma unroll
        for (int i = 0; i < RPT; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                         : "+d"(acc[i][2 * j]), "+d"(acc[i][2 * j + 1])
                         : "d"(av[i]), "d"(bv[j]));
      }
      continue;
    }
#pragma unroll 4
    for (int k = 0; k < BK; ++k) {
      double av[RPT];
#pragma unroll
      for (int q = 0; q < RPT / 2; ++q) {
        double2 const aa = *reinterpret_cast<double2 const *>(&sX[k * XLD + tr * RPT + 2 * q]);
        av[2 * q] = aa.x;
        av[2 * q + 1] = aa.y;
      }
      double bv[CPT];
#pragma unroll
      for (int q = 0; q < CPT / 2; ++q) {
        double2 const bb = *reinterpret_cast<double2 const *>(&sV[k * VLD + 32 * q + 2 * tc]);
        bv[2 * q] = bb.x;
        bv[2 * q + 1] = bb.y;
      }
#pragma unroll
      for (int i = 0; i < RPT; ++i)
#pragma unroll
        for (int j = 0; j < CPT; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
    }
  }

  double * T = a.T + blockIdx.y * a.tStrideSplit;
  if constexpr (kDmma) {
    int const lane = tid & 31, wr = ((tid >> 5) & 1) * (BMT / 2), wc = (tid >> 6) * 32;
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
      int64_t const g = r1base + wr + 8 * i + (lane >> 2);
      if (g >= a.n1) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          int const col = cg * BN + wc + 8 * j + 2 * (lane & 3) + e;
          if (col < a.ncol) T[g * a.ldt + col] = acc[i][2 * j + e];
        }
    }
  } else {
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
      int64_t const g = r1base + tr * RPT + i;
      if (g >= a.n1) continue;
#pragma unroll
      for (int j = 0; j < CPT; ++j) {
        int const col = cg * BN + 32 * (j / 2) + 2 * tc + (j & 1);
        if (col < a.ncol) T[g * a.ldt + col] = acc[i][j];
      }
    }
  }
  if (doCoul) {
#pragma unroll
    for (int o = 1; o < TPR; o <<= 1) vh += __shfl_xor_sync(0xffffffffu, vh, o);
    int64_t const g = r1base + rB;
    if ((tid % TPR) == 0 && g < a.n1) a.VH[blockIdx.y * a.vhStrideSplit + g] = vh;
  }
}

// Symmetric contractions: the Coulomb row sums over the r2 points before each block's first row (the
// pairs kContractFp64 skips), added to the potential: VH[r] += sum_{j < bm floor(r / bm)} g(r, j) c(j),
// FP64 with the exact-coincidence rule and 64-term partial sums.  One block of 64 threads per 128 rows;
// each thread takes rows r and r + 64 (the same bm tile, or consecutive 64-row tiles when bm = 64, so
// every condition below is uniform over the block), and the r2 points pass through shared memory in
// 64-point chunks, the next chunk's load in flight while the current one is summed.
__global__ void __launch_bounds__(64) kCoulombLowerFp64(int64_t n, int bm, const double * __restrict__ p, const double * __restrict__ coul,
                                                       double * VH)
{
  __shared__ double4 sq[2][64];   // x, y, z, c
  int const t = threadIdx.x;
  int64_t const r0 = int64_t(blockIdx.x) * 128 + t, r1 = r0 + 64;
  int64_t const a0 = r0 < n ? r0 : n - 1, a1 = r1 < n ? r1 : n - 1;   // rows past n repeat the last one (not written)
  double const x0 = p[a0], y0 = p[n + a0], z0 = p[2 * n + a0];
  double const x1 = p[a1], y1 = p[n + a1], z1 = p[2 * n + a1];
  int64_t const end0 = (int64_t(blockIdx.x) * 128 / bm) * bm;   // the points before row r0's tile (a multiple of 64)
  int64_t const end1 = ((int64_t(blockIdx.x) * 128 + 64) / bm) * bm;
  // when row r1's tile starts past n, every r1 row is past n (not written): only row r0's points are read
  int64_t const nChunks = (end1 <= n ? end1 : end0) / 64;
  auto load = [&](int64_t k) { int64_t const j = k * 64 + t; return make_double4(p[j], p[n + j], p[2 * n + j], coul[j]); };
  if (nChunks > 0) sq[0][t] = load(0);
  __syncthreads();
  double vh0 = 0.0, vh1 = 0.0;
  for (int64_t k = 0; k < nChunks; ++k) {
    int const buf = int(k & 1);
    bool const more = k + 1 < nChunks;
    double4 const nxt = more ? load(k + 1) : make_double4(0, 0, 0, 0);
    bool const row0 = (k + 1) * 64 <= end0;
    double part0 = 0.0, part1 = 0.0;
#pragma unroll 4
    for (int e = 0; e < 64; ++e) {
      double4 const q = sq[buf][e];
      double dx = x1 - q.x, dy = y1 - q.y, dz = z1 - q.z;
      double d = fma(dx, dx, fma(dy, dy, dz * dz));
      if (d != 0.0) part1 = fma(rsqrt_fp64(d), q.w, part1);
      if (row0) {
        dx = x0 - q.x; dy = y0 - q.y; dz = z0 - q.z;
        d = fma(dx, dx, fma(dy, dy, dz * dz));
        if (d != 0.0) part0 = fma(rsqrt_fp64(d), q.w, part0);
      }
    }
    vh0 += part0;
    vh1 += part1;
    if (more) sq[buf ^ 1][t] = nxt;   // chunk k - 1's buffer: every thread finished it before the last barrier
    __syncthreads();
  }
  if (r0 < n) VH[r0] += vh0;
  if (r1 < n) VH[r1] += vh1;
}

// deterministic sum of split partials: out[i] = sum_s part[s*stride + i]
__global__ void kSumSplits(int64_t n, int nsplit, int64_t stride, const double * part, double * out, int64_t rows, int cols, int ldOut, int ldPart)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    int64_t const r = i / cols;
    int const c = int(i % cols);
    double s = 0.0;
    for (int k = 0; k < nsplit; ++k) s += part[k * stride + r * ldPart + c];
    out[r * ldOut + c] = s;
  }
  (void)rows;
}

// ---- real Fock reduction:  out[k][l] = sum_r w[r] phi[r][k] (cJ phi[r][l] VH[r] - sgnT T[r][l]) ----
constexpr int RB = 16;      // rows per step
constexpr int RCH = 1024;   // rows per block (complex reduction; the real one sizes its row chunks per call)

// one block: `rch` rows (a multiple of RB) into a W x W tile of out (W = 64 or 128; 16 x 16 threads, TT x TT each)
template <int W>
__global__ void __launch_bounds__(NT) kReduceReal(int64_t n1, int nb, int rch, const double * phi, const double * w, const double * VH,
                                                  double cJ, const double * T, int ldt, double sgnT, double * part)
{
  constexpr int TT = W / 16;
  __shared__ __align__(16) double sA[RB][W];
  __shared__ __align__(16) double sY[RB][W];
  int const tid = threadIdx.x;
  int const kg = blockIdx.y * W, lg = blockIdx.z * W;
  int64_t const rbeg = int64_t(blockIdx.x) * rch, rend = min(n1, rbeg + rch);
  int const tk = tid >> 4, tl = tid & 15;
  double acc[TT][TT];
#pragma unroll
  for (int i = 0; i < TT; ++i)
#pragma unroll
    for (int j = 0; j < TT; ++j) acc[i][j] = 0.0;
  for (int64_t r0 = rbeg; r0 < rend; r0 += RB) {
    __syncthreads();
    for (int idx = tid; idx < RB * W; idx += NT) {
      int const rr = idx / W, c = idx % W;
      int64_t const r = r0 + rr;
      double av = 0.0, yv = 0.0;
      if (r < rend) {
        int const k = kg + c, l = lg + c;
        if (k < nb) av = w[r] * phi[r * nb + k];
        if (l < nb) {
          double y = 0.0;
          if (VH) y = cJ * phi[r * nb + l] * VH[r];
          if (T) y -= sgnT * T[r * ldt + l];
          yv = y;
        }
      }
      sA[rr][c] = av;
      sY[rr][c] = yv;
    }
    __syncthreads();
#pragma unroll 2
    for (int rr = 0; rr < RB; ++rr) {
      double av[TT], bv[TT];
#pragma unroll
      for (int q = 0; q < TT / 2; ++q) {
        double2 const x = *reinterpret_cast<double2 const *>(&sA[rr][tk * TT + 2 * q]);
        double2 const y = *reinterpret_cast<double2 const *>(&sY[rr][tl * TT + 2 * q]);
        av[2 * q] = x.x; av[2 * q + 1] = x.y;
        bv[2 * q] = y.x; bv[2 * q + 1] = y.y;
      }
#pragma unroll
      for (int i = 0; i < TT; ++i)
#pragma unroll
        for (int j = 0; j < TT; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
    }
  }
  double * out = part + int64_t(blockIdx.x) * nb * nb;
#pragma unroll
  for (int i = 0; i < TT; ++i) {
    int const k = kg + tk * TT + i;
    if (k >= nb) continue;
#pragma unroll
    for (int j = 0; j < TT; ++j) {
      int const l = lg + tl * TT + j;
      if (l < nb) out[k * nb + l] = acc[i][j];
    }
  }
}

__global__ void kSumChunks(int n, int nchunk, const double * part, double * out)
{
  int const i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int k = 0; k < nchunk; ++k) s += part[int64_t(k) * n + i];
  out[i] += s;
}

// ---- complex Fock reduction (precompute form): out(j,i) += sum_r w conj(A[r][j]) (cJ A[r][i] Faa[r] - Fai[r][i])
constexpr int CRB = 16;
__global__ void __launch_bounds__(NT) kReduceComplex(int64_t n1, int nb, const double2 * A, const double * w, const double2 * Faa,
                                                     double cJ, const double2 * Fai, double2 * part)
{
  extern __shared__ double2 csm[];
  double2 * sA = csm;              // [CRB][nb]
  double2 * sY = csm + CRB * nb;   // [CRB][nb]
  int const tid = threadIdx.x;
  int64_t const rbeg = int64_t(blockIdx.x) * RCH, rend = min(n1, rbeg + RCH);
  int const nn = nb * nb;
  int const per = (nn + NT - 1) / NT;
  double2 acc[16];
  for (int q = 0; q < 16; ++q) acc[q] = make_double2(0, 0);
  for (int64_t r0 = rbeg; r0 < rend; r0 += CRB) {
    __syncthreads();
    for (int idx = tid; idx < CRB * nb; idx += NT) {
      int const rr = idx / nb, c = idx % nb;
      int64_t const r = r0 + rr;
      double2 av = make_double2(0, 0), yv = make_double2(0, 0);
      if (r < rend) {
        double2 const x = A[r * nb + c];
        av = make_double2(w[r] * x.x, -w[r] * x.y);   // w conj(A)
        double2 const f = Faa[r];
        double2 const t = Fai[r * nb + c];
        yv.x = cJ * (x.x * f.x - x.y * f.y) - t.x;
        yv.y = cJ * (x.x * f.y + x.y * f.x) - t.y;
      }
      sA[idx] = av;
      sY[idx] = yv;
    }
    __syncthreads();
    for (int rr = 0; rr < CRB; ++rr)
      for (int q = 0; q < per && q < 16; ++q) {
        int const e = tid + q * NT;
        if (e >= nn) break;
        int const j = e / nb, i = e % nb;
        double2 const x = sA[rr * nb + j], y = sY[rr * nb + i];
        acc[q].x = fma(x.x, y.x, fma(-x.y, y.y, acc[q].x));
        acc[q].y = fma(x.x, y.y, fma(x.y, y.x, acc[q].y));
      }
  }
  double2 * out = part + int64_t(blockIdx.x) * nn;
  for (int q = 0; q < per && q < 16; ++q) {
    int const e = tid + q * NT;
    if (e < nn) out[e] = acc[q];
  }
}

template <int KIND, int BNV, int RPT>
int launchOne(tcscf_ctx * ctx, KArgs const & a, dim3 grid, size_t smem)
{
  TCSCF_CUDA(ctx, cudaFuncSetAttribute(kContractFp64<KIND, BNV, RPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  TCSCF_CUDA(ctx, cudaFuncSetAttribute(kContractFp64<KIND, BNV, RPT>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  kContractFp64<KIND, BNV, RPT><<<grid, NT, smem, ctx->stream>>>(a);
  TCSCF_LAUNCH(ctx);
  return TCSCF_OK;
}

template <int KIND>
int launchKind(tcscf_ctx * ctx, int bn, int rpt, KArgs const & a, dim3 grid, size_t smem)
{
  if (bn == 32) return launchOne<KIND, 32, 4>(ctx, a, grid, smem);
  if (bn == 64) return launchOne<KIND, 64, 4>(ctx, a, grid, smem);
  if constexpr (KIND == 0)
    if (rpt == 8) return launchOne<KIND, 128, 8>(ctx, a, grid, smem);
  return launchOne<KIND, 128, 4>(ctx, a, grid, smem);
}

int launchContract(tcscf_ctx * ctx, int kind, int bn, int rpt, KArgs const & a, unsigned tiles, unsigned nsplit, size_t smem)
{
  unsigned const cgroups = a.ncol <= 128 ? 1u : unsigned((a.ncol + BN - 1) / BN);
  dim3 const grid{tiles, nsplit, cgroups};
  if (kind == 0) return launchKind<0>(ctx, bn, rpt, a, grid, smem);
  if (kind == 1) return launchKind<1>(ctx, bn, rpt, a, grid, smem);
  return launchKind<2>(ctx, bn, rpt, a, grid, smem);
}

}  // namespace

int contractFp64(tcscf_ctx * ctx, Contraction const & c)
{
  TCSCF_CHECK(ctx, c.R >= 0 && c.R <= 128, TCSCF_ERR_UNSUPPORTED, "contraction rank must be <= 128");
  TCSCF_CHECK(ctx, c.ncol > 0 && c.n1 > 0 && c.n2 > 0, TCSCF_ERR_INVALID_ARGUMENT, "empty contraction");
  int const bn = c.ncol <= 32 ? 32 : (c.ncol <= 64 ? 64 : 128);
  int const kind = c.kernel == TCSCF_K_INV_R12 ? 0 : (c.kernel <= TCSCF_K_TC_SCALAR_OPPO ? 1 : 2);
  // 8 x 8 register tiles (128 r1 rows per block) for 1/r12 where the 128-column tile and the rank
  // leave the shared memory room (R <= 64), else 4 x 8 (64 rows).  The transcorrelated kernels spend
  // more of each block generating g, which the one block per SM of the 8 x 8 tile cannot hide: at Be-TC
  // (24 STO, 65,536 x 65,536 points) their precompute took 4.37 s with 8 x 8 and 2.68 s with 4 x 8.
  int const rpt = bn == 128 && c.R <= 64 && kind == 0 ? 8 : 4;
  int const bm = 16 * rpt;
  int64_t const tiles = (c.n1 + bm - 1) / bm;
  int const cgroups = c.ncol <= 128 ? 1 : (c.ncol + BN - 1) / BN;
  int dev = 0;
  cudaGetDevice(&dev);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // split r2 so that small r1 sets still fill the machine (partials are summed deterministically)
  int64_t const want = int64_t(sms) * (rpt == 8 ? 2 : 4);
  int64_t nsplit = (want + tiles * cgroups - 1) / (tiles * cgroups);
  nsplit = std::max<int64_t>(1, std::min<int64_t>(nsplit, (c.n2 + 4 * BK - 1) / (4 * BK)));
  nsplit = std::min<int64_t>(nsplit, 65535);
  int64_t perSplit = (c.n2 + nsplit - 1) / nsplit;
  perSplit = ((perSplit + BK - 1) / BK) * BK;
  nsplit = (c.n2 + perSplit - 1) / perSplit;

  KArgs a{};
  a.n1 = c.n1; a.n2 = c.n2; a.r2PerSplit = perSplit;
  a.R = c.R; a.ncol = c.ncol; a.ldpsi = c.ldpsi; a.ldv = c.ldv; a.ldt = c.ldt;
  a.component = c.component; a.same = (c.kernel == TCSCF_K_TC_SCALAR_SAME || c.kernel == TCSCF_K_GRAD_U_SAME) ? 1 : 0;
  a.p1 = c.p1; a.p2 = c.p2; a.psi1 = c.psi1; a.psi2 = c.psi2; a.coul = c.coul; a.V = c.V;
  if (c.jastrow) {
    a.u.a = c.jastrow->a; a.u.a12 = c.jastrow->a12; a.u.nterms = c.jastrow->nterms;
    for (int k = 0; k < 8; ++k) {
      for (int d = 0; d < 3; ++d) a.u.S[k][d] = c.jastrow->S[k][d];
      a.u.c[k][0] = c.jastrow->c[k][0]; a.u.c[k][1] = c.jastrow->c[k][1];
    }
  }
  double * Tpart = c.T;
  double * VHpart = c.VH;
  if (nsplit > 1) {
    void * p = nullptr;
    size_t const tb = size_t(nsplit) * c.n1 * c.ldt * sizeof(double);
    size_t const vb = c.coul ? size_t(nsplit) * c.n1 * sizeof(double) : 0;
    TCSCF_TRY(scratch(ctx, "contract_split", tb + vb, &p));
    Tpart = static_cast<double *>(p);
    VHpart = c.coul ? Tpart + size_t(nsplit) * c.n1 * c.ldt : nullptr;
    a.tStrideSplit = c.n1 * c.ldt;
    a.vhStrideSplit = c.n1;
  }
  a.T = Tpart;
  a.VH = VHpart;
  TCSCF_CHECK(ctx, !c.sym || (c.p1 == c.p2 && c.n1 == c.n2 && c.psi1 == c.psi2 && c.R > 0 && (c.VH != nullptr) == (c.coul != nullptr)),
              TCSCF_ERR_INVALID_ARGUMENT, "internal: a symmetric contraction needs r1 = r2 and psi1 = psi2");
  a.sym = c.sym ? 1 : 0;
  int const pad = bn == 128 ? 8 : 0;   // the DMMA tiles' padded X and V row strides
  size_t const smem = sizeof(double) * (size_t(c.R) * bm + 3 * bm + BK * (bm + pad) + 2 * (size_t(BK) * (bn + pad) + 4 * BK + size_t(c.R) * BK));
  // the contraction kernel alone is bracketed by the context's timing events (tcscf_last_timing)
  if (!ctx->capturing) cudaEventRecord(ctx->ev[2], ctx->stream);
  TCSCF_TRY(launchContract(ctx, kind, bn, rpt, a, unsigned(tiles), unsigned(nsplit), smem));
  if (!ctx->capturing) cudaEventRecord(ctx->ev[3], ctx->stream);
  if (nsplit > 1) {
    int64_t const n = c.n1 * c.ncol;
    kSumSplits<<<gridBlocks(n, 256), 256, 0, ctx->stream>>>(n, int(nsplit), c.n1 * c.ldt, Tpart, c.T, c.n1, c.ncol, c.ldt, c.ldt);
    TCSCF_LAUNCH(ctx);
    if (c.coul) {
      kSumSplits<<<gridBlocks(c.n1, 256), 256, 0, ctx->stream>>>(c.n1, int(nsplit), c.n1, VHpart, c.VH, c.n1, 1, 1, 1);
      TCSCF_LAUNCH(ctx);
    }
  }
  if (c.sym && c.coul && tiles > 1) {
    kCoulombLowerFp64<<<unsigned((c.n1 + 127) / 128), 64, 0, ctx->stream>>>(c.n1, bm, c.p1, c.coul, c.VH);
    TCSCF_LAUNCH(ctx);
  }
  return TCSCF_OK;
}

int sumSplitsLaunch(tcscf_ctx * ctx, int64_t n, int nsplit, int64_t stride, const double * part, double * out, int64_t rows, int cols,
                    int ldOut, int ldPart)
{
  kSumSplits<<<gridBlocks(n, 256), 256, 0, ctx->stream>>>(n, nsplit, stride, part, out, rows, cols, ldOut, ldPart);
  TCSCF_LAUNCH(ctx);
  return TCSCF_OK;
}

int reduceFockReal(tcscf_ctx * ctx, int64_t n1, int nb, const double * phi, const double * w1, const double * VH, double cJ,
                   const double * T, int ldt, double sgnT, double * out)
{
  // output tiles 64 wide (70 registers a thread: three blocks per SM, where the 128-wide tile's 168
  // allowed one, whose global-to-shared staging then stalled its FP64 FMAs); row chunks sized for about
  // two blocks per SM per output tile (16 to 1024 rows)
  int const W = 64;
  int const g = (nb + W - 1) / W;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  int64_t const want = (n1 + 2 * sms * g * g - 1) / (2 * sms * g * g);
  int const rch = int(std::min<int64_t>(1024, std::max<int64_t>(RB, (want + RB - 1) / RB * RB)));
  int64_t const chunks = (n1 + rch - 1) / rch;
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, "reduce_real", size_t(chunks) * nb * nb * sizeof(double), &p));
  double * part = static_cast<double *>(p);
  dim3 grid{unsigned(chunks), unsigned(g), unsigned(g)};
  if (W == 64) kReduceReal<64><<<grid, NT, 0, ctx->stream>>>(n1, nb, rch, phi, w1, VH, cJ, T, ldt, sgnT, part);
  else kReduceReal<128><<<grid, NT, 0, ctx->stream>>>(n1, nb, rch, phi, w1, VH, cJ, T, ldt, sgnT, part);
  TCSCF_LAUNCH(ctx);
  int const n = nb * nb;
  kSumChunks<<<(n + 255) / 256, 256, 0, ctx->stream>>>(n, int(chunks), part, out);
  TCSCF_LAUNCH(ctx);
  return TCSCF_OK;
}

int reduceFockComplex(tcscf_ctx * ctx, int64_t n1, int nb, const double * A, const double * w, const double * Faa, double cJ,
                      const double * Fai, double * out)
{
  TCSCF_CHECK(ctx, nb * nb <= 16 * NT, TCSCF_ERR_UNSUPPORTED, "precompute-form Fock reduction supports nb <= 64");
  int64_t const chunks = (n1 + RCH - 1) / RCH;
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, "reduce_complex", size_t(chunks) * nb * nb * 2 * sizeof(double), &p));
  size_t const smem = size_t(2) * CRB * nb * sizeof(double2);
  kReduceComplex<<<unsigned(chunks), NT, smem, ctx->stream>>>(n1, nb, reinterpret_cast<const double2 *>(A), w,
                                                              reinterpret_cast<const double2 *>(Faa), cJ,
                                                              reinterpret_cast<const double2 *>(Fai), static_cast<double2 *>(p));
  TCSCF_LAUNCH(ctx);
  int const n = 2 * nb * nb;
  kSumChunks<<<(n + 255) / 256, 256, 0, ctx->stream>>>(n, int(chunks), static_cast<double *>(p), out);
  TCSCF_LAUNCH(ctx);
  return TCSCF_OK;
}

}  // namespace tcscf
