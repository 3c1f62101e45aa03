// tcgen05 (sm_100a) r12 contraction for the direct Fock build in split-BF16 precision with exact
// tensor-core accumulation.
//
// For a tile of 128 r1 points (one TMEM lane each) the kernel streams r2 in blocks of 64:
//   GEMM1 (tensor):  rho(r1,r2) = psi1[r1][:] . psi2[r2][:]            K = 32 or 64 (padded rank)
//   CUDA cores:      g = 1/|r1 - r2| (FP32, Newton-refined), X = g * rho, VH(r1) += g * coul(r2)
//   GEMM2 (tensor):  T[r1][i] += X[r1][r2] . Vt[i][r2]                 Vt = (w2 phi_i(r2))^T, N = NB
//
// Fixed-point BF16 slices.  Each row of psi1 / psi2, each (r1, block) row of X and each (block, i)
// column of Vt carries a power-of-two scale s chosen from its largest entry.  The per-point factors
// psi1, psi2 and Vt (whose rounding is shared by every pair a point takes part in) keep 24 bits:
// u s in [2^23, 2^24) is written as 65536 h + 256 m + l with integers |h| <= 256, |m|, |l| <= 128
// (round to nearest, each exact in BF16); X keeps 24 bits like the factors (four slices) when the
// rank padding is 32, 16 bits (u s = 256 h + l) when it is 64 and shared memory has no room for more.  X's lowest slice l enters only B, so it is stored as
// the BF16 nearest to the remainder (8 significant bits) instead of an integer.  Per r2 block:
//   A = sum h h'                      (integers below 2^16 each, a K <= 64 sum below 2^23: exact)
//   B = sum h m' + m h' + (h l' + l h' + m m')/256   (the level 2^-8 below A; its own FP32 rounding
//                                                     is scaled down by 2^-8 in the result)
// and the product is 256 A + B in units of the block's scales (GEMM2 keeps h m', l h', h l'/256 of
// its 16-bit X).  The hi*hi accumulation being exact, the tensor core's FP32 adder rounding cannot
// bias the result; the products below 2^-24 of the largest term are dropped.  Each block's T is
// added with its scales, as soon as the block completes, into per-thread double-float accumulators
// (FP32 hi + lo updated by Fast2Sum; about 48 bits, no FP64 or conversion pipe work).
// The kernel matrix g exists only as the BF16 X tile in shared memory.
//
// Warp roles (384 threads, one CTA per SM, persistent over (r1 tile, r2 split) work items):
//   warp 0      TMA producer: psi1 tile (once per work item), psi2 / Vt blocks (TMA, no multicast),
//               r2 coordinates + Coulomb source, psi2 row scales and Vt column scales (1-D bulk copies)
//   warp 1      MMA issuer (one elected thread) and TMEM allocator
//   warps 2-3   idle (they complete warpgroup 0, whose registers setmaxnreg hands to the compute warps)
//   warps 4-11  compute: warp w owns TMEM lanes 32*(w%4).. (r1 rows), r2 / column half (w-4)/4
// Every mbarrier wait is bounded by a wall-clock limit; on expiry the kernel records the failure in
// a device status word, drains its own TMA / MMA work with bounded waits, frees TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <array>
#include <vector>

#include "tc_device.cuh"

namespace tcscf {
namespace tc {

// TMA stages (the default rule): three when the tile shapes leave room in shared memory; the autotuner
// may also try two for (NB 64, RP 32)
__host__ __device__ constexpr int stagesFor(int NB, int RP) { return NB == 64 && RP == 32 ? 3 : 2; }
// X precision: XS = 2 slices (16 bits, u s in [2^15, 2^16)) or XS = 3 (24 bits, stored as the four
// slices h, m, l/256, m/256); its tile buffers: two (GEMM2 of block g - 1 overlaps the writing of
// block g) where shared memory allows
__host__ __device__ constexpr int xSlicesFor(int XS) { return XS == 3 ? 4 : 2; }
__host__ __device__ constexpr int xBuffersFor(int NB, int RP, int XS) { return XS == 3 || (NB == 64 && RP == 64) ? 1 : 2; }
__host__ __device__ constexpr int xExpFor(int XS) { return XS == 3 ? 23 : 15; }
// slicing: scale = 2^(k - floor(log2 max|u|)) puts the largest entry in [2^k, 2^(k+1)): k = 23 for
// the three-slice factors, 15 for the two-slice X; entries of a row whose maximum is below
// 2^kMinExp are sliced against 2^kMinExp
constexpr int kFactorExp = 23;
constexpr int kMinExp = -100;

// TMEM columns: rho buffers b = 0, 1 at 128 b (hi*hi) and 128 b + 64 (cross); T at TCOL0 (hi*hi) and
// TCOL0 + NB (cross)
constexpr uint32_t TCOL0 = 256;

// RP: padded rank of rho (GEMM1 K): 32 (64-byte rows, 64B swizzle) or 64 (128-byte rows, 128B swizzle)
template <int NB, int RP, int XS, int NS>
struct __align__(1024) Smem {
  static constexpr int NSTAGE = NS;
  uint8_t v[NSTAGE][3][NB * BK * 2];       // Vt block h / m / l/256: SW128 K-major [NB rows][64]
  static constexpr int XBUF = xBuffersFor(NB, RP, XS);
  uint8_t x[XBUF][xSlicesFor(XS)][BM * BK * 2];   // X tile slices per buffer: SW128 K-major [128 rows][64]
  uint8_t psi2[NSTAGE][3][BK * RP * 2];    // psi2 block h / m / l/256: K-major [64 rows][RP]
  uint8_t psi1[4][BM * RP * 2];            // psi1 tile h / m / l/256 / m/256: K-major [128 rows][RP]
  float4 coords[NSTAGE][BK];               // r2 block as 32 pairs {x0,x1,y0,y1}{z0,z1,c0,c1}
  float a2inv[NSTAGE][BK];                 // 1 / (psi2 row scale) of the block's r2 points
  float cinv[NSTAGE][NB];                  // 1 / (Vt column scale) of the block
  float cinvT[NCW][2][NB / 2];             // each compute warp's copy of its columns' cinv, by block parity
  float rowmax[2][2][BM];                  // [block parity][r2 half][row] max |X'| of the half
  uint64_t full[NSTAGE], empty[NSTAGE];
  uint64_t sfull[2], sfree[2], xfull[2], xfree[2];   // xfull / xfree: per X buffer
  uint64_t rmax[2][4];                     // [block parity][lane quarter]: both r2 halves posted their maxima
  uint64_t tfull, tfree;
  uint64_t p1full, p1free, done;
  uint32_t tmemBase;
  int abort;
};

// instruction descriptor: kind::f16, A = B = BF16 (K-major), D = F32, shape M x N
__host__ __device__ constexpr uint32_t instrDescBf16(int M, int N)
{
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void mmaBf16(uint32_t tmemD, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmemD),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

// the BF16 pair {a, b} rounded to nearest
__device__ __forceinline__ uint32_t bf16PairRn(uint64_t ab)
{
  float a, b;
  f2unpack(ab, a, b);
  __nv_bfloat162 const h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t const *>(&h);
}

// the BF16 pair {a, b} of two FP32 values whose low 16 mantissa bits are zero (exact truncation)
__device__ __forceinline__ uint32_t bf16PairExact(uint64_t ab)
{
  float a, b;
  f2unpack(ab, a, b);
  return __byte_perm(__float_as_uint(a), __float_as_uint(b), 0x7632);
}

// Adds the finished block f (this thread's row, NB/2 columns of T) with the block's scales into the
// double-float accumulators (hi + lo per column, FP32 pairs of columns) by Fast2Sum,
// and hands the TMEM accumulators back to the MMA issuer.
template <int NB, class SmemT>
__device__ __forceinline__ bool flushBlock(SmemT & S, uint32_t taddr, uint32_t f, int cw, float fac, uint64_t (&hi)[NB / 4],
                                           uint64_t (&lo)[NB / 4], int lane, volatile int * abortFlag, int * status)
{
  if (!waitBar(&S.tfull, f & 1, abortFlag, status, 31)) return false;
  fenceAfterSync();
  float const * cs = S.cinvT[cw][f & 1];
  uint64_t const k256 = f2pack(256.0f, 256.0f);
  uint64_t const ff = f2pack(fac, fac);
  constexpr int NQ = NB / 16;   // chunks of 8 columns; the loads of chunk q + 1 overlap the work on chunk q
  float hh[2][8], mm[2][8];
  tmemLoad8(taddr, hh[0]);
  tmemLoad8(taddr + NB, mm[0]);
  tmemWaitLoad8(hh[0], mm[0]);
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    int const cur = q & 1;
    if (q + 1 < NQ) {
      tmemLoad8(taddr + (q + 1) * 8, hh[cur ^ 1]);
      tmemLoad8(taddr + NB + (q + 1) * 8, mm[cur ^ 1]);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      float2 const c2 = *reinterpret_cast<float2 const *>(cs + q * 8 + 2 * i);
      // 256 hh + cross is the block's exact integer sum up to one FP32 rounding; cinv and fac are powers
      // of two, so x is that sum in the units of T
      uint64_t const x = f2mul(f2fma(f2pack(hh[cur][2 * i], hh[cur][2 * i + 1]), k256, f2pack(mm[cur][2 * i], mm[cur][2 * i + 1])),
                               f2mul(f2pack(c2.x, c2.y), ff));
      int const p = q * 4 + i;
      // Fast2Sum: hi + x == sum + (x - (sum - hi)) exactly when |hi| >= |x|, which holds once a
      // row's sum has absorbed its first blocks; otherwise the compensation is approximate at the
      // level of the rounding of the smaller term
      uint64_t const sum = f2add(hi[p], x);
      lo[p] = f2add(lo[p], f2sub(x, f2sub(sum, hi[p])));
      hi[p] = sum;
    }
    if (q + 1 < NQ) tmemWaitLoad8(hh[cur ^ 1], mm[cur ^ 1]);
  }
  fenceBeforeSync();
  __syncwarp();
  if (lane == 0) mbarArrive(&S.tfree);
  return true;
}

// ---- the kernel ------------------------------------------------------------------------------------
template <int NB, int RP, int XS, int NS>
__global__ void __launch_bounds__(NTHREADS, 1)
    kFlashTc(Params P)
{
  extern __shared__ uint8_t smemRaw[];
  Smem<NB, RP, XS, NS> & S = *reinterpret_cast<Smem<NB, RP, XS, NS> *>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
  constexpr int NSTAGE = NS;
  constexpr int XBUF = xBuffersFor(NB, RP, XS);
  constexpr int XSL = xSlicesFor(XS);
  constexpr int kXExp = xExpFor(XS);
  int const warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  volatile int * abortFlag = &S.abort;

  static_assert(TCOL0 + 2 * NB <= 512, "TMEM columns");
  constexpr uint32_t kStageBytes = 3 * NB * BK * 2 + 3 * BK * RP * 2 + BK * sizeof(float4) + BK * sizeof(float) + NB * sizeof(float);
  constexpr uint32_t kPsi1Bytes = 4 * BM * RP * 2;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NSTAGE; ++s) { mbarInit(&S.full[s], 1); mbarInit(&S.empty[s], 1 + NCW); }
    for (int b = 0; b < 2; ++b) {
      mbarInit(&S.sfull[b], 1); mbarInit(&S.sfree[b], NCW);
      mbarInit(&S.xfull[b], NCW); mbarInit(&S.xfree[b], 1);
      for (int q = 0; q < 4; ++q) mbarInit(&S.rmax[b][q], 2);
    }
    mbarInit(&S.tfull, 1); mbarInit(&S.tfree, NCW);
    mbarInit(&S.p1full, 1); mbarInit(&S.p1free, 1); mbarInit(&S.done, 1);
    S.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smemAddr(&S.tmemBase)) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fenceBeforeSync();
  __syncthreads();
  fenceAfterSync();
  uint32_t const tmem = S.tmemBase;

  int const nItems = P.nItems;

  if (warp < 4) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kRegsProducer));
  if (warp == 0) {
    // ---------------------------------------------------------------- TMA producer
    if (lane == 0) {
      uint32_t issuedLoads = 0;
      uint32_t p1Use = 0;
      bool ok = true;
      for (int item = blockIdx.x; item < nItems && ok; item += gridDim.x) {
        int ii, tile, split;
        decodeItem(P, item, ii, tile, split);
        Instance const * I = P.inst + ii;
        CUtensorMap const * maps = I->maps;
        int jb, je;
        itemBlocks(*I, tile, split, jb, je);
        if (je == jb) continue;   // an empty item of a symmetric instance: the MMA issuer skips it too
        if (p1Use > 0 && !(ok = waitBar(&S.p1free, (p1Use - 1) & 1, abortFlag, P.status, 11))) break;
        mbarArriveTx(&S.p1full, kPsi1Bytes);
        for (int k = 0; k < 4; ++k) tmaLoad2d(S.psi1[k], maps + k, 0, tile * BM, &S.p1full);
        ++p1Use;
        for (int j = jb; j < je; ++j) {
          uint32_t const q = issuedLoads++;
          int const s = q % NSTAGE;
          // use u = q / NSTAGE of stage s needs consumption u - 1 of it
          if (q >= uint32_t(NSTAGE) && !(ok = waitBar(&S.empty[s], ((q / NSTAGE) - 1) & 1, abortFlag, P.status, 12))) break;
          mbarArriveTx(&S.full[s], kStageBytes);
          for (int k = 0; k < 3; ++k) tmaLoad2d(S.psi2[s][k], maps + 4 + k, 0, j * BK, &S.full[s]);
          for (int k = 0; k < 3; ++k) tmaLoad2d(S.v[s][k], maps + 7 + k, j * BK, 0, &S.full[s]);
          bulkLoad(S.coords[s], I->r2pairs + int64_t(j) * BK, BK * sizeof(float4), &S.full[s]);
          bulkLoad(S.a2inv[s], I->a2inv + int64_t(j) * BK, BK * sizeof(float), &S.full[s]);
          bulkLoad(S.cinv[s], I->cinv + int64_t(j) * NB, NB * sizeof(float), &S.full[s]);
        }
      }
      // drain: every issued load lands before the CTA can exit (bounded)
      for (uint32_t q = issuedLoads > uint32_t(NSTAGE) ? issuedLoads - NSTAGE : 0; q < issuedLoads; ++q) {
        unsigned long long const t0 = globalTimer();
        while (!mbarTryWait(&S.full[q % NSTAGE], (q / NSTAGE) & 1) && globalTimer() - t0 < kWaitLimitNs) {}
      }
      if (p1Use > 0) {
        unsigned long long const t0 = globalTimer();
        while (!mbarTryWait(&S.p1full, (p1Use - 1) & 1) && globalTimer() - t0 < kWaitLimitNs) {}
      }
    }
  } else if (warp == 1) {
    // ---------------------------------------------------------------- MMA issuer
    if (lane == 0) {
      constexpr uint32_t idesc1 = instrDescBf16(BM, BK);
      constexpr uint32_t idesc2 = instrDescBf16(BM, NB);
      // h x [h'; m'] in one MMA: the h and m slices of an operand are adjacent in shared memory (so
      // the B rows continue), and the two accumulators are adjacent in TMEM (A then B)
      constexpr uint32_t idesc1x2 = instrDescBf16(BM, 2 * BK);
      constexpr uint32_t idesc2x2 = instrDescBf16(BM, 2 * NB);
      uint32_t const aPsi1[4] = {smemAddr(S.psi1[0]), smemAddr(S.psi1[1]), smemAddr(S.psi1[2]), smemAddr(S.psi1[3])};
      uint32_t blockCount = 0;   // global block counter: selects stage, rho / X buffers, T phase
      uint32_t p1Use = 0;
      bool ok = true;
      for (int item = blockIdx.x; item < nItems && ok; item += gridDim.x) {
        int ii, tile, split;
        decodeItem(P, item, ii, tile, split);
        Instance const * I = P.inst + ii;
        int jb, je;
        itemBlocks(*I, tile, split, jb, je);
        int const nblk = je - jb;
        if (nblk == 0) continue;   // nothing loaded for an empty item
        if (!(ok = waitBar(&S.p1full, p1Use & 1, abortFlag, P.status, 21))) break;
        ++p1Use;
        fenceAfterSync();
        uint32_t const base = blockCount;
        auto gemm1 = [&](int jj) -> bool {
          uint32_t const g = base + jj;
          int const s = g % NSTAGE, b = g & 1;
          if (!waitBar(&S.full[s], (g / NSTAGE) & 1, abortFlag, P.status, 22)) return false;
          if (g >= 2 && !waitBar(&S.sfree[b], ((g >> 1) - 1) & 1, abortFlag, P.status, 23)) return false;
          fenceAfterSync();
          uint32_t const dHH = tmem + b * 2 * BK, dX = dHH + BK;
          uint32_t const bPsi2[3] = {smemAddr(S.psi2[s][0]), smemAddr(S.psi2[s][1]), smemAddr(S.psi2[s][2])};
          constexpr uint32_t sbo = RP == 64 ? 1024 : 512, swz = RP == 64 ? 2 : 4;
          auto da = [&](int sl, int k) { return smemDesc(aPsi1[sl] + 32 * k, sbo, swz); };
          auto db = [&](int sl, int k) { return smemDesc(bPsi2[sl] + 32 * k, sbo, swz); };
#pragma unroll
          for (int k = 0; k < RP / 16; ++k) {
            uint32_t const acc = k > 0 ? 1u : 0u;
            // B: h m' + m h' + h l'/256 + l/256 h' + m/256 m'; A: h h'
            mmaBf16(dHH, da(0, k), db(0, k), idesc1x2, acc);   // A += h h', B += h m'
            mmaBf16(dX, da(1, k), db(0, k), idesc1, 1);
            mmaBf16(dX, da(0, k), db(2, k), idesc1, 1);
            mmaBf16(dX, da(2, k), db(0, k), idesc1, 1);
            mmaBf16(dX, da(3, k), db(1, k), idesc1, 1);
          }
          mmaCommit(&S.sfull[b]);
          return true;
        };
        if (nblk > 0 && !(ok = gemm1(0))) break;
        for (int jj = 0; jj < nblk && ok; ++jj) {
          if (jj + 1 < nblk && !(ok = gemm1(jj + 1))) break;
          uint32_t const g = base + jj;
          int const s = g % NSTAGE;
          // the T accumulators are free once the compute warps flushed block g - 1
          if (g >= 1 && !(ok = waitBar(&S.tfree, (g - 1) & 1, abortFlag, P.status, 24))) break;
          int const xb = g % XBUF;
          if (!(ok = waitBar(&S.xfull[xb], (g / XBUF) & 1, abortFlag, P.status, 25))) break;
          fenceAfterSync();
          uint32_t const dHH = tmem + TCOL0, dX = dHH + NB;
          uint32_t aX[XSL];
#pragma unroll
          for (int k = 0; k < XSL; ++k) aX[k] = smemAddr(S.x[xb][k]);
          uint32_t const bV[3] = {smemAddr(S.v[s][0]), smemAddr(S.v[s][1]), smemAddr(S.v[s][2])};
          auto dxa = [&](int sl, int k) { return smemDesc(aX[sl] + 32 * k, 1024, 2); };
          auto dvb = [&](int sl, int k) { return smemDesc(bV[sl] + 32 * k, 1024, 2); };
#pragma unroll
          for (int k = 0; k < BK / 16; ++k) {
            uint32_t const acc = k > 0 ? 1u : 0u;
            mmaBf16(dHH, dxa(0, k), dvb(0, k), idesc2x2, acc);   // A += hX hV, B += hX mV
            if constexpr (XS == 3) {
              // B += mX hV + hX lV/256 + m/256 mV + l/256 hV
              mmaBf16(dX, dxa(1, k), dvb(0, k), idesc2, 1);
              mmaBf16(dX, dxa(0, k), dvb(2, k), idesc2, 1);
              mmaBf16(dX, dxa(3, k), dvb(1, k), idesc2, 1);
              mmaBf16(dX, dxa(2, k), dvb(0, k), idesc2, 1);
            } else {
              // B += lX hV + hX lV/256
              mmaBf16(dX, dxa(1, k), dvb(0, k), idesc2, 1);
              mmaBf16(dX, dxa(0, k), dvb(2, k), idesc2, 1);
            }
          }
          mmaCommit(&S.xfree[xb]);
          mmaCommit(&S.empty[s]);
          mmaCommit(&S.tfull);
          if (jj == nblk - 1) mmaCommit(&S.p1free);
        }
        blockCount += nblk;
      }
      mmaCommit(&S.done);
    }
  }
    // teardown of warpgroup 0: every MMA this CTA issued completes before TMEM is released (bounded)
    fenceBeforeSync();
    __syncthreads();
    if (warp == 1) {
      unsigned long long const t0 = globalTimer();
      while (!mbarTryWait(&S.done, 0) && globalTimer() - t0 < kWaitLimitNs) {}
      fenceAfterSync();
      __syncwarp();
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
    }
  } else {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(kRegsCompute));
    // ---------------------------------------------------------------- compute warps
    int const cw = warp - 4;
    int const quarter = warp & 3;
    int const half = cw >> 2;
    int const row = quarter * 32 + lane;
    uint32_t const laneBase = uint32_t(quarter * 32) << 16;
    uint32_t const tAddr = tmem + laneBase + TCOL0 + uint32_t(half * (NB / 2));
    uint32_t blockCount = 0;
    bool ok = true;
    uint64_t ahi[NB / 4], alo[NB / 4];   // T of this thread's row and columns as FP32 hi + lo, column pairs
    uint64_t const k256 = f2pack(256.0f, 256.0f), kInv256 = f2pack(1.0f / 256.0f, 1.0f / 256.0f), kM256 = f2pack(-256.0f, -256.0f);
    uint64_t const kMagic = f2pack(12582912.0f, 12582912.0f);   // 1.5 * 2^23: adding it rounds |x| < 2^22 to an integer
    uint64_t const kInv65536 = f2pack(1.0f / 65536.0f, 1.0f / 65536.0f), kM65536 = f2pack(-65536.0f, -65536.0f);
    uint64_t const mOne = f2pack(-1.0f, -1.0f), mHalf = f2pack(-0.5f, -0.5f);
    for (int item = blockIdx.x; item < nItems && ok; item += gridDim.x) {
      int ii, tile, split;
      decodeItem(P, item, ii, tile, split);
      Instance const * I = P.inst + ii;
      int jb, je;
      itemBlocks(*I, tile, split, jb, je);
      int const nblk = je - jb;   // 0 for an empty item: its T rows and VH are written as zeros
      // a symmetric instance counts the pairs of its diagonal tile (blocks jDiag - 2, jDiag - 1) at half
      // weight in T; their Coulomb row sums stay whole
      int const jDiag = I->sym ? (tile + 1) * (BM / BK) : 0;
      int const r1 = tile * BM + row;
      float4 const p1 = I->r1xyz[r1];
      // rho = 2^24 a1inv a2inv (256 A + B), X' = g a2inv (256 A + B) = X / (2^24 a1inv), and a block's
      // sum_r2 X' Vt = 2^16 (256 A + B) / (bs c) (XS = 2) or 2^24 (256 A + B) / (bs c) (XS = 3):
      // T += 2^40 (or 2^48) a1inv / bs * cinv (256 A + B)
      float const rowA = (XS == 3 ? 281474976710656.0f : 1099511627776.0f) * I->a1inv[r1];   // 2^48 or 2^40, a power of two
#pragma unroll
      for (int c = 0; c < NB / 4; ++c) { ahi[c] = 0; alo[c] = 0; }
      double vh = 0.0;
      float pendingFac = 0.0f;
      bool pending = false;   // block g - 1 still to be flushed
      uint64_t const p1x = f2pack(p1.x, p1.x), p1y = f2pack(p1.y, p1.y), p1z = f2pack(p1.z, p1.z);
      for (int jj = 0; jj < nblk && ok; ++jj) {
        uint32_t const g = blockCount + jj;
        int const s = g % NSTAGE, b = g & 1;
        if (!(ok = waitBar(&S.full[s], (g / NSTAGE) & 1, abortFlag, P.status, 32))) break;
        // this warp's Vt column scales, kept for the flush of block g after the stage is released
        for (int c = lane; c < NB / 2; c += 32) S.cinvT[cw][b][c] = S.cinv[s][half * (NB / 2) + c];
        // g * a2inv for this warp's 32 r2 points (16 pairs) from the stage alone, while GEMM1 of the
        // block may still run; then X' = g * a2inv * (256 rho_hh + rho_cross)
        float4 const * cc = S.coords[s] + half * 32;
        float2 const * sa = reinterpret_cast<float2 const *>(S.a2inv[s] + half * 32);
        uint64_t xv[16];
        uint64_t vsum2 = 0;
#pragma unroll
        for (int pr = 0; pr < 16; ++pr) {
          float4 const qa = cc[2 * pr], qb = cc[2 * pr + 1];
          uint64_t const dx = f2sub(p1x, f2pack(qa.x, qa.y));
          uint64_t const dy = f2sub(p1y, f2pack(qa.z, qa.w));
          uint64_t const dz = f2sub(p1z, f2pack(qb.x, qb.y));
          uint64_t const r2 = f2fma(dx, dx, f2fma(dy, dy, f2mul(dz, dz)));
          float r2a, r2b;
          f2unpack(r2, r2a, r2b);
          uint64_t y = f2pack(rsqrtApprox(r2a), rsqrtApprox(r2b));
          // one Newton step on the hardware estimate: y += (-y/2) (r2 y^2 - 1)
          uint64_t const em = f2fma(f2mul(r2, y), y, mOne);
          y = f2fma(f2mul(y, mHalf), em, y);
          float ya, yb;
          f2unpack(y, ya, yb);
          // pairs below the FP32 resolution of r1 (nearThreshold, packed as r1's w) are dropped here;
          // the near-pair correction adds those that are not exactly coincident in FP64
          ya = r2a >= p1.w ? ya : 0.0f;
          yb = r2b >= p1.w ? yb : 0.0f;
          y = f2pack(ya, yb);
          vsum2 = f2fma(y, f2pack(qb.z, qb.w), vsum2);
          float2 const a2 = sa[pr];
          xv[pr] = f2mul(y, f2pack(a2.x, a2.y));
        }
        if (!(ok = waitBar(&S.sfull[b], (g >> 1) & 1, abortFlag, P.status, 33))) break;
        fenceAfterSync();
        uint32_t const rhoAddr = tmem + laneBase + uint32_t(b * 2 * BK + half * 32);
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
          float rh[16], rx[16];
          tmemLoad16(rhoAddr + hh * 16, rh);
          tmemLoad16(rhoAddr + BK + hh * 16, rx);
          tmemWaitLoad(rh, rx);
          if (hh == 1) {
            // both rho accumulators of this warp's columns are read: the buffer is free for GEMM1
            fenceBeforeSync();
            __syncwarp();
            if (lane == 0) mbarArrive(&S.sfree[b]);
          }
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            int const pr = hh * 8 + e;
            uint64_t const rho = f2fma(f2pack(rh[2 * e], rh[2 * e + 1]), k256, f2pack(rx[2 * e], rx[2 * e + 1]));
            xv[pr] = f2mul(xv[pr], rho);
          }
        }
        // row maximum of |X'| over the block's 64 r2 points: this warp's 32 and the other half's
        float mx = 0.0f;
#pragma unroll
        for (int pr = 0; pr < 16; ++pr) {
          float xa, xb;
          f2unpack(xv[pr], xa, xb);
          mx = fmaxf(mx, fmaxf(fabsf(xa), fabsf(xb)));
        }
        S.rowmax[b][half][row] = mx;
        __syncwarp();
        if (lane == 0) mbarArrive(&S.rmax[b][quarter]);
        if (!(ok = waitBar(&S.rmax[b][quarter], (g >> 1) & 1, abortFlag, P.status, 35))) break;
        mx = fmaxf(mx, S.rowmax[b][half ^ 1][row]);
        // scale bs = 2^(kXExp - E), E = floor(log2 mx) (clamped below), so |X' bs| < 2^(kXExp + 1)
        int const E = max(int((__float_as_uint(mx) >> 23) & 0xFF) - 127, kMinExp);
        float const bs = __uint_as_float(uint32_t(127 + kXExp - E) << 23);
        float const binv = __uint_as_float(uint32_t(127 + E - kXExp) << 23);   // 2^(E - kXExp), E >= -100
        float fac = rowA * binv;   // a power of two (0 when below FP32 range: those blocks add nothing measurable)
        if (jb + jj < jDiag) fac *= 0.5f;
        // X buffer xb is free once GEMM2 of block g - XBUF completed
        int const xb = g % XBUF;
        if (g >= uint32_t(XBUF) && !(ok = waitBar(&S.xfree[xb], ((g / XBUF) - 1) & 1, abortFlag, P.status, 34))) break;
        uint64_t const bb = f2pack(bs, bs);
#pragma unroll
        for (int ch = 0; ch < 4; ++ch) {
          uint32_t const off = sw128(row, half * 4 + ch);
          if constexpr (XS == 3) {
            // t = X' bs = 65536 h + 256 m + l: h = rint(t / 65536), m = rint(r / 256), l = r - 256 m,
            // r = t - 65536 h; slices h, m, l/256, m/256
            uint32_t sh[4], sm[4], sl[4], sms[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              uint64_t const t = f2mul(xv[ch * 4 + e], bb);
              uint64_t const h = f2sub(f2fma(t, kInv65536, kMagic), kMagic);
              uint64_t const r = f2fma(h, kM65536, t);
              uint64_t const m = f2sub(f2fma(r, kInv256, kMagic), kMagic);
              // the lowest slice only feeds the cross accumulator, which rounds 2^-8 below the result:
              // it is stored rounded to nearest BF16 (8 significant bits), not rounded to an integer
              sh[e] = bf16PairExact(h);
              sm[e] = bf16PairExact(m);
              sl[e] = bf16PairRn(f2mul(f2fma(m, kM256, r), kInv256));
              sms[e] = bf16PairExact(f2mul(m, kInv256));
            }
            *reinterpret_cast<uint4 *>(S.x[xb][0] + off) = make_uint4(sh[0], sh[1], sh[2], sh[3]);
            *reinterpret_cast<uint4 *>(S.x[xb][1] + off) = make_uint4(sm[0], sm[1], sm[2], sm[3]);
            *reinterpret_cast<uint4 *>(S.x[xb][2] + off) = make_uint4(sl[0], sl[1], sl[2], sl[3]);
            *reinterpret_cast<uint4 *>(S.x[xb][3] + off) = make_uint4(sms[0], sms[1], sms[2], sms[3]);
          } else {
            // t = X' bs = 256 h + l, h = rint(t / 256), l = t - 256 h (rounded to nearest BF16: it only
            // feeds the cross accumulator)
            uint32_t hi[4], lo[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              uint64_t const t = f2mul(xv[ch * 4 + e], bb);
              uint64_t const h = f2sub(f2fma(t, kInv256, kMagic), kMagic);
              hi[e] = bf16PairExact(h);
              lo[e] = bf16PairRn(f2fma(h, kM256, t));
            }
            *reinterpret_cast<uint4 *>(S.x[xb][0] + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
            *reinterpret_cast<uint4 *>(S.x[xb][1] + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
          }
        }
        float vs0, vs1;
        f2unpack(vsum2, vs0, vs1);
        vh += double(vs0 + vs1);
        fenceProxyAsync();
        __syncwarp();
        if (lane == 0) { mbarArrive(&S.xfull[xb]); mbarArrive(&S.empty[s]); }
        if (pending && !(ok = flushBlock<NB>(S, tAddr, g - 1, cw, pendingFac, ahi, alo, lane, abortFlag, P.status))) break;
        pending = true;
        pendingFac = fac;
      }
      if (ok && pending) ok = flushBlock<NB>(S, tAddr, blockCount + nblk - 1, cw, pendingFac, ahi, alo, lane, abortFlag, P.status);
      blockCount += nblk;
      if (!ok) break;
      int const n1 = I->n1;
      if (r1 < n1) {
        int const nbReal = I->nb;
        double * T = I->T + int64_t(split) * I->tStride + int64_t(r1) * I->ldt;
#pragma unroll
        for (int c = 0; c < NB / 2; ++c) {
          int const col = half * (NB / 2) + c;
          float h0, h1, l0, l1;
          f2unpack(ahi[c / 2], h0, h1);
          f2unpack(alo[c / 2], l0, l1);
          if (col < nbReal) T[col] = (c & 1) ? double(h1) + double(l1) : double(h0) + double(l0);
        }
      }
      // the two r2-half warps of a row each summed half of the r2 points of every block
      if (r1 < n1) atomicAdd(&I->VH[int64_t(split) * I->vhStride + r1], vh);
    }
    fenceBeforeSync();
    __syncthreads();
  }
}

// ---- operand packing ---------------------------------------------------------------------------------
// floor(log2 m) clamped below at kMinExp (m = 0 included)
__device__ __forceinline__ int sliceExponent(double m)
{
  if (!(m > 0.0)) return kMinExp;
  int e = 0;
  frexp(m, &e);   // m = f 2^e, f in [0.5, 1)
  return max(e - 1, kMinExp);
}

// t (|t| < 2^24) -> BF16 slices h = rint(t / 65536), m = rint((t - 65536 h) / 256),
// l = rint(t - 65536 h - 256 m), stored as h, m and l / 256; h, m, l are integers of at most 8
// significant bits, so each slice is exact
__device__ __forceinline__ void sliceFactor(double t, __nv_bfloat16 & h, __nv_bfloat16 & m, __nv_bfloat16 & l)
{
  double const hd = rint(t * (1.0 / 65536.0));
  double const r = t - 65536.0 * hd;
  double const md = rint(r * (1.0 / 256.0));
  double const ld = rint(r - 256.0 * md);
  h = __float2bfloat16_rn(float(hd));
  m = __float2bfloat16_rn(float(md));
  l = __float2bfloat16_rn(float(ld * (1.0 / 256.0)));
}

// psi [n][ldpsi] FP64 (R columns) -> fixed-point slices h / m / l BF16 [npad][RP] each (zero padded),
// and m / 256 when sms is not null, with the inverse row scale ainv [npad]; one warp per row
__global__ void kPackPsi(int64_t n, int64_t npad, int R, int RP, const double * psi, int ldpsi, __nv_bfloat16 * sh, __nv_bfloat16 * sm,
                         __nv_bfloat16 * sl, __nv_bfloat16 * sms, float * ainv)
{
  int const lane = threadIdx.x & 31;
  for (int64_t r = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; r < npad; r += (int64_t(gridDim.x) * blockDim.x) >> 5) {
    double v[2];
    double m = 0.0;
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      int const b = lane + 32 * u;
      v[u] = (r < n && b < R) ? psi[r * ldpsi + b] : 0.0;
      m = fmax(m, fabs(v[u]));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    int const E = sliceExponent(m);
    double const scale = ldexp(1.0, kFactorExp - E);
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      int const b = lane + 32 * u;
      if (b < RP) {
        sliceFactor(v[u] * scale, sh[r * RP + b], sm[r * RP + b], sl[r * RP + b]);
        if (sms) sms[r * RP + b] = __float2bfloat16_rn(__bfloat162float(sm[r * RP + b]) * (1.0f / 256.0f));
      }
    }
    if (lane == 0) ainv[r] = ldexpf(1.0f, E - kFactorExp);
  }
}

// inverse Vt column scales per r2 block: cinv[blk][c] from max_{r2 in blk} |V[r2][c]|
__global__ void kVtScales(int64_t n, int nBlocks, int nb, int NB, const double * V, int ldv, float * cinv)
{
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < int64_t(nBlocks) * NB; idx += int64_t(gridDim.x) * blockDim.x) {
    int const c = int(idx % NB);
    int64_t const blk = idx / NB;
    double m = 0.0;
    if (c < nb)
      for (int64_t r = blk * BK; r < min(n, (blk + 1) * BK); ++r) m = fmax(m, fabs(V[r * ldv + c]));
    cinv[idx] = ldexpf(1.0f, sliceExponent(m) - kFactorExp);
  }
}

// V [n][ldv] FP64 (nb columns) -> transposed fixed-point slices h / m / l BF16 [NB][npad] each (tiled
// transpose)
__global__ void kPackVt(int64_t n, int64_t npad, int nb, int NB, const double * V, int ldv, const float * cinv, __nv_bfloat16 * sh,
                        __nv_bfloat16 * sm, __nv_bfloat16 * sl)
{
  __shared__ double tile[32][33];
  int64_t const r0 = int64_t(blockIdx.x) * 32;
  int const c0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    int64_t const r = r0 + k;
    int const c = c0 + threadIdx.x;
    tile[k][threadIdx.x] = (r < n && c < nb) ? V[r * ldv + c] : 0.0;
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    int const c = c0 + k;
    int64_t const r = r0 + threadIdx.x;
    if (c < NB && r < npad) {
      double const scale = 1.0 / double(cinv[(r / BK) * NB + c]);   // a power of two
      int64_t const o = int64_t(c) * npad + r;
      sliceFactor(tile[threadIdx.x][k] * scale, sh[o], sm[o], sl[o]);
    }
  }
}

// pts [3][n] -> float4 [npad] (x, y, z, nearThreshold(x, y, z)); padding points sit far away
__global__ void kPackCoords(int64_t n, int64_t npad, const double * pts, float4 * out)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < npad; i += int64_t(gridDim.x) * blockDim.x) {
    float const x = i < n ? float(pts[i]) : 1.0e4f, y = i < n ? float(pts[n + i]) : 1.0e4f, z = i < n ? float(pts[2 * n + i]) : 1.0e4f;
    out[i] = make_float4(x, y, z, nearThreshold(x, y, z));
  }
}

// r2 points in pairs: pair p -> {x_2p, x_2p+1, y_2p, y_2p+1}, {z_2p, z_2p+1, c_2p, c_2p+1} with the
// Coulomb source c (npad even); padding points sit far away with c = 0
__global__ void kPackCoordPairs(int64_t n, int64_t npad, const double * pts, const double * coul, float4 * out)
{
  for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < npad / 2; p += int64_t(gridDim.x) * blockDim.x) {
    float v[2][4];
    for (int u = 0; u < 2; ++u) {
      int64_t const i = 2 * p + u;
      bool const in = i < n;
      v[u][0] = in ? float(pts[i]) : 1.0e4f;
      v[u][1] = in ? float(pts[n + i]) : 1.0e4f;
      v[u][2] = in ? float(pts[2 * n + i]) : 1.0e4f;
      v[u][3] = (in && coul) ? float(coul[i]) : 0.0f;
    }
    out[2 * p] = make_float4(v[0][0], v[1][0], v[0][1], v[1][1]);
    out[2 * p + 1] = make_float4(v[0][2], v[1][2], v[0][3], v[1][3]);
  }
}

// Symmetric instances (r1 and r2 the same points): the Coulomb row sums over the r2 blocks before each
// r1 tile's diagonal, which the tensor kernel skips, added to the potential:
//   VH[r] += sum_{j < BM tile(r)} g(r, j) c(j)
// with the tensor kernel's FP32 arithmetic on the same packed points (its drop rule and its
// Newton-refined rsqrt), FP32 sums per 64-point block added in FP64.  One block of 64 threads per
// (r1 tile, chunk of its lower r2 blocks), the tiles with the most pairs first; each thread takes two
// rows of the tile (r and r + 64), so that every r2 point it loads serves both.  Each chunk's row sums
// go to an FP64 partial, and the partials of a row are added in chunk order (deterministic).
__device__ __forceinline__ uint64_t coulombPair(uint64_t px, uint64_t py, uint64_t pz, float thr, float4 qa, float4 qb)
{
  uint64_t const mOne = f2pack(-1.0f, -1.0f), mHalf = f2pack(-0.5f, -0.5f);
  uint64_t const dx = f2sub(px, f2pack(qa.x, qa.y));
  uint64_t const dy = f2sub(py, f2pack(qa.z, qa.w));
  uint64_t const dz = f2sub(pz, f2pack(qb.x, qb.y));
  uint64_t const r2 = f2fma(dx, dx, f2fma(dy, dy, f2mul(dz, dz)));
  float r2a, r2b;
  f2unpack(r2, r2a, r2b);
  uint64_t y = f2pack(rsqrtApprox(r2a), rsqrtApprox(r2b));
  uint64_t const em = f2fma(f2mul(r2, y), y, mOne);
  y = f2fma(f2mul(y, mHalf), em, y);
  float ya, yb;
  f2unpack(y, ya, yb);
  ya = r2a >= thr ? ya : 0.0f;
  yb = r2b >= thr ? yb : 0.0f;
  return f2pack(ya, yb);
}

// The lower rows of one r1 tile of one contraction over the r2 blocks [jb, je) (a chunk of the blocks
// before the tile): out[t] and out[t + 64] receive the two rows' sums (rows r = BM tile + t, r + 64)
__device__ __forceinline__ void coulombLowerChunk(int tile, int jb, int je, const float4 * __restrict__ r1xyz, const float4 * __restrict__ r2pairs,
                                                  double * out)
{
  // the r2 points pass through shared memory in 64-point blocks (64 float4 in pair layout, one per
  // thread), the next block's load in flight while the current one is summed
  __shared__ float4 sq[2][BK];
  int const t = threadIdx.x;
  int64_t const r0 = int64_t(tile) * BM + t, r1 = r0 + BM / 2;
  float4 const pa = r1xyz[r0], pb = r1xyz[r1];
  uint64_t const ax = f2pack(pa.x, pa.x), ay = f2pack(pa.y, pa.y), az = f2pack(pa.z, pa.z);
  uint64_t const bx = f2pack(pb.x, pb.x), by = f2pack(pb.y, pb.y), bz = f2pack(pb.z, pb.z);
  double vha = 0.0, vhb = 0.0;
  if (je > jb) sq[0][t] = r2pairs[int64_t(jb) * BK + t];
  __syncthreads();
  for (int j = jb; j < je; ++j) {
    int const buf = (j - jb) & 1;
    bool const more = j + 1 < je;
    float4 const nxt = more ? r2pairs[int64_t(j + 1) * BK + t] : make_float4(0, 0, 0, 0);
    uint64_t va = 0, vb = 0;
#pragma unroll 4
    for (int e = 0; e < BK / 2; ++e) {
      float4 const qa = sq[buf][2 * e], qb = sq[buf][2 * e + 1];
      uint64_t const c = f2pack(qb.z, qb.w);
      va = f2fma(coulombPair(ax, ay, az, pa.w, qa, qb), c, va);
      vb = f2fma(coulombPair(bx, by, bz, pb.w, qa, qb), c, vb);
    }
    float u0, u1;
    f2unpack(va, u0, u1);
    vha += double(u0 + u1);
    f2unpack(vb, u0, u1);
    vhb += double(u0 + u1);
    if (more) sq[buf ^ 1][t] = nxt;   // block j - 1's buffer: every thread finished it before the last barrier
    __syncthreads();
  }
  out[t] = vha;
  out[t + BM / 2] = vhb;
}

// The lower blocks of tile p (its 2 p r2 blocks before the diagonal) in kLowerChunks chunks, chunk c the
// blocks [c 2p / S, (c + 1) 2p / S): heavy tiles in short pieces, so that no single block's work sets
// the kernel's tail
constexpr int kLowerChunks = 8;
__device__ __forceinline__ void lowerChunkRange(int tile, int c, int & jb, int & je)
{
  int const n = tile * (BM / BK);
  jb = int(int64_t(n) * c / kLowerChunks);
  je = int(int64_t(n) * (c + 1) / kLowerChunks);
}

// one block per (tile >= 1, chunk), the tiles with the most pairs first: the chunk's row sums into
// part[((tile - 1) kLowerChunks + chunk) BM + row]
__global__ void __launch_bounds__(BM / 2) kCoulombLower(int nTiles, const float4 * __restrict__ r1xyz, const float4 * __restrict__ r2pairs,
                                                       double * part)
{
  int const tile = nTiles - 1 - int(blockIdx.x) / kLowerChunks, c = int(blockIdx.x) % kLowerChunks;
  int jb, je;
  lowerChunkRange(tile, c, jb, je);
  coulombLowerChunk(tile, jb, je, r1xyz, r2pairs, part + (int64_t(tile - 1) * kLowerChunks + c) * BM);
}

// VH[r] += the chunk sums of row r in chunk order, for the rows of tiles >= 1
__global__ void kCoulombLowerSum(int64_t n1, const double * __restrict__ part, double * VH)
{
  for (int64_t r = BM + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n1; r += int64_t(gridDim.x) * blockDim.x) {
    int64_t const tile = r / BM;
    double const * q = part + (tile - 1) * kLowerChunks * BM + r % BM;
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kLowerChunks; ++c) s += q[c * BM];
    VH[r] += s;
  }
}

// the lower rows of several contractions in one launch: block b takes tile tiles[b].y of job tiles[b].x
// (the list holds every (job, tile >= 1) once, the tiles with the most pairs first)
struct CoulombLowerJob {
  const float4 * r1xyz;
  const float4 * r2pairs;
  double * VH;
  int64_t n1;
};
// one block per (listed (job, tile), chunk): the chunk's row sums into part[(entry kLowerChunks + chunk) BM + row]
__global__ void __launch_bounds__(BM / 2) kCoulombLowerBatch(const CoulombLowerJob * __restrict__ jobs, const int2 * __restrict__ tiles,
                                                            double * part)
{
  int const entry = int(blockIdx.x) / kLowerChunks, c = int(blockIdx.x) % kLowerChunks;
  int2 const jt = tiles[entry];
  CoulombLowerJob const j = jobs[jt.x];
  int jb, je;
  lowerChunkRange(jt.y, c, jb, je);
  coulombLowerChunk(jt.y, jb, je, j.r1xyz, j.r2pairs, part + (int64_t(entry) * kLowerChunks + c) * BM);
}

// VH[r] += the chunk sums of the listed (job, tile)'s rows in chunk order; one block of BM threads per entry
__global__ void __launch_bounds__(BM) kCoulombLowerBatchSum(const CoulombLowerJob * __restrict__ jobs, const int2 * __restrict__ tiles,
                                                           const double * __restrict__ part)
{
  int2 const jt = tiles[blockIdx.x];
  CoulombLowerJob const j = jobs[jt.x];
  int const t = threadIdx.x;
  int64_t const r = int64_t(jt.y) * BM + t;
  if (r >= j.n1) return;
  double const * q = part + int64_t(blockIdx.x) * kLowerChunks * BM + t;
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kLowerChunks; ++c) s += q[c * BM];
  j.VH[r] += s;
}

}  // namespace tc

// ------------------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------------------
EncodeTiledFn encodeTiled()
{
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void * p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

bool makeMap2d(CUtensorMap * m, CUtensorMapDataType type, uint32_t elemBytes, void * base, uint64_t inner, uint64_t outer, uint32_t boxInner,
               uint32_t boxOuter, CUtensorMapSwizzle sw)
{
  EncodeTiledFn fn = encodeTiled();
  if (!fn) return false;
  cuuint64_t dims[2] = {inner, outer};
  cuuint64_t strides[1] = {inner * elemBytes};
  cuuint32_t box[2] = {boxInner, boxOuter};
  cuuint32_t es[2] = {1, 1};
  return fn(m, type, 2, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

namespace {

// 2-D BF16 tensor map: inner extent `inner` (contiguous), `outer` rows, box (boxInner, boxOuter)
bool makeMap(CUtensorMap * m, void * base, uint64_t inner, uint64_t outer, uint32_t boxInner, uint32_t boxOuter, CUtensorMapSwizzle sw)
{
  return makeMap2d(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, inner, outer, boxInner, boxOuter, sw);
}

template <int NB, int RP, int XS, int NS>
int launchFlash(tcscf_ctx * ctx, tc::Params const & P, int grid)
{
  size_t const smem = sizeof(tc::Smem<NB, RP, XS, NS>) + 1024;
  static_assert(sizeof(tc::Smem<NB, RP, XS, NS>) + 1024 <= 232448, "shared memory per CTA");
  TCSCF_CUDA(ctx, cudaFuncSetAttribute(tc::kFlashTc<NB, RP, XS, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  tc::kFlashTc<NB, RP, XS, NS><<<grid, tc::NTHREADS, smem, ctx->stream>>>(P);
  TCSCF_LAUNCH(ctx);
  return TCSCF_OK;
}

// tile classes: (NB, RP, XS, TMA stages); XS = 0 is the TF32 kernel (its stage count is its own)
constexpr int kClasses[8][4] = {{64, 32, 2, 3}, {64, 32, 3, 3}, {64, 32, 3, 2}, {64, 64, 2, 2},
                                {128, 32, 2, 2}, {128, 32, 3, 2}, {64, 32, 0, 0}, {128, 32, 0, 0}};

bool classExists(int NB, int RP, int XS, int NS)
{
  for (auto const & cl : kClasses)
    if (cl[0] == NB && cl[1] == RP && cl[2] == XS && cl[3] == NS) return true;
  return false;
}

int launchClass(tcscf_ctx * ctx, int NB, int RP, int XS, int NS, tc::Params const & P, int grid)
{
  if (XS == 0) return launchTf32(ctx, NB, P, grid);
  if (NB == 64 && RP == 32 && XS == 3) return NS == 2 ? launchFlash<64, 32, 3, 2>(ctx, P, grid) : launchFlash<64, 32, 3, 3>(ctx, P, grid);
  if (NB == 64 && RP == 32 && XS == 2) return launchFlash<64, 32, 2, 3>(ctx, P, grid);
  if (NB == 64 && RP == 64 && XS == 2) return launchFlash<64, 64, 2, 2>(ctx, P, grid);
  if (NB == 128 && RP == 32) return XS == 3 ? launchFlash<128, 32, 3, 2>(ctx, P, grid) : launchFlash<128, 32, 2, 2>(ctx, P, grid);
  return fail(ctx, TCSCF_ERR_UNSUPPORTED, "no tensor kernel for this tile class");
}

// bytes of the packed Vt operand: h, m and l slices [NB][n2pad], then the column scales [nBlocks][NB]
size_t packedVtBytes(int NB, int64_t n2pad)
{
  return size_t(3) * NB * n2pad * sizeof(__nv_bfloat16) + size_t(n2pad / tc::BK) * NB * sizeof(float);
}

int packVt(tcscf_ctx * ctx, int64_t n2, int64_t n2pad, int nb, int NB, const double * V, int ldv, void * out)
{
  auto * sh = static_cast<__nv_bfloat16 *>(out);
  auto * sm = sh + size_t(NB) * n2pad;
  auto * sl = sm + size_t(NB) * n2pad;
  auto * cinv = reinterpret_cast<float *>(sl + size_t(NB) * n2pad);
  int const nBlocks = int(n2pad / tc::BK);
  tc::kVtScales<<<gridBlocks(int64_t(nBlocks) * NB, 256), 256, 0, ctx->stream>>>(n2, nBlocks, nb, NB, V, ldv, cinv);
  TCSCF_LAUNCH(ctx);
  dim3 const tb{32, 8, 1};
  dim3 const tg{unsigned((n2pad + 31) / 32), unsigned((NB + 31) / 32), 1};
  tc::kPackVt<<<tg, tb, 0, ctx->stream>>>(n2, n2pad, nb, NB, V, ldv, cinv, sh, sm, sl);
  TCSCF_LAUNCH(ctx);
  return TCSCF_OK;
}

}  // namespace

size_t packedVtOperandBytes(int NB, int64_t n2pad) { return packedVtBytes(NB, n2pad); }

int packVtOperand(tcscf_ctx * ctx, int64_t n2, int64_t n2pad, int nb, int NB, const double * V, int ldv, void * out)
{
  return packVt(ctx, n2, n2pad, nb, NB, V, ldv, out);
}

int packPointsFp32(tcscf_ctx * ctx, int64_t n, int64_t npad, const double * pts, float4 * out)
{
  tc::kPackCoords<<<gridBlocks(npad, 256), 256, 0, ctx->stream>>>(n, npad, pts, out);
  TCSCF_LAUNCH(ctx);
  return TCSCF_OK;
}

int packPointPairsFp32(tcscf_ctx * ctx, int64_t n, int64_t npad, const double * pts, const double * coul, float4 * out)
{
  tc::kPackCoordPairs<<<gridBlocks(npad / 2, 256), 256, 0, ctx->stream>>>(n, npad, pts, coul, out);
  TCSCF_LAUNCH(ctx);
  return TCSCF_OK;
}

int tensorPackedV(tcscf_ctx * ctx, Grid & g2, const double * V, double scale, const void ** packed)
{
  int const NB = g2.nb <= 64 ? 64 : 128;
  int64_t const n2pad = (g2.n + tc::BK - 1) / tc::BK * tc::BK;
  if (!g2.vtCache || g2.vtNB != NB || g2.vtN2pad != n2pad || g2.vtScale != scale) {
    gridRelease(ctx, g2.vtCache);
    g2.vtCache = nullptr;
    TCSCF_TRY(gridAlloc(ctx, &g2.vtCache, packedVtBytes(NB, n2pad)));
    TCSCF_TRY(packVt(ctx, g2.n, n2pad, g2.nb, NB, V, g2.nb, g2.vtCache));
    g2.vtNB = NB;
    g2.vtN2pad = n2pad;
    g2.vtScale = scale;
  }
  *packed = g2.vtCache;
  return TCSCF_OK;
}

bool tensorPathAvailable(Contraction const & c, int precision, std::string * why)
{
  if (precision != TCSCF_PREC_BF16X3 && precision != TCSCF_PREC_TF32) { if (why) *why = "not a tensor-core precision"; return false; }
  if (c.kernel != TCSCF_K_INV_R12) { if (why) *why = "tensor path implements the 1/r12 kernel"; return false; }
  if (c.R < 1) { if (why) *why = "empty density factor"; return false; }
  if (c.ncol > 128) { if (why) *why = "tensor path supports nb <= 128"; return false; }
  if (c.R > tensorRankLimit(c, precision)) { if (why) *why = "one tensor launch holds a density factor rank <= 32 (TF32, or nb > 64) or 64"; return false; }
  if (!encodeTiled()) { if (why) *why = "cuTensorMapEncodeTiled unavailable"; return false; }
  return true;
}

namespace {

int smCount()
{
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

int defaultSplit(int nTiles, int nBlocks, int sms) { return std::max(1, std::min(sms / std::max(1, nTiles), nBlocks / 4)); }

// a requested split count after rounding the r2 blocks per split up (what the launch really runs)
int effectiveSplit(int nBlocks, int want)
{
  int const per = (nBlocks + want - 1) / want;
  return (nBlocks + per - 1) / per;
}

// the autotuner's largest split: every split keeps at least 16 blocks of 64 r2 points
int maxTunedSplit(int nBlocks) { return std::max(1, nBlocks / 16); }

struct Shape {
  int NB, RP, XS, NS;
  int64_t n1pad, n2pad;
  int nTiles, nBlocks, nSplit, perSplit;
};

Shape shapeOf(Contraction const & c, int sms, int precision)
{
  Shape sh{};
  sh.NB = c.ncol <= 64 ? 64 : 128;
  sh.RP = c.R <= 32 ? 32 : 64;
  // 24-bit X wherever shared memory holds its four slices (rank padding 32; 64 leaves no room): with
  // 16-bit X the converged Kr SCF energy (406,000 points) was 1.5e-6 Eh from FP64, with 24-bit X
  // 9e-8, for a 9 % slower kernel; the TF32 kernel (XS = 0) has rank padding 32
  if (precision == TCSCF_PREC_TF32) sh.XS = 0;
  else sh.XS = sh.RP == 32 ? 3 : 2;
  // a class the autotuner asks for (wider T tile, fewer TMA stages): the same arithmetic per column
  if (c.tileNB > sh.NB && sh.XS != 0) sh.NB = c.tileNB;
  sh.NS = sh.XS == 0 ? 0 : tc::stagesFor(sh.NB, sh.RP);
  if (c.stages > 0 && sh.XS != 0 && classExists(sh.NB, sh.RP, sh.XS, c.stages)) sh.NS = c.stages;
  sh.n1pad = (c.n1 + tc::BM - 1) / tc::BM * tc::BM;
  sh.n2pad = (c.n2 + tc::BK - 1) / tc::BK * tc::BK;
  sh.nTiles = int(sh.n1pad / tc::BM);
  sh.nBlocks = int(sh.n2pad / tc::BK);
  // split r2 when there are fewer tiles than SMs (partials summed deterministically afterwards), or
  // as the caller (the autotuner) asks
  sh.nSplit = c.nSplit > 0 ? std::min(c.nSplit, sh.nBlocks) : defaultSplit(sh.nTiles, sh.nBlocks, sms);
  sh.perSplit = (sh.nBlocks + sh.nSplit - 1) / sh.nSplit;
  sh.nSplit = (sh.nBlocks + sh.perSplit - 1) / sh.perSplit;
  return sh;
}

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

}  // namespace

std::vector<int> splitCandidates(int64_t n1, int64_t n2, int sms)
{
  int const nTiles = int((n1 + tc::BM - 1) / tc::BM);
  int const nBlocks = int((n2 + tc::BK - 1) / tc::BK);
  std::vector<int> out{effectiveSplit(nBlocks, defaultSplit(nTiles, nBlocks, sms))};
  for (int s : {1, 2, 3, 4, 6, 8}) {
    if (s > maxTunedSplit(nBlocks)) break;
    int const e = effectiveSplit(nBlocks, s);
    if (std::find(out.begin(), out.end(), e) == out.end()) out.push_back(e);
  }
  return out;
}

int splitForPolicy(Contraction const & c, int precision, int policy)
{
  if (policy == 1) return 0;
  if (policy <= 0) return 1;
  Shape const sh = shapeOf(c, smCount(), precision);
  return std::max(1, std::min(sh.nSplit * policy, std::max(sh.nSplit, maxTunedSplit(sh.nBlocks))));
}

size_t tensorArenaBytes(Contraction const & c, int precision)
{
  Shape const sh = shapeOf(c, smCount(), precision);
  size_t const bf = sizeof(__nv_bfloat16);
  size_t b = 0;
  if (precision == TCSCF_PREC_TF32) b += align256(tf32OperandBytes(sh.NB, sh.n1pad, sh.n2pad));
  else {
    b += 4 * align256(size_t(sh.n1pad) * sh.RP * bf) + 3 * align256(size_t(sh.n2pad) * sh.RP * bf);
    if (!c.vtPacked) b += align256(packedVtBytes(sh.NB, sh.n2pad));
  }
  b += align256(size_t(sh.n1pad) * sizeof(float4)) + align256(size_t(sh.n2pad) * sizeof(float4));
  b += align256(size_t(sh.n1pad) * sizeof(float)) + align256(size_t(sh.n2pad) * sizeof(float));
  if (sh.nSplit > 1 || !c.VH) b += align256(sizeof(double) * size_t(sh.nSplit) * c.n1 * (c.ldt + 1));
  return b + 256;
}

int tensorPrepare(tcscf_ctx * ctx, Contraction const & c, int precision, void * arena, size_t arenaBytes, TensorPrep & tp)
{
  std::string why;
  if (!tensorPathAvailable(c, precision, &why)) return fail(ctx, TCSCF_ERR_UNSUPPORTED, why);
  TCSCF_CHECK(ctx, arenaBytes >= tensorArenaBytes(c, precision), TCSCF_ERR_INVALID_ARGUMENT, "internal: tensor arena too small");
  TCSCF_CHECK(ctx, !c.sym || (c.p1 == c.p2 && c.n1 == c.n2 && c.psi1 == c.psi2 && c.R > 0 && (c.VH != nullptr) == (c.coul != nullptr)),
              TCSCF_ERR_INVALID_ARGUMENT, "internal: a symmetric contraction needs r1 = r2 and psi1 = psi2");
  Shape const sh = shapeOf(c, smCount(), precision);
  int const NB = sh.NB, RP = sh.RP;
  bool const tf32 = precision == TCSCF_PREC_TF32;
  int64_t const n1pad = sh.n1pad, n2pad = sh.n2pad;
  size_t const bf = sizeof(__nv_bfloat16);
  char * q = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(arena) + 255) & ~uintptr_t(255));
  auto take = [&](size_t n) { char * r = q; q += align256(n); return r; };
  __nv_bfloat16 * psi1s[4] = {};
  __nv_bfloat16 * psi2s[3] = {};
  void * vt = nullptr;
  void * tf32Ops = nullptr;
  if (tf32) tf32Ops = take(tf32OperandBytes(NB, n1pad, n2pad));
  else {
    for (auto & a : psi1s) a = reinterpret_cast<__nv_bfloat16 *>(take(size_t(n1pad) * RP * bf));
    for (auto & a : psi2s) a = reinterpret_cast<__nv_bfloat16 *>(take(size_t(n2pad) * RP * bf));
    vt = c.vtPacked ? const_cast<void *>(c.vtPacked) : take(packedVtBytes(NB, n2pad));
  }
  auto * r1c = reinterpret_cast<float4 *>(take(size_t(n1pad) * sizeof(float4)));
  auto * r2c = reinterpret_cast<float4 *>(take(size_t(n2pad) * sizeof(float4)));
  auto * a1inv = reinterpret_cast<float *>(take(size_t(n1pad) * sizeof(float)));
  auto * a2inv = reinterpret_cast<float *>(take(size_t(n2pad) * sizeof(float)));
  double * Tout = c.T;
  double * VHout = c.VH;
  if (sh.nSplit > 1 || !c.VH) {
    // split partials (and a Coulomb sink when the caller does not want the potential)
    double * sp = reinterpret_cast<double *>(take(sizeof(double) * size_t(sh.nSplit) * c.n1 * (c.ldt + 1)));
    if (sh.nSplit > 1) Tout = sp;
    VHout = sp + size_t(sh.nSplit) * c.n1 * c.ldt;
  }
  tc::kPackCoords<<<gridBlocks(n1pad, 256), 256, 0, ctx->stream>>>(c.n1, n1pad, c.p1, r1c);
  TCSCF_LAUNCH(ctx);
  tc::kPackCoordPairs<<<gridBlocks(n2pad / 2, 256), 256, 0, ctx->stream>>>(c.n2, n2pad, c.p2, c.coul, r2c);
  TCSCF_LAUNCH(ctx);
  TCSCF_CUDA(ctx, cudaMemsetAsync(VHout, 0, sizeof(double) * size_t(sh.nSplit) * c.n1, ctx->stream));
  tc::Instance & I = tp.inst;
  I = tc::Instance{};
  I.nTiles = sh.nTiles; I.nSplit = sh.nSplit; I.blocksPerSplit = sh.perSplit; I.nBlocks = sh.nBlocks;
  // TF32 keeps the full contraction: with 11-bit operands its mirrored half would carry the r2-side
  // rounding of V twice (Ne: |dE| 2.1e-5 against 7.5e-7 Eh for the full form)
  I.sym = c.sym && !tf32 ? 1 : 0;
  I.n1 = int(c.n1); I.nb = c.ncol; I.ldt = c.ldt;
  I.r1xyz = r1c; I.r2pairs = r2c;
  I.T = Tout; I.VH = VHout;
  I.tStride = int64_t(c.n1) * c.ldt; I.vhStride = c.n1;
  tp.NB = NB; tp.RP = RP; tp.XS = sh.XS; tp.NS = sh.NS;
  tp.c = c;
  if (tf32) return tf32PackOperands(ctx, c, NB, n1pad, n2pad, tf32Ops, tp.maps);

  auto * vts = static_cast<__nv_bfloat16 *>(vt);   // h, m, l slices [NB][n2pad] each
  auto * cinv = reinterpret_cast<float *>(vts + 3 * size_t(NB) * n2pad);

  // operand preparation (fixed-point BF16 slices with their scales, transposes, FP32 coordinates)
  tc::kPackPsi<<<gridBlocks(n1pad * 32, 256), 256, 0, ctx->stream>>>(c.n1, n1pad, c.R, RP, c.psi1, c.ldpsi, psi1s[0], psi1s[1], psi1s[2],
                                                                      psi1s[3], a1inv);
  TCSCF_LAUNCH(ctx);
  tc::kPackPsi<<<gridBlocks(n2pad * 32, 256), 256, 0, ctx->stream>>>(c.n2, n2pad, c.R, RP, c.psi2, c.ldpsi, psi2s[0], psi2s[1], psi2s[2],
                                                                      nullptr, a2inv);
  TCSCF_LAUNCH(ctx);
  if (!c.vtPacked) TCSCF_TRY(packVt(ctx, c.n2, n2pad, c.ncol, NB, c.V, c.ldv, vt));

  CUtensorMapSwizzle const psw = RP == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B;
  bool okm = true;
  for (int i = 0; i < 4; ++i) okm = okm && makeMap(&tp.maps[i], psi1s[i], RP, n1pad, RP, tc::BM, psw);
  for (int i = 0; i < 3; ++i) {
    okm = okm && makeMap(&tp.maps[4 + i], psi2s[i], RP, n2pad, RP, tc::BK, psw);
    okm = okm && makeMap(&tp.maps[7 + i], vts + size_t(i) * NB * n2pad, n2pad, NB, tc::BK, NB, CU_TENSOR_MAP_SWIZZLE_128B);
  }
  TCSCF_CHECK(ctx, okm, TCSCF_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  I.a1inv = a1inv; I.a2inv = a2inv; I.cinv = cinv;
  return TCSCF_OK;
}

namespace {
// whether a contraction has Coulomb rows below its diagonal tiles to add (symmetric, with a potential)
bool hasLowerRows(tc::Instance const & I, Contraction const & c) { return I.sym && c.VH && I.nTiles >= 2; }
// bytes of the chunk partials of kCoulombLower for nTiles r1 tiles (or of kCoulombLowerBatch for that
// many listed tiles)
size_t lowerPartBytes(int64_t nTiles) { return size_t(std::max<int64_t>(nTiles, 1)) * tc::kLowerChunks * tc::BM * sizeof(double); }

// the Coulomb row sums a symmetric instance skipped, once c.VH holds the rest: the chunks of every tile
// (kCoulombLower) into part (lowerPartBytes(nTiles - 1)), then their sums in chunk order
int coulombLower(tcscf_ctx * ctx, tc::Instance const & I, Contraction const & c, double * part)
{
  if (!hasLowerRows(I, c)) return TCSCF_OK;
  tc::kCoulombLower<<<unsigned((I.nTiles - 1) * tc::kLowerChunks), tc::BM / 2, 0, ctx->stream>>>(I.nTiles, I.r1xyz, I.r2pairs, part);
  TCSCF_LAUNCH(ctx);
  tc::kCoulombLowerSum<<<gridBlocks(c.n1, 256), 256, 0, ctx->stream>>>(c.n1, part, c.VH);
  TCSCF_LAUNCH(ctx);
  return TCSCF_OK;
}
}  // namespace

// Work items of one persistent launch, weighed by their r2 blocks (a symmetric instance's tiles start at
// their diagonal, so their items shrink with the tile index), sorted with the most blocks first and put
// in snake order over rounds of `grid` items: the kernel deals item i to CTA i % grid, so round r goes to
// CTAs 0, 1, ... when r is even and in reverse when r is odd, and every CTA gets about the same number
// of blocks (Kr symmetric build: the busiest CTA 0.2 % above the mean, against 4.7 % for tiles in order).
// The order changes no result: every item writes its own rows of its own split.
void dealItems(std::vector<int4> & items, int grid)
{
  std::stable_sort(items.begin(), items.end(), [](int4 const & a, int4 const & b) { return a.w > b.w; });
  size_t const g = size_t(std::max(grid, 1));
  for (size_t r0 = 0; r0 < items.size(); r0 += g)
    if ((r0 / g) % 2 == 1) std::reverse(items.begin() + int64_t(r0), items.begin() + int64_t(std::min(items.size(), r0 + g)));
}

// the work items (instance k, tile, split, r2 blocks) of one prepared contraction
void appendItems(std::vector<int4> & items, int k, tc::Instance const & I)
{
  for (int t = 0; t < I.nTiles; ++t)
    for (int sp = 0; sp < I.nSplit; ++sp) {
      int jb, je;
      tc::itemBlocks(I, t, sp, jb, je);
      items.push_back(make_int4(k, t, sp, je - jb));
    }
}

extern "C" int tcscf_schedule_items(int64_t n1, int64_t n2, int sym, int nsplit, int grid, int * items, int capacity, int * count)
{
  if (n1 <= 0 || n2 <= 0 || nsplit <= 0 || grid <= 0 || !count || capacity < 0 || (capacity > 0 && !items)) return TCSCF_ERR_INVALID_ARGUMENT;
  if (n1 > (int64_t(1) << 36) || n2 > (int64_t(1) << 36)) return TCSCF_ERR_INVALID_ARGUMENT;   // tile and block counts stay int
  tc::Instance I{};
  I.nTiles = int((n1 + tc::BM - 1) / tc::BM);
  I.nBlocks = int((n2 + tc::BK - 1) / tc::BK);
  I.blocksPerSplit = (I.nBlocks + nsplit - 1) / nsplit;
  I.nSplit = (I.nBlocks + I.blocksPerSplit - 1) / I.blocksPerSplit;
  I.sym = sym != 0;
  std::vector<int4> v;
  appendItems(v, 0, I);
  dealItems(v, std::min(grid, int(v.size())));
  int const n = std::min<int>(capacity, int(v.size()));
  for (int i = 0; i < n; ++i) {
    items[3 * i] = v[size_t(i)].y;
    items[3 * i + 1] = v[size_t(i)].z;
    items[3 * i + 2] = v[size_t(i)].w;
  }
  *count = int(v.size());
  return TCSCF_OK;
}

int tensorRun(tcscf_ctx * ctx, TensorPrep * const * preps, int count, bool recordStart)
{
  int const sms = smCount();
  // instance table and tensor maps in device memory (maps 64-byte aligned), then the work items
  size_t const instBytes = align256(sizeof(tc::Instance) * count);
  size_t const mapBytes = align256(sizeof(CUtensorMap) * tc::kMapsPerInstance * count);
  size_t itemsTotal = 0;
  for (int k = 0; k < count; ++k) itemsTotal += size_t(preps[k]->inst.nTiles) * preps[k]->inst.nSplit;
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, "flash_tc_table", instBytes + mapBytes + align256(sizeof(int4) * itemsTotal) + 256, &p));
  auto * dInst = static_cast<tc::Instance *>(p);
  auto * dMaps = reinterpret_cast<CUtensorMap *>(static_cast<char *>(p) + instBytes);
  auto * dItems = reinterpret_cast<int4 *>(static_cast<char *>(p) + instBytes + mapBytes);
  int * dStatus = reinterpret_cast<int *>(static_cast<char *>(p) + instBytes + mapBytes + align256(sizeof(int4) * itemsTotal));
  std::vector<tc::Instance> hInst(count);
  std::vector<CUtensorMap> hMaps(size_t(count) * tc::kMapsPerInstance);
  for (int k = 0; k < count; ++k) {
    hInst[k] = preps[k]->inst;
    hInst[k].maps = dMaps + size_t(k) * tc::kMapsPerInstance;
    for (int m = 0; m < tc::kMapsPerInstance; ++m) hMaps[size_t(k) * tc::kMapsPerInstance + m] = preps[k]->maps[m];
  }
  TCSCF_CUDA(ctx, cudaMemcpyAsync(dInst, hInst.data(), sizeof(tc::Instance) * count, cudaMemcpyHostToDevice, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemcpyAsync(dMaps, hMaps.data(), sizeof(CUtensorMap) * hMaps.size(), cudaMemcpyHostToDevice, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemsetAsync(dStatus, 0, sizeof(int), ctx->stream));

  // one persistent launch per tile class; within it, the work items dealt by dealItems
  struct Launch {
    int NB, RP, XS, NS, grid;
    tc::Params P;
  };
  std::vector<Launch> launches;
  size_t offset = 0;
  if (recordStart) cudaEventRecord(ctx->ev[2], ctx->stream);
  for (auto const & cl : kClasses) {
    int const NB = cl[0], RP = cl[1], XS = cl[2], NS = cl[3];
    std::vector<int4> items;
    for (int k = 0; k < count; ++k) {
      if (preps[k]->NB != NB || preps[k]->RP != RP || preps[k]->XS != XS || preps[k]->NS != NS) continue;
      appendItems(items, k, preps[k]->inst);
    }
    if (items.empty()) continue;
    int const grid = std::min(int(items.size()), sms);
    dealItems(items, grid);
    TCSCF_CUDA(ctx, cudaMemcpyAsync(dItems + offset, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice, ctx->stream));
    tc::Params P{};
    P.nItems = int(items.size());
    P.items = dItems + offset;
    P.inst = dInst;
    P.status = dStatus;
    launches.push_back({NB, RP, XS, NS, grid, P});
    offset += items.size();
  }
  if (count == 1) {
    for (auto const & l : launches) TCSCF_TRY(launchClass(ctx, l.NB, l.RP, l.XS, l.NS, l.P, l.grid));
  } else {
    // A batch runs as a CUDA graph of its persistent launches, captured once per launch sequence and
    // replayed while the sequence repeats (every SCF iteration of the same instances): the instance
    // table, tensor maps and work items the kernels read are refreshed above, before the replay.
    std::vector<uint64_t> key;
    for (auto const & l : launches) {
      key.insert(key.end(), {uint64_t(l.NB), uint64_t(l.RP), uint64_t(l.XS), uint64_t(l.NS), uint64_t(l.grid), uint64_t(l.P.nItems),
                             uint64_t(reinterpret_cast<uintptr_t>(l.P.items)), uint64_t(reinterpret_cast<uintptr_t>(l.P.inst)),
                             uint64_t(reinterpret_cast<uintptr_t>(l.P.status))});
    }
    if (!ctx->tensorGraph || ctx->tensorGraphKey != key) {
      if (ctx->tensorGraph) {
        cudaGraphExecDestroy(ctx->tensorGraph);
        ctx->tensorGraph = nullptr;
      }
      TCSCF_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
      int lst = TCSCF_OK;
      for (auto const & l : launches)
        if (lst == TCSCF_OK) lst = launchClass(ctx, l.NB, l.RP, l.XS, l.NS, l.P, l.grid);
      cudaGraph_t graph = nullptr;
      cudaError_t const ce = cudaStreamEndCapture(ctx->stream, &graph);
      TCSCF_TRY(lst);
      TCSCF_CHECK(ctx, ce == cudaSuccess && graph, TCSCF_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
      cudaError_t const ie = cudaGraphInstantiate(&ctx->tensorGraph, graph, 0);
      cudaGraphDestroy(graph);
      TCSCF_CHECK(ctx, ie == cudaSuccess, TCSCF_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
      ctx->tensorGraphKey = key;
      ++ctx->graphCaptures;
    } else {
      ++ctx->graphReplays;
      ctx->launchCount += int(launches.size());
    }
    TCSCF_CUDA(ctx, cudaGraphLaunch(ctx->tensorGraph, ctx->stream));
  }
  cudaEventRecord(ctx->ev[3], ctx->stream);
  int st = 0;
  TCSCF_CUDA(ctx, cudaMemcpyAsync(&st, dStatus, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (st != 0) return fail(ctx, TCSCF_ERR_TIMEOUT, "tensor-core contraction: bounded wait expired (code " + std::to_string(st) + ")");
  std::vector<tc::CoulombLowerJob> jobs;
  std::vector<int2> lowerTiles;
  for (int k = 0; k < count; ++k) {
    tc::Instance const & I = preps[k]->inst;
    Contraction const & c = preps[k]->c;
    if (I.nSplit > 1) {
      int64_t const n = int64_t(c.n1) * c.ncol;
      TCSCF_TRY(sumSplitsLaunch(ctx, n, I.nSplit, int64_t(c.n1) * c.ldt, I.T, c.T, c.n1, c.ncol, c.ldt, c.ldt));
      if (c.VH) TCSCF_TRY(sumSplitsLaunch(ctx, c.n1, I.nSplit, c.n1, I.VH, c.VH, c.n1, 1, 1, 1));
    }
    if (count == 1) {
      if (hasLowerRows(I, c)) {
        void * q = nullptr;
        TCSCF_TRY(scratch(ctx, "coulomb_lower_partials", lowerPartBytes(I.nTiles - 1), &q));
        TCSCF_TRY(coulombLower(ctx, I, c, static_cast<double *>(q)));
      }
    } else if (hasLowerRows(I, c)) {
      for (int t = 1; t < I.nTiles; ++t) lowerTiles.push_back(make_int2(int(jobs.size()), t));
      jobs.push_back({I.r1xyz, I.r2pairs, c.VH, c.n1});
    }
  }
  if (!lowerTiles.empty()) {
    // the lower Coulomb rows of all symmetric instances in one launch, the tiles with the most pairs first
    std::stable_sort(lowerTiles.begin(), lowerTiles.end(), [](int2 const & a, int2 const & b) { return a.y > b.y; });
    void * q = nullptr;
    size_t const jobBytes = align256(sizeof(tc::CoulombLowerJob) * jobs.size()), tileBytes = align256(sizeof(int2) * lowerTiles.size());
    TCSCF_TRY(scratch(ctx, "coulomb_lower_jobs", jobBytes + tileBytes + lowerPartBytes(int64_t(lowerTiles.size())) + 256, &q));
    auto * dJobs = static_cast<tc::CoulombLowerJob *>(q);
    auto * dTiles = reinterpret_cast<int2 *>(static_cast<char *>(q) + jobBytes);
    auto * dPart = reinterpret_cast<double *>(static_cast<char *>(q) + jobBytes + tileBytes);
    TCSCF_CUDA(ctx, cudaMemcpyAsync(dJobs, jobs.data(), sizeof(tc::CoulombLowerJob) * jobs.size(), cudaMemcpyHostToDevice, ctx->stream));
    TCSCF_CUDA(ctx, cudaMemcpyAsync(dTiles, lowerTiles.data(), sizeof(int2) * lowerTiles.size(), cudaMemcpyHostToDevice, ctx->stream));
    tc::kCoulombLowerBatch<<<unsigned(lowerTiles.size() * tc::kLowerChunks), tc::BM / 2, 0, ctx->stream>>>(dJobs, dTiles, dPart);
    TCSCF_LAUNCH(ctx);
    tc::kCoulombLowerBatchSum<<<unsigned(lowerTiles.size()), tc::BM, 0, ctx->stream>>>(dJobs, dTiles, dPart);
    TCSCF_LAUNCH(ctx);
    TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));   // the host lists are consumed before they go out of scope
  }
  return TCSCF_OK;
}

int tensorPlanUpload(tcscf_ctx * ctx, TensorPrep & tp, char const * scratchName, TensorPlan & plan)
{
  std::vector<int4> items;
  appendItems(items, 0, tp.inst);
  int const grid = std::min(int(items.size()), smCount());
  dealItems(items, grid);
  size_t const instBytes = align256(sizeof(tc::Instance));
  size_t const mapBytes = align256(sizeof(CUtensorMap) * tc::kMapsPerInstance);
  size_t const itemBytes = align256(sizeof(int4) * items.size());
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, scratchName, instBytes + mapBytes + itemBytes + 256, &p));
  auto * dInst = static_cast<tc::Instance *>(p);
  auto * dMaps = reinterpret_cast<CUtensorMap *>(static_cast<char *>(p) + instBytes);
  auto * dItems = reinterpret_cast<int4 *>(static_cast<char *>(p) + instBytes + mapBytes);
  int * dStatus = reinterpret_cast<int *>(static_cast<char *>(p) + instBytes + mapBytes + itemBytes);
  tc::Instance hInst = tp.inst;
  hInst.maps = dMaps;
  TCSCF_CUDA(ctx, cudaMemcpyAsync(dInst, &hInst, sizeof(tc::Instance), cudaMemcpyHostToDevice, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemcpyAsync(dMaps, tp.maps, sizeof(CUtensorMap) * tc::kMapsPerInstance, cudaMemcpyHostToDevice, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemcpyAsync(dItems, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemsetAsync(dStatus, 0, sizeof(int), ctx->stream));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));   // the host copies are consumed before they go out of scope
  plan.NB = tp.NB; plan.RP = tp.RP; plan.XS = tp.XS; plan.NS = tp.NS;
  plan.nItems = int(items.size());
  plan.grid = grid;
  plan.items = dItems;
  plan.inst = dInst;
  plan.status = dStatus;
  plan.prep = &tp;
  plan.lowerPart = nullptr;
  if (hasLowerRows(tp.inst, tp.c)) {
    // the lower rows' chunk partials, allocated here because the launches may be captured in a graph
    void * q = nullptr;
    TCSCF_TRY(scratch(ctx, (std::string(scratchName) + "_lower").c_str(), lowerPartBytes(tp.inst.nTiles - 1), &q));
    plan.lowerPart = static_cast<double *>(q);
  }
  return TCSCF_OK;
}

int tensorPlanLaunch(tcscf_ctx * ctx, TensorPlan const & plan)
{
  tc::Params P{};
  P.nItems = plan.nItems;
  P.items = static_cast<int4 const *>(plan.items);
  P.inst = static_cast<tc::Instance const *>(plan.inst);
  P.status = plan.status;
  TCSCF_TRY(launchClass(ctx, plan.NB, plan.RP, plan.XS, plan.NS, P, plan.grid));
  tc::Instance const & I = plan.prep->inst;
  Contraction const & c = plan.prep->c;
  if (I.nSplit > 1) {
    int64_t const n = int64_t(c.n1) * c.ncol;
    TCSCF_TRY(sumSplitsLaunch(ctx, n, I.nSplit, int64_t(c.n1) * c.ldt, I.T, c.T, c.n1, c.ncol, c.ldt, c.ldt));
    if (c.VH) TCSCF_TRY(sumSplitsLaunch(ctx, c.n1, I.nSplit, c.n1, I.VH, c.VH, c.n1, 1, 1, 1));
  }
  return coulombLower(ctx, I, c, plan.lowerPart);
}

namespace {

// T[r][j] += A[r][j] for j < ncol (leading dimension ld)
__global__ void kAddTChunk(int64_t n1, int ncol, int ld, const double * A, double * T)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n1 * ncol; i += int64_t(gridDim.x) * blockDim.x) {
    int64_t const r = i / ncol;
    int const j = int(i % ncol);
    T[r * ld + j] += A[r * ld + j];
  }
}

int runTensorOnce(tcscf_ctx * ctx, Contraction const & c, int precision, bool recordStart)
{
  std::string why;
  if (!tensorPathAvailable(c, precision, &why)) return fail(ctx, TCSCF_ERR_UNSUPPORTED, why);
  size_t const bytes = tensorArenaBytes(c, precision);
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, "flash_tc_ops", bytes, &p));
  TensorPrep tp;
  TCSCF_TRY(tensorPrepare(ctx, c, precision, p, bytes, tp));
  TensorPrep * one = &tp;
  return tensorRun(ctx, &one, 1, recordStart);
}

// Times every candidate split of this contraction (operand packing, the persistent launch and the
// split sums, between two events on the context stream; the first candidate, the default rule, runs
// once untimed before) and returns the fastest.  Each run writes the contraction's outputs in full,
// so the caller's final run leaves them as an untuned build would, up to the order of the r2 sums.
// Candidate tile classes of a split-BF16 launch besides the default rule's (same results bit for bit:
// every column of T is computed alike whatever the tile width and stage count): for a 64-column tile
// with rank padding 32 and 24-bit X, two TMA stages instead of three and the 128-column tile.
std::vector<std::pair<int, int>> classCandidates(Contraction const & c, int precision)
{
  Shape const sh = shapeOf(c, smCount(), precision);
  std::vector<std::pair<int, int>> out{{0, 0}};   // (tileNB, stages) = the rule
  if (precision == TCSCF_PREC_BF16X3 && sh.NB == 64 && sh.RP == 32 && sh.XS == 3) {
    out.push_back({64, 2});
    out.push_back({128, 0});
  }
  return out;
}

// Times a candidate schedule (operand packing, the persistent launch and the split sums, between two
// events on the context stream, after one untimed run).
int timeSchedule(tcscf_ctx * ctx, Contraction const & ck, int precision, float * ms)
{
  for (auto & e : ctx->tuneEv)
    if (!e) TCSCF_CUDA(ctx, cudaEventCreate(&e));
  TCSCF_TRY(runTensorOnce(ctx, ck, precision, false));
  TCSCF_CUDA(ctx, cudaEventRecord(ctx->tuneEv[0], ctx->stream));
  TCSCF_TRY(runTensorOnce(ctx, ck, precision, false));
  TCSCF_CUDA(ctx, cudaEventRecord(ctx->tuneEv[1], ctx->stream));
  TCSCF_CUDA(ctx, cudaEventSynchronize(ctx->tuneEv[1]));
  TCSCF_CUDA(ctx, cudaEventElapsedTime(ms, ctx->tuneEv[0], ctx->tuneEv[1]));
  ++ctx->tuneMeasurements;
  return TCSCF_OK;
}

// The schedule of one contraction shape: first the tile class (at the default split), then the r2
// split (with that class); returns {split, tileNB, stages}.  Each run writes the contraction's outputs
// in full, so the caller's final run leaves them as an untuned build would, up to the order of the r2
// block sums.
int tuneSchedule(tcscf_ctx * ctx, Contraction const & c, int precision, std::array<int, 3> * best)
{
  std::vector<int> const cand = splitCandidates(c.n1, c.n2, smCount());
  std::vector<std::pair<int, int>> const classes = classCandidates(c, precision);
  *best = {cand[0], 0, 0};
  float bestMs = 0;
  for (size_t i = 0; i < classes.size(); ++i) {
    Contraction ck = c;
    ck.nSplit = cand[0];
    ck.tileNB = classes[i].first;
    ck.stages = classes[i].second;
    if (ck.tileNB > 0 && ck.tileNB != shapeOf(c, smCount(), precision).NB) ck.vtPacked = nullptr;   // packed at the rule's width
    if (classes.size() == 1) break;
    float ms = 0;
    TCSCF_TRY(timeSchedule(ctx, ck, precision, &ms));
    if (i == 0 || ms < bestMs) { bestMs = ms; (*best)[1] = ck.tileNB; (*best)[2] = ck.stages; }
  }
  if (cand.size() == 1) return TCSCF_OK;
  for (size_t i = 0; i < cand.size(); ++i) {
    Contraction ck = c;
    ck.nSplit = cand[i];
    ck.tileNB = (*best)[1];
    ck.stages = (*best)[2];
    if (ck.tileNB > 0 && ck.tileNB != shapeOf(c, smCount(), precision).NB) ck.vtPacked = nullptr;
    float ms = 0;
    TCSCF_TRY(timeSchedule(ctx, ck, precision, &ms));
    if (i == 0 || ms < bestMs) { bestMs = ms; (*best)[0] = cand[i]; }
  }
  return TCSCF_OK;
}

int contractTensorOnce(tcscf_ctx * ctx, Contraction const & c, int precision, bool recordStart)
{
  if (!ctx->autotune || c.nSplit > 0) return runTensorOnce(ctx, c, precision, recordStart);
  std::string why;
  if (!tensorPathAvailable(c, precision, &why)) return fail(ctx, TCSCF_ERR_UNSUPPORTED, why);
  std::vector<int64_t> const key{c.n1, c.n2, c.ncol <= 64 ? 64 : 128, c.R <= 32 ? 32 : 64, precision, c.sym};
  auto it = ctx->tunedSplit.find(key);
  if (it == ctx->tunedSplit.end()) {
    std::array<int, 3> best{};
    TCSCF_TRY(tuneSchedule(ctx, c, precision, &best));
    it = ctx->tunedSplit.emplace(key, best).first;
  }
  Contraction ck = c;
  ck.nSplit = it->second[0];
  ck.tileNB = it->second[1];
  ck.stages = it->second[2];
  if (ck.tileNB > 0 && ck.tileNB != shapeOf(c, smCount(), precision).NB) ck.vtPacked = nullptr;
  return runTensorOnce(ctx, ck, precision, recordStart);
}

}  // namespace

int tensorRankLimit(Contraction const & c, int precision) { return precision == TCSCF_PREC_TF32 || c.ncol > 64 ? 32 : 64; }

int contractTensor(tcscf_ctx * ctx, Contraction const & c, int precision)
{
  int const lim = tensorRankLimit(c, precision);
  if (c.R <= lim) {
    TCSCF_TRY(contractTensorOnce(ctx, c, precision, true));
    return nearCorrect(ctx, c);
  }
  // rho is linear in the density factor: a rank beyond what one launch's psi tiles hold (32 for TF32
  // or with nb > 64, 64 otherwise) is contracted in column chunks whose T add up (the Coulomb potential,
  // which does not depend on the factor, with the first); ev[2] / ev[3] span all chunks
  double * tmp = nullptr;
  TCSCF_TRY(scratch(ctx, "flash_tc_rank_chunk", sizeof(double) * size_t(c.n1) * c.ldt, reinterpret_cast<void **>(&tmp)));
  for (int r0 = 0; r0 < c.R; r0 += lim) {
    Contraction ck = c;
    ck.R = std::min(lim, c.R - r0);
    ck.psi1 = c.psi1 + r0;
    ck.psi2 = c.psi2 + r0;
    if (r0 > 0) { ck.coul = nullptr; ck.VH = nullptr; ck.T = tmp; }
    ck.near = nullptr;   // the near-pair correction runs once with the whole factor
    TCSCF_TRY(contractTensorOnce(ctx, ck, precision, r0 == 0));
    if (r0 > 0) {
      kAddTChunk<<<gridBlocks(c.n1 * c.ncol, 256), 256, 0, ctx->stream>>>(c.n1, c.ncol, c.ldt, tmp, c.T);
      TCSCF_LAUNCH(ctx);
    }
  }
  cudaEventRecord(ctx->ev[3], ctx->stream);
  return nearCorrect(ctx, c);
}

namespace tc {

// The failure path of the bounded waits: lane 0 of one warp waits through waitBarLimit on an
// mbarrier that nothing arrives at (its phase 0 never completes); the wait gives up after limitNs,
// records code 90 in the status word and the kernel returns.
__global__ void kBoundedWaitSelfTest(unsigned long long limitNs, int * status)
{
  __shared__ uint64_t bar;
  __shared__ int abortWord;
  if (threadIdx.x == 0) {
    mbarInit(&bar, 1);
    abortWord = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  if (threadIdx.x == 0) waitBarLimit(&bar, 0, &abortWord, status, 90, limitNs);
  __syncwarp();
}

}  // namespace tc

int boundedWaitSelfTest(tcscf_ctx * ctx, double limitMs)
{
  TCSCF_CHECK(ctx, limitMs >= 1.0 && limitMs <= 1000.0, TCSCF_ERR_INVALID_ARGUMENT, "limit_ms must be in [1, 1000]");
  int * dStatus = nullptr;
  TCSCF_TRY(scratch(ctx, "wait_selftest", sizeof(int), reinterpret_cast<void **>(&dStatus)));
  TCSCF_CUDA(ctx, cudaMemsetAsync(dStatus, 0, sizeof(int), ctx->stream));
  tc::kBoundedWaitSelfTest<<<1, 32, 0, ctx->stream>>>((unsigned long long)(limitMs * 1e6), dStatus);
  TCSCF_LAUNCH(ctx);
  int st = 0;
  TCSCF_CUDA(ctx, cudaMemcpyAsync(&st, dStatus, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (st != 0) return fail(ctx, TCSCF_ERR_TIMEOUT, "bounded wait expired (code " + std::to_string(st) + ")");
  return TCSCF_OK;
}

}  // namespace tcscf
