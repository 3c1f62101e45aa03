// tcgen05 (sm_100a) precompute form of the r12 contraction, computeF / computeV
// (HartreeFock.hpp:23-229), in split-BF16 precision with exact tensor-core block accumulation:
//
//   T[r1][p] = sum_r2 g(r1, r2) Vp[r2][p],   Vp[r2][p] = w2 phi_k(r2) phi_l(r2)  (basis pairs k <= l)
//
// the reference's precomputeIntegrand (the stored N1 x N2 kernel matrix) followed by computeF's sum,
// with the kernel matrix generated tile by tile and never stored.  g is one of
//   kind 0   1 / r12                                                (HartreeFockTest.cpp:248-253)
//   kind 1   2 / r12 - |grad_1 u(r1,r2)|^2 - |grad_1 u(r2,r1)|^2     (TC scalar, :276-296)
//   kind 2   component `comp` of grad_1 u(r1, r2)                    (:300-318)
// for a Jastrow factor of r12 alone, u = sum_k c_k (r12 / (r12 + a12))^i_k (jastrowFunctions.hpp:9-115
// with every S[k] = (i_k, 0, 0), the form the reference's TC driver uses, HartreeFockTest.cpp:351-360):
// then grad_1 u(r1,r2) = u'(r12) (r1 - r2) / r12 = -grad_1 u(r2,r1), so the TC scalar kernel is
// 2 / r12 - 2 u'^2, with u'(r12) = t^2 P(r12 t), t = 1 / (r12 + a12), P(z) = sum_n p_n z^n and
// p_n = a12 sum_{k: i_k = n + 1} i_k c_k.  An exactly coincident pair (and a separation whose square is
// below nearThreshold, the FP32 resolution of r1) contributes 0 here; the near-pair correction adds the
// pairs that are not exactly coincident back in FP64, so every kind follows the FP64 path's rule.
//
// The kernel values are generated in FP32 from FP32 coordinates (rsqrt and reciprocal estimates each
// refined by one Newton step) and enter the tensor cores as 24-bit fixed-point BF16 slices (four
// slices h, m, l/256, m/256 with a power-of-two scale per (r1 row, r2 block of 64)); Vp enters as
// three 24-bit slices with a scale per (r2 block, column), packed once per call.  Per block the
// hi x hi products accumulate exactly in one TMEM accumulator and the cross products in a second (the
// split-BF16 scheme of the direct Fock build, flash_tc.cu), and each finished block is added with its
// scales into per-thread double-float accumulators.  T's columns run in chunks of NB (64 or 128):
// work items are (r1 tile of 128, column chunk, r2 split); the T accumulators are double-buffered in
// TMEM so the MMAs of block g overlap the flush of block g - 1.
//
// Warp roles (384 threads, one persistent CTA per SM): warp 0 TMA producer (Vp slices by TMA, r2
// coordinates and column scales by 1-D bulk copies; no multicast), warp 1 MMA issuer and TMEM
// allocator, warps 2-3 idle, warps 4-11 compute (TMEM lane quarter w % 4, r2 / column half (w-4)/4).
// Every mbarrier wait is bounded; on expiry the kernel records a status code, drains its own copies
// and MMAs with bounded waits, frees TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>

#include "tc_device.cuh"

namespace tcscf {
namespace tc {
namespace {

constexpr int kPairStages = 3;
// X tile buffers: two where shared memory allows (GEMM of block g - 1 overlaps the writing of block g)
__host__ __device__ constexpr int pairXBuffers(int NB) { return NB == 128 ? 1 : 2; }
constexpr int kPairXSlices = 4;   // h, m, l/256, m/256
constexpr int kMaxPoly = 8;
constexpr int kMinExp = -100;     // rows whose block maximum is below 2^-100 are sliced against 2^-100

struct PairParams {
  int nTiles, nChunks, nSplit, blocksPerSplit, nBlocks;
  int n1, ncol, ldt;
  int kind, comp, same, npoly;
  float a12;
  float poly[kMaxPoly];             // p_n of u'(r12) = t^2 sum_n p_n (r12 t)^n
  const float4 * r1xyz;             // [n1pad] {x, y, z, nearThreshold}
  const float4 * r2pairs;           // [n2pad] pair layout {x0,x1,y0,y1}{z0,z1,0,0}
  const float * cinv;               // [nBlocks][NBtot] inverse column scales of Vp
  int NBtot;
  double * T;                       // [nSplit][n1][ldt]
  int64_t tStride;
  int * status;
};

template <int NB>
struct __align__(1024) PairSmem {
  static constexpr int NSTAGE = kPairStages;
  static constexpr int XBUF = pairXBuffers(NB);
  uint8_t v[NSTAGE][3][NB * BK * 2];               // Vp block h / m / l/256: SW128 K-major [NB rows][64]
  uint8_t x[XBUF][kPairXSlices][BM * BK * 2];      // X tile slices: SW128 K-major [128 rows][64]
  float4 coords[NSTAGE][BK];                       // r2 block as 32 pairs
  float cinv[NSTAGE][NB];                          // inverse column scales of the block's chunk columns
  float cinvT[NCW][2][NB / 2];                     // each compute warp's columns' scales, by block parity
  float rowmax[2][2][BM];                          // [block parity][r2 half][row]
  uint64_t full[NSTAGE], empty[NSTAGE];
  uint64_t xfull[XBUF], xfree[XBUF];
  uint64_t tfull[2], tfree[2];                     // T accumulator buffers
  uint64_t rmax[2][4];
  uint64_t done;
  uint32_t tmemBase;
  int abort;
};

__device__ __forceinline__ uint64_t f2rcp(uint64_t s)
{
  // reciprocal estimates refined by one Newton step t <- t + t (1 - s t)
  float a, b;
  f2unpack(s, a, b);
  float ra, rb;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(ra) : "f"(a));
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rb) : "f"(b));
  uint64_t const t = f2pack(ra, rb);
  uint64_t const e = f2fma(f2mul(s, f2pack(-1.0f, -1.0f)), t, f2pack(1.0f, 1.0f));
  return f2fma(t, e, t);
}

// Kernel values of two pairs (packed): d = r1 - r2 components, r2sq = |d|^2.
template <int KIND>
__device__ __forceinline__ uint64_t pairKernel(PairParams const & P, uint64_t dx, uint64_t dy, uint64_t dz, uint64_t r2sq, float thr)
{
  float r2a, r2b;
  f2unpack(r2sq, r2a, r2b);
  uint64_t y = f2pack(rsqrtApprox(r2a), rsqrtApprox(r2b));
  // one Newton step on the estimate: y += (-y/2) (r2 y^2 - 1)
  uint64_t const em = f2fma(f2mul(r2sq, y), y, f2pack(-1.0f, -1.0f));
  y = f2fma(f2mul(y, f2pack(-0.5f, -0.5f)), em, y);
  uint64_t g;
  if constexpr (KIND == 0) {
    g = y;
  } else {
    uint64_t const r12 = f2mul(r2sq, y);
    uint64_t const t = f2rcp(f2add(r12, f2pack(P.a12, P.a12)));
    uint64_t const z = f2mul(r12, t);
    uint64_t poly = f2pack(P.poly[P.npoly - 1], P.poly[P.npoly - 1]);
    for (int n = P.npoly - 2; n >= 0; --n) poly = f2fma(poly, z, f2pack(P.poly[n], P.poly[n]));
    uint64_t const up = f2mul(f2mul(t, t), poly);   // u'(r12)
    if constexpr (KIND == 1) {
      g = f2fma(f2mul(up, up), f2pack(-2.0f, -2.0f), f2add(y, y));
    } else {
      uint64_t const d = P.comp == 0 ? dx : (P.comp == 1 ? dy : dz);
      g = f2mul(f2mul(up, y), d);
    }
  }
  float ga, gb;
  f2unpack(g, ga, gb);
  ga = r2a >= thr ? ga : 0.0f;
  gb = r2b >= thr ? gb : 0.0f;
  return f2pack(ga, gb);
}

__device__ __forceinline__ uint32_t bf16PairRnP(uint64_t ab)
{
  float a, b;
  f2unpack(ab, a, b);
  __nv_bfloat162 const h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t const *>(&h);
}
__device__ __forceinline__ uint32_t bf16PairExactP(uint64_t ab)
{
  float a, b;
  f2unpack(ab, a, b);
  return __byte_perm(__float_as_uint(a), __float_as_uint(b), 0x7632);
}

__host__ __device__ constexpr uint32_t idescBf16(int M, int N)
{
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void mmaBf16P(uint32_t tmemD, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmemD),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void decodePairItem(PairParams const & P, int item, int & tile, int & chunk, int & split)
{
  int const per = P.nChunks * P.nSplit;
  tile = item / per;
  int const r = item % per;
  chunk = r / P.nSplit;
  split = r % P.nSplit;
}

// Adds T buffer tb of block f (this thread's row and NB/2 columns) with the block's scales into the
// double-float accumulators by Fast2Sum and hands the buffer back to the MMA issuer.
template <int NB, class SmemT>
__device__ __forceinline__ bool flushPairBlock(SmemT & S, uint32_t taddr, uint32_t f, int cw, float fac, uint64_t (&hi)[NB / 4],
                                               uint64_t (&lo)[NB / 4], int lane, volatile int * abortFlag, int * status)
{
  int const tb = f & 1;
  if (!waitBar(&S.tfull[tb], (f >> 1) & 1, abortFlag, status, 131)) return false;
  fenceAfterSync();
  float const * cs = S.cinvT[cw][tb];
  uint64_t const k256 = f2pack(256.0f, 256.0f);
  uint64_t const ff = f2pack(fac, fac);
  uint32_t const base = taddr + uint32_t(tb * 2 * NB);
  constexpr int NQ = NB / 16;
  float hh[2][8], mm[2][8];
  tmemLoad8(base, hh[0]);
  tmemLoad8(base + NB, mm[0]);
  tmemWaitLoad8(hh[0], mm[0]);
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    int const cur = q & 1;
    if (q + 1 < NQ) {
      tmemLoad8(base + (q + 1) * 8, hh[cur ^ 1]);
      tmemLoad8(base + NB + (q + 1) * 8, mm[cur ^ 1]);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      float2 const c2 = *reinterpret_cast<float2 const *>(cs + q * 8 + 2 * i);
      uint64_t const x = f2mul(f2fma(f2pack(hh[cur][2 * i], hh[cur][2 * i + 1]), k256, f2pack(mm[cur][2 * i], mm[cur][2 * i + 1])),
                               f2mul(f2pack(c2.x, c2.y), ff));
      int const p = q * 4 + i;
      uint64_t const sum = f2add(hi[p], x);
      lo[p] = f2add(lo[p], f2sub(x, f2sub(sum, hi[p])));
      hi[p] = sum;
    }
    if (q + 1 < NQ) tmemWaitLoad8(hh[cur ^ 1], mm[cur ^ 1]);
  }
  fenceBeforeSync();
  __syncwarp();
  if (lane == 0) mbarArrive(&S.tfree[tb]);
  return true;
}

template <int NB, int KIND>
__global__ void __launch_bounds__(NTHREADS, 1)
    kPairTc(const __grid_constant__ PairParams P, const __grid_constant__ CUtensorMap mapH, const __grid_constant__ CUtensorMap mapM,
            const __grid_constant__ CUtensorMap mapL)
{
  extern __shared__ uint8_t smemRaw[];
  using SmemT = PairSmem<NB>;
  SmemT & S = *reinterpret_cast<SmemT *>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
  constexpr int NSTAGE = SmemT::NSTAGE;
  constexpr int XBUF = SmemT::XBUF;
  int const warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  volatile int * abortFlag = &S.abort;
  static_assert(4 * NB <= 512, "TMEM columns: two T buffers of two accumulators");
  constexpr uint32_t kStageBytes = 3 * NB * BK * 2 + BK * sizeof(float4) + NB * sizeof(float);
  int const nItems = P.nTiles * P.nChunks * P.nSplit;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NSTAGE; ++s) { mbarInit(&S.full[s], 1); mbarInit(&S.empty[s], 1 + NCW); }
    for (int b = 0; b < XBUF; ++b) { mbarInit(&S.xfull[b], NCW); mbarInit(&S.xfree[b], 1); }
    for (int b = 0; b < 2; ++b) {
      mbarInit(&S.tfull[b], 1); mbarInit(&S.tfree[b], NCW);
      for (int q = 0; q < 4; ++q) mbarInit(&S.rmax[b][q], 2);
    }
    mbarInit(&S.done, 1);
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

  if (warp < 4) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kRegsProducer));
    if (warp == 0) {
      // ---------------------------------------------------------------- TMA producer
      if (lane == 0) {
        uint32_t issued = 0;
        bool ok = true;
        for (int item = blockIdx.x; item < nItems && ok; item += gridDim.x) {
          int tile, chunk, split;
          decodePairItem(P, item, tile, chunk, split);
          int const jb = split * P.blocksPerSplit;
          int const je = min(P.nBlocks, jb + P.blocksPerSplit);
          for (int j = jb; j < je; ++j) {
            uint32_t const q = issued++;
            int const s = q % NSTAGE;
            if (q >= uint32_t(NSTAGE) && !(ok = waitBar(&S.empty[s], ((q / NSTAGE) - 1) & 1, abortFlag, P.status, 112))) break;
            mbarArriveTx(&S.full[s], kStageBytes);
            tmaLoad2d(S.v[s][0], &mapH, j * BK, chunk * NB, &S.full[s]);
            tmaLoad2d(S.v[s][1], &mapM, j * BK, chunk * NB, &S.full[s]);
            tmaLoad2d(S.v[s][2], &mapL, j * BK, chunk * NB, &S.full[s]);
            bulkLoad(S.coords[s], P.r2pairs + int64_t(j) * BK, BK * sizeof(float4), &S.full[s]);
            bulkLoad(S.cinv[s], P.cinv + int64_t(j) * P.NBtot + chunk * NB, NB * sizeof(float), &S.full[s]);
          }
        }
        // drain: every issued copy lands before the CTA can exit (bounded)
        for (uint32_t q = issued > uint32_t(NSTAGE) ? issued - NSTAGE : 0; q < issued; ++q) {
          unsigned long long const t0 = globalTimer();
          while (!mbarTryWait(&S.full[q % NSTAGE], (q / NSTAGE) & 1) && globalTimer() - t0 < kWaitLimitNs) {}
        }
      }
    } else if (warp == 1) {
      // ---------------------------------------------------------------- MMA issuer
      if (lane == 0) {
        constexpr uint32_t idesc = idescBf16(BM, NB);
        constexpr uint32_t idescX2 = idescBf16(BM, 2 * NB);   // h x [h'; m']: adjacent slices, adjacent accumulators
        uint32_t g = 0;
        bool ok = true;
        for (int item = blockIdx.x; item < nItems && ok; item += gridDim.x) {
          int tile, chunk, split;
          decodePairItem(P, item, tile, chunk, split);
          int const jb = split * P.blocksPerSplit;
          int const je = min(P.nBlocks, jb + P.blocksPerSplit);
          for (int j = jb; j < je && ok; ++j, ++g) {
            int const s = g % NSTAGE, tb = g & 1, xb = g % XBUF;
            if (!(ok = waitBar(&S.full[s], (g / NSTAGE) & 1, abortFlag, P.status, 121))) break;
            if (g >= 2 && !(ok = waitBar(&S.tfree[tb], ((g >> 1) - 1) & 1, abortFlag, P.status, 122))) break;
            if (!(ok = waitBar(&S.xfull[xb], (g / XBUF) & 1, abortFlag, P.status, 123))) break;
            fenceAfterSync();
            uint32_t const dA = tmem + uint32_t(tb * 2 * NB), dB = dA + NB;
            uint32_t aX[kPairXSlices];
#pragma unroll
            for (int k = 0; k < kPairXSlices; ++k) aX[k] = smemAddr(S.x[xb][k]);
            uint32_t const bV[3] = {smemAddr(S.v[s][0]), smemAddr(S.v[s][1]), smemAddr(S.v[s][2])};
            auto dxa = [&](int sl, int k) { return smemDesc(aX[sl] + 32 * k, 1024, 2); };
            auto dvb = [&](int sl, int k) { return smemDesc(bV[sl] + 32 * k, 1024, 2); };
#pragma unroll
            for (int k = 0; k < BK / 16; ++k) {
              uint32_t const acc = k > 0 ? 1u : 0u;
              mmaBf16P(dA, dxa(0, k), dvb(0, k), idescX2, acc);   // A += hX hV, B += hX mV
              mmaBf16P(dB, dxa(1, k), dvb(0, k), idesc, 1);       // B += mX hV
              mmaBf16P(dB, dxa(0, k), dvb(2, k), idesc, 1);       // B += hX lV/256
              mmaBf16P(dB, dxa(3, k), dvb(1, k), idesc, 1);       // B += m/256 X mV
              mmaBf16P(dB, dxa(2, k), dvb(0, k), idesc, 1);       // B += l/256 X hV
            }
            mmaCommit(&S.xfree[xb]);
            mmaCommit(&S.empty[s]);
            mmaCommit(&S.tfull[tb]);
          }
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
    uint32_t const tAddr = tmem + laneBase + uint32_t(half * (NB / 2));
    uint32_t g = 0;
    bool ok = true;
    uint64_t ahi[NB / 4], alo[NB / 4];
    uint64_t const kInv256 = f2pack(1.0f / 256.0f, 1.0f / 256.0f), kM256 = f2pack(-256.0f, -256.0f);
    uint64_t const kMagic = f2pack(12582912.0f, 12582912.0f);   // 1.5 * 2^23: adding it rounds |x| < 2^22 to an integer
    uint64_t const kInv65536 = f2pack(1.0f / 65536.0f, 1.0f / 65536.0f), kM65536 = f2pack(-65536.0f, -65536.0f);
    for (int item = blockIdx.x; item < nItems && ok; item += gridDim.x) {
      int tile, chunk, split;
      decodePairItem(P, item, tile, chunk, split);
      int const jb = split * P.blocksPerSplit;
      int const je = min(P.nBlocks, jb + P.blocksPerSplit);
      int const nblk = je - jb;
      int const r1 = tile * BM + row;
      float4 const p1 = P.r1xyz[r1];
#pragma unroll
      for (int c = 0; c < NB / 4; ++c) { ahi[c] = 0; alo[c] = 0; }
      float pendingFac = 0.0f;
      bool pending = false;
      uint64_t const p1x = f2pack(p1.x, p1.x), p1y = f2pack(p1.y, p1.y), p1z = f2pack(p1.z, p1.z);
      for (int jj = 0; jj < nblk && ok; ++jj, ++g) {
        int const s = g % NSTAGE, b = g & 1, xb = g % XBUF;
        if (!(ok = waitBar(&S.full[s], (g / NSTAGE) & 1, abortFlag, P.status, 132))) break;
        // this warp's column scales, kept for the flush of block g after the stage is released
        for (int c = lane; c < NB / 2; c += 32) S.cinvT[cw][b][c] = S.cinv[s][half * (NB / 2) + c];
        float4 const * cc = S.coords[s] + half * 32;
        uint64_t xv[16];
#pragma unroll
        for (int pr = 0; pr < 16; ++pr) {
          float4 const qa = cc[2 * pr], qb = cc[2 * pr + 1];
          uint64_t const dx = f2sub(p1x, f2pack(qa.x, qa.y));
          uint64_t const dy = f2sub(p1y, f2pack(qa.z, qa.w));
          uint64_t const dz = f2sub(p1z, f2pack(qb.x, qb.y));
          uint64_t const r2 = f2fma(dx, dx, f2fma(dy, dy, f2mul(dz, dz)));
          xv[pr] = pairKernel<KIND>(P, dx, dy, dz, r2, p1.w);
        }
        // row maximum of |X| over the block's 64 r2 points: this warp's 32 and the other half's
        float mx = 0.0f;
#pragma unroll
        for (int pr = 0; pr < 16; ++pr) {
          float xa, xb2;
          f2unpack(xv[pr], xa, xb2);
          mx = fmaxf(mx, fmaxf(fabsf(xa), fabsf(xb2)));
        }
        S.rowmax[b][half][row] = mx;
        __syncwarp();
        if (lane == 0) mbarArrive(&S.rmax[b][quarter]);
        if (!(ok = waitBar(&S.rmax[b][quarter], (g >> 1) & 1, abortFlag, P.status, 135))) break;
        mx = fmaxf(mx, S.rowmax[b][half ^ 1][row]);
        // scale bs = 2^(23 - E), E = floor(log2 mx) (clamped below): |X bs| < 2^24
        int const E = max(int((__float_as_uint(mx) >> 23) & 0xFF) - 127, kMinExp);
        float const bs = __uint_as_float(uint32_t(127 + 23 - E) << 23);
        // a block's sum_r2 X Vp = 2^24 (256 A + B) / (bs cs) = 2^(E+1) cinv (256 A + B)
        float const fac = __uint_as_float(uint32_t(127 + E + 1) << 23);
        if (g >= uint32_t(XBUF) && !(ok = waitBar(&S.xfree[xb], ((g / XBUF) - 1) & 1, abortFlag, P.status, 134))) break;
        uint64_t const bb = f2pack(bs, bs);
#pragma unroll
        for (int ch = 0; ch < 4; ++ch) {
          uint32_t const off = sw128(row, half * 4 + ch);
          // t = X bs = 65536 h + 256 m + l: h = rint(t / 65536), m = rint(r / 256), l = r - 256 m with
          // r = t - 65536 h; slices h, m, l/256 (rounded to nearest BF16: it feeds only the cross
          // accumulator), m/256
          uint32_t sh[4], sm[4], sl[4], sms[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            uint64_t const t = f2mul(xv[ch * 4 + e], bb);
            uint64_t const h = f2sub(f2fma(t, kInv65536, kMagic), kMagic);
            uint64_t const r = f2fma(h, kM65536, t);
            uint64_t const m = f2sub(f2fma(r, kInv256, kMagic), kMagic);
            sh[e] = bf16PairExactP(h);
            sm[e] = bf16PairExactP(m);
            sl[e] = bf16PairRnP(f2mul(f2fma(m, kM256, r), kInv256));
            sms[e] = bf16PairExactP(f2mul(m, kInv256));
          }
          *reinterpret_cast<uint4 *>(S.x[xb][0] + off) = make_uint4(sh[0], sh[1], sh[2], sh[3]);
          *reinterpret_cast<uint4 *>(S.x[xb][1] + off) = make_uint4(sm[0], sm[1], sm[2], sm[3]);
          *reinterpret_cast<uint4 *>(S.x[xb][2] + off) = make_uint4(sl[0], sl[1], sl[2], sl[3]);
          *reinterpret_cast<uint4 *>(S.x[xb][3] + off) = make_uint4(sms[0], sms[1], sms[2], sms[3]);
        }
        fenceProxyAsync();
        __syncwarp();
        if (lane == 0) { mbarArrive(&S.xfull[xb]); mbarArrive(&S.empty[s]); }
        if (pending && !(ok = flushPairBlock<NB>(S, tAddr, g - 1, cw, pendingFac, ahi, alo, lane, abortFlag, P.status))) break;
        pending = true;
        pendingFac = fac;
      }
      if (ok && pending) ok = flushPairBlock<NB>(S, tAddr, g - 1, cw, pendingFac, ahi, alo, lane, abortFlag, P.status);
      if (!ok) break;
      if (r1 < P.n1) {
        double * T = P.T + int64_t(split) * P.tStride + int64_t(r1) * P.ldt;
#pragma unroll
        for (int c = 0; c < NB / 2; ++c) {
          int const col = chunk * NB + half * (NB / 2) + c;
          float h0, h1, l0, l1;
          f2unpack(ahi[c / 2], h0, h1);
          f2unpack(alo[c / 2], l0, l1);
          if (col < P.ncol) T[col] = (c & 1) ? double(h1) + double(l1) : double(h0) + double(l0);
        }
      }
    }
    fenceBeforeSync();
    __syncthreads();
  }
}

template <int NB, int KIND>
int launchPairs(tcscf_ctx * ctx, PairParams const & P, CUtensorMap const (&maps)[3], int grid)
{
  size_t const smem = sizeof(PairSmem<NB>) + 1024;
  static_assert(sizeof(PairSmem<NB>) + 1024 <= 232448, "shared memory per CTA");
  TCSCF_CUDA(ctx, cudaFuncSetAttribute(kPairTc<NB, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  kPairTc<NB, KIND><<<grid, NTHREADS, smem, ctx->stream>>>(P, maps[0], maps[1], maps[2]);
  TCSCF_LAUNCH(ctx);
  return TCSCF_OK;
}

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

}  // namespace
}  // namespace tc

bool pairsTensorAvailable(Contraction const & c, int precision, std::string * why)
{
  auto no = [&](char const * m) { if (why) *why = m; return false; };
  if (precision != TCSCF_PREC_BF16X3) return no("the tensor-core precompute form runs in BF16X3");
  if (c.R != 0) return no("the tensor-core precompute form has rho == 1");
  if (c.kernel != TCSCF_K_INV_R12) {
    if (!c.jastrow) return no("TC kernels need the Jastrow parameters");
    for (int k = 0; k < c.jastrow->nterms; ++k) {
      if (c.jastrow->S[k][1] != 0 || c.jastrow->S[k][2] != 0)
        return no("the tensor-core TC kernels take a Jastrow factor of r12 alone (every S[k] = (i, 0, 0)); use FP64");
      if (c.jastrow->S[k][0] < 0 || c.jastrow->S[k][0] > tc::kMaxPoly) return no("Jastrow powers of r12 must be in 0..8 on the tensor path");
    }
    if (!(c.jastrow->a12 > 0)) return no("the Jastrow scale a12 must be positive");
  }
  if (c.ncol < 1) return no("no columns");
  if (!encodeTiled()) return no("cuTensorMapEncodeTiled unavailable");
  return true;
}

int contractPairsTensor(tcscf_ctx * ctx, Contraction const & c, int precision)
{
  std::string why;
  if (!pairsTensorAvailable(c, precision, &why)) return fail(ctx, TCSCF_ERR_UNSUPPORTED, why);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  int const NB = c.ncol <= 64 ? 64 : 128;
  int const nChunks = (c.ncol + NB - 1) / NB;
  int const NBtot = nChunks * NB;
  int64_t const n1pad = (c.n1 + tc::BM - 1) / tc::BM * tc::BM;
  int64_t const n2pad = (c.n2 + tc::BK - 1) / tc::BK * tc::BK;
  TCSCF_CHECK(ctx, n2pad / tc::BK < (int64_t(1) << 30) && n1pad / tc::BM < (int64_t(1) << 30), TCSCF_ERR_UNSUPPORTED, "grid too large");
  int const nTiles = int(n1pad / tc::BM), nBlocks = int(n2pad / tc::BK);
  // r2 split so that the work items fill about 16 waves of the SMs (deterministic split sums afterwards)
  int64_t const items = int64_t(nTiles) * nChunks;
  int nSplit = int(std::max<int64_t>(1, std::min<int64_t>((16 * int64_t(sms) + items - 1) / items, std::max(1, nBlocks / 8))));
  int const perSplit = (nBlocks + nSplit - 1) / nSplit;
  nSplit = (nBlocks + perSplit - 1) / perSplit;
  TCSCF_CHECK(ctx, items * nSplit < (int64_t(1) << 31), TCSCF_ERR_UNSUPPORTED, "too many work items");

  size_t const vtBytes = packedVtOperandBytes(NBtot, n2pad);
  size_t const partBytes = nSplit > 1 ? sizeof(double) * size_t(nSplit) * c.n1 * c.ldt : 0;
  size_t const bytes = tc::align256(vtBytes) + tc::align256(sizeof(float4) * n1pad) + tc::align256(sizeof(float4) * n2pad) +
                       tc::align256(partBytes) + 256 + 256;
  void * arena = nullptr;
  TCSCF_TRY(scratch(ctx, "flash_pairs", bytes, &arena));
  char * q = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(arena) + 255) & ~uintptr_t(255));
  auto take = [&](size_t n) { char * r = q; q += tc::align256(n); return r; };
  void * vt = take(vtBytes);
  auto * r1c = reinterpret_cast<float4 *>(take(sizeof(float4) * n1pad));
  auto * r2c = reinterpret_cast<float4 *>(take(sizeof(float4) * n2pad));
  double * part = partBytes ? reinterpret_cast<double *>(take(partBytes)) : nullptr;
  int * dStatus = reinterpret_cast<int *>(take(sizeof(int)));

  TCSCF_TRY(packVtOperand(ctx, c.n2, n2pad, c.ncol, NBtot, c.V, c.ldv, vt));
  TCSCF_TRY(packPointsFp32(ctx, c.n1, n1pad, c.p1, r1c));
  TCSCF_TRY(packPointPairsFp32(ctx, c.n2, n2pad, c.p2, nullptr, r2c));
  TCSCF_CUDA(ctx, cudaMemsetAsync(dStatus, 0, sizeof(int), ctx->stream));

  auto * vts = static_cast<__nv_bfloat16 *>(vt);
  CUtensorMap maps[3];
  bool okm = true;
  for (int i = 0; i < 3; ++i)
    okm = okm && makeMap2d(&maps[i], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, vts + size_t(i) * NBtot * n2pad, uint64_t(n2pad), uint64_t(NBtot),
                           tc::BK, uint32_t(NB), CU_TENSOR_MAP_SWIZZLE_128B);
  TCSCF_CHECK(ctx, okm, TCSCF_ERR_CUDA, "cuTensorMapEncodeTiled failed");

  tc::PairParams P{};
  P.nTiles = nTiles; P.nChunks = nChunks; P.nSplit = nSplit; P.blocksPerSplit = perSplit; P.nBlocks = nBlocks;
  P.n1 = int(c.n1); P.ncol = c.ncol; P.ldt = c.ldt;
  P.kind = c.kernel == TCSCF_K_INV_R12 ? 0 : (c.kernel <= TCSCF_K_TC_SCALAR_OPPO ? 1 : 2);
  P.comp = c.component;
  P.same = (c.kernel == TCSCF_K_TC_SCALAR_SAME || c.kernel == TCSCF_K_GRAD_U_SAME) ? 1 : 0;
  P.npoly = 1;
  if (P.kind != 0) {
    // u'(r12) = t^2 sum_n p_n z^n, p_n = a12 sum_{k: i_k = n + 1} i_k c_k[same]
    double poly[tc::kMaxPoly] = {};
    int deg = 0;
    for (int k = 0; k < c.jastrow->nterms; ++k) {
      int const i = c.jastrow->S[k][0];
      if (i < 1) continue;
      poly[i - 1] += c.jastrow->a12 * i * c.jastrow->c[k][P.same];
      deg = std::max(deg, i);
    }
    P.npoly = std::max(1, deg);
    for (int n = 0; n < tc::kMaxPoly; ++n) P.poly[n] = float(poly[n]);
    P.a12 = float(c.jastrow->a12);
  }
  P.r1xyz = r1c; P.r2pairs = r2c;
  P.cinv = reinterpret_cast<const float *>(vts + 3 * size_t(NBtot) * n2pad);
  P.NBtot = NBtot;
  P.T = nSplit > 1 ? part : c.T;
  P.tStride = int64_t(c.n1) * c.ldt;
  P.status = dStatus;
  int const grid = int(std::min<int64_t>(items * nSplit, sms));
  cudaEventRecord(ctx->ev[2], ctx->stream);
  int st = TCSCF_OK;
  if (NB == 64) {
    st = P.kind == 0 ? tc::launchPairs<64, 0>(ctx, P, maps, grid)
                     : (P.kind == 1 ? tc::launchPairs<64, 1>(ctx, P, maps, grid) : tc::launchPairs<64, 2>(ctx, P, maps, grid));
  } else {
    st = P.kind == 0 ? tc::launchPairs<128, 0>(ctx, P, maps, grid)
                     : (P.kind == 1 ? tc::launchPairs<128, 1>(ctx, P, maps, grid) : tc::launchPairs<128, 2>(ctx, P, maps, grid));
  }
  cudaEventRecord(ctx->ev[3], ctx->stream);
  TCSCF_TRY(st);
  int hs = 0;
  TCSCF_CUDA(ctx, cudaMemcpyAsync(&hs, dStatus, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (hs != 0) return fail(ctx, TCSCF_ERR_TIMEOUT, "tensor-core precompute contraction: bounded wait expired (code " + std::to_string(hs) + ")");
  if (nSplit > 1) TCSCF_TRY(sumSplitsLaunch(ctx, int64_t(c.n1) * c.ncol, nSplit, int64_t(c.n1) * c.ldt, part, c.T, c.n1, c.ncol, c.ldt, c.ldt));
  return nearCorrect(ctx, c);
}

}  // namespace tcscf
