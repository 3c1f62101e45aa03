// tcgen05 (sm_100a) r12 contraction for the direct Fock build in TF32 (tcgen05.mma kind::tf32) with
// FP32 tensor-core accumulation: the TF32 precision of the Fock build.
//
// The same flash reassociation as the split-BF16 kernel (flash_tc.cu): for a tile of 128 r1 points
// (one TMEM lane each) the kernel streams r2 in blocks of 64,
//   GEMM1 (tensor):  rho(r1,r2) = psi1[r1][:] . psi2[r2][:]            K = 32 (padded rank)
//   CUDA cores:      g = 1/|r1 - r2| (FP32, Newton-refined), X = g * rho, VH(r1) += g * coul(r2)
//   GEMM2 (tensor):  T[r1][i] += X[r1][r2] . Vt[i][r2]                 K = 64, N = NB
// with every operand a single FP32 value rounded to TF32 (10 explicit mantissa bits, round to
// nearest): psi1, psi2 and Vt when they are packed, X when it is written to shared memory.  No
// scales are needed (TF32 keeps the FP32 exponent range).  Each block's FP32 tensor-core sum is
// added, as soon as the block completes, into per-thread double-float accumulators (FP32 hi + lo,
// Fast2Sum), so the only approximations are the TF32 operand roundings and the FP32
// accumulation inside one 64-point block.
//
// Shared-memory operands are K-major with the 128-byte swizzle: a 128-byte row holds 32 FP32 values,
// so the 64-point K extent of GEMM2 is two swizzle atoms (two sub-tiles per operand), and one MMA
// (K = 8, 32 bytes) stays inside one atom.
//
// Warp roles as in flash_tc.cu (384 threads, one persistent CTA per SM): warp 0 TMA producer (no
// multicast), warp 1 MMA issuer and TMEM allocator, warps 2-3 idle, warps 4-11 compute (warp w owns
// TMEM lanes 32*(w%4).. and r2 / column half (w-4)/4).  Every mbarrier wait is bounded; on expiry
// the kernel records the failure in the device status word, drains its own work and frees TMEM.
#include <cuda.h>
#include <cuda_runtime.h>

#include "tc_device.cuh"

namespace tcscf {
namespace tc {

constexpr int RPT = 32;                     // padded rank: one 128-byte row of FP32
__host__ __device__ constexpr int tf32Stages(int NB) { return NB == 64 ? 4 : 3; }
// TMEM columns: rho buffers b = 0, 1 at 64 b; T at TCOLT
constexpr uint32_t TCOLT = 128;

template <int NB>
struct __align__(1024) SmemT32 {
  static constexpr int NSTAGE = tf32Stages(NB);
  uint8_t v[NSTAGE][2][NB * 128];     // Vt block, r2 points 0-31 / 32-63: SW128 K-major [NB rows][32]
  uint8_t x[2][2][BM * 128];          // X tile per buffer, r2 points 0-31 / 32-63: SW128 K-major [128 rows][32]
  uint8_t psi2[NSTAGE][BK * 128];     // psi2 block: SW128 K-major [64 rows][32]
  uint8_t psi1[BM * 128];             // psi1 tile: SW128 K-major [128 rows][32]
  float4 coords[NSTAGE][BK];          // r2 block as 32 pairs {x0,x1,y0,y1}{z0,z1,c0,c1}
  uint64_t full[NSTAGE], empty[NSTAGE];
  uint64_t sfull[2], sfree[2], xfull[2], xfree[2];
  uint64_t tfull, tfree;
  uint64_t p1full, p1free, done;
  uint32_t tmemBase;
  int abort;
};

// instruction descriptor: kind::tf32, A = B = TF32 (K-major), D = F32, shape M x N
__host__ __device__ constexpr uint32_t instrDescTf32(int M, int N)
{
  return (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void mmaTf32(uint32_t tmemD, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmemD),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

// FP32 -> TF32 bit pattern, round to nearest (ties away from zero)
__device__ __forceinline__ uint32_t toTf32(float x)
{
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void tmemWait8(float (&a)[8])
{
  asm volatile("tcgen05.wait::ld.sync.aligned;" : "+f"(a[0]), "+f"(a[1]), "+f"(a[2]), "+f"(a[3]), "+f"(a[4]), "+f"(a[5]), "+f"(a[6]), "+f"(a[7]) :: "memory");
}

// Adds the finished block f (this thread's row, NB/2 columns of T) into the double-float
// accumulators by Fast2Sum and hands the TMEM accumulator back to the MMA issuer.
template <int NB, class SmemT>
__device__ __forceinline__ bool flushTf32(SmemT & S, uint32_t taddr, uint32_t f, uint64_t (&hi)[NB / 4], uint64_t (&lo)[NB / 4], int lane,
                                          volatile int * abortFlag, int * status)
{
  if (!waitBar(&S.tfull, f & 1, abortFlag, status, 31)) return false;
  fenceAfterSync();
  constexpr int NQ = NB / 16;   // chunks of 8 columns; the load of chunk q + 1 overlaps the work on chunk q
  float tt[2][8];
  tmemLoad8(taddr, tt[0]);
  tmemWait8(tt[0]);
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    int const cur = q & 1;
    if (q + 1 < NQ) tmemLoad8(taddr + (q + 1) * 8, tt[cur ^ 1]);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      uint64_t const x = f2pack(tt[cur][2 * i], tt[cur][2 * i + 1]);
      int const p = q * 4 + i;
      // Fast2Sum: hi + x == sum + (x - (sum - hi)) exactly when |hi| >= |x|, which holds once a
      // row's sum has absorbed its first blocks; otherwise the compensation is approximate at the
      // level of the rounding of the smaller term
      uint64_t const sum = f2add(hi[p], x);
      lo[p] = f2add(lo[p], f2sub(x, f2sub(sum, hi[p])));
      hi[p] = sum;
    }
    if (q + 1 < NQ) tmemWait8(tt[cur ^ 1]);
  }
  fenceBeforeSync();
  __syncwarp();
  if (lane == 0) mbarArrive(&S.tfree);
  return true;
}

template <int NB>
__global__ void __launch_bounds__(NTHREADS, 1)
    kFlashTf32(Params P)
{
  extern __shared__ uint8_t smemRaw[];
  SmemT32<NB> & S = *reinterpret_cast<SmemT32<NB> *>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
  constexpr int NSTAGE = tf32Stages(NB);
  int const warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  volatile int * abortFlag = &S.abort;

  static_assert(TCOLT + NB <= 256, "TMEM columns");
  constexpr uint32_t kStageBytes = 2 * NB * 128 + BK * 128 + BK * sizeof(float4);
  constexpr uint32_t kPsi1Bytes = BM * 128;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NSTAGE; ++s) { mbarInit(&S.full[s], 1); mbarInit(&S.empty[s], 1 + NCW); }
    for (int b = 0; b < 2; ++b) {
      mbarInit(&S.sfull[b], 1); mbarInit(&S.sfree[b], NCW);
      mbarInit(&S.xfull[b], NCW); mbarInit(&S.xfree[b], 1);
    }
    mbarInit(&S.tfull, 1); mbarInit(&S.tfree, NCW);
    mbarInit(&S.p1full, 1); mbarInit(&S.p1free, 1); mbarInit(&S.done, 1);
    S.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(smemAddr(&S.tmemBase)) : "memory");
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
          CUtensorMap const * maps = I->maps;   // psi1, psi2, Vt
          int const jb = split * I->blocksPerSplit;
          int const je = min(I->nBlocks, jb + I->blocksPerSplit);
          if (p1Use > 0 && !(ok = waitBar(&S.p1free, (p1Use - 1) & 1, abortFlag, P.status, 11))) break;
          mbarArriveTx(&S.p1full, kPsi1Bytes);
          tmaLoad2d(S.psi1, maps + 0, 0, tile * BM, &S.p1full);
          ++p1Use;
          for (int j = jb; j < je; ++j) {
            uint32_t const q = issuedLoads++;
            int const s = q % NSTAGE;
            if (q >= uint32_t(NSTAGE) && !(ok = waitBar(&S.empty[s], ((q / NSTAGE) - 1) & 1, abortFlag, P.status, 12))) break;
            mbarArriveTx(&S.full[s], kStageBytes);
            tmaLoad2d(S.psi2[s], maps + 1, 0, j * BK, &S.full[s]);
            tmaLoad2d(S.v[s][0], maps + 2, j * BK, 0, &S.full[s]);
            tmaLoad2d(S.v[s][1], maps + 2, j * BK + 32, 0, &S.full[s]);
            bulkLoad(S.coords[s], I->r2pairs + int64_t(j) * BK, BK * sizeof(float4), &S.full[s]);
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
        constexpr uint32_t idesc1 = instrDescTf32(BM, BK);
        constexpr uint32_t idesc2 = instrDescTf32(BM, NB);
        uint32_t const aPsi1 = smemAddr(S.psi1);
        uint32_t blockCount = 0;
        uint32_t p1Use = 0;
        bool ok = true;
        for (int item = blockIdx.x; item < nItems && ok; item += gridDim.x) {
          int ii, tile, split;
          decodeItem(P, item, ii, tile, split);
          Instance const * I = P.inst + ii;
          int const jb = split * I->blocksPerSplit;
          int const je = min(I->nBlocks, jb + I->blocksPerSplit);
          int const nblk = je - jb;
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
            uint32_t const bPsi2 = smemAddr(S.psi2[s]);
#pragma unroll
            for (int k = 0; k < RPT / 8; ++k)
              mmaTf32(tmem + b * BK, smemDesc(aPsi1 + 32 * k, 1024, 2), smemDesc(bPsi2 + 32 * k, 1024, 2), idesc1, k > 0 ? 1u : 0u);
            mmaCommit(&S.sfull[b]);
            return true;
          };
          if (nblk > 0 && !(ok = gemm1(0))) break;
          for (int jj = 0; jj < nblk && ok; ++jj) {
            if (jj + 1 < nblk && !(ok = gemm1(jj + 1))) break;
            uint32_t const g = base + jj;
            int const s = g % NSTAGE, xb = g & 1;
            // the T accumulator is free once the compute warps flushed block g - 1
            if (g >= 1 && !(ok = waitBar(&S.tfree, (g - 1) & 1, abortFlag, P.status, 24))) break;
            if (!(ok = waitBar(&S.xfull[xb], (g >> 1) & 1, abortFlag, P.status, 25))) break;
            fenceAfterSync();
#pragma unroll
            for (int k = 0; k < BK / 8; ++k) {
              uint32_t const aX = smemAddr(S.x[xb][k >> 2]) + 32 * (k & 3);
              uint32_t const bV = smemAddr(S.v[s][k >> 2]) + 32 * (k & 3);
              mmaTf32(tmem + TCOLT, smemDesc(aX, 1024, 2), smemDesc(bV, 1024, 2), idesc2, k > 0 ? 1u : 0u);
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
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(tmem) : "memory");
    }
  } else {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(kRegsCompute));
    // ---------------------------------------------------------------- compute warps
    int const cw = warp - 4;
    int const quarter = warp & 3;
    int const half = cw >> 2;
    int const row = quarter * 32 + lane;
    uint32_t const laneBase = uint32_t(quarter * 32) << 16;
    uint32_t const tAddr = tmem + laneBase + TCOLT + uint32_t(half * (NB / 2));
    uint32_t blockCount = 0;
    bool ok = true;
    uint64_t ahi[NB / 4], alo[NB / 4];   // T of this thread's row and columns as FP32 hi + lo, column pairs
    uint64_t const mOne = f2pack(-1.0f, -1.0f), mHalf = f2pack(-0.5f, -0.5f);
    for (int item = blockIdx.x; item < nItems && ok; item += gridDim.x) {
      int ii, tile, split;
      decodeItem(P, item, ii, tile, split);
      Instance const * I = P.inst + ii;
      int const jb = split * I->blocksPerSplit;
      int const je = min(I->nBlocks, jb + I->blocksPerSplit);
      int const nblk = je - jb;
      int const r1 = tile * BM + row;
      float4 const p1 = I->r1xyz[r1];
#pragma unroll
      for (int c = 0; c < NB / 4; ++c) { ahi[c] = 0; alo[c] = 0; }
      double vh = 0.0;
      bool pending = false;   // block g - 1 still to be flushed
      uint64_t const p1x = f2pack(p1.x, p1.x), p1y = f2pack(p1.y, p1.y), p1z = f2pack(p1.z, p1.z);
      for (int jj = 0; jj < nblk && ok; ++jj) {
        uint32_t const g = blockCount + jj;
        int const s = g % NSTAGE, b = g & 1;
        if (!(ok = waitBar(&S.full[s], (g / NSTAGE) & 1, abortFlag, P.status, 32))) break;
        if (!(ok = waitBar(&S.sfull[b], (g >> 1) & 1, abortFlag, P.status, 33))) break;
        fenceAfterSync();
        // X = g * rho for this warp's 32 r2 points (16 pairs)
        float4 const * cc = S.coords[s] + half * 32;
        uint64_t xv[16];
        uint64_t vsum2 = 0;
        uint32_t const rhoAddr = tmem + laneBase + uint32_t(b * BK + half * 32);
        {
          float rho[2][16];
          tmemLoad16(rhoAddr, rho[0]);
          tmemLoad16(rhoAddr + 16, rho[1]);
          tmemWaitLoad(rho[0], rho[1]);
          // this warp's rho columns are read: the buffer is free for GEMM1
          fenceBeforeSync();
          __syncwarp();
          if (lane == 0) mbarArrive(&S.sfree[b]);
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
            xv[pr] = f2mul(y, f2pack(rho[pr >> 3][2 * (pr & 7)], rho[pr >> 3][2 * (pr & 7) + 1]));
          }
        }
        // X buffer xb is free once GEMM2 of block g - 2 completed; this half writes sub-tile `half`
        int const xb = g & 1;
        if (g >= 2 && !(ok = waitBar(&S.xfree[xb], ((g >> 1) - 1) & 1, abortFlag, P.status, 34))) break;
        uint8_t * xs = S.x[xb][half];
#pragma unroll
        for (int ch = 0; ch < 8; ++ch) {
          float x0, x1, x2, x3;
          f2unpack(xv[2 * ch], x0, x1);
          f2unpack(xv[2 * ch + 1], x2, x3);
          *reinterpret_cast<uint4 *>(xs + sw128(row, ch)) = make_uint4(toTf32(x0), toTf32(x1), toTf32(x2), toTf32(x3));
        }
        float vs0, vs1;
        f2unpack(vsum2, vs0, vs1);
        vh += double(vs0 + vs1);
        fenceProxyAsync();
        __syncwarp();
        if (lane == 0) { mbarArrive(&S.xfull[xb]); mbarArrive(&S.empty[s]); }
        if (pending && !(ok = flushTf32<NB>(S, tAddr, g - 1, ahi, alo, lane, abortFlag, P.status))) break;
        pending = true;
      }
      if (ok && pending) ok = flushTf32<NB>(S, tAddr, blockCount + nblk - 1, ahi, alo, lane, abortFlag, P.status);
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
        // the two r2-half warps of a row each summed half of the r2 points of every block
        atomicAdd(&I->VH[int64_t(split) * I->vhStride + r1], vh);
      }
    }
    fenceBeforeSync();
    __syncthreads();
  }
}

// ---- operand packing ---------------------------------------------------------------------------------
__device__ __forceinline__ float tf32Value(double v) { return __uint_as_float(toTf32(float(v))); }

// psi [n][ldpsi] FP64 (R <= 32 columns) -> TF32-rounded FP32 [npad][32], zero padded
__global__ void kPackPsiTf32(int64_t n, int64_t npad, int R, const double * psi, int ldpsi, float * out)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < npad * RPT; i += int64_t(gridDim.x) * blockDim.x) {
    int64_t const r = i / RPT;
    int const k = int(i % RPT);
    out[i] = (r < n && k < R) ? tf32Value(psi[r * ldpsi + k]) : 0.0f;
  }
}

// V [n2][ldv] FP64 (nb columns) -> Vt TF32-rounded FP32 [NB][n2pad], zero padded (32 x 32 tiles
// transposed through shared memory)
__global__ void kPackVtTf32(int64_t n2, int64_t n2pad, int nb, int NB, const double * V, int ldv, float * out)
{
  __shared__ float t[32][33];
  int64_t const r0 = int64_t(blockIdx.x) * 32;
  int const c0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    int64_t const r = r0 + k;
    int const c = c0 + threadIdx.x;
    t[k][threadIdx.x] = (r < n2 && c < nb) ? tf32Value(V[r * ldv + c]) : 0.0f;
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    int const c = c0 + k;
    int64_t const r = r0 + threadIdx.x;
    if (c < NB && r < n2pad) out[int64_t(c) * n2pad + r] = t[threadIdx.x][k];
  }
}

}  // namespace tc

// ------------------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------------------
namespace {

size_t align256t(size_t n) { return (n + 255) & ~size_t(255); }

template <int NB>
int launchTf32NB(tcscf_ctx * ctx, tc::Params const & P, int grid)
{
  size_t const smem = sizeof(tc::SmemT32<NB>) + 1024;
  static_assert(sizeof(tc::SmemT32<NB>) + 1024 <= 232448, "shared memory per CTA");
  TCSCF_CUDA(ctx, cudaFuncSetAttribute(tc::kFlashTf32<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  tc::kFlashTf32<NB><<<grid, tc::NTHREADS, smem, ctx->stream>>>(P);
  TCSCF_LAUNCH(ctx);
  return TCSCF_OK;
}

}  // namespace

size_t tf32OperandBytes(int NB, int64_t n1pad, int64_t n2pad)
{
  return align256t(sizeof(float) * size_t(n1pad) * tc::RPT) + align256t(sizeof(float) * size_t(n2pad) * tc::RPT) +
         align256t(sizeof(float) * size_t(NB) * n2pad);
}

int tf32PackOperands(tcscf_ctx * ctx, Contraction const & c, int NB, int64_t n1pad, int64_t n2pad, void * dst, CUtensorMap * maps)
{
  TCSCF_CHECK(ctx, c.R >= 1 && c.R <= tc::RPT, TCSCF_ERR_INVALID_ARGUMENT, "internal: TF32 launch rank above 32");
  char * q = static_cast<char *>(dst);
  auto * psi1 = reinterpret_cast<float *>(q);
  q += align256t(sizeof(float) * size_t(n1pad) * tc::RPT);
  auto * psi2 = reinterpret_cast<float *>(q);
  q += align256t(sizeof(float) * size_t(n2pad) * tc::RPT);
  auto * vt = reinterpret_cast<float *>(q);
  tc::kPackPsiTf32<<<gridBlocks(n1pad * tc::RPT, 256), 256, 0, ctx->stream>>>(c.n1, n1pad, c.R, c.psi1, c.ldpsi, psi1);
  TCSCF_LAUNCH(ctx);
  tc::kPackPsiTf32<<<gridBlocks(n2pad * tc::RPT, 256), 256, 0, ctx->stream>>>(c.n2, n2pad, c.R, c.psi2, c.ldpsi, psi2);
  TCSCF_LAUNCH(ctx);
  dim3 const tb{32, 8, 1};
  dim3 const tg{unsigned((n2pad + 31) / 32), unsigned((NB + 31) / 32), 1};
  tc::kPackVtTf32<<<tg, tb, 0, ctx->stream>>>(c.n2, n2pad, c.ncol, NB, c.V, c.ldv, vt);
  TCSCF_LAUNCH(ctx);
  bool ok = makeMap2d(&maps[0], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, psi1, tc::RPT, n1pad, tc::RPT, tc::BM, CU_TENSOR_MAP_SWIZZLE_128B);
  ok = ok && makeMap2d(&maps[1], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, psi2, tc::RPT, n2pad, tc::RPT, tc::BK, CU_TENSOR_MAP_SWIZZLE_128B);
  ok = ok && makeMap2d(&maps[2], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, vt, n2pad, NB, 32, NB, CU_TENSOR_MAP_SWIZZLE_128B);
  TCSCF_CHECK(ctx, ok, TCSCF_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  return TCSCF_OK;
}

int launchTf32(tcscf_ctx * ctx, int NB, tc::Params const & P, int grid)
{
  if (NB == 64) return launchTf32NB<64>(ctx, P, grid);
  if (NB == 128) return launchTf32NB<128>(ctx, P, grid);
  return fail(ctx, TCSCF_ERR_UNSUPPORTED, "no TF32 kernel for this tile class");
}

}  // namespace tcscf
