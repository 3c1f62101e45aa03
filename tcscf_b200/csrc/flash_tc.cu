// tcgen05 (sm_100a) r12 contraction for the direct Fock build, split-BF16 ("bf16x3") precision.
//
// For a tile of 128 r1 points (one TMEM lane each) the kernel streams r2 in blocks of 64:
//   GEMM1 (tensor):  S[r1][r2]  = psi1[r1][:] . psi2[r2][:]        rho(r1,r2), K = 32 (padded rank)
//   CUDA cores:      g = 1/|r1 - r2| (FP32, Newton-refined), X = g * rho, VH(r1) += g * coul(r2)
//   GEMM2 (tensor):  T[r1][i]  += X[r1][r2] . Vt[i][r2]            Vt = (w2 phi_i(r2))^T, N = NB
// Every operand is a hi+lo BF16 pair and each GEMM issues hi*hi + hi*lo + lo*hi; accumulation is
// FP32 in TMEM, flushed every `window` r2 blocks into per-thread FP64 accumulators (the TMEM
// accumulator is double-buffered so the MMA never waits for a flush).  The kernel matrix g is
// generated in registers and only ever exists as the BF16 X tile in shared memory.
//
// Warp roles (384 threads, one CTA per SM, persistent over (r1 tile, r2 split) work items):
//   warp 0      TMA producer: psi1 tile (once per work item), psi2 / Vt blocks (TMA, no multicast),
//               r2 coordinates + Coulomb source (1-D bulk copy)
//   warp 1      MMA issuer (one elected thread) and TMEM allocator
//   warps 2-3   idle (they complete warpgroup 0, whose registers setmaxnreg hands to the compute warps)
//   warps 4-11  compute: warp w owns TMEM lanes 32*(w%4).. (r1 rows), column half (w-4)/4
// Every mbarrier wait is bounded by a wall-clock limit; on expiry the kernel records the failure in
// a device status word, drains its own TMA / MMA work with bounded waits, frees TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>

#include "kernels.cuh"

namespace tcscf {
namespace tc {

constexpr int BM = 128;        // r1 rows per tile
constexpr int BK = 64;         // r2 points per block
// TMA stages: three when the rank padding leaves room in shared memory
__host__ __device__ constexpr int stagesFor(int RP) { return RP == 32 ? 3 : 2; }
constexpr int NCW = 8;         // compute warps
constexpr int NTHREADS = 384;  // warpgroup 0: TMA, MMA, 2 idle warps; warpgroups 1-2: compute
// register split: 384 threads x 168 at launch = 64512 = 128 x 56 (producer warpgroup) + 256 x 224
constexpr int kRegsLaunch = 168, kRegsProducer = 56, kRegsCompute = 224;
static_assert(128 * kRegsProducer + 256 * kRegsCompute <= NTHREADS * kRegsLaunch, "register split exceeds the launch allocation");
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s per wait
// a waiting thread sleeps in mbarrier.try_wait (woken when the phase completes) instead of spinning
// on the issue slots the compute warps need
constexpr uint32_t kSuspendHintNs = 1000000;

// RP: padded rank of rho (GEMM1 K): 32 (64-byte rows, 64B swizzle) or 64 (128-byte rows, 128B swizzle)
template <int NB, int RP>
struct __align__(1024) Smem {
  static constexpr int NSTAGE = stagesFor(RP);
  uint8_t v[NSTAGE][2][NB * BK * 2];       // Vt block hi/lo: SW128 K-major [NB rows][64]
  uint8_t x[2][2][BM * BK * 2];            // X tile hi/lo:   SW128 K-major [128 rows][64]
  uint8_t psi2[NSTAGE][2][BK * RP * 2];    // psi2 block hi/lo: K-major [64 rows][RP]
  uint8_t psi1[2][BM * RP * 2];            // psi1 tile hi/lo:  K-major [128 rows][RP]
  float4 coords[NSTAGE][BK];               // r2 block as 32 pairs {x0,x1,y0,y1}{z0,z1,c0,c1}
  uint64_t full[NSTAGE], empty[NSTAGE];
  uint64_t sfull[2], sfree[2], xfull[2], xfree[2], tfull[2], tfree[2];
  uint64_t p1full, p1free, done;
  uint32_t tmemBase;
  int abort;
};

struct Params {
  int nTiles, nSplit, blocksPerSplit, nBlocks;   // r2 blocks in total, per split
  int n1;                                          // real r1 rows
  int nb;                                          // real columns of T
  int window;                                      // r2 blocks per FP32 accumulation window
  const float4 * r1xyz;                            // [n1pad] x, y, z, 0
  const float4 * r2xyzc;                           // [nBlocks*64] x, y, z, coul
  double * T;                                      // [nSplit][n1][ldt]
  double * VH;                                     // [nSplit][n1]
  int ldt;
  int64_t tStride, vhStride;
  int * status;                                    // device status word (0 = ok)
};

// ---- PTX helpers --------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smemAddr(const void * p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ unsigned long long globalTimer()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbarInit(uint64_t * b, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbarArrive(uint64_t * b)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smemAddr(b)) : "memory");
}
__device__ __forceinline__ void mbarArriveTx(uint64_t * b, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbarTryWait(uint64_t * b, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smemAddr(b)), "r"(parity), "r"(kSuspendHintNs)
      : "memory");
  return ok != 0;
}

// Bounded wait; returns false (after recording the failure) when the limit expires or another role
// has already aborted.
__device__ __forceinline__ bool waitBar(uint64_t * b, uint32_t parity, volatile int * abortFlag, int * status, int code)
{
  if (mbarTryWait(b, parity)) return true;
  unsigned long long const t0 = globalTimer();
  while (true) {
    if (mbarTryWait(b, parity)) return true;
    if (*abortFlag) return false;
    if (globalTimer() - t0 > kWaitLimitNs) {
      *abortFlag = 1;
      atomicCAS(status, 0, code);
      return false;
    }
  }
}

__device__ __forceinline__ void tmaLoad2d(void * dst, const CUtensorMap * map, int x, int y, uint64_t * bar)
{
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(smemAddr(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smemAddr(bar))
      : "memory");
}

__device__ __forceinline__ void bulkLoad(void * dst, const void * src, uint32_t bytes, uint64_t * bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smemAddr(dst)), "l"(src),
               "r"(bytes), "r"(smemAddr(bar))
               : "memory");
}

// UMMA shared-memory descriptor (K-major): start address, stride byte offset between 8-row groups,
// version 1, swizzle mode (2 = 128B, 4 = 64B).
__device__ __forceinline__ uint64_t smemDesc(uint32_t addr, uint32_t sbo, uint32_t swizzle)
{
  uint64_t d = 0;
  d |= uint64_t((addr >> 4) & 0x3FFF);
  d |= uint64_t(1) << 16;                          // leading byte offset (unused for swizzled K-major)
  d |= uint64_t((sbo >> 4) & 0x3FFF) << 32;
  d |= uint64_t(1) << 46;                          // descriptor version (sm_100)
  d |= uint64_t(swizzle & 7) << 61;
  return d;
}

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

__device__ __forceinline__ void mmaCommit(uint64_t * bar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smemAddr(bar)) : "memory");
}

__device__ __forceinline__ void fenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmemLoad16(uint32_t taddr, float * v)
{
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
        "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmemWaitLoad() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---- packed FP32 pairs (sm_100 f32x2 arithmetic on 64-bit register pairs) ---------------------
__device__ __forceinline__ uint64_t f2pack(float a, float b)
{
  uint64_t d;
  asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(a), "f"(b));
  return d;
}
__device__ __forceinline__ void f2unpack(uint64_t v, float & a, float & b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v)); }
__device__ __forceinline__ uint64_t f2sub(uint64_t a, uint64_t b)
{
  uint64_t d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t f2mul(uint64_t a, uint64_t b)
{
  uint64_t d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t f2fma(uint64_t a, uint64_t b, uint64_t c)
{
  uint64_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ float rsqrtApprox(float x)
{
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// byte offset of element (row, k) in a K-major SW128 tile of 64 BF16 columns
__device__ __forceinline__ uint32_t sw128(int row, int chunk)
{
  return uint32_t((row >> 3) * 1024 + (row & 7) * 128 + ((chunk ^ (row & 7)) << 4));
}

__device__ __forceinline__ uint32_t packBf16(float a, float b)
{
  __nv_bfloat162 const h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t const *>(&h);
}

// Adds one finished FP32 TMEM accumulation window (64 of the NB columns of this thread's row) into
// the FP64 accumulators and hands the TMEM buffer back to the MMA issuer.
template <int NB, class SmemT>
__device__ __forceinline__ bool flushWindow(SmemT & S, uint32_t taddr, uint32_t window, double (&acc)[64], int lane,
                                            volatile int * abortFlag, int * status)
{
  uint32_t const t = window & 1;
  if (!waitBar(&S.tfull[t], (window >> 1) & 1, abortFlag, status, 31)) return false;
  fenceAfterSync();
#pragma unroll
  for (int q = 0; q < (NB >= 128 ? 4 : 2); ++q) {
    float v[16];
    tmemLoad16(taddr + q * 16, v);
    tmemWaitLoad();
#pragma unroll
    for (int i = 0; i < 16; ++i) acc[q * 16 + i] += double(v[i]);
  }
  fenceBeforeSync();
  __syncwarp();
  if (lane == 0) mbarArrive(&S.tfree[t]);
  return true;
}

// ---- the kernel ------------------------------------------------------------------------------------
template <int NB, int RP>
__global__ void __launch_bounds__(NTHREADS, 1)
    kFlashTc(const __grid_constant__ CUtensorMap mapPsi1Hi, const __grid_constant__ CUtensorMap mapPsi1Lo,
             const __grid_constant__ CUtensorMap mapPsi2Hi, const __grid_constant__ CUtensorMap mapPsi2Lo,
             const __grid_constant__ CUtensorMap mapVHi, const __grid_constant__ CUtensorMap mapVLo, Params P)
{
  extern __shared__ uint8_t smemRaw[];
  Smem<NB, RP> & S = *reinterpret_cast<Smem<NB, RP> *>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
  constexpr int NSTAGE = stagesFor(RP);
  int const warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  volatile int * abortFlag = &S.abort;

  constexpr uint32_t TCOL0 = 2 * BK;   // TMEM columns: S buffers [0, 128), T buffers [128, 128 + 2 NB)
  constexpr uint32_t kStageBytes = 2 * NB * BK * 2 + 2 * BK * RP * 2 + BK * sizeof(float4);
  constexpr uint32_t kPsi1Bytes = 2 * BM * RP * 2;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NSTAGE; ++s) { mbarInit(&S.full[s], 1); mbarInit(&S.empty[s], 1 + NCW); }
    for (int b = 0; b < 2; ++b) {
      mbarInit(&S.sfull[b], 1); mbarInit(&S.sfree[b], NCW);
      mbarInit(&S.xfull[b], NCW); mbarInit(&S.xfree[b], 1);
      mbarInit(&S.tfull[b], 1); mbarInit(&S.tfree[b], NCW);
    }
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

  int const nItems = P.nTiles * P.nSplit;

  if (warp < 4) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kRegsProducer));
  if (warp == 0) {
    // ---------------------------------------------------------------- TMA producer
    if (lane == 0) {
      uint32_t issuedLoads = 0;
      uint32_t p1Use = 0;
      bool ok = true;
      for (int item = blockIdx.x; item < nItems && ok; item += gridDim.x) {
        int const tile = item / P.nSplit, split = item % P.nSplit;
        int const jb = split * P.blocksPerSplit;
        int const je = min(P.nBlocks, jb + P.blocksPerSplit);
        if (p1Use > 0 && !(ok = waitBar(&S.p1free, (p1Use - 1) & 1, abortFlag, P.status, 11))) break;
        mbarArriveTx(&S.p1full, kPsi1Bytes);
        tmaLoad2d(S.psi1[0], &mapPsi1Hi, 0, tile * BM, &S.p1full);
        tmaLoad2d(S.psi1[1], &mapPsi1Lo, 0, tile * BM, &S.p1full);
        ++p1Use;
        for (int j = jb; j < je; ++j) {
          uint32_t const q = issuedLoads++;
          int const s = q % NSTAGE;
          // use u = q / NSTAGE of stage s needs consumption u - 1 of it
          if (q >= uint32_t(NSTAGE) && !(ok = waitBar(&S.empty[s], ((q / NSTAGE) - 1) & 1, abortFlag, P.status, 12))) break;
          mbarArriveTx(&S.full[s], kStageBytes);
          tmaLoad2d(S.psi2[s][0], &mapPsi2Hi, 0, j * BK, &S.full[s]);
          tmaLoad2d(S.psi2[s][1], &mapPsi2Lo, 0, j * BK, &S.full[s]);
          tmaLoad2d(S.v[s][0], &mapVHi, j * BK, 0, &S.full[s]);
          tmaLoad2d(S.v[s][1], &mapVLo, j * BK, 0, &S.full[s]);
          bulkLoad(S.coords[s], P.r2xyzc + int64_t(j) * BK, BK * sizeof(float4), &S.full[s]);
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
      uint32_t const aPsi1[2] = {smemAddr(S.psi1[0]), smemAddr(S.psi1[1])};
      uint32_t blockCount = 0;   // global block counter: selects stage, S/X buffers
      uint32_t windowCount = 0;  // global window counter: selects the T buffer
      uint32_t p1Use = 0;
      bool ok = true;
      for (int item = blockIdx.x; item < nItems && ok; item += gridDim.x) {
        int const split = item % P.nSplit;
        int const jb = split * P.blocksPerSplit;
        int const je = min(P.nBlocks, jb + P.blocksPerSplit);
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
          uint32_t const d = tmem + b * BK;
          uint32_t const bPsi2[2] = {smemAddr(S.psi2[s][0]), smemAddr(S.psi2[s][1])};
          // the two small cross products accumulate first, the hi*hi product last, so that only
          // the final steps round the full-magnitude accumulator
          constexpr uint32_t sbo = RP == 64 ? 1024 : 512, swz = RP == 64 ? 2 : 4;
          uint32_t acc = 0;
#pragma unroll
          for (int k = 0; k < RP / 16; ++k) {
            mmaBf16(d, smemDesc(aPsi1[0] + 32 * k, sbo, swz), smemDesc(bPsi2[1] + 32 * k, sbo, swz), idesc1, acc); acc = 1;
            mmaBf16(d, smemDesc(aPsi1[1] + 32 * k, sbo, swz), smemDesc(bPsi2[0] + 32 * k, sbo, swz), idesc1, 1);
          }
#pragma unroll
          for (int k = 0; k < RP / 16; ++k)
            mmaBf16(d, smemDesc(aPsi1[0] + 32 * k, sbo, swz), smemDesc(bPsi2[0] + 32 * k, sbo, swz), idesc1, 1);
          mmaCommit(&S.sfull[b]);
          return true;
        };
        if (nblk > 0 && !(ok = gemm1(0))) break;
        for (int jj = 0; jj < nblk && ok; ++jj) {
          if (jj + 1 < nblk && !(ok = gemm1(jj + 1))) break;
          uint32_t const g = base + jj;
          int const s = g % NSTAGE, b = g & 1;
          int const inWin = jj % P.window;
          bool const lastInWin = (inWin == P.window - 1) || (jj == nblk - 1);
          uint32_t const t = windowCount & 1;
          if (inWin == 0 && windowCount >= 2 && !(ok = waitBar(&S.tfree[t], ((windowCount >> 1) - 1) & 1, abortFlag, P.status, 24))) break;
          if (!(ok = waitBar(&S.xfull[b], (g >> 1) & 1, abortFlag, P.status, 25))) break;
          fenceAfterSync();
          uint32_t const d = tmem + TCOL0 + t * NB;
          uint32_t const aX[2] = {smemAddr(S.x[b][0]), smemAddr(S.x[b][1])};
          uint32_t const bV[2] = {smemAddr(S.v[s][0]), smemAddr(S.v[s][1])};
          uint32_t acc = inWin == 0 ? 0u : 1u;
#pragma unroll
          for (int k = 0; k < BK / 16; ++k) {
            mmaBf16(d, smemDesc(aX[0] + 32 * k, 1024, 2), smemDesc(bV[1] + 32 * k, 1024, 2), idesc2, acc); acc = 1;
            mmaBf16(d, smemDesc(aX[1] + 32 * k, 1024, 2), smemDesc(bV[0] + 32 * k, 1024, 2), idesc2, 1);
          }
#pragma unroll
          for (int k = 0; k < BK / 16; ++k)
            mmaBf16(d, smemDesc(aX[0] + 32 * k, 1024, 2), smemDesc(bV[0] + 32 * k, 1024, 2), idesc2, 1);
          mmaCommit(&S.xfree[b]);
          mmaCommit(&S.empty[s]);
          if (lastInWin) { mmaCommit(&S.tfull[t]); ++windowCount; }
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
    uint32_t blockCount = 0, windowCount = 0;
    bool ok = true;
    double acc[64];
    for (int item = blockIdx.x; item < nItems && ok; item += gridDim.x) {
      int const tile = item / P.nSplit, split = item % P.nSplit;
      int const jb = split * P.blocksPerSplit;
      int const je = min(P.nBlocks, jb + P.blocksPerSplit);
      int const nblk = je - jb;
      int const r1 = tile * BM + row;
      float4 const p1 = P.r1xyz[r1];
#pragma unroll
      for (int c = 0; c < 64; ++c) acc[c] = 0.0;
      double vh = 0.0;
      int pendingFlush = -1;   // window whose flush is deferred by one block
      for (int jj = 0; jj < nblk && ok; ++jj) {
        uint32_t const g = blockCount + jj;
        int const s = g % NSTAGE, b = g & 1;
        if (!(ok = waitBar(&S.full[s], (g / NSTAGE) & 1, abortFlag, P.status, 32))) break;
        if (!(ok = waitBar(&S.sfull[b], (g >> 1) & 1, abortFlag, P.status, 33))) break;
        fenceAfterSync();
        float rho[16];
        tmemLoad16(tmem + laneBase + b * BK + half * 32, rho);
        tmemWaitLoad();
        if (g >= 2 && !(ok = waitBar(&S.xfree[b], ((g >> 1) - 1) & 1, abortFlag, P.status, 34))) break;
        // this warp's 32 r2 points: 16 pairs of {x0,x1,y0,y1}{z0,z1,c0,c1}
        float4 const * cc = S.coords[s] + half * 32;
        uint8_t * xhi = S.x[b][0];
        uint8_t * xlo = S.x[b][1];
        uint64_t vsum2 = 0;
        uint64_t const p1x = f2pack(p1.x, p1.x), p1y = f2pack(p1.y, p1.y), p1z = f2pack(p1.z, p1.z);
        uint64_t const mOne = f2pack(-1.0f, -1.0f), mHalf = f2pack(-0.5f, -0.5f);
#pragma unroll 1
        for (int hh = 0; hh < 2; ++hh) {
          if (hh == 1) {
            // second half of this warp's 32 rho columns; the S buffer is then free for the next GEMM1
            tmemLoad16(tmem + laneBase + b * BK + half * 32 + 16, rho);
            tmemWaitLoad();
            fenceBeforeSync();
            __syncwarp();
            if (lane == 0) mbarArrive(&S.sfree[b]);
          }
#pragma unroll
          for (int c2 = 0; c2 < 2; ++c2) {
            int const ch = hh * 2 + c2;
            uint32_t hi[4], lo[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              int const pr = ch * 4 + e;                 // pair index within the warp's 16 pairs
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
              ya = r2a > 0.0f ? ya : 0.0f;                // coincident pair contributes 0
              yb = r2b > 0.0f ? yb : 0.0f;
              y = f2pack(ya, yb);
              vsum2 = f2fma(y, f2pack(qb.z, qb.w), vsum2);
              uint64_t const x = f2mul(y, f2pack(rho[c2 * 8 + 2 * e], rho[c2 * 8 + 2 * e + 1]));
              float xa, xb;
              f2unpack(x, xa, xb);
              // hi = X with the low 16 mantissa bits cleared (exact), lo = BF16(X - hi)
              uint32_t const b0 = __float_as_uint(xa) & 0xFFFF0000u, b1 = __float_as_uint(xb) & 0xFFFF0000u;
              hi[e] = __byte_perm(b0, b1, 0x7632);
              float la, lb;
              f2unpack(f2sub(x, f2pack(__uint_as_float(b0), __uint_as_float(b1))), la, lb);
              lo[e] = packBf16(la, lb);
            }
            uint32_t const off = sw128(row, half * 4 + ch);
            *reinterpret_cast<uint4 *>(xhi + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
            *reinterpret_cast<uint4 *>(xlo + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
          }
        }
        float vs0, vs1;
        f2unpack(vsum2, vs0, vs1);
        float const vsum = vs0 + vs1;
        vh += double(vsum);
        fenceProxyAsync();
        __syncwarp();
        if (lane == 0) { mbarArrive(&S.xfull[b]); mbarArrive(&S.empty[s]); }
        if (pendingFlush >= 0) {
          if (!(ok = flushWindow<NB>(S, tmem + laneBase + TCOL0 + uint32_t(pendingFlush & 1) * NB + half * (NB / 2), uint32_t(pendingFlush),
                                     acc, lane, abortFlag, P.status)))
            break;
          pendingFlush = -1;
        }
        int const inWin = jj % P.window;
        if (inWin == P.window - 1 || jj == nblk - 1) { pendingFlush = int(windowCount); ++windowCount; }
      }
      if (ok && pendingFlush >= 0)
        ok = flushWindow<NB>(S, tmem + laneBase + TCOL0 + uint32_t(pendingFlush & 1) * NB + half * (NB / 2), uint32_t(pendingFlush), acc, lane,
                             abortFlag, P.status);
      blockCount += nblk;
      if (!ok) break;
      if (r1 < P.n1) {
        double * T = P.T + int64_t(split) * P.tStride + int64_t(r1) * P.ldt;
#pragma unroll
        for (int c = 0; c < NB / 2; ++c) {
          int const col = half * (NB / 2) + c;
          if (col < P.nb) T[col] = acc[c];
        }
      }
      // the two column-half warps of a row each summed half of the r2 points of every block
      if (r1 < P.n1) atomicAdd(&P.VH[int64_t(split) * P.vhStride + r1], vh);
    }
    fenceBeforeSync();
    __syncthreads();
  }
}

// ---- operand packing ---------------------------------------------------------------------------------
// psi [n][ldpsi] FP64 (R columns) -> hi/lo BF16 [npad][RP], zero padded
__global__ void kPackPsi(int64_t n, int64_t npad, int R, int RP, const double * psi, int ldpsi, __nv_bfloat16 * hi, __nv_bfloat16 * lo)
{
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < npad * RP; idx += int64_t(gridDim.x) * blockDim.x) {
    int64_t const r = idx / RP;
    int const b = int(idx % RP);
    float const v = (r < n && b < R) ? float(psi[r * ldpsi + b]) : 0.0f;
    double const vd = (r < n && b < R) ? psi[r * ldpsi + b] : 0.0;
    __nv_bfloat16 const h = __float2bfloat16_rn(v);
    hi[idx] = h;
    lo[idx] = __float2bfloat16_rn(float(vd - double(__bfloat162float(h))));
  }
}

// V [n][ldv] FP64 (nb columns) -> transposed hi/lo BF16 [NB][npad] (tiled transpose)
__global__ void kPackVt(int64_t n, int64_t npad, int nb, int NB, const double * V, int ldv, __nv_bfloat16 * hi, __nv_bfloat16 * lo)
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
      double const v = tile[threadIdx.x][k];
      __nv_bfloat16 const h = __float2bfloat16_rn(float(v));
      hi[int64_t(c) * npad + r] = h;
      lo[int64_t(c) * npad + r] = __float2bfloat16_rn(float(v - double(__bfloat162float(h))));
    }
  }
}

// pts [3][n] (+ coul [n]) -> float4 [npad] (x, y, z, coul); padding points sit far away with 0 weight
__global__ void kPackCoords(int64_t n, int64_t npad, const double * pts, const double * coul, float4 * out)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < npad; i += int64_t(gridDim.x) * blockDim.x) {
    if (i < n) out[i] = make_float4(float(pts[i]), float(pts[n + i]), float(pts[2 * n + i]), coul ? float(coul[i]) : 0.0f);
    else out[i] = make_float4(1.0e4f, 1.0e4f, 1.0e4f, 0.0f);
  }
}

// same in pairs: point pair p -> {x_2p, x_2p+1, y_2p, y_2p+1}, {z_2p, z_2p+1, c_2p, c_2p+1} (npad even)
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

}  // namespace tc

// ------------------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------------------
namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *, const cuuint64_t *,
                                   const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

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

// 2-D BF16 tensor map: inner extent `inner` (contiguous), `outer` rows, box (boxInner, boxOuter)
bool makeMap(CUtensorMap * m, void * base, uint64_t inner, uint64_t outer, uint32_t boxInner, uint32_t boxOuter, CUtensorMapSwizzle sw)
{
  EncodeTiledFn fn = encodeTiled();
  if (!fn) return false;
  cuuint64_t dims[2] = {inner, outer};
  cuuint64_t strides[1] = {inner * 2};
  cuuint32_t box[2] = {boxInner, boxOuter};
  cuuint32_t es[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int NB, int RP>
int launchFlash(tcscf_ctx * ctx, CUtensorMap const * maps, tc::Params const & P, int grid)
{
  size_t const smem = sizeof(tc::Smem<NB, RP>) + 1024;
  TCSCF_CUDA(ctx, cudaFuncSetAttribute(tc::kFlashTc<NB, RP>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  tc::kFlashTc<NB, RP><<<grid, tc::NTHREADS, smem, ctx->stream>>>(maps[0], maps[1], maps[2], maps[3], maps[4], maps[5], P);
  TCSCF_LAUNCH(ctx);
  return TCSCF_OK;
}

}  // namespace

int tensorPackedV(tcscf_ctx * ctx, Grid & g2, const double * V, double scale, const void ** hi, const void ** lo)
{
  int const NB = g2.nb <= 64 ? 64 : 128;
  int64_t const n2pad = (g2.n + tc::BK - 1) / tc::BK * tc::BK;
  if (!g2.vtCache || g2.vtNB != NB || g2.vtN2pad != n2pad || g2.vtScale != scale) {
    cudaStreamSynchronize(ctx->stream);
    cudaFree(g2.vtCache);
    g2.vtCache = nullptr;
    TCSCF_CUDA(ctx, cudaMalloc(&g2.vtCache, size_t(2) * NB * n2pad * sizeof(__nv_bfloat16)));
    auto * vh = static_cast<__nv_bfloat16 *>(g2.vtCache);
    dim3 const tb{32, 8, 1};
    dim3 const tg{unsigned((n2pad + 31) / 32), unsigned((NB + 31) / 32), 1};
    tc::kPackVt<<<tg, tb, 0, ctx->stream>>>(g2.n, n2pad, g2.nb, NB, V, g2.nb, vh, vh + size_t(NB) * n2pad);
    TCSCF_LAUNCH(ctx);
    g2.vtNB = NB;
    g2.vtN2pad = n2pad;
    g2.vtScale = scale;
  }
  auto * vh = static_cast<__nv_bfloat16 *>(g2.vtCache);
  *hi = vh;
  *lo = vh + size_t(NB) * n2pad;
  return TCSCF_OK;
}

bool tensorPathAvailable(Contraction const & c, int precision, std::string * why)
{
  if (precision != TCSCF_PREC_BF16X3) { if (why) *why = "only the bf16x3 tensor path is built"; return false; }
  if (c.kernel != TCSCF_K_INV_R12) { if (why) *why = "tensor path implements the 1/r12 kernel"; return false; }
  if (c.R < 1 || c.R > 64) { if (why) *why = "density factor rank must be 1..64 for the tensor path"; return false; }
  if (c.ncol > 128) { if (why) *why = "tensor path supports nb <= 128"; return false; }
  if (!encodeTiled()) { if (why) *why = "cuTensorMapEncodeTiled unavailable"; return false; }
  return true;
}

int contractTensor(tcscf_ctx * ctx, Contraction const & c, int precision)
{
  std::string why;
  if (!tensorPathAvailable(c, precision, &why)) return fail(ctx, TCSCF_ERR_UNSUPPORTED, why);
  int const NB = c.ncol <= 64 ? 64 : 128;
  int const RP = c.R <= 32 ? 32 : 64;
  int64_t const n1pad = (c.n1 + tc::BM - 1) / tc::BM * tc::BM;
  int64_t const n2pad = (c.n2 + tc::BK - 1) / tc::BK * tc::BK;
  int const nTiles = int(n1pad / tc::BM);
  int const nBlocks = int(n2pad / tc::BK);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // split r2 when there are fewer tiles than SMs (partials summed deterministically afterwards)
  int nSplit = std::max(1, std::min(sms / std::max(1, nTiles), nBlocks / 4));
  int const perSplit = (nBlocks + nSplit - 1) / nSplit;
  nSplit = (nBlocks + perSplit - 1) / perSplit;

  size_t const bf = sizeof(__nv_bfloat16);
  size_t bytes = 2 * size_t(n1pad) * RP * bf + 2 * size_t(n2pad) * RP * bf + 2 * size_t(NB) * n2pad * bf
                 + size_t(n1pad) * sizeof(float4) + size_t(n2pad) * sizeof(float4) + 64;
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, "flash_tc_ops", bytes, &p));
  char * q = static_cast<char *>(p);
  auto take = [&](size_t n) { char * r = q; q += (n + 255) & ~size_t(255); return r; };
  auto * psi1hi = reinterpret_cast<__nv_bfloat16 *>(take(size_t(n1pad) * RP * bf));
  auto * psi1lo = reinterpret_cast<__nv_bfloat16 *>(take(size_t(n1pad) * RP * bf));
  auto * psi2hi = reinterpret_cast<__nv_bfloat16 *>(take(size_t(n2pad) * RP * bf));
  auto * psi2lo = reinterpret_cast<__nv_bfloat16 *>(take(size_t(n2pad) * RP * bf));
  auto * vthi = reinterpret_cast<__nv_bfloat16 *>(take(size_t(NB) * n2pad * bf));
  auto * vtlo = reinterpret_cast<__nv_bfloat16 *>(take(size_t(NB) * n2pad * bf));
  auto * r1c = reinterpret_cast<float4 *>(take(size_t(n1pad) * sizeof(float4)));
  auto * r2c = reinterpret_cast<float4 *>(take(size_t(n2pad) * sizeof(float4)));
  int * status = reinterpret_cast<int *>(take(64));
  bool const haveVt = c.vtHi && c.vtLo;
  TCSCF_CHECK(ctx, size_t(q - static_cast<char *>(p)) <= bytes + 16 * 256, TCSCF_ERR_INVALID_ARGUMENT, "internal: scratch layout");

  // operand preparation (BF16 hi/lo split, transposes, FP32 coordinates)
  tc::kPackPsi<<<gridBlocks(n1pad * RP, 256), 256, 0, ctx->stream>>>(c.n1, n1pad, c.R, RP, c.psi1, c.ldpsi, psi1hi, psi1lo);
  TCSCF_LAUNCH(ctx);
  tc::kPackPsi<<<gridBlocks(n2pad * RP, 256), 256, 0, ctx->stream>>>(c.n2, n2pad, c.R, RP, c.psi2, c.ldpsi, psi2hi, psi2lo);
  TCSCF_LAUNCH(ctx);
  dim3 const tb{32, 8, 1};
  dim3 const tg{unsigned((n2pad + 31) / 32), unsigned((NB + 31) / 32), 1};
  if (haveVt) {
    vthi = static_cast<__nv_bfloat16 *>(const_cast<void *>(c.vtHi));
    vtlo = static_cast<__nv_bfloat16 *>(const_cast<void *>(c.vtLo));
  } else {
    tc::kPackVt<<<tg, tb, 0, ctx->stream>>>(c.n2, n2pad, c.ncol, NB, c.V, c.ldv, vthi, vtlo);
    TCSCF_LAUNCH(ctx);
  }
  tc::kPackCoords<<<gridBlocks(n1pad, 256), 256, 0, ctx->stream>>>(c.n1, n1pad, c.p1, nullptr, r1c);
  TCSCF_LAUNCH(ctx);
  tc::kPackCoordPairs<<<gridBlocks(n2pad / 2, 256), 256, 0, ctx->stream>>>(c.n2, n2pad, c.p2, c.coul, r2c);
  TCSCF_LAUNCH(ctx);

  CUtensorMap maps[6];
  CUtensorMapSwizzle const psw = RP == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B;
  bool okm = makeMap(&maps[0], psi1hi, RP, n1pad, RP, tc::BM, psw)
             && makeMap(&maps[1], psi1lo, RP, n1pad, RP, tc::BM, psw)
             && makeMap(&maps[2], psi2hi, RP, n2pad, RP, tc::BK, psw)
             && makeMap(&maps[3], psi2lo, RP, n2pad, RP, tc::BK, psw)
             && makeMap(&maps[4], vthi, n2pad, NB, tc::BK, NB, CU_TENSOR_MAP_SWIZZLE_128B)
             && makeMap(&maps[5], vtlo, n2pad, NB, tc::BK, NB, CU_TENSOR_MAP_SWIZZLE_128B);
  TCSCF_CHECK(ctx, okm, TCSCF_ERR_CUDA, "cuTensorMapEncodeTiled failed");

  double * Tout = c.T;
  double * VHout = c.VH;
  void * sp = nullptr;
  if (nSplit > 1 || !c.VH) {
    // split partials (and a Coulomb sink when the caller does not want the potential)
    TCSCF_TRY(scratch(ctx, "flash_tc_split", sizeof(double) * size_t(nSplit) * c.n1 * (c.ldt + 1), &sp));
    if (nSplit > 1) Tout = static_cast<double *>(sp);
    VHout = static_cast<double *>(sp) + size_t(nSplit) * c.n1 * c.ldt;
  }
  TCSCF_CUDA(ctx, cudaMemsetAsync(VHout, 0, sizeof(double) * size_t(nSplit) * c.n1, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemsetAsync(status, 0, sizeof(int), ctx->stream));

  tc::Params P{};
  P.nTiles = nTiles; P.nSplit = nSplit; P.blocksPerSplit = perSplit; P.nBlocks = nBlocks;
  P.n1 = int(c.n1); P.nb = c.ncol; P.window = ctx->flushWindow;
  P.r1xyz = r1c; P.r2xyzc = r2c; P.T = Tout; P.VH = VHout; P.ldt = c.ldt;
  P.tStride = int64_t(c.n1) * c.ldt; P.vhStride = c.n1; P.status = status;
  int const grid = std::min(nTiles * nSplit, sms);
  if (NB == 64 && RP == 32) TCSCF_TRY((launchFlash<64, 32>(ctx, maps, P, grid)));
  else if (NB == 64) TCSCF_TRY((launchFlash<64, 64>(ctx, maps, P, grid)));
  else if (RP == 32) TCSCF_TRY((launchFlash<128, 32>(ctx, maps, P, grid)));
  else TCSCF_TRY((launchFlash<128, 64>(ctx, maps, P, grid)));

  int st = 0;
  TCSCF_CUDA(ctx, cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (st != 0) return fail(ctx, TCSCF_ERR_TIMEOUT, "tensor-core contraction: bounded wait expired (code " + std::to_string(st) + ")");
  if (nSplit > 1) {
    int64_t const n = int64_t(c.n1) * c.ncol;
    TCSCF_TRY(sumSplitsLaunch(ctx, n, nSplit, int64_t(c.n1) * c.ldt, Tout, c.T, c.n1, c.ncol, c.ldt, c.ldt));
    if (c.VH) TCSCF_TRY(sumSplitsLaunch(ctx, c.n1, nSplit, c.n1, VHout, c.VH, c.n1, 1, 1, 1));
  }
  return TCSCF_OK;
}

}  // namespace tcscf
