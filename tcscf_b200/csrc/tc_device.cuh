// Device-side pieces shared by the tcgen05 flash contraction kernels (split-BF16 flash_tc.cu and
// TF32 flash_tf32.cu): tile sizes, warp roles and register split, work-item decoding, and PTX wrappers
// for mbarriers, TMA, TMEM loads, tcgen05 fences and packed FP32 pair arithmetic.
#pragma once

#include <cuda.h>
#include <cstdint>

#include "kernels.cuh"

namespace tcscf {
namespace tc {

constexpr int BM = 128;        // r1 rows per tile
constexpr int BK = 64;         // r2 points per block

constexpr int NCW = 8;         // compute warps
constexpr int NTHREADS = 384;  // warpgroup 0: TMA, MMA, 2 idle warps; warpgroups 1-2: compute
// register split: 384 threads x 168 at launch = 64512 = 128 x 56 (producer warpgroup) + 256 x 224
constexpr int kRegsLaunch = 168, kRegsProducer = 56, kRegsCompute = 224;
static_assert(128 * kRegsProducer + 256 * kRegsCompute <= NTHREADS * kRegsLaunch, "register split exceeds the launch allocation");
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s per wait
constexpr float kMinNormal = 1.17549435e-38f;                // smallest normal FP32 (2^-126)
// Pairs closer than 2^-16 |r1| are below what FP32 coordinates resolve (their rounding, 2^-24 |r| per
// coordinate, is then more than 1/256 of the separation).  The tensor kernels drop every pair whose FP32
// squared separation is below nearThreshold(r1) (never below the smallest normal FP32, where the
// rsqrt estimate turns the Newton step into NaN), and the near-pair correction (near_pairs.cu) adds
// the pairs that are not exactly coincident back with their FP64 value, so the mixed paths follow the
// FP64 rule: only an exactly coincident pair contributes 0.  Evaluated with explicit round-to-nearest
// operations (no contraction), so every kernel that packs or tests a point gets the same bits.
__device__ __forceinline__ float nearThreshold(float x, float y, float z)
{
  float const s = __fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z));
  return fmaxf(kMinNormal, __fmul_rn(s, 2.3283064365386963e-10f));   // 2^-32 |r1|^2
}
// a waiting thread sleeps in mbarrier.try_wait (woken when the phase completes) instead of spinning
// on the issue slots the compute warps need
constexpr uint32_t kSuspendHintNs = 1000000;

using Instance = TensorInstance;
constexpr int kMapsPerInstance = kTensorMapsPerInstance;

struct Params {
  int nItems;
  const int4 * items;       // work items (instance, r1 tile, r2 split, 0); null: one instance, item = tile * nSplit + split
  const Instance * inst;    // [instances] in device memory
  int * status;             // device status word (0 = ok)
};

// the r2 blocks [jb, je) of work item (tile, split): all blocks, or for a symmetric instance those from
// the tile's own diagonal block (BM / BK blocks per tile) on; empty (je == jb) past the last block
__host__ __device__ __forceinline__ void itemBlocks(Instance const & I, int tile, int split, int & jb, int & je)
{
  jb = (I.sym ? tile * (BM / BK) : 0) + split * I.blocksPerSplit;
  je = jb + I.blocksPerSplit < I.nBlocks ? jb + I.blocksPerSplit : I.nBlocks;
  if (je < jb) je = jb;
}

__device__ __forceinline__ void decodeItem(Params const & P, int item, int & inst, int & tile, int & split)
{
  if (P.items) {
    int4 const it = P.items[item];
    inst = it.x; tile = it.y; split = it.z;
  } else {
    int const ns = P.inst[0].nSplit;
    inst = 0; tile = item / ns; split = item % ns;
  }
}

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

// Bounded wait; returns false (after recording the failure) when limitNs of wall-clock time pass or
// another role has already aborted.
__device__ __forceinline__ bool waitBarLimit(uint64_t * b, uint32_t parity, volatile int * abortFlag, int * status, int code,
                                             unsigned long long limitNs)
{
  if (mbarTryWait(b, parity)) return true;
  unsigned long long const t0 = globalTimer();
  while (true) {
    if (mbarTryWait(b, parity)) return true;
    if (*abortFlag) return false;
    if (globalTimer() - t0 > limitNs) {
      *abortFlag = 1;
      atomicCAS(status, 0, code);
      return false;
    }
  }
}
__device__ __forceinline__ bool waitBar(uint64_t * b, uint32_t parity, volatile int * abortFlag, int * status, int code)
{
  return waitBarLimit(b, parity, abortFlag, status, code, kWaitLimitNs);
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
__device__ __forceinline__ void tmemLoad8(uint32_t taddr, float * v)
{
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmemWaitLoad8(float (&a)[8], float (&b)[8])
{
  asm volatile("tcgen05.wait::ld.sync.aligned;" : "+f"(a[0]), "+f"(a[1]), "+f"(a[2]), "+f"(a[3]), "+f"(a[4]), "+f"(a[5]), "+f"(a[6]), "+f"(a[7]) :: "memory");
  asm volatile("" : "+f"(b[0]), "+f"(b[1]), "+f"(b[2]), "+f"(b[3]), "+f"(b[4]), "+f"(b[5]), "+f"(b[6]), "+f"(b[7]) :: "memory");
}
// wait for the outstanding TMEM loads into a and b; the register operands keep every use of a and b
// after the wait (the asm statements are volatile, so their order is kept)
__device__ __forceinline__ void tmemWaitLoad(float (&a)[16], float (&b)[16])
{
  asm volatile("tcgen05.wait::ld.sync.aligned;" : "+f"(a[0]), "+f"(a[1]), "+f"(a[2]), "+f"(a[3]), "+f"(a[4]), "+f"(a[5]), "+f"(a[6]), "+f"(a[7]), "+f"(a[8]), "+f"(a[9]), "+f"(a[10]), "+f"(a[11]), "+f"(a[12]), "+f"(a[13]), "+f"(a[14]), "+f"(a[15]) :: "memory");
  asm volatile("" : "+f"(b[0]), "+f"(b[1]), "+f"(b[2]), "+f"(b[3]), "+f"(b[4]), "+f"(b[5]), "+f"(b[6]), "+f"(b[7]), "+f"(b[8]), "+f"(b[9]), "+f"(b[10]), "+f"(b[11]), "+f"(b[12]), "+f"(b[13]), "+f"(b[14]), "+f"(b[15]) :: "memory");
}

// ---- packed FP32 pairs (sm_100 f32x2 arithmetic on 64-bit register pairs) ---------------------
__device__ __forceinline__ uint64_t f2pack(float a, float b)
{
  uint64_t d;
  asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(a), "f"(b));
  return d;
}
__device__ __forceinline__ void f2unpack(uint64_t v, float & a, float & b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v)); }
__device__ __forceinline__ uint64_t f2add(uint64_t a, uint64_t b)
{
  uint64_t d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
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

}  // namespace tc

// TF32 path (flash_tf32.cu): bytes of its packed operands (psi1, psi2 and Vt as TF32-rounded FP32),
// their packing into dst with the three tensor maps (psi1, psi2, Vt), and the launch of one tile class
size_t tf32OperandBytes(int NB, int64_t n1pad, int64_t n2pad);
int tf32PackOperands(tcscf_ctx * ctx, Contraction const & c, int NB, int64_t n1pad, int64_t n2pad, void * dst, CUtensorMap * maps);
int launchTf32(tcscf_ctx * ctx, int NB, tc::Params const & P, int grid);

// operand packing shared by the tensor kernels (flash_tc.cu): the transposed fixed-point BF16 slices
// h / m / l/256 [NB][n2pad] of V [n2][ldv] (nb real columns) followed by the per-(r2 block, column)
// inverse scales [n2pad/64][NB]; points [3][n] as FP32 float4 {x, y, z, 0} [npad]; points in pairs
// {x0,x1,y0,y1}{z0,z1,c0,c1} [npad] with the Coulomb source c (0 when coul is null).  Padding points
// sit far away.
size_t packedVtOperandBytes(int NB, int64_t n2pad);
int packVtOperand(tcscf_ctx * ctx, int64_t n2, int64_t n2pad, int nb, int NB, const double * V, int ldv, void * out);
int packPointsFp32(tcscf_ctx * ctx, int64_t n, int64_t npad, const double * pts, float4 * out);
int packPointPairsFp32(tcscf_ctx * ctx, int64_t n, int64_t npad, const double * pts, const double * coul, float4 * out);

// cuTensorMapEncodeTiled from the CUDA driver API (null when unavailable)
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *, const cuuint64_t *,
                                   const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encodeTiled();
// 2-D tensor map over a row-major [outer][inner] array (elemBytes per element), box (boxInner, boxOuter)
bool makeMap2d(CUtensorMap * m, CUtensorMapDataType type, uint32_t elemBytes, void * base, uint64_t inner, uint64_t outer, uint32_t boxInner,
               uint32_t boxOuter, CUtensorMapSwizzle sw);

}  // namespace tcscf
