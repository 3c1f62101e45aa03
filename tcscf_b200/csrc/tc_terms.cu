// Transcorrelated (TC) per-iteration Fock build and the TC SCF driver (FP64).
//
// TCHartreeFock (HartreeFock.cpp:102-609 per-point terms, :1105-1261 iteration, :1150-1224 assembly)
// builds, from the stored scalar tensors Fji (same / opposite spin TC kernels, computeF) and the
// vector tensors Vji (grad u, computeV) on the r1 grid:
//   G2 = two-body scalar + (vector - vector^dagger) terms,  G3 = three-body term,
//   F = h + G2 - G3,  E = sum D(i,j) (h + G2/2 - G3/3)(j,i)                        (HartreeFock.cpp:83-92)
// Each per-point intermediate of the reference (scaled gradients, Vai, Vja, Vjb, Vab norms, V-tilde,
// V-tilde_i, sum_b V_bi . V-tilde_b, occupied density, sum_b conj(V-tilde_b) occ_b) is one kernel
// over (spin, r1[, i]) here; the (j, i) matrix elements are block reductions over r1.  The SCF
// step solves the non-Hermitian pencil F C = S C e on the GPU: S = L L^H (cuSOLVER potrf),
// L^-1 F L^-H (cuBLAS trsm), the general eigen-solve cusolverDnXgeev, C = L^-H Y; then, as the
// reference does (:1298-1353), eigenvalues are sorted by real part and the occupied vectors are
// orthogonalised with the S-metric modified Gram-Schmidt of orthogonalization.hpp:136-154, whose
// vectors after the first are normalised with the Euclidean norm (:152).
#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

#include <cublas_v2.h>

#include "kernels.cuh"
#include "tc_device.cuh"

namespace tcscf {
namespace {

struct Z3 {
  double2 x, y, z;
};

__device__ __forceinline__ double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 zsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 zmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 zconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 zscale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__device__ __forceinline__ Z3 z3load(const double2 * p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ void z3store(double2 * p, Z3 const & a) { p[0] = a.x; p[1] = a.y; p[2] = a.z; }
__device__ __forceinline__ Z3 z3zero() { return {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)}; }
__device__ __forceinline__ void z3axpy(Z3 & a, double2 s, Z3 const & b)
{
  a.x = zadd(a.x, zmul(s, b.x));
  a.y = zadd(a.y, zmul(s, b.y));
  a.z = zadd(a.z, zmul(s, b.z));
}
__device__ __forceinline__ double2 z3dot(Z3 const & a, Z3 const & b) { return zadd(zadd(zmul(a.x, b.x), zmul(a.y, b.y)), zmul(a.z, b.z)); }
__device__ __forceinline__ Z3 z3conj(Z3 const & a) { return {zconj(a.x), zconj(a.y), zconj(a.z)}; }
__device__ __forceinline__ double z3norm(Z3 const & a)
{
  return a.x.x * a.x.x + a.x.y * a.x.y + a.y.x * a.y.x + a.y.y * a.y.y + a.z.x * a.z.x + a.z.y * a.z.y;
}

// Device view of one TC build: inputs and the per-point intermediates ([2] = spin).
struct TcView {
  int64_t n1;
  int nb, nelMax;
  int nel[2];
  int fcx;                               // Fji complex (3-D r2 grid) or real
  const double * Fs;                     // [n1][nb][nb]
  const double * Fo;
  const double2 * Vs;                    // [n1][nb][nb][3]
  const double2 * Vo;
  const double2 * vals;                  // [n1][nb]
  const double2 * grads;                 // [n1][nb][3]
  const double * w;                      // [n1]
  const double2 * D;                     // [2][nb][nb], D_s(i,j) at [s][i][j]
  const double2 * C0;                    // occupied orbitals of spin 0: (i, b) at [b*nb + i]
  const double2 * C1;
  double2 * Faa;                         // [2][n1]
  double2 * Fai;                         // [2][n1][nb]
  double2 * VT;                          // [2][n1][3]   V-tilde (= VaaSPO)
  double2 * SG;                          // [2][n1][3]   scaled gradients
  double * occD;                         // [2][n1]
  double2 * Vai;                         // [2][n1][nb]
  double2 * Vja;                         // [2][n1][nb][3]
  double2 * VTs;                         // [2][n1][nb][3] V-tilde_i
  double2 * Vjbs;                        // [2][n1][nb][nelMax][3]
  double2 * Vjbo;
  double * sumNs;                        // [2][n1]
  double * sumNo;
  double2 * SVD;                         // [2][n1][nb]  sum_b V_bi . V-tilde_b
  double2 * SCV;                         // [2][n1][3]   sum_b conj(V-tilde_b) occ_b
};

__device__ __forceinline__ double2 fget(TcView const & t, const double * F, int64_t r, int j, int i)
{
  int64_t const o = (r * t.nb + j) * t.nb + i;
  return t.fcx ? reinterpret_cast<const double2 *>(F)[o] : make_double2(F[o], 0.0);
}
__device__ __forceinline__ Z3 vget(TcView const & t, const double2 * V, int64_t r, int j, int i)
{
  return z3load(V + ((r * t.nb + j) * t.nb + i) * 3);
}
__device__ __forceinline__ double2 dget(TcView const & t, int s, int i, int j) { return t.D[(int64_t(s) * t.nb + i) * t.nb + j]; }
__device__ __forceinline__ double2 cget(TcView const & t, int s, int i, int b) { return (s == 0 ? t.C0 : t.C1)[int64_t(b) * t.nb + i]; }
__device__ __forceinline__ Z3 gget(TcView const & t, int64_t r, int k) { return z3load(t.grads + (r * t.nb + k) * 3); }

#define TC_GRID_LOOP(total) for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < (total); idx += int64_t(gridDim.x) * blockDim.x)

// per (spin, r1): Faa (calculateIaa on both Fji, :1119-1124), V-tilde (calculateIaa on Vji :1125-1126
// and calculateVTilde :397-434 are the same sum), scaled gradients (:102-140), occupied density (:530-567)
__global__ void kTcPoint(TcView t)
{
  int const nb = t.nb;
  TC_GRID_LOOP(2 * t.n1)
  {
    int const s = int(idx / t.n1), so = 1 - s;
    int64_t const r = idx % t.n1;
    double2 faa = make_double2(0, 0), occ = make_double2(0, 0);
    Z3 vt = z3zero(), sg = z3zero();
    for (int j = 0; j < nb; ++j) {
      double2 const cvj = zconj(t.vals[r * nb + j]);
      for (int i = 0; i < nb; ++i) {
        double2 const ds = dget(t, s, i, j), dop = dget(t, so, i, j);
        faa = zadd(faa, zadd(zmul(fget(t, t.Fs, r, j, i), ds), zmul(fget(t, t.Fo, r, j, i), dop)));
        z3axpy(vt, ds, vget(t, t.Vs, r, j, i));
        z3axpy(vt, dop, vget(t, t.Vo, r, j, i));
        z3axpy(sg, zmul(ds, cvj), gget(t, r, i));
      }
    }
    for (int k = 0; k < nb; ++k) {
      double2 const cvk = zconj(t.vals[r * nb + k]);
      for (int l = 0; l < nb; ++l) occ = zadd(occ, zmul(zmul(dget(t, s, l, k), cvk), t.vals[r * nb + l]));
    }
    t.Faa[idx] = faa;
    z3store(t.VT + idx * 3, vt);
    z3store(t.SG + idx * 3, sg);
    t.occD[idx] = occ.x;
  }
}

// per (spin, r1, i): Fai (calculateFai, :1127), Vai (:217-252), Vja (:256-291, row j = i here) and
// V-tilde_i (:438-480)
__global__ void kTcPointI(TcView t)
{
  int const nb = t.nb;
  TC_GRID_LOOP(2 * t.n1 * nb)
  {
    int const i = int(idx % nb);
    int64_t const sr = idx / nb;
    int const s = int(sr / t.n1);
    int64_t const r = sr % t.n1;
    double2 fai = make_double2(0, 0), vai = make_double2(0, 0);
    Z3 vts = z3zero(), vja = z3zero();
    for (int j = 0; j < nb; ++j) {
      double2 kv = make_double2(0, 0), kc = make_double2(0, 0);
      Z3 kg = z3zero();
      for (int k = 0; k < nb; ++k) {
        kv = zadd(kv, zmul(dget(t, s, k, j), t.vals[r * nb + k]));
        z3axpy(kg, dget(t, s, k, j), gget(t, r, k));
        kc = zadd(kc, zmul(dget(t, s, j, k), zconj(t.vals[r * nb + k])));
      }
      Z3 const vji = vget(t, t.Vs, r, j, i);
      fai = zadd(fai, zmul(kv, fget(t, t.Fs, r, j, i)));
      vai = zadd(vai, z3dot(vji, kg));
      z3axpy(vts, kv, vji);                              // sum_k (sum_l D(l,k) v_l) V(k,i), k := j
      z3axpy(vja, kc, vget(t, t.Vs, r, i, j));           // row i of Vja: sum_j (sum_k D(j,k) v_k^*) V(i,j)
    }
    t.Fai[idx] = fai;
    t.Vai[idx] = vai;
    z3store(t.VTs + idx * 3, vts);
    z3store(t.Vja + idx * 3, vja);
  }
}

// per (spin, r1, j, b < nel): Vjb for the same- and opposite-spin tensors (calculateVjb, :295-337)
__global__ void kTcVjb(TcView t)
{
  int const nb = t.nb, nm = t.nelMax;
  TC_GRID_LOOP(2 * t.n1 * nb * nm)
  {
    int const b = int(idx % nm);
    int64_t k = idx / nm;
    int const j = int(k % nb);
    k /= nb;
    int const s = int(k / t.n1);
    int64_t const r = k % t.n1;
    Z3 rs = z3zero(), ro = z3zero();
    if (b < t.nel[s]) {
      for (int i = 0; i < nb; ++i) {
        double2 const c = cget(t, s, i, b);
        z3axpy(rs, c, vget(t, t.Vs, r, j, i));
        z3axpy(ro, c, vget(t, t.Vo, r, j, i));
      }
    }
    z3store(t.Vjbs + idx * 3, rs);
    z3store(t.Vjbo + idx * 3, ro);
  }
}

// per (spin, r1): sum_ab |Vab|^2 for both tensors (calculateVab, :341-393), and
// sum_b conj(V-tilde_b) occ_b (:571-609)
__global__ void kTcVab(TcView t)
{
  int const nb = t.nb, nm = t.nelMax;
  TC_GRID_LOOP(2 * t.n1)
  {
    int const s = int(idx / t.n1);
    int64_t const r = idx % t.n1;
    int const ne = t.nel[s];
    double ns = 0, no = 0;
    for (int a = 0; a < ne; ++a)
      for (int b = 0; b < ne; ++b) {
        Z3 rs = z3zero(), ro = z3zero();
        for (int j = 0; j < nb; ++j) {
          double2 const cc = zconj(cget(t, s, j, a));
          int64_t const o = ((idx * nb + j) * nm + b) * 3;
          z3axpy(rs, cc, z3load(t.Vjbs + o));
          z3axpy(ro, cc, z3load(t.Vjbo + o));
        }
        ns += z3norm(rs);
        no += z3norm(ro);
      }
    t.sumNs[idx] = ns;
    t.sumNo[idx] = no;
    Z3 cs = z3zero();
    for (int k = 0; k < nb; ++k) {
      Z3 const vk = z3conj(z3load(t.VTs + (idx * nb + k) * 3));
      for (int l = 0; l < nb; ++l) z3axpy(cs, zmul(dget(t, s, l, k), t.vals[r * nb + l]), vk);
    }
    z3store(t.SCV + idx * 3, cs);
  }
}

// per (spin, r1, i): sum_k V(k,i) . (sum_l D(l,k) V-tilde_l)   (calculateSumOverb_Vbi_dot_VTildeb, :484-526)
__global__ void kTcSvd(TcView t)
{
  int const nb = t.nb;
  TC_GRID_LOOP(2 * t.n1 * nb)
  {
    int const i = int(idx % nb);
    int64_t const sr = idx / nb;
    int const s = int(sr / t.n1);
    int64_t const r = sr % t.n1;
    double2 acc = make_double2(0, 0);
    for (int k = 0; k < nb; ++k) {
      Z3 ell = z3zero();
      for (int l = 0; l < nb; ++l) z3axpy(ell, dget(t, s, l, k), z3load(t.VTs + (sr * nb + l) * 3));
      acc = zadd(acc, z3dot(vget(t, t.Vs, r, k, i), ell));
    }
    t.SVD[idx] = acc;
  }
}

// one block per (spin, j, i): the r1 sums of the scalar, vector and three-body terms (:1150-1216);
// out[0] = scalar, out[1] = vector, out[2] = scalar3, each [2][nb][nb]
__global__ void kTcReduce(TcView t, double2 * out)
{
  int const nb = t.nb, nn = nb * nb, nm = t.nelMax;
  int const s = blockIdx.x / nn, so = 1 - s, ji = blockIdx.x % nn, j = ji / nb, i = ji % nb;
  int const ne = t.nel[s];
  double2 sc = make_double2(0, 0), ve = make_double2(0, 0), s3 = make_double2(0, 0);
  for (int64_t r = threadIdx.x; r < t.n1; r += blockDim.x) {
    int64_t const ps = int64_t(s) * t.n1 + r, po = int64_t(so) * t.n1 + r;
    double const w = t.w[r];
    double2 const vi = t.vals[r * nb + i], cvj = zconj(t.vals[r * nb + j]);
    Z3 const gi = gget(t, r, i);
    Z3 const vsji = vget(t, t.Vs, r, j, i), voji = vget(t, t.Vo, r, j, i);
    // two-body scalar
    sc = zadd(sc, zscale(w, zmul(cvj, zsub(zmul(t.Faa[ps], vi), t.Fai[ps * nb + i]))));
    // two-body vector
    Z3 const vt = z3load(t.VT + ps * 3), vto = z3load(t.VT + po * 3);
    double2 va = zmul(cvj, zsub(z3dot(vt, gi), t.Vai[ps * nb + i]));
    va = zadd(va, z3dot(vsji, z3load(t.SG + ps * 3)));
    va = zadd(va, z3dot(voji, z3load(t.SG + po * 3)));
    va = zsub(va, z3dot(z3load(t.Vja + (ps * nb + j) * 3), gi));
    ve = zadd(ve, zscale(w, va));
    // three-body
    Z3 const vti = z3load(t.VTs + (ps * nb + i) * 3), vtj = z3load(t.VTs + (ps * nb + j) * 3);
    double2 x = zmul(zscale(z3norm(vt) - t.sumNs[ps] - t.sumNo[po], cvj), vi);
    x = zadd(x, zscale(2.0, zmul(cvj, zsub(t.SVD[ps * nb + i], z3dot(vt, vti)))));
    x = zadd(x, zscale(2.0, zmul(zsub(zconj(t.SVD[ps * nb + j]), z3dot(z3conj(vtj), vt)), vi)));
    double2 sbS = make_double2(0, 0), sbO = make_double2(0, 0);
    for (int b = 0; b < ne; ++b) {
      int64_t const oj = ((ps * nb + j) * nm + b) * 3, oi = ((ps * nb + i) * nm + b) * 3;
      sbS = zadd(sbS, z3dot(z3load(t.Vjbs + oj), z3conj(z3load(t.Vjbs + oi))));
      sbO = zadd(sbO, z3dot(z3load(t.Vjbo + oj), z3conj(z3load(t.Vjbo + oi))));
    }
    x = zadd(x, zscale(2.0 * t.occD[ps], zsub(z3dot(vsji, vt), sbS)));
    x = zadd(x, zscale(2.0, zsub(z3dot(vti, z3conj(vtj)), z3dot(vsji, z3load(t.SCV + ps * 3)))));
    x = zadd(x, zscale(2.0 * t.occD[po], zsub(z3dot(voji, vto), sbO)));
    x = zsub(x, zscale(2.0, z3dot(voji, z3load(t.SCV + po * 3))));
    s3 = zadd(s3, zscale(w, x));
  }
  double v[6] = {sc.x, sc.y, ve.x, ve.y, s3.x, s3.y};
#pragma unroll
  for (int q = 0; q < 6; ++q)
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
  __shared__ double red[6][32];
  int const lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
    for (int q = 0; q < 6; ++q) red[q][wid] = v[q];
  __syncthreads();
  if (threadIdx.x == 0) {
    double a[6] = {0, 0, 0, 0, 0, 0};
    for (int k = 0; k < int(blockDim.x >> 5); ++k)
      for (int q = 0; q < 6; ++q) a[q] += red[q][k];
    for (int q = 0; q < 3; ++q) out[int64_t(q) * 2 * nn + blockIdx.x] = make_double2(a[2 * q], a[2 * q + 1]);
  }
}

// G2 = scalar/2 + vec - vec^dagger with vec = vector/2, G3 = scalar3/2; masked where h == 0 when
// respectSym (enforceOneElectronSymmetry, :758-780)
__global__ void kTcAssemble(int nb, const double2 * sums, const double * h, int respectSym, double2 * G2, double2 * G3)
{
  int const nn = nb * nb;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < 2 * nn; idx += gridDim.x * blockDim.x) {
    int const s = idx / nn, ji = idx % nn, j = ji / nb, i = ji % nb;
    double2 const scal = sums[idx], vec = sums[2 * nn + idx], vecT = sums[2 * nn + s * nn + i * nb + j], s3 = sums[4 * nn + idx];
    double2 g2 = make_double2(0.5 * scal.x + 0.5 * vec.x - 0.5 * vecT.x, 0.5 * scal.y + 0.5 * vec.y + 0.5 * vecT.y);
    double2 g3 = make_double2(0.5 * s3.x, 0.5 * s3.y);
    if (respectSym && !(fabs(h[ji]) > 0)) { g2 = make_double2(0, 0); g3 = make_double2(0, 0); }
    G2[idx] = g2;
    G3[idx] = g3;
  }
}

// column-major copy of a row-major square matrix (out(j,i) = in[j][i])
__global__ void kToColMajorZ(int nb, const double2 * in, double2 * out)
{
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nb * nb; idx += gridDim.x * blockDim.x) {
    int const j = idx / nb, i = idx % nb;
    out[i * nb + j] = in[idx];
  }
}
__global__ void kRealToZ(int n, const double * in, double2 * out)
{
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) out[idx] = make_double2(in[idx], 0.0);
}

// ---- fused per-point build (nb <= kFusedMaxNb) -------------------------------------------------------
// The kernels above keep every per-point intermediate in HBM and read the Fji / Vji tensors several
// times over (once per intermediate, then again in the reduction, with each thread walking its own
// point's rows).  kTcFused reads them once: one block of kFusedThreads per SM walks the r1 points
// (p = block, block + grid, ...); a point's Vs, Vo ([nb][nb][3] complex), Fs, Fo ([nb][nb]) rows, basis
// values and gradients arrive in shared memory by bulk copies (double-buffered when two points fit);
// all intermediates of kTcPoint ... kTcSvd are formed there for both spins from that one copy, and
// each thread adds the w-weighted scalar, vector and three-body terms of kTcReduce for its fixed
// (spin, j, i) elements in registers.  The per-block sums go to part[block][3][2][nb][nb] and
// kTcPartials adds them in block order (deterministic).  Same terms as kTcReduce, grouped per point:
//   scalar  += conj(v_j) Pw(i)
//   vector  += conj(v_j) Qw(i) + Vs(j,i).w SG_s + Vo(j,i).w SG_o - Vja_s(j).w g_i
//   three   += conj(v_j) Rw(i) + Tw(j) v_i + 2w VTs(i).conj(VTs(j))
//              - 2w occ_s sum_b Vjbs(j,b).conj(Vjbs(i,b)) - 2w occ_o sum_b Vjbo(j,b).conj(Vjbo(i,b))
//              + Vs(j,i).w (2 occ_s VT_s - 2 SCV_s) + Vo(j,i).w (2 occ_o VT_o - 2 SCV_o)
// with Pw = w (Faa v_i - Fai(i)), Qw = w (VT.g_i - Vai(i)), Rw = w ((|VT|^2 - sumNs_s - sumNo_o) v_i
// + 2 (SVD(i) - VT.VTs(i))), Tw = 2w (conj(SVD(j)) - conj(VTs(j)).VT).
constexpr int kFusedThreads = 512;
constexpr int kFusedMaxNb = 32;   // 2 nb^2 elements over 512 threads: at most 4 register slots
constexpr int kFusedWaitCode = 60;

__device__ __forceinline__ double2 zfma(double2 a, double2 b, double2 c)   // a b + c
{
  return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
__device__ __forceinline__ double2 zcfma(double2 a, double2 b, double2 c)  // conj(a) b + c
{
  return make_double2(fma(a.x, b.x, fma(a.y, b.y, c.x)), fma(a.x, b.y, fma(-a.y, b.x, c.y)));
}

// shared-memory layout of kTcFused in double2 units (per-spin arrays are [2][...]); the same
// arithmetic on the host sizes the launch
struct FusedLayout {
  int ldD, fU;
  int D, C, kv, kc, kg, colF, colV, Fai, VTs, Vai, Vja, Vjb, nP, ell, sc, Pw, Qw, Rw, Tw, Xw, Jw, gw, ws;
  int buf, bufStride, total;
  __host__ __device__ FusedLayout(int nb, int nm, int fcx, int nbuf)
  {
    int const nn = nb * nb;
    ldD = (nb & 1) ? nb : nb + 1;   // odd row stride: a warp walking a column of D hits distinct banks
    fU = fcx ? nn : nn / 2;         // real Fji rows (nb even) take half the double2 slots
    int o = 0;
    D = o;    o += 2 * nb * ldD;     // D_s(i, j) at [s][i][j]
    C = o;    o += 2 * nm * nb;      // C_s(i, b) at [s][b][i], zero for b >= nel[s]
    kv = o;   o += 2 * nb;           // sum_k D(k, j) v_k
    kc = o;   o += 2 * nb;           // sum_k D(j, k) conj(v_k)
    kg = o;   o += 6 * nb;           // sum_k D(k, j) g_k
    colF = o; o += 2 * nb;           // column i of the Faa trace
    colV = o; o += 6 * nb;           // column i of the V-tilde trace
    Fai = o;  o += 2 * nb;
    VTs = o;  o += 6 * nb;
    Vai = o;  o += 2 * nb;
    Vja = o;  o += 6 * nb;
    Vjb = o;  o += 12 * nb * nm;     // [s][tensor][j][b][3]
    nP = o;   o += 4 * nm * nm;      // |sum_j conj(C(j,a)) Vjb(j,b)|^2 at [s][tensor][a][b] (.x)
    ell = o;  o += 6 * nb;           // sum_l D(l, k) VTs(l)
    sc = o;   o += 24;               // per spin: Faa, VT[3], SG[3], SCV[3], occ (.x), sumN (.x same, .y oppo)
    Pw = o;   o += 2 * nb;
    Qw = o;   o += 2 * nb;
    Rw = o;   o += 2 * nb;
    Tw = o;   o += 2 * nb;
    Xw = o;   o += 6 * nb;
    Jw = o;   o += 12 * nb * nm;
    gw = o;   o += 3 * nb;
    ws = o;   o += 24;               // per spin: w SG_s, w SG_o, w (2 occ_s VT_s - 2 SCV_s), w (2 occ_o VT_o - 2 SCV_o)
    buf = o;
    bufStride = 6 * nn + 2 * fU + 4 * nb;   // Vs, Vo, Fs, Fo, vals, grads
    total = buf + nbuf * bufStride;
  }
  __host__ __device__ size_t bytes() const { return size_t(total) * sizeof(double2) + 32; }   // + 2 mbarriers, abort word
};

struct TcFusedArgs {
  int64_t n1;
  int nb, nm, nbuf, fcx;
  int nel[2];
  const double * Fs;
  const double * Fo;
  const double2 * Vs;
  const double2 * Vo;
  const double2 * vals;
  const double2 * grads;
  const double * w;
  const double2 * D;
  const double2 * C0;
  const double2 * C1;
  double2 * part;   // [gridDim.x][3][2][nb][nb]
  int * status;
};

template <int SLOTS>
__global__ void __launch_bounds__(kFusedThreads, 1) kTcFused(TcFusedArgs t)
{
  extern __shared__ __align__(16) double2 sm[];
  int const nb = t.nb, nn = nb * nb, nm = t.nm, tid = threadIdx.x;
  FusedLayout const L(nb, nm, t.fcx, t.nbuf);
  int const ld = L.ldD;
  uint64_t * bars = reinterpret_cast<uint64_t *>(sm + L.total);
  int * abortWord = reinterpret_cast<int *>(bars + 2);
  double2 const zero = make_double2(0, 0);

  for (int e = tid; e < 2 * nn; e += kFusedThreads) {
    int const s = e / nn, r = e - s * nn;
    sm[L.D + (s * nb + r / nb) * ld + r % nb] = t.D[e];
  }
  for (int e = tid; e < 2 * nm * nb; e += kFusedThreads) {
    int const s = e / (nm * nb), b = (e / nb) % nm, i = e % nb;
    sm[L.C + e] = b < t.nel[s] ? (s == 0 ? t.C0 : t.C1)[b * nb + i] : zero;
  }
  uint32_t const vBytes = uint32_t(nn) * 48u, fBytes = uint32_t(nn) * (t.fcx ? 16u : 8u);
  uint32_t const txBytes = 2u * vBytes + 2u * fBytes + uint32_t(nb) * 64u;
  auto issue = [&](int64_t p, int b) {
    double2 * B = sm + L.buf + b * L.bufStride;
    tc::mbarArriveTx(&bars[b], txBytes);
    tc::bulkLoad(B, t.Vs + p * nn * 3, vBytes, &bars[b]);
    tc::bulkLoad(B + 3 * nn, t.Vo + p * nn * 3, vBytes, &bars[b]);
    tc::bulkLoad(B + 6 * nn, reinterpret_cast<const char *>(t.Fs) + p * fBytes, fBytes, &bars[b]);
    tc::bulkLoad(B + 6 * nn + L.fU, reinterpret_cast<const char *>(t.Fo) + p * fBytes, fBytes, &bars[b]);
    tc::bulkLoad(B + 6 * nn + 2 * L.fU, t.vals + p * nb, uint32_t(nb) * 16u, &bars[b]);
    tc::bulkLoad(B + 6 * nn + 2 * L.fU + nb, t.grads + p * nb * 3, uint32_t(nb) * 48u, &bars[b]);
  };
  if (tid == 0) {
    tc::mbarInit(&bars[0], 1);
    tc::mbarInit(&bars[1], 1);
    *abortWord = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  int const G = gridDim.x;
  if (tid == 0) {
    if (blockIdx.x < t.n1) issue(blockIdx.x, 0);
    if (t.nbuf == 2 && blockIdx.x + G < t.n1) issue(blockIdx.x + G, 1);
  }

  double2 acc[SLOTS][3];
#pragma unroll
  for (int q = 0; q < SLOTS; ++q) acc[q][0] = acc[q][1] = acc[q][2] = zero;

  int k = 0;
  for (int64_t p = blockIdx.x; p < t.n1; p += G, ++k) {
    int const bi = k % t.nbuf;
    bool const ok = tc::waitBar(&bars[bi], uint32_t(k / t.nbuf) & 1u, abortWord, t.status, kFusedWaitCode);
    if (__syncthreads_or(!ok)) return;
    const double2 * Vs = sm + L.buf + bi * L.bufStride;
    const double2 * Vo = Vs + 3 * nn;
    const double2 * F0 = Vo + 3 * nn;
    const double2 * F1 = F0 + L.fU;
    const double2 * vals = F1 + L.fU;
    const double2 * grads = vals + nb;
    auto F = [&](const double2 * base, int o) -> double2 {
      return t.fcx ? base[o] : make_double2(reinterpret_cast<const double *>(base)[o], 0.0);
    };

    // phase 1: kv, kc, kg (per spin, j); the Faa and V-tilde traces by column; Vjb (per spin, tensor, b, j)
    for (int it = tid; it < 8 * nb + 4 * nb * nm; it += kFusedThreads) {
      int const grp = it / (2 * nb);
      if (grp < 4) {
        int const s = (it / nb) & 1, j = it % nb;
        const double2 * Ds = sm + L.D + s * nb * ld;
        const double2 * Do = sm + L.D + (1 - s) * nb * ld;
        if (grp == 0) {
          double2 kv = zero, kc = zero;
          for (int kk = 0; kk < nb; ++kk) {
            kv = zfma(Ds[kk * ld + j], vals[kk], kv);
            kc = zfma(Ds[j * ld + kk], zconj(vals[kk]), kc);
          }
          sm[L.kv + s * nb + j] = kv;
          sm[L.kc + s * nb + j] = kc;
        } else if (grp == 1) {
          double2 g0 = zero, g1 = zero, g2 = zero;
          for (int kk = 0; kk < nb; ++kk) {
            double2 const d = Ds[kk * ld + j];
            g0 = zfma(d, grads[kk * 3], g0);
            g1 = zfma(d, grads[kk * 3 + 1], g1);
            g2 = zfma(d, grads[kk * 3 + 2], g2);
          }
          double2 * o = sm + L.kg + (s * nb + j) * 3;
          o[0] = g0; o[1] = g1; o[2] = g2;
        } else if (grp == 2) {
          int const i = j;
          double2 f = zero;
          for (int jj = 0; jj < nb; ++jj) {
            f = zfma(F(F0, jj * nb + i), Ds[i * ld + jj], f);
            f = zfma(F(F1, jj * nb + i), Do[i * ld + jj], f);
          }
          sm[L.colF + s * nb + i] = f;
        } else {
          int const i = j;
          double2 v0 = zero, v1 = zero, v2 = zero;
          for (int jj = 0; jj < nb; ++jj) {
            double2 const ds = Ds[i * ld + jj], dop = Do[i * ld + jj];
            const double2 * a = Vs + (jj * nb + i) * 3;
            const double2 * c = Vo + (jj * nb + i) * 3;
            v0 = zfma(c[0], dop, zfma(a[0], ds, v0));
            v1 = zfma(c[1], dop, zfma(a[1], ds, v1));
            v2 = zfma(c[2], dop, zfma(a[2], ds, v2));
          }
          double2 * o = sm + L.colV + (s * nb + i) * 3;
          o[0] = v0; o[1] = v1; o[2] = v2;
        }
      } else {
        int const q = it - 8 * nb;
        int const j = q % nb, b = (q / nb) % nm, st = q / (nb * nm), s = st >> 1, tt = st & 1;
        double2 r0 = zero, r1 = zero, r2 = zero;
        if (b < t.nel[s]) {
          const double2 * V = tt ? Vo : Vs;
          const double2 * Cb = sm + L.C + (s * nm + b) * nb;
          for (int kk = 0; kk < nb; ++kk) {
            int i = kk + j;   // each lane starts on its own column: rows j of a warp hit distinct banks
            if (i >= nb) i -= nb;
            double2 const c = Cb[i];
            const double2 * v = V + (j * nb + i) * 3;
            r0 = zfma(c, v[0], r0);
            r1 = zfma(c, v[1], r1);
            r2 = zfma(c, v[2], r2);
          }
        }
        double2 * o = sm + L.Vjb + (((s * 2 + tt) * nb + j) * nm + b) * 3;
        o[0] = r0; o[1] = r1; o[2] = r2;
      }
    }
    __syncthreads();

    // phase 2: Fai, VTs (per spin, i); Vai, Vja (per spin, i); occ, SG, Faa, VT (per spin); the |Vab|^2 terms
    for (int it = tid; it < 4 * nb + 8 + 4 * nm * nm; it += kFusedThreads) {
      if (it < 2 * nb) {
        int const s = it / nb, i = it % nb;
        double2 fa = zero, a0 = zero, a1 = zero, a2 = zero;
        for (int j = 0; j < nb; ++j) {
          double2 const kv = sm[L.kv + s * nb + j];
          const double2 * v = Vs + (j * nb + i) * 3;
          fa = zfma(kv, F(F0, j * nb + i), fa);
          a0 = zfma(kv, v[0], a0);
          a1 = zfma(kv, v[1], a1);
          a2 = zfma(kv, v[2], a2);
        }
        sm[L.Fai + s * nb + i] = fa;
        double2 * o = sm + L.VTs + (s * nb + i) * 3;
        o[0] = a0; o[1] = a1; o[2] = a2;
      } else if (it < 4 * nb) {
        int const q = it - 2 * nb, s = q / nb, i = q % nb;
        double2 c0 = zero, c1 = zero, c2 = zero, j0 = zero, j1 = zero, j2 = zero;
        for (int jj = 0; jj < nb; ++jj) {
          const double2 * kg = sm + L.kg + (s * nb + jj) * 3;
          const double2 * v = Vs + (jj * nb + i) * 3;
          c0 = zfma(v[0], kg[0], c0);
          c1 = zfma(v[1], kg[1], c1);
          c2 = zfma(v[2], kg[2], c2);
          int j = jj + i;   // skewed walk along row i of Vs
          if (j >= nb) j -= nb;
          double2 const kc = sm[L.kc + s * nb + j];
          const double2 * u = Vs + (i * nb + j) * 3;
          j0 = zfma(kc, u[0], j0);
          j1 = zfma(kc, u[1], j1);
          j2 = zfma(kc, u[2], j2);
        }
        sm[L.Vai + s * nb + i] = zadd(zadd(c0, c1), c2);
        double2 * o = sm + L.Vja + (s * nb + i) * 3;
        o[0] = j0; o[1] = j1; o[2] = j2;
      } else if (it < 4 * nb + 8) {
        int const q = it - 4 * nb, s = q >> 2, which = q & 3;
        double2 * S = sm + L.sc + s * 12;
        if (which == 0) {
          double2 oc = zero;
          for (int kk = 0; kk < nb; ++kk) oc = zcfma(vals[kk], sm[L.kv + s * nb + kk], oc);
          S[10] = make_double2(oc.x, 0.0);
        } else if (which == 1) {
          double2 g0 = zero, g1 = zero, g2 = zero;
          for (int i = 0; i < nb; ++i) {
            double2 const kc = sm[L.kc + s * nb + i];
            g0 = zfma(kc, grads[i * 3], g0);
            g1 = zfma(kc, grads[i * 3 + 1], g1);
            g2 = zfma(kc, grads[i * 3 + 2], g2);
          }
          S[4] = g0; S[5] = g1; S[6] = g2;
        } else if (which == 2) {
          double2 f = zero;
          for (int i = 0; i < nb; ++i) f = zadd(f, sm[L.colF + s * nb + i]);
          S[0] = f;
        } else {
          double2 v0 = zero, v1 = zero, v2 = zero;
          for (int i = 0; i < nb; ++i) {
            const double2 * c = sm + L.colV + (s * nb + i) * 3;
            v0 = zadd(v0, c[0]); v1 = zadd(v1, c[1]); v2 = zadd(v2, c[2]);
          }
          S[1] = v0; S[2] = v1; S[3] = v2;
        }
      } else {
        int const q = it - 4 * nb - 8;
        int const b = q % nm, a = (q / nm) % nm, st = q / (nm * nm), s = st >> 1, tt = st & 1;
        double n = 0;
        if (a < t.nel[s] && b < t.nel[s]) {
          double2 r0 = zero, r1 = zero, r2 = zero;
          for (int j = 0; j < nb; ++j) {
            double2 const c = sm[L.C + (s * nm + a) * nb + j];
            const double2 * v = sm + L.Vjb + (((s * 2 + tt) * nb + j) * nm + b) * 3;
            r0 = zcfma(c, v[0], r0);
            r1 = zcfma(c, v[1], r1);
            r2 = zcfma(c, v[2], r2);
          }
          n = r0.x * r0.x + r0.y * r0.y + r1.x * r1.x + r1.y * r1.y + r2.x * r2.x + r2.y * r2.y;
        }
        sm[L.nP + q] = make_double2(n, 0.0);
      }
    }
    __syncthreads();

    // phase 3: ell (per spin, k), SCV (per spin), sum over a, b of the |Vab|^2 terms (per spin, tensor)
    for (int it = tid; it < 2 * nb + 6; it += kFusedThreads) {
      if (it < 2 * nb) {
        int const s = it / nb, kk = it % nb;
        const double2 * Ds = sm + L.D + s * nb * ld;
        double2 e0 = zero, e1 = zero, e2 = zero;
        for (int l = 0; l < nb; ++l) {
          double2 const d = Ds[l * ld + kk];
          const double2 * v = sm + L.VTs + (s * nb + l) * 3;
          e0 = zfma(d, v[0], e0);
          e1 = zfma(d, v[1], e1);
          e2 = zfma(d, v[2], e2);
        }
        double2 * o = sm + L.ell + (s * nb + kk) * 3;
        o[0] = e0; o[1] = e1; o[2] = e2;
      } else if (it < 2 * nb + 2) {
        int const s = it - 2 * nb;
        double2 c0 = zero, c1 = zero, c2 = zero;
        for (int kk = 0; kk < nb; ++kk) {
          double2 const kv = sm[L.kv + s * nb + kk];
          const double2 * v = sm + L.VTs + (s * nb + kk) * 3;
          c0 = zcfma(v[0], kv, c0);
          c1 = zcfma(v[1], kv, c1);
          c2 = zcfma(v[2], kv, c2);
        }
        double2 * S = sm + L.sc + s * 12;
        S[7] = c0; S[8] = c1; S[9] = c2;
      } else {
        int const q = it - 2 * nb - 2, s = q >> 1, tt = q & 1;
        double n = 0;
        for (int ab = 0; ab < nm * nm; ++ab) n += sm[L.nP + (s * 2 + tt) * nm * nm + ab].x;
        double * S11 = reinterpret_cast<double *>(sm + L.sc + s * 12 + 11);
        S11[tt] = n;
      }
    }
    __syncthreads();

    // phase 4: SVD and the w-scaled per-(spin, i) operands of the element sums; w g_i; the per-spin 3-vectors
    double const w = t.w[p];
    for (int it = tid; it < 3 * nb + 2; it += kFusedThreads) {
      if (it < 2 * nb) {
        int const s = it / nb, i = it % nb, o = 1 - s;
        const double2 * S = sm + L.sc + s * 12;
        const double2 * So = sm + L.sc + o * 12;
        double2 s0 = zero, s1 = zero, s2 = zero;
        for (int kk = 0; kk < nb; ++kk) {
          const double2 * v = Vs + (kk * nb + i) * 3;
          const double2 * e = sm + L.ell + (s * nb + kk) * 3;
          s0 = zfma(v[0], e[0], s0);
          s1 = zfma(v[1], e[1], s1);
          s2 = zfma(v[2], e[2], s2);
        }
        double2 const svd = zadd(zadd(s0, s1), s2);
        double2 const vi = vals[i];
        const double2 * g = grads + i * 3;
        const double2 * vts = sm + L.VTs + (s * nb + i) * 3;
        double2 vtg = zero, vtv = zero, cvv = zero;
        double nvt = 0;
        for (int c = 0; c < 3; ++c) {
          vtg = zfma(S[1 + c], g[c], vtg);
          vtv = zfma(S[1 + c], vts[c], vtv);
          cvv = zcfma(vts[c], S[1 + c], cvv);
          nvt += S[1 + c].x * S[1 + c].x + S[1 + c].y * S[1 + c].y;
        }
        double const coef = nvt - S[11].x - So[11].y;
        sm[L.Pw + s * nb + i] = zscale(w, zsub(zmul(S[0], vi), sm[L.Fai + s * nb + i]));
        sm[L.Qw + s * nb + i] = zscale(w, zsub(vtg, sm[L.Vai + s * nb + i]));
        sm[L.Rw + s * nb + i] = zscale(w, zadd(zscale(coef, vi), zscale(2.0, zsub(svd, vtv))));
        sm[L.Tw + s * nb + i] = zscale(2.0 * w, zsub(zconj(svd), cvv));
        for (int c = 0; c < 3; ++c) sm[L.Xw + (s * nb + i) * 3 + c] = zscale(2.0 * w, vts[c]);
        for (int tt = 0; tt < 2; ++tt) {
          double const f = -2.0 * w * (tt ? So[10].x : S[10].x);
          for (int b = 0; b < nm; ++b) {
            int const o3 = (((s * 2 + tt) * nb + i) * nm + b) * 3;
            for (int c = 0; c < 3; ++c) sm[L.Jw + o3 + c] = zscale(f, sm[L.Vjb + o3 + c]);
          }
        }
      } else if (it < 3 * nb) {
        int const i = it - 2 * nb;
        for (int c = 0; c < 3; ++c) sm[L.gw + i * 3 + c] = zscale(-w, grads[i * 3 + c]);
      } else {
        int const s = it - 3 * nb, o = 1 - s;
        const double2 * S = sm + L.sc + s * 12;
        const double2 * So = sm + L.sc + o * 12;
        double2 * W = sm + L.ws + s * 12;
        for (int c = 0; c < 3; ++c) {
          W[c] = zscale(w, S[4 + c]);
          W[3 + c] = zscale(w, So[4 + c]);
          W[6 + c] = zscale(w, zsub(zscale(2.0 * S[10].x, S[1 + c]), zscale(2.0, S[7 + c])));
          W[9 + c] = zscale(w, zsub(zscale(2.0 * So[10].x, So[1 + c]), zscale(2.0, So[7 + c])));
        }
      }
    }
    __syncthreads();

    // phase 5: this thread's (spin, j, i) elements
#pragma unroll
    for (int q = 0; q < SLOTS; ++q) {
      int const e = tid + q * kFusedThreads;
      if (e < 2 * nn) {
        int const s = e / nn, r = e - s * nn, j = r / nb, i = r - j * nb;
        const double2 * vs = Vs + r * 3;
        const double2 * vo = Vo + r * 3;
        const double2 * W = sm + L.ws + s * 12;
        const double2 * vja = sm + L.Vja + (s * nb + j) * 3;
        const double2 * gw = sm + L.gw + i * 3;
        const double2 * xw = sm + L.Xw + (s * nb + i) * 3;
        const double2 * vtj = sm + L.VTs + (s * nb + j) * 3;
        double2 const vj = vals[j], vi = vals[i];
        acc[q][0] = zcfma(vj, sm[L.Pw + s * nb + i], acc[q][0]);
        double2 ve = zcfma(vj, sm[L.Qw + s * nb + i], acc[q][1]);
        double2 s3 = zcfma(vj, sm[L.Rw + s * nb + i], acc[q][2]);
        s3 = zfma(sm[L.Tw + s * nb + j], vi, s3);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          double2 const a = vs[c], b = vo[c];
          ve = zfma(a, W[c], ve);
          ve = zfma(b, W[3 + c], ve);
          ve = zfma(vja[c], gw[c], ve);
          s3 = zfma(a, W[6 + c], s3);
          s3 = zfma(b, W[9 + c], s3);
          s3 = zfma(xw[c], zconj(vtj[c]), s3);
        }
        for (int tt = 0; tt < 2; ++tt)
          for (int b = 0; b < t.nel[s]; ++b) {
            const double2 * jw = sm + L.Jw + (((s * 2 + tt) * nb + j) * nm + b) * 3;
            const double2 * vb = sm + L.Vjb + (((s * 2 + tt) * nb + i) * nm + b) * 3;
            s3 = zfma(jw[0], zconj(vb[0]), s3);
            s3 = zfma(jw[1], zconj(vb[1]), s3);
            s3 = zfma(jw[2], zconj(vb[2]), s3);
          }
        acc[q][1] = ve;
        acc[q][2] = s3;
      }
    }
    __syncthreads();   // the buffer and the intermediates are free again
    int64_t const next = p + int64_t(t.nbuf) * G;
    if (tid == 0 && next < t.n1) issue(next, bi);
  }
  double2 * out = t.part + int64_t(blockIdx.x) * 6 * nn;
#pragma unroll
  for (int q = 0; q < SLOTS; ++q) {
    int const e = tid + q * kFusedThreads;
    if (e < 2 * nn) {
      out[e] = acc[q][0];
      out[2 * nn + e] = acc[q][1];
      out[4 * nn + e] = acc[q][2];
    }
  }
}

// out[e] = sum over blocks of part[block][e], e < n, in block order
__global__ void kTcPartials(int nparts, int n, const double2 * part, double2 * out)
{
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    double2 a = make_double2(0, 0);
    for (int b = 0; b < nparts; ++b) a = zadd(a, part[int64_t(b) * n + e]);
    out[e] = a;
  }
}

template <int SLOTS>
int launchFused(tcscf_ctx * ctx, TcFusedArgs const & a, int grid, size_t smem)
{
  TCSCF_CUDA(ctx, cudaFuncSetAttribute(kTcFused<SLOTS>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  kTcFused<SLOTS><<<grid, kFusedThreads, smem, ctx->stream>>>(a);
  TCSCF_LAUNCH(ctx);
  return TCSCF_OK;
}

Tensor const * findTensor(tcscf_ctx * ctx, int id)
{
  auto it = ctx->tensors.find(id);
  return it == ctx->tensors.end() ? nullptr : &it->second;
}


struct TcInputs {
  Grid * g1 = nullptr;
  Tensor const * F[2] = {nullptr, nullptr};   // same, opposite
  Tensor const * V[2] = {nullptr, nullptr};
};

int checkTcInputs(tcscf_ctx * ctx, int r1, int fs, int fo, int vs, int vo, int nup, int ndown, TcInputs & in)
{
  in.g1 = findGrid(ctx, r1);
  TCSCF_CHECK(ctx, in.g1 && in.g1->nb > 0 && in.g1->ndim == 3, TCSCF_ERR_INVALID_ARGUMENT, "r1 grid needs a 3-D basis");
  TCSCF_CHECK(ctx, in.g1->grads, TCSCF_ERR_INVALID_ARGUMENT, "the TC build needs the r1 basis gradients");
  int const ids[4] = {fs, fo, vs, vo};
  for (int k = 0; k < 4; ++k) {
    Tensor const * t = findTensor(ctx, ids[k]);
    TCSCF_CHECK(ctx, t, TCSCF_ERR_INVALID_ARGUMENT, "unknown tensor handle");
    TCSCF_CHECK(ctx, t->n1 == in.g1->n && t->nb == in.g1->nb, TCSCF_ERR_INVALID_ARGUMENT, "tensor does not match the r1 grid");
    TCSCF_CHECK(ctx, (k < 2) == !t->vec, TCSCF_ERR_INVALID_ARGUMENT, "expected Fji (computeF) then Vji (computeV) handles");
    if (k < 2) in.F[k] = t; else in.V[k - 2] = t;
  }
  TCSCF_CHECK(ctx, in.F[0]->isComplex == in.F[1]->isComplex, TCSCF_ERR_INVALID_ARGUMENT, "both Fji must come from the same r2 grid kind");
  TCSCF_CHECK(ctx, nup >= 0 && ndown >= 0 && nup <= in.g1->nb && ndown <= in.g1->nb, TCSCF_ERR_INVALID_ARGUMENT, "bad electron counts");
  return TCSCF_OK;
}

// One TC Fock build on device buffers: D [2][nb][nb], C0 / C1 occupied orbitals, h real [nb][nb];
// outputs G2, G3, Fock [2][nb][nb] and the energy (device).  The fused kernel's status word is copied
// to *hostStatus (0: ok), which the caller reads after its next synchronisation.
int tcFockBuildDevice(tcscf_ctx * ctx, TcInputs const & in, int nup, int ndown, const double2 * dD, const double2 * dC0, const double2 * dC1,
                      const double * dH, int respectSym, double2 * dG2, double2 * dG3, double2 * dFock, double * dE, int * hostStatus)
{
  Grid const & g = *in.g1;
  int const nb = g.nb, nm = std::max(1, std::max(nup, ndown));
  int64_t const n1 = g.n;
  *hostStatus = 0;
  int const fcx = in.F[0]->isComplex;
  int nbuf = 0;
  if (nb <= kFusedMaxNb && (fcx || nb % 2 == 0)) {
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
    for (int q = 2; q >= 1 && !nbuf; --q)
      if (FusedLayout(nb, nm, fcx, q).bytes() <= size_t(optin)) nbuf = q;
  }
  if (nbuf) {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    int const grid = int(std::max<int64_t>(1, std::min<int64_t>(sms, n1)));
    size_t const nn6 = 6 * size_t(nb) * nb;
    void * p = nullptr;
    TCSCF_TRY(scratch(ctx, "tc_fused", sizeof(double2) * nn6 * (size_t(grid) + 1) + 256, &p));
    double2 * part = static_cast<double2 *>(p);
    double2 * sums = part + nn6 * grid;
    int * dStatus = reinterpret_cast<int *>(sums + nn6);
    TCSCF_CUDA(ctx, cudaMemsetAsync(dStatus, 0, sizeof(int), ctx->stream));
    TcFusedArgs a{};
    a.n1 = n1; a.nb = nb; a.nm = nm; a.nbuf = nbuf; a.fcx = fcx;
    a.nel[0] = nup; a.nel[1] = ndown;
    a.Fs = in.F[0]->d; a.Fo = in.F[1]->d;
    a.Vs = reinterpret_cast<const double2 *>(in.V[0]->d); a.Vo = reinterpret_cast<const double2 *>(in.V[1]->d);
    a.vals = reinterpret_cast<const double2 *>(g.vals); a.grads = reinterpret_cast<const double2 *>(g.grads); a.w = g.w;
    a.D = dD; a.C0 = dC0; a.C1 = dC1;
    a.part = part; a.status = dStatus;
    size_t const smem = FusedLayout(nb, nm, fcx, nbuf).bytes();
    int const slots = (2 * nb * nb + kFusedThreads - 1) / kFusedThreads;
    if (slots <= 1) TCSCF_TRY(launchFused<1>(ctx, a, grid, smem));
    else if (slots == 2) TCSCF_TRY(launchFused<2>(ctx, a, grid, smem));
    else if (slots == 3) TCSCF_TRY(launchFused<3>(ctx, a, grid, smem));
    else TCSCF_TRY(launchFused<4>(ctx, a, grid, smem));
    kTcPartials<<<gridBlocks(int64_t(nn6), 256), 256, 0, ctx->stream>>>(grid, int(nn6), part, sums);
    TCSCF_LAUNCH(ctx);
    kTcAssemble<<<gridBlocks(2 * nb * nb, 256), 256, 0, ctx->stream>>>(nb, sums, dH, respectSym, dG2, dG3);
    TCSCF_LAUNCH(ctx);
    TCSCF_TRY(finalizeLaunch(ctx, 2, nb, dH, dG2, dG3, dD, respectSym, 1.0, dFock, dE));
    TCSCF_CUDA(ctx, cudaMemcpyAsync(hostStatus, dStatus, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    return TCSCF_OK;
  }
  size_t const perPoint = 1 + nb + 3 + 3 + nb + 3 * nb + 3 * nb + 2 * 3 * size_t(nb) * nm + nb + 3;   // double2 units
  size_t const bytes = sizeof(double2) * (2 * size_t(n1) * perPoint + 6 * size_t(nb) * nb) + sizeof(double) * 2 * 3 * size_t(n1) + 1024;
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, "tc_terms", bytes, &p));
  double2 * z = static_cast<double2 *>(p);
  auto take = [&](size_t n) { double2 * r = z; z += n; return r; };
  TcView t{};
  t.n1 = n1; t.nb = nb; t.nelMax = nm; t.nel[0] = nup; t.nel[1] = ndown;
  t.fcx = in.F[0]->isComplex;
  t.Fs = in.F[0]->d; t.Fo = in.F[1]->d;
  t.Vs = reinterpret_cast<const double2 *>(in.V[0]->d); t.Vo = reinterpret_cast<const double2 *>(in.V[1]->d);
  t.vals = reinterpret_cast<const double2 *>(g.vals); t.grads = reinterpret_cast<const double2 *>(g.grads); t.w = g.w;
  t.D = dD; t.C0 = dC0; t.C1 = dC1;
  size_t const n2 = 2 * size_t(n1);
  t.Faa = take(n2); t.Fai = take(n2 * nb); t.VT = take(n2 * 3); t.SG = take(n2 * 3);
  t.Vai = take(n2 * nb); t.Vja = take(n2 * nb * 3); t.VTs = take(n2 * nb * 3);
  t.Vjbs = take(n2 * nb * nm * 3); t.Vjbo = take(n2 * nb * nm * 3); t.SVD = take(n2 * nb); t.SCV = take(n2 * 3);
  double2 * sums = take(6 * size_t(nb) * nb);
  double * dr = reinterpret_cast<double *>(z);
  t.occD = dr; t.sumNs = dr + n2; t.sumNo = dr + 2 * n2;
  TCSCF_CHECK(ctx, reinterpret_cast<char *>(dr + 3 * n2) <= static_cast<char *>(p) + bytes, TCSCF_ERR_INVALID_ARGUMENT, "internal: tc scratch");

  kTcPoint<<<gridBlocks(2 * n1, 128), 128, 0, ctx->stream>>>(t);
  TCSCF_LAUNCH(ctx);
  kTcPointI<<<gridBlocks(2 * n1 * nb, 128), 128, 0, ctx->stream>>>(t);
  TCSCF_LAUNCH(ctx);
  kTcVjb<<<gridBlocks(2 * n1 * nb * nm, 128), 128, 0, ctx->stream>>>(t);
  TCSCF_LAUNCH(ctx);
  kTcVab<<<gridBlocks(2 * n1, 128), 128, 0, ctx->stream>>>(t);
  TCSCF_LAUNCH(ctx);
  kTcSvd<<<gridBlocks(2 * n1 * nb, 128), 128, 0, ctx->stream>>>(t);
  TCSCF_LAUNCH(ctx);
  kTcReduce<<<unsigned(2 * nb * nb), 256, 0, ctx->stream>>>(t, sums);
  TCSCF_LAUNCH(ctx);
  kTcAssemble<<<gridBlocks(2 * nb * nb, 256), 256, 0, ctx->stream>>>(nb, sums, dH, respectSym, dG2, dG3);
  TCSCF_LAUNCH(ctx);
  return finalizeLaunch(ctx, 2, nb, dH, dG2, dG3, dD, respectSym, 1.0, dFock, dE);
}

// S-metric modified Gram-Schmidt of orthogonalization.hpp:136-154 on nvec row vectors of length n,
// metric S real symmetric [n][n]; after the first vector the normalisation is Euclidean (:152).
void mgsMetric(std::vector<std::complex<double>> & v, int nvec, int n, std::vector<double> const & S)
{
  using cplx = std::complex<double>;
  auto ip = [&](cplx const * a, cplx const * b) {
    cplx d = 0;
    for (int i = 0; i < n; ++i) {
      cplx row = 0;
      for (int j = 0; j < n; ++j) row += S[size_t(i) * n + j] * b[j];
      d += std::conj(a[i]) * row;
    }
    return d;
  };
  auto normE = [&](cplx const * a) { double d = 0; for (int i = 0; i < n; ++i) d += std::norm(a[i]); return std::sqrt(d); };
  if (nvec == 0) return;
  double const s0 = 1.0 / std::sqrt(ip(v.data(), v.data()).real());
  for (int i = 0; i < n; ++i) v[i] *= s0;
  for (int i = 1; i < nvec; ++i) {
    for (int j = i; j < nvec; ++j) {
      cplx const sc = ip(v.data() + size_t(i - 1) * n, v.data() + size_t(j) * n);
      for (int k = 0; k < n; ++k) v[size_t(j) * n + k] -= sc * v[size_t(i - 1) * n + k];
    }
    double const s = 1.0 / normE(v.data() + size_t(i) * n);
    for (int k = 0; k < n; ++k) v[size_t(i) * n + k] *= s;
  }
}

}  // namespace
}  // namespace tcscf

using namespace tcscf;

extern "C" {

int tcscf_tc_fock_build(tcscf_ctx * ctx, int r1, int fji_same, int fji_oppo, int vji_same, int vji_oppo, int n_up, int n_down,
                        const double * density, const double * occ_up, const double * occ_down, const double * h, int respect_symmetry,
                        double * G2, double * G3, double * fock, double * energy)
{
  TCSCF_NVTX();
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  TcInputs in;
  TCSCF_TRY(checkTcInputs(ctx, r1, fji_same, fji_oppo, vji_same, vji_oppo, n_up, n_down, in));
  TCSCF_CHECK(ctx, density && h, TCSCF_ERR_INVALID_ARGUMENT, "density and h are required");
  TCSCF_CHECK(ctx, (occ_up || n_up == 0) && (occ_down || n_down == 0), TCSCF_ERR_INVALID_ARGUMENT, "occupied orbitals are required");
  int const nb = in.g1->nb;
  size_t const nn = size_t(nb) * nb;
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, "tc_io", sizeof(double2) * (nn * 2 * 4 + size_t(nb) * (n_up + n_down) + 2) + sizeof(double) * (nn + 2), &p));
  double2 * dD = static_cast<double2 *>(p);
  double2 * dG2 = dD + 2 * nn;
  double2 * dG3 = dG2 + 2 * nn;
  double2 * dF = dG3 + 2 * nn;
  double2 * dC0 = dF + 2 * nn;
  double2 * dC1 = dC0 + size_t(nb) * n_up;
  double * dH = reinterpret_cast<double *>(dC1 + size_t(nb) * n_down + 1);
  double * dE = dH + nn;
  TCSCF_CUDA(ctx, cudaMemcpyAsync(dD, density, sizeof(double2) * 2 * nn, cudaMemcpyHostToDevice, ctx->stream));
  if (n_up) TCSCF_CUDA(ctx, cudaMemcpyAsync(dC0, occ_up, sizeof(double2) * nb * n_up, cudaMemcpyHostToDevice, ctx->stream));
  if (n_down) TCSCF_CUDA(ctx, cudaMemcpyAsync(dC1, occ_down, sizeof(double2) * nb * n_down, cudaMemcpyHostToDevice, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemcpyAsync(dH, h, sizeof(double) * nn, cudaMemcpyHostToDevice, ctx->stream));
  int kst = 0;
  TCSCF_TRY(tcFockBuildDevice(ctx, in, n_up, n_down, dD, dC0, dC1, dH, respect_symmetry, dG2, dG3, dF, dE, &kst));
  if (G2) TCSCF_CUDA(ctx, cudaMemcpyAsync(G2, dG2, sizeof(double2) * 2 * nn, cudaMemcpyDeviceToHost, ctx->stream));
  if (G3) TCSCF_CUDA(ctx, cudaMemcpyAsync(G3, dG3, sizeof(double2) * 2 * nn, cudaMemcpyDeviceToHost, ctx->stream));
  if (fock) TCSCF_CUDA(ctx, cudaMemcpyAsync(fock, dF, sizeof(double2) * 2 * nn, cudaMemcpyDeviceToHost, ctx->stream));
  double e = 0;
  TCSCF_CUDA(ctx, cudaMemcpyAsync(&e, dE, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  TCSCF_CHECK(ctx, kst == 0, TCSCF_ERR_TIMEOUT, "TC build: bounded wait expired (code " + std::to_string(kst) + ")");
  if (energy) *energy = e;
  if (!(e == e) || std::isinf(e)) return fail(ctx, TCSCF_ERR_NONFINITE, "non-finite TC energy");
  return TCSCF_OK;
}

int tcscf_tc_scf(tcscf_ctx * ctx, int r1, int fji_same, int fji_oppo, int vji_same, int vji_oppo, const double * S, const double * h,
                 int n_up, int n_down, int respect_symmetry, double tol, int max_iter, double * energy, int * iterations, double * density,
                 double * pseudo_energies)
{
  TCSCF_NVTX();
  using cplx = std::complex<double>;
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  TcInputs in;
  TCSCF_TRY(checkTcInputs(ctx, r1, fji_same, fji_oppo, vji_same, vji_oppo, n_up, n_down, in));
  TCSCF_CHECK(ctx, S && h && energy && iterations && density, TCSCF_ERR_INVALID_ARGUMENT, "S, h and the outputs are required");
  TCSCF_CHECK(ctx, max_iter > 0, TCSCF_ERR_INVALID_ARGUMENT, "max_iter must be positive");
  int const nb = in.g1->nb;
  size_t const nn = size_t(nb) * nb;
  int const nel[2] = {n_up, n_down};
  cublasHandle_t blas = nullptr;
  TCSCF_TRY(blasHandle(ctx, &blas));
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, "tc_scf", sizeof(double2) * (nn * 2 * 4 + size_t(nb) * (n_up + n_down) + 2 + 4 * nn + nb) + sizeof(double) * (2 * nn + 2) + 64,
                    &p));
  double2 * dD = static_cast<double2 *>(p);
  double2 * dG2 = dD + 2 * nn;
  double2 * dG3 = dG2 + 2 * nn;
  double2 * dF = dG3 + 2 * nn;
  double2 * dC0 = dF + 2 * nn;
  double2 * dC1 = dC0 + size_t(nb) * n_up;
  double2 * dA = dC1 + size_t(nb) * n_down + 1;
  double2 * dB = dA + nn;
  double2 * dVR = dB + nn;
  double2 * dVL = dVR + nn;
  double2 * dW = dVL + nn;
  double * dH = reinterpret_cast<double *>(dW + nb + 1);
  double * dS = dH + nn;
  double * dE = dS + nn;
  int * dInfo = reinterpret_cast<int *>(dE + 1);
  TCSCF_CUDA(ctx, cudaMemcpyAsync(dH, h, sizeof(double) * nn, cudaMemcpyHostToDevice, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemcpyAsync(dS, S, sizeof(double) * nn, cudaMemcpyHostToDevice, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemsetAsync(dD, 0, sizeof(double2) * 2 * nn, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemsetAsync(dC0, 0, sizeof(double2) * (size_t(nb) * (n_up + n_down) + 1), ctx->stream));

  cusolverDnParams_t params = nullptr;
  TCSCF_CHECK(ctx, cusolverDnCreateParams(&params) == CUSOLVER_STATUS_SUCCESS, TCSCF_ERR_CUDA, "cusolverDnCreateParams failed");
  struct ParamsGuard { cusolverDnParams_t p; ~ParamsGuard() { cusolverDnDestroyParams(p); } } guard{params};
  size_t dws = 0, hws = 0;
  TCSCF_CHECK(ctx, cusolverDnXgeev_bufferSize(ctx->solver, params, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_VECTOR, nb, CUDA_C_64F, dA, nb,
                                              CUDA_C_64F, dW, CUDA_C_64F, dVL, nb, CUDA_C_64F, dVR, nb, CUDA_C_64F, &dws, &hws) == CUSOLVER_STATUS_SUCCESS,
              TCSCF_ERR_LINALG, "cusolverDnXgeev_bufferSize failed");
  int lpotrf = 0;
  TCSCF_CHECK(ctx, cusolverDnZpotrf_bufferSize(ctx->solver, CUBLAS_FILL_MODE_LOWER, nb, reinterpret_cast<cuDoubleComplex *>(dB), nb, &lpotrf) ==
                       CUSOLVER_STATUS_SUCCESS,
              TCSCF_ERR_LINALG, "cusolverDnZpotrf_bufferSize failed");
  void * wk = nullptr;
  TCSCF_TRY(scratch(ctx, "tc_scf_work", std::max(dws, sizeof(double2) * size_t(lpotrf)) + 256, &wk));
  std::vector<char> hwork(hws + 1);

  std::vector<int> sorted(2 * size_t(nb));
  for (int s = 0; s < 2; ++s)
    for (int i = 0; i < nb; ++i) sorted[size_t(s) * nb + i] = i;
  std::vector<cplx> hW(nb), hV(nn), hD(2 * nn);
  std::vector<cplx> occ[2] = {std::vector<cplx>(size_t(nb) * n_up), std::vector<cplx>(size_t(nb) * n_down)};
  std::vector<double> hS(S, S + nn);
  double prev = std::numeric_limits<double>::max();
  cuDoubleComplex const one = make_cuDoubleComplex(1, 0);
  for (int it = 0; it < max_iter; ++it) {
    int kst = 0;
    TCSCF_TRY(tcFockBuildDevice(ctx, in, n_up, n_down, dD, dC0, dC1, dH, respect_symmetry, dG2, dG3, dF, dE, &kst));
    double e = 0;
    TCSCF_CUDA(ctx, cudaMemcpyAsync(&e, dE, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    TCSCF_CHECK(ctx, kst == 0, TCSCF_ERR_TIMEOUT, "TC build: bounded wait expired (code " + std::to_string(kst) + ")");
    *iterations = it + 1;
    TCSCF_CHECK(ctx, e == e && !std::isinf(e), TCSCF_ERR_NONFINITE, "non-finite TC energy");
    if (std::abs(e - prev) < tol) {
      *energy = e;
      TCSCF_CUDA(ctx, cudaMemcpyAsync(density, dD, sizeof(double2) * 2 * nn, cudaMemcpyDeviceToHost, ctx->stream));
      TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      return TCSCF_OK;
    }
    prev = e;
    for (int s = 0; s < 2; ++s) {
      // F C = S C e  ->  (L^-1 F L^-H) Y = Y e,  C = L^-H Y,  S = L L^H
      kToColMajorZ<<<gridBlocks(int64_t(nn), 256), 256, 0, ctx->stream>>>(nb, dF + s * nn, dA);
      TCSCF_LAUNCH(ctx);
      kRealToZ<<<gridBlocks(int64_t(nn), 256), 256, 0, ctx->stream>>>(int(nn), dS, dB);
      TCSCF_LAUNCH(ctx);
      auto * A = reinterpret_cast<cuDoubleComplex *>(dA);
      auto * B = reinterpret_cast<cuDoubleComplex *>(dB);
      auto * VR = reinterpret_cast<cuDoubleComplex *>(dVR);
      TCSCF_CHECK(ctx, cusolverDnZpotrf(ctx->solver, CUBLAS_FILL_MODE_LOWER, nb, B, nb, static_cast<cuDoubleComplex *>(wk), lpotrf, dInfo) ==
                           CUSOLVER_STATUS_SUCCESS,
                  TCSCF_ERR_LINALG, "cusolverDnZpotrf failed");
      int info = 0;
      TCSCF_CUDA(ctx, cudaMemcpyAsync(&info, dInfo, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
      TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      TCSCF_CHECK(ctx, info == 0, TCSCF_ERR_LINALG, "overlap matrix is not positive definite (potrf info " + std::to_string(info) + ")");
      TCSCF_CHECK(ctx, cublasZtrsm(blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, nb, nb, &one, B, nb, A, nb) ==
                               CUBLAS_STATUS_SUCCESS &&
                           cublasZtrsm(blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_C, CUBLAS_DIAG_NON_UNIT, nb, nb, &one, B, nb, A, nb) ==
                               CUBLAS_STATUS_SUCCESS,
                  TCSCF_ERR_LINALG, "cublasZtrsm failed");
      TCSCF_CHECK(ctx, cusolverDnXgeev(ctx->solver, params, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_VECTOR, nb, CUDA_C_64F, dA, nb, CUDA_C_64F,
                                       dW, CUDA_C_64F, dVL, nb, CUDA_C_64F, dVR, nb, CUDA_C_64F, wk, dws, hwork.data(), hws, dInfo) ==
                           CUSOLVER_STATUS_SUCCESS,
                  TCSCF_ERR_LINALG, "cusolverDnXgeev failed");
      TCSCF_CHECK(ctx, cublasZtrsm(blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_C, CUBLAS_DIAG_NON_UNIT, nb, nb, &one, B, nb, VR, nb) ==
                           CUBLAS_STATUS_SUCCESS,
                  TCSCF_ERR_LINALG, "cublasZtrsm failed");
      TCSCF_CUDA(ctx, cudaMemcpyAsync(&info, dInfo, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
      TCSCF_CUDA(ctx, cudaMemcpyAsync(hW.data(), dW, sizeof(double2) * nb, cudaMemcpyDeviceToHost, ctx->stream));
      TCSCF_CUDA(ctx, cudaMemcpyAsync(hV.data(), dVR, sizeof(double2) * nn, cudaMemcpyDeviceToHost, ctx->stream));
      TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      TCSCF_CHECK(ctx, info == 0, TCSCF_ERR_LINALG, "cusolverDnXgeev info " + std::to_string(info));
      // sort by real part, keeping the previous iteration's order as the starting permutation (:1298-1303)
      int * si = sorted.data() + size_t(s) * nb;
      std::sort(si, si + nb, [&](int a, int b) { return hW[a].real() < hW[b].real(); });
      std::vector<cplx> occT(size_t(nel[s]) * nb);
      for (int i = 0; i < nel[s]; ++i) {
        if (pseudo_energies) pseudo_energies[size_t(s) * nb + i] = hW[si[i]].real();
        for (int j = 0; j < nb; ++j) occT[size_t(i) * nb + j] = hV[size_t(si[i]) * nb + j];
      }
      mgsMetric(occT, nel[s], nb, hS);
      occ[s] = occT;   // column-major nb x nel: column b = row b of occT
      // getNewDensity (:20-44): D(u,v) = sum_a C(u,a) conj(C(v,a))
      for (int u = 0; u < nb; ++u)
        for (int v = 0; v < nb; ++v) {
          cplx t = 0;
          for (int a = 0; a < nel[s]; ++a) t += occT[size_t(a) * nb + u] * std::conj(occT[size_t(a) * nb + v]);
          hD[size_t(s) * nn + size_t(u) * nb + v] = t;
        }
    }
    TCSCF_CUDA(ctx, cudaMemcpyAsync(dD, hD.data(), sizeof(double2) * 2 * nn, cudaMemcpyHostToDevice, ctx->stream));
    if (n_up) TCSCF_CUDA(ctx, cudaMemcpyAsync(dC0, occ[0].data(), sizeof(double2) * nb * n_up, cudaMemcpyHostToDevice, ctx->stream));
    if (n_down) TCSCF_CUDA(ctx, cudaMemcpyAsync(dC1, occ[1].data(), sizeof(double2) * nb * n_down, cudaMemcpyHostToDevice, ctx->stream));
    TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));   // host buffers are reused next iteration
  }
  *energy = prev;
  TCSCF_CUDA(ctx, cudaMemcpyAsync(density, dD, sizeof(double2) * 2 * nn, cudaMemcpyDeviceToHost, ctx->stream));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return fail(ctx, TCSCF_ERR_NOT_CONVERGED, "TC SCF did not converge in " + std::to_string(max_iter) + " iterations");
}

}  // extern "C"
