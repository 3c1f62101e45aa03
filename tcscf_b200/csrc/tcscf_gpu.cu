// libtcscf_gpu.so: context, device grids and basis evaluation, one-electron quadrature, density
// factorisation, the Fock-build pipeline (direct and precompute forms) and the SCF driver.
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <algorithm>
#include <vector>

#include "kernels.cuh"

namespace tcscf {

int fail(tcscf_ctx * ctx, int code, std::string const & msg)
{
  if (ctx) ctx->err = msg;
  return code;
}

int blasHandle(tcscf_ctx * ctx, cublasHandle_t * out)
{
  if (!ctx->blas && cublasCreate(&ctx->blas) != CUBLAS_STATUS_SUCCESS) return fail(ctx, TCSCF_ERR_CUDA, "cublasCreate failed");
  if (cublasSetStream(ctx->blas, ctx->stream) != CUBLAS_STATUS_SUCCESS) return fail(ctx, TCSCF_ERR_CUDA, "cublasSetStream failed");
  *out = ctx->blas;
  return TCSCF_OK;
}

int scratch(tcscf_ctx * ctx, char const * name, size_t bytes, void ** out)
{
  Scratch & s = ctx->scratch[name];
  if (s.bytes < bytes || !s.p) {
    if (s.p) { cudaStreamSynchronize(ctx->stream); cudaFree(s.p); s.p = nullptr; s.bytes = 0; }
    size_t const want = std::max<size_t>(bytes, 256);
    cudaError_t const e = cudaMalloc(&s.p, want);
    if (e != cudaSuccess) return fail(ctx, TCSCF_ERR_CUDA, std::string("cudaMalloc(scratch ") + name + "): " + cudaGetErrorString(e));
    s.bytes = want;
  }
  *out = s.p;
  return TCSCF_OK;
}

Grid * findGrid(tcscf_ctx * ctx, int id)
{
  auto it = ctx->grids.find(id);
  return it == ctx->grids.end() ? nullptr : &it->second;
}

int gridAllocBytes(tcscf_ctx * ctx, void ** p, size_t bytes)
{
  *p = nullptr;
  cudaError_t const e = cudaMallocFromPoolAsync(p, std::max<size_t>(bytes, 256), ctx->gridPool, ctx->stream);
  if (e != cudaSuccess) return fail(ctx, TCSCF_ERR_CUDA, std::string("grid buffer allocation: ") + cudaGetErrorString(e));
  if (reinterpret_cast<uintptr_t>(*p) % 256 != 0) {
    cudaFreeAsync(*p, ctx->stream);
    *p = nullptr;
    return fail(ctx, TCSCF_ERR_CUDA, "grid buffer allocation is not 256-byte aligned");
  }
  return TCSCF_OK;
}

void gridRelease(tcscf_ctx * ctx, void * p)
{
  if (p) cudaFreeAsync(p, ctx->stream);
}

void gridReleaseAll(tcscf_ctx * ctx, Grid & g)
{
  gridRelease(ctx, g.pts); gridRelease(ctx, g.w); gridRelease(ctx, g.dsto); gridRelease(ctx, g.phiR);
  gridRelease(ctx, g.vals); gridRelease(ctx, g.grads); gridRelease(ctx, g.vtCache);
  g.pts = g.w = g.phiR = g.vals = g.grads = nullptr;
  g.dsto = nullptr;
  g.vtCache = nullptr;
}

namespace {

// Fully normalised associated Legendre function with the Condon-Shortley phase,
// P(l, m, cos t) = (-1)^m sqrt((2l+1)/(4 pi) (l-m)!/(l+m)!) P_l^m(cos t), i.e. Y_l^m(t, 0), evaluated
// with the standard three-term recurrences in l at fixed m (x = cos t, s = sin t).
__device__ double sphLegendre(int l, int m, double x, double s)
{
  if (m > l || m < 0) return 0.0;
  double pmm = 1.0;
  for (int k = 1; k <= m; ++k) pmm *= -s * sqrt((2.0 * k - 1.0) / (2.0 * k));
  pmm *= sqrt((2.0 * m + 1.0) / (4.0 * kPi));
  if (l == m) return pmm;
  double pm1 = x * sqrt(2.0 * m + 3.0) * pmm;
  if (l == m + 1) return pm1;
  double pll = 0.0;
  for (int ll = m + 2; ll <= l; ++ll) {
    double const a = sqrt((4.0 * ll * ll - 1.0) / (double(ll) * ll - double(m) * m));
    double const b = sqrt((double(ll - 1) * (ll - 1) - double(m) * m) / (4.0 * (ll - 1) * (ll - 1) - 1.0));
    pll = a * (x * pm1 - b * pmm);
    pmm = pm1;
    pm1 = pll;
  }
  return pll;
}

// QMCGrid::setBasisFunctions (integrateAll.hpp:88-137) with SlaterTypeOrbital::operator() and
// ::gradient (SlaterTypeOrbital.hpp:51-106), or the Ochi / hydrogen-like radial parts (basisRadial;
// OchiBasisFunction::gradient, OchiBasis.hpp:58-107, shares the angular terms of the STO gradient).  One thread per (point, function), function index
// fastest, so every store is coalesced.  Also writes the real-harmonic values phiR used by the
// contraction kernels: cos-type sqrt2 R P cos(|m| phi) for m > 0, sin-type sqrt2 R P sin(|m| phi)
// for m < 0, R P for m == 0.
__global__ void kBasis(int64_t n, int nb, int ndim, const double * __restrict__ pts, const DevSto * __restrict__ sto,
                       double * __restrict__ phiR, double * __restrict__ vals, double * __restrict__ grads)
{
  int64_t const total = n * nb;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total; idx += int64_t(gridDim.x) * blockDim.x) {
    int64_t const i = idx / nb;
    int const b = int(idx % nb);
    double const x = pts[i], y = pts[n + i], z = pts[2 * n + i];
    double const r = norm3d(x, y, z);
    double const ct = z / r;
    double const st = sqrt(x * x + y * y) / r;
    double const ph = atan2(y, x);
    DevSto const s = sto[b];
    double R, dR;
    basisRadial(s, r, R, dR);
    int const am = s.m < 0 ? -s.m : s.m;
    double const P = sphLegendre(s.l, am, ct, st);
    double sn, cs;
    sincos(double(s.m) * ph, &sn, &cs);
    double const rp = R * P;
    double pr;
    if (s.rtype == 0) pr = rp;
    else if (s.rtype == 1) pr = 1.4142135623730950488 * rp * cs;
    else pr = -1.4142135623730950488 * rp * sn;
    phiR[idx] = pr;
    if (vals) {
      if (ndim == 3) { vals[2 * idx] = rp * cs; vals[2 * idx + 1] = rp * sn; }
      else vals[idx] = rp * cs;
    }
    if (grads) {
      // SlaterTypeOrbital.hpp:63-106, arithmetic kept (including its m < 0 and pole behaviour)
      double const th = acos(ct);
      double const l = s.l, m = s.m;
      double const dRadialPart = dR;
      double const ylmRe = P * cs, ylmIm = P * sn;
      double const c1 = (s.l != s.m) ? sqrt((l - m) * (l + m + 1)) : 0.0;
      int const m1 = s.m + 1;
      double const P1 = sphLegendre(s.l, m1 < 0 ? -m1 : m1, ct, st);
      double sn1, cs1, snm, csm;
      sincos(double(m1) * ph, &sn1, &cs1);
      sincos(-ph, &snm, &csm);
      // cExp(-phi) * Y_l^{m+1}
      double const y1Re = P1 * cs1, y1Im = P1 * sn1;
      double const ylmp1Re = c1 * (csm * y1Re - snm * y1Im);
      double const ylmp1Im = c1 * (csm * y1Im + snm * y1Re);
      double const rHatRe = dRadialPart * ylmRe, rHatIm = dRadialPart * ylmIm;
      double const tnt = tan(th), sth = sin(th), cth = cos(th);
      double const thRe = (m * ylmRe / tnt + ylmp1Re) * R / r;
      double const thIm = (m * ylmIm / tnt + ylmp1Im) * R / r;
      // i m Ylm R / (r sin t)
      double const phRe = -m * ylmIm * R / (r * sth);
      double const phIm = m * ylmRe * R / (r * sth);
      double sp, cp;
      sincos(ph, &sp, &cp);
      double const rx = cp * sth, ry = sp * sth, rz = cth;
      double const tx = cp * cth, ty = sp * cth, tz = -sth;
      double const px = -sp, py = cp;
      double * g = grads + 6 * idx;
      g[0] = rHatRe * rx + thRe * tx + phRe * px;
      g[1] = rHatIm * rx + thIm * tx + phIm * px;
      g[2] = rHatRe * ry + thRe * ty + phRe * py;
      g[3] = rHatIm * ry + thIm * ty + phIm * py;
      g[4] = rHatRe * rz + thRe * tz;
      g[5] = rHatIm * rz + thIm * tz;
    }
  }
}

// ---- compensated block reduction helpers -------------------------------------------------------
__device__ __forceinline__ void twoSum(double a, double b, double & s, double & e)
{
  s = a + b;
  double const bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

// S_ij / H_ij quadrature, one block per (i, j); complex reference-basis values and gradients.
__global__ void kQuadOverlapCore(int64_t n, int nb, int Z, const double * pts, const double * w, const double2 * vals,
                                 const double2 * grads, double2 * S, double2 * H)
{
  int const i = blockIdx.x / nb, j = blockIdx.x % nb;
  double sRe = 0, sIm = 0, hRe = 0, hIm = 0;
  for (int64_t p = threadIdx.x; p < n; p += blockDim.x) {
    double2 const a = vals[p * nb + i], b = vals[p * nb + j];
    double const ovRe = a.x * b.x + a.y * b.y, ovIm = a.x * b.y - a.y * b.x;  // conj(a) b
    sRe += w[p] * ovRe;
    sIm += w[p] * ovIm;
    if (grads) {
      double const r = norm3d(pts[p], pts[n + p], pts[2 * n + p]);
      double kRe = 0, kIm = 0;
      for (int d = 0; d < 3; ++d) {
        double2 const ga = grads[(p * nb + i) * 3 + d], gb = grads[(p * nb + j) * 3 + d];
        kRe += ga.x * gb.x + ga.y * gb.y;
        kIm += ga.x * gb.y - ga.y * gb.x;
      }
      hRe += w[p] * (0.5 * kRe - Z * ovRe / r);
      hIm += w[p] * (0.5 * kIm - Z * ovIm / r);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    sRe += __shfl_xor_sync(0xffffffffu, sRe, o);
    sIm += __shfl_xor_sync(0xffffffffu, sIm, o);
    hRe += __shfl_xor_sync(0xffffffffu, hRe, o);
    hIm += __shfl_xor_sync(0xffffffffu, hIm, o);
  }
  __shared__ double red[4][32];
  int const wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { red[0][wid] = sRe; red[1][wid] = sIm; red[2][wid] = hRe; red[3][wid] = hIm; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a[4] = {0, 0, 0, 0};
    for (int k = 0; k < int(blockDim.x >> 5); ++k)
      for (int q = 0; q < 4; ++q) a[q] += red[q][k];
    S[blockIdx.x] = make_double2(a[0], a[1]);
    if (H) H[blockIdx.x] = make_double2(a[2], a[3]);
  }
}

// Fixed scratch of tcscf_overlap_core_quadrature_static: S block results, then H (2 MiB).
constexpr int kQuadStaticMaxNb = 256;
static __device__ __align__(256) double2 gQuadStaticScratch[2 * kQuadStaticMaxNb * kQuadStaticMaxNb];

// Device address of gQuadStaticScratch on the context's device, looked up once per device with that
// device current (the caller has made it current).
int quadStaticScratch(tcscf_ctx * ctx, double2 ** out)
{
  constexpr int kMaxDevices = 64;
  static std::mutex lock;
  static double2 * addr[kMaxDevices] = {};
  TCSCF_CHECK(ctx, ctx->device >= 0 && ctx->device < kMaxDevices, TCSCF_ERR_INVALID_ARGUMENT, "device index out of range");
  std::lock_guard<std::mutex> guard(lock);
  if (!addr[ctx->device]) {
    void * p = nullptr;
    cudaError_t const e = cudaGetSymbolAddress(&p, gQuadStaticScratch);
    if (e != cudaSuccess) return fail(ctx, TCSCF_ERR_CUDA, std::string("cudaGetSymbolAddress(gQuadStaticScratch): ") + cudaGetErrorString(e));
    addr[ctx->device] = static_cast<double2 *>(p);
  }
  *out = addr[ctx->device];
  return TCSCF_OK;
}

// U coefficient U[k][i] of the unitary complex -> real-harmonic map phiR_k = sum_i U[k][i] phi_i
__device__ __forceinline__ double2 urow(const DevSto * s, int k, int i)
{
  double const h = 0.70710678118654752440;
  int const t = s[k].rtype;
  if (i == k) return t == 0 ? make_double2(1, 0) : (t == 1 ? make_double2(h, 0) : make_double2(0, h));
  return t == 1 ? make_double2(h, 0) : make_double2(0, -h);
}
__device__ __forceinline__ double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// DR = conj(U) D U^T for each spin; D complex [nspin][nb][nb] (reference basis)
__global__ void kDensityToReal(int nspin, int nb, const DevSto * s, const double2 * D, double2 * DR)
{
  int const total = nspin * nb * nb;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    int const sp = idx / (nb * nb), k = (idx / nb) % nb, l = idx % nb;
    int const ik[2] = {k, s[k].partner};
    int const jl[2] = {l, s[l].partner};
    double2 acc = make_double2(0, 0);
    for (int a = 0; a < 2; ++a) {
      int const i = ik[a];
      if (i < 0) continue;
      double2 const u1 = cconj(urow(s, k, i));
      for (int b = 0; b < 2; ++b) {
        int const j = jl[b];
        if (j < 0) continue;
        double2 const t = cmul(cmul(u1, D[sp * nb * nb + i * nb + j]), urow(s, l, j));
        acc.x += t.x;
        acc.y += t.y;
      }
    }
    DR[idx] = acc;
  }
}

// symmetric real part (column-major == row-major) and the imaginary magnitude, per spin
__global__ void kSplitDensity(int nb, const double2 * DR, double * A, double * maxAbs)
{
  __shared__ double sre[256], sim[256];
  double mr = 0, mi = 0;
  for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
    int const k = idx / nb, l = idx % nb;
    double2 const a = DR[k * nb + l], b = DR[l * nb + k];
    A[idx] = 0.5 * (a.x + b.x);
    mr = fmax(mr, fabs(a.x));
    mi = fmax(mi, fabs(a.y));
  }
  sre[threadIdx.x] = mr;
  sim[threadIdx.x] = mi;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) { sre[threadIdx.x] = fmax(sre[threadIdx.x], sre[threadIdx.x + o]); sim[threadIdx.x] = fmax(sim[threadIdx.x], sim[threadIdx.x + o]); }
    __syncthreads();
  }
  if (threadIdx.x == 0) { maxAbs[0] = sre[0]; maxAbs[1] = sim[0]; }
}

// Hermitian (conj-symmetrised) copy of DR, column-major, for the complex factorisation
__global__ void kHermitianCopy(int nb, const double2 * DR, double2 * Z)
{
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nb * nb; idx += gridDim.x * blockDim.x) {
    int const row = idx % nb, col = idx / nb;   // column-major element (row, col)
    double2 const a = DR[row * nb + col], b = DR[col * nb + row];
    Z[idx] = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
  }
}

// factor matrices X1, X2 [nb][ldx] from the kept eigenpairs (real case): X2 = v sqrt|l|, X1 = sign(l) X2
constexpr int kCholeskyMaxNb = 128;

// Pivoted (diagonal-pivoting) Cholesky factorisation of the real symmetric density A [nb][nb]:
// A = L L^T with the R columns of L written to X1 and X2 ([nb][ldx], both L).  Stops when the largest
// remaining diagonal is <= 1e-12 of the largest initial diagonal; info = {R, 0}, or {R, 1} when the
// remainder is not negligible (largest |entry| above 1e-10 of the largest initial diagonal: the
// density is not positive semi-definite and the caller factors it by eigen-decomposition).  One
// block of 256 threads; shared memory nb * nb doubles (nb <= 128).
__global__ void __launch_bounds__(256) kPivotedCholesky(int nb, const double * A, int ldx, double * X1, double * X2, int * info)
{
  extern __shared__ double S[];
  __shared__ double lcol[kCholeskyMaxNb];
  __shared__ int done[kCholeskyMaxNb];
  __shared__ double rv[256];
  __shared__ int ri[256];
  int const t = threadIdx.x;
  for (int i = t; i < nb * nb; i += 256) S[i] = A[i];
  for (int i = t; i < nb; i += 256) done[i] = 0;
  __syncthreads();
  // block reduction of (value, index): largest value, smallest index among equals
  auto argmax = [&](double v, int idx, double & bv, int & bi) {
    rv[t] = v;
    ri[t] = idx;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
      if (t < o) {
        double const w = rv[t + o];
        int const wi = ri[t + o];
        if (w > rv[t] || (w == rv[t] && wi >= 0 && (ri[t] < 0 || wi < ri[t]))) { rv[t] = w; ri[t] = wi; }
      }
      __syncthreads();
    }
    bv = rv[0];
    bi = ri[0];
    __syncthreads();
  };
  double d0 = 0;
  int unused = 0;
  {
    double m = 0;
    for (int i = t; i < nb; i += 256) m = fmax(m, S[i * nb + i]);
    argmax(m, -1, d0, unused);
  }
  double const tol = 1e-12 * d0;
  int R = 0;
  for (; R < nb; ++R) {
    double best = -1.0;
    int bi = -1;
    for (int i = t; i < nb; i += 256)
      if (!done[i] && S[i * nb + i] > best) { best = S[i * nb + i]; bi = i; }
    double pv;
    int p;
    argmax(best, bi, pv, p);
    if (p < 0 || !(pv > tol)) break;
    double const sq = sqrt(pv), inv = 1.0 / sq;
    for (int i = t; i < nb; i += 256) {
      double const l = done[i] ? 0.0 : (i == p ? sq : S[i * nb + p] * inv);
      lcol[i] = l;
      X1[int64_t(i) * ldx + R] = l;
      X2[int64_t(i) * ldx + R] = l;
    }
    __syncthreads();
    for (int idx = t; idx < nb * nb; idx += 256) S[idx] -= lcol[idx / nb] * lcol[idx % nb];
    if (t == 0) done[p] = 1;
    __syncthreads();
  }
  double r = 0;
  for (int idx = t; idx < nb * nb; idx += 256)
    if (!done[idx / nb] && !done[idx % nb]) r = fmax(r, fabs(S[idx]));
  double rmax;
  argmax(r, -1, rmax, unused);
  if (t == 0) {
    info[0] = R;
    info[1] = (rmax > 1e-10 * d0 || !(rmax == rmax)) ? 1 : 0;
  }
}

// One-sided Jacobi (Hestenes) orthogonalisation of the R = info[0] factor columns L [nb][ldx] of X1
// (skipped when info[1] flags an indefinite density): L <- L W with W orthogonal, chosen so that the
// columns of L W are mutually orthogonal; X X^T = L L^T is unchanged and X's columns become the
// density's eigenvectors scaled by the square roots of its eigenvalues (the factor the fixed-point
// and TF32 contractions are accurate with: no cancellation between columns).  The result goes to
// X1 and X2.  One block of 256 threads: column pairs in round-robin order, one pair per warp at a
// time; at most 30 sweeps, ending when every pair is orthogonal to 1e-15 of its norms.
__global__ void __launch_bounds__(256) kOrthogonalizeFactor(int nb, int ldx, double * X1, double * X2, const int * info)
{
  extern __shared__ double Lc[];   // [R][nb]: column a at Lc + a * nb
  __shared__ int rotated;
  int const R = info[0];
  if (info[1] || R < 2) return;
  int const t = threadIdx.x, warp = t >> 5, lane = t & 31;
  for (int idx = t; idx < R * nb; idx += 256) Lc[idx] = X1[int64_t(idx % nb) * ldx + idx / nb];
  __syncthreads();
  int const Rp = R + (R & 1);   // an even number of slots (the last one idle when R is odd)
  for (int sweep = 0; sweep < 30; ++sweep) {
    if (t == 0) rotated = 0;
    __syncthreads();
    for (int step = 0; step < Rp - 1; ++step) {
      for (int k = warp; k < Rp / 2; k += 8) {
        int const a = k == 0 ? Rp - 1 : (step + k) % (Rp - 1);
        int const b = k == 0 ? step : (step - k + Rp - 1) % (Rp - 1);
        if (a >= R || b >= R) continue;
        double * ca = Lc + a * nb;
        double * cb = Lc + b * nb;
        double al = 0, be = 0, ga = 0;
        for (int i = lane; i < nb; i += 32) {
          al += ca[i] * ca[i];
          be += cb[i] * cb[i];
          ga += ca[i] * cb[i];
        }
        for (int o = 16; o > 0; o >>= 1) {
          al += __shfl_xor_sync(0xffffffffu, al, o);
          be += __shfl_xor_sync(0xffffffffu, be, o);
          ga += __shfl_xor_sync(0xffffffffu, ga, o);
        }
        if (!(fabs(ga) > 1e-15 * sqrt(al * be))) continue;
        double const zeta = (be - al) / (2.0 * ga);
        double const tn = copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        double const c = 1.0 / sqrt(1.0 + tn * tn), sn = c * tn;
        for (int i = lane; i < nb; i += 32) {
          double const x = ca[i], y = cb[i];
          ca[i] = c * x - sn * y;
          cb[i] = sn * x + c * y;
        }
        if (lane == 0) rotated = 1;
      }
      __syncthreads();
    }
    if (!rotated) break;
    __syncthreads();
  }
  for (int idx = t; idx < R * nb; idx += 256) {
    int64_t const o = int64_t(idx % nb) * ldx + idx / nb;
    X1[o] = Lc[idx];
    X2[o] = Lc[idx];
  }
}

// status of a density the pivoted Cholesky does not take (nb > 128): factor by eigen-decomposition
__global__ void kMarkIndefinite(int * info)
{
  if (threadIdx.x == 0) { info[0] = 0; info[1] = 1; }
}

__global__ void kRealFactors(int nb, int nkeep, const int * keep, const double * W, const double * V, int ldx, double * X1, double * X2)
{
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nb * nkeep; idx += gridDim.x * blockDim.x) {
    int const k = idx / nkeep, b = idx % nkeep;
    int const e = keep[b];
    double const lam = W[e];
    double const sq = sqrt(fabs(lam));
    double const v = V[e * nb + k] * sq;
    X2[k * ldx + b] = v;
    X1[k * ldx + b] = lam < 0 ? -v : v;
  }
}

// complex case: X2 = [Re z | Im z], X1re = [l Re z | l Im z], X1im = [l Im z | -l Re z]
__global__ void kComplexFactors(int nb, int nkeep, const int * keep, const double * W, const double2 * Z, int ldx, double * X1re,
                                double * X1im, double * X2)
{
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nb * nkeep; idx += gridDim.x * blockDim.x) {
    int const k = idx / nkeep, b = idx % nkeep;
    int const e = keep[b];
    double const lam = W[e];
    double2 const z = Z[e * nb + k];
    X2[k * ldx + b] = z.x;
    X2[k * ldx + nkeep + b] = z.y;
    X1re[k * ldx + b] = lam * z.x;
    X1re[k * ldx + nkeep + b] = lam * z.y;
    X1im[k * ldx + b] = lam * z.y;
    X1im[k * ldx + nkeep + b] = -lam * z.x;
  }
}

// psi[r][b] = sum_k phi[r][k] X[k][b]  (FP64), b < R, row stride ld
__global__ void kOrbitals(int64_t n, int nb, int R, const double * __restrict__ phi, const double * __restrict__ X, int ldx,
                          double * __restrict__ psi, int ld)
{
  extern __shared__ double sXo[];
  for (int i = threadIdx.x; i < nb * R; i += blockDim.x) sXo[i] = X[(i / R) * ldx + (i % R)];
  __syncthreads();
  int64_t const total = n * R;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total; idx += int64_t(gridDim.x) * blockDim.x) {
    int64_t const r = idx / R;
    int const b = int(idx % R);
    double s = 0;
    const double * pr = phi + r * nb;
    for (int k = 0; k < nb; ++k) s = fma(pr[k], sXo[k * R + b], s);
    psi[r * ld + b] = s;
  }
}

// coul[r] = scale w[r] sum_b psiA[r][b] psiB[r][b]
__global__ void kCoulombSource(int64_t n, int R, const double * psiA, const double * psiB, int ld, const double * w, double scale, double * coul)
{
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n; r += int64_t(gridDim.x) * blockDim.x) {
    double s = 0;
    for (int b = 0; b < R; ++b) s = fma(psiA[r * ld + b], psiB[r * ld + b], s);
    coul[r] = scale * w[r] * s;
  }
}

// V[r][l] = scale w[r] phi[r][l]
__global__ void kWeightedBasis(int64_t n, int nb, const double * phi, const double * w, double scale, double * V)
{
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < n * nb; idx += int64_t(gridDim.x) * blockDim.x)
    V[idx] = scale * w[idx / nb] * phi[idx];
}

// V[r][p(k,l)] = scale w[r] phi[r][k] phi[r][l], k <= l, pair index p = k*nb - k(k-1)/2 + (l-k)
__global__ void kPairProducts(int64_t n, int nb, const double * phi, const double * w, double scale, double * V)
{
  int const np = nb * (nb + 1) / 2;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < n * np; idx += int64_t(gridDim.x) * blockDim.x) {
    int64_t const r = idx / np;
    int p = int(idx % np);
    int k = 0;
    while (p >= nb - k) { p -= nb - k; ++k; }
    int const l = k + p;
    V[idx] = scale * w[r] * phi[r * nb + k] * phi[r * nb + l];
  }
}

__device__ __forceinline__ int pairIndex(int nb, int k, int l)
{
  if (k > l) { int t = k; k = l; l = t; }
  return k * nb - k * (k - 1) / 2 + (l - k);
}

// F(j,i) = sum_{k,l} U[k][j] FR(k,l) conj(U[l][i]) per r1 row; FR packed symmetric [n1][np] (component c of ncomp)
// out complex [n1][nb][nb](*ncomp) or real (x 1) when realOut
__global__ void kPairsToReference(int64_t n1, int nb, const DevSto * s, const double * FR, int ncomp, int comp, int realOut, double * out)
{
  int const np = nb * (nb + 1) / 2;
  int64_t const total = n1 * nb * nb;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total; idx += int64_t(gridDim.x) * blockDim.x) {
    int64_t const r = idx / (nb * nb);
    int const j = int((idx / nb) % nb), i = int(idx % nb);
    int const kj[2] = {j, s[j].partner};
    int const li[2] = {i, s[i].partner};
    double2 acc = make_double2(0, 0);
    for (int a = 0; a < 2; ++a) {
      int const k = kj[a];
      if (k < 0) continue;
      double2 const uk = urow(s, k, j);
      for (int b = 0; b < 2; ++b) {
        int const l = li[b];
        if (l < 0) continue;
        double const f = FR[r * np + pairIndex(nb, k, l)];
        double2 const t = cmul(uk, cconj(urow(s, l, i)));
        acc.x += f * t.x;
        acc.y += f * t.y;
      }
    }
    if (realOut) out[idx] = acc.x;
    else {
      out[2 * (idx * ncomp + comp)] = acc.x;
      out[2 * (idx * ncomp + comp) + 1] = acc.y;
    }
  }
}

// G(j,i) = sum_{k,l} U[k][j] GR(k,l) conj(U[l][i]); GR complex [nspin][nb][nb] given as re/im planes
__global__ void kRealToReference(int nspin, int nb, const DevSto * s, const double * GRre, const double * GRim, double2 * G)
{
  int const total = nspin * nb * nb;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    int const sp = idx / (nb * nb), j = (idx / nb) % nb, i = idx % nb;
    int const kj[2] = {j, s[j].partner};
    int const li[2] = {i, s[i].partner};
    double2 acc = make_double2(0, 0);
    for (int a = 0; a < 2; ++a) {
      int const k = kj[a];
      if (k < 0) continue;
      double2 const uk = urow(s, k, j);
      for (int b = 0; b < 2; ++b) {
        int const l = li[b];
        if (l < 0) continue;
        int64_t const o = int64_t(sp) * nb * nb + k * nb + l;
        double2 const g = make_double2(GRre[o], GRim ? GRim[o] : 0.0);
        double2 const t = cmul(cmul(uk, g), cconj(urow(s, l, i)));
        acc.x += t.x;
        acc.y += t.y;
      }
    }
    G[idx] = acc;
  }
}

// enforceOneElectronSymmetry (HartreeFock.cpp:758-780) and constructSCFOperator (:48-98) with a
// compensated FP64 energy sum.  One block.  energy = factor * Re sum D(i,j) (h(j,i) + G(j,i)/2 - G3(j,i)/3)
__global__ void kFinalize(int nspin, int nb, const double * h, double2 * G, const double2 * G3, const double2 * D, int respectSym,
                          double factor, double2 * fock, double * energy)
{
  __shared__ double ss[512], se[512];
  double s = 0, c = 0;
  int const nn = nb * nb;
  for (int idx = threadIdx.x; idx < nspin * nn; idx += blockDim.x) {
    int const sp = idx / nn, ji = idx % nn, j = ji / nb, i = ji % nb;
    double2 g = G[idx];
    double2 g3 = G3 ? G3[idx] : make_double2(0, 0);
    if (respectSym && !(fabs(h[ji]) > 0)) { g = make_double2(0, 0); g3 = make_double2(0, 0); }
    G[idx] = g;
    double2 f = make_double2(h[ji] + g.x - g3.x, g.y - g3.y);
    if (fock) fock[idx] = f;
    double2 const e = make_double2(h[ji] + g.x / 2 - g3.x / 3, g.y / 2 - g3.y / 3);
    double2 const d = D[int64_t(sp) * nn + i * nb + j];
    double const term = d.x * e.x - d.y * e.y;
    double t, err;
    twoSum(s, term, t, err);
    s = t;
    c += err;
  }
  ss[threadIdx.x] = s;
  se[threadIdx.x] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0, comp = 0;
    for (int k = 0; k < int(blockDim.x); ++k) {
      double t, err;
      twoSum(tot, ss[k], t, err);
      tot = t;
      comp += err + se[k];
    }
    energy[0] = factor * (tot + comp);
  }
}

// Faa(r) (+)= sum_ji F(r,j,i) D(i,j) ; Fai(r,i) (+)= sum_j (sum_k D(k,j) vals(r,k)) F(r,j,i)
// (calculateIaa / calculateFai, HartreeFock.cpp:144-213) for one spin density; one block per row.
template <bool CX>
__global__ void kFaaFai(int64_t n1, int nb, const double * F, const double2 * vals, const double2 * D, double2 * Faa, double2 * Fai)
{
  extern __shared__ double2 sk[];
  int64_t const r = blockIdx.x;
  int const tid = threadIdx.x;
  for (int j = tid; j < nb; j += blockDim.x) {
    double2 a = make_double2(0, 0);
    for (int k = 0; k < nb; ++k) {
      double2 const t = cmul(D[k * nb + j], vals[r * nb + k]);
      a.x += t.x; a.y += t.y;
    }
    sk[j] = a;
  }
  __syncthreads();
  int64_t const base = r * nb * nb;
  auto fval = [&](int j, int i) -> double2 {
    if (CX) return reinterpret_cast<const double2 *>(F)[base + j * nb + i];
    return make_double2(F[base + j * nb + i], 0.0);
  };
  for (int i = tid; i < nb; i += blockDim.x) {
    double2 a = make_double2(0, 0);
    for (int j = 0; j < nb; ++j) {
      double2 const t = cmul(sk[j], fval(j, i));
      a.x += t.x; a.y += t.y;
    }
    Fai[r * nb + i].x += a.x;
    Fai[r * nb + i].y += a.y;
  }
  double sr = 0, si = 0;
  for (int e = tid; e < nb * nb; e += blockDim.x) {
    int const j = e / nb, i = e % nb;
    double2 const t = cmul(fval(j, i), D[i * nb + j]);
    sr += t.x; si += t.y;
  }
  for (int o = 16; o > 0; o >>= 1) { sr += __shfl_xor_sync(0xffffffffu, sr, o); si += __shfl_xor_sync(0xffffffffu, si, o); }
  __shared__ double red[2][32];
  if ((tid & 31) == 0) { red[0][tid >> 5] = sr; red[1][tid >> 5] = si; }
  __syncthreads();
  if (tid == 0) {
    double a = 0, b = 0;
    for (int k = 0; k < int(blockDim.x >> 5); ++k) { a += red[0][k]; b += red[1][k]; }
    Faa[r].x += a;
    Faa[r].y += b;
  }
}

__global__ void kAddInto(int64_t n, const double * a, double * out)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) out[i] += a[i];
}

// out[i][j] += a[j][i] (nb x nb, row-major)
__global__ void kAddTransposed(int nb, const double * a, double * out)
{
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nb * nb; idx += gridDim.x * blockDim.x) out[idx] += a[(idx % nb) * nb + idx / nb];
}

// column-major complex copy of the row-major (j,i) Fock matrix, and of a real row-major S
__global__ void kToColumnMajor(int nb, const double2 * fockRow, const double * S, double2 * A, double2 * B)
{
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nb * nb; idx += gridDim.x * blockDim.x) {
    int const row = idx % nb, col = idx / nb;
    A[idx] = fockRow[row * nb + col];
    B[idx] = make_double2(S[row * nb + col], 0.0);
  }
}

// getNewDensity (HartreeFock.cpp:20-44): D(u,v) = sum_a C(u,a) conj(C(v,a)); C column-major
__global__ void kDensityFromOrbitals(int nb, int nocc, const double2 * C, double2 * D)
{
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nb * nb; idx += gridDim.x * blockDim.x) {
    int const u = idx / nb, v = idx % nb;
    double2 t = make_double2(0, 0);
    for (int a = 0; a < nocc; ++a) {
      double2 const x = cmul(C[a * nb + u], cconj(C[a * nb + v]));
      t.x += x.x; t.y += x.y;
    }
    D[idx] = t;
  }
}

// real-harmonic density DR(u,v) = sum_a C(u,a) C(v,a) from real eigenvectors C (column-major)
__global__ void kRealDensity(int nb, int nocc, const double * C, double * DR)
{
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nb * nb; idx += gridDim.x * blockDim.x) {
    int const u = idx / nb, v = idx % nb;
    double t = 0;
    for (int a = 0; a < nocc; ++a) t += C[a * nb + u] * C[a * nb + v];
    DR[idx] = t;
  }
}

// the occupied eigenvectors of a real-harmonic eigen-solve (columns of the column-major C) as the
// density factor X [nb][ldx] (X[k][a] = C[a][k]): D_R = X X^T, the density kRealDensity forms
__global__ void kFactorFromOrbitals(int nb, int nocc, const double * C, int ldx, double * X)
{
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nb * nocc; idx += gridDim.x * blockDim.x) {
    int const k = idx / nocc, a = idx % nocc;
    X[int64_t(k) * ldx + a] = C[a * nb + k];
  }
}

// ---- Pulay DIIS (optional SCF acceleration; the reference iterates plain Roothaan steps) ---------
// dots[j] = Re <E[slot], E[j]> (Frobenius product of the commutator error matrices of both spins)
// for the used history slots j < count, one block per j
__global__ void kDiisDots(int64_t len, int slot, int count, const double2 * E, double * dots)
{
  __shared__ double red[256];
  int const j = blockIdx.x;
  if (j >= count) return;
  double acc = 0;
  for (int64_t i = threadIdx.x; i < len; i += blockDim.x) {
    double2 const a = E[int64_t(slot) * len + i], b = E[int64_t(j) * len + i];
    acc += a.x * b.x + a.y * b.y;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) dots[j] = red[0];
}

// F = sum_j c[j] Fh[j]
__global__ void kDiisCombine(int64_t len, int count, const double * c, const double2 * Fh, double2 * F)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < len; i += int64_t(gridDim.x) * blockDim.x) {
    double2 a = make_double2(0, 0);
    for (int j = 0; j < count; ++j) {
      double2 const f = Fh[int64_t(j) * len + i];
      a.x += c[j] * f.x;
      a.y += c[j] * f.y;
    }
    F[i] = a;
  }
}

__global__ void kRealToComplex(int64_t n, const double * a, double2 * b)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) b[i] = make_double2(a[i], 0.0);
}

// row-major C = alpha A B + beta C (n x n complex) through column-major cuBLAS: C^T = B^T A^T
int rowMajorZgemm(tcscf_ctx * ctx, cublasHandle_t h, int n, double2 alpha, const double2 * A, const double2 * B, double2 beta, double2 * C)
{
  cuDoubleComplex const al = make_cuDoubleComplex(alpha.x, alpha.y), be = make_cuDoubleComplex(beta.x, beta.y);
  if (cublasZgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &al, reinterpret_cast<const cuDoubleComplex *>(B), n,
                  reinterpret_cast<const cuDoubleComplex *>(A), n, &be, reinterpret_cast<cuDoubleComplex *>(C), n) != CUBLAS_STATUS_SUCCESS)
    return fail(ctx, TCSCF_ERR_CUDA, "cublasZgemm failed");
  return TCSCF_OK;
}

// Solves the DIIS equations [B -1; -1 0] [c; lambda] = [0; -1] (B m x m, row stride ld) by Gaussian
// elimination with partial pivoting; false when singular
bool solveDiis(int m, std::vector<double> const & B, int ld, std::vector<double> & c)
{
  int const n = m + 1;
  std::vector<double> A(size_t(n) * (n + 1), 0.0);
  for (int i = 0; i < m; ++i) {
    for (int j = 0; j < m; ++j) A[i * (n + 1) + j] = B[i * ld + j];
    A[i * (n + 1) + m] = -1;
    A[m * (n + 1) + i] = -1;
  }
  A[m * (n + 1) + n] = -1;
  for (int k = 0; k < n; ++k) {
    int p = k;
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(A[i * (n + 1) + k]) > std::fabs(A[p * (n + 1) + k])) p = i;
    if (!(std::fabs(A[p * (n + 1) + k]) > 0)) return false;
    if (p != k)
      for (int j = 0; j <= n; ++j) std::swap(A[k * (n + 1) + j], A[p * (n + 1) + j]);
    for (int i = k + 1; i < n; ++i) {
      double const f = A[i * (n + 1) + k] / A[k * (n + 1) + k];
      for (int j = k; j <= n; ++j) A[i * (n + 1) + j] -= f * A[k * (n + 1) + j];
    }
  }
  std::vector<double> x(n);
  for (int i = n - 1; i >= 0; --i) {
    double t = A[i * (n + 1) + n];
    for (int j = i + 1; j < n; ++j) t -= A[i * (n + 1) + j] * x[j];
    x[i] = t / A[i * (n + 1) + i];
  }
  c.assign(x.begin(), x.begin() + m);
  for (double v : c)
    if (!(v == v)) return false;
  return true;
}

}  // namespace

int finalizeLaunch(tcscf_ctx * ctx, int nspin, int nb, const double * h, double2 * G, const double2 * G3, const double2 * D, int respectSym,
                   double factor, double2 * fock, double * energy)
{
  kFinalize<<<1, 512, 0, ctx->stream>>>(nspin, nb, h, G, G3, D, respectSym, factor, fock, energy);
  TCSCF_LAUNCH(ctx);
  return TCSCF_OK;
}

// ------------------------------------------------------------------------------------------------
// Fock-build pipeline
// ------------------------------------------------------------------------------------------------
namespace {

struct Factor {
  int R = 0;          // columns of the factor matrices
  bool complex = false;
  bool same = false;  // X1 == X2 (the pivoted Cholesky factor of a positive semi-definite real density)
  double * X1 = nullptr, * X1im = nullptr, * X2 = nullptr;   // device [nb][ldx]
  int ldx = 0;
};

// Factor the spin density's real-harmonic form DR = X1 X2^T (real) or, for a density that is not
// real in the real-harmonic basis, into the real/imaginary pair described in kComplexFactors.
// Device buffers of one density factorisation: the real-harmonic density DR, its symmetrised real
// part A, the factors X1 (X1im) and X2 [nb][ldx], and the status {max |Re DR|, max |Im DR|} with the
// pivoted-Cholesky rank and flag behind it (FactorStatus).
struct FactorStatus {
  double maxAbs[2];
  int rank, indefinite;
};
struct FactorBufs {
  double2 * DR = nullptr;
  double * A = nullptr;
  double * X1 = nullptr, * X1im = nullptr, * X2 = nullptr;
  FactorStatus * status = nullptr;
};
size_t factorBufBytes(int nb)
{
  size_t const nn = size_t(nb) * nb;
  return nn * sizeof(double2) + nn * sizeof(double) + 3 * nn * 2 * sizeof(double) + 2 * sizeof(FactorStatus) + 256;
}
FactorBufs carveFactorBufs(void * p, int nb)
{
  size_t const nn = size_t(nb) * nb;
  char * base = static_cast<char *>(p);
  FactorBufs b;
  b.DR = reinterpret_cast<double2 *>(base); base += nn * sizeof(double2);
  b.A = reinterpret_cast<double *>(base); base += nn * sizeof(double);
  b.X1 = reinterpret_cast<double *>(base); base += nn * 2 * sizeof(double);
  b.X1im = reinterpret_cast<double *>(base); base += nn * 2 * sizeof(double);
  b.X2 = reinterpret_cast<double *>(base); base += nn * 2 * sizeof(double);
  b.status = reinterpret_cast<FactorStatus *>(base);
  return b;
}

// Launches (no host synchronisation) the real-harmonic transform of the spin density, its split
// into real and imaginary magnitudes, and the pivoted Cholesky factorisation of its real part.
int factorLaunch(tcscf_ctx * ctx, Grid & g, const double2 * dD, FactorBufs const & b)
{
  int const nb = g.nb;
  size_t const nn = size_t(nb) * nb;
  kDensityToReal<<<gridBlocks(nn, 256), 256, 0, ctx->stream>>>(1, nb, g.dsto, dD, b.DR);
  TCSCF_LAUNCH(ctx);
  kSplitDensity<<<1, 256, 0, ctx->stream>>>(nb, b.DR, b.A, b.status->maxAbs);
  TCSCF_LAUNCH(ctx);
  if (nb <= kCholeskyMaxNb) {
    TCSCF_CUDA(ctx, cudaFuncSetAttribute(kPivotedCholesky, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(double) * kCholeskyMaxNb * kCholeskyMaxNb)));
    kPivotedCholesky<<<1, 256, sizeof(double) * nn, ctx->stream>>>(nb, b.A, 2 * nb, b.X1, b.X2, &b.status->rank);
    TCSCF_LAUNCH(ctx);
    TCSCF_CUDA(ctx, cudaFuncSetAttribute(kOrthogonalizeFactor, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(double) * kCholeskyMaxNb * kCholeskyMaxNb)));
    kOrthogonalizeFactor<<<1, 256, sizeof(double) * nn, ctx->stream>>>(nb, 2 * nb, b.X1, b.X2, &b.status->rank);
    TCSCF_LAUNCH(ctx);
  } else {
    kMarkIndefinite<<<1, 32, 0, ctx->stream>>>(&b.status->rank);
    TCSCF_LAUNCH(ctx);
  }
  return TCSCF_OK;
}

// Completes the factorisation from the status read back to the host: the pivoted Cholesky factor
// with orthogonalised columns (X1 = X2 = L W) when the density is real and positive semi-definite in
// the real-harmonic basis,
// otherwise the eigen-decomposition (real: DR = X1 X2^T with X1 = V sign(l) sqrt|l|, X2 = V sqrt|l|;
// complex: the real/imaginary pair described in kComplexFactors), keeping the eigenvalues above
// 1e-12 of the largest.
int factorFinish(tcscf_ctx * ctx, Grid & g, FactorBufs const & b, FactorStatus const & st, Factor & f)
{
  int const nb = g.nb;
  size_t const nn = size_t(nb) * nb;
  f.X1 = b.X1; f.X1im = b.X1im; f.X2 = b.X2;
  f.ldx = 2 * nb;
  double const hmax[2] = {st.maxAbs[0], st.maxAbs[1]};
  if (!(hmax[0] == hmax[0]) || !(hmax[1] == hmax[1])) return fail(ctx, TCSCF_ERR_NONFINITE, "non-finite density");
  // an imaginary part below 1e-10 of the real part is rounding (SCF densities from the complex
  // eigen-solver carry ~1e-12): the density is factored as real, dropping it
  f.complex = hmax[1] > 1e-10 * std::max(hmax[0], 1e-300);
  if (hmax[0] == 0 && hmax[1] == 0) { f.R = 0; return TCSCF_OK; }
  if (!f.complex && !st.indefinite) { f.R = st.rank; f.same = true; return TCSCF_OK; }

  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, "fac_eig", nn * sizeof(double2) * 2 + nn * sizeof(double) + 64 * sizeof(double) + nb * sizeof(int) + 1024, &p));
  char * base = static_cast<char *>(p);
  double2 * Z = reinterpret_cast<double2 *>(base); base += nn * sizeof(double2) * 2;
  double * W = reinterpret_cast<double *>(base); base += nn * sizeof(double);
  int * devInfo = reinterpret_cast<int *>(base); base += 64 * sizeof(double);
  int * keep = reinterpret_cast<int *>(base);
  double * A = b.A;
  int lwork = 0;
  std::vector<double> hW(nb);
  if (!f.complex) {
    if (cusolverDnDsyevd_bufferSize(ctx->solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, nb, A, nb, W, &lwork) != CUSOLVER_STATUS_SUCCESS)
      return fail(ctx, TCSCF_ERR_LINALG, "cusolverDnDsyevd_bufferSize failed");
    void * wk = nullptr;
    TCSCF_TRY(scratch(ctx, "syevd_work", size_t(lwork) * sizeof(double) + 64, &wk));
    if (cusolverDnDsyevd(ctx->solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, nb, A, nb, W, static_cast<double *>(wk), lwork, devInfo) != CUSOLVER_STATUS_SUCCESS)
      return fail(ctx, TCSCF_ERR_LINALG, "cusolverDnDsyevd failed");
  } else {
    kHermitianCopy<<<gridBlocks(nn, 256), 256, 0, ctx->stream>>>(nb, b.DR, Z);
    TCSCF_LAUNCH(ctx);
    if (cusolverDnZheevd_bufferSize(ctx->solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, nb, reinterpret_cast<cuDoubleComplex *>(Z), nb, W, &lwork) != CUSOLVER_STATUS_SUCCESS)
      return fail(ctx, TCSCF_ERR_LINALG, "cusolverDnZheevd_bufferSize failed");
    void * wk = nullptr;
    TCSCF_TRY(scratch(ctx, "heevd_work", size_t(lwork) * sizeof(double2) + 64, &wk));
    if (cusolverDnZheevd(ctx->solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, nb, reinterpret_cast<cuDoubleComplex *>(Z), nb, W,
                         static_cast<cuDoubleComplex *>(wk), lwork, devInfo) != CUSOLVER_STATUS_SUCCESS)
      return fail(ctx, TCSCF_ERR_LINALG, "cusolverDnZheevd failed");
  }
  int info = 0;
  TCSCF_CUDA(ctx, cudaMemcpyAsync(hW.data(), W, nb * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemcpyAsync(&info, devInfo, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (info != 0) return fail(ctx, TCSCF_ERR_LINALG, "density eigen-decomposition failed");
  double lmax = 0;
  for (double v : hW) lmax = std::max(lmax, std::fabs(v));
  std::vector<int> hk;
  for (int e = nb - 1; e >= 0; --e)
    if (std::fabs(hW[e]) > 1e-12 * lmax) hk.push_back(e);
  int const nk = int(hk.size());
  if (nk == 0) { f.R = 0; return TCSCF_OK; }
  TCSCF_CUDA(ctx, cudaMemcpyAsync(keep, hk.data(), nk * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  if (!f.complex) {
    kRealFactors<<<gridBlocks(int64_t(nb) * nk, 256), 256, 0, ctx->stream>>>(nb, nk, keep, W, A, f.ldx, f.X1, f.X2);
    f.R = nk;
  } else {
    kComplexFactors<<<gridBlocks(int64_t(nb) * nk, 256), 256, 0, ctx->stream>>>(nb, nk, keep, W, Z, f.ldx, f.X1, f.X1im, f.X2);
    f.R = 2 * nk;
  }
  TCSCF_LAUNCH(ctx);
  // host vectors go out of scope only after the stream has consumed `keep`
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TCSCF_OK;
}

// Factor the spin density's real-harmonic form DR = X1 X2^T (one host synchronisation when the
// pivoted Cholesky factor applies; see factorFinish).
int factorDensity(tcscf_ctx * ctx, Grid & g, const double2 * dD, int spin, Factor & f)
{
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, spin ? "fac1" : "fac0", factorBufBytes(g.nb), &p));
  FactorBufs const b = carveFactorBufs(p, g.nb);
  TCSCF_TRY(factorLaunch(ctx, g, dD, b));
  FactorStatus st;
  TCSCF_CUDA(ctx, cudaMemcpyAsync(&st, b.status, sizeof(FactorStatus), cudaMemcpyDeviceToHost, ctx->stream));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return factorFinish(ctx, g, b, st, f);
}

int checkBasisPair(tcscf_ctx * ctx, Grid * g1, Grid * g2)
{
  TCSCF_CHECK(ctx, g1 && g2, TCSCF_ERR_INVALID_ARGUMENT, "unknown grid handle");
  TCSCF_CHECK(ctx, g1->nb > 0 && g2->nb > 0, TCSCF_ERR_INVALID_ARGUMENT, "setBasisFunctions has not been called on the grid");
  TCSCF_CHECK(ctx, g1->nb == g2->nb, TCSCF_ERR_INVALID_ARGUMENT, "r1Grid.nBasis() != r2Grid.nBasis()");
  TCSCF_CHECK(ctx, g1->ndim == 3, TCSCF_ERR_INVALID_ARGUMENT, "the r1 grid must be three dimensional");
  for (int b = 0; b < g1->nb; ++b) {
    tcscf_sto const & a = g1->basis[b];
    tcscf_sto const & c = g2->basis[b];
    TCSCF_CHECK(ctx, a.alpha == c.alpha && a.n == c.n && a.l == c.l && a.m == c.m && a.family == c.family, TCSCF_ERR_INVALID_ARGUMENT,
                "r1 and r2 grids carry different basis sets");
  }
  return TCSCF_OK;
}

// Direct-form Fock build with device-resident densities dD [nspin][nb][nb] complex.
// Leaves G (masked), Fock (row-major) and the energy on the device.
int fockBuildDevice(tcscf_ctx * ctx, Grid & g1, Grid & g2, int nspin, const double2 * dD, const double * dH, int respectSym,
                    int precision, double2 * dG, double2 * dFock, double * dE, Factor const * given)
{
  int const nb = g1.nb;
  int64_t const n1 = g1.n, n2 = g2.n;
  double const scale = g2.ndim == 2 ? 2 * kPi : 1.0;
  int const ldt = nb;
  int const ldpsi = 2 * nb;
  size_t const bytes = sizeof(double) * (size_t(n2) * nb                 // V
                                         + size_t(n1) * ldpsi + 2 * size_t(n2) * ldpsi  // psi1, psi2, psi1 on r2
                                         + size_t(n2)                              // coul
                                         + size_t(nspin) * n1 * ldt                // T re
                                         + size_t(nspin) * n1 * ldt                // T im
                                         + size_t(nspin) * n1 + n1                 // VH per spin + total
                                         + size_t(nspin) * nb * nb * 2);           // GR re/im
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, "fock", bytes, &p));
  double * V = static_cast<double *>(p);
  double * psi1 = V + size_t(n2) * nb;
  double * psi2 = psi1 + size_t(n1) * ldpsi;
  double * psi1at2 = psi2 + size_t(n2) * ldpsi;
  double * coul = psi1at2 + size_t(n2) * ldpsi;
  double * Tre = coul + n2;
  double * Tim = Tre + size_t(nspin) * n1 * ldt;
  double * VH = Tim + size_t(nspin) * n1 * ldt;
  double * VHtot = VH + size_t(nspin) * n1;
  double * GRre = VHtot + n1;
  double * GRim = GRre + size_t(nspin) * nb * nb;

  cudaEventRecord(ctx->ev[0], ctx->stream);
  int const launch0 = ctx->launchCount;
  kWeightedBasis<<<gridBlocks(n2 * nb, 256), 256, 0, ctx->stream>>>(n2, nb, g2.phiR, g2.w, scale, V);
  TCSCF_LAUNCH(ctx);
  TCSCF_CUDA(ctx, cudaMemsetAsync(VH, 0, sizeof(double) * (size_t(nspin) * n1 + n1), ctx->stream));
  TCSCF_CUDA(ctx, cudaMemsetAsync(GRre, 0, sizeof(double) * size_t(nspin) * nb * nb * 2, ctx->stream));
  bool anyComplex = false;
  bool symSpin[2] = {false, false};
  double contractionMs = 0;
  const void * vtPacked = nullptr;
  if (precision == TCSCF_PREC_BF16X3) TCSCF_TRY(tensorPackedV(ctx, g2, V, scale, &vtPacked));
  for (int s = 0; s < nspin; ++s) {
    Factor f;
    if (given && given[s].X1) f = given[s];   // the caller's factor of this spin's density (its occupied orbitals)
    else TCSCF_TRY(factorDensity(ctx, g1, dD + size_t(s) * nb * nb, s, f));
    double * Ts = Tre + size_t(s) * n1 * ldt;
    double * Ti = Tim + size_t(s) * n1 * ldt;
    if (f.R == 0) {
      TCSCF_CUDA(ctx, cudaMemsetAsync(Ts, 0, sizeof(double) * n1 * ldt, ctx->stream));
      continue;
    }
    int const R = f.R;
    // one grid on both sides and X1 = X2: psi1 = psi2 and X = g rho is symmetric, so the split-BF16 and
    // FP64 contractions compute only the pairs on and above each r1 tile's diagonal (T'), and the
    // exchange matrix is sum W T' plus its transpose (TF32 keeps the full form: tensorPrepare)
    bool const sym = precision != TCSCF_PREC_TF32 && &g1 == &g2 && f.same;
    symSpin[s] = sym;
    for (int part = 0; part < (f.complex ? 2 : 1); ++part) {
      double const * X1 = part == 0 ? f.X1 : f.X1im;
      size_t const sm = sizeof(double) * size_t(nb) * R;
      kOrbitals<<<gridBlocks(n1 * R, 256), 256, sm, ctx->stream>>>(n1, nb, R, g1.phiR, X1, f.ldx, psi1, ldpsi);
      TCSCF_LAUNCH(ctx);
      if (part == 0 && !sym) {
        kOrbitals<<<gridBlocks(n2 * R, 256), 256, sm, ctx->stream>>>(n2, nb, R, g2.phiR, f.X2, f.ldx, psi2, ldpsi);
        TCSCF_LAUNCH(ctx);
        // rho(r2, r2) needs the r1-side factor evaluated on the r2 points
        kOrbitals<<<gridBlocks(n2 * R, 256), 256, sm, ctx->stream>>>(n2, nb, R, g2.phiR, f.X1, f.ldx, psi1at2, ldpsi);
        TCSCF_LAUNCH(ctx);
      }
      double const * p2side = sym ? psi1 : psi2;
      Contraction c;
      c.n1 = n1; c.n2 = n2; c.R = R; c.ncol = nb;
      c.p1 = g1.pts; c.p2 = g2.pts; c.psi1 = psi1; c.psi2 = p2side; c.ldpsi = ldpsi;
      c.V = V; c.ldv = nb; c.T = part == 0 ? Ts : Ti; c.ldt = ldt;
      c.vtPacked = vtPacked;
      c.sym = sym ? 1 : 0;
      if (precision != TCSCF_PREC_FP64) TCSCF_TRY(nearPairsFor(ctx, g1, g2, &c.near));
      if (part == 0) {
        kCoulombSource<<<gridBlocks(n2, 256), 256, 0, ctx->stream>>>(n2, R, sym ? psi1 : psi1at2, p2side, ldpsi, g2.w, scale, coul);
        TCSCF_LAUNCH(ctx);
        c.coul = coul;
        c.VH = VH + size_t(s) * n1;
      }
      // the contraction routines bracket their main kernel with ev[2] / ev[3]
      if (precision == TCSCF_PREC_FP64) TCSCF_TRY(contractFp64(ctx, c));
      else TCSCF_TRY(contractTensor(ctx, c, precision));
      TCSCF_CUDA(ctx, cudaEventSynchronize(ctx->ev[3]));
      float ms = 0;
      cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]);
      contractionMs += ms;
    }
    if (f.complex) anyComplex = true;
    else TCSCF_CUDA(ctx, cudaMemsetAsync(Ti, 0, sizeof(double) * n1 * ldt, ctx->stream));
  }
  for (int s = 0; s < nspin; ++s) {
    kAddInto<<<gridBlocks(n1, 256), 256, 0, ctx->stream>>>(n1, VH + size_t(s) * n1, VHtot);
    TCSCF_LAUNCH(ctx);
  }
  double const cJ = nspin == 1 ? 2.0 : 1.0;
  double * GRhalf = nullptr;
  if (symSpin[0] || symSpin[1]) TCSCF_TRY(scratch(ctx, "fock_sym_half", sizeof(double) * size_t(nb) * nb, reinterpret_cast<void **>(&GRhalf)));
  for (int s = 0; s < nspin; ++s) {
    TCSCF_TRY(reduceFockReal(ctx, n1, nb, g1.phiR, g1.w, VHtot, cJ, Tre + size_t(s) * n1 * ldt, ldt, 1.0, GRre + size_t(s) * nb * nb));
    if (symSpin[s]) {
      // the exchange of the pairs below the diagonal tiles: the transpose of T's own contribution
      // (reduceFockReal adds into its output)
      TCSCF_CUDA(ctx, cudaMemsetAsync(GRhalf, 0, sizeof(double) * size_t(nb) * nb, ctx->stream));
      TCSCF_TRY(reduceFockReal(ctx, n1, nb, g1.phiR, g1.w, nullptr, 0.0, Tre + size_t(s) * n1 * ldt, ldt, 1.0, GRhalf));
      kAddTransposed<<<gridBlocks(int64_t(nb) * nb, 256), 256, 0, ctx->stream>>>(nb, GRhalf, GRre + size_t(s) * nb * nb);
      TCSCF_LAUNCH(ctx);
    }
    if (anyComplex)
      TCSCF_TRY(reduceFockReal(ctx, n1, nb, g1.phiR, g1.w, nullptr, 0.0, Tim + size_t(s) * n1 * ldt, ldt, 1.0, GRim + size_t(s) * nb * nb));
  }
  ctx->lastVH = VHtot;
  ctx->lastT = Tre;
  ctx->lastN1 = n1;
  ctx->lastNb = nb;
  kRealToReference<<<gridBlocks(int64_t(nspin) * nb * nb, 256), 256, 0, ctx->stream>>>(nspin, nb, g1.dsto, GRre, anyComplex ? GRim : nullptr, dG);
  TCSCF_LAUNCH(ctx);
  kFinalize<<<1, 512, 0, ctx->stream>>>(nspin, nb, dH, dG, nullptr, dD, respectSym, nspin == 1 ? 2.0 : 1.0, dFock, dE);
  TCSCF_LAUNCH(ctx);
  cudaEventRecord(ctx->ev[1], ctx->stream);
  TCSCF_CUDA(ctx, cudaEventSynchronize(ctx->ev[1]));
  float tot = 0;
  cudaEventElapsedTime(&tot, ctx->ev[0], ctx->ev[1]);
  ctx->lastTotalMs = tot;
  ctx->lastContractionMs = contractionMs;
  ctx->lastLaunches = ctx->launchCount - launch0;
  return TCSCF_OK;
}

// Batched RCS Fock builds (tcscf_fock_build_batch): every instance's density is factored and its
// tensor operands packed into its own arena; then all tensor contractions run in one persistent
// launch per tile class, and each instance's Fock matrix and energy are finished.  Instances whose
// density factor is complex in the real-harmonic basis, or whose shape the tensor path does not
// take, are built on their own with fockBuildDevice.
int fockBuildBatch(tcscf_ctx * ctx, int count, Grid * const * g1s, Grid * const * g2s, const double2 * const * dDs, const double * const * dHs,
                   int respectSym, int precision, double2 * const * dGs, double2 * const * dFs, double * const * dEs)
{
  cudaEventRecord(ctx->ev[0], ctx->stream);
  int const launch0 = ctx->launchCount;
  // shared temporaries (consumed in stream order by each instance's packing before the next reuses them)
  int64_t maxN1 = 0, maxN2 = 0;
  int maxNb = 0;
  for (int k = 0; k < count; ++k) {
    maxN1 = std::max(maxN1, g1s[k]->n);
    maxN2 = std::max(maxN2, g2s[k]->n);
    maxNb = std::max(maxNb, g1s[k]->nb);
  }
  size_t const tmpBytes = sizeof(double) * (size_t(maxN2) * maxNb + size_t(maxN1) * maxNb + 2 * size_t(maxN2) * maxNb + size_t(maxN2));
  void * tp = nullptr;
  TCSCF_TRY(scratch(ctx, "batch_tmp", tmpBytes, &tp));
  double * V = static_cast<double *>(tp);
  double * psi1 = V + size_t(maxN2) * maxNb;
  double * psi2 = psi1 + size_t(maxN1) * maxNb;
  double * psi1at2 = psi2 + size_t(maxN2) * maxNb;
  double * coul = psi1at2 + size_t(maxN2) * maxNb;

  // per-instance persistent buffers: T, VH, GR and the tensor arena
  std::vector<Contraction> cs(count);
  std::vector<char> tensorOk(count, 0);
  std::vector<size_t> offs(count + 1, 0);
  std::vector<size_t> arenaBytes(count, 0);
  for (int k = 0; k < count; ++k) {
    Grid & g1 = *g1s[k];
    Grid & g2 = *g2s[k];
    int const nb = g1.nb;
    Contraction & c = cs[k];
    c.n1 = g1.n; c.n2 = g2.n; c.R = std::min(nb, 32); c.ncol = nb; c.ldpsi = nb; c.ldt = nb;
    c.p1 = g1.pts; c.p2 = g2.pts;
    c.nSplit = splitForPolicy(c, precision, ctx->batchSplitPolicy);
    arenaBytes[k] = tensorArenaBytes(c, precision);
    size_t const own = (sizeof(double) * (size_t(g1.n) * nb + g1.n + size_t(nb) * nb) + 255) & ~size_t(255);
    offs[k + 1] = offs[k] + own + ((arenaBytes[k] + 255) & ~size_t(255));
  }
  void * bp = nullptr;
  TCSCF_TRY(scratch(ctx, "batch_arena", offs[count] + 256, &bp));
  // every instance's density factorisation is launched first, with one host synchronisation for all
  std::vector<size_t> fOffs(count + 1, 0);
  for (int k = 0; k < count; ++k) fOffs[k + 1] = fOffs[k] + ((factorBufBytes(g1s[k]->nb) + 255) & ~size_t(255));
  void * fp = nullptr;
  TCSCF_TRY(scratch(ctx, "batch_factors", fOffs[count] + 256, &fp));
  void * sp = nullptr;
  TCSCF_TRY(scratch(ctx, "batch_factor_status", sizeof(FactorStatus) * count + 256, &sp));
  auto * dStatus = static_cast<FactorStatus *>(sp);
  std::vector<FactorBufs> fbufs(count);
  for (int k = 0; k < count; ++k) {
    fbufs[k] = carveFactorBufs(static_cast<char *>(fp) + fOffs[k], g1s[k]->nb);
    TCSCF_TRY(factorLaunch(ctx, *g1s[k], dDs[k], fbufs[k]));
    TCSCF_CUDA(ctx, cudaMemcpyAsync(dStatus + k, fbufs[k].status, sizeof(FactorStatus), cudaMemcpyDeviceToDevice, ctx->stream));
  }
  std::vector<FactorStatus> hStatus(count);
  TCSCF_CUDA(ctx, cudaMemcpyAsync(hStatus.data(), dStatus, sizeof(FactorStatus) * count, cudaMemcpyDeviceToHost, ctx->stream));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  std::vector<TensorPrep> preps(count);
  std::vector<TensorPrep *> ready;
  for (int k = 0; k < count; ++k) {
    Grid & g1 = *g1s[k];
    Grid & g2 = *g2s[k];
    int const nb = g1.nb;
    int64_t const n1 = g1.n, n2 = g2.n;
    double const scale = g2.ndim == 2 ? 2 * kPi : 1.0;
    char * base = static_cast<char *>(bp) + offs[k];
    double * T = reinterpret_cast<double *>(base);
    double * VH = T + size_t(n1) * nb;   // followed by the instance's [nb][nb] reduction output
    void * arena = base + ((sizeof(double) * (size_t(n1) * nb + n1 + size_t(nb) * nb) + 255) & ~size_t(255));
    Factor f;
    TCSCF_TRY(factorFinish(ctx, g1, fbufs[k], hStatus[k], f));
    Contraction & c = cs[k];
    // one grid on both sides and X1 = X2: the symmetric split-BF16 contraction (psi2 = psi1)
    bool const sym = precision == TCSCF_PREC_BF16X3 && &g1 == &g2 && f.same;
    c.R = f.R;
    c.T = T; c.VH = VH; c.V = V; c.ldv = nb;
    c.psi1 = psi1; c.psi2 = sym ? psi1 : psi2; c.coul = coul;
    c.sym = sym ? 1 : 0;
    std::string why;
    bool eligible = (precision == TCSCF_PREC_BF16X3 || precision == TCSCF_PREC_TF32) && f.R > 0 && !f.complex &&
                    tensorPathAvailable(c, precision, &why) && tensorArenaBytes(c, precision) <= arenaBytes[k];
    if (eligible) {
      // an instance whose grids hold near-coincident pairs is built on its own (with the FP64 correction)
      NearList const * nl = nullptr;
      TCSCF_TRY(nearPairsFor(ctx, g1, g2, &nl));
      eligible = nl->count == 0;
    }
    if (!eligible) continue;
    kWeightedBasis<<<gridBlocks(n2 * nb, 256), 256, 0, ctx->stream>>>(n2, nb, g2.phiR, g2.w, scale, V);
    TCSCF_LAUNCH(ctx);
    const void * vtPacked = nullptr;
    if (precision == TCSCF_PREC_BF16X3) TCSCF_TRY(tensorPackedV(ctx, g2, V, scale, &vtPacked));
    c.vtPacked = vtPacked;
    size_t const sm = sizeof(double) * size_t(nb) * f.R;
    kOrbitals<<<gridBlocks(n1 * f.R, 256), 256, sm, ctx->stream>>>(n1, nb, f.R, g1.phiR, f.X1, f.ldx, psi1, nb);
    TCSCF_LAUNCH(ctx);
    if (!sym) {
      kOrbitals<<<gridBlocks(n2 * f.R, 256), 256, sm, ctx->stream>>>(n2, nb, f.R, g2.phiR, f.X2, f.ldx, psi2, nb);
      TCSCF_LAUNCH(ctx);
      kOrbitals<<<gridBlocks(n2 * f.R, 256), 256, sm, ctx->stream>>>(n2, nb, f.R, g2.phiR, f.X1, f.ldx, psi1at2, nb);
      TCSCF_LAUNCH(ctx);
    }
    kCoulombSource<<<gridBlocks(n2, 256), 256, 0, ctx->stream>>>(n2, f.R, sym ? psi1 : psi1at2, c.psi2, nb, g2.w, scale, coul);
    TCSCF_LAUNCH(ctx);
    TCSCF_TRY(tensorPrepare(ctx, c, precision, arena, arenaBytes[k], preps[k]));
    tensorOk[k] = 1;
    ready.push_back(&preps[k]);
  }
  if (!ready.empty()) TCSCF_TRY(tensorRun(ctx, ready.data(), int(ready.size())));
  float contractionMs = 0;
  if (!ready.empty()) {
    TCSCF_CUDA(ctx, cudaEventSynchronize(ctx->ev[3]));
    cudaEventElapsedTime(&contractionMs, ctx->ev[2], ctx->ev[3]);
  }
  double * GRhalf = nullptr;
  TCSCF_TRY(scratch(ctx, "batch_sym_half", sizeof(double) * size_t(maxNb) * maxNb, reinterpret_cast<void **>(&GRhalf)));
  for (int k = 0; k < count; ++k) {
    Grid & g1 = *g1s[k];
    int const nb = g1.nb;
    if (!tensorOk[k]) {
      TCSCF_TRY(fockBuildDevice(ctx, g1, *g2s[k], 1, dDs[k], dHs[k], respectSym, precision, dGs[k], dFs[k], dEs[k], nullptr));
      continue;
    }
    Contraction const & c = cs[k];
    double * GR = c.VH + g1.n;
    TCSCF_CUDA(ctx, cudaMemsetAsync(GR, 0, sizeof(double) * nb * nb, ctx->stream));
    TCSCF_TRY(reduceFockReal(ctx, g1.n, nb, g1.phiR, g1.w, c.VH, 2.0, c.T, nb, 1.0, GR));
    if (c.sym) {
      TCSCF_CUDA(ctx, cudaMemsetAsync(GRhalf, 0, sizeof(double) * nb * nb, ctx->stream));
      TCSCF_TRY(reduceFockReal(ctx, g1.n, nb, g1.phiR, g1.w, nullptr, 0.0, c.T, nb, 1.0, GRhalf));
      kAddTransposed<<<gridBlocks(int64_t(nb) * nb, 256), 256, 0, ctx->stream>>>(nb, GRhalf, GR);
      TCSCF_LAUNCH(ctx);
    }
    kRealToReference<<<gridBlocks(int64_t(nb) * nb, 256), 256, 0, ctx->stream>>>(1, nb, g1.dsto, GR, nullptr, dGs[k]);
    TCSCF_LAUNCH(ctx);
    kFinalize<<<1, 512, 0, ctx->stream>>>(1, nb, dHs[k], dGs[k], nullptr, dDs[k], respectSym, 2.0, dFs[k], dEs[k]);
    TCSCF_LAUNCH(ctx);
  }
  cudaEventRecord(ctx->ev[1], ctx->stream);
  TCSCF_CUDA(ctx, cudaEventSynchronize(ctx->ev[1]));
  float tot = 0;
  cudaEventElapsedTime(&tot, ctx->ev[0], ctx->ev[1]);
  ctx->lastTotalMs = tot;
  ctx->lastContractionMs = contractionMs;
  ctx->lastLaunches = ctx->launchCount - launch0;
  return TCSCF_OK;
}

int validateBasis(tcscf_ctx * ctx, const tcscf_sto * basis, int nb, std::vector<DevSto> & out)
{
  TCSCF_CHECK(ctx, basis && nb > 0, TCSCF_ERR_INVALID_ARGUMENT, "empty basis");
  out.resize(nb);
  for (int b = 0; b < nb; ++b) {
    tcscf_sto const & s = basis[b];
    TCSCF_CHECK(ctx, s.family == basis[0].family, TCSCF_ERR_INVALID_ARGUMENT, "a basis holds one family of functions");
    TCSCF_CHECK(ctx, s.l <= kMaxL, TCSCF_ERR_UNSUPPORTED, "angular momentum above 12");
    TCSCF_CHECK(ctx, s.l >= std::abs(s.m), TCSCF_ERR_INVALID_ARGUMENT, "|m| > l");
    if (s.family == TCSCF_BASIS_STO) {
      // SlaterTypeOrbital.hpp:34-36
      TCSCF_CHECK(ctx, s.n >= 1 && s.n >= s.l, TCSCF_ERR_INVALID_ARGUMENT, "invalid STO quantum numbers");
      TCSCF_CHECK(ctx, s.alpha > 0, TCSCF_ERR_INVALID_ARGUMENT, "non-positive STO exponent");
    } else if (s.family == TCSCF_BASIS_OCHI) {
      // OchiBasis.hpp:33-34
      TCSCF_CHECK(ctx, s.n >= 0, TCSCF_ERR_INVALID_ARGUMENT, "negative Ochi Laguerre degree");
      TCSCF_CHECK(ctx, s.alpha > 0, TCSCF_ERR_INVALID_ARGUMENT, "non-positive Ochi exponent");
    } else if (s.family == TCSCF_BASIS_HYDROGEN) {
      // HydrogenLikeBasis.hpp:31-34
      TCSCF_CHECK(ctx, s.alpha > 0 && s.n >= 1 && s.l < s.n, TCSCF_ERR_INVALID_ARGUMENT, "invalid hydrogen-like quantum numbers or Z");
    } else {
      return fail(ctx, TCSCF_ERR_INVALID_ARGUMENT, "unknown basis family");
    }
    DevSto d{};
    d.alpha = s.family == TCSCF_BASIS_HYDROGEN ? s.alpha / s.n : s.alpha;
    d.norm = basisNormalization(s);
    d.n = s.n; d.l = s.l; d.m = s.m;
    d.family = s.family;
    d.rtype = s.m == 0 ? 0 : (s.m > 0 ? 1 : 2);
    d.partner = -1;
    if (s.m != 0) {
      for (int c = 0; c < nb; ++c)
        if (basis[c].alpha == s.alpha && basis[c].n == s.n && basis[c].l == s.l && basis[c].m == -s.m && basis[c].family == s.family) {
          d.partner = c;
          break;
        }
      TCSCF_CHECK(ctx, d.partner >= 0, TCSCF_ERR_UNSUPPORTED, "basis lacks the -m partner of an m != 0 function");
    }
    out[b] = d;
  }
  return TCSCF_OK;
}

// precomputeIntegrand + computeF / computeV (HartreeFock.hpp:23-229): the weighted basis-pair products
// of the r2 grid (real-harmonic basis, k <= l) contracted with the r12 kernel (ncomp = 1: a scalar
// kernel; 3: the components of grad_1 u) in the requested precision, then mapped to the reference's
// complex Fji / Vji layout; written to host memory (out) and / or kept on the device as a handle.
int precomputeTensor(tcscf_ctx * ctx, int r1, int r2, int kernel, const tcscf_ochi * jastrow, int precision, int ncomp, double * out,
                     int keep, int * handle)
{
  Grid * g1 = findGrid(ctx, r1);
  Grid * g2 = findGrid(ctx, r2);
  TCSCF_TRY(checkBasisPair(ctx, g1, g2));
  TCSCF_CHECK(ctx, !jastrow || (jastrow->nterms >= 0 && jastrow->nterms <= 8), TCSCF_ERR_INVALID_ARGUMENT, "at most 8 Jastrow terms");
  TCSCF_CHECK(ctx, out || keep, TCSCF_ERR_INVALID_ARGUMENT, "nothing to do");
  TCSCF_CHECK(ctx, ncomp == 1 || g2->ndim == 3, TCSCF_ERR_INVALID_ARGUMENT, "computeV needs a 3-D r2 grid");
  TCSCF_CHECK(ctx, precision == TCSCF_PREC_FP64 || precision == TCSCF_PREC_BF16X3, TCSCF_ERR_UNSUPPORTED,
              "computeF / computeV run in FP64 or BF16X3");
  int const nb = g1->nb;
  int const np = nb * (nb + 1) / 2;
  int64_t const n1 = g1->n, n2 = g2->n;
  bool const realOut = ncomp == 1 && g2->ndim == 2;
  double const scale = realOut ? 2 * kPi : 1.0;
  Contraction c;
  c.n1 = n1; c.n2 = n2; c.R = 0; c.ncol = np; c.p1 = g1->pts; c.p2 = g2->pts; c.ldv = np; c.ldt = np;
  c.kernel = kernel; c.jastrow = jastrow;
  if (precision != TCSCF_PREC_FP64) {
    std::string why;
    TCSCF_CHECK(ctx, pairsTensorAvailable(c, precision, &why), TCSCF_ERR_UNSUPPORTED, why);
    TCSCF_TRY(nearPairsFor(ctx, *g1, *g2, &c.near));
  }
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, "computeF", sizeof(double) * (size_t(n2) * np + size_t(n1) * np), &p));
  double * pairs = static_cast<double *>(p);
  double * FR = pairs + size_t(n2) * np;
  size_t const outElems = size_t(n1) * nb * nb * (realOut ? 1 : 2) * ncomp;
  double * dOut = nullptr;
  TCSCF_CUDA(ctx, cudaMalloc(&dOut, sizeof(double) * outElems));
  cudaEventRecord(ctx->ev[0], ctx->stream);
  int const launch0 = ctx->launchCount;
  kPairProducts<<<gridBlocks(n2 * np, 256), 256, 0, ctx->stream>>>(n2, nb, g2->phiR, g2->w, scale, pairs);
  ctx->launchCount++;
  int st = TCSCF_OK;
  if (cudaError_t const e = cudaGetLastError(); e != cudaSuccess)   // dOut is released below
    st = fail(ctx, TCSCF_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  c.V = pairs;
  c.T = FR;
  float contraction = 0;
  for (int comp = 0; comp < ncomp && st == TCSCF_OK; ++comp) {
    c.component = comp;
    // the contraction alone is bracketed by ev[2] / ev[3]; tcscf_last_timing reports the components' sum
    cudaEventRecord(ctx->ev[2], ctx->stream);
    st = precision == TCSCF_PREC_FP64 ? contractFp64(ctx, c) : contractPairsTensor(ctx, c, precision);
    cudaEventRecord(ctx->ev[3], ctx->stream);
    if (st == TCSCF_OK) {
      kPairsToReference<<<gridBlocks(n1 * nb * nb, 256), 256, 0, ctx->stream>>>(n1, nb, g1->dsto, FR, ncomp, comp, realOut ? 1 : 0, dOut);
      ctx->launchCount++;
      cudaError_t const e = cudaGetLastError();
      if (e != cudaSuccess) st = fail(ctx, TCSCF_ERR_CUDA, cudaGetErrorString(e));
    }
    cudaStreamSynchronize(ctx->stream);
    float a = 0;
    cudaEventElapsedTime(&a, ctx->ev[2], ctx->ev[3]);
    contraction += a;
  }
  if (st == TCSCF_OK && out) {
    cudaError_t const e = cudaMemcpyAsync(out, dOut, sizeof(double) * outElems, cudaMemcpyDeviceToHost, ctx->stream);
    if (e != cudaSuccess) st = fail(ctx, TCSCF_ERR_CUDA, cudaGetErrorString(e));
  }
  cudaEventRecord(ctx->ev[1], ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  float b = 0;
  cudaEventElapsedTime(&b, ctx->ev[0], ctx->ev[1]);
  ctx->lastContractionMs = contraction;
  ctx->lastTotalMs = b;
  ctx->lastLaunches = ctx->launchCount - launch0;
  if (st != TCSCF_OK || !keep) { cudaFree(dOut); return st; }
  Tensor t;
  t.d = dOut; t.n1 = n1; t.nb = nb; t.isComplex = realOut ? 0 : 1; t.vec = ncomp == 3 ? 1 : 0;
  int const id = ctx->nextId++;
  ctx->tensors[id] = t;
  if (handle) *handle = id;
  return TCSCF_OK;
}

// ---- SCF as one CUDA graph (tcscf_scf_graph) ------------------------------------------------------
// C = op(A) B for small dense row-major matrices (op(A) = A [M][K] or A^T with A [K][M]); one thread
// per output element
__global__ void kSmallGemm(int M, int N, int K, const double * A, int lda, int transA, const double * B, int ldb, double * C, int ldc)
{
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < M * N; idx += gridDim.x * blockDim.x) {
    int const i = idx / N, j = idx % N;
    double s = 0;
    for (int k = 0; k < K; ++k) s = fma(transA ? A[k * lda + i] : A[i * lda + k], B[k * ldb + j], s);
    C[i * ldc + j] = s;
  }
}

// Two-sided cyclic Jacobi eigen-solver of the symmetric m x m matrix A (row-major) in one CTA
// (Golub & Van Loan, Matrix Computations, sym.schur2 rotations in the round-robin parallel ordering:
// m (rounded up to even, the padding index carries a zero row) indices are paired into m/2 disjoint
// rotations per step, m - 1 steps per sweep).  A lives in shared memory, the eigenvectors V (columns,
// row-major [m][m]) in global memory.  A rotation is skipped when |a_pq| <= eps sqrt|a_pp a_qq|; the
// sweeps stop when one performs no rotation (at most 40).  Out: W[m] the eigenvalues (A's diagonal,
// unsorted) and V.
constexpr int kJacobiThreads = 512;
__global__ void __launch_bounds__(kJacobiThreads) kJacobiSym(int m, const double * Ain, double * W, double * V)
{
  extern __shared__ double sJ[];
  __shared__ double cs[64], sn[64];
  __shared__ int pp[64], qq[64];
  __shared__ int rotated;
  int const mp = m + (m & 1);
  int const half = mp / 2;
  int const tid = threadIdx.x;
  for (int idx = tid; idx < mp * mp; idx += blockDim.x) {
    int const i = idx / mp, j = idx % mp;
    sJ[idx] = (i < m && j < m) ? 0.5 * (Ain[i * m + j] + Ain[j * m + i]) : 0.0;
  }
  for (int idx = tid; idx < m * m; idx += blockDim.x) V[idx] = (idx / m == idx % m) ? 1.0 : 0.0;
  __syncthreads();
  for (int sweep = 0; sweep < 40; ++sweep) {
    if (tid == 0) rotated = 0;
    __syncthreads();
    for (int step = 0; step < mp - 1; ++step) {
      if (tid < half) {
        // round-robin pairing: index mp - 1 stays, the others rotate by one each step
        int p = tid == 0 ? mp - 1 : (step + tid) % (mp - 1);
        int q = (step + mp - 1 - tid) % (mp - 1);
        if (tid == 0) q = step % (mp - 1);
        if (p > q) { int const t = p; p = q; q = t; }
        double const apq = sJ[p * mp + q], app = sJ[p * mp + p], aqq = sJ[q * mp + q];
        double c = 1.0, s = 0.0;
        if (apq != 0.0 && fabs(apq) > 2.2204460492503131e-16 * sqrt(fabs(app * aqq))) {
          double const tau = (aqq - app) / (2.0 * apq);
          double const t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
          c = 1.0 / sqrt(1.0 + t * t);
          s = t * c;
          rotated = 1;
        }
        pp[tid] = p; qq[tid] = q; cs[tid] = c; sn[tid] = s;
      }
      __syncthreads();
      // rows: A <- J^T A
      for (int idx = tid; idx < half * mp; idx += blockDim.x) {
        int const k = idx / mp, j = idx % mp;
        if (sn[k] == 0.0) continue;
        int const p = pp[k], q = qq[k];
        double const c = cs[k], s = sn[k];
        double const ap = sJ[p * mp + j], aq = sJ[q * mp + j];
        sJ[p * mp + j] = c * ap - s * aq;
        sJ[q * mp + j] = s * ap + c * aq;
      }
      __syncthreads();
      // columns: A <- A J, V <- V J
      for (int idx = tid; idx < half * mp; idx += blockDim.x) {
        int const k = idx / mp, i = idx % mp;
        if (sn[k] == 0.0) continue;
        int const p = pp[k], q = qq[k];
        double const c = cs[k], s = sn[k];
        double const ap = sJ[i * mp + p], aq = sJ[i * mp + q];
        sJ[i * mp + p] = c * ap - s * aq;
        sJ[i * mp + q] = s * ap + c * aq;
        if (i < m && q < m) {
          double const vp = V[i * m + p], vq = V[i * m + q];
          V[i * m + p] = c * vp - s * vq;
          V[i * m + q] = s * vp + c * vq;
        }
      }
      __syncthreads();
    }
    if (!rotated) break;
    __syncthreads();
  }
  for (int i = tid; i < m; i += blockDim.x) W[i] = sJ[i * mp + i];
}

// Eigenvalues in ascending order (ties by index): Ws[m], and the indices of the nocc lowest; then
// the occupied coefficients C[k][a] = sum_j Xc[k][j] V[j][idx[a]] ([nb][nocc], real-harmonic basis)
// and the density DR = C C^T.  One block.
__global__ void kOccupiedOrbitals(int nb, int m, int nocc, const double * W, const double * V, const double * Xc, double * Ws, double * C,
                                  double * DR)
{
  __shared__ int idx[128];
  for (int t = threadIdx.x; t < m; t += blockDim.x) {
    double const wt = W[t];
    int r = 0;
    for (int j = 0; j < m; ++j) r += (W[j] < wt || (W[j] == wt && j < t)) ? 1 : 0;
    Ws[r] = wt;
    if (r < nocc) idx[r] = t;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nb * nocc; e += blockDim.x) {
    int const k = e / nocc, a = e % nocc;
    double s = 0;
    for (int j = 0; j < m; ++j) s = fma(Xc[k * m + j], V[j * m + idx[a]], s);
    C[e] = s;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    int const u = e / nb, v = e % nb;
    double s = 0;
    for (int a = 0; a < nocc; ++a) s = fma(C[u * nocc + a], C[v * nocc + a], s);
    DR[e] = s;
  }
}

// The convergence test of the SCF loop (RCSHartreeFock::compute, HartreeFock.cpp:857): the energy of
// this iteration's build against the previous one; on convergence, a non-finite energy, an expired
// bounded wait of the tensor kernel or the iteration limit, the loop ends (the graph's WHILE
// condition is cleared) with the density and eigenvalues this build used saved.
struct ScfGraphState {
  double eprev, eres;
  int iter, done, code, pad;
};
__global__ void kScfCheck(ScfGraphState * st, const double * E, const int * tstatus, int maxIter, double tol, int nD, const double2 * D,
                          double2 * Dres, int nW, const double * Wcur, double * Wres, cudaGraphConditionalHandle handle, int useHandle)
{
  __shared__ int stop;
  if (threadIdx.x == 0) {
    double const e = *E;
    int const it = st->iter + 1;
    st->iter = it;
    int code = TCSCF_OK;
    bool s = true;
    if (tstatus && *tstatus != 0) code = TCSCF_ERR_TIMEOUT;
    else if (!isfinite(e)) code = TCSCF_ERR_NONFINITE;
    else if (fabs(e - st->eprev) < tol) code = TCSCF_OK;
    else if (it >= maxIter) code = TCSCF_ERR_NOT_CONVERGED;
    else s = false;
    st->eprev = e;
    if (s) { st->done = 1; st->code = code; st->eres = e; }
    stop = s ? 1 : 0;
  }
  __syncthreads();
  if (stop) {
    for (int i = threadIdx.x; i < nD; i += blockDim.x) Dres[i] = D[i];
    for (int i = threadIdx.x; i < nW; i += blockDim.x) Wres[i] = Wcur[i];
  }
  if (useHandle && threadIdx.x == 0) cudaGraphSetConditional(handle, stop ? 0u : 1u);
}

// One RCS SCF on the device (tcscf_scf_graph).  Every iteration is the same launch sequence on fixed
// buffers: orbitals of the current occupied coefficients C on both grids, the Coulomb source, the r12
// contraction (FP64 or tensor cores) from those factors (D = C C^T, rank nocc), the real Fock
// reduction, the reference-basis G, F and energy (kFinalize), the convergence test, then the new C from
// the Fock matrix: real-harmonic F, Xc^T F Xc with the canonical orthogonaliser Xc of S, Jacobi, the
// nocc lowest eigenvectors.  The first two iterations run directly (the zero-density one, F = h, with
// no contraction; the second allocates every buffer); with capture the rest run as one graph launch
// whose conditional WHILE node repeats the body until the device-side test clears it, so the host
// neither reads nor waits per iteration.
int scfGraph(tcscf_ctx * ctx, Grid & g1, Grid & g2, int nocc, const double * S, const double * h, int respectSym, int precision, double tol,
             int maxIter, int capture, double * energy, int * iterations, double * density, double * eigenvalues, int * graphLaunches)
{
  int const nb = g1.nb;
  int64_t const n1 = g1.n, n2 = g2.n;
  size_t const nn = size_t(nb) * nb;
  double const scale = g2.ndim == 2 ? 2 * kPi : 1.0;
  TCSCF_CHECK(ctx, nb <= 128, TCSCF_ERR_UNSUPPORTED, "the graph SCF's device eigen-solver takes nb <= 128");
  TCSCF_CHECK(ctx, nocc >= 1 && nocc <= nb, TCSCF_ERR_INVALID_ARGUMENT, "occupied orbitals out of range");
  // ---- small buffers
  void * p = nullptr;
  size_t const smallBytes = sizeof(double2) * nn * 7 + sizeof(double) * (nn * 8 + size_t(nb) * nocc + 4 * nb + 64) + sizeof(ScfGraphState) + 4096;
  TCSCF_TRY(scratch(ctx, "scf_graph_small", smallBytes, &p));
  char * q = static_cast<char *>(p);
  auto take = [&](size_t n) { char * r = q; q += (n + 255) & ~size_t(255); return r; };
  auto * dD = reinterpret_cast<double2 *>(take(sizeof(double2) * nn));
  auto * dG = reinterpret_cast<double2 *>(take(sizeof(double2) * nn));
  auto * dF = reinterpret_cast<double2 *>(take(sizeof(double2) * nn));
  auto * FRc = reinterpret_cast<double2 *>(take(sizeof(double2) * nn));
  auto * Sc = reinterpret_cast<double2 *>(take(sizeof(double2) * nn));
  auto * SRc = reinterpret_cast<double2 *>(take(sizeof(double2) * nn));
  auto * Dres = reinterpret_cast<double2 *>(take(sizeof(double2) * nn));
  double * dH = reinterpret_cast<double *>(take(sizeof(double) * nn));
  double * FR = reinterpret_cast<double *>(take(sizeof(double) * nn));
  double * SR = reinterpret_cast<double *>(take(sizeof(double) * nn));
  double * Xc = reinterpret_cast<double *>(take(sizeof(double) * nn));
  double * Tm = reinterpret_cast<double *>(take(sizeof(double) * nn));
  double * Fp = reinterpret_cast<double *>(take(sizeof(double) * nn));
  double * Vm = reinterpret_cast<double *>(take(sizeof(double) * nn));
  double * DR = reinterpret_cast<double *>(take(sizeof(double) * nn));
  double * C = reinterpret_cast<double *>(take(sizeof(double) * nb * nocc));
  double * W = reinterpret_cast<double *>(take(sizeof(double) * nb));
  double * Ws = reinterpret_cast<double *>(take(sizeof(double) * nb));
  double * Wres = reinterpret_cast<double *>(take(sizeof(double) * nb));
  double * fmaxv = reinterpret_cast<double *>(take(sizeof(double) * 4));
  double * dE = reinterpret_cast<double *>(take(sizeof(double) * 4));
  auto * st = reinterpret_cast<ScfGraphState *>(take(sizeof(ScfGraphState)));
  // ---- grid-sized buffers of the build
  int const ldpsi = nocc;
  size_t const bigBytes = sizeof(double) * (size_t(n2) * nb + size_t(n1) * ldpsi + size_t(n2) * ldpsi + n2 + size_t(n1) * nb + n1) + 8 * 256;
  TCSCF_TRY(scratch(ctx, "scf_graph_build", bigBytes, &p));
  q = static_cast<char *>(p);
  double * Vw = reinterpret_cast<double *>(take(sizeof(double) * n2 * nb));
  double * psi1 = reinterpret_cast<double *>(take(sizeof(double) * n1 * ldpsi));
  double * psi2 = reinterpret_cast<double *>(take(sizeof(double) * n2 * ldpsi));
  double * coul = reinterpret_cast<double *>(take(sizeof(double) * n2));
  double * Tb = reinterpret_cast<double *>(take(sizeof(double) * n1 * nb));
  double * VH = reinterpret_cast<double *>(take(sizeof(double) * n1));

  // ---- canonical orthogonaliser Xc = U s^-1/2 of the real-harmonic overlap (eigenvalues above 1e-12
  // of the largest kept)
  TCSCF_CUDA(ctx, cudaMemcpyAsync(SR, S, sizeof(double) * nn, cudaMemcpyHostToDevice, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemcpyAsync(dH, h, sizeof(double) * nn, cudaMemcpyHostToDevice, ctx->stream));
  kRealToComplex<<<gridBlocks(int64_t(nn), 256), 256, 0, ctx->stream>>>(int64_t(nn), SR, Sc);
  TCSCF_LAUNCH(ctx);
  kDensityToReal<<<gridBlocks(nn, 256), 256, 0, ctx->stream>>>(1, nb, g1.dsto, Sc, SRc);
  TCSCF_LAUNCH(ctx);
  kSplitDensity<<<1, 256, 0, ctx->stream>>>(nb, SRc, SR, fmaxv);
  TCSCF_LAUNCH(ctx);
  int m = 0;
  {
    int lwork = 0;
    if (cusolverDnDsyevd_bufferSize(ctx->solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, nb, SR, nb, W, &lwork) != CUSOLVER_STATUS_SUCCESS)
      return fail(ctx, TCSCF_ERR_LINALG, "cusolverDnDsyevd_bufferSize failed");
    void * wk = nullptr;
    TCSCF_TRY(scratch(ctx, "scf_graph_syevd", sizeof(double) * size_t(lwork) + 64 + sizeof(int) * 4, &wk));
    int * info = reinterpret_cast<int *>(static_cast<double *>(wk) + lwork);
    if (cusolverDnDsyevd(ctx->solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, nb, SR, nb, W, static_cast<double *>(wk), lwork, info) !=
        CUSOLVER_STATUS_SUCCESS)
      return fail(ctx, TCSCF_ERR_LINALG, "cusolverDnDsyevd failed");
    std::vector<double> hs(nb), hv(nn);
    int hinfo = 0;
    TCSCF_CUDA(ctx, cudaMemcpyAsync(hs.data(), W, sizeof(double) * nb, cudaMemcpyDeviceToHost, ctx->stream));
    TCSCF_CUDA(ctx, cudaMemcpyAsync(hv.data(), SR, sizeof(double) * nn, cudaMemcpyDeviceToHost, ctx->stream));
    TCSCF_CUDA(ctx, cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    TCSCF_CHECK(ctx, hinfo == 0 && hs[nb - 1] > 0 && std::isfinite(hs[nb - 1]), TCSCF_ERR_LINALG, "overlap matrix is not positive definite");
    std::vector<int> keep;
    for (int j = 0; j < nb; ++j)
      if (hs[j] > 1e-12 * hs[nb - 1]) keep.push_back(j);
    m = int(keep.size());
    TCSCF_CHECK(ctx, m >= nocc, TCSCF_ERR_LINALG, "overlap matrix has fewer independent functions than occupied orbitals");
    std::vector<double> hx(size_t(nb) * m);
    for (int k = 0; k < nb; ++k)   // cuSOLVER's eigenvectors are the columns of a column-major array
      for (int c = 0; c < m; ++c) hx[size_t(k) * m + c] = hv[size_t(keep[c]) * nb + k] / std::sqrt(hs[keep[c]]);
    TCSCF_CUDA(ctx, cudaMemcpyAsync(Xc, hx.data(), sizeof(double) * hx.size(), cudaMemcpyHostToDevice, ctx->stream));
    TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  // ---- static operands and the zero start (D = 0: the first build gives F = h, E = 0)
  TCSCF_CUDA(ctx, cudaMemsetAsync(C, 0, sizeof(double) * nb * nocc, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemsetAsync(dD, 0, sizeof(double2) * nn, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemsetAsync(W, 0, sizeof(double) * nb, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemsetAsync(Ws, 0, sizeof(double) * nb, ctx->stream));
  ScfGraphState st0{std::numeric_limits<double>::max(), 0.0, 0, 0, TCSCF_OK, 0};
  TCSCF_CUDA(ctx, cudaMemcpyAsync(st, &st0, sizeof(st0), cudaMemcpyHostToDevice, ctx->stream));
  kWeightedBasis<<<gridBlocks(n2 * nb, 256), 256, 0, ctx->stream>>>(n2, nb, g2.phiR, g2.w, scale, Vw);
  TCSCF_LAUNCH(ctx);
  bool const tensor = precision != TCSCF_PREC_FP64;
  // one grid on both sides: psi1 = psi2 (both C on the same points), the symmetric split-BF16 or FP64
  // contraction (pairs on and above each r1 tile's diagonal; the exchange plus its transpose)
  bool const sym = precision != TCSCF_PREC_TF32 && &g1 == &g2;
  Contraction c;
  c.n1 = n1; c.n2 = n2; c.R = nocc; c.ncol = nb;
  c.p1 = g1.pts; c.p2 = g2.pts; c.psi1 = psi1; c.psi2 = sym ? psi1 : psi2; c.ldpsi = ldpsi;
  c.V = Vw; c.ldv = nb; c.T = Tb; c.ldt = nb; c.coul = coul; c.VH = VH;
  c.sym = sym ? 1 : 0;
  double * FRhalf = nullptr;
  if (sym) TCSCF_TRY(scratch(ctx, "scf_graph_sym_half", sizeof(double) * nn, reinterpret_cast<void **>(&FRhalf)));
  TensorPrep tp;
  TensorPlan plan;
  void * arena = nullptr;
  size_t arenaBytes = 0;
  if (tensor) {
    TCSCF_TRY(tensorPackedV(ctx, g2, Vw, scale, &c.vtPacked));
    TCSCF_TRY(nearPairsFor(ctx, g1, g2, &c.near));
    std::string why;
    TCSCF_CHECK(ctx, tensorPathAvailable(c, precision, &why), TCSCF_ERR_UNSUPPORTED, "graph SCF tensor path: " + why);
    arenaBytes = tensorArenaBytes(c, precision);
    TCSCF_TRY(scratch(ctx, "scf_graph_tensor", arenaBytes, &arena));
    TCSCF_TRY(tensorPrepare(ctx, c, precision, arena, arenaBytes, tp));
    TCSCF_TRY(tensorPlanUpload(ctx, tp, "scf_graph_plan", plan));
  }
  size_t const jacobiSmem = sizeof(double) * size_t(m + (m & 1)) * (m + (m & 1));
  TCSCF_CUDA(ctx, cudaFuncSetAttribute(kJacobiSym, cudaFuncAttributeMaxDynamicSharedMemorySize, int(jacobiSmem)));

  // zeroDensity: the first iteration's density is zero, so its exchange and Coulomb potentials are
  // zero without a contraction (as tcscf_scf skips a rank-0 factor)
  auto body = [&](cudaGraphConditionalHandle handle, int useHandle, bool zeroDensity) -> int {
    size_t const sm = sizeof(double) * size_t(nb) * nocc;
    if (zeroDensity) {
      TCSCF_CUDA(ctx, cudaMemsetAsync(Tb, 0, sizeof(double) * size_t(n1) * nb, ctx->stream));
      TCSCF_CUDA(ctx, cudaMemsetAsync(VH, 0, sizeof(double) * size_t(n1), ctx->stream));
    } else {
    kOrbitals<<<gridBlocks(n1 * nocc, 256), 256, sm, ctx->stream>>>(n1, nb, nocc, g1.phiR, C, nocc, psi1, ldpsi);
    TCSCF_LAUNCH(ctx);
    if (!sym) {
      kOrbitals<<<gridBlocks(n2 * nocc, 256), 256, sm, ctx->stream>>>(n2, nb, nocc, g2.phiR, C, nocc, psi2, ldpsi);
      TCSCF_LAUNCH(ctx);
    }
    kCoulombSource<<<gridBlocks(n2, 256), 256, 0, ctx->stream>>>(n2, nocc, c.psi2, c.psi2, ldpsi, g2.w, scale, coul);
    TCSCF_LAUNCH(ctx);
    if (tensor) {
      TCSCF_TRY(tensorPrepare(ctx, c, precision, arena, arenaBytes, tp));
      TCSCF_TRY(tensorPlanLaunch(ctx, plan));
      TCSCF_TRY(nearCorrect(ctx, c));
    } else {
      TCSCF_TRY(contractFp64(ctx, c));
    }
    }
    TCSCF_CUDA(ctx, cudaMemsetAsync(FR, 0, sizeof(double) * nn, ctx->stream));
    TCSCF_TRY(reduceFockReal(ctx, n1, nb, g1.phiR, g1.w, VH, 2.0, Tb, nb, 1.0, FR));
    if (sym && !zeroDensity) {
      TCSCF_CUDA(ctx, cudaMemsetAsync(FRhalf, 0, sizeof(double) * nn, ctx->stream));
      TCSCF_TRY(reduceFockReal(ctx, n1, nb, g1.phiR, g1.w, nullptr, 0.0, Tb, nb, 1.0, FRhalf));
      kAddTransposed<<<gridBlocks(int64_t(nn), 256), 256, 0, ctx->stream>>>(nb, FRhalf, FR);
      TCSCF_LAUNCH(ctx);
    }
    kRealToReference<<<gridBlocks(int64_t(nn), 256), 256, 0, ctx->stream>>>(1, nb, g1.dsto, FR, nullptr, dG);
    TCSCF_LAUNCH(ctx);
    kFinalize<<<1, 512, 0, ctx->stream>>>(1, nb, dH, dG, nullptr, dD, respectSym, 2.0, dF, dE);
    TCSCF_LAUNCH(ctx);
    kScfCheck<<<1, 256, 0, ctx->stream>>>(st, dE, tensor ? plan.status : nullptr, maxIter, tol, int(nn), dD, Dres, nb, Ws, Wres, handle,
                                          useHandle);
    TCSCF_LAUNCH(ctx);
    // the next density from this Fock matrix (real in the real-harmonic basis)
    kDensityToReal<<<gridBlocks(nn, 256), 256, 0, ctx->stream>>>(1, nb, g1.dsto, dF, FRc);
    TCSCF_LAUNCH(ctx);
    kSplitDensity<<<1, 256, 0, ctx->stream>>>(nb, FRc, FR, fmaxv);
    TCSCF_LAUNCH(ctx);
    kSmallGemm<<<gridBlocks(int64_t(nb) * m, 256), 256, 0, ctx->stream>>>(nb, m, nb, FR, nb, 0, Xc, m, Tm, m);
    TCSCF_LAUNCH(ctx);
    kSmallGemm<<<gridBlocks(int64_t(m) * m, 256), 256, 0, ctx->stream>>>(m, m, nb, Xc, m, 1, Tm, m, Fp, m);
    TCSCF_LAUNCH(ctx);
    kJacobiSym<<<1, kJacobiThreads, jacobiSmem, ctx->stream>>>(m, Fp, W, Vm);
    TCSCF_LAUNCH(ctx);
    kOccupiedOrbitals<<<1, 256, 0, ctx->stream>>>(nb, m, nocc, W, Vm, Xc, Ws, C, DR);
    TCSCF_LAUNCH(ctx);
    kRealToReference<<<gridBlocks(int64_t(nn), 256), 256, 0, ctx->stream>>>(1, nb, g1.dsto, DR, nullptr, dD);
    TCSCF_LAUNCH(ctx);
    return TCSCF_OK;
  };

  ScfGraphState hst{};
  // the first two iterations directly: the zero-density one, then one that allocates every scratch
  // buffer the body uses
  for (int it = 0; it < 2 && it < maxIter && !hst.done; ++it) {
    TCSCF_TRY(body(0, 0, it == 0));
    TCSCF_CUDA(ctx, cudaMemcpyAsync(&hst, st, sizeof(hst), cudaMemcpyDeviceToHost, ctx->stream));
    TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  *graphLaunches = 0;
  if (!hst.done) {
    if (capture) {
      cudaGraph_t graph = nullptr;
      TCSCF_CUDA(ctx, cudaGraphCreate(&graph, 0));
      cudaGraphConditionalHandle handle;
      cudaGraphNode_t node;
      cudaGraphNodeParams cp = {};
      cudaError_t e = cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault);
      if (e == cudaSuccess) {
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        e = cudaGraphAddNode(&node, graph, nullptr, 0, &cp);
      }
      if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return fail(ctx, TCSCF_ERR_CUDA, std::string("conditional graph node: ") + cudaGetErrorString(e));
      }
      cudaGraph_t bodyGraph = cp.conditional.phGraph_out[0];
      e = cudaStreamBeginCaptureToGraph(ctx->stream, bodyGraph, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
      if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return fail(ctx, TCSCF_ERR_CUDA, std::string("begin capture: ") + cudaGetErrorString(e));
      }
      ctx->capturing = 1;
      int const bst = body(handle, 1, false);
      ctx->capturing = 0;
      cudaGraph_t captured = nullptr;
      e = cudaStreamEndCapture(ctx->stream, &captured);
      if (bst != TCSCF_OK || e != cudaSuccess) {
        cudaGraphDestroy(graph);
        if (bst != TCSCF_OK) return bst;
        return fail(ctx, TCSCF_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(e));
      }
      cudaGraphExec_t exec = nullptr;
      e = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      TCSCF_CHECK(ctx, e == cudaSuccess, TCSCF_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
      e = cudaGraphLaunch(exec, ctx->stream);
      cudaError_t const e2 = cudaStreamSynchronize(ctx->stream);
      cudaGraphExecDestroy(exec);
      TCSCF_CHECK(ctx, e == cudaSuccess && e2 == cudaSuccess, TCSCF_ERR_CUDA,
                  std::string("graph launch: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
      *graphLaunches = 1;
    } else {
      // the same body launched per iteration, with the host reading the loop state after each
      for (int it = 2; it < maxIter && !hst.done; ++it) {
        TCSCF_TRY(body(0, 0, false));
        TCSCF_CUDA(ctx, cudaMemcpyAsync(&hst, st, sizeof(hst), cudaMemcpyDeviceToHost, ctx->stream));
        TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      }
    }
    TCSCF_CUDA(ctx, cudaMemcpyAsync(&hst, st, sizeof(hst), cudaMemcpyDeviceToHost, ctx->stream));
    TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  if (iterations) *iterations = hst.iter;
  if (energy) *energy = hst.eres;
  if (density) TCSCF_CUDA(ctx, cudaMemcpy(density, Dres, sizeof(double2) * nn, cudaMemcpyDeviceToHost));
  if (eigenvalues) {
    std::vector<double> hw(nb, std::numeric_limits<double>::quiet_NaN());
    TCSCF_CUDA(ctx, cudaMemcpy(hw.data(), Wres, sizeof(double) * m, cudaMemcpyDeviceToHost));
    std::copy(hw.begin(), hw.end(), eigenvalues);
  }
  if (hst.code == TCSCF_ERR_TIMEOUT) return fail(ctx, TCSCF_ERR_TIMEOUT, "graph SCF: a bounded wait of the tensor kernel expired");
  if (hst.code == TCSCF_ERR_NONFINITE) return fail(ctx, TCSCF_ERR_NONFINITE, "non-finite energy");
  if (hst.code == TCSCF_ERR_NOT_CONVERGED || !hst.done)
    return fail(ctx, TCSCF_ERR_NOT_CONVERGED, "SCF did not converge in " + std::to_string(maxIter) + " iterations");
  return TCSCF_OK;
}

}  // namespace
}  // namespace tcscf

using namespace tcscf;

extern "C" {

int tcscf_ctx_create(int device, tcscf_ctx ** out)
{
  if (!out) return TCSCF_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return TCSCF_ERR_NO_DEVICE;
  if (device < 0 || device >= count) return TCSCF_ERR_INVALID_ARGUMENT;
  if (cudaSetDevice(device) != cudaSuccess) return TCSCF_ERR_CUDA;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return TCSCF_ERR_CUDA;
  if (prop.major != 10) return TCSCF_ERR_UNSUPPORTED;  // built for sm_100a only
  tcscf_ctx * ctx = new tcscf_ctx();
  ctx->device = device;
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) { delete ctx; return TCSCF_ERR_CUDA; }
  {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (cudaMemPoolCreate(&ctx->gridPool, &props) != cudaSuccess) {
      cudaStreamDestroy(ctx->stream);
      delete ctx;
      return TCSCF_ERR_CUDA;
    }
    // memory of destroyed grids stays in the pool up to this much (a few Kr-sized grids); the rest
    // goes back to the device at the next synchronisation
    uint64_t keep = uint64_t(4) << 30;
    cudaMemPoolSetAttribute(ctx->gridPool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  for (auto & e : ctx->ev) cudaEventCreate(&e);
  if (cusolverDnCreate(&ctx->solver) != CUSOLVER_STATUS_SUCCESS) {
    ctx->solver = nullptr;
    tcscf_ctx_destroy(ctx);   // releases the stream, the grid pool and the events made so far
    return TCSCF_ERR_CUDA;
  }
  cusolverDnSetStream(ctx->solver, ctx->stream);
  // the fixed array of tcscf_overlap_core_quadrature_static: its address is looked up here, where
  // allocation is allowed anyway (a lazily loaded module may allocate its globals on first use), so
  // the entry point itself never does set-up work
  double2 * fixedScratch = nullptr;
  if (quadStaticScratch(ctx, &fixedScratch) != TCSCF_OK) {
    tcscf_ctx_destroy(ctx);
    return TCSCF_ERR_CUDA;
  }
  *out = ctx;
  return TCSCF_OK;
}

int tcscf_ctx_destroy(tcscf_ctx * ctx)
{
  if (!ctx) return TCSCF_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto & kv : ctx->grids) gridReleaseAll(ctx, kv.second);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->gridPool) cudaMemPoolDestroy(ctx->gridPool);
  for (auto & kv : ctx->tensors) cudaFree(kv.second.d);
  for (auto & kv : ctx->scratch) cudaFree(kv.second.p);
  for (auto & kv : ctx->nearPairs)
    if (kv.second.d) cudaFree(kv.second.d);
  for (auto & e : ctx->ev) cudaEventDestroy(e);
  for (auto & e : ctx->tuneEv)
    if (e) cudaEventDestroy(e);
  if (ctx->tensorGraph) cudaGraphExecDestroy(ctx->tensorGraph);
  if (ctx->solver) cusolverDnDestroy(ctx->solver);
  if (ctx->blas) cublasDestroy(ctx->blas);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return TCSCF_OK;
}

const char * tcscf_last_error(tcscf_ctx * ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int tcscf_batch_graph_stats(tcscf_ctx * ctx, int * captures, int * replays)
{
  if (!ctx || !captures || !replays) return TCSCF_ERR_INVALID_ARGUMENT;
  *captures = ctx->graphCaptures;
  *replays = ctx->graphReplays;
  return TCSCF_OK;
}

int tcscf_set_autotune(tcscf_ctx * ctx, int enable)
{
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  ctx->autotune = enable ? 1 : 0;
  return TCSCF_OK;
}

int tcscf_autotune_stats(tcscf_ctx * ctx, int * shapes, int * batches, int * measurements)
{
  if (!ctx || !shapes || !batches || !measurements) return TCSCF_ERR_INVALID_ARGUMENT;
  *shapes = int(ctx->tunedSplit.size());
  *batches = int(ctx->tunedBatchPolicy.size());
  *measurements = ctx->tuneMeasurements;
  return TCSCF_OK;
}

int tcscf_autotune_split_candidates(int64_t n1, int64_t n2, int sms, int * splits, int capacity, int * count)
{
  if (n1 <= 0 || n2 <= 0 || sms <= 0 || !count || capacity < 0 || (capacity > 0 && !splits)) return TCSCF_ERR_INVALID_ARGUMENT;
  if (n1 > (int64_t(1) << 36) || n2 > (int64_t(1) << 36)) return TCSCF_ERR_INVALID_ARGUMENT;  // tile and block counts stay int
  std::vector<int> const c = splitCandidates(n1, n2, sms);
  int const n = std::min<int>(capacity, int(c.size()));
  for (int i = 0; i < n; ++i) splits[i] = c[i];
  *count = n;
  return TCSCF_OK;
}

int tcscf_selftest_bounded_wait(tcscf_ctx * ctx, double limit_ms)
{
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  TCSCF_CUDA(ctx, cudaSetDevice(ctx->device));
  return boundedWaitSelfTest(ctx, limit_ms);
}

int tcscf_ctx_stream(tcscf_ctx * ctx, void ** stream)
{
  if (!ctx || !stream) return TCSCF_ERR_INVALID_ARGUMENT;
  *stream = ctx->stream;
  return TCSCF_OK;
}

int tcscf_synchronize(tcscf_ctx * ctx)
{
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TCSCF_OK;
}

int tcscf_last_timing(tcscf_ctx * ctx, double * contraction_ms, double * total_ms, int * launches)
{
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  if (contraction_ms) *contraction_ms = ctx->lastContractionMs;
  if (total_ms) *total_ms = ctx->lastTotalMs;
  if (launches) *launches = ctx->lastLaunches;
  return TCSCF_OK;
}

int tcscf_last_potentials(tcscf_ctx * ctx, double * VH, double * T)
{
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  TCSCF_CHECK(ctx, ctx->lastVH && ctx->lastT, TCSCF_ERR_INVALID_ARGUMENT, "no direct Fock build has run on this context");
  if (VH) TCSCF_CUDA(ctx, cudaMemcpyAsync(VH, ctx->lastVH, sizeof(double) * ctx->lastN1, cudaMemcpyDeviceToHost, ctx->stream));
  if (T) TCSCF_CUDA(ctx, cudaMemcpyAsync(T, ctx->lastT, sizeof(double) * ctx->lastN1 * ctx->lastNb, cudaMemcpyDeviceToHost, ctx->stream));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TCSCF_OK;
}

int tcscf_grid_create(tcscf_ctx * ctx, const double * points, const double * weights, int64_t n, int ndim, int * grid)
{
  TCSCF_NVTX();
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  TCSCF_CHECK(ctx, points && weights && grid && n > 0 && (ndim == 2 || ndim == 3), TCSCF_ERR_INVALID_ARGUMENT, "invalid grid arguments");
  cudaSetDevice(ctx->device);
  Grid g;
  g.n = n;
  g.ndim = ndim;
  if (gridAlloc(ctx, &g.pts, sizeof(double) * 3 * n) != TCSCF_OK || gridAlloc(ctx, &g.w, sizeof(double) * n) != TCSCF_OK) {
    std::string const msg = ctx->err;
    gridReleaseAll(ctx, g);
    return fail(ctx, TCSCF_ERR_CUDA, msg);
  }
  if (ndim == 3) TCSCF_CUDA(ctx, cudaMemcpyAsync(g.pts, points, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, ctx->stream));
  else {
    TCSCF_CUDA(ctx, cudaMemcpyAsync(g.pts, points, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    TCSCF_CUDA(ctx, cudaMemsetAsync(g.pts + n, 0, sizeof(double) * n, ctx->stream));
    TCSCF_CUDA(ctx, cudaMemcpyAsync(g.pts + 2 * n, points + n, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  }
  TCSCF_CUDA(ctx, cudaMemcpyAsync(g.w, weights, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  int const id = ctx->nextId++;
  ctx->grids[id] = g;
  *grid = id;
  return TCSCF_OK;
}

int tcscf_grid_destroy(tcscf_ctx * ctx, int grid)
{
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  Grid * g = findGrid(ctx, grid);
  TCSCF_CHECK(ctx, g, TCSCF_ERR_INVALID_ARGUMENT, "unknown grid handle");
  nearPairsForget(ctx, g);
  gridReleaseAll(ctx, *g);
  ctx->grids.erase(grid);
  return TCSCF_OK;
}

int tcscf_near_coincident_pairs(tcscf_ctx * ctx, int r1, int r2, int * count)
{
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  TCSCF_CUDA(ctx, cudaSetDevice(ctx->device));
  Grid * g1 = findGrid(ctx, r1);
  Grid * g2 = findGrid(ctx, r2);
  TCSCF_CHECK(ctx, g1 && g2 && count, TCSCF_ERR_INVALID_ARGUMENT, "unknown grid handle or null count");
  NearList const * nl = nullptr;
  TCSCF_TRY(nearPairsFor(ctx, *g1, *g2, &nl));
  *count = nl->count;
  return TCSCF_OK;
}

int tcscf_grid_set_basis(tcscf_ctx * ctx, int grid, const tcscf_sto * basis, int nb, int gradients)
{
  TCSCF_NVTX();
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  Grid * g = findGrid(ctx, grid);
  TCSCF_CHECK(ctx, g, TCSCF_ERR_INVALID_ARGUMENT, "unknown grid handle");
  std::vector<DevSto> ds;
  TCSCF_TRY(validateBasis(ctx, basis, nb, ds));
  TCSCF_CHECK(ctx, !(gradients && basis[0].family == TCSCF_BASIS_HYDROGEN), TCSCF_ERR_UNSUPPORTED,
              "hydrogen-like functions have no gradient (HydrogenLikeBasis.hpp:51-55)");
  gridRelease(ctx, g->dsto); gridRelease(ctx, g->phiR); gridRelease(ctx, g->vals); gridRelease(ctx, g->grads);
  gridRelease(ctx, g->vtCache);
  g->dsto = nullptr; g->phiR = g->vals = g->grads = nullptr;
  g->vtCache = nullptr;
  g->vtNB = 0;
  g->nb = 0;
  TCSCF_TRY(gridAlloc(ctx, &g->dsto, sizeof(DevSto) * nb));
  TCSCF_TRY(gridAlloc(ctx, &g->phiR, sizeof(double) * g->n * nb));
  TCSCF_TRY(gridAlloc(ctx, &g->vals, sizeof(double) * g->n * nb * (g->ndim == 3 ? 2 : 1)));
  if (gradients) TCSCF_TRY(gridAlloc(ctx, &g->grads, sizeof(double) * g->n * nb * 6));
  TCSCF_CUDA(ctx, cudaMemcpyAsync(g->dsto, ds.data(), sizeof(DevSto) * nb, cudaMemcpyHostToDevice, ctx->stream));
  kBasis<<<gridBlocks(g->n * nb, 256), 256, 0, ctx->stream>>>(g->n, nb, g->ndim, g->pts, g->dsto, g->phiR, g->vals, g->grads);
  TCSCF_LAUNCH(ctx);
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  g->nb = nb;
  g->hasGrad = gradients ? 1 : 0;
  g->basis.assign(basis, basis + nb);
  return TCSCF_OK;
}

int tcscf_grid_basis_values(tcscf_ctx * ctx, int grid, double * values, double * gradients)
{
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  Grid * g = findGrid(ctx, grid);
  TCSCF_CHECK(ctx, g && g->nb > 0, TCSCF_ERR_INVALID_ARGUMENT, "grid has no basis");
  if (values)
    TCSCF_CUDA(ctx, cudaMemcpyAsync(values, g->vals, sizeof(double) * g->n * g->nb * (g->ndim == 3 ? 2 : 1), cudaMemcpyDeviceToHost, ctx->stream));
  if (gradients) {
    TCSCF_CHECK(ctx, g->grads, TCSCF_ERR_INVALID_ARGUMENT, "gradients were not stored");
    TCSCF_CUDA(ctx, cudaMemcpyAsync(gradients, g->grads, sizeof(double) * g->n * g->nb * 6, cudaMemcpyDeviceToHost, ctx->stream));
  }
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TCSCF_OK;
}

int tcscf_overlap_core_quadrature(tcscf_ctx * ctx, int grid, int Z, double * S, double * H)
{
  TCSCF_NVTX();
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  Grid * g = findGrid(ctx, grid);
  TCSCF_CHECK(ctx, g && g->nb > 0 && g->ndim == 3, TCSCF_ERR_INVALID_ARGUMENT, "needs a 3-D grid with a basis");
  TCSCF_CHECK(ctx, S, TCSCF_ERR_INVALID_ARGUMENT, "S is required");
  TCSCF_CHECK(ctx, !H || g->grads, TCSCF_ERR_INVALID_ARGUMENT, "H needs stored gradients");
  int const nb = g->nb;
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, "quad_sh", sizeof(double2) * nb * nb * 2, &p));
  double2 * dS = static_cast<double2 *>(p);
  double2 * dH = dS + nb * nb;
  kQuadOverlapCore<<<nb * nb, 256, 0, ctx->stream>>>(g->n, nb, Z, g->pts, g->w, reinterpret_cast<double2 *>(g->vals),
                                                      H ? reinterpret_cast<double2 *>(g->grads) : nullptr, dS, H ? dH : nullptr);
  TCSCF_LAUNCH(ctx);
  TCSCF_CUDA(ctx, cudaMemcpyAsync(S, dS, sizeof(double2) * nb * nb, cudaMemcpyDeviceToHost, ctx->stream));
  if (H) TCSCF_CUDA(ctx, cudaMemcpyAsync(H, dH, sizeof(double2) * nb * nb, cudaMemcpyDeviceToHost, ctx->stream));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TCSCF_OK;
}

// Fixed-scratch form of the S/H quadrature: the block results go to a file-scope device array
// instead of context scratch, so this entry point allocates nothing.  It serves callers that cannot
// allocate device memory at this point: a host whose device memory is already handed out to its own
// pool (grids and tensors sized to fill HBM), and a host that cannot accept the device-wide
// synchronisation that cudaFree implies while its other streams are running.
//   * Limit: nb <= kQuadStaticMaxNb (256), i.e. 2 x 256 x 256 complex doubles = 2 MiB per device;
//     larger bases are rejected with TCSCF_ERR_UNSUPPORTED.
//   * Set-up: tcscf_ctx_create looks up the array's device address (cudaGetSymbolAddress, with the
//     context's device current), so a call of this entry point does no set-up of its own.
//   * Sharing: every call on a device uses the same array, so overlapping calls on one device (other
//     streams or other contexts) race; callers serialise them.  Nothing in the array needs to start
//     at zero: kQuadOverlapCore writes every element it returns (one block per (i, j)).
int tcscf_overlap_core_quadrature_static(tcscf_ctx * ctx, int grid, int Z, double * S, double * H)
{
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  Grid * g = findGrid(ctx, grid);
  TCSCF_CHECK(ctx, g && g->nb > 0 && g->ndim == 3, TCSCF_ERR_INVALID_ARGUMENT, "needs a 3-D grid with a basis");
  TCSCF_CHECK(ctx, S, TCSCF_ERR_INVALID_ARGUMENT, "S is required");
  TCSCF_CHECK(ctx, !H || g->grads, TCSCF_ERR_INVALID_ARGUMENT, "H needs stored gradients");
  int const nb = g->nb;
  TCSCF_CHECK(ctx, nb <= kQuadStaticMaxNb, TCSCF_ERR_UNSUPPORTED,
              "nb = " + std::to_string(nb) + " exceeds the fixed scratch of tcscf_overlap_core_quadrature_static (nb <= " +
                  std::to_string(kQuadStaticMaxNb) + "); use tcscf_overlap_core_quadrature");
  TCSCF_CUDA(ctx, cudaSetDevice(ctx->device));
  double2 * dS = nullptr;
  TCSCF_TRY(quadStaticScratch(ctx, &dS));
  double2 * dH = dS + kQuadStaticMaxNb * kQuadStaticMaxNb;
  kQuadOverlapCore<<<nb * nb, 256, 0, ctx->stream>>>(g->n, nb, Z, g->pts, g->w, reinterpret_cast<double2 *>(g->vals),
                                                      H ? reinterpret_cast<double2 *>(g->grads) : nullptr, dS, H ? dH : nullptr);
  TCSCF_LAUNCH(ctx);
  TCSCF_CUDA(ctx, cudaMemcpyAsync(S, dS, sizeof(double2) * nb * nb, cudaMemcpyDeviceToHost, ctx->stream));
  if (H) TCSCF_CUDA(ctx, cudaMemcpyAsync(H, dH, sizeof(double2) * nb * nb, cudaMemcpyDeviceToHost, ctx->stream));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TCSCF_OK;
}

int tcscf_fock_build(tcscf_ctx * ctx, int r1, int r2, int nspin, const double * density, const double * h, int respect_symmetry,
                     int precision, double * G, double * fock, double * energy)
{
  TCSCF_NVTX();
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  Grid * g1 = findGrid(ctx, r1);
  Grid * g2 = findGrid(ctx, r2);
  TCSCF_TRY(checkBasisPair(ctx, g1, g2));
  TCSCF_CHECK(ctx, nspin == 1 || nspin == 2, TCSCF_ERR_INVALID_ARGUMENT, "nspin must be 1 or 2");
  TCSCF_CHECK(ctx, density && h, TCSCF_ERR_INVALID_ARGUMENT, "density and h are required");
  TCSCF_CHECK(ctx, precision >= TCSCF_PREC_FP64 && precision <= TCSCF_PREC_TF32, TCSCF_ERR_INVALID_ARGUMENT, "unknown precision");
  int const nb = g1->nb;
  size_t const nn = size_t(nb) * nb;
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, "fock_io", sizeof(double2) * nn * nspin * 3 + sizeof(double) * nn + 64, &p));
  double2 * dD = static_cast<double2 *>(p);
  double2 * dG = dD + nn * nspin;
  double2 * dF = dG + nn * nspin;
  double * dH = reinterpret_cast<double *>(dF + nn * nspin);
  double * dE = dH + nn;
  TCSCF_CUDA(ctx, cudaMemcpyAsync(dD, density, sizeof(double2) * nn * nspin, cudaMemcpyHostToDevice, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemcpyAsync(dH, h, sizeof(double) * nn, cudaMemcpyHostToDevice, ctx->stream));
  TCSCF_TRY(fockBuildDevice(ctx, *g1, *g2, nspin, dD, dH, respect_symmetry, precision, dG, dF, dE, nullptr));
  if (G) TCSCF_CUDA(ctx, cudaMemcpyAsync(G, dG, sizeof(double2) * nn * nspin, cudaMemcpyDeviceToHost, ctx->stream));
  if (fock) TCSCF_CUDA(ctx, cudaMemcpyAsync(fock, dF, sizeof(double2) * nn * nspin, cudaMemcpyDeviceToHost, ctx->stream));
  double e = 0;
  TCSCF_CUDA(ctx, cudaMemcpyAsync(&e, dE, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (energy) *energy = e;
  if (!(e == e) || std::isinf(e)) return fail(ctx, TCSCF_ERR_NONFINITE, "non-finite energy");
  return TCSCF_OK;
}

int tcscf_fock_build_device(tcscf_ctx * ctx, int r1, int r2, int nspin, const double * density, const double * h, int respect_symmetry,
                            int precision, double * G, double * fock, double * energy)
{
  TCSCF_NVTX();
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  Grid * g1 = findGrid(ctx, r1);
  Grid * g2 = findGrid(ctx, r2);
  TCSCF_TRY(checkBasisPair(ctx, g1, g2));
  TCSCF_CHECK(ctx, nspin == 1 || nspin == 2, TCSCF_ERR_INVALID_ARGUMENT, "nspin must be 1 or 2");
  TCSCF_CHECK(ctx, density && h && energy, TCSCF_ERR_INVALID_ARGUMENT, "density, h and energy are required");
  TCSCF_CHECK(ctx, precision >= TCSCF_PREC_FP64 && precision <= TCSCF_PREC_TF32, TCSCF_ERR_INVALID_ARGUMENT, "unknown precision");
  size_t const nn = size_t(g1->nb) * g1->nb;
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, "fock_dev_io", sizeof(double2) * nn * nspin * 2, &p));
  double2 * dG = G ? reinterpret_cast<double2 *>(G) : static_cast<double2 *>(p);
  double2 * dF = fock ? reinterpret_cast<double2 *>(fock) : static_cast<double2 *>(p) + nn * nspin;
  TCSCF_TRY(fockBuildDevice(ctx, *g1, *g2, nspin, reinterpret_cast<const double2 *>(density), h, respect_symmetry, precision, dG, dF, energy,
                            nullptr));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TCSCF_OK;
}

int tcscf_compute_F(tcscf_ctx * ctx, int r1, int r2, int kernel, const tcscf_ochi * jastrow, int precision, double * F, int keep,
                    int * fji)
{
  TCSCF_NVTX();
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  TCSCF_CHECK(ctx, kernel >= TCSCF_K_INV_R12 && kernel <= TCSCF_K_TC_SCALAR_OPPO, TCSCF_ERR_INVALID_ARGUMENT, "computeF takes a scalar kernel");
  TCSCF_CHECK(ctx, kernel == TCSCF_K_INV_R12 || jastrow, TCSCF_ERR_INVALID_ARGUMENT, "TC kernels need the Jastrow parameters");
  return precomputeTensor(ctx, r1, r2, kernel, jastrow, precision, 1, F, keep, fji);
}

int tcscf_compute_V(tcscf_ctx * ctx, int r1, int r2, int kernel, const tcscf_ochi * jastrow, int precision, double * V, int keep,
                    int * vji)
{
  TCSCF_NVTX();
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  TCSCF_CHECK(ctx, kernel == TCSCF_K_GRAD_U_SAME || kernel == TCSCF_K_GRAD_U_OPPO, TCSCF_ERR_INVALID_ARGUMENT, "computeV takes a vector kernel");
  TCSCF_CHECK(ctx, jastrow, TCSCF_ERR_INVALID_ARGUMENT, "Jastrow parameters required");
  return precomputeTensor(ctx, r1, r2, kernel, jastrow, precision, 3, V, keep, vji);
}

int tcscf_tensor_destroy(tcscf_ctx * ctx, int handle)
{
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  auto it = ctx->tensors.find(handle);
  TCSCF_CHECK(ctx, it != ctx->tensors.end(), TCSCF_ERR_INVALID_ARGUMENT, "unknown tensor handle");
  cudaStreamSynchronize(ctx->stream);
  cudaFree(it->second.d);
  ctx->tensors.erase(it);
  return TCSCF_OK;
}

int tcscf_fock_build_batch(tcscf_ctx * ctx, int count, const int * r1, const int * r2, const double * const * density,
                           const double * const * h, int respect_symmetry, int precision, double * energy, double * const * fock)
{
  TCSCF_NVTX();
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  TCSCF_CHECK(ctx, count >= 1 && r1 && r2 && density && h && energy, TCSCF_ERR_INVALID_ARGUMENT, "batch: count, grids, densities, h and energy are required");
  TCSCF_CHECK(ctx, precision >= TCSCF_PREC_FP64 && precision <= TCSCF_PREC_TF32, TCSCF_ERR_INVALID_ARGUMENT, "unknown precision");
  std::vector<Grid *> g1s(count), g2s(count);
  size_t io = 0;
  for (int k = 0; k < count; ++k) {
    g1s[k] = findGrid(ctx, r1[k]);
    g2s[k] = findGrid(ctx, r2[k]);
    TCSCF_TRY(checkBasisPair(ctx, g1s[k], g2s[k]));
    TCSCF_CHECK(ctx, density[k] && h[k], TCSCF_ERR_INVALID_ARGUMENT, "batch: every instance needs a density and h");
    size_t const nn = size_t(g1s[k]->nb) * g1s[k]->nb;
    io += sizeof(double2) * 3 * nn + sizeof(double) * nn + 256;
  }
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, "batch_io", io + sizeof(double) * count + 256, &p));
  std::vector<const double2 *> dD(count);
  std::vector<const double *> dH(count);
  std::vector<double2 *> dG(count), dF(count);
  std::vector<double *> dE(count);
  char * q = static_cast<char *>(p);
  double * energies = reinterpret_cast<double *>(q);
  q += (sizeof(double) * count + 255) & ~size_t(255);
  for (int k = 0; k < count; ++k) {
    size_t const nn = size_t(g1s[k]->nb) * g1s[k]->nb;
    auto * d = reinterpret_cast<double2 *>(q);
    dD[k] = d; dG[k] = d + nn; dF[k] = d + 2 * nn;
    auto * hh = reinterpret_cast<double *>(d + 3 * nn);
    dH[k] = hh;
    dE[k] = energies + k;
    q += (sizeof(double2) * 3 * nn + sizeof(double) * nn + 255) & ~size_t(255);
    TCSCF_CUDA(ctx, cudaMemcpyAsync(d, density[k], sizeof(double2) * nn, cudaMemcpyHostToDevice, ctx->stream));
    TCSCF_CUDA(ctx, cudaMemcpyAsync(hh, h[k], sizeof(double) * nn, cudaMemcpyHostToDevice, ctx->stream));
  }
  auto build = [&]() {
    return fockBuildBatch(ctx, count, g1s.data(), g2s.data(), dD.data(), dH.data(), respect_symmetry, precision, dG.data(), dF.data(), dE.data());
  };
  if (ctx->autotune && (precision == TCSCF_PREC_BF16X3 || precision == TCSCF_PREC_TF32)) {
    // batch signature: precision and every instance's grid sizes and basis size
    std::vector<int64_t> key{precision, count};
    for (int k = 0; k < count; ++k) key.insert(key.end(), {g1s[k]->n, g2s[k]->n, int64_t(g1s[k]->nb)});
    auto it = ctx->tunedBatchPolicy.find(key);
    if (it == ctx->tunedBatchPolicy.end()) {
      // each policy's whole batch build runs twice and the second (its graph replayed, scratch
      // grown) is timed between the build's own events; the inputs are read-only, so every run
      // writes the same outputs up to the order of the r2 sums
      int best = 1;
      double bestMs = 0;
      bool first = true;
      for (int policy : {1, 0, 2, 4}) {
        ctx->batchSplitPolicy = policy;
        int st = build();
        if (st == TCSCF_OK) st = build();
        if (st != TCSCF_OK) { ctx->batchSplitPolicy = 1; return st; }
        ++ctx->tuneMeasurements;
        if (first || ctx->lastTotalMs < bestMs) { bestMs = ctx->lastTotalMs; best = policy; }
        first = false;
      }
      it = ctx->tunedBatchPolicy.emplace(key, best).first;
    }
    ctx->batchSplitPolicy = it->second;
  }
  int const bst = build();
  ctx->batchSplitPolicy = 1;
  TCSCF_TRY(bst);
  TCSCF_CUDA(ctx, cudaMemcpyAsync(energy, energies, sizeof(double) * count, cudaMemcpyDeviceToHost, ctx->stream));
  for (int k = 0; k < count; ++k)
    if (fock && fock[k])
      TCSCF_CUDA(ctx, cudaMemcpyAsync(fock[k], dF[k], sizeof(double2) * g1s[k]->nb * g1s[k]->nb, cudaMemcpyDeviceToHost, ctx->stream));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int k = 0; k < count; ++k)
    if (!(energy[k] == energy[k]) || std::isinf(energy[k])) return fail(ctx, TCSCF_ERR_NONFINITE, "non-finite energy in batch instance " + std::to_string(k));
  return TCSCF_OK;
}

int tcscf_fock_build_precomputed(tcscf_ctx * ctx, int r1, int fji, int nspin, const double * density, const double * h,
                                 int respect_symmetry, double * G, double * fock, double * energy)
{
  TCSCF_NVTX();
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  Grid * g1 = findGrid(ctx, r1);
  TCSCF_CHECK(ctx, g1 && g1->nb > 0 && g1->ndim == 3, TCSCF_ERR_INVALID_ARGUMENT, "r1 grid needs a basis");
  auto it = ctx->tensors.find(fji);
  TCSCF_CHECK(ctx, it != ctx->tensors.end() && !it->second.vec, TCSCF_ERR_INVALID_ARGUMENT, "unknown Fji handle");
  Tensor const & t = it->second;
  TCSCF_CHECK(ctx, t.n1 == g1->n && t.nb == g1->nb, TCSCF_ERR_INVALID_ARGUMENT, "Fji does not match the r1 grid");
  TCSCF_CHECK(ctx, nspin == 1 || nspin == 2, TCSCF_ERR_INVALID_ARGUMENT, "nspin must be 1 or 2");
  TCSCF_CHECK(ctx, density && h, TCSCF_ERR_INVALID_ARGUMENT, "density and h are required");
  int const nb = g1->nb;
  int64_t const n1 = g1->n;
  size_t const nn = size_t(nb) * nb;
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, "fock_pre", sizeof(double2) * (nn * nspin * 3 + size_t(nspin) * n1 * (nb + 1) + n1) + sizeof(double) * (nn + 8), &p));
  double2 * dD = static_cast<double2 *>(p);
  double2 * dG = dD + nn * nspin;
  double2 * dF = dG + nn * nspin;
  double2 * Faa = dF + nn * nspin;
  double2 * FaaTot = Faa + size_t(nspin) * n1;
  double2 * Fai = FaaTot + n1;
  double * dH = reinterpret_cast<double *>(Fai + size_t(nspin) * n1 * nb);
  double * dE = dH + nn;
  TCSCF_CUDA(ctx, cudaMemcpyAsync(dD, density, sizeof(double2) * nn * nspin, cudaMemcpyHostToDevice, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemcpyAsync(dH, h, sizeof(double) * nn, cudaMemcpyHostToDevice, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemsetAsync(Faa, 0, sizeof(double2) * (size_t(nspin) * n1 * (nb + 1) + n1), ctx->stream));
  TCSCF_CUDA(ctx, cudaMemsetAsync(dG, 0, sizeof(double2) * nn * nspin, ctx->stream));
  cudaEventRecord(ctx->ev[0], ctx->stream);
  int const launch0 = ctx->launchCount;
  for (int s = 0; s < nspin; ++s) {
    size_t const sm = sizeof(double2) * nb;
    if (t.isComplex)
      kFaaFai<true><<<unsigned(n1), 128, sm, ctx->stream>>>(n1, nb, t.d, reinterpret_cast<double2 *>(g1->vals), dD + s * nn, Faa + s * n1, Fai + s * n1 * nb);
    else
      kFaaFai<false><<<unsigned(n1), 128, sm, ctx->stream>>>(n1, nb, t.d, reinterpret_cast<double2 *>(g1->vals), dD + s * nn, Faa + s * n1, Fai + s * n1 * nb);
    TCSCF_LAUNCH(ctx);
    kAddInto<<<gridBlocks(2 * n1, 256), 256, 0, ctx->stream>>>(2 * n1, reinterpret_cast<double *>(Faa + s * n1), reinterpret_cast<double *>(FaaTot));
    TCSCF_LAUNCH(ctx);
  }
  double const cJ = nspin == 1 ? 2.0 : 1.0;
  for (int s = 0; s < nspin; ++s)
    TCSCF_TRY(reduceFockComplex(ctx, n1, nb, g1->vals, g1->w, reinterpret_cast<double *>(FaaTot), cJ,
                                reinterpret_cast<double *>(Fai + s * n1 * nb), reinterpret_cast<double *>(dG + s * nn)));
  kFinalize<<<1, 512, 0, ctx->stream>>>(nspin, nb, dH, dG, nullptr, dD, respect_symmetry, nspin == 1 ? 2.0 : 1.0, dF, dE);
  TCSCF_LAUNCH(ctx);
  cudaEventRecord(ctx->ev[1], ctx->stream);
  if (G) TCSCF_CUDA(ctx, cudaMemcpyAsync(G, dG, sizeof(double2) * nn * nspin, cudaMemcpyDeviceToHost, ctx->stream));
  if (fock) TCSCF_CUDA(ctx, cudaMemcpyAsync(fock, dF, sizeof(double2) * nn * nspin, cudaMemcpyDeviceToHost, ctx->stream));
  double e = 0;
  TCSCF_CUDA(ctx, cudaMemcpyAsync(&e, dE, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
  ctx->lastTotalMs = ms;
  ctx->lastContractionMs = ms;
  ctx->lastLaunches = ctx->launchCount - launch0;
  if (energy) *energy = e;
  if (!(e == e) || std::isinf(e)) return fail(ctx, TCSCF_ERR_NONFINITE, "non-finite energy");
  return TCSCF_OK;
}

int tcscf_set_scf_options(tcscf_ctx * ctx, int diis, int real_eigensolve)
{
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  TCSCF_CHECK(ctx, diis >= 0 && diis <= 16, TCSCF_ERR_INVALID_ARGUMENT, "DIIS history must be 0..16");
  ctx->diisSize = diis == 1 ? 0 : diis;
  ctx->realEigen = real_eigensolve ? 1 : 0;
  return TCSCF_OK;
}

int tcscf_scf(tcscf_ctx * ctx, int r1, int r2, int nspin, int n_up, int n_down, const double * S, const double * h, int respect_symmetry,
              int precision, double tol, int max_iter, double * energy, int * iterations, double * density, double * eigenvalues)
{
  TCSCF_NVTX();
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  Grid * g1 = findGrid(ctx, r1);
  Grid * g2 = findGrid(ctx, r2);
  TCSCF_TRY(checkBasisPair(ctx, g1, g2));
  TCSCF_CHECK(ctx, nspin == 1 || nspin == 2, TCSCF_ERR_INVALID_ARGUMENT, "nspin must be 1 or 2");
  TCSCF_CHECK(ctx, S && h && max_iter > 0, TCSCF_ERR_INVALID_ARGUMENT, "S, h and max_iter are required");
  // RCSHartreeFock requires an even electron count (HartreeFock.hpp:248)
  TCSCF_CHECK(ctx, nspin == 2 || (n_up + n_down) % 2 == 0, TCSCF_ERR_INVALID_ARGUMENT, "RCS needs an even electron count");
  int const nb = g1->nb;
  int const nocc[2] = {nspin == 1 ? (n_up + n_down) / 2 : n_up, n_down};
  TCSCF_CHECK(ctx, nocc[0] <= nb && nocc[1] <= nb && nocc[0] >= 0 && nocc[1] >= 0, TCSCF_ERR_INVALID_ARGUMENT, "more electrons than basis functions");
  size_t const nn = size_t(nb) * nb;
  void * p = nullptr;
  TCSCF_TRY(scratch(ctx, "scf", sizeof(double2) * (nn * nspin * 3 + nn * 2) + sizeof(double) * (nn * 2 + nb * nspin + 16), &p));
  double2 * dD = static_cast<double2 *>(p);
  double2 * dG = dD + nn * nspin;
  double2 * dF = dG + nn * nspin;
  double2 * A = dF + nn * nspin;
  double2 * B = A + nn;
  double * dH = reinterpret_cast<double *>(B + nn);
  double * dS = dH + nn;
  double * W = dS + nn;
  double * dE = W + nb * nspin;
  int * devInfo = reinterpret_cast<int *>(dE + 8);
  TCSCF_CUDA(ctx, cudaMemsetAsync(dD, 0, sizeof(double2) * nn * nspin, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemcpyAsync(dH, h, sizeof(double) * nn, cudaMemcpyHostToDevice, ctx->stream));
  TCSCF_CUDA(ctx, cudaMemcpyAsync(dS, S, sizeof(double) * nn, cudaMemcpyHostToDevice, ctx->stream));
  int lwork = 0;
  if (cusolverDnZhegvd_bufferSize(ctx->solver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nb,
                                  reinterpret_cast<cuDoubleComplex *>(A), nb, reinterpret_cast<cuDoubleComplex *>(B), nb, W, &lwork) != CUSOLVER_STATUS_SUCCESS)
    return fail(ctx, TCSCF_ERR_LINALG, "cusolverDnZhegvd_bufferSize failed");
  void * wk = nullptr;
  TCSCF_TRY(scratch(ctx, "hegvd_work", sizeof(double2) * size_t(lwork) + 64, &wk));
  // optional Pulay DIIS: history of Fock matrices and commutator errors FDS - SDF (both spins)
  int const nd = ctx->diisSize;
  size_t const len = size_t(nspin) * nn;
  double2 * Fh = nullptr, * Eh = nullptr, * T1 = nullptr, * T2 = nullptr, * Sc = nullptr, * Fd = nullptr;
  double * dDots = nullptr, * dCoef = nullptr;
  cublasHandle_t bh = nullptr;
  std::vector<double> Bm(size_t(nd) * nd, 0.0), hDots(nd), coef;
  int count = 0, head = 0;
  {
    void * q = nullptr;
    TCSCF_TRY(scratch(ctx, "scf_diis", sizeof(double2) * (2 * size_t(nd) * len + 3 * nn + len) + sizeof(double) * 2 * (nd + 1) + 1024, &q));
    Fh = static_cast<double2 *>(q);
    Eh = Fh + size_t(nd) * len;
    T1 = Eh + size_t(nd) * len;
    T2 = T1 + nn;
    Sc = T2 + nn;
    Fd = Sc + nn;
    dDots = reinterpret_cast<double *>(Fd + len);
    dCoef = dDots + nd + 1;
    kRealToComplex<<<gridBlocks(int64_t(nn), 256), 256, 0, ctx->stream>>>(int64_t(nn), dS, Sc);
    TCSCF_LAUNCH(ctx);
    if (nd > 0) TCSCF_TRY(blasHandle(ctx, &bh));
  }
  // Optional real-harmonic eigen-solve (tcscf_set_scf_options): the Fock matrix of a density that is
  // real in the real-harmonic basis is real there too, and the real symmetric problem
  // (cusolverDnDsygvd) gives real eigenvectors, so the next density stays real (one rank-nocc tensor
  // contraction per build) even when the aufbau occupation splits a degenerate shell, where the complex
  // solver of the reference basis returns arbitrary complex combinations (doubling the factor rank
  // and the contractions).  Same eigenvalues; when a degenerate level is partly occupied the two
  // solvers occupy different members of it, so the default keeps the reference's complex path.
  void * rp = nullptr;
  TCSCF_TRY(scratch(ctx, "scf_real", sizeof(double2) * 2 * nn + sizeof(double) * 5 * nn + 256, &rp));
  double2 * FR = static_cast<double2 *>(rp);
  double2 * SRc = FR + nn;
  double * Ar = reinterpret_cast<double *>(SRc + nn);
  double * Br = Ar + nn;
  double * SRre = Br + nn;
  double * DRre = SRre + nn;
  double * fmax = DRre + nn;
  bool realPath = true;
  int lworkR = 0;
  void * wkR = nullptr;
  {
    kDensityToReal<<<gridBlocks(nn, 256), 256, 0, ctx->stream>>>(1, nb, g1->dsto, Sc, SRc);
    TCSCF_LAUNCH(ctx);
    kSplitDensity<<<1, 256, 0, ctx->stream>>>(nb, SRc, SRre, fmax);
    TCSCF_LAUNCH(ctx);
    double hm[2];
    TCSCF_CUDA(ctx, cudaMemcpyAsync(hm, fmax, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    realPath = ctx->realEigen && hm[1] <= 1e-12 * hm[0];
    if (realPath) {
      if (cusolverDnDsygvd_bufferSize(ctx->solver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nb, Ar, nb, Br, nb, W,
                                      &lworkR) != CUSOLVER_STATUS_SUCCESS)
        return fail(ctx, TCSCF_ERR_LINALG, "cusolverDnDsygvd_bufferSize failed");
      TCSCF_TRY(scratch(ctx, "sygvd_work", sizeof(double) * size_t(lworkR) + 64, &wkR));
    }
  }
  double2 const one = make_double2(1, 0), zero = make_double2(0, 0), mone = make_double2(-1, 0);
  double e = std::numeric_limits<double>::max();
  // density factors from the previous iteration's real-harmonic eigen-solve (every spin solved real)
  Factor given[2];
  bool givenOk = false;
  double * Xocc = nullptr;
  if (realPath) TCSCF_TRY(scratch(ctx, "scf_occ_factor", sizeof(double) * 2 * nn + 64, reinterpret_cast<void **>(&Xocc)));
  for (int it = 0; it < max_iter; ++it) {
    TCSCF_TRY(fockBuildDevice(ctx, *g1, *g2, nspin, dD, dH, respect_symmetry, precision, dG, dF, dE, givenOk ? given : nullptr));
    double ne = 0;
    TCSCF_CUDA(ctx, cudaMemcpyAsync(&ne, dE, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (!(ne == ne) || std::isinf(ne)) return fail(ctx, TCSCF_ERR_NONFINITE, "non-finite energy");
    if (iterations) *iterations = it + 1;
    if (std::fabs(ne - e) < tol) {
      if (energy) *energy = ne;
      if (density) TCSCF_CUDA(ctx, cudaMemcpy(density, dD, sizeof(double2) * nn * nspin, cudaMemcpyDeviceToHost));
      if (eigenvalues) TCSCF_CUDA(ctx, cudaMemcpy(eigenvalues, W, sizeof(double) * nb * nspin, cudaMemcpyDeviceToHost));
      return TCSCF_OK;
    }
    e = ne;
    const double2 * Fuse = dF;
    if (nd > 0 && it >= 1) {
      int const slot = head;
      head = (head + 1) % nd;
      count = std::min(count + 1, nd);
      for (int s = 0; s < nspin; ++s) {
        double2 const * Fs = dF + s * nn;
        double2 const * Ds = dD + s * nn;
        double2 * Es = Eh + slot * len + s * nn;
        TCSCF_TRY(rowMajorZgemm(ctx, bh, nb, one, Ds, Sc, zero, T1));     // D S
        TCSCF_TRY(rowMajorZgemm(ctx, bh, nb, one, Fs, T1, zero, Es));     // F D S
        TCSCF_TRY(rowMajorZgemm(ctx, bh, nb, one, Sc, Ds, zero, T2));     // S D
        TCSCF_TRY(rowMajorZgemm(ctx, bh, nb, mone, T2, Fs, one, Es));     // - S D F
        TCSCF_CUDA(ctx, cudaMemcpyAsync(Fh + slot * len + s * nn, Fs, sizeof(double2) * nn, cudaMemcpyDeviceToDevice, ctx->stream));
      }
      kDiisDots<<<count, 256, 0, ctx->stream>>>(int64_t(len), slot, count, Eh, dDots);
      TCSCF_LAUNCH(ctx);
      TCSCF_CUDA(ctx, cudaMemcpyAsync(hDots.data(), dDots, sizeof(double) * count, cudaMemcpyDeviceToHost, ctx->stream));
      TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      for (int j = 0; j < count; ++j) Bm[slot * nd + j] = Bm[j * nd + slot] = hDots[j];
      if (count >= 2) {
        // equations scaled by the largest error norm for conditioning
        double mx = 0;
        for (int j = 0; j < count; ++j) mx = std::max(mx, Bm[j * nd + j]);
        std::vector<double> Bs(size_t(count) * count);
        for (int i = 0; i < count; ++i)
          for (int j = 0; j < count; ++j) Bs[i * count + j] = mx > 0 ? Bm[i * nd + j] / mx : Bm[i * nd + j];
        if (mx > 0 && solveDiis(count, Bs, count, coef)) {
          TCSCF_CUDA(ctx, cudaMemcpyAsync(dCoef, coef.data(), sizeof(double) * count, cudaMemcpyHostToDevice, ctx->stream));
          kDiisCombine<<<gridBlocks(int64_t(len), 256), 256, 0, ctx->stream>>>(int64_t(len), count, dCoef, Fh, Fd);
          TCSCF_LAUNCH(ctx);
          Fuse = Fd;
        }
      }
    }
    int solvedReal = 0;
    given[0] = given[1] = Factor{};
    for (int s = 0; s < nspin; ++s) {
      if (realPath) {
        kDensityToReal<<<gridBlocks(nn, 256), 256, 0, ctx->stream>>>(1, nb, g1->dsto, Fuse + s * nn, FR);
        TCSCF_LAUNCH(ctx);
        kSplitDensity<<<1, 256, 0, ctx->stream>>>(nb, FR, Ar, fmax);
        TCSCF_LAUNCH(ctx);
        double hm[2];
        TCSCF_CUDA(ctx, cudaMemcpyAsync(hm, fmax, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        if (!(hm[0] == hm[0]) || !(hm[1] == hm[1])) return fail(ctx, TCSCF_ERR_NONFINITE, "non-finite Fock matrix");
        if (hm[1] <= 1e-10 * hm[0]) {
          TCSCF_CUDA(ctx, cudaMemcpyAsync(Br, SRre, sizeof(double) * nn, cudaMemcpyDeviceToDevice, ctx->stream));
          if (cusolverDnDsygvd(ctx->solver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nb, Ar, nb, Br, nb, W + s * nb,
                               static_cast<double *>(wkR), lworkR, devInfo) != CUSOLVER_STATUS_SUCCESS)
            return fail(ctx, TCSCF_ERR_LINALG, "cusolverDnDsygvd failed");
          int info = 0;
          TCSCF_CUDA(ctx, cudaMemcpyAsync(&info, devInfo, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
          TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
          if (info != 0) return fail(ctx, TCSCF_ERR_LINALG, "generalized eigen-solve failed (info " + std::to_string(info) + ")");
          kRealDensity<<<gridBlocks(nn, 256), 256, 0, ctx->stream>>>(nb, nocc[s], Ar, DRre);
          TCSCF_LAUNCH(ctx);
          kRealToReference<<<gridBlocks(nn, 256), 256, 0, ctx->stream>>>(1, nb, g1->dsto, DRre, nullptr, dD + s * nn);
          TCSCF_LAUNCH(ctx);
          // the next build factors this density as its occupied orbitals themselves (D_R = C C^T):
          // smooth from one iteration to the next, unlike a pivoted factorisation of D
          if (nocc[s] > 0) {
            kFactorFromOrbitals<<<gridBlocks(int64_t(nb) * nocc[s], 256), 256, 0, ctx->stream>>>(nb, nocc[s], Ar, nb, Xocc + size_t(s) * nn);
            TCSCF_LAUNCH(ctx);
            given[s].R = nocc[s];
            given[s].X1 = given[s].X2 = Xocc + size_t(s) * nn;
            given[s].ldx = nb;
            given[s].complex = false;
            given[s].same = true;
          }
          ++solvedReal;
          continue;
        }
      }
      kToColumnMajor<<<gridBlocks(nn, 256), 256, 0, ctx->stream>>>(nb, Fuse + s * nn, dS, A, B);
      TCSCF_LAUNCH(ctx);
      if (cusolverDnZhegvd(ctx->solver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nb,
                           reinterpret_cast<cuDoubleComplex *>(A), nb, reinterpret_cast<cuDoubleComplex *>(B), nb, W + s * nb,
                           static_cast<cuDoubleComplex *>(wk), lwork, devInfo) != CUSOLVER_STATUS_SUCCESS)
        return fail(ctx, TCSCF_ERR_LINALG, "cusolverDnZhegvd failed");
      int info = 0;
      TCSCF_CUDA(ctx, cudaMemcpyAsync(&info, devInfo, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
      TCSCF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      if (info != 0) return fail(ctx, TCSCF_ERR_LINALG, "generalized eigen-solve failed (info " + std::to_string(info) + ")");
      kDensityFromOrbitals<<<gridBlocks(nn, 256), 256, 0, ctx->stream>>>(nb, nocc[s], A, dD + s * nn);
      TCSCF_LAUNCH(ctx);
    }
    givenOk = solvedReal == nspin;
  }
  if (energy) *energy = e;
  if (density) TCSCF_CUDA(ctx, cudaMemcpy(density, dD, sizeof(double2) * nn * nspin, cudaMemcpyDeviceToHost));
  if (eigenvalues) TCSCF_CUDA(ctx, cudaMemcpy(eigenvalues, W, sizeof(double) * nb * nspin, cudaMemcpyDeviceToHost));
  return fail(ctx, TCSCF_ERR_NOT_CONVERGED, "Did not converge.");
}

int tcscf_scf_graph(tcscf_ctx * ctx, int r1, int r2, int n_up, int n_down, const double * S, const double * h, int respect_symmetry,
                    int precision, double tol, int max_iter, int capture, double * energy, int * iterations, double * density,
                    double * eigenvalues, int * graph_launches)
{
  TCSCF_NVTX();
  if (!ctx) return TCSCF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  Grid * g1 = findGrid(ctx, r1);
  Grid * g2 = findGrid(ctx, r2);
  TCSCF_TRY(checkBasisPair(ctx, g1, g2));
  TCSCF_CHECK(ctx, S && h && max_iter > 0, TCSCF_ERR_INVALID_ARGUMENT, "S, h and max_iter are required");
  TCSCF_CHECK(ctx, (n_up + n_down) % 2 == 0 && n_up == n_down, TCSCF_ERR_INVALID_ARGUMENT, "the graph SCF is restricted closed shell");
  TCSCF_CHECK(ctx, precision >= TCSCF_PREC_FP64 && precision <= TCSCF_PREC_TF32, TCSCF_ERR_INVALID_ARGUMENT, "unknown precision");
  int launches = 0;
  int const st = scfGraph(ctx, *g1, *g2, (n_up + n_down) / 2, S, h, respect_symmetry, precision, tol, max_iter, capture, energy, iterations,
                          density, eigenvalues, &launches);
  if (graph_launches) *graph_launches = launches;
  return st;
}

}  // extern "C"
