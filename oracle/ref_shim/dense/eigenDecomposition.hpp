// The eigen-solves the reference's SCF drivers call through LvArray::dense with the LAPACK backend,
// for the oracle's reference build (test infrastructure): hegvd -> zhegvd (A x = lambda B x, A and B
// Hermitian, given by the triangle named, B positive definite; A overwritten with the eigenvectors,
// eigenvalues ascending) and ggev -> zggev (right eigenvectors only, as the transcorrelated driver asks).
// LAPACK is reached through function pointers that the build's entry points set from a shared library
// (scipy's bundled OpenBLAS), the same LAPACK the oracle uses.  Operands are copied into contiguous
// column-major buffers (the slices the drivers pass are column-major already, but may be strided).
// Only complex<double> operands are supported; the single-precision instantiations throw.
#pragma once

#include <complex>
#include <cstddef>
#include <stdexcept>
#include <type_traits>
#include <vector>

#include "common.hpp"

namespace LvArray {
namespace dense {
namespace lapack {
using cplx = std::complex<double>;
using zhegvd_t = void (*)(int const *, char const *, char const *, int const *, cplx *, int const *, cplx *, int const *, double *,
                          cplx *, int const *, double *, int const *, int *, int const *, int *, size_t, size_t);
using zggev_t = void (*)(char const *, char const *, int const *, cplx *, int const *, cplx *, int const *, cplx *, cplx *, cplx *,
                         int const *, cplx *, int const *, cplx *, int const *, double *, int *, size_t, size_t);
inline zhegvd_t & zhegvd()
{
  static zhegvd_t f = nullptr;
  return f;
}
inline zggev_t & zggev()
{
  static zggev_t f = nullptr;
  return f;
}

template <typename SLICE>
std::vector<cplx> gather(SLICE const & M, int n)
{
  std::vector<cplx> out(size_t(n) * n);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) out[size_t(j) * n + i] = cplx(M(i, j));
  return out;
}
template <typename SLICE>
void scatter(std::vector<cplx> const & in, SLICE const & M, int n)
{
  using E = std::remove_reference_t<decltype(M(0, 0))>;
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) M(i, j) = E(in[size_t(j) * n + i]);
}
}  // namespace lapack

template <typename OPTIONS, typename A_SLICE, typename B_SLICE, typename W_SLICE, typename WORKSPACE>
void hegvd(BuiltInBackends, OPTIONS const & options, A_SLICE const & A, B_SLICE const & B, W_SLICE const & eigenvalues, WORKSPACE &,
           SymmetricMatrixStorageType storage)
{
  using E = std::remove_cv_t<std::remove_reference_t<decltype(A(0, 0))>>;
  if constexpr (!std::is_same_v<E, std::complex<double>>) {
    throw std::runtime_error("hegvd: only complex<double> in the oracle's reference build");
  } else {
    LVARRAY_ERROR_IF(!lapack::zhegvd(), "hegvd: LAPACK not loaded");
    LVARRAY_ERROR_IF(options.problem != EigenDecompositionOptions::Ax_eq_lambdaBx, "hegvd: only A x = lambda B x");
    int const n = int(A.size(0));
    std::vector<lapack::cplx> a = lapack::gather(A, n), b = lapack::gather(B, n);
    std::vector<double> w(static_cast<size_t>(n));
    int itype = 1, info = 0, lwork = -1, lrwork = -1, liwork = -1, iq = 0;
    char const jobz = options.type == EigenDecompositionOptions::EIGENVALUES ? 'N' : 'V';
    char const uplo = storage == SymmetricMatrixStorageType::UPPER_TRIANGULAR ? 'U' : 'L';
    lapack::cplx wq;
    double rq = 0;
    lapack::zhegvd()(&itype, &jobz, &uplo, &n, a.data(), &n, b.data(), &n, w.data(), &wq, &lwork, &rq, &lrwork, &iq, &liwork, &info, 1, 1);
    lwork = int(wq.real()) + 1;
    lrwork = int(rq) + 1;
    liwork = iq + 1;
    std::vector<lapack::cplx> work(static_cast<size_t>(lwork));
    std::vector<double> rwork(static_cast<size_t>(lrwork));
    std::vector<int> iwork(static_cast<size_t>(liwork));
    lapack::zhegvd()(&itype, &jobz, &uplo, &n, a.data(), &n, b.data(), &n, w.data(), work.data(), &lwork, rwork.data(), &lrwork,
                     iwork.data(), &liwork, &info, 1, 1);
    LVARRAY_ERROR_IF(info != 0, "zhegvd info " << info);
    for (int i = 0; i < n; ++i) eigenvalues[i] = w[size_t(i)];
    lapack::scatter(a, A, n);
    lapack::scatter(b, B, n);
  }
}

template <typename OPTIONS, typename A_SLICE, typename B_SLICE, typename ALPHA_SLICE, typename BETA_SLICE, typename VL_SLICE, typename VR_SLICE,
          typename WORKSPACE>
void ggev(BuiltInBackends, OPTIONS const & options, A_SLICE const & A, B_SLICE const & B, ALPHA_SLICE const & alpha, BETA_SLICE const & beta,
          VL_SLICE const &, VR_SLICE const & VR, WORKSPACE &)
{
  using E = std::remove_cv_t<std::remove_reference_t<decltype(A(0, 0))>>;
  if constexpr (!std::is_same_v<E, std::complex<double>>) {
    throw std::runtime_error("ggev: only complex<double> in the oracle's reference build");
  } else {
    LVARRAY_ERROR_IF(!lapack::zggev(), "ggev: LAPACK not loaded");
    LVARRAY_ERROR_IF(options.type != EigenDecompositionOptions::EIGENVALUES_AND_RIGHT_VECTORS, "ggev: only right eigenvectors");
    int const n = int(A.size(0));
    std::vector<lapack::cplx> a = lapack::gather(A, n), b = lapack::gather(B, n), vr(size_t(n) * n), al(static_cast<size_t>(n)), be(static_cast<size_t>(n));
    int info = 0, lwork = -1, one = 1;
    lapack::cplx wq, vl;
    std::vector<double> rwork(static_cast<size_t>(8 * n));
    lapack::zggev()("N", "V", &n, a.data(), &n, b.data(), &n, al.data(), be.data(), &vl, &one, vr.data(), &n, &wq, &lwork, rwork.data(), &info, 1,
                    1);
    lwork = int(wq.real()) + 1;
    std::vector<lapack::cplx> work(static_cast<size_t>(lwork));
    lapack::zggev()("N", "V", &n, a.data(), &n, b.data(), &n, al.data(), be.data(), &vl, &one, vr.data(), &n, work.data(), &lwork,
                    rwork.data(), &info, 1, 1);
    LVARRAY_ERROR_IF(info != 0, "zggev info " << info);
    for (int i = 0; i < n; ++i) {
      alpha[i] = al[size_t(i)];
      beta[i] = be[size_t(i)];
    }
    lapack::scatter(vr, VR, n);
  }
}

}  // namespace dense
}  // namespace LvArray
