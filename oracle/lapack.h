// Test infrastructure only (CPU oracle).  LAPACK/BLAS entry points of the
// OpenBLAS build that scipy bundles (LP64, symbols prefixed "scipy_").  The
// reference links MKL for the same routines (sim-trhepd-rheed/src/Makefile:7).
#pragma once
#include <complex>
#include <cstddef>

extern "C" {
using zc = std::complex<double>;
void scipy_zgemm_(const char* ta, const char* tb, const int* m, const int* n, const int* k,
                  const zc* alpha, const zc* a, const int* lda, const zc* b, const int* ldb,
                  const zc* beta, zc* c, const int* ldc, size_t, size_t);
void scipy_zgetrf_(const int* m, const int* n, zc* a, const int* lda, int* ipiv, int* info);
void scipy_zgetrs_(const char* tr, const int* n, const int* nrhs, const zc* a, const int* lda,
                   const int* ipiv, zc* b, const int* ldb, int* info, size_t);
void scipy_ztrsm_(const char* side, const char* uplo, const char* ta, const char* diag,
                  const int* m, const int* n, const zc* alpha, const zc* a, const int* lda, zc* b,
                  const int* ldb, size_t, size_t, size_t, size_t);
void scipy_zgeev_(const char* jobvl, const char* jobvr, const int* n, zc* a, const int* lda,
                  zc* w, zc* vl, const int* ldvl, zc* vr, const int* ldvr, zc* work,
                  const int* lwork, double* rwork, int* info, size_t, size_t);
void scipy_zherk_(const char* uplo, const char* tr, const int* n, const int* k,
                  const double* alpha, const zc* a, const int* lda, const double* beta, zc* c,
                  const int* ldc, size_t, size_t);
void scipy_zpotrf_(const char* uplo, const int* n, zc* a, const int* lda, int* info, size_t);
void scipy_openblas_set_num_threads(int);
}

namespace oracle {
using cplx = std::complex<double>;
// C = alpha*op(A)*op(B) + beta*C, column-major
inline void zgemm(char ta, char tb, int m, int n, int k, cplx alpha, const cplx* a, int lda,
                  const cplx* b, int ldb, cplx beta, cplx* c, int ldc) {
  scipy_zgemm_(&ta, &tb, &m, &n, &k, &alpha, a, &lda, b, &ldb, &beta, c, &ldc, 1, 1);
}
inline int zgetrf(int m, int n, cplx* a, int lda, int* ipiv) {
  int info = 0;
  scipy_zgetrf_(&m, &n, a, &lda, ipiv, &info);
  return info;
}
inline int zgetrs(char tr, int n, int nrhs, const cplx* a, int lda, const int* ipiv, cplx* b,
                  int ldb) {
  int info = 0;
  scipy_zgetrs_(&tr, &n, &nrhs, a, &lda, ipiv, b, &ldb, &info, 1);
  return info;
}
inline void ztrsm(char side, char uplo, char ta, char diag, int m, int n, cplx alpha,
                  const cplx* a, int lda, cplx* b, int ldb) {
  scipy_ztrsm_(&side, &uplo, &ta, &diag, &m, &n, &alpha, a, &lda, b, &ldb, 1, 1, 1, 1);
}
// C = alpha*op(A)^H op(A) + beta*C (Hermitian rank-k update), column-major
inline void zherk(char uplo, char tr, int n, int k, double alpha, const cplx* a, int lda,
                  double beta, cplx* c, int ldc) {
  scipy_zherk_(&uplo, &tr, &n, &k, &alpha, a, &lda, &beta, c, &ldc, 1, 1);
}
inline int zpotrf(char uplo, int n, cplx* a, int lda) {
  int info = 0;
  scipy_zpotrf_(&uplo, &n, a, &lda, &info, 1);
  return info;
}
}  // namespace oracle
