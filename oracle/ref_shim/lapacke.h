// Test infrastructure only: maps the LAPACKE names the reference engine calls onto numpy's
// bundled ILP64 OpenBLAS (64-bit lapack_int), for the oracle/_ref build of the reference.
#pragma once
#include <cstdint>

typedef std::int64_t lapack_int;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

extern "C" {
lapack_int scipy_LAPACKE_dstevd64_(int layout, char jobz, lapack_int n, double* d, double* e, double* z,
                                   lapack_int ldz);
lapack_int scipy_LAPACKE_dstevx64_(int layout, char jobz, char range, lapack_int n, double* d, double* e, double vl,
                                   double vu, lapack_int il, lapack_int iu, double abstol, lapack_int* m, double* w,
                                   double* z, lapack_int ldz, lapack_int* ifail);
lapack_int scipy_LAPACKE_dsyevd64_(int layout, char jobz, char uplo, lapack_int n, double* a, lapack_int lda,
                                   double* w);
}

inline lapack_int LAPACKE_dstevd(int layout, char jobz, lapack_int n, double* d, double* e, double* z,
                                 lapack_int ldz) {
    return scipy_LAPACKE_dstevd64_(layout, jobz, n, d, e, z, ldz);
}
inline lapack_int LAPACKE_dstevx(int layout, char jobz, char range, lapack_int n, double* d, double* e, double vl,
                                 double vu, lapack_int il, lapack_int iu, double abstol, lapack_int* m, double* w,
                                 double* z, lapack_int ldz, lapack_int* ifail) {
    return scipy_LAPACKE_dstevx64_(layout, jobz, range, n, d, e, vl, vu, il, iu, abstol, m, w, z, ldz, ifail);
}
inline lapack_int LAPACKE_dsyevd(int layout, char jobz, char uplo, lapack_int n, double* a, lapack_int lda,
                                 double* w) {
    return scipy_LAPACKE_dsyevd64_(layout, jobz, uplo, n, a, lda, w);
}
