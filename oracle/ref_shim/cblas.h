// Test infrastructure only: maps the CBLAS names the reference engine calls onto the ILP64
// OpenBLAS that numpy bundles (scipy_openblas64_), so the reference's own CPU code compiles
// unmodified into oracle/_ref. Only the entry points the reference headers use are declared.
#pragma once
#include <cstdint>

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef CBLAS_LAYOUT CBLAS_ORDER;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;

extern "C" {
double scipy_cblas_dznrm264_(std::int64_t n, const void* x, std::int64_t incx);
void scipy_cblas_zscal64_(std::int64_t n, const void* alpha, void* x, std::int64_t incx);
void scipy_cblas_zaxpy64_(std::int64_t n, const void* alpha, const void* x, std::int64_t incx, void* y,
                          std::int64_t incy);
void scipy_cblas_zdotc_sub64_(std::int64_t n, const void* x, std::int64_t incx, const void* y, std::int64_t incy,
                              void* ret);
void scipy_cblas_zgemm64_(CBLAS_ORDER, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, std::int64_t m, std::int64_t n,
                          std::int64_t k, const void* alpha, const void* A, std::int64_t lda, const void* B,
                          std::int64_t ldb, const void* beta, void* C, std::int64_t ldc);
void scipy_cblas_dgemm64_(CBLAS_ORDER, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, std::int64_t m, std::int64_t n,
                          std::int64_t k, double alpha, const double* A, std::int64_t lda, const double* B,
                          std::int64_t ldb, double beta, double* C, std::int64_t ldc);
}

inline double cblas_dznrm2(std::int64_t n, const void* x, std::int64_t incx) {
    return scipy_cblas_dznrm264_(n, x, incx);
}
inline void cblas_zscal(std::int64_t n, const void* a, void* x, std::int64_t incx) {
    scipy_cblas_zscal64_(n, a, x, incx);
}
inline void cblas_zaxpy(std::int64_t n, const void* a, const void* x, std::int64_t incx, void* y, std::int64_t incy) {
    scipy_cblas_zaxpy64_(n, a, x, incx, y, incy);
}
inline void cblas_zdotc_sub(std::int64_t n, const void* x, std::int64_t incx, const void* y, std::int64_t incy,
                            void* r) {
    scipy_cblas_zdotc_sub64_(n, x, incx, y, incy, r);
}
inline void cblas_zgemm(CBLAS_ORDER o, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, std::int64_t m, std::int64_t n,
                        std::int64_t k, const void* alpha, const void* A, std::int64_t lda, const void* B,
                        std::int64_t ldb, const void* beta, void* C, std::int64_t ldc) {
    scipy_cblas_zgemm64_(o, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}
inline void cblas_dgemm(CBLAS_ORDER o, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, std::int64_t m, std::int64_t n,
                        std::int64_t k, double alpha, const double* A, std::int64_t lda, const double* B,
                        std::int64_t ldb, double beta, double* C, std::int64_t ldc) {
    scipy_cblas_dgemm64_(o, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}
