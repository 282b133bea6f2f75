/*
 * cblas_shim.c -- TEST INFRASTRUCTURE ONLY.
 *
 * The CBLAS functions of oracle/ref/cblas/cblas.h, each widening its integer
 * arguments and calling the same routine of the OpenBLAS that numpy bundles
 * (exported with a scipy_ prefix and a 64_ suffix, 64-bit integers).  The
 * reference names no BLAS version (ATLAS is its Makefile default,
 * testSuite/common/build/linux/Makefile.common:63-81); any conforming BLAS
 * computes the same products up to rounding order.
 */
#include "cblas.h"

typedef long i64;

#define EXT(name) scipy_cblas_##name##64_
extern void EXT(sgemm)(int, int, int, i64, i64, i64, float, const float*, i64, const float*, i64, float, float*, i64);
extern void EXT(dgemm)(int, int, int, i64, i64, i64, double, const double*, i64, const double*, i64, double, double*,
                       i64);
extern void EXT(strsm)(int, int, int, int, int, i64, i64, float, const float*, i64, float*, i64);
extern void EXT(dtrsm)(int, int, int, int, int, i64, i64, double, const double*, i64, double*, i64);
extern void EXT(strmm)(int, int, int, int, int, i64, i64, float, const float*, i64, float*, i64);
extern void EXT(dtrmm)(int, int, int, int, int, i64, i64, double, const double*, i64, double*, i64);
extern void EXT(sger)(int, i64, i64, float, const float*, i64, const float*, i64, float*, i64);
extern void EXT(dger)(int, i64, i64, double, const double*, i64, const double*, i64, double*, i64);
extern void EXT(sscal)(i64, float, float*, i64);
extern void EXT(dscal)(i64, double, double*, i64);
extern void EXT(saxpy)(i64, float, const float*, i64, float*, i64);
extern void EXT(daxpy)(i64, double, const double*, i64, double*, i64);

void cblas_sgemm(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, int m, int n, int k, float al,
                 const float* a, int lda, const float* b, int ldb, float be, float* c, int ldc) {
    EXT(sgemm)(o, ta, tb, m, n, k, al, a, lda, b, ldb, be, c, ldc);
}
void cblas_dgemm(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, int m, int n, int k, double al,
                 const double* a, int lda, const double* b, int ldb, double be, double* c, int ldc) {
    EXT(dgemm)(o, ta, tb, m, n, k, al, a, lda, b, ldb, be, c, ldc);
}
void cblas_strsm(enum CBLAS_ORDER o, enum CBLAS_SIDE s, enum CBLAS_UPLO u, enum CBLAS_TRANSPOSE t, enum CBLAS_DIAG d,
                 int m, int n, float al, const float* a, int lda, float* b, int ldb) {
    EXT(strsm)(o, s, u, t, d, m, n, al, a, lda, b, ldb);
}
void cblas_dtrsm(enum CBLAS_ORDER o, enum CBLAS_SIDE s, enum CBLAS_UPLO u, enum CBLAS_TRANSPOSE t, enum CBLAS_DIAG d,
                 int m, int n, double al, const double* a, int lda, double* b, int ldb) {
    EXT(dtrsm)(o, s, u, t, d, m, n, al, a, lda, b, ldb);
}
void cblas_strmm(enum CBLAS_ORDER o, enum CBLAS_SIDE s, enum CBLAS_UPLO u, enum CBLAS_TRANSPOSE t, enum CBLAS_DIAG d,
                 int m, int n, float al, const float* a, int lda, float* b, int ldb) {
    EXT(strmm)(o, s, u, t, d, m, n, al, a, lda, b, ldb);
}
void cblas_dtrmm(enum CBLAS_ORDER o, enum CBLAS_SIDE s, enum CBLAS_UPLO u, enum CBLAS_TRANSPOSE t, enum CBLAS_DIAG d,
                 int m, int n, double al, const double* a, int lda, double* b, int ldb) {
    EXT(dtrmm)(o, s, u, t, d, m, n, al, a, lda, b, ldb);
}
void cblas_sger(enum CBLAS_ORDER o, int m, int n, float al, const float* x, int incx, const float* y, int incy,
                float* a, int lda) {
    EXT(sger)(o, m, n, al, x, incx, y, incy, a, lda);
}
void cblas_dger(enum CBLAS_ORDER o, int m, int n, double al, const double* x, int incx, const double* y, int incy,
                double* a, int lda) {
    EXT(dger)(o, m, n, al, x, incx, y, incy, a, lda);
}
void cblas_sscal(int n, float al, float* x, int incx) { EXT(sscal)(n, al, x, incx); }
void cblas_dscal(int n, double al, double* x, int incx) { EXT(dscal)(n, al, x, incx); }
void cblas_saxpy(int n, float al, const float* x, int incx, float* y, int incy) { EXT(saxpy)(n, al, x, incx, y, incy); }
void cblas_daxpy(int n, double al, const double* x, int incx, double* y, int incy) {
    EXT(daxpy)(n, al, x, incx, y, incy);
}
