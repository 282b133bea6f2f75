/*
 * cblas.h -- TEST INFRASTRUCTURE ONLY.
 *
 * The subset of the CBLAS interface the reference's BLAS apps call
 * (testSuite/matrixMultiplyBlas/source/code/src/matrixMultiplyBlas.cpp:44-48,
 * testSuite/luDecomposition/source/code/src/luDecomposition.cpp:48-62), so
 * those files compile unchanged here.  commonAPI.h includes <cblas.h> inside
 * extern "C" when ENABLE_BLAS is defined.  The enumerator values are the
 * CBLAS standard's (the BLAS library on the other side of the call reads
 * them).  oracle/ref/cblas_shim.c implements the functions on the OpenBLAS
 * that numpy bundles (64-bit integer interface).
 */
#ifndef PMB_ORACLE_CBLAS_H
#define PMB_ORACLE_CBLAS_H

enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 };
enum CBLAS_DIAG { CblasNonUnit = 131, CblasUnit = 132 };
enum CBLAS_SIDE { CblasLeft = 141, CblasRight = 142 };

void cblas_sgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, int m, int n, int k,
                 float alpha, const float* a, int lda, const float* b, int ldb, float beta, float* c, int ldc);
void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, int m, int n, int k,
                 double alpha, const double* a, int lda, const double* b, int ldb, double beta, double* c, int ldc);
void cblas_strsm(enum CBLAS_ORDER order, enum CBLAS_SIDE side, enum CBLAS_UPLO uplo, enum CBLAS_TRANSPOSE ta,
                 enum CBLAS_DIAG diag, int m, int n, float alpha, const float* a, int lda, float* b, int ldb);
void cblas_dtrsm(enum CBLAS_ORDER order, enum CBLAS_SIDE side, enum CBLAS_UPLO uplo, enum CBLAS_TRANSPOSE ta,
                 enum CBLAS_DIAG diag, int m, int n, double alpha, const double* a, int lda, double* b, int ldb);
void cblas_strmm(enum CBLAS_ORDER order, enum CBLAS_SIDE side, enum CBLAS_UPLO uplo, enum CBLAS_TRANSPOSE ta,
                 enum CBLAS_DIAG diag, int m, int n, float alpha, const float* a, int lda, float* b, int ldb);
void cblas_dtrmm(enum CBLAS_ORDER order, enum CBLAS_SIDE side, enum CBLAS_UPLO uplo, enum CBLAS_TRANSPOSE ta,
                 enum CBLAS_DIAG diag, int m, int n, double alpha, const double* a, int lda, double* b, int ldb);
void cblas_sger(enum CBLAS_ORDER order, int m, int n, float alpha, const float* x, int incx, const float* y, int incy,
                float* a, int lda);
void cblas_dger(enum CBLAS_ORDER order, int m, int n, double alpha, const double* x, int incx, const double* y,
                int incy, double* a, int lda);
void cblas_sscal(int n, float alpha, float* x, int incx);
void cblas_dscal(int n, double alpha, double* x, int incx);
void cblas_saxpy(int n, float alpha, const float* x, int incx, float* y, int incy);
void cblas_daxpy(int n, double alpha, const double* x, int incx, double* y, int incy);

#endif
