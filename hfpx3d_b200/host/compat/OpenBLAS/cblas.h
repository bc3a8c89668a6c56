/* The CBLAS declarations that the reference's il/ headers compile against
 * under -DIL_OPENBLAS -DIL_BLAS (il/linear_algebra/dense/blas/blas.h:26-29,
 * dot.h), with the enumerator values of the CBLAS standard.  Declarations
 * only: a program that calls one of these links it from a BLAS library.  The
 * reference's driver (main.cpp with the engine's system_assembly and
 * LAPACKE libraries) calls none of them. */
#ifndef HFPX_COMPAT_CBLAS_H
#define HFPX_COMPAT_CBLAS_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef enum CBLAS_TRANSPOSE {
  CblasNoTrans = 111,
  CblasTrans = 112,
  CblasConjTrans = 113,
  CblasConjNoTrans = 114
} CBLAS_TRANSPOSE;
typedef enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;
typedef enum CBLAS_DIAG { CblasNonUnit = 131, CblasUnit = 132 } CBLAS_DIAG;
typedef enum CBLAS_SIDE { CblasLeft = 141, CblasRight = 142 } CBLAS_SIDE;
typedef CBLAS_ORDER CBLAS_LAYOUT;

void cblas_daxpy(int n, double alpha, const double *x, int incx, double *y, int incy);
void cblas_saxpby(int n, float alpha, const float *x, int incx, float beta, float *y, int incy);
void cblas_daxpby(int n, double alpha, const double *x, int incx, double beta, double *y, int incy);
void cblas_sgemv(CBLAS_ORDER order, CBLAS_TRANSPOSE trans, int m, int n, float alpha, const float *a, int lda,
                 const float *x, int incx, float beta, float *y, int incy);
void cblas_dgemv(CBLAS_ORDER order, CBLAS_TRANSPOSE trans, int m, int n, double alpha, const double *a, int lda,
                 const double *x, int incx, double beta, double *y, int incy);
void cblas_sgemm(CBLAS_ORDER order, CBLAS_TRANSPOSE transa, CBLAS_TRANSPOSE transb, int m, int n, int k,
                 float alpha, const float *a, int lda, const float *b, int ldb, float beta, float *c, int ldc);
void cblas_dgemm(CBLAS_ORDER order, CBLAS_TRANSPOSE transa, CBLAS_TRANSPOSE transb, int m, int n, int k,
                 double alpha, const double *a, int lda, const double *b, int ldb, double beta, double *c, int ldc);
void cblas_dsymm(CBLAS_ORDER order, CBLAS_SIDE side, CBLAS_UPLO uplo, int m, int n, double alpha, const double *a,
                 int lda, const double *b, int ldb, double beta, double *c, int ldc);
double cblas_ddot(int n, const double *x, int incx, const double *y, int incy);

#ifdef __cplusplus
}
#endif

#endif
