/* The LAPACKE declarations that code reaching LAPACK through
 * <OpenBLAS/lapacke.h> compiles against -- the reference's il::LU
 * (il/linear_algebra/dense/factorization/LU.h) -- for linking with
 * libhfpx_lapacke.so, which implements LAPACKE_dgetrf, LAPACKE_dgetrs and
 * LAPACKE_dgesv on the engine.  LP64: lapack_int is a 32-bit int, as in the
 * reference's OpenBLAS builds.  dgetri, dgecon, dgbsv and dgtsv are declared
 * so that the il/ headers (LU.h, linearSolve.h) compile; a program that calls
 * them links them from a LAPACK library. */
#ifndef HFPX_COMPAT_LAPACKE_H
#define HFPX_COMPAT_LAPACKE_H

#ifndef lapack_int
#define lapack_int int
#endif

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
#define LAPACK_WORK_MEMORY_ERROR -1010

#ifdef __cplusplus
extern "C" {
#endif

lapack_int LAPACKE_dgetrf(int matrix_layout, lapack_int m, lapack_int n, double *a, lapack_int lda,
                          lapack_int *ipiv);
lapack_int LAPACKE_dgetrs(int matrix_layout, char trans, lapack_int n, lapack_int nrhs, const double *a,
                          lapack_int lda, const lapack_int *ipiv, double *b, lapack_int ldb);
lapack_int LAPACKE_dgetri(int matrix_layout, lapack_int n, double *a, lapack_int lda, const lapack_int *ipiv);
lapack_int LAPACKE_dgecon(int matrix_layout, char norm, lapack_int n, const double *a, lapack_int lda,
                          double anorm, double *rcond);
lapack_int LAPACKE_dgesv(int matrix_layout, lapack_int n, lapack_int nrhs, double *a, lapack_int lda,
                         lapack_int *ipiv, double *b, lapack_int ldb);
lapack_int LAPACKE_dgbsv(int matrix_layout, lapack_int n, lapack_int kl, lapack_int ku, lapack_int nrhs,
                         double *ab, lapack_int ldab, lapack_int *ipiv, double *b, lapack_int ldb);
lapack_int LAPACKE_dgtsv(int matrix_layout, lapack_int n, lapack_int nrhs, double *dl, double *d, double *du,
                         double *b, lapack_int ldb);

#ifdef __cplusplus
}
#endif

#endif
