// LAPACKE_dgetrf and LAPACKE_dgetrs on the engine (FP64, LAPACK's partial
// pivoting and ipiv convention), so that a program reaching LAPACK through
// LAPACKE -- the reference's il::LU, il/linear_algebra/dense/factorization/
// LU.h:79-120 -- runs its factorisation and solves on the GPU when linked
// with this library ahead of OpenBLAS.  Column-major, square, trans 'N'
// only; anything else returns LAPACK's "illegal argument" code.  When the
// engine cannot run (no GPU, out of memory) the calls print the engine's
// message and return LAPACK_WORK_MEMORY_ERROR: there is no CPU fallback.
//
//   HFPX_LAPACKE_DEVICE   GPU to use (default 0)
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../../include/hfpx_engine.h"
#include "compat/OpenBLAS/lapacke.h"

namespace {

hfpx_ctx* ctx() {
  static hfpx_ctx* c = [] {
    const char* e = std::getenv("HFPX_LAPACKE_DEVICE");
    hfpx_ctx* p = nullptr;
    if (hfpx_ctx_create(e ? std::atoi(e) : 0, &p) != HFPX_OK) {
      std::fprintf(stderr, "hfpx lapacke: no engine context\n");
      return static_cast<hfpx_ctx*>(nullptr);
    }
    return p;
  }();
  return c;
}

lapack_int fail(const char* what) {
  std::fprintf(stderr, "hfpx lapacke: %s: %s\n", what, ctx() ? hfpx_ctx_last_error(ctx()) : "no context");
  return LAPACK_WORK_MEMORY_ERROR;
}

}  // namespace

extern "C" lapack_int LAPACKE_dgetrf(int layout, lapack_int m, lapack_int n, double* a, lapack_int lda,
                                     lapack_int* ipiv) {
  if (layout != LAPACK_COL_MAJOR) return -1;
  if (m < 0) return -2;
  if (n != m) return -3;  // square matrices only
  if (lda < (m > 1 ? m : 1)) return -5;
  if (n == 0) return 0;
  hfpx_ctx* c = ctx();
  if (!c) return LAPACK_WORK_MEMORY_ERROR;
  hfpx_matrix* mat = nullptr;
  if (hfpx_matrix_upload(c, a, n, lda, &mat) != HFPX_OK) return fail("upload");
  int64_t info = 0;
  const int rc = hfpx_lu_factor(c, mat, HFPX_LU_FP64, &info);
  if (rc != HFPX_OK && rc != HFPX_ERR_SINGULAR) {
    hfpx_matrix_destroy(mat);
    return fail("factorisation");
  }
  std::vector<int32_t> p(n);
  if (hfpx_matrix_download(c, mat, a, lda) != HFPX_OK || hfpx_matrix_pivots(c, mat, p.data()) != HFPX_OK) {
    hfpx_matrix_destroy(mat);
    return fail("download");
  }
  hfpx_matrix_destroy(mat);
  for (lapack_int i = 0; i < n; ++i) ipiv[i] = p[i] + 1;
  return (lapack_int)info;  // 0, or the 1-based column of the first zero pivot
}

extern "C" lapack_int LAPACKE_dgetrs(int layout, char trans, lapack_int n, lapack_int nrhs, const double* a,
                                     lapack_int lda, const lapack_int* ipiv, double* b, lapack_int ldb) {
  if (layout != LAPACK_COL_MAJOR) return -1;
  if (trans != 'N' && trans != 'n') return -2;
  if (n < 0) return -3;
  if (nrhs < 0) return -4;
  if (lda < (n > 1 ? n : 1)) return -6;
  if (ldb < (n > 1 ? n : 1)) return -9;
  if (n == 0 || nrhs == 0) return 0;
  hfpx_ctx* c = ctx();
  if (!c) return LAPACK_WORK_MEMORY_ERROR;
  std::vector<int32_t> p(n);
  for (lapack_int i = 0; i < n; ++i) p[i] = ipiv[i] - 1;
  hfpx_matrix* mat = nullptr;
  if (hfpx_matrix_upload_lu(c, a, n, lda, p.data(), &mat) != HFPX_OK) return fail("upload of the factors");
  hfpx_solve_info si{};
  const int rc = hfpx_lu_solve(c, mat, b, nrhs, ldb, 0.0, 0, &si);
  hfpx_matrix_destroy(mat);
  return rc == HFPX_OK ? 0 : fail("solve");
}

// dgesv = dgetrf + dgetrs on one device copy of A (il::linearSolve,
// il/linear_algebra/dense/factorization/linearSolve.h:28-76).  Row-major
// input is transposed on the host, as LAPACKE's own row-major path does, so A
// and B come back in the caller's layout.  On a zero pivot the factors and
// ipiv are returned with info > 0 and B is left as it was.
extern "C" lapack_int LAPACKE_dgesv(int layout, lapack_int n, lapack_int nrhs, double* a, lapack_int lda,
                                    lapack_int* ipiv, double* b, lapack_int ldb) {
  const bool row = layout == LAPACK_ROW_MAJOR;
  if (!row && layout != LAPACK_COL_MAJOR) return -1;
  if (n < 0) return -2;
  if (nrhs < 0) return -3;
  if (lda < (n > 1 ? n : 1)) return -5;
  if (ldb < (row ? (nrhs > 1 ? nrhs : 1) : (n > 1 ? n : 1))) return -8;
  if (n == 0) return 0;
  hfpx_ctx* c = ctx();
  if (!c) return LAPACK_WORK_MEMORY_ERROR;
  // column-major copies: A as an n x n, B as an n x nrhs
  std::vector<double> at, bt;
  const double* acol = a;
  lapack_int ldac = lda;
  if (row) {
    at.resize((size_t)n * n);
    for (lapack_int i = 0; i < n; ++i)
      for (lapack_int j = 0; j < n; ++j) at[(size_t)i + (size_t)n * j] = a[(size_t)i * lda + j];
    acol = at.data();
    ldac = n;
  }
  hfpx_matrix* mat = nullptr;
  if (hfpx_matrix_upload(c, acol, n, ldac, &mat) != HFPX_OK) return fail("upload");
  int64_t info = 0;
  int rc = hfpx_lu_factor(c, mat, HFPX_LU_FP64, &info);
  if (rc != HFPX_OK && rc != HFPX_ERR_SINGULAR) {
    hfpx_matrix_destroy(mat);
    return fail("factorisation");
  }
  if (info == 0 && nrhs > 0) {
    double* bcol = b;
    lapack_int ldbc = ldb;
    if (row) {
      bt.resize((size_t)n * nrhs);
      for (lapack_int i = 0; i < n; ++i)
        for (lapack_int j = 0; j < nrhs; ++j) bt[(size_t)i + (size_t)n * j] = b[(size_t)i * ldb + j];
      bcol = bt.data();
      ldbc = n;
    }
    hfpx_solve_info si{};
    if (hfpx_lu_solve(c, mat, bcol, nrhs, ldbc, 0.0, 0, &si) != HFPX_OK) {
      hfpx_matrix_destroy(mat);
      return fail("solve");
    }
    if (row)
      for (lapack_int i = 0; i < n; ++i)
        for (lapack_int j = 0; j < nrhs; ++j) b[(size_t)i * ldb + j] = bt[(size_t)i + (size_t)n * j];
  }
  std::vector<int32_t> p(n);
  rc = hfpx_matrix_download(c, mat, row ? at.data() : a, ldac);
  if (rc == HFPX_OK) rc = hfpx_matrix_pivots(c, mat, p.data());
  hfpx_matrix_destroy(mat);
  if (rc != HFPX_OK) return fail("download");
  if (row)
    for (lapack_int i = 0; i < n; ++i)
      for (lapack_int j = 0; j < n; ++j) a[(size_t)i * lda + j] = at[(size_t)i + (size_t)n * j];
  for (lapack_int i = 0; i < n; ++i) ipiv[i] = p[i] + 1;
  return (lapack_int)info;
}
