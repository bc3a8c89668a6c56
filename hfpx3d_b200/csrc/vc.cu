// Volume-control truncation on the device: the bordered system of a subset
// of the DoF, and solves of it with the factors of the full system.
//
// mod_3dbem_system_vc (src/Solvers/system_assembly.cpp:560-629) builds, from
// the bordered VC matrix (make_3dbem_matrix_vc, :458-557) and a "truncated"
// DoF handle (some DoF fixed, e.g. by contact or cohesion in the reference's
// Development/c_f_iteration.cpp), the (used + 1)^2 matrix of the kept DoF
// plus the volume row and pressure column.  As written it requires the
// matrix to be orig_ndof square and then reads row and column full_ndof of
// it, one past the end; here the border is the bordered matrix's own last
// row and column.
//   hfpx_matrix_truncate: that gather, on the device (no host round trip of
//     the matrix);
//   hfpx_lu_solve_fixed: the truncated system solved with the factors of the
//     full one, no refactorisation: with F the k dropped DoF and E_F their
//     unit columns, x = y + X mu where y = A^-1 b0 (b0 = b with the F
//     entries zeroed), X = A^-1 E_F, and mu solves the k x k capacitance
//     system (E_F^T X) mu = -E_F^T y, so that x_F = 0 and the kept rows of
//     A x equal b.  Cost: k + 1 solves with the existing factors and a k x k
//     dense solve, instead of a new factorisation.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <vector>
#include "engine_internal.h"

namespace hfpx {
namespace {

__global__ void truncate_kernel(const double* __restrict__ A, int64_t lda, const int64_t* __restrict__ map, int64_t m,
                                double* __restrict__ B, int64_t ldb) {
  const int64_t j = blockIdx.y;
  const int64_t src_col = map[j];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
    B[i + ldb * j] = A[map[i] + lda * src_col];
}

// X (n x k, zero) gets X[fixed[i], i] = 1
__global__ void unit_columns_kernel(const int64_t* __restrict__ fixed, int64_t k, double* __restrict__ X, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < k) X[fixed[i] + n * i] = 1.0;
}

// C[i + k j] = X[fixed[i] + n j]; yf[i] = y[fixed[i]]
__global__ void gather_fixed_kernel(const int64_t* __restrict__ fixed, int64_t k, const double* __restrict__ X,
                                    const double* __restrict__ y, int64_t n, double* __restrict__ C,
                                    double* __restrict__ yf) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < k * k) {
    const int64_t i = t % k, j = t / k;
    C[t] = X[fixed[i] + n * j];
  }
  if (t < k) yf[t] = y[fixed[t]];
}

__global__ void zero_fixed_kernel(const int64_t* __restrict__ fixed, int64_t k, double* __restrict__ v) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < k) v[fixed[i]] = 0.0;
}

// dense LU with partial pivoting of the k x k capacitance matrix (column
// major), solving C mu = r in place of r; false when C is singular
bool host_solve(std::vector<double>& C, std::vector<double>& r, int64_t k) {
  for (int64_t c = 0; c < k; ++c) {
    int64_t p = c;
    for (int64_t i = c + 1; i < k; ++i)
      if (std::fabs(C[i + k * c]) > std::fabs(C[p + k * c])) p = i;
    if (C[p + k * c] == 0.0) return false;
    if (p != c) {
      for (int64_t j = 0; j < k; ++j) std::swap(C[c + k * j], C[p + k * j]);
      std::swap(r[c], r[p]);
    }
    for (int64_t i = c + 1; i < k; ++i) {
      const double l = C[i + k * c] / C[c + k * c];
      if (l == 0.0) continue;
      for (int64_t j = c + 1; j < k; ++j) C[i + k * j] -= l * C[c + k * j];
      r[i] -= l * r[c];
    }
  }
  for (int64_t i = k - 1; i >= 0; --i) {
    double s = r[i];
    for (int64_t j = i + 1; j < k; ++j) s -= C[i + k * j] * r[j];
    r[i] = s / C[i + k * i];
  }
  return true;
}

struct Dev {
  void* p = nullptr;
  ~Dev() {
    if (p) cudaFree(p);
  }
};

}  // namespace
}  // namespace hfpx

using namespace hfpx;

extern "C" {

int hfpx_matrix_truncate(hfpx_ctx* c, const hfpx_matrix* m, const int64_t* keep, int64_t n_keep, int keep_border,
                         hfpx_matrix** out) {
  if (!c || !out) return HFPX_ERR_ARG;
  *out = nullptr;
  if (!m || !keep || n_keep < 1) return set_error(c, HFPX_ERR_ARG, "bad truncation arguments");
  if (m->factored == 1) return set_error(c, HFPX_ERR_STATE, "the matrix holds FP64 LU factors, not the operator");
  if (m->op_mixed) return set_error(c, HFPX_ERR_STATE, "truncation needs the FP64 matrix");
  const int64_t n_dd = keep_border ? m->n - 1 : m->n;
  if (n_dd < 1 || n_keep > n_dd) return set_error(c, HFPX_ERR_ARG, "more kept DoF than the matrix has");
  {
    std::vector<char> seen((size_t)n_dd, 0);
    for (int64_t i = 0; i < n_keep; ++i) {
      if (keep[i] < 0 || keep[i] >= n_dd || seen[(size_t)keep[i]])
        return set_error(c, HFPX_ERR_ARG, "kept DoF must be distinct indices of the DD unknowns");
      seen[(size_t)keep[i]] = 1;
    }
  }
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  const int64_t mn = n_keep + (keep_border ? 1 : 0);
  std::vector<int64_t> map(keep, keep + n_keep);
  if (keep_border) map.push_back(m->n - 1);
  Dev dmap;
  int rc = check_cuda(c, cudaMalloc(&dmap.p, sizeof(int64_t) * mn), "map");
  if (!rc)
    rc = check_cuda(c, cudaMemcpyAsync(dmap.p, map.data(), sizeof(int64_t) * mn, cudaMemcpyHostToDevice, c->stream),
                    "map");
  hfpx_matrix* t = nullptr;
  if (!rc) {
    // a matrix of mn unknowns with the engine's layout (ld rounded to 32)
    t = new (std::nothrow) hfpx_matrix;
    if (!t) rc = set_error(c, HFPX_ERR_NOMEM, "matrix");
  }
  if (!rc) {
    t->n = mn;
    t->ld = (mn + 31) / 32 * 32;
    rc = check_cuda(c, cudaMalloc(&t->d_a, sizeof(double) * t->ld * mn), "truncated matrix");
    if (!rc) rc = check_cuda(c, cudaMalloc(&t->d_piv, sizeof(int32_t) * mn), "pivots");
  }
  if (!rc) {
    ++g_launches;
    const unsigned gx = (unsigned)std::min<int64_t>((mn + 255) / 256, 64);
    truncate_kernel<<<dim3(gx, (unsigned)mn), 256, 0, c->stream>>>(m->d_a, m->ld, (const int64_t*)dmap.p, mn, t->d_a,
                                                                    t->ld);
    rc = check_cuda(c, cudaGetLastError(), "truncation");
  }
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "truncation");
  if (rc) {
    hfpx_matrix_destroy(t);
    return rc;
  }
  *out = t;
  return HFPX_OK;
}

int hfpx_lu_solve_fixed(hfpx_ctx* c, const hfpx_matrix* m, const int64_t* fixed, int64_t k, double* b, double tol,
                        hfpx_solve_info* info) {
  if (!c) return HFPX_ERR_ARG;
  if (!m || !b || (k > 0 && !fixed) || k < 0) return set_error(c, HFPX_ERR_ARG, "bad arguments");
  if (!m->factored) return set_error(c, HFPX_ERR_STATE, "factor the matrix first (hfpx_lu_factor)");
  const int64_t n = m->n;
  if (k > 4096 || k >= n) return set_error(c, HFPX_ERR_ARG, "at most 4096 fixed DoF, fewer than the unknowns");
  {
    std::vector<char> seen((size_t)n, 0);
    for (int64_t i = 0; i < k; ++i) {
      if (fixed[i] < 0 || fixed[i] >= n) return set_error(c, HFPX_ERR_ARG, "fixed DoF out of range");
      if (seen[(size_t)fixed[i]]) return set_error(c, HFPX_ERR_ARG, "repeated fixed DoF");
      seen[(size_t)fixed[i]] = 1;
    }
  }
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  Dev dy, dX, dfix, dC;
  int rc = check_cuda(c, cudaMalloc(&dy.p, sizeof(double) * n), "rhs");
  if (!rc && k > 0) rc = check_cuda(c, cudaMalloc(&dX.p, sizeof(double) * n * k), "unit columns");
  if (!rc && k > 0) rc = check_cuda(c, cudaMalloc(&dfix.p, sizeof(int64_t) * k), "fixed");
  if (!rc && k > 0) rc = check_cuda(c, cudaMalloc(&dC.p, sizeof(double) * (k * k + k)), "capacitance");
  double* y = (double*)dy.p;
  double* X = (double*)dX.p;
  const int64_t* fx = (const int64_t*)dfix.p;
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(y, b, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream), "rhs");
  if (!rc && k > 0) {
    rc = check_cuda(c, cudaMemcpyAsync(dfix.p, fixed, sizeof(int64_t) * k, cudaMemcpyHostToDevice, c->stream), "fixed");
    if (!rc) rc = check_cuda(c, cudaMemsetAsync(X, 0, sizeof(double) * n * k, c->stream), "unit columns");
    if (!rc) {
      g_launches += 2;
      unit_columns_kernel<<<(unsigned)((k + 255) / 256), 256, 0, c->stream>>>(fx, k, X, n);
      zero_fixed_kernel<<<(unsigned)((k + 255) / 256), 256, 0, c->stream>>>(fx, k, y);
    }
    // X = A^-1 E_F with the existing factors
    if (!rc) rc = hfpx_lu_solve_device(c, m, X, k, n, tol, 50, nullptr);
  }
  hfpx_solve_info yi{};
  if (!rc) rc = hfpx_lu_solve_device(c, m, y, 1, n, tol, 50, &yi);  // y = A^-1 b0
  if (!rc && k > 0) {
    double* C = (double*)dC.p;
    ++g_launches;
    gather_fixed_kernel<<<(unsigned)((k * k + 255) / 256), 256, 0, c->stream>>>(fx, k, X, y, n, C, C + k * k);
    std::vector<double> hC((size_t)(k * k)), hr((size_t)k);
    rc = check_cuda(c, cudaMemcpyAsync(hC.data(), C, sizeof(double) * k * k, cudaMemcpyDeviceToHost, c->stream), "C");
    if (!rc) rc = check_cuda(c, cudaMemcpyAsync(hr.data(), C + k * k, sizeof(double) * k, cudaMemcpyDeviceToHost,
                                                c->stream), "y_F");
    if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "capacitance");
    if (!rc) {
      for (double& v : hr) v = -v;
      if (!host_solve(hC, hr, k)) rc = set_error(c, HFPX_ERR_SINGULAR, "the truncated system is singular");
    }
    // x = y + X mu, then exact zeros at F
    if (!rc) rc = check_cuda(c, cudaMemcpyAsync(C, hr.data(), sizeof(double) * k, cudaMemcpyHostToDevice, c->stream),
                             "mu");
    if (!rc) {
      cublasHandle_t h = static_cast<cublasHandle_t>(c->cublas);
      cublasSetPointerMode(h, CUBLAS_POINTER_MODE_HOST);
      const double one = 1.0;
      if (cublasDgemv(h, CUBLAS_OP_N, (int)n, (int)k, &one, X, (int)n, C, 1, &one, y, 1) != CUBLAS_STATUS_SUCCESS)
        rc = set_error(c, HFPX_ERR_CUDA, "x = y + X mu");
      ++g_launches;
      zero_fixed_kernel<<<(unsigned)((k + 255) / 256), 256, 0, c->stream>>>(fx, k, y);
    }
  }
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(b, y, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream), "x");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "solve");
  if (info) *info = yi;
  return rc;
}

}  // extern "C"
