// Learned near-field preconditioner: a graph network over element adjacency
// that predicts corrections to the Neumann blocks of precond.cu, trained on
// the GPU on meshes and matrices this engine generates.  No counterpart in
// the reference (which solves directly, il::LU at
// il/linear_algebra/dense/factorization/LU.h:79-120); the operator it
// preconditions is the one make_3dbem_matrix_s fills
// (src/Solvers/system_assembly.cpp:30-219).
//
// Graph: one node per element, one directed edge i -> j per neighbour i of
// element j (elements sharing a vertex; NearPattern).  Inputs, all in the
// frame of element j (rotation Q_j = 6 copies of its frame R_j, the frame
// make_el_r_tensor builds, element_utilities.cpp:62-87) and scaled by its
// size s_j = sqrt(2 area_j) and the shear modulus G, so that they do not
// depend on where the element sits or how large the crack is:
//   node j:  8 geometry features, then (G / s_j) Q_j D_j^-1 Q_j^T (324);
//   edge ij: 12 geometry features, then Q_j D_i^-1 A_ij Q_j^T (324);
// Network (4 message-passing layers, 64 wide):
//   h = relu(Xn Wn + bn), z = relu(Xe We + be)
//   per layer: m = relu([h_i, h_j, z_ij] Wm + bm), a_j = mean_i m_ij,
//              h_j += relu([h_j, a_j] Wu + bu)
//   outputs: edge ij  [h_i, h_j, z_ij] Woe + boe (324),
//            node j   h_j Won + bon (324)
// The outputs are the corrections (G / s_j) Q_j (M_ij - M^N_ij) Q_j^T of the
// blocks of column j, M^N the Neumann blocks.  Training regresses them on
// the same quantity for the exact local inverse (HFPX_PC_LOCAL_INVERSE):
// mean squared error over all entries.
//
// Precision: weights and activations are stored in BF16; every product
// accumulates in FP32; gradients, the Adam moments and the master weights
// are FP32.  All kernels here are the engine's own (no library GEMM).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <utility>
#include <random>
#include <string>
#include <vector>
#include "engine_internal.h"

namespace hfpx {
namespace gnn {

constexpr int kH = 64;            // hidden width
constexpr int kLayers = 4;
constexpr int kFN = 336;          // node input: 8 geometry + 324 + 4 zero
constexpr int kFE = 336;          // edge input: 12 geometry + 324
constexpr int kGeoN = 8, kGeoE = 12;
constexpr int kOut = 324;         // one 18 x 18 block

// parameter tensors: (rows, cols) of each weight, bias of length cols
struct Shape {
  int rows, cols;
};
constexpr int kTensors = 2 + 2 * kLayers + 2;
inline Shape tensor_shape(int t) {
  if (t == 0) return {kFN, kH};                              // Wn
  if (t == 1) return {kFE, kH};                              // We
  if (t < 2 + 2 * kLayers) return ((t - 2) % 2 == 0) ? Shape{3 * kH, kH} : Shape{2 * kH, kH};  // Wm, Wu
  if (t == 2 + 2 * kLayers) return {3 * kH, kOut};           // Woe
  return {kH, kOut};                                         // Won
}

}  // namespace gnn
}  // namespace hfpx

using namespace hfpx;
using namespace hfpx::gnn;

struct hfpx_gnn {
  int device = 0;
  int64_t n_params = 0;
  int64_t w_off[kTensors] = {}, b_off[kTensors] = {};
  float* d_w = nullptr;          // master FP32 parameters (weights, then bias, per tensor)
  __nv_bfloat16* d_wb = nullptr; // BF16 copy used by the products
  float* d_g = nullptr;          // gradients
  float* d_m = nullptr;          // Adam first moment
  float* d_v = nullptr;          // Adam second moment
  int64_t step = 0;
};

// A graph of one mesh: structure, inputs, optional targets, activations.
struct hfpx_gnn_graph {
  int64_t n_nodes = 0, n_edges = 0;
  std::shared_ptr<NearPattern> pat;   // the mesh's
  float* d_size = nullptr;        // s_j
  float* d_rot = nullptr;         // R_j (9, row-major: rows e1, e2, e3)
  double* d_dinv = nullptr;       // D_j^-1
  double* d_neu = nullptr;        // Neumann blocks (pattern order)
  __nv_bfloat16* xn = nullptr;    // n x kFN
  __nv_bfloat16* xe = nullptr;    // E x kFE
  float* tn = nullptr;            // n x 324 targets (null without)
  float* te = nullptr;            // E x 324
  // activations and their gradients
  __nv_bfloat16 *h[kLayers + 1] = {}, *z = nullptr, *cm[kLayers] = {}, *m[kLayers] = {}, *cu[kLayers] = {},
                *u[kLayers] = {}, *ce = nullptr;
  float *oe = nullptr, *on = nullptr;
  float *dh = nullptr, *dh2 = nullptr, *dz = nullptr, *dce = nullptr, *doe = nullptr, *don = nullptr, *dm = nullptr,
        *dcu = nullptr, *du = nullptr, *dagg = nullptr;
  float* part = nullptr;          // split-row partial sums of the weight gradients
  int64_t part_floats = 0;
  float* loss = nullptr;          // device loss accumulator (2 doubles worth)
  std::vector<void*> allocs;
};

namespace hfpx {
namespace gnn {

// ------------------------------------------------------------ products
// C[M x N] = act(A[M x K] B + bias), B[K x N] row-major (or, with TB_T, the
// transpose of a row-major N x K matrix), all accumulated in FP32; A and B
// are BF16 or FP32, C BF16 or FP32; beta = 1 adds the product to C.
constexpr int kTM = 64, kTN = 64, kTK = 16;

template <class T>
__device__ __forceinline__ float ld(const T* p) {
  if constexpr (sizeof(T) == 2)
    return __bfloat162float(*p);
  else
    return *p;
}
template <class T>
__device__ __forceinline__ void st(T* p, float v) {
  if constexpr (sizeof(T) == 2)
    *p = __float2bfloat16_rn(v);
  else
    *p = v;
}

template <class TA, class TB, class TC, bool TB_T>
__global__ void __launch_bounds__(256) gemm_kernel(int64_t M, int N, int K, const TA* __restrict__ A, int64_t lda,
                                                   const TB* __restrict__ B, int64_t ldb,
                                                   const float* __restrict__ bias, TC* __restrict__ C, int64_t ldc,
                                                   int relu, int beta) {
  __shared__ float sa[kTK][kTM + 4];
  __shared__ float sb[kTK][kTN + 4];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int64_t m0 = (int64_t)blockIdx.x * kTM;
  const int n0 = blockIdx.y * kTN;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += kTK) {
    for (int t = threadIdx.x; t < kTM * kTK; t += 256) {
      const int r = t / kTK, k = t % kTK;
      const int64_t gm = m0 + r;
      sa[k][r] = (gm < M && k0 + k < K) ? ld(A + gm * lda + k0 + k) : 0.f;
    }
    for (int t = threadIdx.x; t < kTK * kTN; t += 256) {
      const int k = t / kTN, c = t % kTN;
      const int gk = k0 + k, gn = n0 + c;
      float v = 0.f;
      if (gk < K && gn < N) v = TB_T ? ld(B + (int64_t)gn * ldb + gk) : ld(B + (int64_t)gk * ldb + gn);
      sb[k][c] = v;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kTK; ++k) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = sa[k][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = sb[k][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int64_t gm = m0 + ty * 4 + i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gn = n0 + tx * 4 + j;
      if (gn >= N) continue;
      float v = acc[i][j];
      if (bias) v += bias[gn];
      TC* p = C + gm * ldc + gn;
      if (beta) v += ld(p);
      if (relu) v = fmaxf(v, 0.f);
      st(p, v);
    }
  }
}

// Weight gradient partials: P[chunk][K x N] = sum over the chunk's rows m of
// A[m][k] dY[m][n] (A BF16 activations, dY FP32), then a fixed-order sum
// over chunks: deterministic.
constexpr int kChunk = 512;
template <class TA>
__global__ void __launch_bounds__(256) wgrad_partial_kernel(int64_t M, int N, int K, const TA* __restrict__ A,
                                                            int64_t lda, const float* __restrict__ dY, int64_t ldy,
                                                            float* __restrict__ part) {
  __shared__ float sa[kTK][kTM + 4];
  __shared__ float sb[kTK][kTN + 4];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int k0 = blockIdx.x * kTM, n0 = blockIdx.y * kTN;
  const int64_t r0 = (int64_t)blockIdx.z * kChunk, r1 = min(M, r0 + kChunk);
  float acc[4][4] = {};
  for (int64_t rr = r0; rr < r1; rr += kTK) {
    for (int t = threadIdx.x; t < kTK * kTM; t += 256) {
      const int r = t / kTM, k = t % kTM;
      const int64_t gm = rr + r;
      sa[r][k] = (gm < r1 && k0 + k < K) ? ld(A + gm * lda + k0 + k) : 0.f;
    }
    for (int t = threadIdx.x; t < kTK * kTN; t += 256) {
      const int r = t / kTN, c = t % kTN;
      const int64_t gm = rr + r;
      sb[r][c] = (gm < r1 && n0 + c < N) ? dY[gm * ldy + n0 + c] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kTK; ++r) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = sa[r][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = sb[r][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
  float* P = part + (size_t)blockIdx.z * K * N;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int k = k0 + ty * 4 + i;
    if (k >= K) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + tx * 4 + j;
      if (n < N) P[(size_t)k * N + n] = acc[i][j];
    }
  }
}

// G[k][n] (+)= sum over chunks of P; bias gradient: gb[n] (+)= sum over rows of dY
__global__ void wgrad_reduce_kernel(const float* __restrict__ part, int chunks, int64_t kn, float* __restrict__ G) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= kn) return;
  float s = 0.f;
  for (int q = 0; q < chunks; ++q) s += part[(size_t)q * kn + t];
  G[t] += s;
}
__global__ void bgrad_kernel(int64_t M, int N, const float* __restrict__ dY, int64_t ldy, float* __restrict__ gb) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.f;
  for (int64_t m = 0; m < M; ++m) s += dY[m * ldy + n];
  gb[n] += s;
}

// ----------------------------------------------------------- graph ops
// C[e] = [h[src e], h[dst e], z[e]] (BF16, 3 kH wide)
__global__ void gather3_kernel(int64_t E, const int32_t* __restrict__ src, const int32_t* __restrict__ dst,
                               const __nv_bfloat16* __restrict__ h, const __nv_bfloat16* __restrict__ z,
                               __nv_bfloat16* __restrict__ C) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= E * 3 * kH) return;
  const int64_t e = t / (3 * kH);
  const int c = (int)(t % (3 * kH));
  __nv_bfloat16 v;
  if (c < kH)
    v = h[(int64_t)src[e] * kH + c];
  else if (c < 2 * kH)
    v = h[(int64_t)dst[e] * kH + c - kH];
  else
    v = z[e * kH + c - 2 * kH];
  C[t] = v;
}
// C[j] = [h[j], a[j]] with a[j] the mean of m over column j's edges (edges of
// a column are contiguous: ptr)
__global__ void mean_concat_kernel(int64_t n, const int32_t* __restrict__ ptr, const __nv_bfloat16* __restrict__ h,
                                   const __nv_bfloat16* __restrict__ m, __nv_bfloat16* __restrict__ C) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n * kH) return;
  const int64_t j = t / kH;
  const int c = (int)(t % kH);
  const int e0 = ptr[j], e1 = ptr[j + 1];
  float s = 0.f;
  for (int e = e0; e < e1; ++e) s += __bfloat162float(m[(int64_t)e * kH + c]);
  C[j * 2 * kH + c] = h[j * kH + c];
  C[j * 2 * kH + kH + c] = __float2bfloat16_rn(e1 > e0 ? s / (float)(e1 - e0) : 0.f);
}
// h_out = h_in + u (BF16)
__global__ void residual_kernel(int64_t count, const __nv_bfloat16* __restrict__ a, const __nv_bfloat16* __restrict__ b,
                                __nv_bfloat16* __restrict__ out) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < count) out[t] = __float2bfloat16_rn(__bfloat162float(a[t]) + __bfloat162float(b[t]));
}
// dY *= (Y > 0)
__global__ void relu_bwd_kernel(int64_t count, const __nv_bfloat16* __restrict__ y, float* __restrict__ dy) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < count && !(__bfloat162float(y[t]) > 0.f)) dy[t] = 0.f;
}
// backward of gather3: dh[j] += sum over column j's edges of dC[e][kH..2kH)
// (dst part) + sum over the edges whose source is j of dC[e][0..kH) (those
// are the reverses of column j's edges), dz[e] += dC[e][2kH..3kH)
__global__ void scatter3_kernel(int64_t n, int64_t E, const int32_t* __restrict__ ptr,
                                const int32_t* __restrict__ rev, const float* __restrict__ dC,
                                float* __restrict__ dh, float* __restrict__ dz, int dz_accumulate) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < n * kH) {
    const int64_t j = t / kH;
    const int c = (int)(t % kH);
    float s = dh[t];
    for (int e = ptr[j]; e < ptr[j + 1]; ++e) {
      s += dC[(int64_t)e * 3 * kH + kH + c];
      s += dC[(int64_t)rev[e] * 3 * kH + c];
    }
    dh[t] = s;
  }
  if (t < E * kH) {
    const int64_t e = t / kH;
    const int c = (int)(t % kH);
    const float v = dC[e * 3 * kH + 2 * kH + c];
    dz[t] = dz_accumulate ? dz[t] + v : v;
  }
}
// backward of mean_concat: dh[j] += dC[j][0..kH); dm[e] = dC[dst e][kH..) / deg
__global__ void mean_concat_bwd_kernel(int64_t n, int64_t E, const int32_t* __restrict__ ptr,
                                       const int32_t* __restrict__ dst, const float* __restrict__ dC,
                                       float* __restrict__ dh, float* __restrict__ dm) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < n * kH) {
    const int64_t j = t / kH;
    const int c = (int)(t % kH);
    dh[t] += dC[j * 2 * kH + c];
  }
  if (t < E * kH) {
    const int64_t e = t / kH;
    const int c = (int)(t % kH);
    const int64_t j = dst[e];
    const int deg = ptr[j + 1] - ptr[j];
    dm[t] = dC[j * 2 * kH + kH + c] / (float)deg;
  }
}
// squared error of the outputs against the targets and its gradient
// 2 (o - t) / count; loss accumulated in FP64 per block then atomically
__global__ void mse_kernel(int64_t count, const float* __restrict__ o, const float* __restrict__ tg,
                           float* __restrict__ d, double inv_count, double* __restrict__ loss) {
  __shared__ double red[256];
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double s = 0.0;
  if (t < count) {
    const float r = o[t] - tg[t];
    d[t] = (float)(2.0 * inv_count) * r;
    s = (double)r * r;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int k = 128; k > 0; k >>= 1) {
    if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, red[0] * inv_count);
}
// Adam on the master weights, then the BF16 copy
__global__ void adam_kernel(int64_t count, float* __restrict__ w, __nv_bfloat16* __restrict__ wb,
                            const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= count) return;
  const float gi = g[t];
  const float mi = b1 * m[t] + (1.f - b1) * gi;
  const float vi = b2 * v[t] + (1.f - b2) * gi * gi;
  m[t] = mi;
  v[t] = vi;
  const float wi = w[t] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[t] = wi;
  wb[t] = __float2bfloat16_rn(wi);
}
__global__ void to_bf16_kernel(int64_t count, const float* __restrict__ a, __nv_bfloat16* __restrict__ b) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < count) b[t] = __float2bfloat16_rn(a[t]);
}

// ------------------------------------------------ inputs and targets
// R X R^T on each 3 x 3 sub-block of an 18 x 18 column-major block (R
// row-major 3 x 3), in shared memory; inverse = 1 applies R^T X R
__device__ void rotate18(const float* R, const double* X, double* Y, bool inverse) {
  const int t = threadIdx.x;
  if (t >= 324) return;
  const int row = t % 18, col = t / 18;
  const int a = row / 3, p = row % 3, b = col / 3, q = col % 3;
  double s = 0.0;
  for (int pp = 0; pp < 3; ++pp)
    for (int qq = 0; qq < 3; ++qq) {
      const double rp = inverse ? R[pp * 3 + p] : R[p * 3 + pp];
      const double rq = inverse ? R[qq * 3 + q] : R[q * 3 + qq];
      s += rp * X[(3 * a + pp) + 18 * (3 * b + qq)] * rq;
    }
  Y[t] = s;
}

// One CTA per block b (self blocks first, then edges, as NearPattern): the
// normalised operator input (X row, after its geometry features) and, when
// `target` is given, the normalised target (local inverse minus Neumann).
__global__ void __launch_bounds__(352) inputs_kernel(const OpView A, int64_t n_el,
                                                     const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                                     const int32_t* __restrict__ dst, const double* __restrict__ dinv,
                                                     const double* __restrict__ neu,
                                                     const double* __restrict__ target, const float* __restrict__ rot,
                                                     const float* __restrict__ size, double G,
                                                     __nv_bfloat16* __restrict__ xn, __nv_bfloat16* __restrict__ xe,
                                                     float* __restrict__ tn, float* __restrict__ te) {
  __shared__ double s_x[324], s_y[324], s_t[324];
  __shared__ float s_r[9];
  const int64_t b = blockIdx.x;
  const int t = threadIdx.x;
  const bool self = b < n_el;
  const int64_t e = self ? -1 : b - n_el;
  const int64_t j = self ? b : dst[e];
  const int64_t i = self ? b : idx[e];
  const int64_t blk = self ? j + ptr[j] : j + 1 + e;
  const double sc = G / (double)size[j];
  if (t < 9) s_r[t] = rot[9 * j + t];
  if (t < 324) {
    if (self) {
      s_x[t] = sc * dinv[(size_t)324 * j + t];
    } else {
      // D_i^-1 A_ij
      const int r = t % 18, c = t / 18;
      double s = 0.0;
      for (int k = 0; k < 18; ++k) s += dinv[(size_t)324 * i + r + 18 * k] * A.at_blk(18 * i + k, 18 * j + c, blk);
      s_x[t] = s;
    }
  }
  __syncthreads();
  rotate18(s_r, s_x, s_y, false);
  __syncthreads();
  if (t < 324) {
    if (self)
      xn[j * kFN + kGeoN + t] = __float2bfloat16_rn((float)s_y[t]);
    else
      xe[e * kFE + kGeoE + t] = __float2bfloat16_rn((float)s_y[t]);
  }
  if (!target) return;
  if (t < 324) s_t[t] = sc * (target[(size_t)324 * blk + t] - neu[(size_t)324 * blk + t]);
  __syncthreads();
  rotate18(s_r, s_t, s_y, false);
  __syncthreads();
  if (t < 324) {
    if (self)
      tn[j * 324 + t] = (float)s_y[t];
    else
      te[e * 324 + t] = (float)s_y[t];
  }
}

// M = M^N + (s_j / G) Q_j^T O Q_j for every block (outputs O of the network)
__global__ void __launch_bounds__(352) apply_outputs_kernel(int64_t n_el, const int32_t* __restrict__ ptr,
                                                            const int32_t* __restrict__ dst,
                                                            const float* __restrict__ on,
                                                            const float* __restrict__ oe,
                                                            const float* __restrict__ rot,
                                                            const float* __restrict__ size, double G,
                                                            double* __restrict__ blocks) {
  __shared__ double s_x[324], s_y[324];
  __shared__ float s_r[9];
  const int64_t b = blockIdx.x;
  const int t = threadIdx.x;
  const bool self = b < n_el;
  const int64_t e = self ? -1 : b - n_el;
  const int64_t j = self ? b : dst[e];
  const int64_t blk = self ? j + ptr[j] : j + 1 + e;
  if (t < 9) s_r[t] = rot[9 * j + t];
  if (t < 324) s_x[t] = self ? on[j * 324 + t] : oe[e * 324 + t];
  __syncthreads();
  rotate18(s_r, s_x, s_y, true);
  __syncthreads();
  if (t < 324) blocks[(size_t)324 * blk + t] += ((double)size[j] / G) * s_y[t];
}

inline unsigned blocks_for(int64_t count, int bs = 256) { return (unsigned)((count + bs - 1) / bs); }

}  // namespace gnn
}  // namespace hfpx

// ------------------------------------------------------------------ host
namespace hfpx {
namespace gnn {
namespace {

template <class T>
T* galloc(hfpx_gnn_graph* g, size_t count, int* rc, hfpx_ctx* c) {
  if (*rc) return nullptr;
  void* p = nullptr;
  *rc = pool_alloc(c, &p, sizeof(T) * std::max<size_t>(1, count), "network buffers");
  if (!*rc) g->allocs.push_back(p);
  return static_cast<T*>(p);
}

// geometry of one element: frame rows (e1, e2, e3) as make_el_r_tensor
// builds them, centroid, size s = sqrt(2 area)
struct Geo {
  double r[9], c[3], s, l1, x2, y2;
};
Geo element_geo(const double* v) {
  Geo g;
  double a[3], b[3];
  for (int k = 0; k < 3; ++k) {
    a[k] = v[3 + k] - v[k];
    b[k] = v[6 + k] - v[k];
    g.c[k] = (v[k] + v[3 + k] + v[6 + k]) / 3.0;
  }
  const double la = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  double n[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
  const double ln = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  double e1[3], e3[3];
  for (int k = 0; k < 3; ++k) {
    e1[k] = a[k] / la;
    e3[k] = n[k] / ln;
  }
  const double e2[3] = {e3[1] * e1[2] - e3[2] * e1[1], e3[2] * e1[0] - e3[0] * e1[2], e3[0] * e1[1] - e3[1] * e1[0]};
  for (int k = 0; k < 3; ++k) {
    g.r[k] = e1[k];
    g.r[3 + k] = e2[k];
    g.r[6 + k] = e3[k];
  }
  g.s = std::sqrt(ln);  // 2 area = |a x b|
  g.l1 = la / g.s;
  g.x2 = (b[0] * e1[0] + b[1] * e1[1] + b[2] * e1[2]) / g.s;
  g.y2 = (b[0] * e2[0] + b[1] * e2[1] + b[2] * e2[2]) / g.s;
  return g;
}

void rot_apply(const double* r, const double* x, double* y) {
  for (int p = 0; p < 3; ++p) y[p] = r[3 * p] * x[0] + r[3 * p + 1] * x[1] + r[3 * p + 2] * x[2];
}

void lin(hfpx_ctx* c, int64_t M, int N, int K, const void* A, bool a_bf16, int64_t lda, const __nv_bfloat16* W,
         const float* bias, void* C, bool c_bf16, int64_t ldc, bool relu, bool beta) {
  const dim3 grid((unsigned)((M + kTM - 1) / kTM), (unsigned)((N + kTN - 1) / kTN));
  ++g_launches;
  if (a_bf16 && c_bf16)
    gemm_kernel<__nv_bfloat16, __nv_bfloat16, __nv_bfloat16, false><<<grid, 256, 0, c->stream>>>(
        M, N, K, (const __nv_bfloat16*)A, lda, W, N, bias, (__nv_bfloat16*)C, ldc, relu, beta);
  else if (a_bf16)
    gemm_kernel<__nv_bfloat16, __nv_bfloat16, float, false><<<grid, 256, 0, c->stream>>>(
        M, N, K, (const __nv_bfloat16*)A, lda, W, N, bias, (float*)C, ldc, relu, beta);
}
// dX (M x K, FP32) (+)= dY (M x N, FP32) W^T, W K x N BF16
void lin_dx(hfpx_ctx* c, int64_t M, int N, int K, const float* dY, int64_t ldy, const __nv_bfloat16* W, float* dX,
            int64_t ldx, bool beta) {
  const dim3 grid((unsigned)((M + kTM - 1) / kTM), (unsigned)((K + kTN - 1) / kTN));
  ++g_launches;
  gemm_kernel<float, __nv_bfloat16, float, true><<<grid, 256, 0, c->stream>>>(M, K, N, dY, ldy, W, N, nullptr, dX, ldx,
                                                                              0, beta);
}
// gW (K x N) += A^T dY, gb (N) += column sums of dY
void lin_dw(hfpx_ctx* c, hfpx_gnn_graph* g, int64_t M, int N, int K, const __nv_bfloat16* A, int64_t lda,
            const float* dY, int64_t ldy, float* gW, float* gb) {
  const int chunks = (int)((M + kChunk - 1) / kChunk);
  const dim3 grid((unsigned)((K + kTM - 1) / kTM), (unsigned)((N + kTN - 1) / kTN), (unsigned)chunks);
  g_launches += 3;
  wgrad_partial_kernel<__nv_bfloat16><<<grid, 256, 0, c->stream>>>(M, N, K, A, lda, dY, ldy, g->part);
  wgrad_reduce_kernel<<<blocks_for((int64_t)K * N), 256, 0, c->stream>>>(g->part, chunks, (int64_t)K * N, gW);
  bgrad_kernel<<<blocks_for(N, 64), 64, 0, c->stream>>>(M, N, dY, ldy, gb);
}

int ensure_activations(hfpx_ctx* c, hfpx_gnn_graph* g) {
  if (g->oe) return 0;
  int rc = 0;
  const int64_t n = g->n_nodes, E = g->n_edges;
  for (int l = 0; l <= kLayers; ++l) g->h[l] = galloc<__nv_bfloat16>(g, n * kH, &rc, c);
  g->z = galloc<__nv_bfloat16>(g, E * kH, &rc, c);
  for (int l = 0; l < kLayers; ++l) {
    g->cm[l] = galloc<__nv_bfloat16>(g, E * 3 * kH, &rc, c);
    g->m[l] = galloc<__nv_bfloat16>(g, E * kH, &rc, c);
    g->cu[l] = galloc<__nv_bfloat16>(g, n * 2 * kH, &rc, c);
    g->u[l] = galloc<__nv_bfloat16>(g, n * kH, &rc, c);
  }
  g->ce = galloc<__nv_bfloat16>(g, E * 3 * kH, &rc, c);
  g->oe = galloc<float>(g, E * kOut, &rc, c);
  g->on = galloc<float>(g, n * kOut, &rc, c);
  g->dh = galloc<float>(g, n * kH, &rc, c);
  g->dh2 = galloc<float>(g, n * kH, &rc, c);
  g->du = galloc<float>(g, n * kH, &rc, c);
  g->dz = galloc<float>(g, E * kH, &rc, c);
  g->dce = galloc<float>(g, E * 3 * kH, &rc, c);
  g->doe = galloc<float>(g, E * kOut, &rc, c);
  g->don = galloc<float>(g, n * kOut, &rc, c);
  g->dm = galloc<float>(g, E * kH, &rc, c);
  g->dcu = galloc<float>(g, n * 2 * kH, &rc, c);
  const int64_t rows = std::max(n, E);
  const int64_t chunks = (rows + kChunk - 1) / kChunk;
  g->part_floats = chunks * (int64_t)std::max(kFE * kH, 3 * kH * kOut);
  g->part = galloc<float>(g, g->part_floats, &rc, c);
  g->loss = galloc<float>(g, 2, &rc, c);  // one double
  return rc;
}

int forward(hfpx_ctx* c, const hfpx_gnn* net, hfpx_gnn_graph* g) {
  int rc = ensure_activations(c, g);
  if (rc) return rc;
  const int64_t n = g->n_nodes, E = g->n_edges;
  const __nv_bfloat16* W = net->d_wb;
  const float* Bf = net->d_w;
  auto w = [&](int t) { return W + net->w_off[t]; };
  auto b = [&](int t) { return Bf + net->b_off[t]; };
  lin(c, n, kH, kFN, g->xn, true, kFN, w(0), b(0), g->h[0], true, kH, true, false);
  lin(c, E, kH, kFE, g->xe, true, kFE, w(1), b(1), g->z, true, kH, true, false);
  for (int l = 0; l < kLayers; ++l) {
    g_launches += 3;
    gather3_kernel<<<blocks_for(E * 3 * kH), 256, 0, c->stream>>>(E, g->pat->d_idx, g->pat->d_dst, g->h[l], g->z,
                                                                   g->cm[l]);
    lin(c, E, kH, 3 * kH, g->cm[l], true, 3 * kH, w(2 + 2 * l), b(2 + 2 * l), g->m[l], true, kH, true, false);
    mean_concat_kernel<<<blocks_for(n * kH), 256, 0, c->stream>>>(n, g->pat->d_ptr, g->h[l], g->m[l], g->cu[l]);
    lin(c, n, kH, 2 * kH, g->cu[l], true, 2 * kH, w(3 + 2 * l), b(3 + 2 * l), g->u[l], true, kH, true, false);
    residual_kernel<<<blocks_for(n * kH), 256, 0, c->stream>>>(n * kH, g->h[l], g->u[l], g->h[l + 1]);
  }
  ++g_launches;
  gather3_kernel<<<blocks_for(E * 3 * kH), 256, 0, c->stream>>>(E, g->pat->d_idx, g->pat->d_dst, g->h[kLayers], g->z,
                                                                 g->ce);
  const int te = 2 + 2 * kLayers, tn = te + 1;
  lin(c, E, kOut, 3 * kH, g->ce, true, 3 * kH, w(te), b(te), g->oe, false, kOut, false, false);
  lin(c, n, kOut, kH, g->h[kLayers], true, kH, w(tn), b(tn), g->on, false, kOut, false, false);
  return check_cuda(c, cudaGetLastError(), "network forward");
}

// loss = mean over all output entries of (o - t)^2; gradients into net->d_g
int backward(hfpx_ctx* c, hfpx_gnn* net, hfpx_gnn_graph* g) {
  const int64_t n = g->n_nodes, E = g->n_edges;
  const int64_t cnt = (n + E) * kOut;
  const double inv = 1.0 / (double)cnt;
  float* G = net->d_g;
  auto gw = [&](int t) { return G + net->w_off[t]; };
  auto gb = [&](int t) { return G + net->b_off[t]; };
  auto w = [&](int t) { return net->d_wb + net->w_off[t]; };
  int rc = check_cuda(c, cudaMemsetAsync(g->loss, 0, sizeof(double), c->stream), "loss");
  if (!rc) rc = check_cuda(c, cudaMemsetAsync(G, 0, sizeof(float) * net->n_params, c->stream), "gradients");
  if (rc) return rc;
  double* loss = reinterpret_cast<double*>(g->loss);
  g_launches += 2;
  mse_kernel<<<blocks_for(E * kOut), 256, 0, c->stream>>>(E * kOut, g->oe, g->te, g->doe, inv, loss);
  mse_kernel<<<blocks_for(n * kOut), 256, 0, c->stream>>>(n * kOut, g->on, g->tn, g->don, inv, loss);
  const int te = 2 + 2 * kLayers, tn = te + 1;
  // heads
  lin_dw(c, g, E, kOut, 3 * kH, g->ce, 3 * kH, g->doe, kOut, gw(te), gb(te));
  lin_dx(c, E, kOut, 3 * kH, g->doe, kOut, w(te), g->dce, 3 * kH, false);
  lin_dw(c, g, n, kOut, kH, g->h[kLayers], kH, g->don, kOut, gw(tn), gb(tn));
  lin_dx(c, n, kOut, kH, g->don, kOut, w(tn), g->dh, kH, false);
  ++g_launches;
  scatter3_kernel<<<blocks_for(std::max(n, E) * kH), 256, 0, c->stream>>>(n, E, g->pat->d_ptr, g->pat->d_rev, g->dce,
                                                                           g->dh, g->dz, 0);
  for (int l = kLayers - 1; l >= 0; --l) {
    // h[l+1] = h[l] + u[l]: dh is dL/dh[l+1]
    cudaMemcpyAsync(g->du, g->dh, sizeof(float) * n * kH, cudaMemcpyDeviceToDevice, c->stream);
    cudaMemcpyAsync(g->dh2, g->dh, sizeof(float) * n * kH, cudaMemcpyDeviceToDevice, c->stream);
    ++g_launches;
    relu_bwd_kernel<<<blocks_for(n * kH), 256, 0, c->stream>>>(n * kH, g->u[l], g->du);
    lin_dw(c, g, n, kH, 2 * kH, g->cu[l], 2 * kH, g->du, kH, gw(3 + 2 * l), gb(3 + 2 * l));
    lin_dx(c, n, kH, 2 * kH, g->du, kH, w(3 + 2 * l), g->dcu, 2 * kH, false);
    g_launches += 2;
    mean_concat_bwd_kernel<<<blocks_for(std::max(n, E) * kH), 256, 0, c->stream>>>(n, E, g->pat->d_ptr, g->pat->d_dst,
                                                                                    g->dcu, g->dh2, g->dm);
    relu_bwd_kernel<<<blocks_for(E * kH), 256, 0, c->stream>>>(E * kH, g->m[l], g->dm);
    lin_dw(c, g, E, kH, 3 * kH, g->cm[l], 3 * kH, g->dm, kH, gw(2 + 2 * l), gb(2 + 2 * l));
    lin_dx(c, E, kH, 3 * kH, g->dm, kH, w(2 + 2 * l), g->dce, 3 * kH, false);
    ++g_launches;
    scatter3_kernel<<<blocks_for(std::max(n, E) * kH), 256, 0, c->stream>>>(n, E, g->pat->d_ptr, g->pat->d_rev,
                                                                             g->dce, g->dh2, g->dz, 1);
    std::swap(g->dh, g->dh2);
  }
  g_launches += 2;
  relu_bwd_kernel<<<blocks_for(n * kH), 256, 0, c->stream>>>(n * kH, g->h[0], g->dh);
  relu_bwd_kernel<<<blocks_for(E * kH), 256, 0, c->stream>>>(E * kH, g->z, g->dz);
  lin_dw(c, g, n, kH, kFN, g->xn, kFN, g->dh, kH, gw(0), gb(0));
  lin_dw(c, g, E, kH, kFE, g->xe, kFE, g->dz, kH, gw(1), gb(1));
  return check_cuda(c, cudaGetLastError(), "network backward");
}

int adam(hfpx_ctx* c, hfpx_gnn* net, float lr) {
  ++net->step;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, (float)net->step), c2 = 1.f - std::pow(b2, (float)net->step);
  ++g_launches;
  adam_kernel<<<blocks_for(net->n_params), 256, 0, c->stream>>>(net->n_params, net->d_w, net->d_wb, net->d_g, net->d_m,
                                                                net->d_v, lr, b1, b2, 1e-8f, c1, c2);
  return check_cuda(c, cudaGetLastError(), "Adam step");
}

int net_alloc(hfpx_ctx* c, hfpx_gnn* net) {
  int64_t off = 0;
  for (int t = 0; t < kTensors; ++t) {
    const Shape s = tensor_shape(t);
    net->w_off[t] = off;
    off += (int64_t)s.rows * s.cols;
    net->b_off[t] = off;
    off += s.cols;
  }
  net->n_params = off;
  net->device = c->device;
  int rc = 0;
  for (float** p : {&net->d_w, &net->d_g, &net->d_m, &net->d_v})
    if (!rc) rc = check_cuda(c, cudaMalloc(p, sizeof(float) * off), "network parameters");
  if (!rc) rc = check_cuda(c, cudaMalloc(&net->d_wb, sizeof(__nv_bfloat16) * off), "network parameters");
  if (!rc) rc = check_cuda(c, cudaMemsetAsync(net->d_m, 0, sizeof(float) * off, c->stream), "Adam state");
  if (!rc) rc = check_cuda(c, cudaMemsetAsync(net->d_v, 0, sizeof(float) * off, c->stream), "Adam state");
  return rc;
}

int net_upload(hfpx_ctx* c, hfpx_gnn* net, const float* host) {
  int rc = check_cuda(c, cudaMemcpyAsync(net->d_w, host, sizeof(float) * net->n_params, cudaMemcpyHostToDevice,
                                         c->stream),
                      "parameters");
  if (!rc) {
    ++g_launches;
    to_bf16_kernel<<<blocks_for(net->n_params), 256, 0, c->stream>>>(net->n_params, net->d_w, net->d_wb);
    rc = check_cuda(c, cudaGetLastError(), "parameters");
  }
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "parameters");
  return rc;
}

}  // namespace

void graph_destroy(hfpx_gnn_graph* g);

// The mesh-only part of a graph: the pattern, the frames and sizes, the
// geometry columns of the inputs (the operator columns are filled per
// matrix by graph_fill).
// The mesh-only inputs of the network (host): per element its geometry row
// and per pattern edge its geometry row (the operator columns stay zero),
// its frame and size.
bool host_inputs(const hfpx_mesh* mesh, const NearPattern& pat, GraphHostInputs* out) {
  const int64_t n = mesh->n_el, E = pat.n_edges;
  if ((int64_t)mesh->h_vert.size() < 9 * n || (int64_t)mesh->h_vid.size() < 3 * n) return false;
  // host geometry: frames, sizes, features
  std::vector<Geo> geo(n);
  for (int64_t e = 0; e < n; ++e) geo[e] = element_geo(&mesh->h_vert[9 * e]);
  double smean = 0.0;
  for (const Geo& q : geo) smean += q.s;
  smean /= (double)n;
  // how many elements share each element edge (1: a boundary edge): the
  // (vertex pair, 3 e + k) keys sorted, counted by runs
  std::vector<std::pair<std::pair<int64_t, int64_t>, int32_t>> ek((size_t)(3 * n));
  for (int64_t e = 0; e < n; ++e)
    for (int k = 0; k < 3; ++k) {
      int64_t a = mesh->h_vid[3 * e + k], b = mesh->h_vid[3 * e + (k + 1) % 3];
      if (a > b) std::swap(a, b);
      ek[(size_t)(3 * e + k)] = {{a, b}, (int32_t)(3 * e + k)};
    }
  std::sort(ek.begin(), ek.end());
  std::vector<int32_t> edge_count((size_t)(3 * n));
  for (size_t i = 0; i < ek.size();) {
    size_t j = i;
    while (j < ek.size() && ek[j].first == ek[i].first) ++j;
    for (size_t q = i; q < j; ++q) edge_count[(size_t)ek[q].second] = (int32_t)(j - i);
    i = j;
  }
  // the geometry columns only (the first kGeoN / kGeoE of each row)
  std::vector<__nv_bfloat16> xn((size_t)n * kGeoN), xe((size_t)E * kGeoE);
  std::vector<float> rot((size_t)9 * n), size(n);
  for (int64_t j = 0; j < n; ++j) {
    const Geo& q = geo[j];
    int boundary = 0;
    for (int k = 0; k < 3; ++k)
      if (edge_count[(size_t)(3 * j + k)] == 1) ++boundary;
    const int deg = pat.ptr[j + 1] - pat.ptr[j];
    double curv = 0.0;
    for (int32_t e = pat.ptr[j]; e < pat.ptr[j + 1]; ++e) {
      const Geo& p = geo[pat.idx[e]];
      curv += 1.0 - (p.r[6] * q.r[6] + p.r[7] * q.r[7] + p.r[8] * q.r[8]);
    }
    curv = deg ? curv / deg : 0.0;
    const float f[kGeoN] = {(float)std::log(q.s / smean), (float)q.l1, (float)q.x2, (float)q.y2, boundary / 3.f,
                            deg / 12.f, (float)(10.0 * curv), 1.f};
    for (int k = 0; k < kGeoN; ++k) xn[(size_t)j * kGeoN + k] = __float2bfloat16_rn(f[k]);
    for (int k = 0; k < 9; ++k) rot[9 * j + k] = (float)q.r[k];
    size[j] = (float)q.s;
    for (int32_t e = pat.ptr[j]; e < pat.ptr[j + 1]; ++e) {
      const int64_t i = pat.idx[e];
      const Geo& p = geo[i];
      double d[3] = {(p.c[0] - q.c[0]) / q.s, (p.c[1] - q.c[1]) / q.s, (p.c[2] - q.c[2]) / q.s}, dl[3], nl[3], el[3];
      rot_apply(q.r, d, dl);
      rot_apply(q.r, p.r + 6, nl);
      rot_apply(q.r, p.r, el);
      int shared = 0;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) shared += mesh->h_vid[3 * i + a] == mesh->h_vid[3 * j + b];
      const float fe[kGeoE] = {(float)dl[0], (float)dl[1], (float)dl[2], (float)nl[0], (float)nl[1], (float)nl[2],
                               (float)el[0], (float)el[1], (float)el[2], (float)std::log(p.s / q.s),
                               (float)(shared - 1), 1.f};
      for (int k = 0; k < kGeoE; ++k) xe[(size_t)e * kGeoE + k] = __float2bfloat16_rn(fe[k]);
    }
  }
  out->xn.resize(xn.size());
  out->xe.resize(xe.size());
  static_assert(sizeof(__nv_bfloat16) == sizeof(uint16_t), "bf16 bits");
  std::memcpy(out->xn.data(), xn.data(), sizeof(uint16_t) * xn.size());
  std::memcpy(out->xe.data(), xe.data(), sizeof(uint16_t) * xe.size());
  out->rot = std::move(rot);
  out->size = std::move(size);
  return true;
}

int graph_prepare(hfpx_ctx* c, const hfpx_mesh* mesh, hfpx_gnn_graph** out) {
  *out = nullptr;
  hfpx_gnn_graph* g = new (std::nothrow) hfpx_gnn_graph;
  if (!g) return set_error(c, HFPX_ERR_NOMEM, "graph");
  g->pat = mesh_pattern(c, mesh);
  if (!g->pat) {
    delete g;
    return set_error(c, HFPX_ERR_NOMEM, "near-field pattern");
  }
  int rc = 0;
  const int64_t n = mesh->n_el, E = g->pat->n_edges;
  g->n_nodes = n;
  g->n_edges = E;
  // the geometry inputs: from the mesh's set-up thread, or made here
  SetupClock::time_point t0 = SetupClock::now();
  GraphHostInputs local;
  const GraphHostInputs* in = nullptr;
  MeshHostSetup* hs = const_cast<hfpx_mesh*>(mesh)->host_setup.get();
  if (hs) {
    hs->wait(3);
    if (hs->graph_ok) in = &hs->graph;
  }
  if (!in) {
    if (!host_inputs(mesh, *g->pat, &local)) rc = set_error(c, HFPX_ERR_STATE, "mesh has no host geometry");
    in = &local;
  }
  setup_note(hs && hs->graph_ok ? "network graph inputs (wait for the set-up thread)" : "network graph inputs",
             ms_since(t0));
  t0 = SetupClock::now();
  g->d_size = galloc<float>(g, n, &rc, c);
  g->d_rot = galloc<float>(g, 9 * n, &rc, c);
  g->xn = galloc<__nv_bfloat16>(g, (size_t)n * kFN, &rc, c);
  g->xe = galloc<__nv_bfloat16>(g, (size_t)E * kFE, &rc, c);
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(g->d_size, in->size.data(), sizeof(float) * n, cudaMemcpyHostToDevice, c->stream), "sizes");
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(g->d_rot, in->rot.data(), sizeof(float) * 9 * n, cudaMemcpyHostToDevice, c->stream), "frames");
  // the input rows: zero, then the geometry columns from the host (the
  // operator columns are written per matrix by graph_fill)
  if (!rc) rc = check_cuda(c, cudaMemsetAsync(g->xn, 0, sizeof(__nv_bfloat16) * (size_t)n * kFN, c->stream), "inputs");
  if (!rc) rc = check_cuda(c, cudaMemsetAsync(g->xe, 0, sizeof(__nv_bfloat16) * (size_t)E * kFE, c->stream), "inputs");
  // (one contiguous upload each, then a strided copy on the device: a
  // strided copy from pageable host memory goes row by row)
  uint16_t* sxn = galloc<uint16_t>(g, (size_t)n * kGeoN, &rc, c);
  uint16_t* sxe = galloc<uint16_t>(g, (size_t)E * kGeoE, &rc, c);
  if (!rc && n > 0)
    rc = check_cuda(c, cudaMemcpyAsync(sxn, in->xn.data(), sizeof(uint16_t) * in->xn.size(), cudaMemcpyHostToDevice,
                                       c->stream), "inputs");
  if (!rc && E > 0)
    rc = check_cuda(c, cudaMemcpyAsync(sxe, in->xe.data(), sizeof(uint16_t) * in->xe.size(), cudaMemcpyHostToDevice,
                                       c->stream), "inputs");
  if (!rc && n > 0)
    rc = check_cuda(c, cudaMemcpy2DAsync(g->xn, sizeof(uint16_t) * kFN, sxn, sizeof(uint16_t) * kGeoN,
                                         sizeof(uint16_t) * kGeoN, (size_t)n, cudaMemcpyDeviceToDevice, c->stream),
                    "inputs");
  if (!rc && E > 0)
    rc = check_cuda(c, cudaMemcpy2DAsync(g->xe, sizeof(uint16_t) * kFE, sxe, sizeof(uint16_t) * kGeoE,
                                         sizeof(uint16_t) * kGeoE, (size_t)E, cudaMemcpyDeviceToDevice, c->stream),
                    "inputs");
  // the host vectors are pageable: finish the copies before they go
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "graph inputs");
  setup_note("network graph: uploads (with the queued work)", ms_since(t0));
  if (rc) {
    graph_destroy(g);
    return rc;
  }
  *out = g;
  return 0;
}

// The operator columns of the inputs (and, with a target, the training
// targets) of matrix m: dinv and neu are the diagonal-block inverses and the
// Neumann blocks of m in the pattern's order.
int graph_fill(hfpx_ctx* c, hfpx_gnn_graph* g, const hfpx_matrix* m, double G, const double* dinv, const double* neu,
               const double* target) {
  ++g_launches;
  inputs_kernel<<<(unsigned)g->pat->blocks(), 352, 0, c->stream>>>(
      op_view(m), g->n_nodes, g->pat->d_ptr, g->pat->d_idx, g->pat->d_dst, dinv, neu, target, g->d_rot, g->d_size,
      G, g->xn, g->xe, target ? g->tn : nullptr, target ? g->te : nullptr);
  return check_cuda(c, cudaGetLastError(), "network inputs");
}

// A training graph: its own diagonal inverses, Neumann blocks and the exact
// local inverse as the target.
int graph_create(hfpx_ctx* c, const hfpx_mesh* mesh, const hfpx_matrix* m, double G, bool with_targets,
                 hfpx_gnn_graph** out) {
  *out = nullptr;
  hfpx_gnn_graph* g = nullptr;
  int rc = graph_prepare(c, mesh, &g);
  if (rc) return rc;
  const int64_t n = g->n_nodes, E = g->n_edges, nb = g->pat->blocks();
  g->d_dinv = galloc<double>(g, 324 * n, &rc, c);
  g->d_neu = galloc<double>(g, 324 * (size_t)nb, &rc, c);
  double* target = nullptr;
  if (with_targets) {
    g->tn = galloc<float>(g, (size_t)n * kOut, &rc, c);
    g->te = galloc<float>(g, (size_t)E * kOut, &rc, c);
    target = galloc<double>(g, 324 * (size_t)nb, &rc, c);
  }
  int* err = (int*)ctx_scratch(c, kScrTcErr, sizeof(int));
  if (!rc && !err) rc = set_error(c, HFPX_ERR_NOMEM, "status word");
  if (!rc) rc = check_cuda(c, cudaMemsetAsync(err, 0, sizeof(int), c->stream), "status");
  if (!rc) rc = check_cuda(c, cudaMemsetAsync(g->d_neu, 0, sizeof(double) * 324 * nb, c->stream), "blocks");
  const OpView A = op_view(m);
  if (!rc) rc = gather_diag_inverse(c, A, *g->pat, g->d_dinv, err);
  if (!rc) rc = neumann_blocks(c, A, *g->pat, g->d_dinv, g->d_neu, true);
  if (!rc && target) rc = local_inverse_blocks(c, A, *g->pat, target);
  if (!rc) rc = graph_fill(c, g, m, G, g->d_dinv, g->d_neu, target);
  int herr = 0;
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "status");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "network inputs");
  if (!rc && herr) rc = set_error(c, HFPX_ERR_SINGULAR, "a diagonal block of the matrix is singular");
  if (rc) {
    graph_destroy(g);
    return rc;
  }
  *out = g;
  return 0;
}

void graph_destroy(hfpx_gnn_graph* g) {
  if (!g) return;
  g->pat.reset();
  pool_free_many(g->allocs.data(), g->allocs.size());
  delete g;
}

}  // namespace gnn

// The learned corrections, added to pc's Neumann blocks.  The graph of the
// mesh (pattern, geometry inputs, activation buffers) is built by the first
// call and kept with the mesh; each call fills in the operator inputs from
// pc's diagonal inverses and Neumann blocks and runs one forward pass.
int gnn_correct_blocks(hfpx_ctx* c, const hfpx_gnn* net, const hfpx_mesh* mesh, const hfpx_matrix* m,
                       hfpx_precond* pc, double shear_m) {
  hfpx_mesh* mm = const_cast<hfpx_mesh*>(mesh);
  if (!mm->gnn_graph) {
    int rc = gnn::graph_prepare(c, mesh, &mm->gnn_graph);
    if (rc) return rc;
  }
  hfpx_gnn_graph* g = mm->gnn_graph;
  int rc = gnn::graph_fill(c, g, m, shear_m, pc->d_dinv, pc->d_blocks, nullptr);
  if (!rc) rc = gnn::forward(c, net, g);
  if (!rc) {
    ++g_launches;
    gnn::apply_outputs_kernel<<<(unsigned)g->pat->blocks(), 352, 0, c->stream>>>(
        g->n_nodes, g->pat->d_ptr, g->pat->d_dst, g->on, g->oe, g->d_rot, g->d_size, shear_m, pc->d_blocks);
    rc = check_cuda(c, cudaGetLastError(), "learned blocks");
  }
  return rc;
}

void gnn_graph_release(hfpx_gnn_graph* g) { gnn::graph_destroy(g); }

bool graph_host_inputs(const hfpx_mesh* mesh, const NearPattern& pat, GraphHostInputs* out) {
  return gnn::host_inputs(mesh, pat, out);
}

}  // namespace hfpx

// ------------------------------------------------------------------ C-ABI
extern "C" {

int hfpx_gnn_create(hfpx_ctx* c, uint64_t seed, hfpx_gnn** out) {
  if (!c || !out) return HFPX_ERR_ARG;
  *out = nullptr;
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  hfpx_gnn* net = new (std::nothrow) hfpx_gnn;
  if (!net) return set_error(c, HFPX_ERR_NOMEM, "network");
  int rc = gnn::net_alloc(c, net);
  if (!rc) {
    // He-uniform hidden weights, zero biases; the output heads start at zero,
    // so an untrained network gives the Neumann blocks unchanged
    std::vector<float> h((size_t)net->n_params, 0.f);
    std::mt19937_64 rng(seed);
    for (int t = 0; t < gnn::kTensors - 2; ++t) {
      const gnn::Shape s = gnn::tensor_shape(t);
      const float lim = std::sqrt(6.f / (float)s.rows);
      std::uniform_real_distribution<float> u(-lim, lim);
      for (int64_t k = 0; k < (int64_t)s.rows * s.cols; ++k) h[net->w_off[t] + k] = u(rng);
    }
    rc = gnn::net_upload(c, net, h.data());
  }
  if (rc) {
    hfpx_gnn_destroy(net);
    return rc;
  }
  *out = net;
  return HFPX_OK;
}

int hfpx_gnn_destroy(hfpx_gnn* net) {
  if (!net) return HFPX_OK;
  for (void* p : {(void*)net->d_w, (void*)net->d_wb, (void*)net->d_g, (void*)net->d_m, (void*)net->d_v})
    if (p) cudaFree(p);
  delete net;
  return HFPX_OK;
}

int64_t hfpx_gnn_param_count(const hfpx_gnn* net) { return net ? net->n_params : -1; }

int hfpx_gnn_get_params(hfpx_ctx* c, const hfpx_gnn* net, float* out) {
  if (!c) return HFPX_ERR_ARG;
  if (!net || !out) return set_error(c, HFPX_ERR_ARG, "null argument");
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  int rc = check_cuda(c, cudaMemcpyAsync(out, net->d_w, sizeof(float) * net->n_params, cudaMemcpyDeviceToHost, c->stream),
                      "parameters");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "parameters");
  return rc;
}

int hfpx_gnn_set_params(hfpx_ctx* c, hfpx_gnn* net, const float* in) {
  if (!c) return HFPX_ERR_ARG;
  if (!net || !in) return set_error(c, HFPX_ERR_ARG, "null argument");
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  for (int64_t k = 0; k < net->n_params; ++k)
    if (!std::isfinite(in[k])) return set_error(c, HFPX_ERR_ARG, "non-finite parameter");
  return gnn::net_upload(c, net, in);
}

// File: "HFPXGNN1", int32 tensors, then (rows, cols) per tensor, int64 Adam
// step, then the FP32 parameters (each weight row-major, then its bias).
int hfpx_gnn_save(hfpx_ctx* c, const hfpx_gnn* net, const char* path) {
  if (!c) return HFPX_ERR_ARG;
  if (!net || !path) return set_error(c, HFPX_ERR_ARG, "null argument");
  std::vector<float> h((size_t)net->n_params);
  int rc = hfpx_gnn_get_params(c, net, h.data());
  if (rc) return rc;
  FILE* f = std::fopen(path, "wb");
  if (!f) return set_error(c, HFPX_ERR_ARG, std::string("cannot write ") + path);
  const char magic[8] = {'H', 'F', 'P', 'X', 'G', 'N', 'N', '1'};
  const int32_t nt = gnn::kTensors;
  bool ok = std::fwrite(magic, 1, 8, f) == 8 && std::fwrite(&nt, 4, 1, f) == 1;
  for (int t = 0; t < gnn::kTensors && ok; ++t) {
    const gnn::Shape s = gnn::tensor_shape(t);
    const int32_t rcn[2] = {s.rows, s.cols};
    ok = std::fwrite(rcn, 4, 2, f) == 2;
  }
  ok = ok && std::fwrite(&net->step, 8, 1, f) == 1 && std::fwrite(h.data(), 4, h.size(), f) == h.size();
  ok = (std::fclose(f) == 0) && ok;
  return ok ? HFPX_OK : set_error(c, HFPX_ERR_ARG, std::string("write failed: ") + path);
}

int hfpx_gnn_load(hfpx_ctx* c, const char* path, hfpx_gnn** out) {
  if (!c || !out) return HFPX_ERR_ARG;
  *out = nullptr;
  if (!path) return set_error(c, HFPX_ERR_ARG, "null path");
  FILE* f = std::fopen(path, "rb");
  if (!f) return set_error(c, HFPX_ERR_ARG, std::string("cannot read ") + path);
  char magic[8];
  int32_t nt = 0;
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "HFPXGNN1", 8) == 0 && std::fread(&nt, 4, 1, f) == 1 &&
            nt == gnn::kTensors;
  for (int t = 0; t < gnn::kTensors && ok; ++t) {
    int32_t rcn[2];
    const gnn::Shape s = gnn::tensor_shape(t);
    ok = std::fread(rcn, 4, 2, f) == 2 && rcn[0] == s.rows && rcn[1] == s.cols;
  }
  int64_t step = 0;
  ok = ok && std::fread(&step, 8, 1, f) == 1;
  hfpx_gnn* net = nullptr;
  int rc = HFPX_OK;
  if (ok) rc = hfpx_gnn_create(c, 0, &net);
  std::vector<float> h;
  if (ok && !rc) {
    h.resize((size_t)net->n_params);
    ok = std::fread(h.data(), 4, h.size(), f) == h.size();
  }
  std::fclose(f);
  if (!ok) {
    hfpx_gnn_destroy(net);
    return rc ? rc : set_error(c, HFPX_ERR_ARG, std::string("not a network file of this layout: ") + path);
  }
  if (!rc) rc = hfpx_gnn_set_params(c, net, h.data());
  if (rc) {
    hfpx_gnn_destroy(net);
    return rc;
  }
  net->step = step;
  *out = net;
  return HFPX_OK;
}

int hfpx_gnn_graph_create(hfpx_ctx* c, const hfpx_mesh* mesh, const hfpx_matrix* m, double shear_m, int with_targets,
                          hfpx_gnn_graph** out) {
  if (!c || !out) return HFPX_ERR_ARG;
  *out = nullptr;
  if (!mesh || !m) return set_error(c, HFPX_ERR_ARG, "null mesh or matrix");
  if (m->n != 18 * mesh->n_el)
    return set_error(c, HFPX_ERR_ARG, "the network needs a matrix of 18 DoF per element (no fixed DoF, no border)");
  if (m->factored == 1) return set_error(c, HFPX_ERR_STATE, "the matrix holds FP64 LU factors, not the operator");
  if (!(shear_m > 0)) return set_error(c, HFPX_ERR_ARG, "bad shear modulus");
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  return gnn::graph_create(c, mesh, m, shear_m, with_targets != 0, out);
}

int hfpx_gnn_graph_destroy(hfpx_gnn_graph* g) {
  gnn::graph_destroy(g);
  return HFPX_OK;
}

int hfpx_gnn_graph_dims(const hfpx_gnn_graph* g, int64_t* n_nodes, int64_t* n_edges) {
  if (!g || !n_nodes || !n_edges) return HFPX_ERR_ARG;
  *n_nodes = g->n_nodes;
  *n_edges = g->n_edges;
  return HFPX_OK;
}

int hfpx_gnn_graph_data(hfpx_ctx* c, const hfpx_gnn_graph* g, float* xn, float* xe, int32_t* src, int32_t* dst,
                        float* tn, float* te) {
  if (!c) return HFPX_ERR_ARG;
  if (!g) return set_error(c, HFPX_ERR_ARG, "null graph");
  if ((tn || te) && !g->tn) return set_error(c, HFPX_ERR_STATE, "the graph has no targets");
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  // the graph's buffers are written on the context's stream
  if (int rc = check_cuda(c, cudaStreamSynchronize(c->stream), "graph")) return rc;
  const int64_t n = g->n_nodes, E = g->n_edges;
  std::vector<__nv_bfloat16> b;
  int rc = 0;
  auto down_bf16 = [&](const __nv_bfloat16* d, int64_t count, float* out) {
    b.resize((size_t)count);
    if (!rc) rc = check_cuda(c, cudaMemcpy(b.data(), d, sizeof(__nv_bfloat16) * count, cudaMemcpyDeviceToHost), "data");
    if (!rc)
      for (int64_t k = 0; k < count; ++k) out[k] = __bfloat162float(b[k]);
  };
  if (xn) down_bf16(g->xn, n * gnn::kFN, xn);
  if (xe) down_bf16(g->xe, E * gnn::kFE, xe);
  if (src) std::memcpy(src, g->pat->idx.data(), sizeof(int32_t) * E);
  if (dst) std::memcpy(dst, g->pat->dst.data(), sizeof(int32_t) * E);
  if (tn && !rc) rc = check_cuda(c, cudaMemcpy(tn, g->tn, sizeof(float) * n * gnn::kOut, cudaMemcpyDeviceToHost), "targets");
  if (te && !rc) rc = check_cuda(c, cudaMemcpy(te, g->te, sizeof(float) * E * gnn::kOut, cudaMemcpyDeviceToHost), "targets");
  return rc;
}

int hfpx_gnn_forward(hfpx_ctx* c, const hfpx_gnn* net, hfpx_gnn_graph* g, float* out_nodes, float* out_edges) {
  if (!c) return HFPX_ERR_ARG;
  if (!net || !g) return set_error(c, HFPX_ERR_ARG, "null argument");
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  int rc = gnn::forward(c, net, g);
  if (!rc && out_nodes)
    rc = check_cuda(c, cudaMemcpyAsync(out_nodes, g->on, sizeof(float) * g->n_nodes * gnn::kOut, cudaMemcpyDeviceToHost,
                                       c->stream), "outputs");
  if (!rc && out_edges)
    rc = check_cuda(c, cudaMemcpyAsync(out_edges, g->oe, sizeof(float) * g->n_edges * gnn::kOut, cudaMemcpyDeviceToHost,
                                       c->stream), "outputs");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "network forward");
  return rc;
}

int hfpx_gnn_gradients(hfpx_ctx* c, hfpx_gnn* net, hfpx_gnn_graph* g, double* loss, float* grads) {
  if (!c) return HFPX_ERR_ARG;
  if (!net || !g || !loss) return set_error(c, HFPX_ERR_ARG, "null argument");
  if (!g->tn) return set_error(c, HFPX_ERR_STATE, "the graph has no targets");
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  int rc = gnn::forward(c, net, g);
  if (!rc) rc = gnn::backward(c, net, g);
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(loss, g->loss, sizeof(double), cudaMemcpyDeviceToHost, c->stream), "loss");
  if (!rc && grads)
    rc = check_cuda(c, cudaMemcpyAsync(grads, net->d_g, sizeof(float) * net->n_params, cudaMemcpyDeviceToHost, c->stream),
                    "gradients");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "network gradients");
  return rc;
}

int hfpx_gnn_train(hfpx_ctx* c, hfpx_gnn* net, hfpx_gnn_graph* g, int steps, double lr, double* losses) {
  if (!c) return HFPX_ERR_ARG;
  if (!net || !g || steps < 1 || !(lr > 0)) return set_error(c, HFPX_ERR_ARG, "bad training arguments");
  if (!g->tn) return set_error(c, HFPX_ERR_STATE, "the graph has no targets");
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  int rc = 0;
  for (int s = 0; s < steps && !rc; ++s) {
    rc = gnn::forward(c, net, g);
    if (!rc) rc = gnn::backward(c, net, g);
    if (!rc && losses)
      rc = check_cuda(c, cudaMemcpyAsync(losses + s, g->loss, sizeof(double), cudaMemcpyDeviceToHost, c->stream), "loss");
    if (!rc) rc = gnn::adam(c, net, (float)lr);
  }
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "network training");
  return rc;
}

}  // extern "C"
