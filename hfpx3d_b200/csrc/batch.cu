// The batched workload: many meshes of uneven sizes, each with many load
// cases, assembled, factored and solved in one CUDA-graph launch.
//
// Reference counterpart, per mesh: make_3dbem_matrix_s
// (src/Solvers/system_assembly.cpp:30-219), add_s_inf_to_3dbem_rhs (:222-274)
// and il::LU's dgetrf/dgetrs (il/linear_algebra/dense/factorization/LU.h:79-120),
// called once per mesh and once per load case by a caller's loop.
//
// Design (one GPU, every mesh at once, level-synchronous):
//   * assembly: one launch over (mesh, source element, target tile) tasks
//     writes each mesh's mixed-precision operator (FP32 entries, FP32 low
//     parts on the near-field blocks) and its FP32 copy for the factor;
//   * right-hand sides: the traction right-hand side is linear in the in-situ
//     stress (rhs = -n . s_inf per collocation point), so the 6 unit stress
//     states are solved and every load case is their combination;
//   * factorisation: right-looking blocked LU of every FP32 copy, block nb
//     (multiple of 32), 32-column panels with tournament pivoting (TSLU:
//     every chunk of rows proposes 32 pivot rows by partial pivoting, one
//     more partial-pivoting pass over the proposals picks the panel's rows;
//     Grigori, Demmel, Xiang 2011), full-row interchanges recorded as LAPACK
//     ipiv, U rows of each panel by the unit-lower panel inverse, the block's
//     own rows and columns updated per panel, then one trailing update per
//     block (C -= L21 U12), a tiled SIMT FP32 GEMM over every mesh's tiles;
//   * solve: FP32 forward / backward substitution of the 6 basis right-hand
//     sides, one CTA per mesh, FP64 iterative refinement against the
//     mixed-precision operator (products in FP64) to the requested max-norm
//     residual; converged meshes skip later refinement steps;
//   * every launch of a stage covers all meshes that still have work there
//     (a precomputed item list per launch), and the whole run is captured
//     once into a CUDA graph and replayed.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>
#include "engine_internal.h"

namespace hfpx {
namespace {

constexpr int kPw = 32;              // panel width
constexpr int kBasis = 6;            // unit in-situ stress states
constexpr int kMaxChunks = 40;       // leaf chunks per panel (rows / leaf rows)
constexpr int kBt = 256;             // threads of the panel kernels

// Per-mesh data the kernels read (device array, one per mesh).
struct BMesh {
  float* F;          // FP32 factor (ld x n), LU in place
  const float* A;    // FP32 operator entries
  const float* lo;   // near-field low parts (blocks x 324)
  const int32_t* rptr;  // near-field row view of the mesh's pattern
  const int32_t* rblk;
  const int32_t* rcol;
  int32_t* piv;      // ipiv (0-based, LAPACK order)
  int32_t* perm;     // row permutation of the factor
  float* diag;       // the current panel's L11\U11 (32 x 32, column-major)
  int32_t* prow;     // the current panel's pivot rows (32)
  int32_t* cand;     // leaf proposals (kMaxChunks x 32)
  double* B;         // right-hand sides (n x kBasis), then the solutions' residuals
  double* X;         // solutions (n x kBasis)
  float* W;          // FP32 work vector block (n x kBasis)
  int64_t n, ld, n_el;
  int info;          // first zero pivot (1-based column), 0 none
  int done;          // refinement converged
  int iters;         // refinement corrections applied
  double bmax[kBasis];
};

// ------------------------------------------------------- panel: leaves
// Item: mesh, first row, rows, chunk index, panel column c0, width w.
struct LeafItem {
  int32_t mesh, r0, rows, chunk, c0, w;
};

// Partial pivoting on one chunk of rows (rows x w in shared memory, row i
// of the chunk at a + i lda): the w rows it chooses, in order, go to cho[].
// Rows are not moved: a chosen row is marked and left out of later steps,
// so each column takes two CTA barriers (the candidates' maxima, then the
// elimination).  After the call a chosen row j holds its multipliers in
// columns < j and its U row from column j on (L11\U11 row j).  Ties go to
// the lower row id (the first maximum, as LAPACK's idamax).
__device__ void chunk_gepp(float* a, int lda, const int32_t* rid, int rows, int w, unsigned char* chosen, int* cho) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  __shared__ float s_val[kBt / 32];
  __shared__ int s_id[kBt / 32], s_pos[kBt / 32];
  for (int i = tid; i < rows; i += kBt) chosen[i] = 0;
  __syncthreads();
  const int steps = min(rows, w);
  for (int j = 0; j < steps; ++j) {
    float best = -1.f;
    int bi = 0x7fffffff, bp = 0;
    for (int i = tid; i < rows; i += kBt) {
      if (chosen[i]) continue;
      const float v = fabsf(a[i * lda + j]);
      const int r = rid[i];
      if (v > best || (v == best && r < bi)) {
        best = v;
        bi = r;
        bp = i;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const float ov = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      const int op = __shfl_xor_sync(0xffffffffu, bp, o);
      if (ov > best || (ov == best && oi < bi)) {
        best = ov;
        bi = oi;
        bp = op;
      }
    }
    if (lane == 0) {
      s_val[warp] = best;
      s_id[warp] = bi;
      s_pos[warp] = bp;
    }
    __syncthreads();
    // every thread finds the same winner
    float b = s_val[0];
    int id = s_id[0], p = s_pos[0];
    for (int k = 1; k < kBt / 32; ++k)
      if (s_val[k] > b || (s_val[k] == b && s_id[k] < id)) {
        b = s_val[k];
        id = s_id[k];
        p = s_pos[k];
      }
    if (tid == 0) {
      cho[j] = p;
      chosen[p] = 1;
    }
    const float piv = a[p * lda + j];
    const float inv = piv != 0.f ? 1.f / piv : 0.f;
    const float* pr = a + p * lda;
    for (int i = tid; i < rows; i += kBt) {
      if (i == p || chosen[i]) continue;
      float* ar = a + i * lda;
      const float l = ar[j] * inv;
      ar[j] = l;
      for (int c = j + 1; c < w; ++c) ar[c] = fmaf(-l, pr[c], ar[c]);
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kBt) leaf_kernel(BMesh* __restrict__ meshes, const LeafItem* __restrict__ items,
                                                   int leaf_rows) {
  extern __shared__ __align__(16) unsigned char smem[];
  const LeafItem it = items[blockIdx.x];
  const BMesh& M = meshes[it.mesh];
  float* a = reinterpret_cast<float*>(smem);
  const int lda = kPw + 1;
  int32_t* rid = reinterpret_cast<int32_t*>(a + (size_t)leaf_rows * lda);
  unsigned char* chosen = reinterpret_cast<unsigned char*>(rid + leaf_rows);
  __shared__ int cho[kPw];
  for (int t = threadIdx.x; t < it.rows * it.w; t += kBt) {
    const int i = t % it.rows, c = t / it.rows;
    a[i * lda + c] = M.F[(int64_t)(it.r0 + i) + M.ld * (it.c0 + c)];
  }
  for (int i = threadIdx.x; i < it.rows; i += kBt) rid[i] = it.r0 + i;
  __syncthreads();
  chunk_gepp(a, lda, rid, it.rows, it.w, chosen, cho);
  for (int j = threadIdx.x; j < kPw; j += kBt)
    M.cand[it.chunk * kPw + j] = j < min(it.rows, it.w) ? rid[cho[j]] : -1;
}

// --------------------------------------------------- panel: tournament
// Item: mesh, panel column c0, width w, chunks.  Partial pivoting over the
// chunks' proposals (their original rows) picks the panel's w pivot rows;
// the top w x w block of that elimination is L11\U11 of the pivot rows in
// order.  One thread then turns the pivot rows into LAPACK's interchanges.
struct PanelItem {
  int32_t mesh, c0, w, chunks;
};

__global__ void __launch_bounds__(kBt) tourn_kernel(BMesh* __restrict__ meshes, const PanelItem* __restrict__ items,
                                                    int cap) {
  extern __shared__ __align__(16) unsigned char smem[];
  const PanelItem it = items[blockIdx.x];
  BMesh& M = meshes[it.mesh];
  const int lda = kPw + 1;
  float* a = reinterpret_cast<float*>(smem);  // cap candidate rows (the launch's largest chunk count x 32)
  int32_t* rid = reinterpret_cast<int32_t*>(a + (size_t)cap * lda);
  unsigned char* chosen = reinterpret_cast<unsigned char*>(rid + cap);
  __shared__ int cho[kPw];
  __shared__ int n_rows;
  if (threadIdx.x == 0) {
    int k = 0;
    for (int c = 0; c < it.chunks; ++c)
      for (int j = 0; j < kPw; ++j) {
        const int r = M.cand[c * kPw + j];
        if (r >= 0) rid[k++] = r;
      }
    n_rows = k;
  }
  __syncthreads();
  const int rows = n_rows;
  for (int t = threadIdx.x; t < rows * it.w; t += kBt) {
    const int i = t % rows, c = t / rows;
    a[i * lda + c] = M.F[(int64_t)rid[i] + M.ld * (it.c0 + c)];
  }
  __syncthreads();
  chunk_gepp(a, lda, rid, rows, it.w, chosen, cho);
  // L11\U11 (column-major 32 x 32): row j is the j-th chosen row; the pivot rows
  for (int t = threadIdx.x; t < it.w * it.w; t += kBt) {
    const int i = t % it.w, c = t / it.w;
    M.diag[i + kPw * c] = a[cho[i] * lda + c];
  }
  for (int j = threadIdx.x; j < it.w; j += kBt) M.prow[j] = rid[cho[j]];
  if (threadIdx.x == 0) {
    for (int j = 0; j < it.w; ++j)
      if (a[cho[j] * lda + j] == 0.f && M.info == 0) M.info = it.c0 + j + 1;
    // interchanges: position c0 + j receives pivot row prow[j]; rows moved
    // earlier are tracked in a small map (position -> original row)
    int pos[2 * kPw], org[2 * kPw], n_map = 0;
    auto content = [&](int p) {
      for (int k = 0; k < n_map; ++k)
        if (pos[k] == p) return org[k];
      return p;
    };
    auto set = [&](int p, int r) {
      for (int k = 0; k < n_map; ++k)
        if (pos[k] == p) {
          org[k] = r;
          return;
        }
      pos[n_map] = p;
      org[n_map] = r;
      ++n_map;
    };
    for (int j = 0; j < it.w; ++j) {
      const int target = rid[cho[j]];
      int where = target;
      for (int k = 0; k < n_map; ++k)
        if (org[k] == target) {
          where = pos[k];
          break;
        }
      const int here = it.c0 + j;
      M.piv[here] = where;
      if (where != here) {
        const int ch = content(here);
        set(where, ch);
        set(here, target);
      }
    }
  }
}

// ------------------------------------------------ panel: interchanges
// Item: mesh, first column, columns, panel column c0, width w.  Each thread
// applies the panel's interchanges, in order, to one column.
struct ColItem {
  int32_t mesh, q0, cols, c0, w;
};

__global__ void __launch_bounds__(256) swap_rows_kernel(BMesh* __restrict__ meshes, const ColItem* __restrict__ items) {
  const ColItem it = items[blockIdx.x];
  const BMesh& M = meshes[it.mesh];
  __shared__ int32_t p[kPw];
  if (threadIdx.x < it.w) p[threadIdx.x] = M.piv[it.c0 + threadIdx.x];
  __syncthreads();
  const int q = threadIdx.x;
  if (q >= it.cols) return;
  float* col = M.F + M.ld * (int64_t)(it.q0 + q);
  for (int j = 0; j < it.w; ++j) {
    const int r = it.c0 + j, s = p[j];
    if (s != r) {
      const float t = col[r];
      col[r] = col[s];
      col[s] = t;
    }
  }
}

// ------------------------------------------------- panel: L21 and L11\U11
// Item: mesh, first row, rows, panel column c0, width w.  Rows of the panel
// block take L11\U11; rows below solve l U11 = a.
struct RowItem {
  int32_t mesh, r0, rows, c0, w;
};

__global__ void __launch_bounds__(256) l21_kernel(BMesh* __restrict__ meshes, const RowItem* __restrict__ items) {
  const RowItem it = items[blockIdx.x];
  const BMesh& M = meshes[it.mesh];
  __shared__ float d[kPw * kPw];
  for (int t = threadIdx.x; t < it.w * kPw; t += blockDim.x) d[t] = M.diag[t];
  __syncthreads();
  const int i = threadIdx.x;
  if (i >= it.rows) return;
  const int64_t r = it.r0 + i;
  float* row = M.F + r + M.ld * (int64_t)it.c0;
  if (r < it.c0 + it.w) {
    const int j0 = (int)(r - it.c0);
    for (int c = 0; c < it.w; ++c) row[M.ld * c] = d[j0 + kPw * c];
    return;
  }
  float l[kPw];
#pragma unroll
  for (int c = 0; c < kPw; ++c)
    if (c < it.w) l[c] = row[M.ld * c];
#pragma unroll
  for (int c = 0; c < kPw; ++c)
    if (c < it.w) {
      float v = l[c];
#pragma unroll
      for (int k = 0; k < c; ++k) v = fmaf(-l[k], d[k + kPw * c], v);
      const float u = d[c + kPw * c];
      l[c] = u != 0.f ? v / u : 0.f;
    }
#pragma unroll
  for (int c = 0; c < kPw; ++c)
    if (c < it.w) row[M.ld * c] = l[c];
}

// ------------------------------------------------- panel: U rows
// U rows of a panel = L11^-1 A12 for the item's columns: one thread per
// column, forward substitution with the panel's unit lower L11 (read from
// the factor, where the panel step left it).
__global__ void __launch_bounds__(256) u12_kernel(BMesh* __restrict__ meshes, const ColItem* __restrict__ items) {
  const ColItem it = items[blockIdx.x];
  const BMesh& M = meshes[it.mesh];
  __shared__ float d[kPw * kPw];
  for (int t = threadIdx.x; t < it.w * kPw; t += blockDim.x) {
    const int i = t % kPw, k = t / kPw;
    d[t] = i < it.w ? M.F[(int64_t)(it.c0 + i) + M.ld * (it.c0 + k)] : 0.f;
  }
  __syncthreads();
  const int q = threadIdx.x;
  if (q >= it.cols) return;
  float* col = M.F + M.ld * (int64_t)(it.q0 + q) + it.c0;
  float x[kPw];
#pragma unroll
  for (int i = 0; i < kPw; ++i)
    if (i < it.w) x[i] = col[i];
#pragma unroll
  for (int i = 0; i < kPw; ++i)
    if (i < it.w) {
      float v = x[i];
#pragma unroll
      for (int k = 0; k < i; ++k) v = fmaf(-d[i + kPw * k], x[k], v);
      x[i] = v;
    }
#pragma unroll
  for (int i = 0; i < kPw; ++i)
    if (i < it.w) col[i] = x[i];
}

// --------------------------------------------------------- tiled GEMM
// C -= L U on 64 x 64 tiles of one mesh's factor: C = F[r0.., q0..],
// L = F[r0.., k0 .. k0 + K), U = F[k0 .., q0..]; rows < r_end, columns <
// q_end.  256 threads, 4 x 4 outputs each, K in steps of 32 staged in
// shared memory; each thread's 16 entries of C are loaded together before
// they are written back.  Small tiles keep many CTAs per SM in flight: the
// rank-32 updates of the panels are bound by the latency of their loads.
struct GemmItem {
  int32_t mesh, r0, q0, r_end, q_end, k0, K;
};
constexpr int kGm = 64, kGk = 32;

__global__ void __launch_bounds__(256) bgemm_kernel(BMesh* __restrict__ meshes, const GemmItem* __restrict__ items) {
  const GemmItem it = items[blockIdx.x];
  const BMesh& M = meshes[it.mesh];
  __shared__ float Ls[kGk][kGm + 1];
  __shared__ float Us[kGk][kGm + 1];
  const int tid = threadIdx.x;
  const int tr = tid % 16, tc = tid / 16;  // rows tr + 16 i, columns tc + 16 j
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
  const int64_t ld = M.ld;
  float* F = M.F;
  for (int kk = 0; kk < it.K; kk += kGk) {
    for (int t = tid; t < kGm * kGk; t += 256) {
      const int r = t % kGm, k = t / kGm;
      const int64_t gr = it.r0 + r;
      const int gk = kk + k;
      Ls[k][r] = (gr < it.r_end && gk < it.K) ? F[gr + ld * (it.k0 + gk)] : 0.f;
    }
    for (int t = tid; t < kGm * kGk; t += 256) {
      const int k = t % kGk, q = t / kGk;
      const int64_t gq = it.q0 + q;
      const int gk = kk + k;
      Us[k][q] = (gq < it.q_end && gk < it.K) ? F[(it.k0 + gk) + ld * gq] : 0.f;
    }
    __syncthreads();
#pragma unroll 8
    for (int k = 0; k < kGk; ++k) {
      float lv[4], uv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) lv[i] = Ls[k][tr + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) uv[j] = Us[k][tc + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(lv[i], uv[j], acc[i][j]);
    }
    __syncthreads();
  }
  float c[4][4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int64_t gq = it.q0 + tc + 16 * j;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int64_t gr = it.r0 + tr + 16 * i;
      c[i][j] = (gq < it.q_end && gr < it.r_end) ? F[gr + ld * gq] : 0.f;
    }
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int64_t gq = it.q0 + tc + 16 * j;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int64_t gr = it.r0 + tr + 16 * i;
      if (gq < it.q_end && gr < it.r_end) F[gr + ld * gq] = c[i][j] - acc[i][j];
    }
  }
}

// ---------------------------------------- trailing update on tcgen05
// FP16 K-major operands of the block's trailing update C -= L21 U12 for the
// engine's grouped tensor-core kernel: the rows of L21 each scaled by a power
// of two into [2^14, 2^15) (the inverse kept per row for the epilogue), U12
// scaled as a whole the same way (alpha = -the inverse).
struct HalfItem {
  int32_t mesh, l0, count, k0, bend;  // local rows (L21) or columns (U12) [l0, l0 + count) of [bend, n)
};

__device__ __forceinline__ float pow2_scale(float amax, float* inv) {
  if (!(amax > 0.f)) {
    *inv = 1.f;
    return 1.f;
  }
  int ex;
  frexpf(amax, &ex);  // amax = f 2^ex, f in [0.5, 1)
  *inv = ldexpf(1.f, ex - 15);
  return ldexpf(1.f, 15 - ex);
}

constexpr int kHr = 32;  // L21 rows per CTA
__global__ void __launch_bounds__(256) l21_half_kernel(BMesh* __restrict__ meshes, const HalfItem* __restrict__ items,
                                                       __half* __restrict__ L16, const int64_t* __restrict__ l16off,
                                                       float* __restrict__ rs, const int64_t* __restrict__ rsoff,
                                                       int nb) {
  extern __shared__ float tile[];  // kHr x (nb + 1)
  const HalfItem it = items[blockIdx.x];
  const BMesh& M = meshes[it.mesh];
  const int ldt = nb + 1;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int t = tid; t < kHr * nb; t += 256) {
    const int r = t % kHr, c = t / kHr;
    tile[r * ldt + c] = r < it.count ? M.F[(int64_t)(it.bend + it.l0 + r) + M.ld * (it.k0 + c)] : 0.f;
  }
  __syncthreads();
  __shared__ float sc[kHr];
  for (int r = warp; r < kHr; r += 8) {
    float m = 0.f;
    for (int c = lane; c < nb; c += 32) m = fmaxf(m, fabsf(tile[r * ldt + c]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) {
      float inv;
      sc[r] = pow2_scale(m, &inv);
      if (r < it.count) rs[rsoff[it.mesh] + it.l0 + r] = inv;
    }
  }
  __syncthreads();
  __half* out = L16 + l16off[it.mesh] + (int64_t)it.l0 * nb;
  for (int t = tid; t < it.count * nb; t += 256) {
    const int r = t / nb, c = t % nb;
    out[(int64_t)r * nb + c] = __float2half_rn(tile[r * ldt + c] * sc[r]);
  }
}

__global__ void __launch_bounds__(256) u12_amax_kernel(BMesh* __restrict__ meshes, const HalfItem* __restrict__ items,
                                                       unsigned* __restrict__ amax, int nb) {
  const HalfItem it = items[blockIdx.x];
  const BMesh& M = meshes[it.mesh];
  float m = 0.f;
  for (int t = threadIdx.x; t < it.count * nb; t += 256) {
    const int q = t / nb, k = t % nb;
    m = fmaxf(m, fabsf(M.F[(int64_t)(it.k0 + k) + M.ld * (it.bend + it.l0 + q)]));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(amax + it.mesh, __float_as_uint(m));
}

__global__ void __launch_bounds__(256) u12_half_kernel(BMesh* __restrict__ meshes, const HalfItem* __restrict__ items,
                                                       const unsigned* __restrict__ amax, __half* __restrict__ U16,
                                                       const int64_t* __restrict__ u16off, float* __restrict__ alpha,
                                                       int nb) {
  const HalfItem it = items[blockIdx.x];
  const BMesh& M = meshes[it.mesh];
  float inv;
  const float su = pow2_scale(__uint_as_float(amax[it.mesh]), &inv);
  if (it.l0 == 0 && threadIdx.x == 0) alpha[it.mesh] = -inv;
  __half* out = U16 + u16off[it.mesh] + (int64_t)it.l0 * nb;
  for (int t = threadIdx.x; t < it.count * nb; t += 256) {
    const int q = t / nb, k = t % nb;
    out[(int64_t)q * nb + k] = __float2half_rn(M.F[(int64_t)(it.k0 + k) + M.ld * (it.bend + it.l0 + q)] * su);
  }
}

__global__ void zero_u32_kernel(unsigned* p, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = 0u;
}

// --------------------------------------------------------------- solve
// The factor's row permutation from ipiv (one CTA per mesh, in shared memory).
__global__ void __launch_bounds__(256) perm_kernel(BMesh* __restrict__ meshes, int max_n) {
  extern __shared__ int32_t sp[];
  BMesh& M = meshes[blockIdx.x];
  const int n = (int)M.n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) sp[i] = i;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int i = 0; i < n; ++i) {
      const int p = M.piv[i];
      if (p != i) {
        const int t = sp[i];
        sp[i] = sp[p];
        sp[p] = t;
      }
    }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) M.perm[i] = sp[i];
  (void)max_n;
}

// W = P r in FP32 (r = B, the current residual), then W = U^-1 L^-1 W, and
// X += W in FP64.  One thread-block cluster of kSc CTAs per mesh (meshes
// largest first, so the longest solves start first).  The triangles are
// taken in 32-row blocks: every CTA of the cluster solves the block's 32 x 32
// triangle itself (a warp per right-hand side, shuffles, the block staged in
// shared memory), then updates its slice of the rows beyond the block; a
// cluster barrier (release / acquire at cluster scope) separates the blocks,
// so the cluster's SMs share the factor's bandwidth.
constexpr int kSt = 256, kSc = 4;

// rows [r0, r1) of W (n x 6) -= T[rows, c0 .. c0 + bw) Y (Y = yb, bw x 6),
// T the factor; all 32 loads of a row issued together when bw is 32
__device__ __forceinline__ void rows_update(const float* __restrict__ F, int64_t ld, float* __restrict__ W, int n,
                                            int r0, int r1, int c0, int bw, const float (*yb)[kBasis]) {
  for (int i = r0 + threadIdx.x; i < r1; i += kSt) {
    float acc[kBasis];
#pragma unroll
    for (int c = 0; c < kBasis; ++c) acc[c] = W[i + (int64_t)n * c];
    const float* row = F + i + ld * (int64_t)c0;
    if (bw == kPw) {
      float l[kPw];
#pragma unroll
      for (int k = 0; k < kPw; ++k) l[k] = row[ld * k];
#pragma unroll
      for (int k = 0; k < kPw; ++k)
#pragma unroll
        for (int c = 0; c < kBasis; ++c) acc[c] = fmaf(-l[k], yb[k][c], acc[c]);
    } else {
      for (int k = 0; k < bw; ++k) {
        const float l = row[ld * k];
#pragma unroll
        for (int c = 0; c < kBasis; ++c) acc[c] = fmaf(-l, yb[k][c], acc[c]);
      }
    }
#pragma unroll
    for (int c = 0; c < kBasis; ++c) W[i + (int64_t)n * c] = acc[c];
  }
}

__device__ __forceinline__ void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ unsigned cluster_rank_u() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

// this CTA's slice of rows [r0, r1) (contiguous, in 32-row units)
__device__ __forceinline__ void cta_slice(int r0, int r1, unsigned rank, int& s0, int& s1) {
  const int span = r1 - r0;
  const int per = ((span + kSc - 1) / kSc + 31) / 32 * 32;
  s0 = min(r1, r0 + (int)rank * per);
  s1 = min(r1, s0 + per);
}

__global__ void __cluster_dims__(kSc, 1, 1) __launch_bounds__(kSt, 2)
    solve_kernel(BMesh* __restrict__ meshes, const int32_t* __restrict__ order, int first) {
  BMesh& M = meshes[order[blockIdx.x / kSc]];
  if (!first && M.done) return;  // the whole cluster returns together
  const unsigned rank = cluster_rank_u();
  if (!first && threadIdx.x == 0 && rank == 0) ++M.iters;
  const int n = (int)M.n;
  const int64_t ld = M.ld;
  const float* F = M.F;
  float* W = M.W;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  __shared__ float yb[kPw][kBasis];
  __shared__ float Db[kPw][kPw + 1];  // the current 32 x 32 diagonal block
  {
    int s0, s1;
    cta_slice(0, n, rank, s0, s1);
    for (int t = tid; t < (s1 - s0) * kBasis; t += kSt) {
      const int i = s0 + t % (s1 - s0), c = t / (s1 - s0);
      W[i + (int64_t)n * c] = (float)M.B[M.perm[i] + (int64_t)n * c];
    }
  }
  cluster_barrier();
  // forward: unit lower L
  for (int b0 = 0; b0 < n; b0 += kPw) {
    const int bw = min(kPw, n - b0);
    for (int t = tid; t < kPw * kPw; t += kSt) {
      const int r = t % kPw, k = t / kPw;
      if (r < bw && k < bw) Db[r][k] = F[(b0 + r) + ld * (b0 + k)];
    }
    __syncthreads();
    if (warp < kBasis) {
      float y = lane < bw ? W[b0 + lane + (int64_t)n * warp] : 0.f;
      for (int k = 0; k < bw; ++k) {
        const float yk = __shfl_sync(0xffffffffu, y, k);
        if (lane > k && lane < bw) y = fmaf(-Db[lane][k], yk, y);
      }
      if (lane < bw) yb[lane][warp] = y;
    }
    __syncthreads();
    int s0, s1;
    cta_slice(b0 + bw, n, rank, s0, s1);
    rows_update(F, ld, W, n, s0, s1, b0, bw, yb);
    cluster_barrier();  // every CTA has read W[b0 .. b0 + bw) and updated its rows
    if (rank == 0 && warp < kBasis && lane < bw) W[b0 + lane + (int64_t)n * warp] = yb[lane][warp];
  }
  cluster_barrier();
  // backward: upper U, blocks from the bottom; rows above the block take
  // the block's contribution
  const int nb_blocks = (n + kPw - 1) / kPw;
  for (int bb = nb_blocks - 1; bb >= 0; --bb) {
    const int b0 = bb * kPw, bw = min(kPw, n - b0);
    for (int t = tid; t < kPw * kPw; t += kSt) {
      const int r = t % kPw, k = t / kPw;
      if (r < bw && k < bw) Db[r][k] = F[(b0 + r) + ld * (b0 + k)];
    }
    __syncthreads();
    if (warp < kBasis) {
      float y = lane < bw ? W[b0 + lane + (int64_t)n * warp] : 0.f;
      for (int k = bw - 1; k >= 0; --k) {
        if (lane == k) {
          const float u = Db[k][k];
          y = u != 0.f ? y / u : 0.f;
        }
        const float yk = __shfl_sync(0xffffffffu, y, k);
        if (lane < k) y = fmaf(-Db[lane][k], yk, y);
      }
      if (lane < bw) yb[lane][warp] = y;
    }
    __syncthreads();
    int s0, s1;
    cta_slice(0, b0, rank, s0, s1);
    rows_update(F, ld, W, n, s0, s1, b0, bw, yb);
    cluster_barrier();
    if (rank == 0 && warp < kBasis && lane < bw) W[b0 + lane + (int64_t)n * warp] = yb[lane][warp];
  }
  cluster_barrier();
  {
    int s0, s1;
    cta_slice(0, n, rank, s0, s1);
    for (int t = tid; t < (s1 - s0) * kBasis; t += kSt) {
      const int64_t i = s0 + t % (s1 - s0), c = t / (s1 - s0);
      const double v = (double)W[i + n * c];
      M.X[i + n * c] = first ? v : M.X[i + n * c] + v;
    }
  }
}

// R = Bs - A X with the mixed-precision operator: the FP32 entries times X
// in FP64 over 256-row tiles (item: mesh, first row), plus the near-field
// low parts; the result overwrites B (the refinement's next right-hand
// side), Bs holds the original right-hand sides.
struct ResItem {
  int32_t mesh, r0;
};
constexpr int kRt = 256, kRc = 512;
__global__ void __launch_bounds__(kRt) resid_kernel(BMesh* __restrict__ meshes, const ResItem* __restrict__ items,
                                                    const double* __restrict__ Bs_all, const int64_t* __restrict__ boff) {
  const ResItem it = items[blockIdx.x];
  BMesh& M = meshes[it.mesh];
  if (M.done) return;
  const int n = (int)M.n;
  __shared__ double xs[kRc][kBasis];
  const int i = it.r0 + threadIdx.x;
  double acc[kBasis];
#pragma unroll
  for (int c = 0; c < kBasis; ++c) acc[c] = 0.0;
  for (int j0 = 0; j0 < n; j0 += kRc) {
    const int cw = min(kRc, n - j0);
    __syncthreads();
    for (int t = threadIdx.x; t < cw * kBasis; t += kRt) {
      const int j = t % cw, c = t / cw;
      xs[j][c] = M.X[j0 + j + (int64_t)n * c];
    }
    __syncthreads();
    if (i < n) {
      const float* a = M.A + i + M.ld * (int64_t)j0;
      for (int j = 0; j < cw; ++j) {
        const double v = (double)a[M.ld * (int64_t)j];
#pragma unroll
        for (int c = 0; c < kBasis; ++c) acc[c] = fma(v, xs[j][c], acc[c]);
      }
    }
  }
  if (i >= n) return;
  // near-field low parts of row i (element i / 18, local row i % 18)
  const int e = i / 18, lr = i % 18;
  for (int32_t k = M.rptr[e]; k < M.rptr[e + 1]; ++k) {
    const float* blk = M.lo + (int64_t)M.rblk[k] * 324 + lr;
    const int64_t col0 = 18 * (int64_t)M.rcol[k];
    for (int cc = 0; cc < 18; ++cc) {
      const double v = (double)blk[18 * cc];
#pragma unroll
      for (int c = 0; c < kBasis; ++c) acc[c] = fma(v, M.X[col0 + cc + (int64_t)n * c], acc[c]);
    }
  }
  const double* Bs = Bs_all + boff[it.mesh];
#pragma unroll
  for (int c = 0; c < kBasis; ++c) M.B[i + (int64_t)n * c] = Bs[i + (int64_t)n * c] - acc[c];
}

// per mesh: max over right-hand sides of |r|_inf / |b|_inf; converged meshes
// are done (their later refinement steps are skipped)
__global__ void __launch_bounds__(256) converge_kernel(BMesh* __restrict__ meshes, double tol, double* __restrict__ res) {
  BMesh& M = meshes[blockIdx.x];
  if (M.done) return;
  const int64_t n = M.n;
  __shared__ double s[kBasis][8];
  double m[kBasis];
#pragma unroll
  for (int c = 0; c < kBasis; ++c) m[c] = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x)
#pragma unroll
    for (int c = 0; c < kBasis; ++c) m[c] = fmax(m[c], fabs(M.B[i + n * c]));
#pragma unroll
  for (int c = 0; c < kBasis; ++c) {
    for (int o = 16; o > 0; o >>= 1) m[c] = fmax(m[c], __shfl_xor_sync(0xffffffffu, m[c], o));
    if ((threadIdx.x & 31) == 0) s[c][threadIdx.x >> 5] = m[c];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double worst = 0.0;
    for (int c = 0; c < kBasis; ++c) {
      double v = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v = fmax(v, s[c][w]);
      worst = fmax(worst, M.bmax[c] > 0.0 ? v / M.bmax[c] : 0.0);
    }
    res[blockIdx.x] = worst;
    if (worst <= tol) M.done = 1;
  }
}

// |b|_inf of each basis right-hand side; the run's per-mesh state reset
__global__ void __launch_bounds__(256) bmax_kernel(BMesh* __restrict__ meshes) {
  BMesh& M = meshes[blockIdx.x];
  const int64_t n = M.n;
  __shared__ double s[kBasis][8];
  double m[kBasis];
#pragma unroll
  for (int c = 0; c < kBasis; ++c) m[c] = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x)
#pragma unroll
    for (int c = 0; c < kBasis; ++c) m[c] = fmax(m[c], fabs(M.B[i + n * c]));
#pragma unroll
  for (int c = 0; c < kBasis; ++c) {
    for (int o = 16; o > 0; o >>= 1) m[c] = fmax(m[c], __shfl_xor_sync(0xffffffffu, m[c], o));
    if ((threadIdx.x & 31) == 0) s[c][threadIdx.x >> 5] = m[c];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int c = 0; c < kBasis; ++c) {
      double v = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v = fmax(v, s[c][w]);
      M.bmax[c] = v;
    }
    M.done = 0;
    M.info = 0;
    M.iters = 0;
  }
}

// The load cases' solutions: X_cases (n x n_cases) = X (n x 6) S (6 x n_cases)
// for each mesh's cases (S: 6 x n_cases per mesh, column-major).
__global__ void __launch_bounds__(256) combine_kernel(BMesh* __restrict__ meshes, const double* __restrict__ S_all,
                                                      int n_cases, double* __restrict__ Xc_all,
                                                      const int64_t* __restrict__ xoff) {
  const BMesh& M = meshes[blockIdx.y];
  const int64_t n = M.n;
  const double* S = S_all + (int64_t)6 * n_cases * blockIdx.y;
  double* Xc = Xc_all + xoff[blockIdx.y];
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n * n_cases;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t % n, j = t / n;
    double v = 0.0;
#pragma unroll
    for (int c = 0; c < kBasis; ++c) v = fma(M.X[i + n * c], S[c + 6 * j], v);
    Xc[t] = v;
  }
}

}  // namespace
}  // namespace hfpx

// ====================================================================== host
struct hfpx_batch {
  int64_t n_mesh = 0;
  std::vector<const hfpx_mesh*> meshes;
  std::vector<std::shared_ptr<NearPattern>> pats;
  std::vector<int64_t> n, ld, aoff, rsoff;
  int nb = 128, leaf_rows = 512, num_sms = 148;
  double G = 1.0, nu = 0.25;
  int64_t max_n = 0;
  // device state
  hfpx::BatchAsmMesh* d_am = nullptr;
  void* d_bm = nullptr;  // BMesh[n_mesh]
  void* d_tasks = nullptr;
  int64_t n_tasks = 0;
  float *d_A = nullptr, *d_F = nullptr, *d_lo = nullptr, *d_W = nullptr, *d_diag = nullptr;
  int32_t *d_ints = nullptr, *d_dof = nullptr;
  double *d_B = nullptr, *d_Bs = nullptr, *d_X = nullptr, *d_res = nullptr;
  int64_t* d_boff = nullptr;
  int* d_status = nullptr;
  // the launch schedule of the factorisation: kind, item bytes offset, item
  // count, auxiliary (dynamic shared memory)
  struct Launch {
    int kind;
    size_t off;
    int64_t count;
    int aux;
    size_t off2;
  };
  // trailing updates on tcgen05 (nb a multiple of 64): FP16 operand copies
  // (n x nb per mesh), row scales, per-mesh alpha and U12 maxima, tensor maps
  bool use_tc = false;
  __half *d_l16 = nullptr, *d_u16 = nullptr;
  float *d_rs = nullptr, *d_alpha = nullptr;
  unsigned* d_amax = nullptr;
  void* d_maps = nullptr;
  int* d_tcerr = nullptr;
  // C's tensor maps of every trailing update (the reduce-add epilogue),
  // 128 bytes each, 64-byte aligned
  struct alignas(64) Map128 {
    unsigned char bytes[128];
  };
  std::vector<Map128> cmaps;
  void* d_cmaps = nullptr;
  bool tc_reduce = true;
  int64_t *d_hoff = nullptr, *d_rsoff = nullptr;
  std::vector<Launch> sched;
  void* d_items = nullptr;
  std::vector<hfpx::ResItem> res_items;
  hfpx::ResItem* d_res_items = nullptr;
  int32_t* d_order = nullptr;  // meshes by size, largest first
  // load cases
  int n_cases = 0;
  double *d_S = nullptr, *d_Xc = nullptr;
  int64_t* d_xoff = nullptr;
  std::vector<int64_t> xoff;
  // the captured run, with events after the assembly (and right-hand
  // sides), the factorisation and the solves
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  double tol = 0.0;
  int max_iter = 0, graph_cases = -1;
};

namespace hfpx {
namespace {

enum LaunchKind { kLeaf, kTourn, kSwap, kL21, kU12, kGemm, kZeroAmax, kU12Amax, kU12Half, kL21Half, kTcUpdate };

template <class T>
size_t put_bytes(std::vector<unsigned char>& bytes, const std::vector<T>& items) {
  const size_t off = (bytes.size() + 15) / 16 * 16;
  bytes.resize(off + sizeof(T) * items.size());
  std::memcpy(bytes.data() + off, items.data(), sizeof(T) * items.size());
  return off;
}

template <class T>
void push_items(std::vector<unsigned char>& bytes, std::vector<hfpx_batch::Launch>& sched, int kind,
                const std::vector<T>& items, int aux) {
  if (items.empty()) return;
  const size_t off = put_bytes(bytes, items);
  sched.push_back({kind, off, (int64_t)items.size(), aux, 0});
}

void gemm_tiles(std::vector<GemmItem>& out, int m, int64_t r_lo, int64_t r_hi, int64_t q_lo, int64_t q_hi, int64_t k0,
                int K) {
  if (r_lo >= r_hi || q_lo >= q_hi || K <= 0) return;
  for (int64_t r0 = r_lo; r0 < r_hi; r0 += kGm)
    for (int64_t q0 = q_lo; q0 < q_hi; q0 += kGm)
      out.push_back({m, (int32_t)r0, (int32_t)q0, (int32_t)r_hi, (int32_t)q_hi, (int32_t)k0, K});
}

// The factorisation's launches for block size nb and leaf chunks of R rows.
void build_schedule(hfpx_batch* b, std::vector<unsigned char>& bytes) {
  const int nb = b->nb, R = b->leaf_rows;
  int64_t kmax = 0;
  for (int64_t m = 0; m < b->n_mesh; ++m) kmax = std::max(kmax, (b->n[m] + nb - 1) / nb);
  for (int64_t k = 0; k < kmax; ++k) {
    for (int p = 0; p < nb / kPw; ++p) {
      std::vector<LeafItem> leaf;
      std::vector<PanelItem> tourn;
      std::vector<ColItem> swp, u12;
      std::vector<RowItem> l21;
      std::vector<GemmItem> gm;
      int max_chunks = 0;
      for (int64_t mi = 0; mi < b->n_mesh; ++mi) {
        const int m = (int)mi;
        const int64_t n = b->n[mi], c0 = k * nb + kPw * p;
        if (c0 >= n) continue;
        const int w = (int)std::min<int64_t>(kPw, n - c0);
        const int64_t bend = std::min<int64_t>(n, (k + 1) * nb);
        int ch = 0;
        for (int64_t r0 = c0; r0 < n; r0 += R, ++ch)
          leaf.push_back({m, (int32_t)r0, (int32_t)std::min<int64_t>(R, n - r0), ch, (int32_t)c0, w});
        max_chunks = std::max(max_chunks, ch);
        tourn.push_back({m, (int32_t)c0, w, ch});
        for (int64_t q0 = 0; q0 < n; q0 += 256)
          swp.push_back({m, (int32_t)q0, (int32_t)std::min<int64_t>(256, n - q0), (int32_t)c0, w});
        for (int64_t r0 = c0; r0 < n; r0 += 256)
          l21.push_back({m, (int32_t)r0, (int32_t)std::min<int64_t>(256, n - r0), (int32_t)c0, w});
        for (int64_t q0 = c0 + w; q0 < bend; q0 += 256)
          u12.push_back({m, (int32_t)q0, (int32_t)std::min<int64_t>(256, bend - q0), (int32_t)c0, w});
        // the block's own columns, all rows below the panel
        gemm_tiles(gm, m, c0 + w, n, c0 + w, bend, c0, w);
      }
      push_items(bytes, b->sched, kLeaf, leaf, (int)(R * ((kPw + 1) * 4 + 4 + 1)));
      push_items(bytes, b->sched, kTourn, tourn, (int)(max_chunks * kPw * ((kPw + 1) * 4 + 4 + 1)));
      push_items(bytes, b->sched, kSwap, swp, 0);
      push_items(bytes, b->sched, kL21, l21, 0);
      push_items(bytes, b->sched, kU12, u12, 0);
      push_items(bytes, b->sched, kGemm, gm, 0);
    }
    // the block row right of the block, once all of the block's interchanges
    // are applied: U12 = L11^-1 A12 panel by panel (the panel's U rows, then
    // the block rows below them)
    for (int p = 0; p < nb / kPw; ++p) {
      std::vector<ColItem> u12;
      std::vector<GemmItem> gm;
      for (int64_t mi = 0; mi < b->n_mesh; ++mi) {
        const int m = (int)mi;
        const int64_t n = b->n[mi], c0 = k * nb + kPw * p, bend = (k + 1) * nb;
        if (bend >= n) continue;  // no columns right of the block
        const int w = kPw;
        for (int64_t q0 = bend; q0 < n; q0 += 256)
          u12.push_back({m, (int32_t)q0, (int32_t)std::min<int64_t>(256, n - q0), (int32_t)c0, w});
        gemm_tiles(gm, m, c0 + w, bend, bend, n, c0, w);
      }
      push_items(bytes, b->sched, kU12, u12, 0);
      push_items(bytes, b->sched, kGemm, gm, 0);
    }
    if (b->use_tc) {
      // FP16 copies of L21 (rows) and U12 (columns), then one grouped
      // tensor-core launch over every mesh's tiles
      std::vector<HalfItem> lh, uh;
      std::vector<TcProblem> probs;
      std::vector<int64_t> tstart(1, 0);
      for (int64_t mi = 0; mi < b->n_mesh; ++mi) {
        const int m = (int)mi;
        const int64_t n = b->n[mi], k0 = k * nb, bend = (k + 1) * nb;
        if (bend >= n) continue;
        const int64_t rest = n - bend;
        for (int64_t l0 = 0; l0 < rest; l0 += kHr)
          lh.push_back({m, (int32_t)l0, (int32_t)std::min<int64_t>(kHr, rest - l0), (int32_t)k0, (int32_t)bend});
        for (int64_t l0 = 0; l0 < rest; l0 += 64)
          uh.push_back({m, (int32_t)l0, (int32_t)std::min<int64_t>(64, rest - l0), (int32_t)k0, (int32_t)bend});
        TcProblem P;
        P.C = nullptr;  // set on the device side below: F + bend (ld + 1)
        P.ldc = b->ld[mi];
        P.m = (int32_t)rest;
        P.n = (int32_t)rest;
        P.k = nb;
        P.map = 2 * m;
        P.alpha = b->d_alpha + m;
        P.row_scale = b->d_rs + b->rsoff[mi];
        P.C = b->d_F + b->aoff[mi] + bend * (b->ld[mi] + 1);
        P.cmap = -1;
        P.pad = 0;
        if (b->tc_reduce) {
          hfpx_batch::Map128 cm;
          if (tc_make_c_map(&cm, P.C, rest, rest, b->ld[mi])) {
            P.cmap = (int32_t)b->cmaps.size();
            b->cmaps.push_back(cm);
          } else {
            b->tc_reduce = false;  // fall back to the reading epilogue everywhere
          }
        }
        probs.push_back(P);
        tstart.push_back(tstart.back() + ((rest + 127) / 128) * ((rest + 255) / 256));
      }
      if (!probs.empty()) {
        b->sched.push_back({kZeroAmax, 0, b->n_mesh, 0, 0});
        push_items(bytes, b->sched, kU12Amax, uh, 0);
        push_items(bytes, b->sched, kU12Half, uh, 0);
        push_items(bytes, b->sched, kL21Half, lh, (int)(sizeof(float) * kHr * (nb + 1)));
        const size_t po = put_bytes(bytes, probs), to = put_bytes(bytes, tstart);
        b->sched.push_back({kTcUpdate, po, (int64_t)probs.size(), (int)std::min<int64_t>(tstart.back(), b->num_sms), to});
      }
    } else {
      std::vector<GemmItem> trail;
      for (int64_t mi = 0; mi < b->n_mesh; ++mi) {
        const int64_t n = b->n[mi], k0 = k * nb, bend = (k + 1) * nb;
        if (bend < n) gemm_tiles(trail, (int)mi, bend, n, bend, n, k0, nb);
      }
      push_items(bytes, b->sched, kGemm, trail, 0);
    }
  }
}

PerDeviceOnce g_attr_leaf, g_attr_tourn, g_attr_perm, g_attr_half;

int batch_setup(hfpx_ctx* c, const hfpx_batch* b) {
  if (batch_assemble_setup(c->stream)) return set_error(c, HFPX_ERR_CUDA, "batched assembly set-up");
  cudaError_t e = smem_attr_once(g_attr_leaf, leaf_kernel, 512 * ((kPw + 1) * 4 + 4 + 1));
  if (e == cudaSuccess) e = smem_attr_once(g_attr_tourn, tourn_kernel, kMaxChunks * kPw * ((kPw + 1) * 4 + 4 + 1));
  if (e == cudaSuccess) e = smem_attr_once(g_attr_perm, perm_kernel, 48 * 1024);
  if (e == cudaSuccess) e = smem_attr_once(g_attr_half, l21_half_kernel, (int)(sizeof(float) * kHr * (1024 + 1)));
  int rc = check_cuda(c, e, "batched kernel attributes");
  if (!rc && b->use_tc) rc = tc_grouped_setup(c);
  return rc;
}

// every launch of one run, on the context's stream
void batch_launches(hfpx_ctx* c, hfpx_batch* b) {
  cudaStream_t s = c->stream;
  BMesh* bm = static_cast<BMesh*>(b->d_bm);
  const unsigned nm = (unsigned)b->n_mesh;
  cudaEventRecordWithFlags(b->ev[0], s, cudaEventRecordExternal);
  // far pairs in FP32 by quadrature only with HFPX_FAR32=1 (as for
  // hfpx_assemble_mixed: the default keeps the reference's closed form)
  const char* ef = std::getenv("HFPX_FAR32");
  launch_batch_assemble(b->d_am, b->d_tasks, b->n_tasks, b->G, b->nu, b->d_status, s,
                        (ef && std::string(ef) == "1") ? 1 : 0);
  int64_t nbs = 0;
  for (int64_t m = 0; m < b->n_mesh; ++m) nbs += b->n[m] * kBasis;
  launch_batch_basis_rhs(b->d_am, b->n_mesh, b->d_Bs, b->d_boff, s);
  cudaMemcpyAsync(b->d_B, b->d_Bs, sizeof(double) * nbs, cudaMemcpyDeviceToDevice, s);
  ++g_launches;
  bmax_kernel<<<nm, 256, 0, s>>>(bm);
  cudaEventRecordWithFlags(b->ev[1], s, cudaEventRecordExternal);
  const unsigned char* items = static_cast<const unsigned char*>(b->d_items);
  for (const auto& L : b->sched) {
    const void* it = items + L.off;
    const unsigned grid = (unsigned)L.count;
    ++g_launches;
    switch (L.kind) {
      case kLeaf:
        leaf_kernel<<<grid, kBt, L.aux, s>>>(bm, static_cast<const LeafItem*>(it), b->leaf_rows);
        break;
      case kTourn:
        tourn_kernel<<<grid, kBt, L.aux, s>>>(bm, static_cast<const PanelItem*>(it), L.aux / ((kPw + 1) * 4 + 4 + 1));
        break;
      case kSwap:
        swap_rows_kernel<<<grid, 256, 0, s>>>(bm, static_cast<const ColItem*>(it));
        break;
      case kL21:
        l21_kernel<<<grid, 256, 0, s>>>(bm, static_cast<const RowItem*>(it));
        break;
      case kU12:
        u12_kernel<<<grid, 256, 0, s>>>(bm, static_cast<const ColItem*>(it));
        break;
      case kGemm:
        bgemm_kernel<<<grid, 256, 0, s>>>(bm, static_cast<const GemmItem*>(it));
        break;
      case kZeroAmax:
        zero_u32_kernel<<<(grid + 255) / 256, 256, 0, s>>>(b->d_amax, (int)L.count);
        break;
      case kU12Amax:
        u12_amax_kernel<<<grid, 256, 0, s>>>(bm, static_cast<const HalfItem*>(it), b->d_amax, b->nb);
        break;
      case kU12Half:
        u12_half_kernel<<<grid, 256, 0, s>>>(bm, static_cast<const HalfItem*>(it), b->d_amax, b->d_u16, b->d_hoff,
                                              b->d_alpha, b->nb);
        break;
      case kL21Half:
        l21_half_kernel<<<grid, 256, L.aux, s>>>(bm, static_cast<const HalfItem*>(it), b->d_l16, b->d_hoff, b->d_rs,
                                                 b->d_rsoff, b->nb);
        break;
      default:  // kTcUpdate
        --g_launches;  // counted by the launcher
        tc_update_grouped(s, L.aux, b->d_maps, static_cast<const TcProblem*>(it),
                          reinterpret_cast<const int64_t*>(items + L.off2), (int)L.count, b->d_tcerr,
                          b->tc_reduce ? b->d_cmaps : nullptr);
        break;
    }
  }
  cudaEventRecordWithFlags(b->ev[2], s, cudaEventRecordExternal);
  ++g_launches;
  perm_kernel<<<nm, 256, sizeof(int32_t) * b->max_n, s>>>(bm, (int)b->max_n);
  ++g_launches;
  solve_kernel<<<nm * kSc, kSt, 0, s>>>(bm, b->d_order, 1);
  const unsigned nr = (unsigned)b->res_items.size();
  for (int it = 0; it <= b->max_iter; ++it) {
    g_launches += 2;
    resid_kernel<<<nr, kRt, 0, s>>>(bm, b->d_res_items, b->d_Bs, b->d_boff);
    converge_kernel<<<nm, 256, 0, s>>>(bm, b->tol, b->d_res);
    if (it == b->max_iter) break;
    ++g_launches;
    solve_kernel<<<nm * kSc, kSt, 0, s>>>(bm, b->d_order, 0);
  }
  if (b->n_cases > 0) {
    ++g_launches;
    combine_kernel<<<dim3(16, nm), 256, 0, s>>>(bm, b->d_S, b->n_cases, b->d_Xc, b->d_xoff);
  }
  cudaEventRecordWithFlags(b->ev[3], s, cudaEventRecordExternal);
}

void batch_free(hfpx_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  for (cudaEvent_t e : b->ev)
    if (e) cudaEventDestroy(e);
  void* ps[] = {b->d_am, b->d_bm, b->d_tasks, b->d_A, b->d_F, b->d_lo, b->d_W, b->d_diag, b->d_ints, b->d_dof,
                b->d_B, b->d_Bs, b->d_X, b->d_res, b->d_boff, b->d_status, b->d_items, b->d_res_items, b->d_S,
                b->d_Xc, b->d_xoff, b->d_l16, b->d_u16, b->d_rs, b->d_alpha, b->d_amax, b->d_maps, b->d_tcerr,
                b->d_hoff, b->d_rsoff, b->d_order, b->d_cmaps};
  for (void* p : ps)
    if (p) cudaFree(p);
  delete b;
}

template <class T>
int dalloc(hfpx_ctx* c, T** p, size_t count, const char* what) {
  return check_cuda(c, cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(1, count)), what);
}

}  // namespace
}  // namespace hfpx

using namespace hfpx;

extern "C" {

int hfpx_batch_create(hfpx_ctx* c, int64_t n_mesh, const hfpx_mesh* const* meshes, double G, double nu, int nb,
                      int leaf_rows, hfpx_batch** out) {
  if (!c || !out) return HFPX_ERR_ARG;
  *out = nullptr;
  if (n_mesh < 1 || !meshes) return set_error(c, HFPX_ERR_ARG, "no meshes");
  if (!(G > 0) || !(nu > -1.0 && nu < 0.5)) return set_error(c, HFPX_ERR_ARG, "bad elastic constants");
  nb = nb > 0 ? nb : 128;
  leaf_rows = leaf_rows > 0 ? leaf_rows : 512;
  if (nb % kPw || nb > 1024) return set_error(c, HFPX_ERR_ARG, "block size must be a multiple of 32, at most 1024");
  if (leaf_rows != 256 && leaf_rows != 512) return set_error(c, HFPX_ERR_ARG, "leaf rows must be 256 or 512");
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  hfpx_batch* b = new (std::nothrow) hfpx_batch;
  if (!b) return set_error(c, HFPX_ERR_NOMEM, "batch");
  b->n_mesh = n_mesh;
  b->nb = nb;
  b->leaf_rows = leaf_rows;
  b->G = G;
  b->nu = nu;
  b->num_sms = std::max(1, c->num_sms);
  // trailing updates on the tensor cores (the FP16 grouped kernel) when the
  // block is a multiple of its 64-deep k-steps; otherwise, or with
  // HFPX_BATCH_TC=0, the SIMT FP32 update
  const char* etc = std::getenv("HFPX_BATCH_TC");
  b->use_tc = nb % 64 == 0 && !(etc && std::string(etc) == "0");
  // the reduce-add epilogue (HFPX_BATCH_TC_REDUCE=0: the epilogue reads and writes C)
  const char* etr = std::getenv("HFPX_BATCH_TC_REDUCE");
  b->tc_reduce = !(etr && std::string(etr) == "0");
  int rc = 0;
  for (int64_t m = 0; m < n_mesh && !rc; ++m) {
    const hfpx_mesh* me = meshes[m];
    if (!me) {
      rc = set_error(c, HFPX_ERR_ARG, "null mesh");
      break;
    }
    const int64_t n = 18 * me->n_el;
    if (n > (int64_t)kMaxChunks * leaf_rows) rc = set_error(c, HFPX_ERR_ARG, "a mesh is too large for the batch");
    if (n > 11000) rc = set_error(c, HFPX_ERR_ARG, "a mesh is too large for the batch (at most 611 elements)");
    b->meshes.push_back(me);
    b->n.push_back(n);
    b->ld.push_back((n + 31) / 32 * 32);
    b->max_n = std::max(b->max_n, n);
    auto pat = rc ? nullptr : mesh_pattern(c, me);
    if (!rc && !pat) rc = set_error(c, HFPX_ERR_NOMEM, "near-field pattern");
    if (!rc && pat->maxdeg > kMaxNearDeg) rc = set_error(c, HFPX_ERR_ARG, "an element has more than 64 neighbours");
    b->pats.push_back(pat);
  }
  // pools: operator and factor (ld x n FP32 each), near-field low parts,
  // DoF maps, the solve's blocks (n x 6)
  b->aoff.assign(n_mesh, 0);
  std::vector<int64_t>& aoff = b->aoff;
  std::vector<int64_t> loff(n_mesh), doff(n_mesh), voff(n_mesh);
  int64_t atot = 0, ltot = 0, dtot = 0, vtot = 0;
  for (int64_t m = 0; m < n_mesh && !rc; ++m) {
    aoff[m] = atot;
    atot += b->ld[m] * b->n[m];
    loff[m] = ltot;
    ltot += 324 * b->pats[m]->blocks();
    doff[m] = dtot;
    dtot += b->n[m];
    voff[m] = vtot;
    vtot += b->n[m] * kBasis;
  }
  if (!rc) rc = dalloc(c, &b->d_A, atot, "batch operators");
  if (!rc) rc = dalloc(c, &b->d_F, atot, "batch factors");
  if (!rc) rc = dalloc(c, &b->d_lo, ltot, "batch near-field low parts");
  if (!rc) rc = dalloc(c, &b->d_dof, dtot, "batch DoF maps");
  if (!rc) rc = dalloc(c, &b->d_ints, 2 * dtot + n_mesh * (kPw + kMaxChunks * kPw), "batch pivots");
  if (!rc) rc = dalloc(c, &b->d_diag, n_mesh * kPw * kPw, "batch panel blocks");
  if (!rc) rc = dalloc(c, &b->d_B, vtot, "batch right-hand sides");
  if (!rc) rc = dalloc(c, &b->d_Bs, vtot, "batch right-hand sides");
  if (!rc) rc = dalloc(c, &b->d_X, vtot, "batch solutions");
  if (!rc) rc = dalloc(c, &b->d_W, vtot, "batch work vectors");
  if (!rc) rc = dalloc(c, &b->d_res, n_mesh, "batch residuals");
  if (!rc) rc = dalloc(c, &b->d_boff, n_mesh, "batch offsets");
  if (!rc) rc = dalloc(c, &b->d_status, 2, "batch status");
  if (!rc) rc = dalloc(c, &b->d_am, n_mesh, "batch meshes");
  if (!rc) rc = check_cuda(c, cudaMalloc(&b->d_bm, sizeof(BMesh) * n_mesh), "batch meshes");
  if (!rc) {
    // DoF maps (default numbering, element-major as dof_h: e + n_el * l)
    std::vector<int32_t> dof(dtot);
    std::vector<BatchAsmMesh> am(n_mesh);
    std::vector<BMesh> bm(n_mesh);
    int32_t* ints = b->d_ints;
    for (int64_t m = 0; m < n_mesh; ++m) {
      const int64_t ne = b->meshes[m]->n_el;
      for (int64_t l = 0; l < 18; ++l)
        for (int64_t e = 0; e < ne; ++e) dof[doff[m] + e + ne * l] = (int32_t)(18 * e + l);
      am[m] = {b->meshes[m]->d_elem, b->d_dof + doff[m], b->d_A + aoff[m], b->d_F + aoff[m], b->d_lo + loff[m],
               b->pats[m]->d_ptr, b->pats[m]->d_idx, ne, b->ld[m]};
      BMesh& M = bm[m];
      std::memset(&M, 0, sizeof(M));
      M.F = b->d_F + aoff[m];
      M.A = b->d_A + aoff[m];
      M.lo = b->d_lo + loff[m];
      M.rptr = b->pats[m]->d_rptr;
      M.rblk = b->pats[m]->d_rblk;
      M.rcol = b->pats[m]->d_rcol;
      M.piv = ints + doff[m];
      M.perm = ints + dtot + doff[m];
      M.prow = ints + 2 * dtot + m * kPw;
      M.cand = ints + 2 * dtot + n_mesh * kPw + m * kMaxChunks * kPw;
      M.diag = b->d_diag + m * kPw * kPw;
      M.B = b->d_B + voff[m];
      M.X = b->d_X + voff[m];
      M.W = b->d_W + voff[m];
      M.n = b->n[m];
      M.ld = b->ld[m];
      M.n_el = ne;
    }
    rc = check_cuda(c, cudaMemcpy(b->d_dof, dof.data(), sizeof(int32_t) * dtot, cudaMemcpyHostToDevice), "DoF maps");
    if (!rc)
      rc = check_cuda(c, cudaMemcpy(b->d_am, am.data(), sizeof(BatchAsmMesh) * n_mesh, cudaMemcpyHostToDevice),
                      "meshes");
    if (!rc) rc = check_cuda(c, cudaMemcpy(b->d_bm, bm.data(), sizeof(BMesh) * n_mesh, cudaMemcpyHostToDevice), "meshes");
    if (!rc) rc = check_cuda(c, cudaMemcpy(b->d_boff, voff.data(), sizeof(int64_t) * n_mesh, cudaMemcpyHostToDevice),
                             "offsets");
  }
  if (!rc) {
    // assembly tasks (mesh, source element, target tile)
    std::vector<int4> tasks;
    for (int64_t m = 0; m < n_mesh; ++m) {
      const int64_t ne = b->meshes[m]->n_el, tiles = (6 * ne + 127) / 128;
      for (int64_t sidx = 0; sidx < ne; ++sidx)
        for (int64_t x = 0; x < tiles; ++x) tasks.push_back(make_int4((int)m, (int)sidx, (int)x, 0));
    }
    b->n_tasks = (int64_t)tasks.size();
    rc = check_cuda(c, cudaMalloc(&b->d_tasks, sizeof(int4) * tasks.size()), "assembly tasks");
    if (!rc)
      rc = check_cuda(c, cudaMemcpy(b->d_tasks, tasks.data(), sizeof(int4) * tasks.size(), cudaMemcpyHostToDevice),
                      "assembly tasks");
  }
  if (!rc && b->use_tc) {
    // FP16 operand copies (n x nb per mesh), row scales, tensor maps
    std::vector<int64_t> hoff(n_mesh);
    int64_t htot = 0;
    for (int64_t m = 0; m < n_mesh; ++m) {
      hoff[m] = htot;
      htot += b->n[m] * nb;
    }
    b->rsoff = doff;
    rc = dalloc(c, &b->d_l16, htot, "batch FP16 L21");
    if (!rc) rc = dalloc(c, &b->d_u16, htot, "batch FP16 U12");
    if (!rc) rc = dalloc(c, &b->d_rs, dtot, "batch row scales");
    if (!rc) rc = dalloc(c, &b->d_alpha, n_mesh, "batch update scales");
    if (!rc) rc = dalloc(c, &b->d_amax, n_mesh, "batch U12 maxima");
    if (!rc) rc = dalloc(c, &b->d_tcerr, 1, "batch update status");
    if (!rc) rc = dalloc(c, &b->d_hoff, n_mesh, "batch offsets");
    if (!rc) rc = dalloc(c, &b->d_rsoff, n_mesh, "batch offsets");
    if (!rc) rc = check_cuda(c, cudaMalloc(&b->d_maps, 128 * 2 * n_mesh), "tensor maps");
    if (!rc) rc = check_cuda(c, cudaMemset(b->d_tcerr, 0, sizeof(int)), "update status");
    if (!rc) rc = check_cuda(c, cudaMemset(b->d_l16, 0, sizeof(__half) * htot), "FP16 copies");
    if (!rc) rc = check_cuda(c, cudaMemset(b->d_u16, 0, sizeof(__half) * htot), "FP16 copies");
    if (!rc)
      rc = check_cuda(c, cudaMemcpy(b->d_hoff, hoff.data(), sizeof(int64_t) * n_mesh, cudaMemcpyHostToDevice), "offsets");
    if (!rc)
      rc = check_cuda(c, cudaMemcpy(b->d_rsoff, doff.data(), sizeof(int64_t) * n_mesh, cudaMemcpyHostToDevice),
                      "offsets");
    if (!rc) {
      struct alignas(64) Map {
        unsigned char bytes[128];
      };
      std::vector<Map> maps(2 * n_mesh);
      for (int64_t m = 0; m < n_mesh && !rc; ++m)
        if (!tc_make_operand_map(&maps[2 * m], b->d_l16 + hoff[m], b->n[m], nb, nb, 128) ||
            !tc_make_operand_map(&maps[2 * m + 1], b->d_u16 + hoff[m], b->n[m], nb, nb, 256))
          rc = set_error(c, HFPX_ERR_CUDA, "tensor map encoding");
      if (!rc)
        rc = check_cuda(c, cudaMemcpy(b->d_maps, maps.data(), 128 * 2 * n_mesh, cudaMemcpyHostToDevice), "tensor maps");
    }
  }
  if (!rc) {
    std::vector<unsigned char> bytes;
    build_schedule(b, bytes);
    if (b->use_tc && b->tc_reduce && !b->cmaps.empty()) {
      rc = check_cuda(c, cudaMalloc(&b->d_cmaps, 128 * b->cmaps.size()), "C tensor maps");
      if (!rc)
        rc = check_cuda(c, cudaMemcpy(b->d_cmaps, b->cmaps.data(), 128 * b->cmaps.size(), cudaMemcpyHostToDevice),
                        "C tensor maps");
    } else {
      b->tc_reduce = false;
    }
    if (!rc) rc = check_cuda(c, cudaMalloc(&b->d_items, std::max<size_t>(16, bytes.size())), "schedule");
    if (!rc && !bytes.empty())
      rc = check_cuda(c, cudaMemcpy(b->d_items, bytes.data(), bytes.size(), cudaMemcpyHostToDevice), "schedule");
    std::vector<int32_t> order(n_mesh);
    for (int64_t m = 0; m < n_mesh; ++m) order[m] = (int32_t)m;
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return b->n[x] > b->n[y]; });
    for (int32_t m : order)
      for (int64_t r0 = 0; r0 < b->n[m]; r0 += kRt) b->res_items.push_back({m, (int32_t)r0});
    if (!rc) rc = dalloc(c, &b->d_order, n_mesh, "mesh order");
    if (!rc)
      rc = check_cuda(c, cudaMemcpy(b->d_order, order.data(), sizeof(int32_t) * n_mesh, cudaMemcpyHostToDevice),
                      "mesh order");
    if (!rc) rc = dalloc(c, &b->d_res_items, b->res_items.size(), "residual items");
    if (!rc)
      rc = check_cuda(c, cudaMemcpy(b->d_res_items, b->res_items.data(), sizeof(ResItem) * b->res_items.size(),
                                    cudaMemcpyHostToDevice),
                      "residual items");
  }
  if (!rc) rc = batch_setup(c, b);
  for (int i = 0; i < 4 && !rc; ++i) rc = check_cuda(c, cudaEventCreate(&b->ev[i]), "batch events");
  if (rc) {
    batch_free(b);
    return rc;
  }
  *out = b;
  return HFPX_OK;
}

int hfpx_batch_set_loads(hfpx_ctx* c, hfpx_batch* b, const double* s_inf, int64_t n_cases) {
  if (!c) return HFPX_ERR_ARG;
  if (!b || !s_inf || n_cases < 1 || n_cases > 4096) return set_error(c, HFPX_ERR_ARG, "bad load cases");
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  int rc = 0;
  if (b->n_cases != n_cases) {
    if (b->d_S) cudaFree(b->d_S);
    if (b->d_Xc) cudaFree(b->d_Xc);
    if (b->d_xoff) cudaFree(b->d_xoff);
    b->d_S = b->d_Xc = nullptr;
    b->d_xoff = nullptr;
    b->n_cases = 0;
    b->xoff.assign(b->n_mesh, 0);
    int64_t tot = 0;
    for (int64_t m = 0; m < b->n_mesh; ++m) {
      b->xoff[m] = tot;
      tot += b->n[m] * n_cases;
    }
    rc = dalloc(c, &b->d_S, 6 * n_cases * b->n_mesh, "load cases");
    if (!rc) rc = dalloc(c, &b->d_Xc, tot, "load-case solutions");
    if (!rc) rc = dalloc(c, &b->d_xoff, b->n_mesh, "offsets");
    if (!rc)
      rc = check_cuda(c, cudaMemcpy(b->d_xoff, b->xoff.data(), sizeof(int64_t) * b->n_mesh, cudaMemcpyHostToDevice),
                      "offsets");
    if (rc) return rc;
    b->n_cases = (int)n_cases;
  }
  return check_cuda(c, cudaMemcpy(b->d_S, s_inf, sizeof(double) * 6 * n_cases * b->n_mesh, cudaMemcpyHostToDevice),
                    "load cases");
}

int hfpx_batch_run(hfpx_ctx* c, hfpx_batch* b, double tol, int max_iter, hfpx_batch_info* info) {
  if (!c) return HFPX_ERR_ARG;
  if (!b) return set_error(c, HFPX_ERR_ARG, "null batch");
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  tol = tol > 0 ? tol : 1e-10;
  max_iter = max_iter > 0 ? std::min(max_iter, 30) : 10;
  int rc = 0;
  if (!b->exec || b->tol != tol || b->max_iter != max_iter || b->graph_cases != b->n_cases) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    b->tol = tol;
    b->max_iter = max_iter;
    b->graph_cases = b->n_cases;
    cudaGraph_t g = nullptr;
    rc = check_cuda(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "capture");
    if (!rc) {
      batch_launches(c, b);
      rc = check_cuda(c, cudaStreamEndCapture(c->stream, &g), "capture");
    }
    if (!rc) rc = check_cuda(c, cudaGraphInstantiate(&b->exec, g, 0), "graph instantiate");
    if (g) cudaGraphDestroy(g);
    if (rc) return rc;
  }
  rc = check_cuda(c, cudaGraphLaunch(b->exec, c->stream), "batch launch");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "batch run");
  if (rc) return rc;
  std::vector<double> res(b->n_mesh);
  std::vector<BMesh> bm(b->n_mesh);
  rc = check_cuda(c, cudaMemcpy(res.data(), b->d_res, sizeof(double) * b->n_mesh, cudaMemcpyDeviceToHost), "residuals");
  if (!rc) rc = check_cuda(c, cudaMemcpy(bm.data(), b->d_bm, sizeof(BMesh) * b->n_mesh, cudaMemcpyDeviceToHost), "state");
  int status[2] = {0, 0};
  if (!rc) rc = check_cuda(c, cudaMemcpy(status, b->d_status, sizeof(status), cudaMemcpyDeviceToHost), "status");
  if (rc) return rc;
  if (status[0] & 1) return set_error(c, HFPX_ERR_CUDA, "element staging copy timed out");
  if (b->use_tc) {
    int tcerr = 0;
    rc = check_cuda(c, cudaMemcpy(&tcerr, b->d_tcerr, sizeof(int), cudaMemcpyDeviceToHost), "update status");
    if (rc) return rc;
    if (tcerr) return set_error(c, HFPX_ERR_CUDA, "batched tensor-core update: a pipeline wait timed out");
  }
  double worst = 0.0;
  int64_t singular = -1;
  int iters = 0;
  for (int64_t m = 0; m < b->n_mesh; ++m) {
    worst = std::max(worst, res[m]);
    iters = std::max(iters, bm[m].iters);
    if (bm[m].info && singular < 0) singular = m;
  }
  if (info) {
    info->n_mesh = b->n_mesh;
    info->residual = worst;
    info->converged = worst <= tol;
    info->singular_mesh = singular;
    info->off_plane_pairs = status[1];
    info->iterations = iters;
  }
  if (singular >= 0) return set_error(c, HFPX_ERR_SINGULAR, "a mesh's matrix is singular");
  if (!(worst <= tol)) return set_error(c, HFPX_ERR_NOT_CONVERGED, "refinement did not reach the tolerance");
  return HFPX_OK;
}

int hfpx_batch_solution(hfpx_ctx* c, const hfpx_batch* b, int64_t mesh, double* x) {
  if (!c) return HFPX_ERR_ARG;
  if (!b || !x || mesh < 0 || mesh >= b->n_mesh) return set_error(c, HFPX_ERR_ARG, "bad solution arguments");
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  if (b->n_cases > 0)
    return check_cuda(c, cudaMemcpy(x, b->d_Xc + b->xoff[mesh], sizeof(double) * b->n[mesh] * b->n_cases,
                                    cudaMemcpyDeviceToHost), "solution");
  int64_t voff = 0;
  for (int64_t m = 0; m < mesh; ++m) voff += b->n[m] * kBasis;
  return check_cuda(c, cudaMemcpy(x, b->d_X + voff, sizeof(double) * b->n[mesh] * kBasis, cudaMemcpyDeviceToHost),
                    "solution");
}

int hfpx_batch_residuals(hfpx_ctx* c, const hfpx_batch* b, double* res) {
  if (!c) return HFPX_ERR_ARG;
  if (!b || !res) return set_error(c, HFPX_ERR_ARG, "bad arguments");
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  return check_cuda(c, cudaMemcpy(res, b->d_res, sizeof(double) * b->n_mesh, cudaMemcpyDeviceToHost), "residuals");
}

int64_t hfpx_batch_launches(const hfpx_batch* b) { return b ? (int64_t)b->sched.size() + 3 : -1; }

int hfpx_batch_phases(hfpx_ctx* c, const hfpx_batch* b, double* ms) {
  if (!c) return HFPX_ERR_ARG;
  if (!b || !ms || !b->exec) return set_error(c, HFPX_ERR_STATE, "no run yet");
  for (int i = 0; i < 3; ++i) {
    float t = 0.f;
    if (int rc = check_cuda(c, cudaEventElapsedTime(&t, b->ev[i], b->ev[i + 1]), "batch phases")) return rc;
    ms[i] = t;
  }
  return HFPX_OK;
}

int hfpx_batch_destroy(hfpx_batch* b) {
  if (b) batch_free(b);
  return HFPX_OK;
}

}  // extern "C"
