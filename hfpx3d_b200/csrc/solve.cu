// The mixed-precision refinement's memory-bound pieces, one right-hand side:
//   * triangular solves with the FP32 factors (forward with unit L, backward
//     with U) as one persistent sweep over 128-row tiles, the factor blocks
//     streamed through shared memory by asynchronous copies;
//   * the FP64 residual r = b - A x and its largest magnitude.
// Both replace cuBLAS calls of the refinement (dgetrs-style solve at
// il/linear_algebra/dense/factorization/LU.h:106-120 applied to FP32 factors,
// and the FP64 residual of the refinement loop), with fixed summation orders
// so repeated solves give the same bits.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include "engine_internal.h"

namespace hfpx {

// ------------------------------------------------------ triangular solves
// Solve order s = 0 .. T-1 over the 128-row tiles (tile s forward, tile
// T-1-s backward).  One CTA per SM, launched cooperatively; CTA g owns the
// solves s = g, g + G, ... and keeps their right-hand sides in shared
// memory.  For each s in turn, a CTA with work left
//   * takes x_s: its owner computes x_s = D_s^-1 y_s with the inverse of the
//     diagonal block (precomputed once per factorisation) and publishes it
//     as 128 8-byte words (value + the solve's epoch); the others poll those
//     words (one L2 round trip, no flag, no fence);
//   * first the next solve's tile: its owner subtracts A(t_{s+1}, t_s) x_s
//     (that block and the next inverse loaded before the wait), solves and
//     publishes: the critical path per tile is one word exchange and two
//     128 x 128 products;
//   * then subtracts A(t', t_s) x_s from its other owned tiles t' later in
//     solve order (the owner of s + 2 takes its solve as soon as x_{s+1}
//     arrives, between those blocks).  Those blocks are one stream per CTA, in the order they
//     are used, fed into a two-block shared-memory ring by asynchronous
//     16-byte copies (cp.async, one commit group per block), so the next
//     blocks load while the CTA waits for x and works the critical path.
// Every word wait gives up after kTrsvTimeoutNs, records the failure and
// ends the kernel (after its copies in flight complete).
constexpr int kTb = 128;
constexpr int kSwThreads = 256;
constexpr int kSwMaxOwn = 16;  // solves per CTA: n <= 16 * 148 * 128 rows
constexpr int kSwRing = 2;
constexpr unsigned long long kTrsvTimeoutNs = 200ull * 1000 * 1000;
constexpr size_t kSwSmemFloats = (size_t)(kSwRing + 1) * kTb * kTb + kSwMaxOwn * kTb + 3 * kTb + 4 * kTb + 2 * kTb;
constexpr size_t kSwSmem = sizeof(float) * kSwSmemFloats;

__device__ __forceinline__ unsigned long long trsv_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void xw_store(uint64_t* p, float v, uint32_t tag) {
  const uint64_t w = ((uint64_t)tag << 32) | __float_as_uint(v);
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(w) : "memory");
}
__device__ __forceinline__ uint64_t xw_load(const uint64_t* p) {
  uint64_t w;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(w) : "l"(p) : "memory");
  return w;
}
__device__ __forceinline__ uint32_t sw_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void sw_copy16(float* dst, const float* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sw_smem(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void sw_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// wait until at most `pending` of this thread's copy groups are in flight
__device__ __forceinline__ void sw_wait_groups(int pending) {
  if (pending <= 0) asm volatile("cp.async.wait_group 0;" ::: "memory");
  else asm volatile("cp.async.wait_group 1;" ::: "memory");
}

template <bool UPPER>
__global__ void __launch_bounds__(kSwThreads, 1) trsv_sweep_kernel(const float* __restrict__ A, int64_t lda, int n,
                                                                   const float* __restrict__ dinv,
                                                                   float* __restrict__ x, uint64_t* __restrict__ xw,
                                                                   uint32_t epoch, int* __restrict__ err) {
  extern __shared__ __align__(16) float sm[];
  float* s_ring = sm;                          // [kSwRing][kTb * kTb], column-major blocks
  float* s_dinv = s_ring + kSwRing * kTb * kTb;  // [kTb * kTb] inverse for the next owned solve
  float* s_y = s_dinv + kTb * kTb;             // [kSwMaxOwn][kTb]
  float* s_x = s_y + kSwMaxOwn * kTb;          // [kTb] x of the strip being applied
  float* s_xo = s_x + kTb;                     // [kTb] x of this CTA's latest solve
  float* s_red = s_xo + kTb;                   // [2 parities][2 halves][kTb]
  float* s_redc = s_red + 4 * kTb;             // [2 halves][kTb] (critical path)
  float* s_x2 = s_redc + 2 * kTb;              // [kTb] x_{s+1} taken early (see below)
  __shared__ int s_fail;
  const int G = gridDim.x, g = blockIdx.x, tid = threadIdx.x;
  const int T = (n + kTb - 1) / kTb;
  const int r = tid & (kTb - 1), half = tid >> 7;
  constexpr int kHalf = kTb / 2;
  auto tile_of = [&](int s) { return UPPER ? T - 1 - s : s; };
  auto rows_of = [&](int t) { return min(kTb, n - t * kTb); };
  const int nown = g < T ? (T - 1 - g) / G + 1 : 0;
  const int last_own = g + (nown - 1) * G;  // solve index of the last owned tile
  // first owned index with solve index > s + 1
  auto i_first = [&](int s) { return s + 1 - g >= 0 ? (s + 1 - g) / G + 1 : 0; };
  for (int i = 0; i < nown; ++i) {
    const int t = tile_of(g + i * G);
    if (tid < kTb) s_y[i * kTb + tid] = tid < rows_of(t) ? x[(int64_t)t * kTb + tid] : 0.f;
  }
  // stale ring contents meet zero x entries only: start them finite
  for (int i = tid; i < kSwRing * kTb * kTb; i += kSwThreads) s_ring[i] = 0.f;
  if (tid == 0) s_fail = 0;
  if (nown > 0) {
    const float* src = dinv + (size_t)tile_of(g) * kTb * kTb;
    for (int i = tid; i < kTb * kTb; i += kSwThreads) s_dinv[i] = src[i];
  }
  __syncthreads();
  // the block stream: (strip ps, owned index pi) in the order used
  int ps = 0, pi = i_first(0);
  while (ps < T && pi >= nown) {
    ++ps;
    if (ps < T) pi = i_first(ps);
  }
  int inflight = 0;   // blocks issued and not yet used (the same in every thread)
  int slot_next = 0;  // slot of the next block to use
  // every thread copies its 16-byte pieces of the next block of the stream
  // into `slot` (piece q: column q / 32, rows 4 (q % 32) ..), one group, and
  // the stream advances
  auto issue = [&](int slot) {
    if (ps >= T) return;
    const int rt = tile_of(g + pi * G), ct = tile_of(ps);
    const int rows = rows_of(rt), cols = rows_of(ct);
    float* dst = s_ring + (size_t)slot * kTb * kTb;
    const float* src = A + (int64_t)rt * kTb + lda * (int64_t)ct * kTb;
    for (int q = tid; q < kTb * kTb / 4; q += kSwThreads) {
      const int c = q >> 5, ro = (q & 31) * 4;
      if (c < cols && ro < rows) sw_copy16(dst + c * kTb + ro, src + ro + lda * c);
    }
    sw_commit();
    ++inflight;
    ++pi;
    while (ps < T && pi >= nown) {
      ++ps;
      if (ps < T) pi = i_first(ps);
    }
  };
  for (int k = 0; k < kSwRing; ++k) issue(k);
  // y_s holds every update from earlier solves: x_s = D_s^-1 y_s into s_xo,
  // published at once (words + the caller's x)
  auto solve_own = [&](int s) {
    const int ts = tile_of(s), c0 = ts * kTb, cols = rows_of(ts);
    const float* ys = s_y + (s / G) * kTb;
    float acc = 0.f;
#pragma unroll 16
    for (int u = 0; u < kHalf; ++u) {
      const int c = half * kHalf + u;
      acc = fmaf(s_dinv[r + kTb * c], ys[c], acc);
    }
    s_redc[half * kTb + r] = acc;
    __syncthreads();
    if (tid < kTb) {
      const float v = tid < cols ? s_redc[tid] + s_redc[kTb + tid] : 0.f;
      s_xo[tid] = v;
      xw_store(xw + (size_t)s * kTb + tid, v, epoch);
      if (tid < cols) x[(int64_t)c0 + tid] = v;
    }
    __syncthreads();
  };
  if (g == 0) solve_own(0);
  int nblk = 0;    // blocks used so far (selects the s_red parity)
  int early = -1;  // strip whose critical step (solve of strip + 1) was taken early
  float pa[kHalf];
  for (int s = 0; s < T; ++s) {
    const bool mine = s % G == g;
    const bool mine_next = s + 1 < T && (s + 1) % G == g;
    const bool crit = mine_next && early != s;
    if (!mine_next && last_own <= s + 1) {
      if (nown == 0 || last_own <= s) break;  // nothing of this CTA is left
      continue;
    }
    const int ts = tile_of(s), c0 = ts * kTb, cols = rows_of(ts);
    // the next owned solve: its block of this strip and its inverse, early
    if (crit) {
      const int tn = tile_of(s + 1), rn = rows_of(tn);
#pragma unroll
      for (int u = 0; u < kHalf; ++u) {
        const int c = half * kHalf + u;
        pa[u] = (r < rn && c < cols) ? A[(int64_t)tn * kTb + r + lda * (c0 + c)] : 0.f;
      }
      const float* src = dinv + (size_t)tn * kTb * kTb;
      for (int i = tid; i < kTb * kTb; i += kSwThreads) s_dinv[i] = src[i];
    }
    if (mine) {
      if (tid < kTb) s_x[tid] = s_xo[tid];
    } else if (tid < kTb) {
      const uint64_t* p = xw + (size_t)s * kTb + tid;
      uint64_t w = xw_load(p);
      if ((uint32_t)(w >> 32) != epoch) {
        const unsigned long long t0 = trsv_ns();
        do {
          w = xw_load(p);
          if (trsv_ns() - t0 > kTrsvTimeoutNs) { s_fail = 1; break; }
        } while ((uint32_t)(w >> 32) != epoch);
      }
      s_x[tid] = __uint_as_float((uint32_t)w);
    }
    __syncthreads();
    if (s_fail) break;
    if (crit) {
      float acc = 0.f;
#pragma unroll
      for (int u = 0; u < kHalf; ++u) acc = fmaf(pa[u], s_x[half * kHalf + u], acc);
      s_redc[half * kTb + r] = acc;
      __syncthreads();
      if (tid < kTb) s_y[((s + 1) / G) * kTb + tid] -= s_redc[tid] + s_redc[kTb + tid];
      __syncthreads();
      solve_own(s + 1);
    }
    // The solve of s + 2, if this CTA owns it, need not wait for this strip's
    // other blocks: once its strip-s block (the first in the ring) is applied
    // and x_{s+1} has arrived (probed between blocks, the probe's load in
    // flight during a block), it is taken here and strip s + 1 skips it.
    bool pending2 = s + 2 < T && (s + 2) % G == g;
    if (pending2) {
      const int tn = tile_of(s + 2), rn = rows_of(tn), t1 = tile_of(s + 1), cn = rows_of(t1);
#pragma unroll
      for (int u = 0; u < kHalf; ++u) {
        const int c = half * kHalf + u;
        pa[u] = (r < rn && c < cn) ? A[(int64_t)tn * kTb + r + lda * ((int64_t)t1 * kTb + c)] : 0.f;
      }
      const float* src = dinv + (size_t)tn * kTb * kTb;
      for (int i = tid; i < kTb * kTb; i += kSwThreads) s_dinv[i] = src[i];
    }
    // this strip's blocks of the other owned tiles, from the ring
    for (int i = i_first(s); i < nown; ++i) {
      uint64_t w2 = 0;
      if (pending2 && tid < kTb) w2 = xw_load(xw + (size_t)(s + 1) * kTb + tid);
      const int k = slot_next;
      sw_wait_groups(inflight - 1);  // the block of slot k is the oldest group
      __syncthreads();               // ... and every thread's pieces of it landed
      --inflight;
      const float* blk = s_ring + (size_t)k * kTb * kTb;
      float acc = 0.f;
#pragma unroll 16
      for (int u = 0; u < kHalf; ++u) {
        const int c = half * kHalf + u;
        acc = fmaf(blk[r + kTb * c], s_x[c], acc);
      }
      float* red = s_red + (nblk & 1) * 2 * kTb;
      red[half * kTb + r] = acc;
      __syncthreads();  // every read of slot k and every partial sum done
      if (tid < kTb) s_y[i * kTb + tid] -= red[tid] + red[kTb + tid];
      issue(k);
      slot_next = (k + 1) % kSwRing;
      ++nblk;
      if (pending2 && __syncthreads_and(tid >= kTb || (uint32_t)(w2 >> 32) == epoch)) {
        if (tid < kTb) s_x2[tid] = __uint_as_float((uint32_t)w2);
        __syncthreads();
        float acc2 = 0.f;
#pragma unroll
        for (int u = 0; u < kHalf; ++u) acc2 = fmaf(pa[u], s_x2[half * kHalf + u], acc2);
        s_redc[half * kTb + r] = acc2;
        __syncthreads();
        if (tid < kTb) s_y[((s + 2) / G) * kTb + tid] -= s_redc[tid] + s_redc[kTb + tid];
        __syncthreads();
        solve_own(s + 2);
        early = s + 1;
        pending2 = false;
      }
    }
  }
  // copies still in flight land before the CTA exits
  sw_wait_groups(0);
  if (s_fail && tid == 0) atomicExch(err, 1);
}

// Inverses of the 128 x 128 diagonal blocks of the factors: unit lower L
// (forward) or upper U (backward), by substitution on the identity, one
// column per thread; the ragged last block is padded with the identity.
template <bool UPPER>
__global__ void __launch_bounds__(kTb) tri_inverse_kernel(const float* __restrict__ A, int64_t lda, int n,
                                                          float* __restrict__ dinv) {
  extern __shared__ float sm[];
  float* s_a = sm;                     // [kTb][kTb + 1] row-major
  float* s_v = s_a + kTb * (kTb + 1);  // [kTb][kTb + 1]: s_v[i][j] = inverse (i, j)
  const int t = blockIdx.x, r0 = t * kTb, rows = min(kTb, n - r0), j = threadIdx.x;
  for (int i = 0; i < kTb; ++i)
    s_a[i * (kTb + 1) + j] = (i < rows && j < rows) ? A[(int64_t)r0 + i + lda * (r0 + j)] : (i == j ? 1.f : 0.f);
  __syncthreads();
  if (!UPPER) {
    for (int i = 0; i < kTb; ++i) {
      float v = i == j ? 1.f : 0.f;
      for (int k = j; k < i; ++k) v = fmaf(-s_a[i * (kTb + 1) + k], s_v[k * (kTb + 1) + j], v);
      s_v[i * (kTb + 1) + j] = i < j ? 0.f : v;
    }
  } else {
    for (int i = kTb - 1; i >= 0; --i) {
      float v = i == j ? 1.f : 0.f;
      for (int k = i + 1; k <= j; ++k) v = fmaf(-s_a[i * (kTb + 1) + k], s_v[k * (kTb + 1) + j], v);
      s_v[i * (kTb + 1) + j] = i > j ? 0.f : v / s_a[i * (kTb + 1) + i];
    }
  }
  __syncthreads();
  float* out = dinv + (size_t)t * kTb * kTb;
  for (int i = 0; i < kTb; ++i) out[i + (size_t)kTb * j] = s_v[i * (kTb + 1) + j];
}

int trsv_tiles(int64_t n) { return (int)((n + kTb - 1) / kTb); }

int tri_inverses(hfpx_ctx* c, const float* A, int64_t lda, int64_t n, float* dinv_lower, float* dinv_upper) {
  static PerDeviceOnce attr0, attr1;
  const size_t smem = sizeof(float) * 2 * kTb * (kTb + 1);
  smem_attr_once(attr0, tri_inverse_kernel<false>, (int)smem);
  smem_attr_once(attr1, tri_inverse_kernel<true>, (int)smem);
  const unsigned T = (unsigned)trsv_tiles(n);
  ++g_launches;
  tri_inverse_kernel<false><<<T, kTb, smem, c->stream>>>(A, lda, (int)n, dinv_lower);
  ++g_launches;
  tri_inverse_kernel<true><<<T, kTb, smem, c->stream>>>(A, lda, (int)n, dinv_upper);
  return check_cuda(c, cudaGetLastError(), "diagonal block inverses");
}

// x (n) holds the right-hand side on entry, the solution on return.  The
// exchange words and the failure word live in the context; the epoch tags
// each solve, so the words need no clearing between solves.
int trsv_f32(hfpx_ctx* c, const float* A, int64_t lda, int64_t n, const float* dinv, float* x, bool upper) {
  if (n <= 0) return 0;
  const int64_t T = trsv_tiles(n);
  const int G = std::min(c->num_sms, (int)T);
  if ((T + G - 1) / G > kSwMaxOwn) return set_error(c, HFPX_ERR_ARG, "matrix too large for the tile solve");
  auto* xw = (uint64_t*)ctx_scratch(c, kScrTrsvFlags, sizeof(uint64_t) * T * kTb);
  int* err = (int*)ctx_scratch(c, kScrTrsvErr, sizeof(int));
  if (!xw || !err) return set_error(c, HFPX_ERR_NOMEM, "trsv state");
  if (c->trsv_cap < T) {
    // (re)allocated: words and failure word start at zero (epoch 0 unused)
    cudaMemsetAsync(xw, 0, sizeof(uint64_t) * T * kTb, c->stream);
    cudaMemsetAsync(err, 0, sizeof(int), c->stream);
    c->trsv_cap = T;
    c->trsv_epoch = 0;
  }
  if (++c->trsv_epoch <= 0) c->trsv_epoch = 1;
  static PerDeviceOnce attr0, attr1;
  smem_attr_once(attr0, trsv_sweep_kernel<false>, (int)kSwSmem);
  smem_attr_once(attr1, trsv_sweep_kernel<true>, (int)kSwSmem);
  int nn = (int)n;
  uint32_t ep = (uint32_t)c->trsv_epoch;
  void* args[] = {&A, &lda, &nn, &dinv, &x, &xw, &ep, &err};
  ++g_launches;
  cudaError_t e = cudaLaunchCooperativeKernel(upper ? (void*)trsv_sweep_kernel<true> : (void*)trsv_sweep_kernel<false>,
                                              dim3(G), dim3(kSwThreads), args, kSwSmem, c->stream);
  return check_cuda(c, e, "triangular solve launch");
}

int trsv_status(hfpx_ctx* c) {
  if (c->trsv_cap == 0) return 0;  // no solve has run (the word is set up by the first)
  int* err = (int*)ctx_scratch(c, kScrTrsvErr, sizeof(int));
  if (!err) return 0;
  int e = 0;
  int rc = check_cuda(c, cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "trsv status");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "trsv status");
  if (!rc && e) rc = set_error(c, HFPX_ERR_CUDA, "triangular solve wait timed out");
  return rc;
}

// ---------------------------------------------------------- FP64 residual
// r = b - A x: blocks of 512 rows (two per thread, 16-byte loads) times
// column chunks; the chunks' partial sums are added in chunk order by a
// second kernel, which also records max |r| (non-negative doubles order as
// their bits).
constexpr int kGvThreads = 256;
constexpr int kGvRows = 2 * kGvThreads;
constexpr int kGvChunk = 4096;

__global__ void __launch_bounds__(kGvThreads) resid_partial_kernel(const double* __restrict__ A, int64_t lda, int n,
                                                                   const double* __restrict__ x,
                                                                   double* __restrict__ part) {
  __shared__ double s_x[kGvChunk];
  const int nch = gridDim.y;
  const int per = (n + nch - 1) / nch;
  const int c_lo = blockIdx.y * per, c_hi = min(n, c_lo + per);
  for (int j = c_lo + threadIdx.x; j < c_hi; j += kGvThreads) s_x[j - c_lo] = x[j];
  __syncthreads();
  const int i0 = blockIdx.x * kGvRows + 2 * threadIdx.x;
  double a0 = 0.0, a1 = 0.0;
  if (i0 + 1 < n) {
    const double* col = A + i0;
    int j = c_lo;
    for (; j + 4 <= c_hi; j += 4) {
      const double2 v0 = *reinterpret_cast<const double2*>(col + lda * j);
      const double2 v1 = *reinterpret_cast<const double2*>(col + lda * (j + 1));
      const double2 v2 = *reinterpret_cast<const double2*>(col + lda * (j + 2));
      const double2 v3 = *reinterpret_cast<const double2*>(col + lda * (j + 3));
      const double x0 = s_x[j - c_lo], x1 = s_x[j + 1 - c_lo], x2 = s_x[j + 2 - c_lo], x3 = s_x[j + 3 - c_lo];
      a0 = fma(v0.x, x0, a0);
      a1 = fma(v0.y, x0, a1);
      a0 = fma(v1.x, x1, a0);
      a1 = fma(v1.y, x1, a1);
      a0 = fma(v2.x, x2, a0);
      a1 = fma(v2.y, x2, a1);
      a0 = fma(v3.x, x3, a0);
      a1 = fma(v3.y, x3, a1);
    }
    for (; j < c_hi; ++j) {
      const double2 v = *reinterpret_cast<const double2*>(col + lda * j);
      a0 = fma(v.x, s_x[j - c_lo], a0);
      a1 = fma(v.y, s_x[j - c_lo], a1);
    }
  } else if (i0 < n) {
    for (int j = c_lo; j < c_hi; ++j) a0 = fma(A[i0 + lda * j], s_x[j - c_lo], a0);
  }
  if (i0 < n) part[(int64_t)blockIdx.y * n + i0] = a0;
  if (i0 + 1 < n) part[(int64_t)blockIdx.y * n + i0 + 1] = a1;
}

// The same partial products from the FP32 copy of the matrix: 4 rows per
// thread (one 16-byte load per column), products and sums in FP64 with x in
// FP64, so the only error is the FP32 rounding of the matrix entries.
constexpr int kGvRows32 = 4 * kGvThreads;
__global__ void __launch_bounds__(kGvThreads) resid_partial_f32_kernel(const float* __restrict__ A, int64_t lda, int n,
                                                                       const double* __restrict__ x,
                                                                       double* __restrict__ part) {
  __shared__ double s_x[kGvChunk];
  const int nch = gridDim.y;
  const int per = (n + nch - 1) / nch;
  const int c_lo = blockIdx.y * per, c_hi = min(n, c_lo + per);
  for (int j = c_lo + threadIdx.x; j < c_hi; j += kGvThreads) s_x[j - c_lo] = x[j];
  __syncthreads();
  const int i0 = blockIdx.x * kGvRows32 + 4 * threadIdx.x;
  double a[4] = {0.0, 0.0, 0.0, 0.0};
  if (i0 + 3 < n) {
    const float* col = A + i0;
    int j = c_lo;
    for (; j + 4 <= c_hi; j += 4) {
      const float4 v0 = *reinterpret_cast<const float4*>(col + lda * j);
      const float4 v1 = *reinterpret_cast<const float4*>(col + lda * (j + 1));
      const float4 v2 = *reinterpret_cast<const float4*>(col + lda * (j + 2));
      const float4 v3 = *reinterpret_cast<const float4*>(col + lda * (j + 3));
      const double x0 = s_x[j - c_lo], x1 = s_x[j + 1 - c_lo], x2 = s_x[j + 2 - c_lo], x3 = s_x[j + 3 - c_lo];
      a[0] = fma((double)v0.x, x0, a[0]);
      a[1] = fma((double)v0.y, x0, a[1]);
      a[2] = fma((double)v0.z, x0, a[2]);
      a[3] = fma((double)v0.w, x0, a[3]);
      a[0] = fma((double)v1.x, x1, a[0]);
      a[1] = fma((double)v1.y, x1, a[1]);
      a[2] = fma((double)v1.z, x1, a[2]);
      a[3] = fma((double)v1.w, x1, a[3]);
      a[0] = fma((double)v2.x, x2, a[0]);
      a[1] = fma((double)v2.y, x2, a[1]);
      a[2] = fma((double)v2.z, x2, a[2]);
      a[3] = fma((double)v2.w, x2, a[3]);
      a[0] = fma((double)v3.x, x3, a[0]);
      a[1] = fma((double)v3.y, x3, a[1]);
      a[2] = fma((double)v3.z, x3, a[2]);
      a[3] = fma((double)v3.w, x3, a[3]);
    }
    for (; j < c_hi; ++j) {
      const float4 v = *reinterpret_cast<const float4*>(col + lda * j);
      const double xj = s_x[j - c_lo];
      a[0] = fma((double)v.x, xj, a[0]);
      a[1] = fma((double)v.y, xj, a[1]);
      a[2] = fma((double)v.z, xj, a[2]);
      a[3] = fma((double)v.w, xj, a[3]);
    }
  } else {
#pragma unroll
    for (int r = 0; r < 4; ++r)
      if (i0 + r < n)
        for (int j = c_lo; j < c_hi; ++j) a[r] = fma((double)A[i0 + r + lda * j], s_x[j - c_lo], a[r]);
  }
#pragma unroll
  for (int r = 0; r < 4; ++r)
    if (i0 + r < n) part[(int64_t)blockIdx.y * n + i0 + r] = a[r];
}

// extra (optional): one more term of each row's product, added after the
// chunk sums (the near-field low parts of a mixed-precision operator)
__global__ void resid_finish_kernel(const double* __restrict__ b, const double* __restrict__ part, int n, int nch,
                                    double* __restrict__ r, unsigned long long* __restrict__ rmax,
                                    const double* __restrict__ extra) {
  __shared__ double s_m[8];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double m = 0.0;
  if (i < n) {
    double s = 0.0;
    for (int k = 0; k < nch; ++k) s += part[(int64_t)k * n + i];
    if (extra) s += extra[i];
    const double v = b[i] - s;
    r[i] = v;
    m = fabs(v);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) s_m[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, s_m[w]);
    atomicMax(rmax, (unsigned long long)__double_as_longlong(m));
  }
}

__global__ void absmax_kernel(const double* __restrict__ v, int n, unsigned long long* __restrict__ out) {
  __shared__ double s_m[8];
  double m = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = fmax(m, fabs(v[i]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) s_m[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, s_m[w]);
    atomicMax(out, (unsigned long long)__double_as_longlong(m));
  }
}

// Column chunks: at least n / kGvChunk (the chunk's x fits shared memory)
// and 16; the partial-sum buffer holds up to 4 times that many.
static int64_t resid_chunks_min(int64_t n) { return std::max<int64_t>(16, (n + kGvChunk - 1) / kGvChunk); }
int resid_chunks(int64_t n) { return (int)(4 * resid_chunks_min(n)); }

// The chunk count for a grid of ceil(n / rows) x nch blocks: the one (from
// the minimum up to 4 times it) whose blocks fill the last wave of resident
// blocks best, so that the matrix stream keeps every SM's loads in flight to
// the end.  A function of n and the device only, so sums are reproducible.
template <class K>
static int resid_grid_chunks(hfpx_ctx* c, int64_t n, int rows, K kernel) {
  const int64_t lo = resid_chunks_min(n);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kGvThreads, 0) != cudaSuccess || per_sm < 1) {
    cudaGetLastError();
    return (int)lo;
  }
  const int64_t R = (int64_t)per_sm * std::max(1, c->num_sms);
  const int64_t gx = (n + rows - 1) / rows;
  int64_t best = lo;
  double best_fill = 0.0;
  for (int64_t nch = lo; nch <= 4 * lo; ++nch) {
    const int64_t B = gx * nch;
    const double fill = (double)B / (double)(((B + R - 1) / R) * R);
    if (fill > best_fill + 1e-3) {
      best_fill = fill;
      best = nch;
    }
  }
  return (int)best;
}

int residual_f64(hfpx_ctx* c, const double* A, int64_t lda, int64_t n, const double* x, const double* b, double* r,
                 double* part, unsigned long long* d_max) {
  const int nch = resid_grid_chunks(c, n, kGvRows, resid_partial_kernel);
  cudaMemsetAsync(d_max, 0, sizeof(unsigned long long), c->stream);
  ++g_launches;
  resid_partial_kernel<<<dim3((unsigned)((n + kGvRows - 1) / kGvRows), (unsigned)nch), kGvThreads, 0, c->stream>>>(
      A, lda, (int)n, x, part);
  ++g_launches;
  resid_finish_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(b, part, (int)n, nch, r, d_max, nullptr);
  return check_cuda(c, cudaGetLastError(), "residual launch");
}

int residual_f32m(hfpx_ctx* c, const float* A, int64_t lda, int64_t n, const double* x, const double* b, double* r,
                  double* part, unsigned long long* d_max) {
  const int nch = resid_grid_chunks(c, n, kGvRows32, resid_partial_f32_kernel);
  cudaMemsetAsync(d_max, 0, sizeof(unsigned long long), c->stream);
  ++g_launches;
  resid_partial_f32_kernel<<<dim3((unsigned)((n + kGvRows32 - 1) / kGvRows32), (unsigned)nch), kGvThreads, 0,
                             c->stream>>>(A, lda, (int)n, x, part);
  ++g_launches;
  resid_finish_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(b, part, (int)n, nch, r, d_max, nullptr);
  return check_cuda(c, cudaGetLastError(), "residual launch");
}

// y = L x for the near-field low parts of a mixed-precision operator, one
// warp per block row (element i): lane r < 18 sums row 18 i + r over the
// row's blocks (row view rptr/rblk/rcol) in a fixed order, in FP64.
__global__ void __launch_bounds__(256) near_lo_kernel(const float* __restrict__ lo, int64_t n_el,
                                                      const int32_t* __restrict__ rptr,
                                                      const int32_t* __restrict__ rblk,
                                                      const int32_t* __restrict__ rcol,
                                                      const double* __restrict__ x, double* __restrict__ y) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n_el || lane >= 18) return;
  double s = 0.0;
  for (int32_t k = rptr[i]; k < rptr[i + 1]; ++k) {
    const float* B = lo + (int64_t)rblk[k] * 324 + lane;
    const double* xc = x + 18 * (int64_t)rcol[k];
#pragma unroll 6
    for (int c = 0; c < 18; ++c) s = fma((double)B[18 * c], xc[c], s);
  }
  y[18 * i + lane] = s;
}

int residual_mixed(hfpx_ctx* c, const hfpx_matrix* m, const double* x, const double* b, double* r, double* part,
                   unsigned long long* d_max) {
  const int64_t n = m->n;
  if (!m->op_mixed || !m->d_f || !m->d_lo || !m->pat) return set_error(c, HFPX_ERR_STATE, "not a mixed-precision operator");
  double* y = (double*)ctx_scratch(c, kScrMixedY, sizeof(double) * n);
  if (!y) return set_error(c, HFPX_ERR_NOMEM, "mixed product buffer");
  const NearPattern& p = *m->pat;
  ++g_launches;
  near_lo_kernel<<<(unsigned)((p.n_el * 32 + 255) / 256), 256, 0, c->stream>>>(m->d_lo, p.n_el, p.d_rptr, p.d_rblk,
                                                                              p.d_rcol, x, y);
  const int nch = resid_grid_chunks(c, n, kGvRows32, resid_partial_f32_kernel);
  cudaMemsetAsync(d_max, 0, sizeof(unsigned long long), c->stream);
  ++g_launches;
  resid_partial_f32_kernel<<<dim3((unsigned)((n + kGvRows32 - 1) / kGvRows32), (unsigned)nch), kGvThreads, 0,
                             c->stream>>>(m->d_f, m->ld, (int)n, x, part);
  ++g_launches;
  resid_finish_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(b, part, (int)n, nch, r, d_max, y);
  return check_cuda(c, cudaGetLastError(), "mixed residual launch");
}

int absmax_f64(hfpx_ctx* c, const double* v, int64_t n, unsigned long long* d_max) {
  cudaMemsetAsync(d_max, 0, sizeof(unsigned long long), c->stream);
  ++g_launches;
  absmax_kernel<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((int64_t)c->num_sms * 4, (n + 255) / 256)), 256, 0,
                  c->stream>>>(v, (int)n, d_max);
  return check_cuda(c, cudaGetLastError(), "absmax launch");
}

}  // namespace hfpx
