// Dense LU with partial pivoting (the work of il::LU / LAPACK dgetrf+dgetrs,
// il/linear_algebra/dense/factorization/LU.h:79-120) and the mixed-precision
// solve.
//
// Blocked right-looking LU, block nb = 2048 FP32 / 768 FP64 (HFPX_LU_NB),
// depth-1 look-ahead:
//   panel  (n-k) x nb : recursive halving (dgetrf2 order); the <=32-column
//          base case is one cooperative kernel: for FP32 the rows sit in
//          registers and the pivot search is exchanged through L2 words
//          (panel_ll_kernel), for FP64 the panel sits in shared memory with
//          one grid barrier per column (panel_base_kernel);
//   swaps  applied to the columns left and right of the panel as gathers;
//   U12 = L11^-1 A12, A22 -= L21 U12 (trailing update).
// FP64 mode factors the FP64 matrix in place (trailing update and triangular
// solves: cuBLAS FP64, i.e. FP64 tensor cores).  Mixed mode factors an FP32
// copy (U12 by an inverse-L11 TF32 GEMM, FP16 tensor-core trailing updates
// with FP32 accumulation) and recovers FP64 accuracy by iterative refinement
// against the untouched FP64 matrix.
#include <cooperative_groups.h>
#include <cublas_v2.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <mutex>
#include <vector>
#include "engine_internal.h"

namespace cg = cooperative_groups;

namespace hfpx {

constexpr int kBaseW = 32;
constexpr int kLuNbMax = 2048;    // largest FP32 block (row-swap plans hold 2 nb rows)
constexpr int kLuNbMax64 = 1024;  // largest FP64 block (the gather's register budget)
// Block size of the right-looking LU: each trailing update reads and writes
// the remaining matrix once, so HBM traffic ~ N^3 / (3 nb) x 8 bytes (FP32);
// larger blocks move work into the (overlapped) panel.  Defaults measured at
// N = 72 000: FP32 (mixed) 2048, FP64 768.  HFPX_LU_NB overrides both
// (multiple of 32 in [64, kLuNbMax]; FP64 at most kLuNbMax64).
static int lu_block_size(bool fp32) {
  static const int env = [] {
    const char* e = std::getenv("HFPX_LU_NB");
    const int v = e ? std::atoi(e) : 0;
    return (v >= 64 && v <= kLuNbMax && v % kBaseW == 0) ? v : 0;
  }();
  if (env) return fp32 ? env : std::min(env, kLuNbMax64);
  return fp32 ? kLuNbMax : 768;
}
constexpr int kPanelThreads = 256;

// ------------------------------------------------------ panel base kernel
template <class T>
struct PanelScratch {
  T* cand;        // [2][grid][kBaseW] candidate pivot rows
  double* cmax;   // [2][grid]
  int* cidx;      // [2][grid]
  T* rowj;        // [2][kBaseW] old row j
};

template <class T>
__global__ void __launch_bounds__(kPanelThreads) panel_base_kernel(
    T* __restrict__ A, int64_t lda, int64_t m, int w, int rpc, int32_t* __restrict__ piv,
    PanelScratch<T> sc, int64_t* __restrict__ info, int64_t col_offset) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* chunk = reinterpret_cast<T*>(smem_raw);               // [w][rpc]
  T* prow = chunk + (size_t)w * rpc;                        // [kBaseW]
  __shared__ double rmax[kPanelThreads / 32];
  __shared__ int ridx[kPanelThreads / 32];
  __shared__ int s_p;
  cg::grid_group grid = cg::this_grid();
  const int b = blockIdx.x, G = gridDim.x, tid = threadIdx.x;
  const int64_t r0 = (int64_t)b * rpc;
  const int nrow = (int)std::max<int64_t>(0, std::min<int64_t>(rpc, m - r0));
  for (int c = 0; c < w; ++c)
    for (int i = tid; i < nrow; i += kPanelThreads) chunk[(size_t)c * rpc + i] = A[(r0 + i) + lda * c];
  __syncthreads();
  const int lane = tid & 31, warp = tid >> 5;
  // (max, first index) pair reduction within a warp
  auto warp_argmax = [&](double& best, int& bidx) {
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_down_sync(0xffffffffu, best, o);
      const int oi = __shfl_down_sync(0xffffffffu, bidx, o);
      if (ov > best || (ov == best && oi < bidx)) { best = ov; bidx = oi; }
    }
  };
  // thread-local arg-max of |a(i,0)|
  double best = -1.0;
  int bidx = INT32_MAX;
  for (int i = tid; i < nrow; i += kPanelThreads) {
    const double v = fabs((double)chunk[i]);
    if (v > best) { best = v; bidx = (int)(r0 + i); }
  }
  for (int j = 0; j < w; ++j) {
    const int buf = j & 1;
    const int lj = j - (int)r0;
    // CTA arg-max of |a(i,j)|, i >= j (first index on ties); warp 0 publishes
    // it with the candidate row and, in the owner of row j, the old row j
    warp_argmax(best, bidx);
    if (lane == 0) { rmax[warp] = best; ridx[warp] = bidx; }
    __syncthreads();
    if (warp == 0) {
      best = lane < kPanelThreads / 32 ? rmax[lane] : -1.0;
      bidx = lane < kPanelThreads / 32 ? ridx[lane] : INT32_MAX;
      warp_argmax(best, bidx);
      best = __shfl_sync(0xffffffffu, best, 0);
      bidx = __shfl_sync(0xffffffffu, bidx, 0);
      if (lane == 0) { sc.cmax[buf * G + b] = best; sc.cidx[buf * G + b] = bidx; }
      const int li = bidx - (int)r0;
      if (li >= 0 && li < nrow && lane < w) sc.cand[((size_t)buf * G + b) * kBaseW + lane] = chunk[(size_t)lane * rpc + li];
      if (lj >= 0 && lj < nrow && lane < w) sc.rowj[buf * kBaseW + lane] = chunk[(size_t)lane * rpc + lj];
    }
    grid.sync();
    // global pivot, identical in every CTA (warp 0 scans the CTAs' candidates)
    if (warp == 0) {
      double gb = -1.0;
      int gi = INT32_MAX, gw = 0;
      for (int q = lane; q < G; q += 32) {
        const double v = sc.cmax[buf * G + q];
        const int ix = sc.cidx[buf * G + q];
        if (v > gb || (v == gb && ix < gi)) { gb = v; gi = ix; gw = q; }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, gb, o);
        const int oi = __shfl_down_sync(0xffffffffu, gi, o);
        const int ow = __shfl_down_sync(0xffffffffu, gw, o);
        if (ov > gb || (ov == gb && oi < gi)) { gb = ov; gi = oi; gw = ow; }
      }
      if (lane == 0) { s_p = gi; rmax[0] = gb; ridx[0] = gw; }
    }
    __syncthreads();
    const int p = s_p, win = ridx[0];
    if (tid < w) {
      const T pr = sc.cand[((size_t)buf * G + win) * kBaseW + tid];
      prow[tid] = pr;
      if (p != j) {  // swap rows j and p
        const int lp = p - (int)r0;
        if (lp >= 0 && lp < nrow) chunk[(size_t)tid * rpc + lp] = sc.rowj[buf * kBaseW + tid];
        if (lj >= 0 && lj < nrow) chunk[(size_t)tid * rpc + lj] = pr;
      }
    }
    if (b == 0 && tid == 0) {
      piv[j] = p;
      if (rmax[0] == 0.0 && info && *info == 0) *info = col_offset + j + 1;
    }
    __syncthreads();
    // scale column j and rank-1 update of columns j+1..w-1 for rows i > j,
    // tracking the arg-max of the updated column j+1 for the next step
    best = -1.0;
    bidx = INT32_MAX;
    const T pv = prow[j];
    const T inv = pv != (T)0 ? (T)1 / pv : (T)0;
    for (int i = tid; i < nrow; i += kPanelThreads) {
      if (r0 + i <= j) continue;
      T l = chunk[(size_t)j * rpc + i];
      if (pv != (T)0) {
        l *= inv;
        chunk[(size_t)j * rpc + i] = l;
        for (int c = j + 1; c < w; ++c) chunk[(size_t)c * rpc + i] -= l * prow[c];
      }
      if (j + 1 < w) {
        const double v = fabs((double)chunk[(size_t)(j + 1) * rpc + i]);
        if (v > best) { best = v; bidx = (int)(r0 + i); }
      }
    }
  }
  __syncthreads();
  for (int c = 0; c < w; ++c)
    for (int i = tid; i < nrow; i += kPanelThreads) A[(r0 + i) + lda * c] = chunk[(size_t)c * rpc + i];
}

// ------------------------------------------ register-resident FP32 panel
// Same factorisation as panel_base_kernel<float> (same pivots, same
// arithmetic per element, so the same bits), restructured for latency:
//  * each thread keeps kLLRows whole rows of the <= 32-column panel in
//    registers, so the rank-1 update touches no shared memory.  The rows are
//    kept shifted: at column j register column c holds panel column j + c,
//    so every register index is a compile-time constant (no selects, one
//    compact loop body: an unrolled per-column variant of this loop ran out
//    of the instruction cache).  The rank-1 update writes into the shifted
//    place, a(c) <- a(c + 1) - l p(c + 1), and column j, final once step j is
//    done, goes to the row's slot in A;
//  * the pivot search is exchanged through L2 in "LL" words: 8 bytes holding
//    4 bytes of data and a 4-byte tag naming the launch and column.  A word
//    is written and read as one 8-byte access, so a reader that sees the
//    expected tag holds the data: no grid barrier and no fence.  Every CTA
//    publishes its arg-max (key, row, the candidate row); every CTA then
//    polls all of them in one L2 round trip and picks the same pivot;
//  * rows are interchanged by relabelling, not by moving data: each register
//    row carries the panel row it currently stands for.  Swapping rows j and
//    p swaps the two labels; the pivot row's data stays where it is and, now
//    labelled j, takes no further updates.  At the end the rows whose label
//    is not their slot (<= 2 w of them) move to it with all of the block
//    panel's columns (ll_finish; skipped when no column interchanged rows);
//  * the exchange of column j + 1 overlaps the rest of step j's update (see
//    panel_ll_kernel).
// Words of column j sit in buffer j & 1: a CTA can only write column j + 2
// after all CTAs published column j + 1, i.e. after all finished reading j.
// Tags are unique within one factorisation and the buffers are zeroed before
// it (tag 0 is never used), so stale words never match.  Every poll gives up
// after kLLTimeoutNs, records the failure and ends the kernel.
constexpr int kLLThreads = 256;
constexpr int kLLRows = 6;
constexpr int kLLCap = kLLThreads * kLLRows;  // panel rows per CTA
constexpr int kLLSlot = 2 + kBaseW;           // words per CTA per column
constexpr int kLLUnits = 8;                   // words each thread polls
constexpr int kLLMaxCtas = kLLThreads * kLLUnits / kLLSlot;
constexpr unsigned long long kLLTimeoutNs = 200ull * 1000 * 1000;

__device__ __forceinline__ void ll_store(uint64_t* p, uint32_t data, uint32_t tag) {
  const uint64_t v = ((uint64_t)tag << 32) | data;
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t ll_load(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Register row k of this thread to shared memory.  The if-chain over
// compile-time K keeps every register index static.
template <int K = 0>
__device__ __forceinline__ void ll_row_to_smem(const float (&a)[kLLRows][kBaseW], int k, float* dst) {
  if (k == K) {
#pragma unroll
    for (int c = 0; c < kBaseW; ++c) dst[c] = a[K][c];
  } else if constexpr (K + 1 < kLLRows) {
    ll_row_to_smem<K + 1>(a, k, dst);
  }
}

// Waits until every CTA of the grid has stored tag in its word of bar (one
// word per CTA), bounded by kLLTimeoutNs; release fence before the store,
// acquire fence after.  Returns false (and sets s_fail) on a timeout.
__device__ bool ll_grid_barrier(uint64_t* bar, uint32_t tag, int& s_fail) {
  const int tid = threadIdx.x;
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    ll_store(bar + blockIdx.x, 0u, tag);
  }
  if (tid < (int)gridDim.x) {
    const uint64_t t0 = global_ns();
    while ((uint32_t)(ll_load(bar + tid) >> 32) != tag) {
      if (global_ns() - t0 > kLLTimeoutNs) {
        s_fail = 1;
        break;
      }
    }
    __threadfence();
  }
  __syncthreads();
  return !s_fail;
}

// Rows of a register-resident panel that end at another row (lab[k] !=
// g0 + k kLLThreads, the slot register row k came from) take their values to
// it on the enclosing block panel's columns [-left, w + right): with mid = w
// all of them, with mid = 0 the columns outside the panel only (left:
// [-left, 0), right: [w, w + right); the recursive panel's halves then need
// no row swaps between them).  A moved row's old values go to xtmp first
// (ll_moves_stash), at slot = its final label if < w, else w + its first row
// (a row starting at w or below only ever moves to a label < w, so the slots
// are distinct); after a barrier over the CTAs they go to the final row
// (ll_moves_apply).
struct MoveShared {
  int nmv;
  int src[2 * kBaseW], dst[2 * kBaseW], slot[2 * kBaseW];
};

__device__ __forceinline__ int64_t ll_move_col(int cc, int left, int mid, int w) {
  return cc < left + mid ? (int64_t)(cc - left) : (int64_t)(w + cc - left - mid);
}

__device__ void ll_moves_stash(MoveShared& ms, const float* __restrict__ A, int64_t lda, int w,
                               const int (&lab)[kLLRows], int g0, int left, int mid, int right,
                               float* __restrict__ xtmp, const int& s_fail) {
  const int tid = threadIdx.x;
  if (tid == 0) ms.nmv = 0;
  __syncthreads();
  if (!s_fail && left + mid + right > 0) {
#pragma unroll
    for (int k = 0; k < kLLRows; ++k) {
      const int phys = g0 + k * kLLThreads;
      if (lab[k] >= 0 && lab[k] != phys) {
        const int q = atomicAdd(&ms.nmv, 1);
        ms.src[q] = phys;
        ms.dst[q] = lab[k];
        ms.slot[q] = lab[k] < w ? lab[k] : w + phys;
      }
    }
  }
  __syncthreads();
  const int nmv = ms.nmv, ncol = left + mid + right;
  for (int i = tid; i < nmv * ncol; i += kLLThreads) {
    const int q = i / ncol, cc = i - q * ncol;
    xtmp[(size_t)ms.slot[q] * ncol + cc] = A[(int64_t)ms.src[q] + lda * ll_move_col(cc, left, mid, w)];
  }
}

__device__ void ll_moves_apply(const MoveShared& ms, float* __restrict__ A, int64_t lda, int w, int left, int mid,
                               int right, const float* __restrict__ xtmp) {
  const int nmv = ms.nmv, ncol = left + mid + right;
  for (int i = threadIdx.x; i < nmv * ncol; i += kLLThreads) {
    const int q = i / ncol, cc = i - q * ncol;
    A[(int64_t)ms.dst[q] + lda * ll_move_col(cc, left, mid, w)] = xtmp[(size_t)ms.slot[q] * ncol + cc];
  }
}

// End of panel_ll_kernel, whose rows are in their slots: the moved rows to
// their labels on all block-panel columns (barrier words bar, tag btag).
__device__ void ll_finish(MoveShared& ms, float* __restrict__ A, int64_t lda, int w, const int (&lab)[kLLRows],
                          int g0, int left, int right, float* __restrict__ xtmp, uint64_t* bar, uint32_t btag,
                          int* err, int& s_fail) {
  ll_moves_stash(ms, A, lda, w, lab, g0, left, w, right, xtmp, s_fail);
  if (!ll_grid_barrier(bar, btag, s_fail)) {
    if (threadIdx.x == 0) atomicExch(err, 1);
    return;
  }
  __threadfence();
  ll_moves_apply(ms, A, lda, w, left, w, right, xtmp);
}

// CTA arg-max of |a(i, jj)| (register column 0) over the rows labelled >= jj,
// lowest label on ties, in every thread.  Arg-max keys are |a| bits + 1
// (non-negative floats order as their bits), 0 for "no row".  Holds one CTA
// barrier between the two reductions.
__device__ __forceinline__ void ll_cta_argmax(const float (&a)[kLLRows][kBaseW], const int (&lab)[kLLRows], int jj,
                                              unsigned* s_wk, unsigned* s_wi, unsigned& bkey, unsigned& bidx) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // the thread's rows pairwise (a tree, not a chain); a row without a key
  // carries label 0xFFFFFFFF, so equal keys keep the lower label
  static_assert(kLLRows == 6, "the tree below pairs 6 rows");
  unsigned kk[kLLRows], ii[kLLRows];
#pragma unroll
  for (int k = 0; k < kLLRows; ++k) {
    const bool on = lab[k] >= jj;
    kk[k] = on ? __float_as_uint(fabsf(a[k][0])) + 1u : 0u;
    ii[k] = on ? (unsigned)lab[k] : 0xFFFFFFFFu;
  }
  auto pick = [](unsigned& k1, unsigned& i1, unsigned k2, unsigned i2) {
    const bool two = k2 > k1 || (k2 == k1 && i2 < i1);
    k1 = two ? k2 : k1;
    i1 = two ? i2 : i1;
  };
  pick(kk[0], ii[0], kk[1], ii[1]);
  pick(kk[2], ii[2], kk[3], ii[3]);
  pick(kk[4], ii[4], kk[5], ii[5]);
  pick(kk[0], ii[0], kk[2], ii[2]);
  pick(kk[0], ii[0], kk[4], ii[4]);
  bkey = kk[0];
  bidx = ii[0];
  {
    const unsigned wm = __reduce_max_sync(0xffffffffu, bkey);
    const unsigned wi = __reduce_min_sync(0xffffffffu, bkey == wm ? bidx : 0xFFFFFFFFu);
    if (lane == 0) { s_wk[warp] = wm; s_wi[warp] = wi; }
  }
  __syncthreads();
  const unsigned k2 = lane < kLLThreads / 32 ? s_wk[lane] : 0u;
  const unsigned i2 = lane < kLLThreads / 32 ? s_wi[lane] : 0xFFFFFFFFu;
  bkey = __reduce_max_sync(0xffffffffu, k2);
  bidx = __reduce_min_sync(0xffffffffu, k2 == bkey ? i2 : 0xFFFFFFFFu);
}

// Register row k of this thread and its multiplier lz[k] to shared memory
// (dst[0..kBaseW), then dst[kBaseW]) as they stand: during step j's update
// register column 0 already holds the updated value, the others not yet.
template <int K = 0>
__device__ __forceinline__ void ll_row_lz_to_smem(const float (&a)[kLLRows][kBaseW], const float (&lz)[kLLRows], int k,
                                                  float* dst) {
  if (k == K) {
#pragma unroll
    for (int c = 0; c < kBaseW; ++c) dst[c] = a[K][c];
    dst[kBaseW] = lz[K];
  } else if constexpr (K + 1 < kLLRows) {
    ll_row_lz_to_smem<K + 1>(a, lz, k, dst);
  }
}

// Publishes this CTA's candidate for one column in its words `mine` (tag):
// thread 0 the key and row, the warp holding the candidate row the row, one
// word per lane (v: this lane's column of it); a CTA without candidates
// publishes zeros.  `hit`: this warp holds the row.
__device__ __forceinline__ void ll_publish(uint64_t* mine, unsigned bkey, unsigned bidx, uint32_t tag, int w,
                                           bool hit, float v) {
  const int tid = threadIdx.x, lane = tid & 31;
  if (tid == 0) {
    ll_store(mine, bkey, tag);
    ll_store(mine + 1, bidx, tag);
  }
  if (hit) {
    if (lane < w) ll_store(mine + 2 + lane, __float_as_uint(v), tag);
  } else if (bkey == 0u && tid < 32 && lane < w) {
    ll_store(mine + 2 + lane, 0u, tag);
  }
}

// piv[j] = pivot row + piv_add; left/right: columns of the enclosing block
// panel on either side that take the interchanges too (ll_finish).
// Step j, once the pivot p and its row are known: the labels swap, every row
// takes the update of its register column 0 only (column j + 1 of the panel),
// the CTA's candidate for column j + 1 is found and published, and only then
// do the other 30 register columns take their update and column j go to A, so
// that work overlaps the exchange of column j + 1.
__global__ void __launch_bounds__(kLLThreads, 1) panel_ll_kernel(
    float* __restrict__ A, int64_t lda, int64_t m, int w, int rpc, int32_t* __restrict__ piv,
    uint64_t* __restrict__ slots, int64_t* __restrict__ info, int64_t col_offset, uint32_t tag0,
    int* __restrict__ err, int left, int right, float* __restrict__ xtmp, int piv_add) {
  // the polled words of columns j (buffer j & 1), laid out as in `slots`:
  // per CTA (key, row, candidate row); words never written stay zero, so
  // candidate columns past w read as zeros
  __shared__ __align__(16) uint32_t s_w[2][kLLMaxCtas * kLLSlot];
  __shared__ unsigned s_wk[kLLThreads / 32];
  __shared__ unsigned s_wi[kLLThreads / 32];
  __shared__ float s_stage[kLLThreads / 32][kBaseW + 1];  // a warp's candidate row (+ its multiplier)
  __shared__ int s_fail;
  const int b = blockIdx.x, G = gridDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t r0 = (int64_t)b * rpc;
  const int nrow = (int)max((int64_t)0, min((int64_t)rpc, m - r0));
  const int g0 = (int)r0 + tid;       // panel row first held in a[k]: g0 + k * kLLThreads
  const int nrow_left = nrow - tid;   // a[k] holds a row iff k * kLLThreads < nrow_left
  float a[kLLRows][kBaseW];
  int lab[kLLRows];                   // panel row a[k] stands for, -1: none
#pragma unroll
  for (int k = 0; k < kLLRows; ++k) {
    lab[k] = k * kLLThreads < nrow_left ? g0 + k * kLLThreads : -1;
#pragma unroll
    for (int c = 0; c < kBaseW; ++c)
      a[k][c] = (lab[k] >= 0 && c < w) ? A[(int64_t)lab[k] + lda * c] : 0.f;
  }
  for (int i = tid; i < 2 * kLLMaxCtas * kLLSlot; i += kLLThreads) (&s_w[0][0])[i] = 0u;
  const float* st = s_stage[warp];
  if (tid == 0) s_fail = 0;
  // words this thread polls: CTA q's (key, row, candidate row)
  const int per = 2 + w, units = G * per;
  int off[kLLUnits];
#pragma unroll
  for (int u = 0; u < kLLUnits; ++u) {
    const int x = tid + u * kLLThreads;
    off[u] = x < units ? (x / per) * kLLSlot + x % per : -1;
  }
  bool swapped = false;  // an interchange happened (the same in every CTA)
  // column 0's candidate, the rows as loaded
  {
    unsigned bkey, bidx;
    ll_cta_argmax(a, lab, 0, s_wk, s_wi, bkey, bidx);
    int kc = -1;
#pragma unroll
    for (int k = 0; k < kLLRows; ++k) kc = ((unsigned)lab[k] == bidx && bkey != 0u) ? k : kc;
    const bool hit = __ballot_sync(0xffffffffu, kc >= 0) != 0u;
    if (kc >= 0) ll_row_to_smem(a, kc, s_stage[warp]);
    __syncwarp();
    ll_publish(slots + (size_t)b * kLLSlot, bkey, bidx, tag0 + 1u, w, hit, st[lane]);
  }
  for (int j = 0; j < w; ++j) {
    const int buf = j & 1;
    const uint32_t tag = tag0 + (uint32_t)j + 1u;
    // poll every CTA's words for this column
    const uint64_t* xb = slots + (size_t)buf * G * kLLSlot;
    uint32_t* sw = s_w[buf];
    bool need[kLLUnits];
#pragma unroll
    for (int u = 0; u < kLLUnits; ++u) need[u] = off[u] >= 0;
    uint64_t t_start = 0;
    bool failed = false;
    for (;;) {
      uint64_t v[kLLUnits];
#pragma unroll
      for (int u = 0; u < kLLUnits; ++u) v[u] = need[u] ? ll_load(xb + off[u]) : 0;
      bool pending = false;
#pragma unroll
      for (int u = 0; u < kLLUnits; ++u) {
        if (!need[u]) continue;
        if ((uint32_t)(v[u] >> 32) != tag) { pending = true; continue; }
        need[u] = false;
        sw[off[u]] = (uint32_t)v[u];
      }
      if (!pending) break;
      const uint64_t now = global_ns();
      if (t_start == 0) t_start = now;
      else if (now - t_start > kLLTimeoutNs) { failed = true; break; }
    }
    if (failed) s_fail = 1;
    __syncthreads();
    if (s_fail) {
      if (tid == 0) atomicExch(err, 1);
      break;
    }
    // global pivot, identical in every warp of every CTA
    unsigned gk = 0u, gi = 0xFFFFFFFFu, gq = 0u;
    for (int q = lane; q < G; q += 32) {
      const unsigned kq = sw[q * kLLSlot], iq = sw[q * kLLSlot + 1];
      if (kq > gk || (kq == gk && iq < gi)) { gk = kq; gi = iq; gq = (unsigned)q; }
    }
    const unsigned gmax = __reduce_max_sync(0xffffffffu, gk);
    const unsigned pu = __reduce_min_sync(0xffffffffu, gk == gmax ? gi : 0xFFFFFFFFu);
    const int p = (int)pu;
    // the lane holding the winner (labels are unique; with no row left
    // anywhere every lane holds key 0 and label 0xFFFFFFFF: lane 0, CTA 0)
    const unsigned wl = __ffs(__ballot_sync(0xffffffffu, gk == gmax && gi == pu)) - 1;
    const uint32_t* prow = sw + __shfl_sync(0xffffffffu, gq, wl) * kLLSlot + 2;
    if (b == 0 && tid == 0) {
      piv[j] = p + piv_add;
      if (gmax == 1u && info && *info == 0) *info = col_offset + j + 1;  // |pivot| == 0
    }
    // interchange rows j and p: swap the labels
    if (p != j) {
      swapped = true;
#pragma unroll
      for (int k = 0; k < kLLRows; ++k) lab[k] = lab[k] == j ? p : (lab[k] == p ? j : lab[k]);
    }
    const float pv = __uint_as_float(prow[0]);
    const bool nz = pv != 0.f;
    const float inv = nz ? 1.f / pv : 0.f;
    // Column j of every row is final after this step (the multiplier of a
    // row below, U of the pivot and of earlier pivots); the registers shift
    // left by one as the rows below take the rank-1 update (multiplier 0 for
    // the others: a plain shift).  Register column 0 first.
    float l[kLLRows], lz[kLLRows];
    const float p1 = __uint_as_float(prow[1]);
#pragma unroll
    for (int k = 0; k < kLLRows; ++k) {
      const bool below = nz && lab[k] > j;
      l[k] = below ? a[k][0] * inv : a[k][0];
      lz[k] = below ? l[k] : 0.f;
      a[k][0] = fmaf(-lz[k], p1, a[k][1]);
    }
    if (j + 1 < w) {
      unsigned bkey, bidx;
      ll_cta_argmax(a, lab, j + 1, s_wk, s_wi, bkey, bidx);
      int kc = -1;
#pragma unroll
      for (int k = 0; k < kLLRows; ++k) kc = ((unsigned)lab[k] == bidx && bkey != 0u) ? k : kc;
      const bool hit = __ballot_sync(0xffffffffu, kc >= 0) != 0u;
      // the candidate row after step j, one column per lane: the owner's
      // registers as they stand, then the same fmaf as the update below
      if (kc >= 0) ll_row_lz_to_smem(a, lz, kc, s_stage[warp]);
      __syncwarp();
      float v = 0.f;
      if (hit) {
        v = lane == 0 ? st[0]
                      : (lane + 1 < kBaseW ? fmaf(-st[kBaseW], __uint_as_float(prow[lane + 1]), st[lane + 1]) : 0.f);
      }
      ll_publish(slots + ((size_t)(buf ^ 1) * G + b) * kLLSlot, bkey, bidx, tag + 1u, w, hit, v);
    }
    // the rest of the update and column j, behind the exchange of column j + 1
#pragma unroll
    for (int k = 0; k < kLLRows; ++k) {
      if (lab[k] >= 0) A[(int64_t)(g0 + k * kLLThreads) + lda * j] = l[k];
#pragma unroll
      for (int c = 1; c + 1 < kBaseW; ++c) a[k][c] = fmaf(-lz[k], __uint_as_float(prow[c + 1]), a[k][c + 1]);
      a[k][kBaseW - 1] = 0.f;
    }
  }
  // without interchanges every row is in its slot: no moves, no barrier
  __shared__ MoveShared ms;
  if (swapped)
    ll_finish(ms, A, lda, w, lab, g0, left, right, xtmp, slots + (size_t)2 * kLLMaxCtas * kLLSlot, tag0 + 63u, err,
              s_fail);
}

// ------------------------------------------ tournament-pivoting FP32 panel
// For the mixed-precision factorisation only (FP64 keeps LAPACK's partial
// pivoting).  Same register layout as panel_ll_kernel, but the pivots of all
// w columns are chosen with one exchange over the grid instead of one per
// column: TSLU, the panel step of communication-avoiding LU (Grigori, Demmel
// and Xiang, "CALU: a communication optimal LU factorization algorithm",
// SIAM J. Matrix Anal. Appl. 32 (2011) 1317-1350), with a flat tournament:
//  1. each CTA runs partial pivoting on its own rows, exchanging through
//     shared memory only, and publishes the original values of the <= w rows
//     it chose;
//  2. after one grid barrier every CTA loads all G w candidates (<= 1536, one
//     per register row) and runs partial pivoting on them.  The same inputs
//     and the same arithmetic in every CTA give every CTA the same w pivot
//     rows and the same rows of U, with no broadcast;
//  3. each CTA turns the pivots into LAPACK interchanges (row j <-> row
//     piv[j], in order), reloads its rows and, after a second barrier (other
//     CTAs' rows move onto rows this CTA reloads), eliminates them with the
//     known U, writing each row at its final place.
// With one CTA step 2 is skipped: step 1 is partial pivoting on the whole panel.
//
// The partial pivoting of steps 1 and 2 is blocked, kLeaf columns at a time,
// so that every register index is a compile-time constant: the leaf's columns
// sit in register columns [0, kLeaf) and take the rank-1 steps; the leaf's
// pivot rows give U12 = L11^-1 A12 (one small forward substitution in shared
// memory); the other rows take A22 -= L21 U12; then the registers shift left
// by kLeaf.  Step 3 runs the same elimination with U from step 2 (a pivot row
// stops at its own column), so each pivot row ends bit-identical to its U row.
// Zero pivots are reported as partial pivoting does: info = first column
// whose chosen pivot is 0.  The refinement against the FP64 matrix, not the
// pivot sequence, pins the mixed solution.
constexpr int kTsluMaxCtas = kLLCap / kBaseW;  // candidates fill one CTA's registers: 48
constexpr int kLeaf = 8;
constexpr int kTrail = kBaseW - kLeaf;
constexpr int kLLWarps = kLLThreads / 32;

struct TsluShared {
  float stage[kLeaf][kLLWarps][kLeaf];  // leaf step s: each warp's arg-max row, leaf columns
  unsigned key[kLeaf][kLLWarps];
  unsigned idx[kLeaf][kLLWarps];
  int win[kLeaf];                       // warp whose row won leaf step s
  float u12[kLeaf][kTrail];             // the leaf's pivot rows, trailing columns -> U12
  int sel[kBaseW];                      // label chosen at column j, -1: none left
  float fin[kBaseW][kBaseW];            // row j: U(j, c) for c >= j
  int pos[kLLCap];                      // own row -> pivot column, then -> final label
  int zero;                             // first column with a zero pivot (kBaseW: none)
};

// Register row k's leaf columns to shared memory (if-chain: static indices).
template <int K = 0>
__device__ __forceinline__ void leaf_row_to_smem(const float (&a)[kLLRows][kBaseW], int k, float* dst) {
  if (k == K) {
#pragma unroll
    for (int c = 0; c < kLeaf; ++c) dst[c] = a[K][c];
  } else if constexpr (K + 1 < kLLRows) {
    leaf_row_to_smem<K + 1>(a, k, dst);
  }
}

// Blocked partial pivoting over columns [0, w) of the rows this CTA holds
// (lab[k] >= 0); ties go to the lower label, as in panel_ll_kernel.
// sh.sel[j] <- label chosen at column j, sh.zero <- first zero pivot, and
// with want_fin sh.fin[j] <- U(j, c >= j).  The registers are consumed.
__device__ __forceinline__ void tslu_gepp(float (&a)[kLLRows][kBaseW], const int (&lab)[kLLRows], int w,
                                          bool want_fin, TsluShared& sh) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  bool act[kLLRows];
#pragma unroll
  for (int k = 0; k < kLLRows; ++k) act[k] = lab[k] >= 0;
  if (tid == 0) sh.zero = kBaseW;
#pragma unroll 1
  for (int j0 = 0; j0 < w; j0 += kLeaf) {
    const int lw = min(kLeaf, w - j0);
    int cs[kLLRows];  // leaf step at which register row k was chosen, -1: not in this leaf
#pragma unroll
    for (int k = 0; k < kLLRows; ++k) cs[k] = -1;
#pragma unroll
    for (int s = 0; s < kLeaf; ++s) {
      if (s >= lw) break;
      unsigned bkey = 0u, bidx = 0xFFFFFFFFu;
#pragma unroll
      for (int k = 0; k < kLLRows; ++k) {
        const unsigned kk = act[k] ? __float_as_uint(fabsf(a[k][s])) + 1u : 0u;
        if (kk > bkey || (kk == bkey && kk != 0u && (unsigned)lab[k] < bidx)) {
          bkey = kk;
          bidx = (unsigned)lab[k];
        }
      }
      const unsigned wm = __reduce_max_sync(0xffffffffu, bkey);
      const unsigned wi = __reduce_min_sync(0xffffffffu, bkey == wm ? bidx : 0xFFFFFFFFu);
      if (wm != 0u) {
        int kc = -1;
#pragma unroll
        for (int k = 0; k < kLLRows; ++k) kc = (act[k] && (unsigned)lab[k] == wi) ? k : kc;
        if (kc >= 0) leaf_row_to_smem(a, kc, sh.stage[s][warp]);
      }
      if (lane == 0) {
        sh.key[s][warp] = wm;
        sh.idx[s][warp] = wi;
      }
      __syncthreads();
      const unsigned k2 = lane < kLLWarps ? sh.key[s][lane] : 0u;
      const unsigned i2 = lane < kLLWarps ? sh.idx[s][lane] : 0xFFFFFFFFu;
      const unsigned gk = __reduce_max_sync(0xffffffffu, k2);
      const unsigned gi = __reduce_min_sync(0xffffffffu, k2 == gk ? i2 : 0xFFFFFFFFu);
      const unsigned gw = __reduce_max_sync(0xffffffffu, (k2 == gk && i2 == gi) ? (unsigned)lane : 0u);
      if (tid == 0) {
        sh.sel[j0 + s] = gk != 0u ? (int)gi : -1;
        sh.win[s] = (int)gw;
        if (gk <= 1u) sh.zero = min(sh.zero, j0 + s);  // no row left, or |pivot| == 0
      }
      if (gk == 0u) continue;
#pragma unroll
      for (int k = 0; k < kLLRows; ++k) {
        if (act[k] && (unsigned)lab[k] == gi) {
          act[k] = false;
          cs[k] = s;
        }
      }
      const float* prow = sh.stage[s][gw];
      const float pv = prow[s];
      if (pv == 0.f) continue;
      const float inv = 1.f / pv;
      float pc[kLeaf];
#pragma unroll
      for (int c = s + 1; c < kLeaf; ++c) pc[c] = prow[c];
#pragma unroll
      for (int k = 0; k < kLLRows; ++k) {
        if (!act[k]) continue;
        const float l = a[k][s] * inv;
        a[k][s] = l;
#pragma unroll
        for (int c = s + 1; c < kLeaf; ++c) a[k][c] = fmaf(-l, pc[c], a[k][c]);
      }
    }
    // the leaf's pivot rows, trailing columns as at the leaf's start
#pragma unroll
    for (int k = 0; k < kLLRows; ++k) {
      if (cs[k] < 0) continue;
      float* d = sh.u12[cs[k]];
#pragma unroll
      for (int c = 0; c < kTrail; ++c) d[c] = a[k][kLeaf + c];
    }
    __syncthreads();
    // U12 = L11^-1 A12; L11(i, i2) = multiplier of the pivot row of step i at leaf column i2
    if (tid < kTrail) {
      float u[kLeaf];
#pragma unroll
      for (int i = 0; i < kLeaf; ++i) {
        const bool ok = i < lw && sh.sel[j0 + i] >= 0;
        u[i] = ok ? sh.u12[i][tid] : 0.f;
        if (ok) {
          const float* li = sh.stage[i][sh.win[i]];
#pragma unroll
          for (int i2 = 0; i2 < i; ++i2) u[i] = fmaf(-li[i2], u[i2], u[i]);
        }
      }
#pragma unroll
      for (int i = 0; i < kLeaf; ++i) sh.u12[i][tid] = u[i];
    }
    __syncthreads();
    if (want_fin) {
      for (int e = tid; e < kLeaf * kBaseW; e += kLLThreads) {
        const int i = e / kBaseW, col = e - i * kBaseW, j = j0 + i;
        if (i < lw && col >= j && sh.sel[j] >= 0)
          sh.fin[j][col] = col < j0 + kLeaf ? sh.stage[i][sh.win[i]][col - j0] : sh.u12[i][col - j0 - kLeaf];
      }
    }
    // A22 -= L21 U12 on the rows still in play (kLeaf trailing columns at a
    // time, to bound the registers), then the registers shift by a leaf
#pragma unroll
    for (int cb = 0; cb < kTrail; cb += kLeaf) {
#pragma unroll
      for (int i = 0; i < kLeaf; ++i) {
        float u[kLeaf];
#pragma unroll
        for (int c = 0; c < kLeaf; ++c) u[c] = sh.u12[i][cb + c];
#pragma unroll
        for (int k = 0; k < kLLRows; ++k) {
          if (!act[k]) continue;
          const float l = a[k][i];
#pragma unroll
          for (int c = 0; c < kLeaf; ++c) a[k][kLeaf + cb + c] = fmaf(-l, u[c], a[k][kLeaf + cb + c]);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kLLRows; ++k) {
#pragma unroll
      for (int c = 0; c < kTrail; ++c) a[k][c] = a[k][c + kLeaf];
#pragma unroll
      for (int c = kTrail; c < kBaseW; ++c) a[k][c] = 0.f;
    }
    __syncthreads();
  }
}

// Step 3: the rows of this CTA (original values) eliminated with U = sh.fin.
// rk[k] packs register row k's final label (bits 0-16) and the column it is
// the pivot of, plus 1 (bits 17-22; 0: none); -1: no row.  A pivot row stops
// at its own column.  Each leaf's columns are written to A as they finish.
constexpr int kRkBits = 17;
static_assert(kTsluMaxCtas * kLLCap <= (1 << kRkBits), "tournament rows fit the packed label");
__device__ __forceinline__ int rk_pcol(int rk) { return (rk >> kRkBits) - 1; }

__device__ __forceinline__ void tslu_eliminate(float (&a)[kLLRows][kBaseW], const int (&rk)[kLLRows], int w,
                                               const TsluShared& sh, float* __restrict__ A, int64_t lda) {
#pragma unroll 1
  for (int j0 = 0; j0 < w; j0 += kLeaf) {
    const int lw = min(kLeaf, w - j0);
#pragma unroll
    for (int s = 0; s < kLeaf; ++s) {
      if (s >= lw) break;
      const int j = j0 + s;
      const float* U = sh.fin[j];
      const float pv = U[j];
      if (pv == 0.f) continue;
      const float inv = 1.f / pv;
      float pc[kLeaf];
#pragma unroll
      for (int c = s + 1; c < kLeaf; ++c) pc[c] = U[j0 + c];
#pragma unroll
      for (int k = 0; k < kLLRows; ++k) {
        const int p = rk_pcol(rk[k]);
        if (rk[k] < 0 || (p >= 0 && p <= j)) continue;
        const float l = a[k][s] * inv;
        a[k][s] = l;
#pragma unroll
        for (int c = s + 1; c < kLeaf; ++c) a[k][c] = fmaf(-l, pc[c], a[k][c]);
      }
    }
    // trailing columns: multipliers of the leaf steps each row took part in
    // (all kLeaf, up to its own column for this leaf's pivot rows, none for
    // rows done in earlier leaves)
#pragma unroll
    for (int cb = 0; cb < kTrail; cb += kLeaf) {
      if (j0 + kLeaf + cb >= kBaseW) break;
#pragma unroll
      for (int i = 0; i < kLeaf; ++i) {
        if (i >= lw) break;
        float u[kLeaf];
        const float* U = sh.fin[j0 + i] + j0 + kLeaf + cb;
#pragma unroll
        for (int c = 0; c < kLeaf; ++c) u[c] = U[c];
#pragma unroll
        for (int k = 0; k < kLLRows; ++k) {
          const int p = rk_pcol(rk[k]);
          if (rk[k] < 0 || (p >= 0 && p <= j0 + i)) continue;
          const float l = a[k][i];
#pragma unroll
          for (int c = 0; c < kLeaf; ++c) a[k][kLeaf + cb + c] = fmaf(-l, u[c], a[k][kLeaf + cb + c]);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kLLRows; ++k) {
      if (rk[k] >= 0) {
        float* row = A + (int64_t)(rk[k] & ((1 << kRkBits) - 1)) + lda * j0;
#pragma unroll
        for (int c = 0; c < kLeaf; ++c)
          if (c < lw) row[lda * c] = a[k][c];
      }
#pragma unroll
      for (int c = 0; c < kTrail; ++c) a[k][c] = a[k][c + kLeaf];
#pragma unroll
      for (int c = kTrail; c < kBaseW; ++c) a[k][c] = 0.f;
    }
  }
}

// The pivots sh.sel[0..w) (labels) as LAPACK interchanges, by one warp:
// piv[j] = place of row sel[j] after the interchanges of columns < j.  Lane
// x < w tracks the row now at place x; lane j also keeps the one place >= w
// that column j's interchange may create (far_pos, holding row far_row).  The
// final label of every row of [r0, r0 + nrow) that moved goes to sh.pos.
__device__ void tslu_interchanges(int w, int64_t r0, int nrow, int32_t* __restrict__ piv, int piv_add,
                                  bool write_piv, TsluShared& sh) {
  const int x = threadIdx.x & 31;
  int row_at = x, far_pos = -1, far_row = -1;
  for (int j = 0; j < w; ++j) {
    const int p = sh.sel[j];
    const unsigned near = __ballot_sync(0xffffffffu, x < w && row_at == p);
    const unsigned far = __ballot_sync(0xffffffffu, far_pos >= 0 && far_row == p);
    int cur;
    if (near) cur = __ffs(near) - 1;
    else if (far) cur = __shfl_sync(0xffffffffu, far_pos, __ffs(far) - 1);
    else cur = p;
    const int rj = __shfl_sync(0xffffffffu, row_at, j);
    if (x == 0 && write_piv) piv[j] = cur + piv_add;
    if (cur != j) {
      if (x == j) row_at = p;
      if (cur < w) {
        if (x == cur) row_at = rj;
      } else if (far) {
        if (x == __ffs(far) - 1) far_row = rj;
      } else if (x == j) {
        far_pos = cur;
        far_row = rj;
      }
    }
  }
  if (x < w && row_at >= r0 && row_at < r0 + nrow) sh.pos[row_at - r0] = x;
  if (far_pos >= 0 && far_row >= r0 && far_row < r0 + nrow) sh.pos[far_row - r0] = far_pos;
}

__global__ void __launch_bounds__(kLLThreads, 1) panel_tslu_kernel(
    float* __restrict__ A, int64_t lda, int64_t m, int w, int rpc, int32_t* __restrict__ piv,
    uint64_t* __restrict__ slots, float* __restrict__ cand, int64_t* __restrict__ info, int64_t col_offset,
    uint32_t tag0, int* __restrict__ err, int left, int right, float* __restrict__ xtmp, int piv_add) {
  __shared__ TsluShared sh;
  __shared__ MoveShared ms;
  __shared__ int s_fail;
  const int b = blockIdx.x, G = gridDim.x, tid = threadIdx.x;
  const int64_t r0 = (int64_t)b * rpc;
  const int nrow = (int)max((int64_t)0, min((int64_t)rpc, m - r0));
  const int g0 = (int)r0 + tid;
  const int nrow_left = nrow - tid;
  uint64_t* bar = slots + (size_t)2 * kLLMaxCtas * kLLSlot;  // kLLMaxCtas words per barrier
  int* cidx = reinterpret_cast<int*>(cand + (size_t)kTsluMaxCtas * kBaseW * kBaseW);
  float a[kLLRows][kBaseW];
  int lab[kLLRows];
#pragma unroll
  for (int k = 0; k < kLLRows; ++k) {
    lab[k] = k * kLLThreads < nrow_left ? g0 + k * kLLThreads : -1;
#pragma unroll
    for (int c = 0; c < kBaseW; ++c) a[k][c] = (lab[k] >= 0 && c < w) ? A[(int64_t)lab[k] + lda * c] : 0.f;
  }
  if (tid == 0) s_fail = 0;
  const int rounds = G > 1 ? 2 : 1;
#pragma unroll 1
  for (int rd = 0; rd < rounds; ++rd) {
    if (rd == 1) {
      // candidates: original values of the rows chosen in round 0 at
      // cand[(b kBaseW + i) kBaseW + c], their labels at cidx
      for (int e = tid; e < kBaseW * kBaseW; e += kLLThreads) {
        const int i = e / kBaseW, c = e - i * kBaseW;
        const int r = i < w ? sh.sel[i] : -1;
        cand[((size_t)b * kBaseW + i) * kBaseW + c] = (r >= 0 && c < w) ? A[(int64_t)r + lda * c] : 0.f;
        if (c == 0) cidx[b * kBaseW + i] = r;
      }
      if (!ll_grid_barrier(bar + kLLMaxCtas, tag0 + 62u, s_fail)) {
        if (tid == 0) atomicExch(err, 1);
        return;
      }
      // list entry e = q kBaseW + i in register row e / kLLThreads of thread e % kLLThreads
#pragma unroll
      for (int k = 0; k < kLLRows; ++k) {
        const int e = tid + k * kLLThreads;
        lab[k] = e < G * kBaseW ? __ldcg(cidx + e) : -1;
        const float4* src = reinterpret_cast<const float4*>(cand + (size_t)e * kBaseW);
#pragma unroll
        for (int c4 = 0; c4 < kBaseW / 4; ++c4) {
          const float4 v = lab[k] >= 0 ? __ldcg(src + c4) : make_float4(0.f, 0.f, 0.f, 0.f);
          a[k][4 * c4] = v.x;
          a[k][4 * c4 + 1] = v.y;
          a[k][4 * c4 + 2] = v.z;
          a[k][4 * c4 + 3] = v.w;
        }
      }
    }
    tslu_gepp(a, lab, w, rd == rounds - 1, sh);
  }
  if (b == 0 && tid == 0 && info && sh.zero < w && *info == 0) *info = col_offset + sh.zero + 1;
  // own rows: pivot column, then final label
  for (int i = tid; i < nrow; i += kLLThreads) sh.pos[i] = -1;
  __syncthreads();
  if (tid < w) {
    const int r = sh.sel[tid];
    if (r >= r0 && r < r0 + nrow) sh.pos[r - r0] = tid;
  }
  __syncthreads();
  int rk[kLLRows];  // pivot column + 1, then packed with the final label
#pragma unroll
  for (int k = 0; k < kLLRows; ++k) {
    lab[k] = k * kLLThreads < nrow_left ? g0 + k * kLLThreads : -1;
    rk[k] = lab[k] >= 0 ? sh.pos[lab[k] - r0] + 1 : 0;
  }
  __syncthreads();
  for (int i = tid; i < nrow; i += kLLThreads) sh.pos[i] = -1;
  __syncthreads();
  if (tid < 32) tslu_interchanges(w, r0, nrow, piv, piv_add, b == 0, sh);
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kLLRows; ++k) {
    const int moved = lab[k] >= 0 ? sh.pos[lab[k] - r0] : -1;
    lab[k] = moved >= 0 ? moved : lab[k];  // final label from here on
    rk[k] = lab[k] >= 0 ? lab[k] | (rk[k] << kRkBits) : -1;
  }
  // the block panel's other columns of moved rows to xtmp; then nobody reads
  // this panel's rows any more, and every CTA writes its rows at their places
  ll_moves_stash(ms, A, lda, w, lab, g0, left, 0, right, xtmp, s_fail);
#pragma unroll
  for (int k = 0; k < kLLRows; ++k) {
    const int r = k * kLLThreads < nrow_left ? g0 + k * kLLThreads : -1;
#pragma unroll
    for (int c = 0; c < kBaseW; ++c) a[k][c] = (r >= 0 && c < w) ? A[(int64_t)r + lda * c] : 0.f;
  }
  if (!ll_grid_barrier(bar, tag0 + 63u, s_fail)) {
    if (tid == 0) atomicExch(err, 1);
    return;
  }
  __threadfence();
  tslu_eliminate(a, rk, w, sh, A, lda);
  ll_moves_apply(ms, A, lda, w, left, 0, right, xtmp);
}

// -------------------------------------------------------------- row swaps
// The interchanges piv[0..k) (LAPACK dlaswp order: row i <-> row piv[i] -
// base, i = 0, 1, ...) are turned once into the permutation they make of the
// rows they touch (a "plan": new row dst[e] = old row src[e]), then applied
// to every column as one gather: contiguous reads of the leading rows
// instead of k dependent strided swaps per column.
constexpr int kSwapMax = kLuNbMax;              // interchanges per plan (block size cap)
constexpr int kSwapHash = 8192;                 // rows >= k touched, open addressing (<= 25 % full)
constexpr int kSwapHashShift = 32 - 13;         // multiplicative hash to 13 bits
constexpr int kSwapPlanInts = 1 + 4 * kSwapMax; // count, src[2 kSwapMax], dst[2 kSwapMax]
constexpr int kSwapThreads = 256;
// plan entries each thread gathers: all 2 kSwapMax for FP32, 2 kLuNbMax64 for FP64
template <class T>
constexpr int swap_per() { return 2 * (sizeof(T) == 8 ? kLuNbMax64 : kSwapMax) / kSwapThreads; }
constexpr int kSwapCols = 4;                    // columns per gather pass
constexpr size_t kSwapPlanSmem = sizeof(int32_t) * (2 * kSwapMax + 2 * kSwapHash);

// add != 0: piv[i] += add afterwards (pivots of a sub-panel made relative to
// the enclosing panel).
__global__ void __launch_bounds__(kSwapThreads) swap_plan_kernel(int32_t* __restrict__ piv, int k, int base,
                                                                  int32_t* __restrict__ plan, int add) {
  extern __shared__ int32_t swsm[];  // kSwapPlanSmem bytes
  int32_t* content = swsm;
  int32_t* spiv = content + kSwapMax;
  int32_t* hkey = spiv + kSwapMax;
  int32_t* hval = hkey + kSwapHash;
  __shared__ int moved;
  const int tid = threadIdx.x;
  int any = 0;
  for (int i = tid; i < k; i += kSwapThreads) {
    content[i] = i;
    spiv[i] = piv[i] - base;
    any |= spiv[i] != i;
    if (add) piv[i] += add;
  }
  // no interchange at all (the same answer in every thread): an empty plan
  // without the serial walk below
  if (!__syncthreads_or(any)) {
    if (tid == 0) plan[0] = 0;
    return;
  }
  for (int i = tid; i < kSwapHash; i += kSwapThreads) hkey[i] = -1;
  if (tid == 0) moved = 0;
  __syncthreads();
  if (tid == 0) {
    // content[x]: original row now at position x (x < k; rows >= k in the hash)
    for (int i = 0; i < k; ++i) {
      const int p = spiv[i];
      if (p == i) continue;
      int* slot;
      if (p < k) {
        slot = &content[p];
      } else {
        unsigned h = ((unsigned)p * 2654435761u) >> kSwapHashShift;
        while (hkey[h] != -1 && hkey[h] != p) h = (h + 1) & (kSwapHash - 1);
        if (hkey[h] == -1) { hkey[h] = p; hval[h] = p; }
        slot = &hval[h];
      }
      const int t = content[i];
      content[i] = *slot;
      *slot = t;
    }
  }
  __syncthreads();
  // the leading rows that changed, in order (neighbouring rows stay
  // neighbours in a warp's gather), then the rows below k that changed, in
  // any order; no interchange at all leaves an empty plan
  int32_t* src = plan + 1;
  int32_t* dst = plan + 1 + 2 * kSwapMax;
  __shared__ int wcount[kSwapThreads / 32];
  const int lane = tid & 31, warp = tid >> 5;
  int nlead = 0;
  for (int i0 = 0; i0 < k; i0 += kSwapThreads) {
    const int i = i0 + tid;
    const bool f = i < k && content[i] != i;
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wcount[warp] = __popc(bal);
    __syncthreads();
    int off = nlead, tot = 0;
#pragma unroll
    for (int w = 0; w < kSwapThreads / 32; ++w) {
      off += w < warp ? wcount[w] : 0;
      tot += wcount[w];
    }
    if (f) {
      const int e = off + __popc(bal & ((1u << lane) - 1u));
      src[e] = content[i];
      dst[e] = i;
    }
    __syncthreads();
    nlead += tot;
  }
  for (int h = tid; h < kSwapHash; h += kSwapThreads)
    if (hkey[h] >= 0 && hval[h] != hkey[h]) {
      const int e = nlead + atomicAdd(&moved, 1);
      src[e] = hval[h];
      dst[e] = hkey[h];
    }
  __syncthreads();
  if (tid == 0) plan[0] = nlead + moved;
}

template <class T>
__global__ void __launch_bounds__(kSwapThreads) swap_apply_kernel(T* __restrict__ A, int64_t lda, int64_t ncols,
                                                                   const int32_t* __restrict__ plan) {
  constexpr int kSwapPer = swap_per<T>();
  const int cnt = plan[0];
  if (cnt == 0) return;  // no interchange (the same in every thread)
  const int tid = threadIdx.x;
  int s[kSwapPer], d[kSwapPer];
#pragma unroll
  for (int r = 0; r < kSwapPer; ++r) {
    const int e = tid + r * kSwapThreads;
    s[r] = e < cnt ? plan[1 + e] : -1;
    d[r] = e < cnt ? plan[1 + 2 * kSwapMax + e] : -1;
  }
  for (int64_t c0 = (int64_t)blockIdx.x * kSwapCols; c0 < ncols; c0 += (int64_t)gridDim.x * kSwapCols) {
    T v[kSwapCols][kSwapPer];
#pragma unroll
    for (int q = 0; q < kSwapCols; ++q)
#pragma unroll
      for (int r = 0; r < kSwapPer; ++r)
        if (s[r] >= 0 && c0 + q < ncols) v[q][r] = A[s[r] + lda * (c0 + q)];
    __syncthreads();  // every read of these columns before any write
#pragma unroll
    for (int q = 0; q < kSwapCols; ++q)
#pragma unroll
      for (int r = 0; r < kSwapPer; ++r)
        if (s[r] >= 0 && c0 + q < ncols) A[d[r] + lda * (c0 + q)] = v[q][r];
  }
}

// --------------------------------------------------------------- BLAS glue
static inline cublasHandle_t H(hfpx_ctx* c) { return static_cast<cublasHandle_t>(c->cublas); }

// A stream with the cuBLAS handle bound to it.
struct Lane {
  cudaStream_t s;
  cublasHandle_t h;
  int sms;  // the device's SM count (grid caps)
};
static Lane main_lane(hfpx_ctx* c) { return {c->stream, H(c), c->num_sms}; }
static Lane panel_lane(hfpx_ctx* c) {
  return {c->stream_panel, static_cast<cublasHandle_t>(c->cublas_panel), c->num_sms};
}

static void trsm_llu(Lane l, int64_t m, int64_t n, const double* L, int64_t ldl, double* B, int64_t ldb) {
  if (m <= 0 || n <= 0) return;
  const double one = 1.0;
  cublasDtrsm(l.h, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_UNIT, (int)m, (int)n, &one,
              L, (int)ldl, B, (int)ldb);
}
static void trsm_llu(Lane l, int64_t m, int64_t n, const float* L, int64_t ldl, float* B, int64_t ldb) {
  if (m <= 0 || n <= 0) return;
  const float one = 1.0f;
  cublasStrsm(l.h, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_UNIT, (int)m, (int)n, &one,
              L, (int)ldl, B, (int)ldb);
}
static void gemm_sub(Lane l, int64_t m, int64_t n, int64_t k, const double* A, int64_t lda, const double* B,
                     int64_t ldb, double* C, int64_t ldc) {
  if (m <= 0 || n <= 0 || k <= 0) return;
  const double mone = -1.0, one = 1.0;
  cublasDgemm(l.h, CUBLAS_OP_N, CUBLAS_OP_N, (int)m, (int)n, (int)k, &mone, A, (int)lda, B, (int)ldb, &one, C,
              (int)ldc);
}
static void gemm_sub(Lane l, int64_t m, int64_t n, int64_t k, const float* A, int64_t lda, const float* B,
                     int64_t ldb, float* C, int64_t ldc) {
  if (m <= 0 || n <= 0 || k <= 0) return;
  const float mone = -1.0f, one = 1.0f;
  cublasSgemm(l.h, CUBLAS_OP_N, CUBLAS_OP_N, (int)m, (int)n, (int)k, &mone, A, (int)lda, B, (int)ldb, &one, C,
              (int)ldc);
}

// ------------------------------------------------- FP16 trailing update
// The FP32 factorisation's trailing update C -= L21 U12 runs on FP16 tensor
// cores with FP32 accumulation.  FP16 and TF32 both keep 11 significant
// bits, so the factor keeps TF32 quality at twice the tensor throughput.
// L21 holds multipliers (|l| <= 1 under partial pivoting) and converts as
// is; U12 is scaled by a power of two, from its largest magnitude, to put
// that entry in [2^14, 2^15), and the GEMM's alpha (read from device memory)
// undoes the scale exactly.
__global__ void amax_kernel(const float* __restrict__ a, int64_t lda, int64_t rows, int64_t cols,
                            unsigned* __restrict__ amax) {
  __shared__ float wmax[8];
  float m = 0.f;
  const int64_t tot = rows * cols;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = i / rows, r = i - c * rows;
    m = fmaxf(m, fabsf(a[r + lda * c]));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmaxf(m, wmax[w]);
    atomicMax(amax, __float_as_uint(m));  // non-negative floats order as their bits
  }
}

// h = a * 2^(15 - e), amax = f 2^e with f in [0.5, 1); no scaling when amax
// is null.  coef (if given) = {-2^(e - 15), 1}: alpha and beta of the update.
__global__ void to_half_kernel(const float* __restrict__ a, int64_t lda, int64_t rows, int64_t cols,
                               __half* __restrict__ h, int64_t ldh, const unsigned* __restrict__ amax,
                               float* __restrict__ coef) {
  int e = 15;
  if (amax) {
    const float m = __uint_as_float(*amax);
    if (m > 0.f) frexpf(m, &e);
  }
  const float sc = ldexpf(1.f, 15 - e);
  if (coef && blockIdx.x == 0 && threadIdx.x == 0) {
    coef[0] = -ldexpf(1.f, e - 15);
    coef[1] = 1.f;
  }
  const int64_t tot = rows * cols;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = i / rows, r = i - c * rows;
    h[r + ldh * c] = __float2half_rn(a[r + lda * c] * sc);
  }
}

// grid of 256-thread CTAs for a grid-stride loop over tot elements: at most
// 16 resident CTAs per SM
static unsigned grid_for(const Lane& l, int64_t tot) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>((tot + 255) / 256, (int64_t)std::max(1, l.sms) * 16));
}

// C = coef[0] A B^T + coef[1] C with A (m x k) and B (n x k) FP16, both
// K-major (ld elements between rows), FP32 C, FP32 accumulation: the cuBLAS
// comparison arm of the engine's own tensor-core update (gemm_tc.cu).
static void gemm16_cublas(Lane l, int64_t m, int64_t n, int64_t k, const __half* A, int64_t lda, const __half* B,
                          int64_t ldb, float* C, int64_t ldc, const float* d_coef) {
  if (m <= 0 || n <= 0 || k <= 0) return;
  cublasSetPointerMode(l.h, CUBLAS_POINTER_MODE_DEVICE);
  cublasGemmEx(l.h, CUBLAS_OP_T, CUBLAS_OP_N, (int)m, (int)n, (int)k, d_coef, A, CUDA_R_16F, (int)lda, B, CUDA_R_16F,
               (int)ldb, d_coef + 1, C, CUDA_R_32F, (int)ldc, CUBLAS_COMPUTE_32F, CUBLAS_GEMM_DEFAULT);
  cublasSetPointerMode(l.h, CUBLAS_POINTER_MODE_HOST);
}

// HFPX_LU_GEMM=cublas runs the FP16 trailing update through cuBLAS instead of
// the engine's tcgen05 kernel (for comparison).
static bool own_update_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("HFPX_LU_GEMM");
    return !(e && std::string(e) == "cublas");
  }();
  return on;
}

// K stride of the FP16 operands: kb rounded up to 8 elements (16 bytes, the
// row-stride granule of the tensor copies)
static inline int64_t ld16(int kb) { return ((int64_t)kb + 7) / 8 * 8; }

// Per-row power-of-two scales of L21: row i's largest magnitude f 2^e
// (f in [0.5, 1)) goes to [2^14, 2^15) in FP16, so small multipliers keep
// their 11 bits instead of falling into FP16's subnormal range (below 6.1e-5)
// or to zero (below 6e-8); 2^(e - 15) undoes it in the update's epilogue.
// The row maxima come from a 2-D grid (256 rows x 64 columns per CTA, one
// row per thread: a warp reads 32 consecutive rows of a column at a time),
// combined by atomicMax on the non-negative floats' bits.
constexpr int kRowScaleCols = 64;
__global__ void row_amax_kernel(const float* __restrict__ a, int64_t lda, int64_t rows, int cols,
                                unsigned* __restrict__ amax) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const int c0 = blockIdx.y * kRowScaleCols, c1 = min(cols, c0 + kRowScaleCols);
  float m = 0.f;
  for (int c = c0; c < c1; ++c) m = fmaxf(m, fabsf(a[r + lda * c]));
  atomicMax(amax + r, __float_as_uint(m));
}
// per row: rs = 2^(e - 15) (the epilogue's factor) and its exact inverse
// (the conversion's), from the row maxima
__global__ void row_scale_kernel(const unsigned* __restrict__ amax, int64_t rows, float* __restrict__ rs,
                                 float* __restrict__ inv) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const float m = __uint_as_float(amax[r]);
  int e = 15;
  if (m > 0.f) frexpf(m, &e);
  rs[r] = ldexpf(1.f, e - 15);
  inv[r] = ldexpf(1.f, 15 - e);
}

// l16 (rows x ldk, K-major FP16) = L21 (rows x cols, column-major FP32, lda)
// times the inverse row scale inv (a power of two, exact; null: unscaled),
// transposed through a 32 x 33 shared tile so that the reads (down the
// columns) and the writes (along the rows) are both coalesced.
__global__ void __launch_bounds__(256) to_half_rows_kernel(const float* __restrict__ a, int64_t lda, int64_t rows,
                                                           int cols, const float* __restrict__ inv,
                                                           __half* __restrict__ h, int64_t ldk) {
  __shared__ float t[32][33];
  const int64_t r0 = (int64_t)blockIdx.x * 32;
  const int c0 = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int i = ty; i < 32; i += 8) {
    const int64_t r = r0 + tx;
    const int cc = c0 + i;
    t[i][tx] = (r < rows && cc < cols) ? a[r + lda * cc] : 0.f;
  }
  __syncthreads();
  for (int i = ty; i < 32; i += 8) {
    const int64_t r = r0 + i;
    const int cc = c0 + tx;
    if (r < rows && cc < cols) h[r * ldk + cc] = __float2half_rn(inv ? t[tx][i] * inv[r] : t[tx][i]);
  }
}

// HFPX_LU_UPDATE=tf32 keeps the trailing update on TF32 tensor cores.
static bool fp16_update_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("HFPX_LU_UPDATE");
    return !(e && std::string(e) == "tf32");
  }();
  return on;
}

// ------------------------------------------------------------- profiling
// HFPX_PROFILE=1 in the environment: every LU phase is synchronised and
// timed on the host, and a per-phase summary goes to stderr after each
// factorisation / solve.  Off by default (no synchronisation, no cost).
struct PhaseProfile {
  bool on = false;
  double t[8] = {0};
  int n[8] = {0};
  const char* name[8] = {"panel", "laswp", "trsm", "gemm", "convert", "trsv", "residual", "other"};
  std::chrono::steady_clock::time_point t0;
  cudaStream_t s = nullptr;
  void begin(cudaStream_t st) {
    if (!on) return;
    s = st;
    cudaDeviceSynchronize();
    t0 = std::chrono::steady_clock::now();
  }
  void end(int k) {
    if (!on) return;
    cudaDeviceSynchronize();
    const auto t1 = std::chrono::steady_clock::now();
    t[k] += std::chrono::duration<double, std::milli>(t1 - t0).count();
    n[k] += 1;
    t0 = t1;
  }
  void report(const char* what) {
    if (!on) return;
    std::fprintf(stderr, "[hfpx profile] %s:", what);
    for (int k = 0; k < 8; ++k)
      if (n[k]) std::fprintf(stderr, " %s %.1f ms (%d)", name[k], t[k], n[k]);
    std::fprintf(stderr, "\n");
    for (int k = 0; k < 8; ++k) { t[k] = 0; n[k] = 0; }
  }
};
static PhaseProfile& prof() {
  static PhaseProfile p = [] {
    PhaseProfile q;
    const char* e = std::getenv("HFPX_PROFILE");
    q.on = e && *e == '1';
    return q;
  }();
  return p;
}

// HFPX_PROFILE=2: no synchronisation; timing events around every wait of the
// look-ahead show which stream is on the critical path.  Per step: the main
// stream's stall waiting for the panel, the panel stream's stall waiting for
// the next block column, the panel's own duration, and the main stream's
// work; summary to stderr after each factorisation.
struct StepTimeline {
  bool on = false;
  struct Step {
    int64_t rest;
    cudaEvent_t m_idle, m_go, p_idle, p_go, p_done, m_done;
  };
  std::vector<Step> steps;
  void add(int64_t rest) {
    Step s{rest, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    for (cudaEvent_t* e : {&s.m_idle, &s.m_go, &s.p_idle, &s.p_go, &s.p_done, &s.m_done}) cudaEventCreate(e);
    steps.push_back(s);
  }
  void report() {
    if (!on || steps.empty()) return;
    auto el = [](cudaEvent_t a, cudaEvent_t b) {
      float ms = 0.f;
      return cudaEventElapsedTime(&ms, a, b) == cudaSuccess ? (double)ms : 0.0;
    };
    double m_stall = 0, p_stall = 0, panel = 0, main = 0;
    std::fprintf(stderr, "[hfpx timeline] step rest panel_ms main_ms main_wait_ms panel_wait_ms\n");
    for (size_t i = 0; i < steps.size(); ++i) {
      const Step& s = steps[i];
      const double ms = el(s.m_idle, s.m_go), ps = el(s.p_idle, s.p_go), pd = el(s.p_go, s.p_done),
                   md = el(s.m_go, s.m_done);
      m_stall += ms;
      p_stall += ps;
      panel += pd;
      main += md;
      if (i % std::max<size_t>(1, steps.size() / 8) == 0 || i + 1 == steps.size())
        std::fprintf(stderr, "[hfpx timeline] %4zu %7lld %8.3f %8.3f %8.3f %8.3f\n", i, (long long)s.rest, pd, md, ms, ps);
    }
    std::fprintf(stderr, "[hfpx timeline] total: panel %.1f ms, main %.1f ms, main waiting %.1f ms, panel waiting %.1f ms\n",
                 panel, main, m_stall, p_stall);
    for (Step& s : steps)
      for (cudaEvent_t e : {s.m_idle, s.m_go, s.p_idle, s.p_go, s.p_done, s.m_done}) cudaEventDestroy(e);
    steps.clear();
    cudaGetLastError();  // elapsed times of the last step's unrecorded events
  }
};
static StepTimeline& timeline() {
  static StepTimeline t = [] {
    StepTimeline q;
    const char* e = std::getenv("HFPX_PROFILE");
    q.on = e && *e == '2';
    return q;
  }();
  return t;
}

// --------------------------------------------------------------- driver
template <class T>
struct LuWork {
  PanelScratch<T> sc{};
  int64_t* d_info = nullptr;
  int grid = 0;
  // register-resident FP32 panel: exchange words [2][kLLMaxCtas][kLLSlot]
  // (zeroed), failure word, launches so far (names the tags)
  uint64_t* ll_slots = nullptr;
  int* ll_err = nullptr;
  uint32_t ll_launches = 0;
  // FP32: L11^-1 (nb x nb) and a copy of A12 (nb x n) for U12 = L11^-1 A12
  // as one TF32 GEMM
  T* linv = nullptr;
  T* a12 = nullptr;
  // row-swap plans: one for the panel stream's own swaps, one per block
  // (read by the right and left swaps of that block on two streams)
  int32_t* plan_panel = nullptr;
  int32_t* plans = nullptr;
  // FP32 with the FP16 trailing update: L21 (rest x nb) and scaled U12
  // (nb x rest) in FP16, U12's largest magnitude and the update's alpha/beta
  // (layouts: l16 rest x ld16(kb) K-major, u16 ld16(kb) x n column-major)
  __half* l16 = nullptr;
  __half* u16 = nullptr;
  unsigned* amax = nullptr;
  float* coef = nullptr;
  // the tensor-core update's failure word, and its CTA cap (the SMs the
  // main stream may take at this step)
  int* tc_err = nullptr;
  int gemm_ctas = 0;
  // per-row maxima and scales of the FP16 L21 (own update only; cuBLAS takes
  // it unscaled)
  unsigned* row_amax = nullptr;
  float* row_scale = nullptr;   // n_rows scales, then n_rows inverse scales
  int64_t n_rows = 0;
  // moved rows of one base panel across the block panel: [2 kBaseW][nb]
  float* xtmp = nullptr;
  // tournament candidates: [kTsluMaxCtas][kBaseW][kBaseW] rows, then labels
  float* tslu = nullptr;
  // panel_update32_kernel's ticket counter (zero between launches)
  unsigned* pu32_ticket = nullptr;
  // panel stream's U12 by inverse (panel_u12_by_inverse): inv(L11), the
  // inverse's scratch and a copy of A12, for a left half of up to nb / 2
  float* pinv = nullptr;
};

// Remaining size below which the main stream leaves SMs to the panel stream
// (HFPX_LU_CAP_REST; 0: never, a large value: always).  Measured on a B200 at
// N = 72 000 (bench, nb 1536): below ~62 000 remaining rows a panel outlasts
// the trailing update; factor 501 ms with this threshold, 505 ms capped at
// every step, 521 ms never capped.
static int64_t lu_cap_rest() {
  static const int64_t v = [] {
    const char* e = std::getenv("HFPX_LU_CAP_REST");
    return e ? std::max<int64_t>(0, std::atoll(e)) : (int64_t)62000;
  }();
  return v;
}

// FP32 base panels: partial pivoting in the register-resident kernel by
// default; HFPX_LU_PANEL=smem takes the shared-memory kernel, =tslu the
// tournament-pivoting kernel where its candidates fit.
enum class PanelKind { Tournament, Register, Shared };
static PanelKind panel_kind() {
  static const PanelKind k = [] {
    const char* e = std::getenv("HFPX_LU_PANEL");
    const std::string s = e ? e : "";
    return s == "smem" ? PanelKind::Shared : s == "tslu" ? PanelKind::Tournament : PanelKind::Register;
  }();
  return k;
}
static bool ll_panel_enabled() { return panel_kind() != PanelKind::Shared; }

// The register-resident panel takes m rows.
template <class T>
static bool ll_fits(const LuWork<T>& wk, int64_t m) {
  return sizeof(T) == 4 && wk.ll_slots && wk.xtmp && (m + kLLCap - 1) / kLLCap <= kLLMaxCtas && ll_panel_enabled();
}
// ... and with tournament pivoting.
template <class T>
static bool tslu_fits(const LuWork<T>& wk, int64_t m) {
  return wk.tslu && ll_fits(wk, m) && (m + kLLCap - 1) / kLLCap <= kTsluMaxCtas;
}

struct PanelSpan {
  int c0 = 0, bw = 0;
  bool eager = false;
};

__global__ void identity_kernel(float* a, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i < n) a[i + (int64_t)n * j] = i == j ? 1.f : 0.f;
}

// Inverses of the 32 x 32 diagonal blocks of the unit lower L (lda) into X
// (ld ldx; its strictly upper part and diagonal already hold the identity's):
// one CTA per block, thread c forward-substitutes column c of the inverse.
__global__ void __launch_bounds__(kBaseW) unit_lower_diag_inv_kernel(const float* __restrict__ L, int64_t lda,
                                                                     float* __restrict__ X, int64_t ldx) {
  __shared__ float s[kBaseW][kBaseW + 1];
  const int c = threadIdx.x;
  const int64_t o = (int64_t)blockIdx.x * kBaseW;
  for (int t = 0; t < kBaseW; ++t) s[c][t] = L[o + c + lda * (o + t)];
  __syncwarp();
  float x[kBaseW];
#pragma unroll
  for (int i = 0; i < kBaseW; ++i) {
    float acc = i == c ? 1.f : 0.f;  // rows above c stay 0: every x_t with t < c is 0
#pragma unroll
    for (int t = 0; t < i; ++t) acc = fmaf(-s[i][t], x[t], acc);
    x[i] = acc;
  }
#pragma unroll
  for (int i = 1; i < kBaseW; ++i)
    if (i > c) X[o + i + ldx * (o + c)] = x[i];
}

// inv(L11) for a kb x kb unit lower L11 with kb = 32 * 2^k, level by level:
// the 32 x 32 diagonal blocks, then for b = 32, 64, .. kb / 2 every 2b x 2b
// diagonal block [L1 0; L2 L3] from its halves' inverses,
// inv = [inv(L1) 0; -inv(L3) L2 inv(L1) inv(L3)], as two strided-batched
// GEMMs (the pairs sit at a fixed stride down the diagonal).  Replaces the
// kb x kb triangular solve on the identity (13 launches at kb = 2048).
// X holds the identity on entry; T: scratch of kb * kb / 4 floats.
static bool unit_lower_inverse(Lane l, int kb, const float* L, int64_t lda, float* X, float* T) {
  const int blocks = kb / kBaseW;
  if (kb < 2 * kBaseW || kb % kBaseW || (blocks & (blocks - 1))) return false;
  ++g_launches;
  unit_lower_diag_inv_kernel<<<blocks, kBaseW, 0, l.s>>>(L, lda, X, kb);
  const float one = 1.f, zero = 0.f, mone = -1.f;
  for (int b = kBaseW; b < kb; b *= 2) {
    const int nbatch = kb / (2 * b);
    const long long sL = 2LL * b * (lda + 1), sX = 2LL * b * (kb + 1), sT = (long long)b * b;
    // T = L2 inv(L1), then X21 = -inv(L3) T
    cublasSgemmStridedBatched(l.h, CUBLAS_OP_N, CUBLAS_OP_N, b, b, b, &one, L + b, (int)lda, sL, X, kb, sX, &zero, T,
                              b, sT, nbatch);
    cublasSgemmStridedBatched(l.h, CUBLAS_OP_N, CUBLAS_OP_N, b, b, b, &mone, X + b + (int64_t)b * kb, kb, sX, T, b,
                              sT, &zero, X + b, kb, sX, nbatch);
  }
  return true;
}

// U12 = L11^-1 A12 for columns [c0, c0 + nc) of the trailing block row (B:
// its column 0).  FP32: with the inverse of the unit lower L11 (made by the
// step's first call, with_inverse: unit_lower_inverse, or a kb x kb
// triangular solve on the identity), one TF32 GEMM; the triangular solve over
// the block row is the slow path it replaces.  FP64: triangular solve.
template <class T>
static void block_row_solve(Lane l, LuWork<T>& wk, int kb, int64_t c0, int64_t nc, const T* L, int64_t lda, T* B,
                            bool with_inverse) {
  if (nc <= 0) return;
  B += lda * c0;
  if constexpr (sizeof(T) == 4) {
    if (wk.linv && wk.a12) {
      if (with_inverse) {
        ++g_launches;
        identity_kernel<<<dim3((kb + 127) / 128, kb), 128, 0, l.s>>>(wk.linv, kb);
        if (!unit_lower_inverse(l, kb, L, lda, wk.linv, wk.a12)) trsm_llu(l, kb, kb, L, lda, wk.linv, kb);
      }
      cudaMemcpy2DAsync(wk.a12, sizeof(T) * kb, B, sizeof(T) * lda, sizeof(T) * kb, nc, cudaMemcpyDeviceToDevice, l.s);
      const float one = 1.f, zero = 0.f;
      cublasSgemm(l.h, CUBLAS_OP_N, CUBLAS_OP_N, kb, (int)nc, kb, &one, wk.linv, kb, wk.a12, kb, &zero, B, (int)lda);
      return;
    }
  }
  trsm_llu(l, kb, nc, L, lda, B, lda);
}

// Trailing update of step k (FP32 with the FP16 update): the FP16 copy of
// L21 (rest x kb, K-major), once per step ...
template <class T>
static void prepare_l21(Lane l, LuWork<T>& wk, int kb, int64_t rest, const T* L21, int64_t lda) {
  if constexpr (sizeof(T) == 4) {
    if (wk.l16 && rest > 0) {
      const bool scaled = wk.row_scale && wk.row_amax && own_update_enabled();
      if (scaled) {
        cudaMemsetAsync(wk.row_amax, 0, sizeof(unsigned) * rest, l.s);
        ++g_launches;
        row_amax_kernel<<<dim3((unsigned)((rest + 255) / 256), (unsigned)((kb + kRowScaleCols - 1) / kRowScaleCols)),
                          256, 0, l.s>>>(L21, lda, rest, kb, wk.row_amax);
      }
      float* inv = scaled ? wk.row_scale + (size_t)wk.n_rows : nullptr;
      if (scaled) {
        ++g_launches;
        row_scale_kernel<<<(unsigned)((rest + 255) / 256), 256, 0, l.s>>>(wk.row_amax, rest, wk.row_scale, inv);
      }
      ++g_launches;
      to_half_rows_kernel<<<dim3((unsigned)((rest + 31) / 32), (unsigned)((kb + 31) / 32)), 256, 0, l.s>>>(
          L21, lda, rest, kb, scaled ? inv : nullptr, wk.l16, ld16(kb));
    }
  }
}
// ... and of U12's columns [c0, c0 + nc), scaled by their own largest
// magnitude into the GEMM's alpha (wk.amax and wk.coef are reused by the next
// range: same stream, so the GEMM of this range has read them first)
template <class T>
static void prepare_u12(Lane l, LuWork<T>& wk, int kb, int64_t c0, int64_t nc, const T* U12, int64_t lda) {
  if constexpr (sizeof(T) == 4) {
    if (wk.l16 && nc > 0) {
      U12 += lda * c0;
      cudaMemsetAsync(wk.amax, 0, sizeof(unsigned), l.s);
      ++g_launches;
      amax_kernel<<<grid_for(l, nc * kb), 256, 0, l.s>>>(U12, lda, kb, nc, wk.amax);
      ++g_launches;
      to_half_kernel<<<grid_for(l, nc * kb), 256, 0, l.s>>>(U12, lda, kb, nc, wk.u16 + (size_t)ld16(kb) * c0, ld16(kb),
                                                            wk.amax, wk.coef);
    }
  }
}

template <class T>
static int update_gemm(hfpx_ctx* c, Lane l, LuWork<T>& wk, int kb, int64_t rest, int64_t c0, int64_t nc, const T* L21,
                       const T* U12, T* C, int64_t lda) {
  if constexpr (sizeof(T) == 4) {
    if (wk.l16) {
      const int64_t k16 = ld16(kb);
      const __half* B = wk.u16 + (size_t)k16 * c0;
      if (own_update_enabled() && wk.tc_err)
        return tc_update_f16(c, l.s, rest, nc, kb, wk.l16, k16, B, k16, C, lda, wk.coef,
                             wk.row_amax ? wk.row_scale : nullptr, wk.tc_err, wk.gemm_ctas);
      gemm16_cublas(l, rest, nc, kb, wk.l16, k16, B, k16, C, lda, wk.coef);
      return 0;
    }
  }
  gemm_sub(l, rest, nc, kb, L21, lda, U12 + lda * c0, lda, C, lda);
  return 0;
}

// CTAs for a panel of m rows: enough for the panel to fit in shared memory,
// at least kPanelCtas when there are rows for them, never more than the SMs.
// Fewer CTAs than SMs leave room for the trailing update running beside it
// and make the per-column grid barrier cheaper.
constexpr int kPanelCtas = 48;
constexpr size_t kPanelSmemCap = 200 * 1024;

template <class T>
static int panel_ctas(hfpx_ctx* c, int64_t m, int w) {
  const int64_t per_cta_rows = (int64_t)((kPanelSmemCap - kBaseW * sizeof(T)) / (w * sizeof(T)));
  const int64_t need = (m + per_cta_rows - 1) / per_cta_rows;
  const int64_t want = std::min<int64_t>(kPanelCtas, std::max<int64_t>(1, (m + 31) / 32));
  return (int)std::min<int64_t>(c->num_sms, std::max(need, want));
}

template <class T>
static int panel_base(hfpx_ctx* c, Lane l, LuWork<T>& wk, T* A, int64_t lda, int64_t m, int w, int32_t* piv,
                      int64_t col_offset, const PanelSpan& sp) {
  if constexpr (sizeof(T) == 4) {
    if (ll_fits(wk, m)) {
      int G = (int)((m + kLLCap - 1) / kLLCap);
      int rpc = (int)((m + G - 1) / G);
      uint32_t tag0 = (++wk.ll_launches) << 6;
      int left = sp.eager ? sp.c0 : 0, right = sp.eager ? sp.bw - sp.c0 - w : 0, piv_add = sp.eager ? sp.c0 : 0;
      ++g_launches;
      if (tslu_fits(wk, m)) {
        void* targs[] = {&A,          &lda, &m,         &w,    &rpc,   &piv,     &wk.ll_slots, &wk.tslu,
                         &wk.d_info, &col_offset, &tag0, &wk.ll_err, &left, &right, &wk.xtmp,     &piv_add};
        return check_cuda(c,
                          cudaLaunchCooperativeKernel((void*)panel_tslu_kernel, dim3(G), dim3(kLLThreads), targs, 0,
                                                      l.s),
                          "panel_tslu_kernel launch");
      }
      void* args[] = {&A,  &lda,       &m,           &w,    &rpc,  &piv,    &wk.ll_slots, &wk.d_info,
                      &col_offset, &tag0, &wk.ll_err, &left, &right, &wk.xtmp, &piv_add};
      return check_cuda(c, cudaLaunchCooperativeKernel((void*)panel_ll_kernel, dim3(G), dim3(kLLThreads), args, 0, l.s),
                        "panel_ll_kernel launch");
    }
  }
  int G = panel_ctas<T>(c, m, w);
  int rpc = (int)((m + G - 1) / G);
  size_t smem = (size_t)w * rpc * sizeof(T) + kBaseW * sizeof(T);
  if (smem > kPanelSmemCap) return set_error(c, HFPX_ERR_ARG, "panel too tall for shared memory");
  static PerDeviceOnce attr;  // one per instantiation of T
  smem_attr_once(attr, panel_base_kernel<T>, (int)kPanelSmemCap);
  void* args[] = {&A, &lda, &m, &w, &rpc, &piv, &wk.sc, &wk.d_info, &col_offset};
  ++g_launches;
  cudaError_t e =
      cudaLaunchCooperativeKernel((void*)panel_base_kernel<T>, dim3(G), dim3(kPanelThreads), args, smem, l.s);
  return check_cuda(c, e, "panel_base_kernel launch");
}

static void swap_plan(Lane l, int32_t* piv, int k, int base, int32_t* plan, int add = 0) {
  if (k <= 0) return;
  ++g_launches;
  static PerDeviceOnce attr;
  smem_attr_once(attr, swap_plan_kernel, (int)kSwapPlanSmem);
  swap_plan_kernel<<<1, kSwapThreads, kSwapPlanSmem, l.s>>>(piv, k, base, plan, add);
}

template <class T>
static void swap_apply(Lane l, T* A, int64_t lda, int64_t ncols, const int32_t* plan) {
  if (ncols <= 0) return;
  const int64_t blocks = std::min<int64_t>((ncols + kSwapCols - 1) / kSwapCols, (int64_t)std::max(1, l.sms) * 8);
  ++g_launches;
  swap_apply_kernel<T><<<(unsigned)blocks, kSwapThreads, 0, l.s>>>(A, lda, ncols, plan);
}

// dlaswp: interchanges piv[0..k) (minus base) on columns [0, ncols) of A,
// through the plan buffer.
template <class T>
static void laswp(Lane l, T* A, int64_t lda, int64_t ncols, int32_t* piv, int k, int base, int32_t* plan) {
  if (ncols <= 0 || k <= 0) return;
  swap_plan(l, piv, k, base, plan);
  swap_apply(l, A, lda, ncols, plan);
}

// Lowest level of the FP32 panel recursion, a 32-column left half: dgetrf2's
// U12 = L11^-1 A12 (unit lower L11) and A22 -= L21 U12 in one launch, where
// cuBLAS spends a TRSM launch of ~20 us on the 32 x 32 triangle alone.
// Every CTA solves U12 (w2 <= 32 columns) in shared memory, the same
// arithmetic in each, and one CTA stores it (below); then each thread takes
// one row of A22 through the 32-term update in FP32 (U12 broadcast from
// shared memory, L21 and A22 read once, coalesced down the columns).  U12 overwrites A12
// in place, so it is stored by the last CTA to have read A12: each CTA takes
// a ticket once its copy is in shared memory, and the CTA holding the last
// ticket stores U12 and puts the counter back to 0 for the next launch (the
// launches of one factorisation are ordered on one stream).  No CTA waits for
// another.
constexpr int kPu32Threads = 256;
__global__ void __launch_bounds__(kPu32Threads) panel_update32_kernel(float* __restrict__ A, int64_t lda, int64_t m,
                                                                      int w2, unsigned* __restrict__ ticket) {
  __shared__ float s_l[kBaseW][kBaseW + 1];  // L11(i, t)
  __shared__ __align__(16) float s_u[kBaseW][kBaseW];  // A12 -> U12 (t, c)
  __shared__ bool s_last;
  const int tid = threadIdx.x;
  for (int e = tid; e < kBaseW * kBaseW; e += kPu32Threads) {
    const int i = e % kBaseW, t = e / kBaseW;  // column-major: neighbouring threads, neighbouring rows
    s_l[i][t] = A[i + lda * t];
    s_u[i][t] = t < w2 ? A[i + lda * (kBaseW + t)] : 0.f;
  }
  __syncthreads();
  if (tid == 0) s_last = atomicAdd(ticket, 1u) == gridDim.x - 1u;
  if (tid < kBaseW) {
    // forward substitution down column c of U12 (row i takes rows t < i)
    const int c = tid;
    float u[kBaseW];
#pragma unroll
    for (int i = 0; i < kBaseW; ++i) u[i] = s_u[i][c];
#pragma unroll
    for (int t = 0; t < kBaseW; ++t)
#pragma unroll
      for (int i = t + 1; i < kBaseW; ++i) u[i] = fmaf(-s_l[i][t], u[t], u[i]);
#pragma unroll
    for (int i = 0; i < kBaseW; ++i) s_u[i][c] = u[i];
  }
  __syncthreads();
  if (s_last) {
    for (int e = tid; e < kBaseW * w2; e += kPu32Threads) {
      const int i = e % kBaseW, t = e / kBaseW;
      A[i + lda * (kBaseW + t)] = s_u[i][t];
    }
    if (tid == 0) *ticket = 0u;
  }
  const int64_t r = kBaseW + (int64_t)blockIdx.x * kPu32Threads + tid;
  if (r >= m) return;
  float acc[kBaseW];
#pragma unroll
  for (int c = 0; c < kBaseW; ++c) acc[c] = c < w2 ? A[r + lda * (kBaseW + c)] : 0.f;
#pragma unroll 4
  for (int t = 0; t < kBaseW; ++t) {
    const float l = A[r + lda * t];
    const float4* ut = reinterpret_cast<const float4*>(s_u[t]);
#pragma unroll
    for (int q = 0; q < kBaseW / 4; ++q) {
      const float4 v = ut[q];
      acc[4 * q] = fmaf(-l, v.x, acc[4 * q]);
      acc[4 * q + 1] = fmaf(-l, v.y, acc[4 * q + 1]);
      acc[4 * q + 2] = fmaf(-l, v.z, acc[4 * q + 2]);
      acc[4 * q + 3] = fmaf(-l, v.w, acc[4 * q + 3]);
    }
  }
#pragma unroll
  for (int c = 0; c < kBaseW; ++c)
    if (c < w2) A[r + lda * (kBaseW + c)] = acc[c];
}

// U12 = L11^-1 A12 of a recursion node whose left half is w1 >= 512 wide
// (FP32, panel stream): inv(L11) by unit_lower_inverse into the panel's own
// buffer, A12 copied beside it, one TF32 GEMM back into A12.  A cuBLAS
// triangular solve of that shape is launch- and latency-bound (~140 us at
// w1 = 1024 on a B200); this is 13 launches of small GEMMs.  Smaller halves
// keep the triangular solve.  False: not taken.
constexpr int kPanelInvMin = 512;
static bool panel_u12_by_inverse(Lane l, LuWork<float>& wk, int w1, int w2, float* A, int64_t lda) {
  const int blocks = w1 / kBaseW;
  if (!wk.pinv || w1 < kPanelInvMin || w1 % kBaseW || (blocks & (blocks - 1)) || w2 > w1) return false;
  float* X = wk.pinv;
  float* T = X + (size_t)w1 * w1;
  float* C = T + (size_t)w1 * w1;  // the inverse's scratch needs w1 * w1 / 4
  ++g_launches;
  identity_kernel<<<dim3((w1 + 127) / 128, w1), 128, 0, l.s>>>(X, w1);
  unit_lower_inverse(l, w1, A, lda, X, T);
  cudaMemcpy2DAsync(C, sizeof(float) * w1, A + lda * w1, sizeof(float) * lda, sizeof(float) * w1, w2,
                    cudaMemcpyDeviceToDevice, l.s);
  const float one = 1.f, zero = 0.f;
  cublasSgemm(l.h, CUBLAS_OP_N, CUBLAS_OP_N, w1, w2, w1, &one, X, w1, C, w1, &zero, A + lda * w1, (int)lda);
  return true;
}

// dgetrf2-style recursion on an m x w panel (pivots relative to A's top row).
// sp.c0: column (and row) offset of this sub-panel inside its block panel of
// sp.bw columns.  sp.eager: every base panel applies its own interchanges to
// the whole block panel, so the recursion swaps nothing between its halves.
template <class T>
static int panel_rec(hfpx_ctx* c, Lane l, LuWork<T>& wk, T* A, int64_t lda, int64_t m, int w, int32_t* piv,
                     int64_t col_offset, PanelSpan sp) {
  PhaseProfile& P = prof();
  if (w <= kBaseW) {
    P.begin(l.s);
    const int rc = panel_base(c, l, wk, A, lda, m, w, piv, col_offset, sp);
    P.end(0);
    return rc;
  }
  // left half rounded up to whole base panels (768 -> 384 -> 192 -> 96 ->
  // 64 + 32), so every base panel but a ragged last one is 32 wide
  const int w1 = (w / 2 + kBaseW - 1) / kBaseW * kBaseW, w2 = w - w1;
  int rc = panel_rec(c, l, wk, A, lda, m, w1, piv, col_offset, sp);
  if (rc) return rc;
  P.begin(l.s);
  if (!sp.eager) laswp(l, A + lda * w1, lda, w2, piv, w1, 0, wk.plan_panel);
  P.end(1);
  bool fused = false;
  if constexpr (sizeof(T) == 4) {
    if (w1 == kBaseW && w2 <= kBaseW && m > w1 && wk.pu32_ticket) {
      ++g_launches;
      panel_update32_kernel<<<(unsigned)((m - w1 + kPu32Threads - 1) / kPu32Threads), kPu32Threads, 0, l.s>>>(
          A, lda, m, w2, wk.pu32_ticket);
      P.end(3);
      fused = true;
    }
  }
  if (!fused) {
    bool solved = false;
    if constexpr (sizeof(T) == 4) solved = panel_u12_by_inverse(l, wk, w1, w2, A, lda);
    if (!solved) trsm_llu(l, w1, w2, A, lda, A + lda * w1, lda);
    P.end(2);
    gemm_sub(l, m - w1, w2, w1, A + w1, lda, A + lda * w1, lda, A + w1 + lda * w1, lda);
    P.end(3);
  }
  PanelSpan sr = sp;
  sr.c0 += w1;
  rc = panel_rec(c, l, wk, A + w1 + lda * w1, lda, m - w1, w2, piv + w1, col_offset + w1, sr);
  if (rc) return rc;
  if (!sp.eager) {
    P.begin(l.s);
    // the right half's interchanges on the left half's columns; its pivots
    // become relative to this panel's top
    swap_plan(l, piv + w1, w2, 0, wk.plan_panel, w1);
    swap_apply(l, A + w1, lda, w1, wk.plan_panel);
    P.end(1);
  }
  return 0;
}

// Factor block panel [0, w) of A (m rows), pivots relative to its top.
template <class T>
static int block_panel(hfpx_ctx* c, Lane l, LuWork<T>& wk, T* A, int64_t lda, int64_t m, int w, int32_t* piv,
                       int64_t col_offset) {
  PanelSpan sp;
  sp.bw = w;
  sp.eager = wk.xtmp != nullptr && ll_fits(wk, m);
  return panel_rec(c, l, wk, A, lda, m, w, piv, col_offset, sp);
}

// Pivots of block b are relative to the block's first row until the end.
__global__ void globalise_piv_kernel(int32_t* piv, int64_t n, int nb) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) piv[i] += (int32_t)((i / nb) * nb);
}

// Right-looking blocked LU with depth-1 look-ahead.  Step k on the main
// stream: for the next block column only, the swaps of panel k, its part of
// U12 = L11^-1 A12 and its update; then (while the panel stream factors that
// next block column) the same for everything right of it.
// Swaps on the columns left of each panel wait for the step that last read
// those columns and run on a third stream.
template <class T>
// src64 (FP32 only): A is first filled from this FP64 matrix (same ld), the
// first block column before the first panel, the rest beside it.
static int lu_factor(hfpx_ctx* c, T* A, int64_t lda, int64_t n, int32_t* piv, int64_t* info_out,
                     const double* src64 = nullptr) {
  LuWork<T> wk;
  const int G = c->num_sms;
  // work buffers live in the context and are reused by later factorisations
  auto alloc = [&](int slot, size_t bytes) -> void* { return ctx_scratch(c, slot, bytes); };
  wk.sc.cand = (T*)alloc(kScrPanelCand, sizeof(T) * 2 * G * kBaseW);
  wk.sc.cmax = (double*)alloc(kScrPanelMax, sizeof(double) * 2 * G);
  wk.sc.cidx = (int*)alloc(kScrPanelIdx, sizeof(int) * 2 * G);
  wk.sc.rowj = (T*)alloc(kScrPanelRowj, sizeof(T) * 2 * kBaseW);
  wk.d_info = (int64_t*)alloc(kScrInfo, sizeof(int64_t));
  const int64_t n_blocks = (n + lu_block_size(sizeof(T) == 4) - 1) / lu_block_size(sizeof(T) == 4);
  wk.plan_panel = (int32_t*)alloc(kScrPlanPanel, sizeof(int32_t) * kSwapPlanInts);
  wk.plans = (int32_t*)alloc(kScrPlans, sizeof(int32_t) * kSwapPlanInts * (size_t)n_blocks);
  // two column buffers of per-CTA words, two barriers of one word per CTA,
  // then panel_update32_kernel's ticket
  const size_t ll_bytes = sizeof(uint64_t) * (2 * kLLMaxCtas * kLLSlot + 2 * kLLMaxCtas + 1);
  if (sizeof(T) == 4) {
    wk.ll_slots = (uint64_t*)alloc(kScrLLSlots, ll_bytes);
    if (wk.ll_slots) wk.pu32_ticket = reinterpret_cast<unsigned*>(wk.ll_slots + 2 * kLLMaxCtas * kLLSlot + 2 * kLLMaxCtas);
    wk.ll_err = (int*)alloc(kScrLLErr, sizeof(int));
    // optional: without it the panels keep partial pivoting
    if (panel_kind() == PanelKind::Tournament)
      wk.tslu = (float*)alloc(kScrTslu, (sizeof(float) * kBaseW + sizeof(int)) * kTsluMaxCtas * kBaseW);
    // optional: without room for them the block row takes the triangular solve
    const size_t nb = (size_t)lu_block_size(sizeof(T) == 4);
    wk.xtmp = (float*)alloc(kScrXtmp, sizeof(float) * 2 * kBaseW * nb);
    wk.linv = (T*)alloc(kScrLinv, sizeof(T) * nb * nb);
    wk.a12 = (T*)alloc(kScrA12, sizeof(T) * nb * (size_t)n);
    if (!wk.linv || !wk.a12) wk.linv = wk.a12 = nullptr;
    // optional: without it the recursion's wide halves keep the triangular solve
    const size_t w1max = (nb / 2 + kBaseW - 1) / kBaseW * kBaseW;  // widest left half of a block panel
    if (wk.linv) wk.pinv = (float*)alloc(kScrPanelInv, sizeof(float) * w1max * w1max * 3);
    // optional too: without them the update stays on TF32
    if (fp16_update_enabled()) {
      wk.l16 = (__half*)alloc(kScrL16, sizeof(__half) * nb * (size_t)n);
      wk.u16 = (__half*)alloc(kScrU16, sizeof(__half) * nb * (size_t)n);
      wk.amax = (unsigned*)alloc(kScrAmax, sizeof(unsigned));
      wk.coef = (float*)alloc(kScrCoef, 2 * sizeof(float));
      wk.tc_err = (int*)alloc(kScrTcErr, sizeof(int));
      wk.row_scale = (float*)alloc(kScrRowScale, sizeof(float) * 3 * (size_t)n);
      wk.n_rows = n;
      if (wk.row_scale) wk.row_amax = reinterpret_cast<unsigned*>(wk.row_scale + 2 * n);
      if (!wk.l16 || !wk.u16 || !wk.amax || !wk.coef) wk.l16 = wk.u16 = nullptr;
    }
  }
  int rc = 0;
  if (!wk.sc.cand || !wk.sc.cmax || !wk.sc.cidx || !wk.sc.rowj || !wk.d_info || !wk.plan_panel || !wk.plans ||
      (sizeof(T) == 4 && (!wk.ll_slots || !wk.ll_err)))
    rc = set_error(c, HFPX_ERR_NOMEM, "LU scratch");
  if (!rc && wk.ll_slots) {
    cudaMemsetAsync(wk.ll_slots, 0, ll_bytes, c->stream);
    cudaMemsetAsync(wk.ll_err, 0, sizeof(int), c->stream);
  }
  if (!rc && wk.tc_err) cudaMemsetAsync(wk.tc_err, 0, sizeof(int), c->stream);
  wk.gemm_ctas = c->num_sms;
  const Lane M = main_lane(c), Pn = panel_lane(c);
  const cudaStream_t S = c->stream_left;
  const int kNb = lu_block_size(sizeof(T) == 4);
  cudaEvent_t ev_panel = nullptr, ev_next = nullptr, ev_rest = nullptr, ev_left = nullptr, ev_start = nullptr;
  for (cudaEvent_t* e : {&ev_panel, &ev_next, &ev_rest, &ev_left, &ev_start})
    if (!rc) rc = check_cuda(c, cudaEventCreateWithFlags(e, cudaEventDisableTiming), "LU events");
  PhaseProfile& P = prof();
  if (!rc) {
    cudaMemsetAsync(wk.d_info, 0, sizeof(int64_t), c->stream);
    const int kb0 = (int)std::min<int64_t>(kNb, n);
    if constexpr (sizeof(T) == 4)
      if (src64) launch_convert_f32(src64, lda, kb0, A, M.s);
    // the panel and swap streams start after everything queued on the main stream
    cudaEventRecord(ev_start, M.s);
    cudaStreamWaitEvent(Pn.s, ev_start, 0);
    cudaStreamWaitEvent(S, ev_start, 0);
    rc = block_panel(c, Pn, wk, A, lda, n, kb0, piv, 0);
    if (!rc) swap_plan(Pn, piv, kb0, 0, wk.plans);
    cudaEventRecord(ev_panel, Pn.s);
    if constexpr (sizeof(T) == 4)
      if (src64 && n > kb0) launch_convert_f32(src64 + lda * kb0, lda, n - kb0, A + lda * kb0, M.s);
  }
  for (int64_t k = 0; k < n && !rc; k += kNb) {
    const int kb = (int)std::min<int64_t>(kNb, n - k);
    T* Akk = A + k + lda * k;
    StepTimeline& TL = timeline();
    StepTimeline::Step* ts = nullptr;
    if (TL.on) {
      TL.add(n - k - kb);
      ts = &TL.steps.back();
      cudaEventRecord(ts->m_idle, M.s);
    }
    cudaStreamWaitEvent(M.s, ev_panel, 0);
    if (ts) cudaEventRecord(ts->m_go, M.s);
    // left swaps of panel k, after the step that read those columns last
    cudaStreamWaitEvent(S, ev_panel, 0);
    if (k > 0) cudaStreamWaitEvent(S, ev_rest, 0);
    const int32_t* plan_k = wk.plans + (size_t)(k / kNb) * kSwapPlanInts;
    swap_apply(Lane{S, nullptr, c->num_sms}, A + k, lda, k, plan_k);
    if (k + kb < n) {
      const int64_t rest = n - k - kb;
      if constexpr (sizeof(T) == 4) {
        // While the trailing update outlasts the panel, the main stream's
        // cuBLAS kernels take every SM; once the panel chain is the longer
        // one (rest below lu_cap_rest()), they leave 48 SMs to it so that a
        // panel (<= 47 CTAs, one per SM) never waits for SMs.
        const int target = rest < lu_cap_rest() ? std::max(1, c->num_sms - kPanelCtas) : 0;
        cublasSetSmCountTarget(M.h, target);
        wk.gemm_ctas = target ? target : c->num_sms;
      }
      const int kn = (int)std::min<int64_t>(kNb, rest);
      // first everything the next panel needs: the next block column's
      // interchanges, U12 and update; the rest of the block row after
      P.begin(M.s);
      swap_apply(M, A + k + lda * (k + kb), lda, kn, plan_k);
      P.end(1);
      block_row_solve(M, wk, kb, 0, kn, Akk, lda, Akk + lda * kb, true);
      P.end(2);
      prepare_l21(M, wk, kb, rest, Akk + kb, lda);
      prepare_u12(M, wk, kb, 0, kn, Akk + lda * kb, lda);
      rc = update_gemm(c, M, wk, kb, rest, 0, kn, Akk + kb, Akk + lda * kb, Akk + kb + lda * kb, lda);
      if (rc) break;
      P.end(3);
      cudaEventRecord(ev_next, M.s);
      if (ts) cudaEventRecord(ts->p_idle, Pn.s);
      cudaStreamWaitEvent(Pn.s, ev_next, 0);
      if (ts) cudaEventRecord(ts->p_go, Pn.s);
      rc = block_panel(c, Pn, wk, Akk + kb + lda * kb, lda, rest, kn, piv + k + kb, k + kb);
      if (!rc) swap_plan(Pn, piv + k + kb, kn, 0, wk.plans + (size_t)((k + kb) / kNb) * kSwapPlanInts);
      if (ts) cudaEventRecord(ts->p_done, Pn.s);
      cudaEventRecord(ev_panel, Pn.s);
      if (rc) break;
      P.begin(M.s);
      swap_apply(M, A + k + lda * (k + kb + kn), lda, rest - kn, plan_k);
      P.end(1);
      block_row_solve(M, wk, kb, kn, rest - kn, Akk, lda, Akk + lda * kb, false);
      P.end(2);
      prepare_u12(M, wk, kb, kn, rest - kn, Akk + lda * kb, lda);
      rc = update_gemm(c, M, wk, kb, rest, kn, rest - kn, Akk + kb, Akk + lda * kb, Akk + kb + lda * (kb + kn), lda);
      if (rc) break;
      P.end(3);
      cudaEventRecord(ev_rest, M.s);
      if (ts) cudaEventRecord(ts->m_done, M.s);
    }
    if (!rc) rc = check_cuda(c, cudaGetLastError(), "LU step launch");
  }
  if (ev_left) {
    cudaEventRecord(ev_left, S);
    cudaStreamWaitEvent(M.s, ev_left, 0);
    cudaEventRecord(ev_panel, Pn.s);
    cudaStreamWaitEvent(M.s, ev_panel, 0);
  }
  if (!rc) {
    ++g_launches;
    globalise_piv_kernel<<<(unsigned)((n + 255) / 256), 256, 0, M.s>>>(piv, n, kNb);
  }
  P.report(sizeof(T) == 8 ? "LU fp64" : "LU fp32");
  int64_t info = 0;
  int ll_err = 0, tc_err = 0;
  if (!rc) {
    rc = check_cuda(c, cudaMemcpyAsync(&info, wk.d_info, sizeof(int64_t), cudaMemcpyDeviceToHost, M.s), "info");
    if (!rc && wk.ll_err)
      rc = check_cuda(c, cudaMemcpyAsync(&ll_err, wk.ll_err, sizeof(int), cudaMemcpyDeviceToHost, M.s), "panel status");
    if (!rc && wk.tc_err)
      rc = check_cuda(c, cudaMemcpyAsync(&tc_err, wk.tc_err, sizeof(int), cudaMemcpyDeviceToHost, M.s), "update status");
    if (!rc) rc = check_cuda(c, cudaStreamSynchronize(M.s), "LU factorisation");
  }
  cudaStreamSynchronize(Pn.s);
  cudaStreamSynchronize(S);
  timeline().report();
  if (!rc && ll_err) rc = set_error(c, HFPX_ERR_CUDA, "panel pivot exchange timed out");
  if (!rc && tc_err)
    rc = set_error(c, HFPX_ERR_CUDA, "tensor-core update: a pipeline wait timed out (code " + std::to_string(tc_err) + ")");
  for (cudaEvent_t e : {ev_panel, ev_next, ev_rest, ev_left, ev_start})
    if (e) cudaEventDestroy(e);
  *info_out = info;
  if (!rc && info != 0) rc = set_error(c, HFPX_ERR_SINGULAR, "matrix is singular: zero pivot at column " + std::to_string(info));
  return rc;
}

static void set_math(hfpx_ctx* c, cublasMath_t mode) {
  cublasSetMathMode(H(c), mode);
  cublasSetMathMode(static_cast<cublasHandle_t>(c->cublas_panel), mode);
}

int lu_factor_fp64(hfpx_ctx* c, hfpx_matrix* m) {
  m->f32_current = 0;
  set_math(c, CUBLAS_DEFAULT_MATH);
  int rc = lu_factor<double>(c, m->d_a, m->ld, m->n, m->d_piv, &m->info);
  m->factored = rc == 0 || rc == HFPX_ERR_SINGULAR ? 1 : 0;
  return rc;
}

int lu_factor_fp32(hfpx_ctx* c, hfpx_matrix* m) {
  if (!m->d_f) {
    if (cudaMalloc(&m->d_f, sizeof(float) * (size_t)m->ld * m->n) != cudaSuccess) {
      m->d_f = nullptr;
      return set_error(c, HFPX_ERR_NOMEM, "FP32 working copy");
    }
  }
  set_math(c, CUBLAS_TF32_TENSOR_OP_MATH);
  // the assembly already wrote the FP32 copy when the matrix had one:
  // nothing to convert; the factors then replace it
  const double* src = m->f32_current ? nullptr : m->d_a;
  m->f32_current = 0;
  int rc = lu_factor<float>(c, m->d_f, m->ld, m->n, m->d_piv, &m->info, src);
  cublasSetSmCountTarget(H(c), 0);
  set_math(c, CUBLAS_DEFAULT_MATH);
  m->factored = rc == 0 || rc == HFPX_ERR_SINGULAR ? 2 : 0;
  m->dinv_valid = 0;
  return rc;
}

// ----------------------------------------------------------------- solves
template <class T>
__global__ void permute_rows_kernel(const T* __restrict__ src, T* __restrict__ dst, const int32_t* __restrict__ perm,
                                    int64_t n, int64_t nrhs, int64_t ld) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n * nrhs) return;
  const int64_t c = i / n, r = i - c * n;
  dst[r + ld * c] = src[perm[r] + ld * c];
}

// out[j] = max_i |a[i + lda j]|, one CTA per column (the refinement's
// per-column infinity norms in one launch and one copy to the host)
__global__ void __launch_bounds__(256) colmax_kernel(const double* __restrict__ a, int64_t n, int64_t lda,
                                                     double* __restrict__ out) {
  __shared__ double red[256];
  const double* col = a + lda * (int64_t)blockIdx.x;
  double m = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += 256) m = fmax(m, fabs(col[i]));
  red[threadIdx.x] = m;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

__global__ void d2f_kernel(const double* __restrict__ a, float* __restrict__ b, int64_t n, int64_t nrhs, int64_t lda,
                           int64_t ldb) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n * nrhs) return;
  const int64_t c = i / n, r = i - c * n;
  b[r + ldb * c] = (float)a[r + lda * c];
}

__global__ void axpy_f2d_kernel(const float* __restrict__ d, double* __restrict__ x, int64_t n, int64_t nrhs,
                                int64_t ldd, int64_t ldx) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n * nrhs) return;
  const int64_t c = i / n, r = i - c * n;
  x[r + ldx * c] += (double)d[r + ldd * c];
}

// Row permutation from the sequential interchanges (host: O(n)).
static int build_perm(hfpx_ctx* c, const hfpx_matrix* m, int32_t** d_perm) {
  std::vector<int32_t> piv(m->n), perm(m->n);
  int rc = check_cuda(c, cudaMemcpyAsync(piv.data(), m->d_piv, sizeof(int32_t) * m->n, cudaMemcpyDeviceToHost, c->stream),
                      "pivots");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "pivots");
  if (rc) return rc;
  for (int64_t i = 0; i < m->n; ++i) perm[i] = (int32_t)i;
  for (int64_t i = 0; i < m->n; ++i) std::swap(perm[i], perm[piv[i]]);
  *d_perm = (int32_t*)ctx_scratch(c, kScrPerm, sizeof(int32_t) * m->n);
  if (!*d_perm) return set_error(c, HFPX_ERR_NOMEM, "perm");
  // the host vector goes out of scope: copy synchronously with the stream
  rc = check_cuda(c, cudaMemcpyAsync(*d_perm, perm.data(), sizeof(int32_t) * m->n, cudaMemcpyHostToDevice, c->stream),
                  "perm");
  return rc ? rc : check_cuda(c, cudaStreamSynchronize(c->stream), "perm");
}

template <class T>
static int solve_factored(hfpx_ctx* c, const hfpx_matrix* m, const T* LU, T* d_b, int64_t nrhs, int64_t ldb,
                          const int32_t* d_perm) {
  const int64_t n = m->n;
  T* tmp = (T*)ctx_scratch(c, kScrSolveTmp, sizeof(T) * (size_t)ldb * nrhs);
  if (!tmp) return set_error(c, HFPX_ERR_NOMEM, "solve tmp");
  const int64_t tot = n * nrhs;
  ++g_launches;
  permute_rows_kernel<T><<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(d_b, tmp, d_perm, n, nrhs, ldb);
  cublasSetMathMode(H(c), CUBLAS_DEFAULT_MATH);
  const T one = 1;
  if constexpr (sizeof(T) == 8) {
    cublasDtrsm(H(c), CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_UNIT, (int)n, (int)nrhs, &one,
                (const double*)LU, (int)m->ld, (double*)tmp, (int)ldb);
    cublasDtrsm(H(c), CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, (int)n, (int)nrhs,
                &one, (const double*)LU, (int)m->ld, (double*)tmp, (int)ldb);
  } else {
    cublasStrsm(H(c), CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_UNIT, (int)n, (int)nrhs, &one,
                (const float*)LU, (int)m->ld, (float*)tmp, (int)ldb);
    cublasStrsm(H(c), CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, (int)n, (int)nrhs,
                &one, (const float*)LU, (int)m->ld, (float*)tmp, (int)ldb);
  }
  return check_cuda(c, cudaMemcpy2DAsync(d_b, ldb * sizeof(T), tmp, ldb * sizeof(T), n * sizeof(T), nrhs,
                                         cudaMemcpyDeviceToDevice, c->stream),
                    "solve copy");
}

int lu_solve_fp64(hfpx_ctx* c, const hfpx_matrix* m, double* d_b, int64_t nrhs, int64_t ldb) {
  int32_t* d_perm = nullptr;
  int rc = build_perm(c, m, &d_perm);
  if (!rc) rc = solve_factored<double>(c, m, m->d_a, d_b, nrhs, ldb, d_perm);
  return rc;
}

int lu_solve_fp32(hfpx_ctx* c, const hfpx_matrix* m, float* d_b, int64_t nrhs, int64_t ldb) {
  int32_t* d_perm = nullptr;
  int rc = build_perm(c, m, &d_perm);
  if (!rc) rc = solve_factored<float>(c, m, m->d_f, d_b, nrhs, ldb, d_perm);
  return rc;
}

// HFPX_SOLVE=cublas keeps the single right-hand side on cuBLAS solves.
static bool own_solve_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("HFPX_SOLVE");
    return !(e && std::string(e) == "cublas");
  }();
  return on;
}

// The single right-hand side uses the engine's tile-sweep triangular solves
// (solve.cu: ~4 ms per triangle at N = 72 000, against ~6 for cuBLAS);
// HFPX_TRSV=cublas selects cuBLAS instead.
static bool own_trsv_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("HFPX_TRSV");
    return !(e && std::string(e) == "cublas");
  }();
  return on;
}

// y = (P L U)^-1 v with the FP32 factors of a mixed factorisation, for one
// FP64 vector v: v -> FP32 (rf), row interchanges (into y), then the two
// triangular solves in place.  The diagonal-block inverses of the tile
// solves are made once per factorisation.
static int precond_f32(hfpx_ctx* c, const hfpx_matrix* m, const int32_t* d_perm, const double* v, float* rf,
                       float* y) {
  const int64_t n = m->n;
  const unsigned nb = (unsigned)((n + 255) / 256);
  ++g_launches;
  d2f_kernel<<<nb, 256, 0, c->stream>>>(v, rf, n, 1, n, n);
  ++g_launches;
  permute_rows_kernel<float><<<nb, 256, 0, c->stream>>>(rf, y, d_perm, n, 1, n);
  if (own_trsv_enabled()) {
    const size_t blk = (size_t)trsv_tiles(n) * 128 * 128;
    if (!m->dinv_valid) {
      if (!m->d_dinv && cudaMalloc(&m->d_dinv, sizeof(float) * 2 * blk) != cudaSuccess) {
        m->d_dinv = nullptr;
        cudaGetLastError();
        return set_error(c, HFPX_ERR_NOMEM, "diagonal block inverses");
      }
      int rc = tri_inverses(c, m->d_f, m->ld, n, m->d_dinv, m->d_dinv + blk);
      if (rc) return rc;
      m->dinv_valid = 1;
    }
    int rc = trsv_f32(c, m->d_f, m->ld, n, m->d_dinv, y, false);
    if (!rc) rc = trsv_f32(c, m->d_f, m->ld, n, m->d_dinv + blk, y, true);
    return rc;
  }
  // cuBLAS strsm with one column measured faster than strsv here
  const float one = 1.f;
  cublasSetMathMode(H(c), CUBLAS_DEFAULT_MATH);
  cublasStrsm(H(c), CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_UNIT, (int)n, 1, &one, m->d_f,
              (int)m->ld, y, (int)n);
  cublasStrsm(H(c), CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, (int)n, 1, &one,
              m->d_f, (int)m->ld, y, (int)n);
  return check_cuda(c, cudaGetLastError(), "triangular solves");
}

// One right-hand side: the engine's residual (solve.cu; |r|_inf comes back
// as one 8-byte copy per step) and triangular solves.
static int refine_one(hfpx_ctx* c, const hfpx_matrix* m, double* d_b, double tol, int max_iter, hfpx_solve_info* info) {
  const int64_t n = m->n;
  double* x = (double*)ctx_scratch(c, kScrRefX, sizeof(double) * n);
  double* r = (double*)ctx_scratch(c, kScrRefR, sizeof(double) * n);
  float* rf = (float*)ctx_scratch(c, kScrRefRf, sizeof(float) * n);
  float* y = (float*)ctx_scratch(c, kScrSolveTmp, sizeof(float) * n);
  double* part = (double*)ctx_scratch(c, kScrResidPart, sizeof(double) * n * resid_chunks(n));
  unsigned long long* dmax = (unsigned long long*)ctx_scratch(c, kScrResidMax, sizeof(unsigned long long));
  if (!x || !r || !rf || !y || !part || !dmax) return set_error(c, HFPX_ERR_NOMEM, "refinement buffers");
  int32_t* d_perm = nullptr;
  int rc = build_perm(c, m, &d_perm);
  if (rc) return rc;
  auto read_max = [&](double* v) {
    unsigned long long bits = 0;
    int e = check_cuda(c, cudaMemcpyAsync(&bits, dmax, sizeof(bits), cudaMemcpyDeviceToHost, c->stream), "max");
    if (!e) e = check_cuda(c, cudaStreamSynchronize(c->stream), "max");
    std::memcpy(v, &bits, sizeof(double));
    return e;
  };
  double bnorm = 0.0, worst = INFINITY;
  rc = absmax_f64(c, d_b, n, dmax);
  if (!rc) rc = read_max(&bnorm);
  if (!(bnorm > 0.0)) bnorm = 1.0;
  const unsigned nb = (unsigned)((n + 255) / 256);
  int it = 0;
  if (!rc) {
    cudaMemsetAsync(x, 0, sizeof(double) * n, c->stream);
    cudaMemcpyAsync(r, d_b, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream);
    for (it = 1; it <= max_iter; ++it) {
      rc = precond_f32(c, m, d_perm, r, rf, y);
      if (rc) break;
      ++g_launches;
      axpy_f2d_kernel<<<nb, 256, 0, c->stream>>>(y, x, n, 1, n, n);
      rc = residual_f64(c, m->d_a, m->ld, n, x, d_b, r, part, dmax);
      double rmax = 0.0;
      if (!rc) rc = read_max(&rmax);
      if (rc) break;
      worst = rmax / bnorm;
      if (prof().on) std::fprintf(stderr, "[hfpx profile] refinement %d: residual %.3e\n", it, worst);
      if (worst <= tol) break;
    }
  }
  if (!rc) rc = trsv_status(c);
  if (!rc) {
    cudaMemcpyAsync(d_b, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream);
    rc = check_cuda(c, cudaStreamSynchronize(c->stream), "refinement");
  }
  if (info) {
    info->iterations = std::min(it, max_iter);
    info->residual = worst;
    info->converged = worst <= tol;
  }
  if (!rc && !(worst <= tol)) rc = set_error(c, HFPX_ERR_NOT_CONVERGED, "refinement did not reach the tolerance");
  return rc;
}

// GMRES(restart) on the FP64 matrix with a right preconditioner M:
// A M u = b, x = M u, in the flexible form (the vectors z_j = M v_j are
// kept, so x += Z y needs no further application of M).  One step is one
// application of M (apply) and one FP64 product with A (the residual kernel
// against a zero right-hand side gives -A z); the Arnoldi vectors are
// orthogonalised by classical Gram-Schmidt applied twice (four cuBLAS
// DGEMVs), the small Hessenberg least-squares problem is solved on the host
// with Givens rotations.  A cycle stops when the rotated residual
// |g_{j+1}| / |b|_2 is below tol / 4; then the residual r = b - A x decides,
// in the max norm like the refinement: |r|_inf / |b|_inf <= tol, else the
// next cycle starts from it.  The products A z_j are kept, so r = b - [A z] y
// costs one small DGEMV instead of another pass over A (the same r as b - A x
// up to rounding far below the tolerance).  d_b: right-hand side in, x out.
constexpr int kGmresMax = 64;

int gmres_core(hfpx_ctx* c, const double* A, int64_t lda, int64_t n, double* d_b, double tol, int restart,
               int max_iter, hfpx_solve_info* info, const std::function<int(const double*, double*)>& apply,
               const float* Af, double relax_below, const hfpx_matrix* mixed_op) {
  if (mixed_op) Af = nullptr;  // the operator is the mixed one: no relaxed products
  const int k = std::max(1, std::min(restart, kGmresMax));
  double* V = (double*)ctx_scratch(c, kScrGmresV, sizeof(double) * n * (k + 1));
  double* Z = (double*)ctx_scratch(c, kScrGmresZ, sizeof(double) * n * 2 * k);  // Z, then A Z
  double* dh = (double*)ctx_scratch(c, kScrGmresH, sizeof(double) * 2 * (kGmresMax + 1));
  double* zero = (double*)ctx_scratch(c, kScrGmresZero, sizeof(double) * n);
  double* x = (double*)ctx_scratch(c, kScrRefX, sizeof(double) * n);
  double* r = (double*)ctx_scratch(c, kScrRefR, sizeof(double) * n);
  double* part = (double*)ctx_scratch(c, kScrResidPart, sizeof(double) * n * resid_chunks(n));
  unsigned long long* dmax = (unsigned long long*)ctx_scratch(c, kScrResidMax, sizeof(unsigned long long));
  double* est = (double*)ctx_scratch(c, kScrGmresEst, sizeof(double) * n);
  if (!V || !Z || !dh || !zero || !x || !r || !part || !dmax || !est)
    return set_error(c, HFPX_ERR_NOMEM, "GMRES buffers");
  double* AZ = Z + (size_t)n * k;
  int rc = 0;
  cublasHandle_t h = H(c);
  cublasSetPointerMode(h, CUBLAS_POINTER_MODE_HOST);
  cublasSetMathMode(h, CUBLAS_DEFAULT_MATH);
  auto sync = [&](const char* what) { return check_cuda(c, cudaStreamSynchronize(c->stream), what); };
  auto read_max = [&](double* v) {
    unsigned long long bits = 0;
    int e = check_cuda(c, cudaMemcpyAsync(&bits, dmax, sizeof(bits), cudaMemcpyDeviceToHost, c->stream), "max");
    if (!e) e = sync("max");
    std::memcpy(v, &bits, sizeof(double));
    return e;
  };
  double bmax = 0.0, bnorm2 = 0.0, worst = INFINITY;
  rc = absmax_f64(c, d_b, n, dmax);
  if (!rc) rc = read_max(&bmax);
  if (!rc) cublasDnrm2(h, (int)n, d_b, 1, &bnorm2);
  if (!(bmax > 0.0)) bmax = 1.0;
  if (!(bnorm2 > 0.0)) bnorm2 = 1.0;
  cudaMemsetAsync(zero, 0, sizeof(double) * n, c->stream);
  cudaMemsetAsync(x, 0, sizeof(double) * n, c->stream);
  cudaMemcpyAsync(r, d_b, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream);
  double Hm[kGmresMax + 1][kGmresMax];  // Hessenberg columns, rotated in place
  double cs[kGmresMax], sn[kGmresMax], g[kGmresMax + 1], hv[kGmresMax + 1], h2[kGmresMax + 1];
  int steps = 0;
  double rnorm = bnorm2;  // |r|_2 of the cycle's start
  while (!rc && steps < max_iter) {
    // v_0 = r / |r|_2
    if (steps > 0) {
      cublasDnrm2(h, (int)n, r, 1, &rnorm);
      rc = sync("GMRES restart");
      if (rc || !(rnorm > 0.0)) break;
    }
    cudaMemcpyAsync(V, r, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream);
    const double inv0 = 1.0 / rnorm;
    cublasDscal(h, (int)n, &inv0, V, 1);
    for (int i = 0; i <= k; ++i) g[i] = 0.0;
    g[0] = rnorm;
    int j = 0;
    bool cycle_relaxed = false;
    for (; j < k && steps < max_iter; ++j, ++steps) {
      double* vj = V + (size_t)n * j;
      double* zj = Z + (size_t)n * j;
      double* w = V + (size_t)n * (j + 1);
      // z_j = M v_j (the preconditioner), w = A z_j: once the residual is
      // small the product may be inexact by about tol / |r| (relaxed
      // Krylov), so below relax_below it reads the FP32 copy of A
      rc = apply(vj, zj);
      if (rc) break;
      const bool relaxed = Af && std::fabs(g[j]) / bnorm2 <= relax_below;
      cycle_relaxed = cycle_relaxed || relaxed;
      rc = relaxed    ? residual_f32m(c, Af, lda, n, zj, zero, w, part, dmax)   // w = -A z_j
           : mixed_op ? residual_mixed(c, mixed_op, zj, zero, w, part, dmax)
                      : residual_f64(c, A, lda, n, zj, zero, w, part, dmax);
      if (rc) break;
      const double mone = -1.0, one = 1.0, zero_s = 0.0;
      cublasDscal(h, (int)n, &mone, w, 1);
      cudaMemcpyAsync(AZ + (size_t)n * j, w, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream);
      // h = V^T w; w -= V h; twice
      cublasDgemv(h, CUBLAS_OP_T, (int)n, j + 1, &one, V, (int)n, w, 1, &zero_s, dh, 1);
      cublasDgemv(h, CUBLAS_OP_N, (int)n, j + 1, &mone, V, (int)n, dh, 1, &one, w, 1);
      cublasDgemv(h, CUBLAS_OP_T, (int)n, j + 1, &one, V, (int)n, w, 1, &zero_s, dh + kGmresMax + 1, 1);
      cublasDgemv(h, CUBLAS_OP_N, (int)n, j + 1, &mone, V, (int)n, dh + kGmresMax + 1, 1, &one, w, 1);
      double beta = 0.0;
      cublasDnrm2(h, (int)n, w, 1, &beta);  // synchronises (host pointer mode)
      rc = check_cuda(c, cudaMemcpyAsync(hv, dh, sizeof(double) * (j + 1), cudaMemcpyDeviceToHost, c->stream), "h");
      if (!rc)
        rc = check_cuda(c, cudaMemcpyAsync(h2, dh + kGmresMax + 1, sizeof(double) * (j + 1), cudaMemcpyDeviceToHost,
                                           c->stream),
                        "h");
      if (!rc) rc = sync("GMRES step");
      if (rc) break;
      for (int i = 0; i <= j; ++i) Hm[i][j] = hv[i] + h2[i];
      Hm[j + 1][j] = beta;
      if (beta > 0.0) {
        const double ib = 1.0 / beta;
        cublasDscal(h, (int)n, &ib, w, 1);
      }
      // earlier rotations, then the one that zeroes H(j+1, j)
      for (int i = 0; i < j; ++i) {
        const double a = Hm[i][j], bb = Hm[i + 1][j];
        Hm[i][j] = cs[i] * a + sn[i] * bb;
        Hm[i + 1][j] = -sn[i] * a + cs[i] * bb;
      }
      const double a = Hm[j][j], bb = Hm[j + 1][j];
      const double den = std::hypot(a, bb);
      cs[j] = den > 0.0 ? a / den : 1.0;
      sn[j] = den > 0.0 ? bb / den : 0.0;
      Hm[j][j] = den;
      Hm[j + 1][j] = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      if (prof().on)
        std::fprintf(stderr, "[hfpx profile] GMRES step %d: |g| / |b|_2 %.3e\n", steps + 1, std::fabs(g[j + 1]) / bnorm2);
      if (!(beta > 0.0)) {
        ++j;
        ++steps;
        break;
      }
      // The stopping rule is on the max norm, |r|_inf <= tol |b|_inf, and
      // |g| is the 2-norm of the residual: a residual concentrated at the
      // crack tip, against an even b, has |r|_inf / |b|_inf well above
      // |r|_2 / |b|_2.  Once |g| <= sqrt(n) tol |b|_inf the max norm may
      // already be below tol, so from there each step forms the residual the
      // cycle's products give, r_0 - [A z] y (a pass over n x (j + 1)
      // stored products, no product with A), and stops on its max norm.
      if (std::fabs(g[j + 1]) <= std::sqrt((double)n) * tol * bmax) {
        double yv[kGmresMax];
        for (int i = j; i >= 0; --i) {
          double t = g[i];
          for (int l = i + 1; l <= j; ++l) t -= Hm[i][l] * yv[l];
          yv[i] = Hm[i][i] != 0.0 ? t / Hm[i][i] : 0.0;
        }
        rc = check_cuda(c, cudaMemcpyAsync(dh, yv, sizeof(double) * (j + 1), cudaMemcpyHostToDevice, c->stream), "y");
        if (!rc) rc = check_cuda(c, cudaMemcpyAsync(est, r, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream),
                                 "estimate");
        if (rc) break;
        const double mone_e = -1.0, one_e = 1.0;
        cublasDgemv(h, CUBLAS_OP_N, (int)n, j + 1, &mone_e, AZ, (int)n, dh, 1, &one_e, est, 1);
        double emax = 0.0;
        rc = absmax_f64(c, est, n, dmax);
        if (!rc) rc = read_max(&emax);
        if (rc) break;
        if (prof().on)
          std::fprintf(stderr, "[hfpx profile] GMRES step %d: estimated |r|_inf / |b|_inf %.3e\n", steps + 1,
                       emax / bmax);
        if (emax <= 0.5 * tol * bmax) {
          ++j;
          ++steps;
          break;
        }
      }
    }
    if (rc || j == 0) break;
    // y = R^-1 g (back substitution), x += Z y
    double yv[kGmresMax];
    for (int i = j - 1; i >= 0; --i) {
      double t = g[i];
      for (int l = i + 1; l < j; ++l) t -= Hm[i][l] * yv[l];
      yv[i] = Hm[i][i] != 0.0 ? t / Hm[i][i] : 0.0;
    }
    rc = check_cuda(c, cudaMemcpyAsync(dh, yv, sizeof(double) * j, cudaMemcpyHostToDevice, c->stream), "y");
    if (rc) break;
    const double one = 1.0, mone = -1.0;
    cublasDgemv(h, CUBLAS_OP_N, (int)n, j, &one, Z, (int)n, dh, 1, &one, x, 1);
    if (cycle_relaxed) {
      // products from the FP32 copy: the cycle's residual is b - A x in FP64
      rc = residual_f64(c, A, lda, n, x, d_b, r, part, dmax);
    } else {
      // r = r_0 - [A z] y (r holds the cycle's starting residual)
      cublasDgemv(h, CUBLAS_OP_N, (int)n, j, &mone, AZ, (int)n, dh, 1, &one, r, 1);
      rc = absmax_f64(c, r, n, dmax);
    }
    double rmax = 0.0;
    if (!rc) rc = read_max(&rmax);
    if (rc) break;
    worst = rmax / bmax;
    if (prof().on) std::fprintf(stderr, "[hfpx profile] GMRES cycle end: residual %.3e\n", worst);
    if (worst <= tol) break;
  }
  if (!rc) rc = check_cuda(c, cudaGetLastError(), "GMRES");
  if (!rc) {
    cudaMemcpyAsync(d_b, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream);
    rc = sync("GMRES");
  }
  if (info) {
    info->iterations = steps;
    info->residual = worst;
    info->converged = worst <= tol;
  }
  if (!rc && !(worst <= tol)) rc = set_error(c, HFPX_ERR_NOT_CONVERGED, "GMRES did not reach the tolerance");
  return rc;
}


// The mixed-LU preconditioned form: M = (P L U)^-1 of the FP32 factors,
// applied in FP32 and widened to FP64.
int gmres_solve(hfpx_ctx* c, const hfpx_matrix* m, double* d_b, double tol, int restart, int max_iter,
                hfpx_solve_info* info) {
  const int64_t n = m->n;
  float* rf = (float*)ctx_scratch(c, kScrRefRf, sizeof(float) * n);
  float* y = (float*)ctx_scratch(c, kScrSolveTmp, sizeof(float) * n);
  if (!rf || !y) return set_error(c, HFPX_ERR_NOMEM, "GMRES buffers");
  int32_t* d_perm = nullptr;
  int rc = build_perm(c, m, &d_perm);
  if (rc) return rc;
  const unsigned nb = (unsigned)((n + 255) / 256);
  auto apply = [&](const double* v, double* z) {
    int e = precond_f32(c, m, d_perm, v, rf, y);
    if (e) return e;
    cudaMemsetAsync(z, 0, sizeof(double) * n, c->stream);
    ++g_launches;
    axpy_f2d_kernel<<<nb, 256, 0, c->stream>>>(y, z, n, 1, n, n);
    return 0;
  };
  rc = gmres_core(c, m->d_a, m->ld, n, d_b, tol, restart, max_iter, info, apply);
  if (!rc) rc = trsv_status(c);
  return rc;
}

int refine_solve(hfpx_ctx* c, const hfpx_matrix* m, double* d_b, int64_t nrhs, int64_t ldb, double tol, int max_iter,
                 hfpx_solve_info* info) {
  if (nrhs == 1 && own_solve_enabled()) return refine_one(c, m, d_b, tol, max_iter, info);
  const int64_t n = m->n;
  double* x = (double*)ctx_scratch(c, kScrRefX, sizeof(double) * ldb * nrhs);
  double* r = (double*)ctx_scratch(c, kScrRefR, sizeof(double) * ldb * nrhs);
  float* rf = (float*)ctx_scratch(c, kScrRefRf, sizeof(float) * ldb * nrhs);
  double* cmax = (double*)ctx_scratch(c, kScrRefColMax, sizeof(double) * nrhs);
  int32_t* d_perm = nullptr;
  int rc = 0;
  if (!x || !r || !rf || !cmax) rc = set_error(c, HFPX_ERR_NOMEM, "refinement buffers");
  if (!rc) rc = build_perm(c, m, &d_perm);
  std::vector<double> bnorm(nrhs, 0.0), rnorm(nrhs, 0.0);
  const int64_t tot = n * nrhs;
  const unsigned nb = (unsigned)((tot + 255) / 256);
  int it = 0;
  double worst = INFINITY;
  if (!rc) {
    cudaMemsetAsync(x, 0, sizeof(double) * ldb * nrhs, c->stream);
    cudaMemcpyAsync(r, d_b, sizeof(double) * ldb * nrhs, cudaMemcpyDeviceToDevice, c->stream);
    // per-column infinity norms: one launch, one copy
    auto colmax = [&](const double* a, std::vector<double>& out) -> int {
      ++g_launches;
      colmax_kernel<<<(unsigned)nrhs, 256, 0, c->stream>>>(a, n, ldb, cmax);
      int e = check_cuda(c, cudaMemcpyAsync(out.data(), cmax, sizeof(double) * nrhs, cudaMemcpyDeviceToHost,
                                            c->stream), "column norms");
      if (!e) e = check_cuda(c, cudaStreamSynchronize(c->stream), "column norms");
      return e;
    };
    rc = colmax(d_b, bnorm);
    for (double& v : bnorm) v = v > 0 ? v : 1.0;
    for (it = 1; !rc && it <= max_iter; ++it) {
      ++g_launches;
      d2f_kernel<<<nb, 256, 0, c->stream>>>(r, rf, n, nrhs, ldb, ldb);
      rc = solve_factored<float>(c, m, m->d_f, rf, nrhs, ldb, d_perm);
      if (rc) break;
      ++g_launches;
      axpy_f2d_kernel<<<nb, 256, 0, c->stream>>>(rf, x, n, nrhs, ldb, ldb);
      cudaMemcpyAsync(r, d_b, sizeof(double) * ldb * nrhs, cudaMemcpyDeviceToDevice, c->stream);
      const double mone = -1.0, one = 1.0;
      cublasDgemm(H(c), CUBLAS_OP_N, CUBLAS_OP_N, (int)n, (int)nrhs, (int)n, &mone, m->d_a, (int)m->ld, x, (int)ldb,
                  &one, r, (int)ldb);
      worst = 0.0;
      if ((rc = colmax(r, rnorm))) break;
      for (int64_t j = 0; j < nrhs; ++j) worst = std::max(worst, rnorm[j] / bnorm[j]);
      if (worst <= tol) break;
    }
    if (!rc) cudaMemcpyAsync(d_b, x, sizeof(double) * ldb * nrhs, cudaMemcpyDeviceToDevice, c->stream);
    if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "refinement");
  }
  if (info) {
    info->iterations = std::min(it, max_iter);
    info->residual = worst;
    info->converged = worst <= tol;
  }
  if (!rc && !(worst <= tol)) rc = set_error(c, HFPX_ERR_NOT_CONVERGED, "refinement did not reach the tolerance");
  return rc;
}

// ------------------------------------------------- allocation-free panel LU
// For callers that cannot allocate device memory: hosts that hand all of the
// device's memory to an arena or pool of their own at start-up (a cudaMalloc
// then fails, or takes memory the arena counts on), and real-time or embedded
// loops that forbid allocation after start-up (cudaMalloc and cudaFree can
// synchronise the device and take unbounded time).  The pivot-search scratch
// of the panel kernel lives in this file-scope array instead of in
// cudaMalloc'd buffers.  Every GPU that loads the library holds it until the
// process exits; all calls share it, so calls that overlap on the GPU (other
// streams, other host threads) race and must be serialised by the caller.
constexpr int kNoAllocMaxCtas = 256;
constexpr size_t kNoAllocCand = sizeof(double) * 2 * kNoAllocMaxCtas * kBaseW;
constexpr size_t kNoAllocCmax = sizeof(double) * 2 * kNoAllocMaxCtas;
constexpr size_t kNoAllocCidx = sizeof(int) * 2 * kNoAllocMaxCtas;
constexpr size_t kNoAllocRowj = sizeof(double) * 2 * kBaseW;
constexpr size_t kNoAllocBytes = kNoAllocCand + kNoAllocCmax + kNoAllocCidx + kNoAllocRowj + sizeof(int64_t);
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of the array, looked up by the first call on each device
// with that device current (the caller has made it current).  In host code the
// symbol's name is a host-side stand-in, not a device address, so only the
// looked-up pointer is passed to kernels.  The lookup runs under a lock, so
// first calls from several host threads do not race on the cache.
static unsigned char* noalloc_scratch(hfpx_ctx* c) {
  constexpr int kMaxDevices = 64;
  static std::atomic<unsigned char*> addr[kMaxDevices];
  static std::mutex lock;
  if (c->device < 0 || c->device >= kMaxDevices) return nullptr;
  if (unsigned char* p = addr[c->device].load(std::memory_order_acquire)) return p;
  std::lock_guard<std::mutex> g(lock);
  if (unsigned char* p = addr[c->device].load(std::memory_order_relaxed)) return p;
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) return nullptr;
  if (cudaFuncSetAttribute(panel_base_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) !=
      cudaSuccess)
    return nullptr;
  addr[c->device].store(static_cast<unsigned char*>(p), std::memory_order_release);
  return static_cast<unsigned char*>(p);
}

int lu_panel_factor_noalloc(hfpx_ctx* c, double* d_a, int64_t lda, int64_t m, int w, int32_t* d_piv,
                            int64_t* info) {
  if (!d_a || !d_piv || !info) return set_error(c, HFPX_ERR_ARG, "null argument");
  if (w < 1 || w > kBaseW) return set_error(c, HFPX_ERR_ARG, "panel width must be 1..32 columns");
  if (m < w || lda < m) return set_error(c, HFPX_ERR_ARG, "need m >= w and lda >= m");
  const int G = (int)std::min<int64_t>(std::min<int64_t>(c->num_sms, kNoAllocMaxCtas), std::max<int64_t>(1, (m + 31) / 32));
  const int rpc = (int)((m + G - 1) / G);
  const size_t smem = (size_t)w * rpc * sizeof(double) + kBaseW * sizeof(double);
  if (smem > 200 * 1024)
    return set_error(c, HFPX_ERR_ARG, "panel too tall: at most " + std::to_string((long long)G * (200 * 1024 / 8 - kBaseW) / w) +
                                          " rows for this width on this GPU");
  unsigned char* base = noalloc_scratch(c);
  if (!base) return set_error(c, HFPX_ERR_CUDA, "cannot resolve the device address of the scratch array");
  PanelScratch<double> sc;
  sc.cand = reinterpret_cast<double*>(base);
  sc.cmax = reinterpret_cast<double*>(base + kNoAllocCand);
  sc.cidx = reinterpret_cast<int*>(base + kNoAllocCand + kNoAllocCmax);
  sc.rowj = reinterpret_cast<double*>(base + kNoAllocCand + kNoAllocCmax + kNoAllocCidx);
  int64_t* d_info = reinterpret_cast<int64_t*>(base + kNoAllocCand + kNoAllocCmax + kNoAllocCidx + kNoAllocRowj);
  // the array keeps the previous call's contents: the zero-pivot word starts at 0
  int rc = check_cuda(c, cudaMemsetAsync(d_info, 0, sizeof(int64_t), c->stream), "clear info");
  int64_t col_offset = 0;
  void* args[] = {&d_a, &lda, &m, &w, const_cast<int*>(&rpc), &d_piv, &sc, &d_info, &col_offset};
  if (!rc) {
    ++g_launches;
    rc = check_cuda(c, cudaLaunchCooperativeKernel((void*)panel_base_kernel<double>, dim3(G), dim3(kPanelThreads), args,
                                                   smem, c->stream),
                    "panel launch");
  }
  // Inside a stream capture the call records the clear and the kernel only:
  // a host read (or a synchronisation) would end the capture with an error.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (!rc) rc = check_cuda(c, cudaStreamIsCapturing(c->stream, &cap), "capture status");
  if (!rc && cap != cudaStreamCaptureStatusNone) {
    *info = 0;
    return HFPX_OK;
  }
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(info, d_info, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream), "info");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "panel factorisation");
  if (!rc && *info != 0) rc = set_error(c, HFPX_ERR_SINGULAR, "zero pivot at column " + std::to_string(*info));
  return rc;
}

}  // namespace hfpx
