// Trailing update of the mixed LU on the 5th-generation tensor cores:
//
//     C (m x n, FP32, column-major, ldc)  +=  alpha * A B^T
//     A: m x k FP16, K-major (row i at A + i * lda_k),
//     B: n x k FP16, K-major (column j of the k x n factor at B + j * ldb_k),
//     alpha read from device memory (the power-of-two scale of the FP16 copy
//     of U12, with its sign).
//
// This is the O(N^3) contraction of the factorisation: LAPACK dgetrf's
// trailing update A22 -= L21 U12, the step il::LU reaches through
// LAPACKE_dgetrf (il/linear_algebra/dense/factorization/LU.h:87).
//
// Design (one CTA per SM, persistent over 128 x 256 output tiles):
//   * warp 0, one lane: TMA producer.  Each k-block of 64 brings a 128 x 64
//     tile of A and a 256 x 64 tile of B into shared memory with
//     cp.async.bulk.tensor (128-byte swizzle, plain loads of this GPU's own
//     memory), four stages on full/empty mbarriers;
//   * warp 1: allocates 512 TMEM columns (two 128 x 256 FP32 accumulators);
//     one lane issues tcgen05.mma kind::f16 (M 128, N 256, K 16; four per
//     k-block) and tcgen05.commit to release stages and publish finished
//     accumulators;
//   * warps 2..9: epilogue.  Warp w reads TMEM lanes 32 (w % 4) .. + 31 (one
//     output row per thread) and half of the 256 columns with tcgen05.ld, and
//     applies C += alpha s_i acc with coalesced 128-byte column segments (s_i
//     an optional per-row scale: the LU keeps each row of L21 scaled into the
//     normal FP16 range and undoes it here).  The second accumulator lets the
//     next tile's MMAs run during the epilogue.
// Every wait is bounded (%globaltimer); a wait that runs out sets the
// failure word and an abort flag, every role leaves its loop, outstanding
// copies and MMAs are waited for (bounded), TMEM is freed and the kernel
// returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include "engine_internal.h"

namespace hfpx {
namespace {

constexpr int kBM = 128, kBN = 256, kBK = 64, kStages = 4;
constexpr int kEpiWarps = 8;
constexpr int kThreads = 64 + 32 * kEpiWarps;
constexpr uint32_t kStageA = kBM * kBK * 2;   // 16 KB
constexpr uint32_t kStageB = kBN * kBK * 2;   // 32 KB
constexpr uint32_t kTmemCols = 2 * kBN;       // two accumulators
constexpr int kGroupM = 16;                   // tile raster: row blocks per group (default)
constexpr unsigned long long kWaitNs = 1000000000ull;  // 1 s per wait

struct alignas(1024) TcSmem {
  uint8_t a[kStages][kStageA];
  uint8_t b[kStages][kStageB];
  uint64_t full[kStages], empty[kStages], tfull[2], tempty[2], drain;
  uint32_t tmem_base;
  int abort;
};
constexpr size_t kSmemBytes = sizeof(TcSmem) + 1024;  // + alignment slack of the dynamic base

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for the phase of `parity` to complete, at most kWaitNs; on time-out
// (or when another role has aborted) set the abort flag and the failure
// word and return false.
__device__ __forceinline__ bool wait_phase(uint64_t* b, uint32_t parity, volatile int* abort, int* err, int code) {
  if (mbar_try_wait(b, parity)) return true;
  const unsigned long long t0 = now_ns();
  for (uint32_t it = 1;; ++it) {
    if (mbar_try_wait(b, parity)) return true;
    if ((it & 63) == 0) {
      if (*abort) return false;
      if (now_ns() - t0 > kWaitNs) {
        *abort = 1;
        atomicExch(err, code);
        return false;
      }
    }
  }
}
// after an abort: wait for a phase that an operation already in flight (a
// copy or an MMA) will complete, bounded, without looking at the flag
__device__ __forceinline__ void drain_phase(uint64_t* b, uint32_t parity) {
  const unsigned long long t0 = now_ns();
  while (!mbar_try_wait(b, parity))
    if (now_ns() - t0 > kWaitNs) return;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// the tile's block of C into L2 ahead of its epilogue (no shared memory, no
// completion to wait for)
__device__ __forceinline__ void tma_prefetch_2d(const CUtensorMap* map, int x, int y) {
  asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];" ::"l"(reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y)
               : "memory");
}

// K-major operand tile in shared memory with the 128-byte swizzle: rows of
// 64 FP16 (128 bytes), 8-row atoms of 1024 bytes one after another (stride
// byte offset 1024), leading byte offset unused for swizzled K-major (1),
// descriptor version 1, layout 2 = 128-byte swizzle.  Advancing K by 16
// elements inside the atom adds 32 bytes to the start address.
__device__ __forceinline__ uint64_t smem_desc(const void* tile, int k16) {
  const uint32_t addr = smem_u32(tile) + 32u * (uint32_t)k16;
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;                 // leading byte offset (16 B units)
  d |= (uint64_t)(1024u >> 4) << 32;       // stride byte offset
  d |= (uint64_t)1u << 46;                 // version (sm_100)
  d |= (uint64_t)2u << 61;                 // 128-byte swizzle
  return d;
}
// kind::f16 instruction descriptor: D FP32 (bits 4-5 = 1), A and B FP16
// (bits 7-9, 10-12 = 0), both K-major (bits 15, 16 = 0), N >> 3 at bit 17,
// M >> 4 at bit 24.
constexpr uint32_t kIdesc = (1u << 4) | ((uint32_t)(kBN >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem_d), "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

// Output tiles in groups of `group` row blocks: inside a group the row block
// changes fastest, so the CTAs working at one time share B tiles (and A tiles
// across neighbouring groups) in L2.
struct TileMap {
  int64_t tiles_m, tiles_n;
  int group;
  __device__ void coords(int64_t t, int64_t& mb, int64_t& nb) const {
    const int64_t per_group = (int64_t)group * tiles_n;
    const int64_t g = t / per_group, r = t - g * per_group;
    const int64_t gm = min((int64_t)group, tiles_m - g * group);
    mb = g * group + r % gm;
    nb = r / gm;
  }
};

__global__ void __launch_bounds__(kThreads, 1)
    update_tc_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                     const __grid_constant__ CUtensorMap map_c, int prefetch_c, float* __restrict__ C, int64_t ldc,
                     int64_t m, int64_t n, int k, int group, const float* __restrict__ d_alpha,
                     const float* __restrict__ row_scale, int* __restrict__ err) {
  extern __shared__ uint8_t smem_raw[];
  TcSmem& s = *reinterpret_cast<TcSmem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const TileMap tm{(m + kBM - 1) / kBM, (n + kBN - 1) / kBN, group};
  const int64_t tiles = tm.tiles_m * tm.tiles_n;
  const int nk = (k + kBK - 1) / kBK;
  volatile int* abort = &s.abort;

  if (threadIdx.x == 0) {
    for (int i = 0; i < kStages; ++i) {
      mbar_init(&s.full[i], 1);
      mbar_init(&s.empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&s.tfull[i], 1);
      mbar_init(&s.tempty[i], kEpiWarps);
    }
    mbar_init(&s.drain, 1);
    s.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_a)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_b)) : "memory");
    if (prefetch_c) asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_c)) : "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s.tmem_base;

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      uint32_t armed = 0, armed_par = 0;  // stages with a copy in flight, and its phase
      for (int64_t t = blockIdx.x; t < tiles && !*abort; t += gridDim.x) {
        int64_t mb, nb;
        tm.coords(t, mb, nb);
        if (prefetch_c) tma_prefetch_2d(&map_c, (int)(mb * kBM), (int)(nb * kBN));
        for (int kb = 0; kb < nk; ++kb) {
          if (!wait_phase(&s.empty[stage], phase ^ 1u, abort, err, 0x101)) break;
          armed &= ~(1u << stage);
          mbar_expect_tx(&s.full[stage], kStageA + kStageB);
          tma_load_2d(s.a[stage], &map_a, &s.full[stage], kb * kBK, (int)(mb * kBM));
          tma_load_2d(s.b[stage], &map_b, &s.full[stage], kb * kBK, (int)(nb * kBN));
          armed |= 1u << stage;
          armed_par = (armed_par & ~(1u << stage)) | (phase << stage);
          if (++stage == kStages) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      if (*abort)  // copies still in flight must land before the CTA exits
        for (int i = 0; i < kStages; ++i)
          if (armed & (1u << i)) drain_phase(&s.full[i], (armed_par >> i) & 1u);
    }
    __syncwarp();
  } else if (warp == 1) {
    // ----------------------------------------------------------------- MMA
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      int it = 0;
      bool issued = false;
      for (int64_t t = blockIdx.x; t < tiles && !*abort; t += gridDim.x, ++it) {
        const int acc = it & 1;
        const uint32_t acc_phase = (uint32_t)(it >> 1) & 1u;
        if (!wait_phase(&s.tempty[acc], acc_phase ^ 1u, abort, err, 0x102)) break;
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(acc * kBN);
        bool ok = true;
        for (int kb = 0; kb < nk; ++kb) {
          if (!wait_phase(&s.full[stage], phase, abort, err, 0x103)) {
            ok = false;
            break;
          }
          tc_fence_after();
#pragma unroll
          for (int k16 = 0; k16 < kBK / 16; ++k16)
            mma_f16(d, smem_desc(s.a[stage], k16), smem_desc(s.b[stage], k16), (kb | k16) != 0);
          issued = true;
          mma_commit(&s.empty[stage]);
          if (++stage == kStages) {
            stage = 0;
            phase ^= 1u;
          }
        }
        if (!ok) break;
        mma_commit(&s.tfull[acc]);
      }
      if (*abort && issued) {  // MMAs still in flight must finish before TMEM is freed
        mma_commit(&s.drain);
        drain_phase(&s.drain, 0);
      }
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------------ epilogue
    const int q = warp & 3;                 // TMEM lane quarter this warp may read
    const int half = (warp - 2) >> 2;       // columns [128 half, 128 half + 128)
    const float alpha = *d_alpha;
    int it = 0;
    for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x, ++it) {
      const int acc = it & 1;
      const uint32_t acc_phase = (uint32_t)(it >> 1) & 1u;
      bool ok = wait_phase(&s.tfull[acc], acc_phase, abort, err, 0x104);
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) break;
      tc_fence_after();
      int64_t mb, nb;
      tm.coords(t, mb, nb);
      const int64_t row = mb * kBM + q * 32 + lane;
      const bool row_ok = row < m;
      const float ra = row_ok && row_scale ? alpha * row_scale[row] : alpha;
      const int64_t col0 = nb * kBN + half * 128;
#pragma unroll 1
      for (int ch = 0; ch < 4; ++ch) {
        float v[32];
        tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * kBN + half * 128 + ch * 32), v);
        const int64_t cb = col0 + ch * 32;
        // columns of this chunk inside the matrix (0 for rows below it)
        const int ncol = row_ok ? (int)min((int64_t)32, max((int64_t)0, n - cb)) : 0;
        float* p = C + row + ldc * cb;
        // two groups of 16 column segments in flight
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          float c[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) c[j] = 16 * h + j < ncol ? __ldcg(p + ldc * (16 * h + j)) : 0.f;
#pragma unroll
          for (int j = 0; j < 16; ++j)
            if (16 * h + j < ncol) __stcg(p + ldc * (16 * h + j), fmaf(ra, v[16 * h + j], c[j]));
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&s.tempty[acc]);
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// ------------------------------------------------------- 2-SM variant
// A cluster of two CTAs on two SMs computes one 256 x 256 output tile with
// tcgen05.mma.cta_group::2 (M 256, N 256, K 16).  CTA r of the pair (r =
// %cluster_ctarank) holds rows [128 r, 128 r + 128) of the tile's A rows and
// of its B rows (output columns) in its own shared memory at the same
// offsets; the leader (r = 0) issues the MMAs, and each CTA's TMEM receives
// its 128 output rows x all 256 columns.  Per k-block each SM loads 32 KB
// instead of the 1-SM kernel's 48 KB for the same 128 x 256 x 64 of MMA
// work: the operand traffic from L2 into shared memory, which bounds the
// 1-SM kernel, drops by a third.
//   * both CTAs' producers wait on their own `empty` barrier and load their
//     halves with plain (non-multicast) TMA loads that complete on the
//     leader's `full` barrier; the leader arms it for both halves;
//   * the leader's MMA thread commits each stage to both CTAs' `empty`
//     barriers and each finished accumulator to both CTAs' `tfull`;
//   * both CTAs' epilogue warps arrive on the leader's `tempty` (the peer's
//     remotely), so the leader reuses an accumulator only when both halves
//     are read;
//   * a cluster barrier after the set-up (barriers initialised, TMEM
//     allocated in both CTAs) and before the teardown.
constexpr int kStages2 = 6;
constexpr uint32_t kHalf = 128 * kBK * 2;  // 16 KB: 128 rows x 64 FP16
struct alignas(1024) TcSmem2 {
  uint8_t a[kStages2][kHalf];
  uint8_t b[kStages2][kHalf];
  uint64_t full[kStages2], empty[kStages2], tfull[2], tempty[2], drain;
  uint32_t tmem_base;
  int abort;
};
constexpr size_t kSmemBytes2 = sizeof(TcSmem2) + 1024;
// kind::f16, D FP32, A and B FP16 K-major, N 256, M 256 (the pair)
constexpr uint32_t kIdesc2 = (1u << 4) | ((uint32_t)(256 >> 3) << 17) | ((uint32_t)(256 >> 4) << 24);

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// shared::cluster address of the same variable in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t cluster_addr(const void* p, uint32_t rank) {
  uint32_t a;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_u32(p)), "r"(rank));
  return a;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// TMA load into this CTA's shared memory completing on a barrier of the pair
// (the leader's), given as a shared::cluster address
__device__ __forceinline__ void tma_load_2d_pair(void* dst, const CUtensorMap* map, uint32_t bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], "
      "[%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
      : "memory");
}
__device__ __forceinline__ void mma_f16_pair(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem_d), "l"(da), "l"(db), "r"(kIdesc2), "r"(accumulate)
      : "memory");
}
// arrive on the barrier at this offset in both CTAs of the pair when the
// MMAs issued so far have completed
__device__ __forceinline__ void mma_commit_pair(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
          smem_u32(bar)),
      "h"((uint16_t)3)
      : "memory");
}
__device__ __forceinline__ void mma_commit_pair_local(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];" ::"r"(bar) : "memory");
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreads, 1)
    update_tc2_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                      const __grid_constant__ CUtensorMap map_c, int prefetch_c, float* __restrict__ C, int64_t ldc,
                      int64_t m, int64_t n, int k, int group, const float* __restrict__ d_alpha,
                      const float* __restrict__ row_scale, int* __restrict__ err) {
  extern __shared__ uint8_t smem_raw[];
  TcSmem2& s = *reinterpret_cast<TcSmem2*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();
  const bool leader = rank == 0;
  const int64_t pair = blockIdx.x >> 1, pairs = gridDim.x >> 1;
  const TileMap tm{(m + 255) / 256, (n + 255) / 256, group};
  const int64_t tiles = tm.tiles_m * tm.tiles_n;
  const int nk = (k + kBK - 1) / kBK;
  volatile int* abort = &s.abort;

  if (threadIdx.x == 0) {
    for (int i = 0; i < kStages2; ++i) {
      mbar_init(&s.full[i], 1);
      mbar_init(&s.empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&s.tfull[i], 1);
      mbar_init(&s.tempty[i], 2 * kEpiWarps);
    }
    mbar_init(&s.drain, 1);
    s.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_a)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_b)) : "memory");
    if (prefetch_c) asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_c)) : "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  cluster_sync_all();
  tc_fence_after();
  const uint32_t tmem = s.tmem_base;

  if (warp == 0) {
    // ------------------------------------------------------ producers (both)
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      uint32_t armed = 0, armed_par = 0;  // leader: stages armed for both halves, and their phase
      for (int64_t t = pair; t < tiles && !*abort; t += pairs) {
        int64_t mb, nb;
        tm.coords(t, mb, nb);
        const int row0 = (int)(mb * 256 + 128 * rank), col0 = (int)(nb * 256 + 128 * rank);
        if (prefetch_c) tma_prefetch_2d(&map_c, row0, (int)(nb * 256));
        for (int kb = 0; kb < nk; ++kb) {
          if (!wait_phase(&s.empty[stage], phase ^ 1u, abort, err, 0x201)) break;
          if (leader) {
            armed &= ~(1u << stage);
            mbar_expect_tx(&s.full[stage], 4 * kHalf);  // A and B halves of both CTAs
            armed |= 1u << stage;
            armed_par = (armed_par & ~(1u << stage)) | (phase << stage);
          }
          const uint32_t fb = cluster_addr(&s.full[stage], 0);
          tma_load_2d_pair(s.a[stage], &map_a, fb, kb * kBK, row0);
          tma_load_2d_pair(s.b[stage], &map_b, fb, kb * kBK, col0);
          if (++stage == kStages2) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      if (*abort && leader)  // copies of both halves land on the leader's barriers
        for (int i = 0; i < kStages2; ++i)
          if (armed & (1u << i)) drain_phase(&s.full[i], (armed_par >> i) & 1u);
    }
    __syncwarp();
  } else if (warp == 1) {
    // ------------------------------------------------- MMA (leader only)
    if (lane == 0 && leader) {
      int stage = 0;
      uint32_t phase = 0;
      int it = 0;
      bool issued = false;
      for (int64_t t = pair; t < tiles && !*abort; t += pairs, ++it) {
        const int acc = it & 1;
        const uint32_t acc_phase = (uint32_t)(it >> 1) & 1u;
        if (!wait_phase(&s.tempty[acc], acc_phase ^ 1u, abort, err, 0x202)) break;
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(acc * kBN);
        bool ok = true;
        for (int kb = 0; kb < nk; ++kb) {
          if (!wait_phase(&s.full[stage], phase, abort, err, 0x203)) {
            ok = false;
            break;
          }
          tc_fence_after();
#pragma unroll
          for (int k16 = 0; k16 < kBK / 16; ++k16)
            mma_f16_pair(d, smem_desc(s.a[stage], k16), smem_desc(s.b[stage], k16), (kb | k16) != 0);
          issued = true;
          mma_commit_pair(&s.empty[stage]);
          if (++stage == kStages2) {
            stage = 0;
            phase ^= 1u;
          }
        }
        if (!ok) break;
        mma_commit_pair(&s.tfull[acc]);
      }
      if (*abort && issued) {
        mma_commit_pair_local(&s.drain);
        drain_phase(&s.drain, 0);
      }
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------ epilogue (both)
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    const float alpha = *d_alpha;
    const uint32_t tempty_leader0 = cluster_addr(&s.tempty[0], 0), tempty_leader1 = cluster_addr(&s.tempty[1], 0);
    int it = 0;
    for (int64_t t = pair; t < tiles; t += pairs, ++it) {
      const int acc = it & 1;
      const uint32_t acc_phase = (uint32_t)(it >> 1) & 1u;
      bool ok = wait_phase(&s.tfull[acc], acc_phase, abort, err, 0x204);
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) break;
      tc_fence_after();
      int64_t mb, nb;
      tm.coords(t, mb, nb);
      const int64_t row = mb * 256 + 128 * rank + q * 32 + lane;
      const bool row_ok = row < m;
      const float ra = row_ok && row_scale ? alpha * row_scale[row] : alpha;
      const int64_t col0 = nb * 256 + half * 128;
#pragma unroll 1
      for (int ch = 0; ch < 4; ++ch) {
        float v[32];
        tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * kBN + half * 128 + ch * 32), v);
        const int64_t cb = col0 + ch * 32;
        const int ncol = row_ok ? (int)min((int64_t)32, max((int64_t)0, n - cb)) : 0;
        float* p = C + row + ldc * cb;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          float c[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) c[j] = 16 * h + j < ncol ? __ldcg(p + ldc * (16 * h + j)) : 0.f;
#pragma unroll
          for (int j = 0; j < 16; ++j)
            if (16 * h + j < ncol) __stcg(p + ldc * (16 * h + j), fmaf(ra, v[16 * h + j], c[j]));
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_cluster(acc ? tempty_leader1 : tempty_leader0);
    }
  }

  tc_fence_before();
  __syncthreads();
  // the peer's copies and remote arrivals target the leader's barriers, and
  // both CTAs read their TMEM: neither leaves before the other is done
  cluster_sync_all();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// ------------------------------------------------------ grouped form
// Many independent updates in one persistent launch (the batched LU's
// trailing updates, one problem per mesh): problem p is C_p += alpha_p s_i
// (A_p B_p^T) with its tensor maps at maps[map_p], maps[map_p + 1] (in
// global memory, written before the launch), its output tiles numbered
// tile_start[p] .. tile_start[p + 1).  The roles and the pipeline are the
// 1-SM kernel's; each tile looks its problem up.
__device__ __forceinline__ int tile_problem(const int64_t* __restrict__ tile_start, int n_probs, int64_t t) {
  int lo = 0, hi = n_probs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tile_start[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// REDUCE: the epilogue adds the scaled accumulator into C with TMA
// reduce-add copies (cp.reduce.async.bulk.tensor, 32 x 32 boxes staged in
// shared memory per epilogue warp, C's tensor map at cmaps[cmap]): the SMs
// never read C, L2 applies the additions.
struct alignas(1024) TcSmemR {
  TcSmem base;
  float red[kEpiWarps][32 * 32];
};
constexpr size_t kSmemBytesR = sizeof(TcSmemR) + 1024;
static_assert(kSmemBytesR <= 232448, "shared memory of the reduce-add epilogue");

__device__ __forceinline__ void tma_reduce_add_2d(const CUtensorMap* map, const void* src, int x, int y) {
  asm volatile("cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.tile.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(smem_u32(src)), "r"(x), "r"(y)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

template <bool REDUCE>
__global__ void __launch_bounds__(kThreads, 1)
    update_tc_grouped_kernel(const CUtensorMap* __restrict__ maps, const TcProblem* __restrict__ probs,
                             const int64_t* __restrict__ tile_start, int n_probs, int* __restrict__ err,
                             const CUtensorMap* __restrict__ cmaps) {
  extern __shared__ uint8_t smem_raw[];
  TcSmemR& sr = *reinterpret_cast<TcSmemR*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  TcSmem& s = sr.base;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t tiles = tile_start[n_probs];
  volatile int* abort = &s.abort;
  auto tile_of = [&](int64_t t, int& p, int64_t& mb, int64_t& nb) {
    p = tile_problem(tile_start, n_probs, t);
    const int64_t l = t - tile_start[p];
    const int64_t tn = (probs[p].n + kBN - 1) / kBN;
    mb = l / tn;
    nb = l - mb * tn;
  };

  if (threadIdx.x == 0) {
    for (int i = 0; i < kStages; ++i) {
      mbar_init(&s.full[i], 1);
      mbar_init(&s.empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&s.tfull[i], 1);
      mbar_init(&s.tempty[i], kEpiWarps);
    }
    mbar_init(&s.drain, 1);
    s.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s.tmem_base;

  if (warp == 0) {
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      uint32_t armed = 0, armed_par = 0;
      for (int64_t t = blockIdx.x; t < tiles && !*abort; t += gridDim.x) {
        int p;
        int64_t mb, nb;
        tile_of(t, p, mb, nb);
        const CUtensorMap* ma = maps + probs[p].map;
        const int nk = (probs[p].k + kBK - 1) / kBK;
        // the maps were written to global memory before the launch: acquire
        // them for the tensor-map proxy before the copies read them
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(ma))
                     : "memory");
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(ma + 1))
                     : "memory");
        for (int kb = 0; kb < nk; ++kb) {
          if (!wait_phase(&s.empty[stage], phase ^ 1u, abort, err, 0x301)) break;
          armed &= ~(1u << stage);
          mbar_expect_tx(&s.full[stage], kStageA + kStageB);
          tma_load_2d(s.a[stage], ma, &s.full[stage], kb * kBK, (int)(mb * kBM));
          tma_load_2d(s.b[stage], ma + 1, &s.full[stage], kb * kBK, (int)(nb * kBN));
          armed |= 1u << stage;
          armed_par = (armed_par & ~(1u << stage)) | (phase << stage);
          if (++stage == kStages) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      if (*abort)
        for (int i = 0; i < kStages; ++i)
          if (armed & (1u << i)) drain_phase(&s.full[i], (armed_par >> i) & 1u);
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      int it = 0;
      bool issued = false;
      for (int64_t t = blockIdx.x; t < tiles && !*abort; t += gridDim.x, ++it) {
        int p;
        int64_t mb, nb;
        tile_of(t, p, mb, nb);
        const int nk = (probs[p].k + kBK - 1) / kBK;
        const int acc = it & 1;
        const uint32_t acc_phase = (uint32_t)(it >> 1) & 1u;
        if (!wait_phase(&s.tempty[acc], acc_phase ^ 1u, abort, err, 0x302)) break;
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(acc * kBN);
        bool ok = true;
        for (int kb = 0; kb < nk; ++kb) {
          if (!wait_phase(&s.full[stage], phase, abort, err, 0x303)) {
            ok = false;
            break;
          }
          tc_fence_after();
#pragma unroll
          for (int k16 = 0; k16 < kBK / 16; ++k16)
            mma_f16(d, smem_desc(s.a[stage], k16), smem_desc(s.b[stage], k16), (kb | k16) != 0);
          issued = true;
          mma_commit(&s.empty[stage]);
          if (++stage == kStages) {
            stage = 0;
            phase ^= 1u;
          }
        }
        if (!ok) break;
        mma_commit(&s.tfull[acc]);
      }
      if (*abort && issued) {
        mma_commit(&s.drain);
        drain_phase(&s.drain, 0);
      }
    }
    __syncwarp();
  } else {
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    int it = 0;
    for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x, ++it) {
      const int acc = it & 1;
      const uint32_t acc_phase = (uint32_t)(it >> 1) & 1u;
      bool ok = wait_phase(&s.tfull[acc], acc_phase, abort, err, 0x304);
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) break;
      tc_fence_after();
      int p;
      int64_t mb, nb;
      tile_of(t, p, mb, nb);
      const TcProblem& P = probs[p];
      const float alpha = *P.alpha;
      const int64_t row = mb * kBM + q * 32 + lane;
      const bool row_ok = row < P.m;
      const float ra = row_ok && P.row_scale ? alpha * P.row_scale[row] : alpha;
      const int64_t col0 = nb * kBN + half * 128;
      if (REDUCE) {
        // this warp's 32 rows x 32 columns per chunk, column-major in its
        // staging box, added into C by one TMA reduce-add per chunk
        float* box = sr.red[warp - 2];
        const int64_t row0 = mb * kBM + q * 32;
        const CUtensorMap* cm = cmaps + P.cmap;
#pragma unroll 1
        for (int ch = 0; ch < 4; ++ch) {
          float v[32];
          tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * kBN + half * 128 + ch * 32), v);
          const int64_t cb = col0 + ch * 32;
          // the previous chunk's copy has read the box
          if (lane == 0) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
          __syncwarp();
          const float sc = row_ok ? ra : 0.f;
#pragma unroll
          for (int j = 0; j < 32; ++j) box[32 * j + lane] = sc * v[j];
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          __syncwarp();
          if (lane == 0 && row0 < P.m && cb < P.n) tma_reduce_add_2d(cm, box, (int)row0, (int)cb);
        }
      } else {
#pragma unroll 1
        for (int ch = 0; ch < 4; ++ch) {
          float v[32];
          tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * kBN + half * 128 + ch * 32), v);
          const int64_t cb = col0 + ch * 32;
          const int ncol = row_ok ? (int)min((int64_t)32, max((int64_t)0, (int64_t)P.n - cb)) : 0;
          float* pc = P.C + row + P.ldc * cb;
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            float c[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) c[j] = 16 * h + j < ncol ? __ldcg(pc + P.ldc * (16 * h + j)) : 0.f;
#pragma unroll
            for (int j = 0; j < 16; ++j)
              if (16 * h + j < ncol) __stcg(pc + P.ldc * (16 * h + j), fmaf(ra, v[16 * h + j], c[j]));
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&s.tempty[acc]);
    }
    // the reduce-add copies complete before the CTA's shared memory goes away
    if (REDUCE && lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    __syncwarp();
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// rows x k FP16, K-major with ld elements between rows; box = box_rows x 64
bool make_map(CUtensorMap* map, const void* base, int64_t rows, int64_t k, int64_t ld, uint32_t box_rows) {
  auto fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)(ld * 2)};
  const cuuint32_t box[2] = {(cuuint32_t)kBK, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// C (m x n FP32, column-major, ldc) for the L2 prefetch: boxes of 128 rows x
// 256 columns, the output tile
bool make_map_c(CUtensorMap* map, const float* C, int64_t m, int64_t n, int64_t ldc) {
  auto fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)m, (cuuint64_t)n};
  const cuuint64_t strides[1] = {(cuuint64_t)(ldc * 4)};
  const cuuint32_t box[2] = {(cuuint32_t)kBM, (cuuint32_t)kBN};
  const cuuint32_t estr[2] = {1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(C), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// HFPX_TC_GROUP (1..64) overrides the raster group, for tuning sweeps
int raster_group() {
  static const int g = [] {
    const char* e = std::getenv("HFPX_TC_GROUP");
    const int v = e ? std::atoi(e) : 0;
    return v >= 1 && v <= 64 ? v : kGroupM;
  }();
  return g;
}

}  // namespace

bool tc_update_supported(int64_t lda_k, int64_t ldb_k, const void* A, const void* B) {
  // TMA: 16-byte aligned bases and row strides
  return lda_k % 8 == 0 && ldb_k % 8 == 0 && (reinterpret_cast<uintptr_t>(A) & 15) == 0 &&
         (reinterpret_cast<uintptr_t>(B) & 15) == 0 && encode_fn() != nullptr;
}

int tc_update_f16(hfpx_ctx* c, cudaStream_t st, int64_t m, int64_t n, int64_t k, const void* A, int64_t lda_k,
                  const void* B, int64_t ldb_k, float* C, int64_t ldc, const float* d_alpha, const float* d_row_scale,
                  int* d_err, int max_ctas) {
  if (m <= 0 || n <= 0 || k <= 0) return HFPX_OK;
  if (m > INT32_MAX || n > INT32_MAX || k > INT32_MAX || !tc_update_supported(lda_k, ldb_k, A, B))
    return set_error(c, HFPX_ERR_ARG, "tensor-core update: unsupported operand layout");
  // the 2-SM kernel unless HFPX_TC_2SM=0 (or a single SM may be used)
  const int cap = max_ctas > 0 ? std::min(max_ctas, c->num_sms) : c->num_sms;
  const char* env2 = std::getenv("HFPX_TC_2SM");
  const bool two_sm = cap >= 2 && !(env2 && std::string(env2) == "0");
  CUtensorMap ma, mb, mc;
  if (!make_map(&ma, A, m, k, lda_k, kBM) || !make_map(&mb, B, n, k, ldb_k, two_sm ? 128 : kBN))
    return set_error(c, HFPX_ERR_CUDA, "tensor-core update: tensor map encoding failed");
  // C's prefetch needs a 16-byte aligned base and row stride (it only warms
  // L2: without it the epilogue reads C from HBM)
  int prefetch_c = (reinterpret_cast<uintptr_t>(C) & 15) == 0 && ldc % 4 == 0 && make_map_c(&mc, C, m, n, ldc);
  if (!prefetch_c) std::memset(&mc, 0, sizeof(mc));
  ++g_launches;
  if (two_sm) {
    static PerDeviceOnce attr2;
    if (int rc = check_cuda(c, smem_attr_once(attr2, update_tc2_kernel, (int)kSmemBytes2),
                            "tensor-core update attribute"))
      return rc;
    const int64_t tiles = ((m + 255) / 256) * ((n + 255) / 256);
    const int64_t pairs = std::max<int64_t>(1, std::min<int64_t>(tiles, cap / 2));
    update_tc2_kernel<<<(unsigned)(2 * pairs), kThreads, kSmemBytes2, st>>>(
        ma, mb, mc, prefetch_c, C, ldc, m, n, (int)k, raster_group(), d_alpha, d_row_scale, d_err);
  } else {
    static PerDeviceOnce attr;
    if (int rc = check_cuda(c, smem_attr_once(attr, update_tc_kernel, (int)kSmemBytes), "tensor-core update attribute"))
      return rc;
    const int64_t tiles = ((m + kBM - 1) / kBM) * ((n + kBN - 1) / kBN);
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(tiles, cap));
    update_tc_kernel<<<grid, kThreads, kSmemBytes, st>>>(ma, mb, mc, prefetch_c, C, ldc, m, n, (int)k, raster_group(),
                                                         d_alpha, d_row_scale, d_err);
  }
  return check_cuda(c, cudaGetLastError(), "tensor-core update launch");
}

bool tc_make_operand_map(void* map, const void* base, int64_t rows, int64_t k, int64_t ld_k, int box_rows) {
  return make_map(static_cast<CUtensorMap*>(map), base, rows, k, ld_k, (uint32_t)box_rows);
}

int tc_grouped_setup(hfpx_ctx* c) {
  static PerDeviceOnce attr, attr_r;
  int rc = check_cuda(c, smem_attr_once(attr, update_tc_grouped_kernel<false>, (int)kSmemBytes),
                      "grouped update attribute");
  if (!rc)
    rc = check_cuda(c, smem_attr_once(attr_r, update_tc_grouped_kernel<true>, (int)kSmemBytesR),
                    "grouped update attribute");
  return rc;
}

bool tc_make_c_map(void* map, const float* C, int64_t m, int64_t n, int64_t ldc) {
  auto fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)m, (cuuint64_t)n};
  const cuuint64_t strides[1] = {(cuuint64_t)(ldc * 4)};
  const cuuint32_t box[2] = {32, 32};
  const cuuint32_t estr[2] = {1, 1};
  return fn(static_cast<CUtensorMap*>(map), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(C), dims, strides,
            box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

void tc_update_grouped(cudaStream_t st, int grid, const void* d_maps, const TcProblem* d_probs,
                       const int64_t* d_tile_start, int n_probs, int* d_err, const void* d_cmaps) {
  ++g_launches;
  if (d_cmaps)
    update_tc_grouped_kernel<true><<<(unsigned)grid, kThreads, kSmemBytesR, st>>>(
        static_cast<const CUtensorMap*>(d_maps), d_probs, d_tile_start, n_probs, d_err,
        static_cast<const CUtensorMap*>(d_cmaps));
  else
    update_tc_grouped_kernel<false><<<(unsigned)grid, kThreads, kSmemBytes, st>>>(
        static_cast<const CUtensorMap*>(d_maps), d_probs, d_tile_start, n_probs, d_err, nullptr);
}

}  // namespace hfpx
