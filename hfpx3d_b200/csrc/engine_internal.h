// Internal declarations shared by the engine's translation units.
#pragma once
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/hfpx_engine.h"

struct hfpx_ctx {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  void* cublas = nullptr;          // cublasHandle_t
  // LU look-ahead: panels on a high-priority stream with their own cuBLAS
  // handle, deferred left-side row swaps on a third stream
  cudaStream_t stream_panel = nullptr, stream_left = nullptr;
  void* cublas_panel = nullptr;
  void* cusolver = nullptr;        // cusolverDnHandle_t (small dense LU), made on first use
  std::string last_error;
  int* d_flags = nullptr;          // device status words (see kernels)
  // device work buffers kept between calls (grown on demand, freed with the
  // context), so repeated factorisations and solves allocate nothing
  static constexpr int kScratchSlots = 64;
  void* scratch[kScratchSlots] = {};
  size_t scratch_bytes[kScratchSlots] = {};
  // tile triangular solves: tiles the flag array covers, epoch of the last
  // solve, tickets handed out so far
  int64_t trsv_cap = 0;
  int trsv_epoch = 0;
  unsigned long long trsv_base = 0;
  // the coarse level's set-up runs on its own stream beside the near-field
  // blocks (made on first use)
  cudaStream_t stream_coarse = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
};

// Near-field pattern of a mesh: the elements sharing a vertex with element j
// are its neighbours N(j); the pattern of block column j is P(j) = {j} + N(j).
// Blocks of a near-field operator are stored column by column: column j's
// self block at j + ptr[j], its neighbour blocks after it in idx order, so
// edge e (src idx[e] -> column dst[e]) is block dst[e] + 1 + e.
struct NearPattern {
  int64_t n_el = 0, n_edges = 0;
  int maxdeg = 0;
  std::vector<int32_t> ptr, idx, dst, rev;   // rev[e]: the edge (dst[e] -> idx[e])
  // row view for products: row i's blocks rblk[k] with column rcol[k], k in [rptr[i], rptr[i+1])
  std::vector<int32_t> rptr, rblk, rcol;
  int32_t *d_ptr = nullptr, *d_idx = nullptr, *d_dst = nullptr, *d_rev = nullptr;
  int32_t *d_rptr = nullptr, *d_rblk = nullptr, *d_rcol = nullptr;
  int64_t blocks() const { return n_el + n_edges; }
};

struct hfpx_gnn_graph;

// Read-only view of an operator for the kernels that gather its entries (the
// near-field preconditioners, the network's inputs): the FP64 matrix A, or a
// mixed-precision operator (Af every entry in FP32, lo the low parts of the
// near-field blocks on the pattern ptr/idx: block (i, j) of column j is
// j + ptr[j] for i == j, j + 1 + e for idx[e] == i).
struct OpView {
  const double* A = nullptr;
  const float* Af = nullptr;
  int64_t ld = 0;
  const float* lo = nullptr;
  const int32_t* ptr = nullptr;
  const int32_t* idx = nullptr;
#ifdef __CUDACC__
  // entry (r, c) whose near-field block index is known (blk < 0: none)
  __device__ __forceinline__ double at_blk(int64_t r, int64_t c, int64_t blk) const {
    if (A) return A[r + ld * c];
    double v = (double)Af[r + ld * c];
    if (lo && blk >= 0) v += (double)lo[blk * 324 + 18 * (c % 18) + (r % 18)];
    return v;
  }
  // any entry: the block is looked up in column c / 18's pattern
  __device__ __forceinline__ double at(int64_t r, int64_t c) const {
    if (A) return A[r + ld * c];
    int64_t blk = -1;
    if (lo) {
      const int64_t i = r / 18, j = c / 18;
      if (i == j) {
        blk = j + ptr[j];
      } else {
        for (int32_t e = ptr[j]; e < ptr[j + 1]; ++e)
          if (idx[e] == i) {
            blk = j + 1 + e;
            break;
          }
      }
    }
    return at_blk(r, c, blk);
  }
#endif
};

// Coarse space of a mesh for the two-level preconditioner: the elements
// grouped into aggregates (k-means of their centroids), and on each aggregate
// the DD components' linear functions 1, xi, eta in the aggregate's tangent
// plane, sampled at the element nodes.  Coarse unknown 9 a + 3 m + k is
// basis function m (1, xi, eta) of DD component k on aggregate a; P (n x nc)
// has P[18 e + 3 node + k, 9 agg(e) + 3 m + k] = w[(6 e + node) 3 + m].
struct CoarseSpace {
  int64_t n_el = 0, n_agg = 0, nc = 0;
  int agg_size = 0, max_agg = 0;
  std::vector<int32_t> agg_of, ptr, el;   // element -> aggregate; elements of aggregate a: el[ptr[a] .. ptr[a+1])
  std::vector<double> w;                  // n_el x 6 nodes x 3 basis values
  int32_t *d_ptr = nullptr, *d_el = nullptr, *d_agg_of = nullptr;
  double* d_w = nullptr;
};

// The network's geometry inputs of a mesh (host arrays, the bf16 values as
// their bit patterns): the geometry columns of the node rows (n x 8) and of
// the edge rows (E x 12), frames (9 per element) and sizes.
struct GraphHostInputs {
  std::vector<uint16_t> xn, xe;
  std::vector<float> rot, size;
};

// Mesh-only set-up of the near-field preconditioners, made on a host thread
// started by hfpx_mesh_create (meshes of kMeshSetupMinElems elements or
// more) while the device assembles: the near-field pattern's host arrays,
// the coarse aggregates and basis (default aggregate size) and the
// network's geometry inputs, in that order.  Consumers wait for the part
// they need and copy it; a part that failed is rebuilt where it is needed.
struct MeshHostSetup {
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv;
  int done = 0;                 // parts finished: 1 pattern, 2 + coarse, 3 + graph inputs
  bool pattern_ok = false, coarse_ok = false, graph_ok = false;
  NearPattern pattern;          // host arrays only
  CoarseSpace coarse;           // host arrays only
  GraphHostInputs graph;
  // wait until `part` (1, 2, 3) is finished
  void wait(int part) {
    std::unique_lock<std::mutex> l(mu);
    cv.wait(l, [&] { return done >= part; });
  }
};
constexpr int64_t kMeshSetupMinElems = 1000;

struct hfpx_mesh {
  int64_t n_el = 0;
  void* d_elem = nullptr;          // ElemRec[n_el]
  // host copies for the near-field pattern and the learned preconditioner's
  // geometry features: vertex ids (3 per element) and vertex coordinates
  // (9 per element, vertex j's x, y, z at 3 j)
  std::vector<int64_t> h_vid;
  std::vector<double> h_vert;
  // built on first use and kept with the mesh: the near-field pattern and the
  // learned preconditioner's graph (geometry inputs and buffers)
  std::shared_ptr<NearPattern> pattern;
  std::shared_ptr<CoarseSpace> coarse;
  hfpx_gnn_graph* gnn_graph = nullptr;
  std::unique_ptr<MeshHostSetup> host_setup;   // null for small meshes
};

struct hfpx_gnn;

struct hfpx_precond {
  int kind = 0;
  int64_t n_el = 0, n = 0;
  const hfpx_mesh* mesh = nullptr;    // the mesh it was made for (updates read it)
  std::shared_ptr<NearPattern> pat;   // the mesh's
  double* d_blocks = nullptr;      // blocks() x 18 x 18, each column-major
  double* d_dinv = nullptr;        // inverses of the diagonal blocks, n_el x 18 x 18
  // two-level form (kind with HFPX_PC_COARSE): the coarse space, A P
  // (n x nc, column-major), the coarse operator P^T A P factored, its
  // explicit inverse, and work vectors
  std::shared_ptr<CoarseSpace> cs;
  double* d_ap = nullptr;
  double* d_ac = nullptr;          // P^T A P, then its LU factors (nc x nc)
  int32_t* d_acpiv = nullptr;
  int* d_acinfo = nullptr;
  void* d_acwork = nullptr;        // the factorisation's workspace
  size_t acwork_bytes = 0;
  double* d_acinv = nullptr;
  double *d_q = nullptr, *d_cc = nullptr, *d_t = nullptr;
};

struct hfpx_matrix {
  int64_t n = 0, ld = 0;
  double* d_a = nullptr;           // FP64 n x n column-major (ld); null for a mixed-precision operator
  float* d_f = nullptr;            // FP32 working copy (mixed mode), ld
  int f32_current = 0;             // d_f holds the operator (written by the assembly), not factors
  // Mixed-precision operator (hfpx_assemble_mixed): d_f holds every entry
  // rounded to FP32 and d_lo, on the near-field blocks of `pat` (each
  // element with itself and with the elements sharing a vertex, 18 x 18
  // column-major blocks in the pattern's block order), the FP32 rounding of
  // what that rounding lost, so hi + lo is the FP64 entry to about 2^-48.
  int op_mixed = 0;
  float* d_lo = nullptr;
  int64_t lo_blocks = 0;
  std::shared_ptr<NearPattern> pat;
  int32_t* d_piv = nullptr;        // pivots (0-based global rows), n
  int factored = 0;                // 0 none, 1 fp64 in place, 2 fp32 copy
  int64_t info = 0;
  // inverses of the FP32 factors' 128 x 128 diagonal blocks (L, then U),
  // made by the first single-right-hand-side solve after a factorisation
  mutable float* d_dinv = nullptr;
  mutable int dinv_valid = 0;
};

namespace hfpx {
// HFPX_PROFILE=1: host times of the set-up phases (pattern, coarse space,
// network graph) to stderr
using SetupClock = std::chrono::steady_clock;
inline double ms_since(SetupClock::time_point t0) {
  return std::chrono::duration<double, std::milli>(SetupClock::now() - t0).count();
}
bool setup_profile();
void setup_note(const char* what, double ms);

// launches of this engine's own kernels in this process (library kernels excluded)
extern std::atomic<long long> g_launches;

// Per-device set-up flags.  Kernel attributes and __constant__ data belong to
// one device's context, so "done" is one bit per device, set only after the
// set-up succeeded on the current device.
struct PerDeviceOnce {
  std::atomic<unsigned long long> done{0};
  // true when the current device still needs the set-up (devices >= 64 always do)
  bool pending(int* dev_out = nullptr) const {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return true;
    if (dev_out) *dev_out = dev;
    return dev >= 64 || !(done.load() & (1ull << dev));
  }
  void mark() {
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && dev < 64) done.fetch_or(1ull << dev);
  }
};
// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) once per device
template <class F>
inline cudaError_t smem_attr_once(PerDeviceOnce& once, F* func, int bytes) {
  if (!once.pending()) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) once.mark();
  return e;
}
int set_error(hfpx_ctx* c, int code, const std::string& msg);
int check_cuda(hfpx_ctx* c, cudaError_t e, const char* what);
// Work buffer `slot` of the context with at least `bytes` bytes (null when
// the device is out of memory; the CUDA error state is cleared).  A slot
// that grows is reallocated after the context's streams finish with it.
void* ctx_scratch(hfpx_ctx* c, int slot, size_t bytes);
// scratch slots
enum : int {
  kScrPanelCand, kScrPanelMax, kScrPanelIdx, kScrPanelRowj, kScrInfo, kScrPlanPanel, kScrPlans, kScrLLSlots,
  kScrLLErr, kScrLinv, kScrA12, kScrL16, kScrU16, kScrAmax, kScrCoef, kScrPerm, kScrSolveTmp, kScrRefX,
  kScrRefR, kScrRefRf, kScrDof, kScrXtmp, kScrResidPart, kScrResidMax, kScrTrsvFlags, kScrTrsvTicket,
  kScrTrsvErr, kScrTslu, kScrGmresV, kScrGmresZ, kScrGmresH, kScrGmresZero, kScrHostNods, kScrHostConn,
  kScrHostSinf, kScrHostRhs, kScrPanelInv, kScrTcErr, kScrRowScale, kScrStressDd, kScrStressPts, kScrStressSinf,
  kScrStressOut, kScrStressInfl, kScrStressVec, kScrStressSum, kScrGmresEst, kScrMixedY, kScrMixedBlk, kScrGrowList,
  kScrRefColMax, kScrCount
};

// assembly.cu
size_t elem_record_bytes();
void launch_element_precompute(const double* d_nods, int64_t ld_nods, const int64_t* d_conn,
                               int64_t ld_conn, int64_t n_el, double beta, void* d_elem,
                               cudaStream_t s);
// d_f (optional): an FP32 copy of the matrix written in the same pass.
// d_a null: the mixed-precision operator, d_f every entry in FP32 and d_lo
// (on the near-field pattern np_ptr/np_idx, at most kMaxNearDeg neighbours
// per element) the low parts of the near-field blocks.  far32: in-plane
// pairs at least 8 source-element sizes apart, outside the near-field
// pattern, are integrated in FP32 by a 16-point rule (mixed operator only).
constexpr int kMaxNearDeg = 64;
void launch_assemble(const void* d_elem, int64_t n_el, const int32_t* d_dof, double G, double nu,
                     int is_dd_local, double* d_a, int64_t ld, float* d_f, int* d_general_count,
                     cudaStream_t s, float* d_lo = nullptr, const int32_t* np_ptr = nullptr,
                     const int32_t* np_idx = nullptr, int far32 = 0);
// One mesh of a batched assembly: its element records, DoF map, the FP32
// operator A (hi parts) with its near-field low parts lo on the pattern
// np_ptr/np_idx, and the FP32 copy F the factorisation overwrites (ld rows).
struct BatchAsmMesh {
  const void* elems;
  const int32_t* dof;
  float* A;
  float* F;
  float* lo;
  const int32_t* np_ptr;
  const int32_t* np_idx;
  int64_t n_el;
  int64_t ld;
};
// tasks: n_tasks int4 (mesh, source element, target tile of 128
// collocation points, 0), one CTA each
int batch_assemble_setup(cudaStream_t s);
void launch_batch_assemble(const BatchAsmMesh* d_meshes, const void* d_tasks, int64_t n_tasks, double G, double nu,
                           int* d_status, cudaStream_t s, int far32);
// the 6 unit in-situ stress states' right-hand sides of every mesh (no
// fixed DoF), mesh m's n x 6 block at d_B + d_boff[m]
void launch_batch_basis_rhs(const BatchAsmMesh* d_meshes, int64_t n_mesh, double* d_B, const int64_t* d_boff,
                            cudaStream_t s);
// the pairs of an incremental assembly (FP64 only): every target of the
// sources slist[0..n_s), and the targets tlist[0..n_t) of the sources
// slist2[0..n_s2)
void launch_assemble_partial(const void* d_elem, int64_t n_el, const int32_t* d_dof, double G, double nu,
                             int is_dd_local, double* d_a, int64_t ld, int* d_status, cudaStream_t s,
                             const int32_t* slist, int64_t n_s, const int32_t* slist2, int64_t n_s2,
                             const int32_t* tlist, int64_t n_t);
void launch_vc_border(const void* d_elem, int64_t n_el, const int32_t* d_dof, int64_t n_dof,
                      int is_dd_local, double* d_a, int64_t ld, cudaStream_t s);
void launch_rhs(const void* d_elem, int64_t n_el, const int32_t* d_dof, const double* d_sinf,
                int64_t n_rhs, double* d_rhs, int64_t ld_rhs, cudaStream_t s);
void launch_stress(const void* d_elem, int64_t n_el, double G, double nu, int is_dd_local,
                   const double* d_dd, const double* d_pts, int64_t n_pts, const double* d_sinf,
                   double* d_out, cudaStream_t s);
void launch_stress_influence(const void* d_elem, int64_t n_el, double G, double nu, int is_dd_local,
                             const double* d_pts, int64_t n_pts, double* d_M, int64_t ldm, cudaStream_t s);
void launch_dd_to_vec(const double* d_dd, int64_t n_el, int64_t n_cases, double* d_D, cudaStream_t s);
void launch_stress_out(const double* d_S, int64_t n_pts, int64_t n_cases, const double* d_sinf, double* d_out,
                       cudaStream_t s);
void launch_local_block(double G, double nu, double h, double zr, double zi, const double* d_tau,
                        const double* d_sfm, double* d_out, cudaStream_t s);
void launch_convert_f32(const double* d_a, int64_t ld, int64_t n, float* d_f, cudaStream_t s);

// lu.cu
int lu_factor_fp64(hfpx_ctx* c, hfpx_matrix* m);
int lu_factor_fp32(hfpx_ctx* c, hfpx_matrix* m);
int lu_solve_fp64(hfpx_ctx* c, const hfpx_matrix* m, double* d_b, int64_t nrhs, int64_t ldb);
int lu_solve_fp32(hfpx_ctx* c, const hfpx_matrix* m, float* d_b, int64_t nrhs, int64_t ldb);
int refine_solve(hfpx_ctx* c, const hfpx_matrix* m, double* d_b, int64_t nrhs, int64_t ldb,
                 double tol, int max_iter, hfpx_solve_info* info);
int lu_panel_factor_noalloc(hfpx_ctx* c, double* d_a, int64_t lda, int64_t m, int w, int32_t* d_piv,
                            int64_t* info);
int gmres_solve(hfpx_ctx* c, const hfpx_matrix* m, double* d_b, double tol, int restart, int max_iter,
                hfpx_solve_info* info);

// gemm_tc.cu: C (m x n FP32, column-major, ldc) += alpha s_i (A B^T)_ij on
// tcgen05 tensor cores, A (m x k) and B (n x k) FP16 K-major with row strides
// lda_k, ldb_k (multiples of 8), alpha = *d_alpha, s_i = d_row_scale[i]
// (null: 1); d_err a zeroed failure word (set when a pipeline wait times
// out); at most max_ctas CTAs (<= 0: all SMs).
bool tc_update_supported(int64_t lda_k, int64_t ldb_k, const void* A, const void* B);
int tc_update_f16(hfpx_ctx* c, cudaStream_t s, int64_t m, int64_t n, int64_t k, const void* A, int64_t lda_k,
                  const void* B, int64_t ldb_k, float* C, int64_t ldc, const float* d_alpha, const float* d_row_scale,
                  int* d_err, int max_ctas);

// the grouped form (the batched LU's trailing updates): problem p is
// C += alpha s_i (A B^T), m x n x k, its operand maps at maps[map], maps[map + 1]
// (tensor maps of 128 bytes each in device memory, made by
// tc_make_operand_map with box rows 128 for A and 256 for B), its tiles
// tile_start[p] .. tile_start[p + 1) (128 x 256 outputs each)
struct TcProblem {
  float* C;
  int64_t ldc;
  int32_t m, n, k, map;
  const float* alpha;
  const float* row_scale;
  int32_t cmap, pad;  // C's tensor map (32 x 32 boxes) for the reduce-add epilogue
};
bool tc_make_operand_map(void* map, const void* base, int64_t rows, int64_t k, int64_t ld_k, int box_rows);
// C (m x n FP32, column-major, ldc) for the reduce-add epilogue: 32 x 32 boxes
bool tc_make_c_map(void* map, const float* C, int64_t m, int64_t n, int64_t ldc);
int tc_grouped_setup(hfpx_ctx* c);
// d_cmaps (optional): the problems' C maps; the epilogue then adds into C
// with TMA reduce-add copies instead of reading and writing C
void tc_update_grouped(cudaStream_t st, int grid, const void* d_maps, const TcProblem* d_probs,
                       const int64_t* d_tile_start, int n_probs, int* d_err, const void* d_cmaps = nullptr);

// precond.cu: near-field preconditioners on the FP64 matrix (block-Jacobi,
// first-order Neumann, exact local inverse, learned) and their product
int build_pattern(hfpx_ctx* c, const hfpx_mesh* mesh, NearPattern* p);
// the host arrays of a mesh's pattern (false: no connectivity, or not symmetric)
bool pattern_host(const hfpx_mesh* mesh, NearPattern* p);
int upload_pattern(hfpx_ctx* c, NearPattern* p);
// coarse.cu: aggregates and basis of a mesh (host), the default aggregate size
bool build_coarse(const hfpx_mesh* m, int agg_size, CoarseSpace* cs);
int env_agg_size();
// gnn.cu: the network's geometry inputs of a mesh (host)
bool graph_host_inputs(const hfpx_mesh* mesh, const NearPattern& pat, GraphHostInputs* out);
// engine.cu: start the mesh's set-up thread (meshes of kMeshSetupMinElems or more)
void start_mesh_setup(hfpx_mesh* m);
void free_pattern(NearPattern* p);
// the mesh's coarse space with about agg_size elements per aggregate (built
// on first use and kept with the mesh; rebuilt for another size)
std::shared_ptr<CoarseSpace> mesh_coarse(hfpx_ctx* c, const hfpx_mesh* mesh, int agg_size);
// A P, P^T A P and its inverse for pc (storage allocated) from the matrix m
// (its FP32 copy when current, else the FP64 matrix)
int coarse_setup(hfpx_ctx* c, hfpx_precond* pc, const hfpx_matrix* m);
// z = Pc + M (v - A P c), c = (P^T A P)^-1 P^T v: the coarse correction,
// then the near-field preconditioner M on what it leaves
int coarse_apply(hfpx_ctx* c, const hfpx_precond* pc, const double* v, double* z);
int coarse_alloc(hfpx_ctx* c, hfpx_precond* pc);
void coarse_free(hfpx_precond* pc);
int precond_apply_near(hfpx_ctx* c, const hfpx_precond* pc, const double* v, double* z);
// device memory from an engine-owned stream-ordered pool that keeps freed
// blocks reserved (queued on the context's stream); pool_free first waits for
// the device, as cudaFree does
int pool_alloc(hfpx_ctx* c, void** p, size_t bytes, const char* what);
void pool_free(void* p);
void pool_free_many(void* const* p, size_t count);
// the mesh's pattern, built on first use (null on failure)
std::shared_ptr<NearPattern> mesh_pattern(hfpx_ctx* c, const hfpx_mesh* mesh);
void gnn_graph_release(hfpx_gnn_graph* g);
int precond_apply(hfpx_ctx* c, const hfpx_precond* pc, const double* v, double* z);
// the view of the operator a matrix holds (FP64, or mixed precision)
OpView op_view(const hfpx_matrix* m);
int gather_diag_inverse(hfpx_ctx* c, const OpView& A, const NearPattern& p, double* dinv, int* d_err);
int neumann_blocks(hfpx_ctx* c, const OpView& A, const NearPattern& p, const double* dinv, double* blocks,
                   bool offdiag);
// gnn.cu: the learned corrections added to the Neumann blocks of pc
int gnn_correct_blocks(hfpx_ctx* c, const hfpx_gnn* net, const hfpx_mesh* mesh, const hfpx_matrix* m,
                       hfpx_precond* pc, double shear_m);
int local_inverse_blocks(hfpx_ctx* c, const OpView& A, const NearPattern& p, double* blocks);
// lu.cu: flexible GMRES on the FP64 matrix with a right preconditioner
// apply(v, z): z = M v (FP64, device), for one right-hand side
// Af (optional): the FP32 copy of A; products use it once the rotated
// residual is below relax_below (relative), with an FP64 residual at the end
// of such a cycle.  mixed_op (optional): a mixed-precision operator; every
// product and residual is then its own (A and Af unused)
int gmres_core(hfpx_ctx* c, const double* A, int64_t lda, int64_t n, double* d_b, double tol, int restart,
               int max_iter, hfpx_solve_info* info, const std::function<int(const double*, double*)>& apply,
               const float* Af = nullptr, double relax_below = 0.0, const hfpx_matrix* mixed_op = nullptr);

// solve.cu: one right-hand side of the refinement
int trsv_tiles(int64_t n);
int tri_inverses(hfpx_ctx* c, const float* A, int64_t lda, int64_t n, float* dinv_lower, float* dinv_upper);
int trsv_f32(hfpx_ctx* c, const float* A, int64_t lda, int64_t n, const float* dinv, float* x, bool upper);
int trsv_status(hfpx_ctx* c);
int resid_chunks(int64_t n);
int residual_f64(hfpx_ctx* c, const double* A, int64_t lda, int64_t n, const double* x, const double* b, double* r,
                 double* part, unsigned long long* d_max);
// the same with the FP32 copy of the matrix (products and sums in FP64)
int residual_f32m(hfpx_ctx* c, const float* A, int64_t lda, int64_t n, const double* x, const double* b, double* r,
                  double* part, unsigned long long* d_max);
int absmax_f64(hfpx_ctx* c, const double* v, int64_t n, unsigned long long* d_max);
// r = b - A x for a mixed-precision operator: the FP32 entries (products and
// sums in FP64) plus the near-field blocks' low parts
int residual_mixed(hfpx_ctx* c, const hfpx_matrix* m, const double* x, const double* b, double* r, double* part,
                   unsigned long long* d_max);
}  // namespace hfpx
