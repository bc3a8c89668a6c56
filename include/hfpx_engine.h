/* hfpx_engine.h -- C-ABI of the B200 engine for HFPx3D's
 * assembly -> dense solve -> stress path.
 *
 * Every entry point replaces one function of the reference's C++ call surface
 * (namespace hfp3d, plus il::LU); the comment above each declaration names it
 * by file:line inside the HFPx3D project.  Plain pointers and sizes only:
 *   - all host arrays are column-major with the leading dimension given;
 *   - mesh: nods is ld_nods x n_nodes (rows 0..2 coordinates, rows 3..4 the
 *     tip flags the DoF handle reads), conn is ld_conn x n_el int64 0-based;
 *   - dof_h is n_el x 18 int64 column-major, -1 marks a fixed DoF;
 *   - device objects (context, mesh, matrix) are opaque engine-owned handles;
 *     host buffers stay caller-owned.
 * Every function returns an hfpx_status; no exception crosses the boundary.
 * hfpx_ctx_last_error() gives the message of the last failure on a context.
 * A context owns one CUDA stream and is not shared across host threads.
 */
#ifndef HFPX_ENGINE_H
#define HFPX_ENGINE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hfpx_ctx hfpx_ctx;
typedef struct hfpx_mesh hfpx_mesh;
typedef struct hfpx_matrix hfpx_matrix;

typedef enum {
  HFPX_OK = 0,
  HFPX_ERR_ARG = 1,          /* bad argument (the reference aborts via IL_EXPECT_FAST) */
  HFPX_ERR_CUDA = 2,         /* CUDA runtime / library failure */
  HFPX_ERR_SINGULAR = 3,     /* zero pivot; info holds the 1-based column (LU.h:92-99) */
  HFPX_ERR_NOMEM = 4,        /* device allocation failed */
  HFPX_ERR_STATE = 5,        /* object in the wrong state (e.g. solve before factor) */
  HFPX_ERR_NOT_CONVERGED = 6 /* refinement did not reach the tolerance */
} hfpx_status;

typedef enum {
  HFPX_LU_FP64 = 0,   /* FP64 LU in place, FP64 triangular solves */
  HFPX_LU_MIXED = 1   /* FP32 LU of a copy (trailing updates in FP16 with FP32
                         accumulation on the engine's tcgen05 kernel, each row
                         of L21 and U12 as a whole scaled by a power of two;
                         TF32 in-panel products), FP64 iterative refinement
                         against the FP64 matrix */
} hfpx_lu_mode;

typedef struct {
  int iterations;          /* refinement steps taken (0 for FP64 mode) */
  double residual;         /* final max_j ||b_j - A x_j||_inf / ||b_j||_inf */
  int converged;
} hfpx_solve_info;

/* ---- context ---------------------------------------------------------- */
int hfpx_ctx_create(int device, hfpx_ctx **ctx);
int hfpx_ctx_destroy(hfpx_ctx *ctx);
const char *hfpx_ctx_last_error(const hfpx_ctx *ctx);
/* The context's cudaStream_t, for callers that time or order work around it. */
int hfpx_ctx_stream(hfpx_ctx *ctx, void **stream);
int hfpx_ctx_synchronize(hfpx_ctx *ctx);

/* ---- DoF handle: make_dof_h_crack, src/Core/surface_mesh_utilities.cpp:28-112
 * (approximation order 2).  Host-only; writes dof_h and returns n_dof (< 0 on
 * a bad argument). */
int64_t hfpx_dof_handle(const double *nods, int64_t ld_nods, int64_t n_nodes,
                        const int64_t *conn, int64_t ld_conn, int64_t n_el,
                        int tip_type, int64_t *dof_h);

/* ---- mesh: uploads the mesh and computes, once per element, what
 * make_el_r_tensor / make_el_tau_crd / make_el_sfm_uniform / el_cp_uniform
 * (src/Core/element_utilities.cpp:62-238, 364-395) give; the reference
 * recomputes these inside its pair loops (system_assembly.cpp:64-113).
 * For meshes of 1000 elements or more it also starts one host thread that
 * makes the near-field preconditioners' mesh-only set-up (pattern, coarse
 * aggregates, network inputs) while the caller goes on (assembly);
 * hfpx_mesh_destroy joins it. */
int hfpx_mesh_create(hfpx_ctx *ctx, const double *nods, int64_t ld_nods, int64_t n_nodes,
                     const int64_t *conn, int64_t ld_conn, int64_t n_el, double beta,
                     hfpx_mesh **mesh);
int hfpx_mesh_destroy(hfpx_mesh *mesh);

/* ---- assembly: make_3dbem_matrix_s, src/Solvers/system_assembly.cpp:30-219
 * (vc_border == 0), or make_3dbem_matrix_vc, :458-557 (vc_border != 0: one
 * extra row of shape-function-weighted normals, one extra column of -normals,
 * corner 0).  The matrix stays in device memory. */
int hfpx_assemble(hfpx_ctx *ctx, const hfpx_mesh *mesh, const int64_t *dof_h, int64_t n_dof,
                  double shear_m, double poiss_r, int is_dd_local, int vc_border,
                  hfpx_matrix **matrix);
/* Same as hfpx_assemble into an existing matrix of matching size (n_dof, or
 * n_dof + 1 with vc_border), reusing its device storage; clears any
 * factorisation it held. */
int hfpx_assemble_into(hfpx_ctx *ctx, const hfpx_mesh *mesh, const int64_t *dof_h, int64_t n_dof,
                       double shear_m, double poiss_r, int is_dd_local, int vc_border,
                       hfpx_matrix *matrix);
/* The same operator as hfpx_assemble (make_3dbem_matrix_s,
 * system_assembly.cpp:30-219) held in mixed precision: every entry rounded
 * to FP32 (4 bytes per entry instead of 8), and on the near-field blocks
 * (each element with itself and with every element sharing a vertex: the
 * log/atan-singular pairs) the FP32 rounding of what that rounding lost, so
 * those entries keep about 48 bits.  The far field, whose entries decay as
 * the cube of the distance, carries the FP32 rounding only.  Products and
 * residuals with it accumulate in FP64 (hfpx_residual_device,
 * hfpx_gmres_precond); the near-field preconditioners and the network read
 * its near blocks to about 2^-48.  It needs 18 DoF per element in the
 * default numbering (no fixed DoF) and has no volume-control border; it
 * cannot be LU-factored or truncated (HFPX_ERR_STATE).  hfpx_assemble_into
 * on it re-assembles in the same form; hfpx_matrix_download gives hi + lo. */
int hfpx_assemble_mixed(hfpx_ctx *ctx, const hfpx_mesh *mesh, const int64_t *dof_h, int64_t n_dof,
                        double shear_m, double poiss_r, int is_dd_local, hfpx_matrix **matrix);
/* 1 for a mixed-precision operator (hfpx_assemble_mixed), else 0. */
int hfpx_matrix_is_mixed(const hfpx_matrix *matrix);
/* Incremental assembly of a growing crack, the step the reference leaves as
 * "todo: growing mesh" (src/Development/c_f_iteration.cpp:289) around its
 * full re-assembly (make_3dbem_matrix_s, system_assembly.cpp:30-219):
 * `mesh` is the mesh `old` was assembled for with elements appended (its
 * first n_el_old elements unchanged), dof_h its DoF handle (n_dof).  The
 * old elements must keep their DoF numbers (they number the old matrix's
 * n_old DoF; the appended elements' DoF come after), as the default
 * numbering does.  *out (new, FP64) is the whole mesh's operator: the old
 * block copied on the device, and only the new block rows and columns
 * assembled (pairs with an appended source or target).  Removing elements is
 * hfpx_matrix_truncate with the DoF of the elements that stay. */
int hfpx_assemble_grow(hfpx_ctx *ctx, const hfpx_mesh *mesh, int64_t n_el_old, const int64_t *dof_h,
                       int64_t n_dof, double shear_m, double poiss_r, int is_dd_local, const hfpx_matrix *old,
                       hfpx_matrix **out);
/* Upload a caller matrix (n x n, column-major, ld_host) for il::LU use. */
int hfpx_matrix_upload(hfpx_ctx *ctx, const double *a, int64_t n, int64_t ld_host,
                       hfpx_matrix **matrix);
int hfpx_matrix_dims(const hfpx_matrix *matrix, int64_t *n, int64_t *ld);
/* Copy the FP64 matrix (or, after an FP64 factorisation, its LU factors) to host. */
int hfpx_matrix_download(hfpx_ctx *ctx, const hfpx_matrix *matrix, double *a, int64_t ld_host);
/* Rows [i0, i0 + rows) x columns [j0, j0 + cols) of the same, into a host
 * block (ld_host >= rows): the reference's do_save_matrix output
 * (main.cpp:130-145) one block at a time, for matrices larger than host
 * memory. */
int hfpx_matrix_download_block(hfpx_ctx *ctx, const hfpx_matrix *matrix, int64_t i0, int64_t j0,
                               int64_t rows, int64_t cols, double *a, int64_t ld_host);
int hfpx_matrix_destroy(hfpx_matrix *matrix);

/* ---- right-hand side: add_s_inf_to_3dbem_rhs, system_assembly.cpp:222-274.
 * s_inf is 6 x n_rhs (Voigt xx,yy,zz,xy,xz,yz, tension positive); rhs is
 * ld_rhs x n_rhs on the host; rhs[dof] -= (n . s_inf)_l is added to what the
 * caller passes in. */
int hfpx_rhs_sinf(hfpx_ctx *ctx, const hfpx_mesh *mesh, const int64_t *dof_h, int64_t n_dof,
                  const double *s_inf, int64_t n_rhs, double *rhs, int64_t ld_rhs);

/* ---- dense LU: il::LU<il::Array2D<double>>(A, il::io, status),
 * il/linear_algebra/dense/factorization/LU.h:79-99 (LAPACK dgetrf).  Partial
 * pivoting by rows.  info = 0, or the 1-based column of a zero pivot
 * (HFPX_ERR_SINGULAR). */
int hfpx_lu_factor(hfpx_ctx *ctx, hfpx_matrix *matrix, int mode, int64_t *info);
/* lu.solve(y), LU.h:106-120 (LAPACK dgetrs), for nrhs columns of b (host,
 * ld_b x nrhs) overwritten with x.  In mixed mode x is refined in FP64 until
 * the relative residual is below tol (<= 0 selects 1e-12) or max_iter steps. */
int hfpx_lu_solve(hfpx_ctx *ctx, const hfpx_matrix *matrix, double *b, int64_t nrhs,
                  int64_t ld_b, double tol, int max_iter, hfpx_solve_info *info);

/* The row interchanges of an FP64 factorisation (dgetrf's ipiv, 0-based:
 * row i was interchanged with row ipiv[i], i = 0 .. n-1 in order). */
int hfpx_matrix_pivots(hfpx_ctx *ctx, const hfpx_matrix *matrix, int32_t *ipiv);
/* A matrix holding FP64 LU factors made elsewhere (dgetrf layout: unit L
 * below the diagonal, U on and above; ipiv 0-based as above), ready for
 * hfpx_lu_solve: the dgetrs of LU.h:106-120 given a caller's factors. */
int hfpx_matrix_upload_lu(hfpx_ctx *ctx, const double *lu, int64_t n, int64_t ld_host,
                          const int32_t *ipiv, hfpx_matrix **matrix);

/* Same as hfpx_lu_solve with b already in device memory (ld_b >= n). */
int hfpx_lu_solve_device(hfpx_ctx *ctx, const hfpx_matrix *matrix, double *d_b, int64_t nrhs,
                         int64_t ld_b, double tol, int max_iter, hfpx_solve_info *info);

/* ---- volume-control truncation: mod_3dbem_system_vc,
 * src/Solvers/system_assembly.cpp:560-629.  *out (new) is the square matrix
 * of the kept DD unknowns: out(i, j) = matrix(keep[i], keep[j]), keep
 * distinct indices below n_dd (n_dd = n - 1 when keep_border, else n), in
 * the truncated numbering's order; with keep_border the volume row and the
 * pressure column of the bordered matrix (make_3dbem_matrix_vc, :458-557)
 * follow as row and column n_keep, corner included.  The reference reads the
 * border one row past an orig_ndof-square matrix; here it is the bordered
 * matrix's own last row and column.  The matrix must hold the operator (not
 * FP64 factors); a mixed factorisation keeps it, so truncation can follow.
 * The right-hand side (delta_t by the truncated numbering, delta_v last) is
 * a host gather and not part of this call. */
int hfpx_matrix_truncate(hfpx_ctx *ctx, const hfpx_matrix *matrix, const int64_t *keep, int64_t n_keep,
                         int keep_border, hfpx_matrix **out);
/* The truncated system solved with the factors of the full one (no new
 * factorisation): on return b (host, n) holds x with x[fixed[i]] = 0 and
 * (A x)[r] = b[r] for every row r not in fixed.  The kept entries of x
 * solve the system hfpx_matrix_truncate makes from the complement of
 * `fixed`.  k + 1 solves with the existing factors (tol as in
 * hfpx_lu_solve) and a k x k capacitance system; at most 4096 distinct
 * fixed indices.  HFPX_ERR_SINGULAR when the truncated system is singular.
 * info is that of the solve of b. */
int hfpx_lu_solve_fixed(hfpx_ctx *ctx, const hfpx_matrix *matrix, const int64_t *fixed, int64_t k, double *b,
                        double tol, hfpx_solve_info *info);

/* ---- iterative solve: flexible GMRES(restart) on the FP64 matrix,
 * right-preconditioned by the FP32 factors of its mixed factorisation
 * (hfpx_lu_factor with HFPX_LU_MIXED), for one right-hand side b (host, n),
 * overwritten with x.  The reference solves only directly (LU.h:106-120);
 * this is the Krylov alternative to hfpx_lu_solve's refinement, with the same
 * stopping rule |b - A x|_inf / |b|_inf <= tol (<= 0 selects 1e-12).
 * restart <= 0 selects 50 (at most 64), max_iter <= 0 200 steps;
 * info->iterations counts preconditioner solves.  HFPX_ERR_STATE without a
 * mixed factorisation, HFPX_ERR_NOT_CONVERGED with x returned anyway. */
int hfpx_gmres(hfpx_ctx *ctx, const hfpx_matrix *matrix, double *b, double tol, int restart,
               int max_iter, hfpx_solve_info *info);
/* Same with b already in device memory. */
int hfpx_gmres_device(hfpx_ctx *ctx, const hfpx_matrix *matrix, double *d_b, double tol,
                      int restart, int max_iter, hfpx_solve_info *info);

/* Partial-pivoting LU of one tall panel already in device memory, in place,
 * without allocating anything: no counterpart in the reference.  For callers
 * that cannot call cudaMalloc: hosts whose device memory all belongs to an
 * arena of their own (an allocation would fail or take memory the arena
 * counts on), and real-time loops that forbid allocation after start-up
 * (cudaMalloc can synchronise the device and take unbounded time).
 * d_a: m x w column-major (lda >= m, 1 <= w <= 32, m >= w), overwritten with
 * L (unit lower, below the diagonal) and U; d_piv: w int32 pivot rows
 * (0-based, relative to the panel's first row, applied in order as LAPACK
 * dgetf2's ipiv); info (host): 0, or the 1-based column of the first zero
 * pivot (HFPX_ERR_SINGULAR).  Taller panels than the shared memory of all SMs
 * can hold (about 118000 rows at w = 32 on a B200) are rejected with
 * HFPX_ERR_ARG.  Its pivot-search scratch is one static device array of
 * about 138 KB shared by every call: the first call on a device looks up its
 * address (make that first call before any stream capture), and calls that
 * overlap on the GPU race.  Called while the context's stream is being
 * captured (hfpx_ctx_stream), it records its work only: info is set to 0
 * and a zero pivot is not reported (each replay of the graph factors the
 * panel in place). */
int hfpx_lu_panel_factor_noalloc(hfpx_ctx *ctx, double *d_a, int64_t lda, int64_t m, int w,
                                 int32_t *d_piv, int64_t *info);

/* The trailing-update contraction of hfpx_lu_factor's mixed mode on device
 * buffers: C += alpha A B^T, the GEMM inside LAPACK dgetrf's blocked loop
 * (A22 -= L21 U12) that il::LU reaches at
 * il/linear_algebra/dense/factorization/LU.h:87.  Runs on the engine's own
 * tcgen05 tensor-core kernel: A (m x k) and B (n x k) FP16, each K-major
 * (lda_k, ldb_k >= k elements between rows, multiples of 8, 16-byte aligned
 * bases), C (m x n) FP32 column-major (ldc >= m), FP32 accumulation, alpha
 * read from device memory (d_alpha).  Synchronises the context's stream. */
int hfpx_gemm_f16_update(hfpx_ctx *ctx, int64_t m, int64_t n, int64_t k, const void *d_a, int64_t lda_k,
                         const void *d_b, int64_t ldb_k, float *d_c, int64_t ldc, const float *d_alpha);

/* r = b - A x with the FP64 matrix (device vectors of n; b null: r = -A x),
 * the product of the refinement and of GMRES: no counterpart in the
 * reference, which solves directly (LU.h:106-120).  Deterministic (fixed
 * chunk sums, no atomics); queued on the context's stream, not synchronised. */
int hfpx_residual_device(hfpx_ctx *ctx, const hfpx_matrix *matrix, const double *d_x, const double *d_b,
                         double *d_r);

/* Number of this engine's own kernels launched on the context so far
 * (library kernels such as cuBLAS are not counted). */
int64_t hfpx_ctx_launch_count(const hfpx_ctx *ctx);

/* ---- near-field preconditioners for GMRES on the FP64 operator: no
 * counterpart in the reference, which solves directly (il::LU,
 * il/linear_algebra/dense/factorization/LU.h:79-120).  Block-sparse right
 * preconditioners M ~ A^-1 on the pattern of element adjacency (elements
 * sharing a vertex), built from the assembled FP64 matrix of a mesh without
 * fixed DoF (n = 18 n_el, no volume-control border):
 *   HFPX_PC_BLOCK_JACOBI   the inverses of the 18 x 18 diagonal blocks;
 *   HFPX_PC_NEUMANN        those plus -D_i^-1 A_ij D_j^-1 for neighbours;
 *   HFPX_PC_LOCAL_INVERSE  column j = (A[P(j), P(j)])^-1 e_j on the pattern
 *                          P(j) of element j (the square-pattern sparse
 *                          approximate inverse), by batched dense LU;
 *   HFPX_PC_LEARNED        the Neumann blocks plus corrections predicted by
 *                          the graph network `net` (hfpx_gnn_*).
 * The matrix must hold the operator (not FP64 LU factors); shear_m scales
 * the learned corrections. */
typedef struct hfpx_precond hfpx_precond;
typedef struct hfpx_gnn hfpx_gnn;
typedef enum {
  HFPX_PC_BLOCK_JACOBI = 0,
  HFPX_PC_NEUMANN = 1,
  HFPX_PC_LOCAL_INVERSE = 2,
  HFPX_PC_LEARNED = 3,
  /* or'ed with a kind above: the two-level form, a coarse correction over
   * aggregates of about 30 elements (HFPX_PC_AGG overrides the size) with
   * linear DD on each, before the near-field preconditioner:
   * z = P c + M (v - A P c), c = (P^T A P)^-1 P^T v */
  HFPX_PC_COARSE = 16
} hfpx_pc_kind;
int hfpx_precond_create(hfpx_ctx *ctx, const hfpx_mesh *mesh, const hfpx_matrix *matrix, int kind,
                        const hfpx_gnn *net, double shear_m, hfpx_precond **precond);
/* The blocks of precond made again from matrix, a re-assembly of the
 * operator on the same mesh (which must still exist), into the storage the
 * preconditioner already holds: no device allocation, so a time-stepping
 * loop that re-assembles into one matrix (hfpx_assemble_into) and updates
 * one preconditioner allocates nothing per step.  net as for create. */
int hfpx_precond_update(hfpx_ctx *ctx, hfpx_precond *precond, const hfpx_matrix *matrix, const hfpx_gnn *net,
                        double shear_m);
int hfpx_precond_destroy(hfpx_precond *precond);
/* The coarse level of a two-level preconditioner (HFPX_PC_COARSE): the number
 * of aggregates, each element's aggregate (n_el), the basis values
 * (n_el x 6 nodes x 3: 1, xi, eta), A P (n x 9 n_agg, column-major, from the
 * last create or update) and the coarse operator's inverse (9 n_agg square);
 * null arrays are skipped. */
int hfpx_precond_coarse(hfpx_ctx *ctx, const hfpx_precond *precond, int64_t *n_agg, int32_t *agg_of_el,
                        double *weights, double *ap, double *acinv);
/* The blocks (18 x 18 column-major each) and their block row and column:
 * call with null arrays to get n_blocks first. */
int hfpx_precond_blocks(hfpx_ctx *ctx, const hfpx_precond *precond, int64_t *n_blocks, int32_t *block_row,
                        int32_t *block_col, double *blocks);
/* Flexible GMRES(restart) on the FP64 matrix (not factored), right-
 * preconditioned by precond (null: none), for one right-hand side b (host,
 * n; overwritten with x); stopping rule |b - A x|_inf / |b|_inf <= tol (<= 0
 * selects 1e-12); restart <= 0 selects 50 (at most 64), max_iter <= 0 1000
 * steps.  HFPX_ERR_NOT_CONVERGED with x returned anyway. */
int hfpx_gmres_precond(hfpx_ctx *ctx, const hfpx_matrix *matrix, const hfpx_precond *precond, double *b,
                       double tol, int restart, int max_iter, hfpx_solve_info *info);
/* Same with b already in device memory. */
int hfpx_gmres_precond_device(hfpx_ctx *ctx, const hfpx_matrix *matrix, const hfpx_precond *precond,
                              double *d_b, double tol, int restart, int max_iter, hfpx_solve_info *info);

/* ---- the graph network of HFPX_PC_LEARNED: no counterpart in the
 * reference.  One node per element, one directed edge per pair of elements
 * sharing a vertex; 4 message-passing layers 64 wide, BF16 weights and
 * activations with FP32 accumulation, trained on the GPU by the engine's own
 * forward and backward kernels with Adam.  It predicts, for every block of
 * the near-field pattern, the correction that takes the Neumann block to the
 * exact local inverse's (in the frame and scale of the block's column
 * element); training regresses on that correction (mean squared error). */
typedef struct hfpx_gnn_graph hfpx_gnn_graph;
/* A new network (seeded He initialisation; output heads zero, so it starts
 * as the Neumann preconditioner). */
int hfpx_gnn_create(hfpx_ctx *ctx, uint64_t seed, hfpx_gnn **net);
int hfpx_gnn_destroy(hfpx_gnn *net);
int64_t hfpx_gnn_param_count(const hfpx_gnn *net);
/* FP32 master parameters, tensor by tensor (each weight row-major, in x
 * out, then its bias): Wn, We, (Wm, Wu) per layer, Woe, Won. */
int hfpx_gnn_get_params(hfpx_ctx *ctx, const hfpx_gnn *net, float *params);
int hfpx_gnn_set_params(hfpx_ctx *ctx, hfpx_gnn *net, const float *params);
int hfpx_gnn_save(hfpx_ctx *ctx, const hfpx_gnn *net, const char *path);
int hfpx_gnn_load(hfpx_ctx *ctx, const char *path, hfpx_gnn **net);
/* The graph of a mesh and its assembled FP64 matrix (n = 18 n_el): inputs,
 * and with with_targets the training targets (exact local inverse). */
int hfpx_gnn_graph_create(hfpx_ctx *ctx, const hfpx_mesh *mesh, const hfpx_matrix *matrix, double shear_m,
                          int with_targets, hfpx_gnn_graph **graph);
int hfpx_gnn_graph_destroy(hfpx_gnn_graph *graph);
int hfpx_gnn_graph_dims(const hfpx_gnn_graph *graph, int64_t *n_nodes, int64_t *n_edges);
/* Inputs (n_nodes x 336, n_edges x 336, as the network reads them), edge
 * endpoints (src = neighbour i, dst = column element j) and targets
 * (n_nodes x 324, n_edges x 324); any pointer may be null. */
int hfpx_gnn_graph_data(hfpx_ctx *ctx, const hfpx_gnn_graph *graph, float *xn, float *xe, int32_t *src,
                        int32_t *dst, float *tn, float *te);
/* Outputs of one forward pass (n_nodes x 324, n_edges x 324). */
int hfpx_gnn_forward(hfpx_ctx *ctx, const hfpx_gnn *net, hfpx_gnn_graph *graph, float *out_nodes,
                     float *out_edges);
/* Loss and the gradient of every parameter (layout of get_params), no update. */
int hfpx_gnn_gradients(hfpx_ctx *ctx, hfpx_gnn *net, hfpx_gnn_graph *graph, double *loss, float *grads);
/* `steps` Adam steps (learning rate lr) on one graph; losses (steps) may be null. */
int hfpx_gnn_train(hfpx_ctx *ctx, hfpx_gnn *net, hfpx_gnn_graph *graph, int steps, double lr, double *losses);

/* ---- stress: make_3dbem_stress_f_s, system_assembly.cpp:279-455.
 * dd is (6 n_el) x 3 nodal DD (row 6 e + node), pts 3 x n_pts, out n_pts x 6
 * [Sxx,Syy,Szz,Sxy,Sxz,Syz]; s_inf (6) is added.  Deterministic (no atomics). */
int hfpx_stress(hfpx_ctx *ctx, const hfpx_mesh *mesh, double shear_m, double poiss_r,
                int is_dd_local, const double *dd, const double *pts, int64_t n_pts,
                const double *s_inf, double *out);

/* ---- stress for many load cases at once (the batched workload's
 * postprocessing): the 6 n_pts x 18 n_el influence matrix of the points
 * (the blocks make_3dbem_stress_f_s sums, system_assembly.cpp:306-437) is
 * formed once on the device and applied to all cases with one FP64 GEMM.
 * dd: n_cases blocks of (6 n_el) x 3 as for hfpx_stress (block k at
 * dd + 18 n_el k); s_inf: 6 x n_cases; out: n_cases blocks of n_pts x 6.
 * n_cases == 1 runs hfpx_stress. */
int hfpx_stress_batch(hfpx_ctx *ctx, const hfpx_mesh *mesh, double shear_m, double poiss_r,
                      int is_dd_local, const double *dd, int64_t n_cases, const double *pts,
                      int64_t n_pts, const double *s_inf, double *out);

/* ---- the batched workload: many meshes of uneven sizes (no fixed DoF,
 * 18 DoF per element in the default numbering), each with many load cases,
 * assembled, factored and solved in one CUDA-graph launch.  Per mesh this is
 * the reference's make_3dbem_matrix_s (system_assembly.cpp:30-219),
 * add_s_inf_to_3dbem_rhs (:222-274) and il::LU factor + solve
 * (il/linear_algebra/dense/factorization/LU.h:79-120) once per load case.
 * The right-hand side is linear in the in-situ stress, so the 6 unit stress
 * states are solved to the tolerance and each load case is their
 * combination.  The operator of each mesh is held in mixed precision (FP32
 * entries, near-field blocks to about 2^-48, as hfpx_assemble_mixed); the
 * factorisation is FP32 with tournament-pivoted panels; the solutions are
 * refined in FP64 against the operator.  The meshes (hfpx_mesh_create) must
 * outlive the batch; at most 611 elements per mesh.  nb: block size (a
 * multiple of 32, <= 0: 128), leaf_rows: rows per panel chunk (256 or 512,
 * <= 0: 512); both are tile choices of the autotuner. */
typedef struct hfpx_batch hfpx_batch;
typedef struct {
  int64_t n_mesh;
  double residual;          /* max over meshes and unit states of |b - A x|_inf / |b|_inf */
  int converged;
  int64_t singular_mesh;    /* first mesh with a zero pivot, -1 none */
  int off_plane_pairs;      /* pairs evaluated by the off-plane path */
  int iterations;           /* most refinement corrections any mesh took */
} hfpx_batch_info;
int hfpx_batch_create(hfpx_ctx *ctx, int64_t n_mesh, const hfpx_mesh *const *meshes, double shear_m,
                      double poiss_r, int nb, int leaf_rows, hfpx_batch **batch);
/* Load cases: s_inf is 6 x n_cases per mesh (Voigt, tension positive),
 * mesh after mesh; each case's solution is the combination of the unit
 * states' solutions. */
int hfpx_batch_set_loads(hfpx_ctx *ctx, hfpx_batch *batch, const double *s_inf, int64_t n_cases);
/* One run: assembly, right-hand sides, factorisation, solves and FP64
 * refinement to |b - A x|_inf / |b|_inf <= tol (<= 0: 1e-10) in at most
 * max_iter steps (<= 0: 10), and the load cases' solutions, as one CUDA
 * graph (captured by the first run, replayed after). */
int hfpx_batch_run(hfpx_ctx *ctx, hfpx_batch *batch, double tol, int max_iter, hfpx_batch_info *info);
/* Mesh `mesh`'s solutions: n x n_cases (or n x 6 unit states without load
 * cases), column-major. */
int hfpx_batch_solution(hfpx_ctx *ctx, const hfpx_batch *batch, int64_t mesh, double *x);
/* Each mesh's final relative residual (n_mesh). */
int hfpx_batch_residuals(hfpx_ctx *ctx, const hfpx_batch *batch, double *res);
/* Launches of the factorisation's schedule (plus the fixed ones). */
int64_t hfpx_batch_launches(const hfpx_batch *batch);
/* Device times (ms) of the last run's phases: assembly with the right-hand
 * sides, factorisation, solves with refinement and the load cases. */
int hfpx_batch_phases(hfpx_ctx *ctx, const hfpx_batch *batch, double *ms);
int hfpx_batch_destroy(hfpx_batch *batch);

/* ---- the volume-control iteration with cohesion and friction:
 * vc_cf_iteration, src/Development/c_f_iteration.cpp:27-436, with match_f_c
 * and update_mrd (src/Development/cohesion_friction.cpp:22-130, :134-194).
 * The state is the reference's Mesh_Data_T solution part
 * (src/Core/surface_mesh_utilities.h:51-101), per collocation point
 * (n_cp = 6 n_el, point 6 el + local node): dd n_cp x 3 column-major (the
 * nodal DD), pp the nodal pressures, the Frac_State_T arrays and the
 * material ids; dof_h (n_el x 18, written by the iteration) is the
 * truncated DoF handle of the step, dof_h_dd.  Materials are the
 * reference's F_C_Param_T (model_parameters.h:22-31) with its contact
 * model ids (Properties_T::c_model_id(mat, 0 / 1)). */
typedef struct {
  double cr_open;      /* critical opening */
  double peak_ts;      /* peak tensile stress */
  double cr_slip;      /* critical slip */
  double peak_sc;      /* peak shear cohesion */
  double peak_sf;      /* peak friction coefficient */
  double res_sf;       /* residual friction coefficient */
  int cohesion_model;  /* 0 box (Dugdale), 1 linear weakening, other: none */
  int friction_model;  /* 0 constant (peak), 1 linear slip weakening, other: residual */
} hfpx_cf_material;

typedef struct {
  double *dd;                 /* n_cp x 3, ld n_cp (in/out) */
  double *pp;                 /* n_cp (in/out) */
  double *mr_open, *mr_slip;  /* max. relative opening / slip (in; update_mrd writes) */
  double *friction_coef, *slip_cohesion, *open_cohesion;  /* written by match_f_c */
  const int32_t *mat_id;      /* n_cp, 0 .. n_mat - 1 */
  int64_t *dof_h;             /* n_el x 18 column-major (out; may be null) */
} hfpx_cf_state;

typedef struct {
  double residual;    /* |increments|_1 + |traction adjustments|_1 (:430-433) */
  double volume;      /* crack volume before the step (the volume row times dd) */
  double pressure;    /* injection pressure after the step */
  double delta_p;     /* its increment */
  int64_t n_dof;      /* active DD unknowns of the step (dof_h_dd.n_dof) */
  int64_t n_fixed;    /* unknowns fixed at intact collocation points */
  int solver;         /* 0: solved with the full system's factors, 1: truncated system factored */
  int refinement;     /* refinement steps of the solve */
} hfpx_cf_info;

/* match_f_c on the device: cohesion and friction of every point from its
 * DD (read as local, as the reference reads them) and damage state. */
int hfpx_cf_match(hfpx_ctx *ctx, int64_t n_cp, const hfpx_cf_material *mats, int n_mat, hfpx_cf_state *state);
/* update_mrd on the device: the maximum relative opening and slip reached. */
int hfpx_cf_update_mrd(hfpx_ctx *ctx, int64_t n_cp, const hfpx_cf_material *mats, int n_mat,
                       hfpx_cf_state *state);
/* One iteration: match_f_c, the elastic tractions of the current DD (one
 * product with the bordered matrix, whose volume row gives the volume),
 * per point the traction check (opening, cohesion, slip, intact) and the
 * traction adjustments, the truncated system (the DoF of intact points
 * fixed; mod_3dbem_system_vc, system_assembly.cpp:560-629) solved for the
 * DD increments and the pressure increment that injects new_vol, then the
 * DD (negative openings clamped) and the pressures of opened points.
 * `matrix` is the bordered matrix of orig_dof_h (make_3dbem_matrix_vc,
 * n_dof + 1 unknowns): unfactored, or factored with HFPX_LU_MIXED, which
 * keeps the operator.  With mixed factors and few fixed DoF (k + 1 <
 * 0.02 n_keep^3 / n^2, where the k + 1 refined solves cost less than a new
 * factorisation) the step reuses them (hfpx_lu_solve_fixed); otherwise it
 * factors the truncated system (hfpx_matrix_truncate, HFPX_LU_MIXED);
 * flags bit 2 reuses the mixed factors whenever there are any (k <= 4096).  inj_cp is the
 * injection point (6 el + node, load.inj_loc(0, 0..1)).  flags bit 0: add
 * all three components of the traction adjustments to the right-hand side
 * (the reference adds the first two, :262-268); bit 1: add them with the
 * opposite sign.  The reference's sign adds A dd = dt with dt = -(excess
 * traction) to the traction A dd it subtracts, which doubles the excess,
 * and its iteration grows; with bit 1 the excess is removed and the
 * iteration settles.  Where the reference's
 * statements disagree with each other the engine takes one reading:
 * DoF renumbering in element order (the reference's shared counter races
 * under OpenMP), DoF untouched by the checks stay active, tractions and the
 * volume from the original numbering, the clamped DD left in local
 * coordinates.  HFPX_ERR_SINGULAR when every DoF is fixed.  The call
 * allocates its O(n) device buffers (and, on the truncated path, the
 * truncated matrix) per step and returns with the stream synchronised. */
int hfpx_vc_cf_iteration(hfpx_ctx *ctx, const hfpx_mesh *mesh, const hfpx_matrix *matrix,
                         const int64_t *orig_dof_h, int64_t n_dof, const hfpx_cf_material *mats, int n_mat,
                         const double *s_inf, int64_t inj_cp, double new_vol, int is_dd_local, int flags,
                         double tol, hfpx_cf_state *state, hfpx_cf_info *info);

/* ---- one element at one point: make_local_3dbem_submatrix,
 * src/Elasticity/elasticity_kernel_integration.cpp:34-205 (kernel 1).
 * tau: 3 complex (re,im), sfm: 6x6 complex row-major (re,im); out 6x18
 * row-major local stress influence.  Runs the device kernel once. */
int hfpx_local_submatrix(hfpx_ctx *ctx, double shear_m, double poiss_r, double h, double zr,
                         double zi, const double *tau, const double *sfm, double *out);

/* ---- element frame on the host (same arithmetic as the device precompute):
 * make_el_sfm_uniform + make_el_tau_crd, element_utilities.cpp:89-238.
 * vert[k + 3 j] = coordinate k of vertex j; r row-major 3x3. */
int hfpx_element_frame(const double *vert, double *r, double *tau, double *sfm);

#ifdef __cplusplus
}
#endif
#endif
