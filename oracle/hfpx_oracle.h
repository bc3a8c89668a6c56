/* Test infrastructure: CPU oracle for the HFPx3D assembly -> solve -> stress path.
 *
 * A plain-C restatement of the reference's algorithm, used only by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker.  The
 * product never links it.  It is pinned against the reference compiled from
 * its own sources (oracle/_ref, see oracle/Makefile) and against the reference's
 * MATLAB golden vectors (tests/golden/).
 *
 * Layouts (identical to the C-ABI in include/hfpx_engine.h):
 *   nods   ld_nods x n_nodes, column-major (rows 0..2 coordinates, rows 3..4 tip flags)
 *   conn   ld_conn x n_el, column-major, int64, 0-based
 *   dof_h  n_el x 18, column-major, int64, -1 = fixed DoF
 *   matrix n x n, column-major, leading dimension ld
 */
#ifndef HFPX_ORACLE_H
#define HFPX_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Element frame: rows e1,e2,e3 (row-major 3x3), vertex tau coordinates
 * (3 complex as re,im pairs) and shape-function matrix (6x6 complex, row-major,
 * re,im pairs).  vert[k + 3*j] = coordinate k of vertex j. */
void ora_element_frame(const double *vert, double *r, double *tau, double *sfm);

/* (h, z) of a point in an element's local frame. */
void ora_pt_hz(const double *vert, const double *pt, double *h, double *zr, double *zi);

/* 6x18 local stress-influence block (row-major) of an element at a point (h, z). */
void ora_local_block(double G, double nu, double h, double zr, double zi,
                     const double *tau, const double *sfm, double *out);

/* DoF handle for a crack mesh; returns n_dof. */
int64_t ora_dof_handle(const double *nods, int64_t ld_nods, int64_t n_nodes,
                       const int64_t *conn, int64_t ld_conn, int64_t n_el,
                       int tip_type, int64_t *dof_h);

/* Dense collocation matrix (vc != 0 adds the volume-control row/column and a
 * zero corner).  out has n = n_dof (+1) rows and leading dimension ld. */
int ora_assemble(const double *nods, int64_t ld_nods, int64_t n_nodes,
                 const int64_t *conn, int64_t ld_conn, int64_t n_el,
                 const int64_t *dof_h, int64_t n_dof,
                 double G, double nu, double beta, int is_dd_local, int vc,
                 double *out, int64_t ld);

/* Same matrix restricted to target elements [t0, t1): rows of those elements
 * only, written into a full-size column-major buffer (for sampled timing). */
int ora_assemble_rows(const double *nods, int64_t ld_nods, int64_t n_nodes,
                      const int64_t *conn, int64_t ld_conn, int64_t n_el,
                      const int64_t *dof_h, int64_t n_dof,
                      double G, double nu, double beta, int is_dd_local,
                      int64_t t0, int64_t t1, double *out, int64_t ld);

/* rhs[dof] -= (n . s_inf)_l over all collocation points; rhs has n_dof entries. */
void ora_rhs(const double *nods, int64_t ld_nods, const int64_t *conn, int64_t ld_conn,
             int64_t n_el, const int64_t *dof_h, const double *s_inf, double *rhs);

/* Stress at points; dd is (6 n_el) x 3 column-major, pts 3 x n_pts column-major,
 * out n_pts x 6 column-major [Sxx,Syy,Szz,Sxy,Sxz,Syz]. */
void ora_stress(const double *nods, int64_t ld_nods, const int64_t *conn, int64_t ld_conn,
                int64_t n_el, double G, double nu, int is_dd_local, const double *dd,
                const double *pts, int64_t n_pts, const double *s_inf, double *out);

/* Nodal DD array (6 n_el) x 3 column-major from a solution vector. */
void ora_dd_from_solution(const double *sol, const int64_t *dof_h, int64_t n_el, double *dd);

/* Sneddon's penny-shaped crack: opening and full stress field at a point. */
void ora_sneddon_dd(double G, double nu, double a, double p, const double *x, double *dd);
void ora_sneddon_stress(double G, double nu, double a, double p, const double *x, double *s);

#ifdef __cplusplus
}
#endif
#endif
