// Test infrastructure only: the reference's CPU path, run and timed the way
// its own main.cpp runs and times it, for bench.py's CPU-baseline leg and its
// reference arm.  Compiled by oracle/Makefile (target cpu) into
// oracle/_ref/libhfpx_ref_cpu.so from the reference's sources where they lie,
// with OpenMP (as the reference's CMakeLists.txt builds it) and linked to the
// OpenBLAS build bundled with scipy, the LAPACK the reference's il::LU calls
// (il/linear_algebra/dense/factorization/LU.h:87, 115).  Nothing in the
// product links or loads it.
//
//   "Assembly" (main.cpp:89-124): make_dof_h_crack, make_3dbem_matrix_s (or
//       make_3dbem_matrix_vc with the never-written corner set to 0) and
//       add_s_inf_to_3dbem_rhs;
//   "Solution" (main.cpp:150-175): il::LU of the matrix and lu.solve(rhs).
//       main.cpp hands il::LU a copy of the matrix; here it is moved in, so
//       the timer covers the factorisation and the solve only.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <il/Array.h>
#include <il/Array2D.h>
#include <il/linear_algebra/dense/factorization/LU.h>
#include "src/Core/model_parameters.h"
#include "src/Core/surface_mesh_utilities.h"
#include "src/Solvers/system_assembly.h"

namespace {

hfp3d::Mesh_Geom_T mesh_of(const double* nods, int64_t ld_nods, int64_t n_nodes, const int64_t* conn,
                           int64_t ld_conn, int64_t n_el) {
  hfp3d::Mesh_Geom_T m;
  m.nods = il::Array2D<double>{(il::int_t)ld_nods, (il::int_t)n_nodes, 0.0};
  for (int64_t j = 0; j < n_nodes; ++j)
    for (int64_t i = 0; i < ld_nods; ++i) m.nods(i, j) = nods[i + ld_nods * j];
  m.conn = il::Array2D<il::int_t>{(il::int_t)ld_conn, (il::int_t)n_el, 0};
  for (int64_t j = 0; j < n_el; ++j)
    for (int64_t i = 0; i < ld_conn; ++i) m.conn(i, j) = conn[i + ld_conn * j];
  return m;
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

extern "C" {

// One assembly + solve of the reference on a mesh (tip_type 0, global DD).
// vc != 0: the volume-control bordered system with injected volume `volume`.
// x (optional): the solution, n_dof (+1 with vc) entries.  Returns 0, or
// 1 + the singular column reported by il::LU.
int ref_cpu_path(const double* nods, int64_t ld_nods, int64_t n_nodes, const int64_t* conn, int64_t ld_conn,
                 int64_t n_el, double G, double nu, double beta, int vc, const double* s_inf, double volume,
                 double* t_assembly, double* t_solution, double* x, int64_t* n_out) {
  hfp3d::Mesh_Data_T md;
  md.mesh = mesh_of(nods, ld_nods, n_nodes, conn, ld_conn, n_el);
  hfp3d::Num_Param_T np;
  np.beta = beta;
  np.tip_type = 0;
  np.is_dd_local = false;
  hfp3d::Load_T load;
  for (int k = 0; k < 6; ++k) load.s_inf[k] = s_inf[k];

  auto t0 = std::chrono::steady_clock::now();
  md.dof_h_dd = hfp3d::make_dof_h_crack(md.mesh, 2, np.tip_type);
  hfp3d::SAE_T sae;
  sae.matrix = vc ? hfp3d::make_3dbem_matrix_vc(G, nu, md.mesh, np, il::io, md.dof_h_dd)
                  : hfp3d::make_3dbem_matrix_s(G, nu, md.mesh, np, il::io, md.dof_h_dd);
  sae.n_dof = md.dof_h_dd.n_dof;
  sae.rhs_v = il::Array<double>{sae.n_dof, 0.0};
  hfp3d::add_s_inf_to_3dbem_rhs(md, load, il::io, sae);
  const il::int_t n = sae.matrix.size(0);
  il::Array<double> rhs{n, 0.0};
  for (il::int_t i = 0; i < sae.n_dof; ++i) rhs[i] = sae.rhs_v[i];
  if (vc) {
    sae.matrix(n - 1, n - 1) = 0.0;
    rhs[n - 1] = volume;
  }
  *t_assembly = seconds_since(t0);

  t0 = std::chrono::steady_clock::now();
  il::Status status{};
  il::LU<il::Array2D<double>> lu(std::move(sae.matrix), il::io, status);
  if (!status.ok()) {
    const int64_t r = status.toInteger("rank");
    *t_solution = seconds_since(t0);
    return (int)(1 + r);
  }
  il::Array<double> sol = lu.solve(rhs);
  *t_solution = seconds_since(t0);
  *n_out = n;
  if (x) std::memcpy(x, sol.data(), sizeof(double) * n);
  return 0;
}

}  // extern "C"
