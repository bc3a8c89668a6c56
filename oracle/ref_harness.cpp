// Test infrastructure only: a C-ABI wrapper around the reference HFPx3D
// sources, compiled by oracle/Makefile into oracle/_ref/libhfpx_ref.so.
// It is the pinned checker for the CPU restatement in oracle/hfpx_oracle.c
// and for the golden fixtures under tests/golden/.  Nothing in the product
// links or loads it.
//
// Every function copies plain column-major arrays into the reference's
// il:: containers, calls the reference function named in its comment and
// copies the result back out.  Layout conventions:
//   nods : ld_nods x n_nodes column-major (rows 0..2 = x,y,z; rows 3,4 tip flags)
//   conn : ld_conn x n_el    column-major, int64, 0-based node indices
//   dof_h: n_el x 18         column-major, int64 (-1 = fixed DoF)
//   matrices: column-major with leading dimension = row count.

#include <complex>
#include <cstdint>
#include <cstring>
#include <il/Array.h>
#include <il/Array2D.h>
#include <il/StaticArray.h>
#include <il/StaticArray2D.h>
#include "src/Core/element_utilities.h"
#include "src/Core/surface_mesh_utilities.h"
#include "src/Core/model_parameters.h"
#include "src/Elasticity/elasticity_kernel_integration.h"
#include "src/Elasticity/h_potential.h"
#include "src/Solvers/system_assembly.h"

namespace {

hfp3d::Mesh_Geom_T make_mesh(const double* nods, int64_t ld_nods, int64_t n_nodes,
                             const int64_t* conn, int64_t ld_conn, int64_t n_el) {
  hfp3d::Mesh_Geom_T m;
  m.nods = il::Array2D<double>{(il::int_t)ld_nods, (il::int_t)n_nodes, 0.0};
  for (int64_t j = 0; j < n_nodes; ++j)
    for (int64_t i = 0; i < ld_nods; ++i) m.nods(i, j) = nods[i + ld_nods * j];
  m.conn = il::Array2D<il::int_t>{(il::int_t)ld_conn, (il::int_t)n_el, 0};
  for (int64_t j = 0; j < n_el; ++j)
    for (int64_t i = 0; i < ld_conn; ++i) m.conn(i, j) = conn[i + ld_conn * j];
  return m;
}

il::StaticArray2D<double, 3, 3> vert33(const double* v) {
  il::StaticArray2D<double, 3, 3> a;
  for (int j = 0; j < 3; ++j)
    for (int k = 0; k < 3; ++k) a(k, j) = v[k + 3 * j];
  return a;
}

void copy_dof(const hfp3d::DoF_Handle_T& d, int64_t n_el, int64_t* dof_h) {
  for (int64_t j = 0; j < 18; ++j)
    for (int64_t e = 0; e < n_el; ++e) dof_h[e + n_el * j] = d.dof_h(e, j);
}

}  // namespace

extern "C" {

// element_utilities.cpp: make_el_sfm_uniform + make_el_tau_crd.
// r_out: 3x3 row-major (rows e1,e2,e3); tau_out: 3 complex as (re,im);
// sfm_out: 6x6 complex row-major as (re,im) pairs.
int ref_element_frame(const double* vert, double* r_out, double* tau_out, double* sfm_out) {
  il::StaticArray2D<double, 3, 3> v = vert33(vert), r;
  il::StaticArray2D<std::complex<double>, 6, 6> sfm = hfp3d::make_el_sfm_uniform(v, il::io, r);
  il::StaticArray<std::complex<double>, 3> tau = hfp3d::make_el_tau_crd(v, r);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r_out[3 * i + j] = r(i, j);
  for (int i = 0; i < 3; ++i) { tau_out[2 * i] = tau[i].real(); tau_out[2 * i + 1] = tau[i].imag(); }
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      sfm_out[2 * (6 * i + j)] = sfm(i, j).real();
      sfm_out[2 * (6 * i + j) + 1] = sfm(i, j).imag();
    }
  return 0;
}

// element_utilities.cpp: make_el_pt_hz.
int ref_pt_hz(const double* vert, const double* pt, double* h, double* zr, double* zi) {
  il::StaticArray2D<double, 3, 3> v = vert33(vert);
  il::StaticArray2D<double, 3, 3> r = hfp3d::make_el_r_tensor(v);
  il::StaticArray<double, 3> p;
  for (int k = 0; k < 3; ++k) p[k] = pt[k];
  hfp3d::HZ hz = hfp3d::make_el_pt_hz(v, p, r);
  *h = hz.h; *zr = hz.z.real(); *zi = hz.z.imag();
  return 0;
}

// elasticity_kernel_integration.cpp: make_local_3dbem_submatrix (kernel 1).
// out: 6x18 row-major.
int ref_local_submatrix(double G, double nu, double h, double zr, double zi,
                        const double* tau, const double* sfm, double* out) {
  il::StaticArray<std::complex<double>, 3> t;
  for (int i = 0; i < 3; ++i) t[i] = std::complex<double>(tau[2 * i], tau[2 * i + 1]);
  il::StaticArray2D<std::complex<double>, 6, 6> s;
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j)
      s(i, j) = std::complex<double>(sfm[2 * (6 * i + j)], sfm[2 * (6 * i + j) + 1]);
  il::StaticArray2D<double, 6, 18> m =
      hfp3d::make_local_3dbem_submatrix(1, G, nu, h, std::complex<double>(zr, zi), t, s);
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 18; ++j) out[18 * i + j] = m(i, j);
  return 0;
}

// h_potential.cpp: s_ij_lim_h.  out: 6x4x3 complex, index ((j*4+c)*3+k), (re,im).
int ref_s_ij_lim(double nu, double eix_re, double eix_im, double d_re, double d_im, double* out) {
  il::StaticArray3D<std::complex<double>, 6, 4, 3> c =
      hfp3d::s_ij_lim_h(nu, std::complex<double>(eix_re, eix_im), std::complex<double>(d_re, d_im));
  for (int j = 0; j < 6; ++j)
    for (int a = 0; a < 4; ++a)
      for (int k = 0; k < 3; ++k) {
        int q = (j * 4 + a) * 3 + k;
        out[2 * q] = c(j, a, k).real();
        out[2 * q + 1] = c(j, a, k).imag();
      }
  return 0;
}

// surface_mesh_utilities.cpp: make_dof_h_crack (approximation order 2).
int64_t ref_dof_handle(const double* nods, int64_t ld_nods, int64_t n_nodes,
                       const int64_t* conn, int64_t ld_conn, int64_t n_el,
                       int tip_type, int64_t* dof_h) {
  hfp3d::Mesh_Geom_T m = make_mesh(nods, ld_nods, n_nodes, conn, ld_conn, n_el);
  hfp3d::DoF_Handle_T d = hfp3d::make_dof_h_crack(m, 2, tip_type);
  copy_dof(d, n_el, dof_h);
  return d.n_dof;
}

// system_assembly.cpp: make_3dbem_matrix_s (vc == 0) or make_3dbem_matrix_vc
// (vc != 0; the never-written corner entry is set to 0 here).
// out: n x n column-major with n = n_dof (+1 when vc).
int ref_assemble(const double* nods, int64_t ld_nods, int64_t n_nodes,
                 const int64_t* conn, int64_t ld_conn, int64_t n_el,
                 double G, double nu, double beta, int tip_type, int is_dd_local, int vc,
                 double* out, int64_t* dof_h, int64_t* n_dof) {
  hfp3d::Mesh_Geom_T m = make_mesh(nods, ld_nods, n_nodes, conn, ld_conn, n_el);
  hfp3d::Num_Param_T np;
  np.beta = beta; np.tip_type = tip_type; np.is_dd_local = (is_dd_local != 0);
  hfp3d::DoF_Handle_T d = hfp3d::make_dof_h_crack(m, 2, tip_type);
  il::Array2D<double> a = vc ? hfp3d::make_3dbem_matrix_vc(G, nu, m, np, il::io, d)
                             : hfp3d::make_3dbem_matrix_s(G, nu, m, np, il::io, d);
  const int64_t n = a.size(0);
  if (vc) a(n - 1, n - 1) = 0.0;
  for (int64_t j = 0; j < n; ++j) std::memcpy(out + n * j, &a(0, j), sizeof(double) * n);
  copy_dof(d, n_el, dof_h);
  *n_dof = d.n_dof;
  return 0;
}

// system_assembly.cpp: add_s_inf_to_3dbem_rhs.  rhs has n_dof entries, zeroed first.
int ref_rhs(const double* nods, int64_t ld_nods, int64_t n_nodes,
            const int64_t* conn, int64_t ld_conn, int64_t n_el,
            int tip_type, const double* s_inf, double* rhs) {
  hfp3d::Mesh_Data_T md;
  md.mesh = make_mesh(nods, ld_nods, n_nodes, conn, ld_conn, n_el);
  md.dof_h_dd = hfp3d::make_dof_h_crack(md.mesh, 2, tip_type);
  hfp3d::Load_T load;
  for (int k = 0; k < 6; ++k) load.s_inf[k] = s_inf[k];
  hfp3d::SAE_T sae;
  sae.rhs_v = il::Array<double>{md.dof_h_dd.n_dof, 0.0};
  hfp3d::add_s_inf_to_3dbem_rhs(md, load, il::io, sae);
  for (il::int_t i = 0; i < md.dof_h_dd.n_dof; ++i) rhs[i] = sae.rhs_v[i];
  return 0;
}

// system_assembly.cpp: make_3dbem_stress_f_s.
// dd: (6 n_el) x 3 column-major nodal DD; pts: 3 x n_pts column-major;
// out: n_pts x 6 column-major [Sxx,Syy,Szz,Sxy,Sxz,Syz].
int ref_stress(const double* nods, int64_t ld_nods, int64_t n_nodes,
               const int64_t* conn, int64_t ld_conn, int64_t n_el,
               double G, double nu, int is_dd_local, const double* dd,
               const double* pts, int64_t n_pts, const double* s_inf, double* out) {
  hfp3d::Mesh_Data_T md;
  md.mesh = make_mesh(nods, ld_nods, n_nodes, conn, ld_conn, n_el);
  md.dd = il::Array2D<double>{(il::int_t)(6 * n_el), 3, 0.0};
  for (int64_t j = 0; j < 3; ++j)
    for (int64_t i = 0; i < 6 * n_el; ++i) md.dd(i, j) = dd[i + 6 * n_el * j];
  hfp3d::Load_T load;
  for (int k = 0; k < 6; ++k) load.s_inf[k] = s_inf[k];
  hfp3d::Num_Param_T np;
  np.is_dd_local = (is_dd_local != 0);
  il::Array2D<double> p{3, (il::int_t)n_pts, 0.0};
  for (int64_t j = 0; j < n_pts; ++j)
    for (int64_t i = 0; i < 3; ++i) p(i, j) = pts[i + 3 * j];
  il::Array2D<double> s = hfp3d::make_3dbem_stress_f_s(G, nu, md, load, np, p);
  for (int64_t j = 0; j < 6; ++j)
    for (int64_t i = 0; i < n_pts; ++i) out[i + n_pts * j] = s(i, j);
  return 0;
}

}  // extern "C"
