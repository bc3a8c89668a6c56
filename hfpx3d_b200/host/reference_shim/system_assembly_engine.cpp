// Engine-backed replacement for the reference's src/Solvers/system_assembly.cpp.
// It defines the same functions with the same signatures
// (src/Solvers/system_assembly.h:35-63) against the reference's own headers and
// il:: types, and hands the work to libhfpx_engine.so through its C-ABI
// (include/hfpx_engine.h).  Linked in place of system_assembly.cpp (and,
// for il::LU, with libhfpx_lapacke.so ahead of OpenBLAS), it puts the
// reference's main.cpp -- or any other caller of these functions -- on the GPU
// without a change to its source.
//
// Argument checks follow the reference: its IL_EXPECT_FAST preconditions
// (system_assembly.cpp:39-42, 287-290, 468-471) and every engine error abort
// with a message.  There is no CPU fallback.
//
// mod_3dbem_system_vc (system_assembly.cpp:560-629) is defined for the
// bordered matrix its one caller passes (Development/c_f_iteration.cpp:285):
// the reference version requires an orig_ndof-square matrix and then reads
// its border one row past the end; here the border is the bordered matrix's
// own last row and column, gathered on the device (hfpx_matrix_truncate).
//
//   HFPX_DEVICE   GPU to use (default 0)
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include <il/Array.h>
#include <il/Array2D.h>

#include "hfpx_engine.h"
#include "src/Solvers/system_assembly.h"

namespace {

hfpx_ctx* ctx() {
  static hfpx_ctx* c = [] {
    const char* e = std::getenv("HFPX_DEVICE");
    hfpx_ctx* p = nullptr;
    const int rc = hfpx_ctx_create(e ? std::atoi(e) : 0, &p);
    if (rc != HFPX_OK) {
      std::fprintf(stderr, "hfpx system_assembly: no engine context (status %d)\n", rc);
      std::abort();
    }
    return p;
  }();
  return c;
}

void check(int rc, const char* what) {
  if (rc == HFPX_OK) return;
  std::fprintf(stderr, "hfpx system_assembly: %s: %s (status %d)\n", what, hfpx_ctx_last_error(ctx()), rc);
  std::abort();
}

void expect(bool cond, const char* what) {
  if (cond) return;
  std::fprintf(stderr, "hfpx system_assembly: precondition failed: %s\n", what);
  std::abort();
}

// il::Array2D keeps its columns stride(1) = capacity(0) apart.  The engine's
// dof_h, dd and point arrays have no leading dimension of their own (columns
// size(0) apart); this gives such a view, packing only when the two differ.
template <typename T>
class Packed {
 public:
  explicit Packed(const il::Array2D<T>& a) : p_(a.data()) {
    const il::int_t n0 = a.size(0), n1 = a.size(1), ld = a.stride(1);
    if (ld == n0 || n1 <= 1) return;
    buf_.resize((size_t)(n0 * n1));
    for (il::int_t j = 0; j < n1; ++j)
      for (il::int_t i = 0; i < n0; ++i) buf_[(size_t)(i + n0 * j)] = a(i, j);
    p_ = buf_.data();
  }
  const T* get() const { return p_; }

 private:
  const T* p_;
  std::vector<T> buf_;
};

// The mesh on the device for the duration of one call.  nods and conn go in
// with their own leading dimensions (3 x n_nodes and >= 3 x n_el; the rows
// past the third, as in the reference, are ignored).
class DeviceMesh {
 public:
  DeviceMesh(const hfp3d::Mesh_Geom_T& m, double beta) {
    static_assert(sizeof(il::int_t) == sizeof(int64_t), "il::int_t is the engine's int64_t");
    check(hfpx_mesh_create(ctx(), m.nods.data(), m.nods.stride(1), m.nods.size(1),
                           reinterpret_cast<const int64_t*>(m.conn.data()), m.conn.stride(1), m.conn.size(1),
                           beta, &h_),
          "mesh upload");
  }
  ~DeviceMesh() { hfpx_mesh_destroy(h_); }
  DeviceMesh(const DeviceMesh&) = delete;
  DeviceMesh& operator=(const DeviceMesh&) = delete;
  const hfpx_mesh* get() const { return h_; }

 private:
  hfpx_mesh* h_ = nullptr;
};

void expect_mesh(const hfp3d::Mesh_Geom_T& mesh) {
  expect(mesh.conn.size(0) >= 3, "mesh.conn.size(0) >= 3");
  expect(mesh.conn.size(1) >= 1, "mesh.conn.size(1) >= 1");
  expect(mesh.nods.size(0) >= 3, "mesh.nods.size(0) >= 3");
  expect(mesh.nods.size(1) >= 3, "mesh.nods.size(1) >= 3");
}

// make_3dbem_matrix_s / _vc (system_assembly.cpp:30-219, 458-557): the
// matrix is formed on the device and returned on the host, as the reference
// returns it.  vc adds the volume row and pressure column; the corner stays 0.
il::Array2D<double> host_matrix(double shear_m, double poiss_r, const hfp3d::Mesh_Geom_T& mesh,
                                const hfp3d::Num_Param_T& n_par, hfp3d::DoF_Handle_T& dof_hndl, bool vc) {
  expect_mesh(mesh);
  if (dof_hndl.n_dof == 0 || dof_hndl.dof_h.size(0) == 0)
    dof_hndl = hfp3d::make_dof_h_crack(mesh, 2, n_par.tip_type);
  expect(dof_hndl.dof_h.size(0) == mesh.conn.size(1) && dof_hndl.dof_h.size(1) == 18,
         "dof_hndl.dof_h is n_el x 18");
  DeviceMesh dm(mesh, n_par.beta);
  Packed<il::int_t> dof(dof_hndl.dof_h);
  const il::int_t n = dof_hndl.n_dof + (vc ? 1 : 0);
  hfpx_matrix* a = nullptr;
  check(hfpx_assemble(ctx(), dm.get(), reinterpret_cast<const int64_t*>(dof.get()), dof_hndl.n_dof, shear_m,
                      poiss_r, n_par.is_dd_local ? 1 : 0, vc ? 1 : 0, &a),
        "assembly");
  il::Array2D<double> out{n, n};
  const int rc = hfpx_matrix_download(ctx(), a, out.data(), out.stride(1));
  hfpx_matrix_destroy(a);
  check(rc, "matrix download");
  return out;
}

}  // namespace

namespace hfp3d {

il::Array2D<double> make_3dbem_matrix_s(double shear_m, double poiss_r, const Mesh_Geom_T& mesh,
                                        const Num_Param_T& n_par, il::io_t, DoF_Handle_T& dof_hndl) {
  return host_matrix(shear_m, poiss_r, mesh, n_par, dof_hndl, false);
}

il::Array2D<double> make_3dbem_matrix_vc(double shear_m, double poiss_r, const Mesh_Geom_T& mesh,
                                         const Num_Param_T& n_par, il::io_t, DoF_Handle_T& dof_hndl) {
  return host_matrix(shear_m, poiss_r, mesh, n_par, dof_hndl, true);
}

// add_s_inf_to_3dbem_rhs (system_assembly.cpp:222-274): sae.rhs_v is reset
// to zeros when its size is not n_dof, then rhs[dof] -= (n . s_inf)_l.
void add_s_inf_to_3dbem_rhs(const Mesh_Data_T& mesh_data, const Load_T& load, il::io_t, SAE_T& sae) {
  const il::int_t n_dof = mesh_data.dof_h_dd.n_dof;
  if (sae.rhs_v.size() != n_dof) sae.rhs_v = il::Array<double>{n_dof, 0.0};
  if (n_dof == 0) return;
  expect(mesh_data.dof_h_dd.dof_h.size(0) == mesh_data.mesh.conn.size(1), "dof_h_dd.dof_h is n_el x 18");
  DeviceMesh dm(mesh_data.mesh, 0.125);  // the collocation offset does not enter the normals
  Packed<il::int_t> dof(mesh_data.dof_h_dd.dof_h);
  double s_inf[6];
  for (int k = 0; k < 6; ++k) s_inf[k] = load.s_inf[k];
  check(hfpx_rhs_sinf(ctx(), dm.get(), reinterpret_cast<const int64_t*>(dof.get()), n_dof, s_inf, 1,
                      sae.rhs_v.data(), n_dof),
        "right-hand side");
}

// make_3dbem_stress_f_s (system_assembly.cpp:279-455): stresses at the points
// m_pts_crd (3 x n_pts) from the nodal DD m_data.dd ((6 n_el) x 3), plus s_inf.
il::Array2D<double> make_3dbem_stress_f_s(double shear_m, double poiss_r, const Mesh_Data_T& m_data,
                                          const Load_T& load, const Num_Param_T& n_par,
                                          const il::Array2D<double>& m_pts_crd) {
  expect_mesh(m_data.mesh);
  const il::int_t n_el = m_data.mesh.conn.size(1);
  const il::int_t n_pts = m_pts_crd.size(1);
  expect(m_data.dd.size(0) == 6 * n_el && m_data.dd.size(1) == 3, "m_data.dd is (6 n_el) x 3");
  expect(m_pts_crd.size(0) >= 3, "m_pts_crd.size(0) >= 3");
  il::Array2D<double> out{n_pts, 6, 0.0};
  if (n_pts == 0) return out;
  DeviceMesh dm(m_data.mesh, n_par.beta);
  Packed<double> dd(m_data.dd);
  // the engine reads the points as packed xyz triples
  std::vector<double> pts((size_t)(3 * n_pts));
  for (il::int_t p = 0; p < n_pts; ++p)
    for (int k = 0; k < 3; ++k) pts[(size_t)(3 * p + k)] = m_pts_crd(k, p);
  double s_inf[6];
  for (int k = 0; k < 6; ++k) s_inf[k] = load.s_inf[k];
  std::vector<double> res((size_t)(6 * n_pts));
  check(hfpx_stress(ctx(), dm.get(), shear_m, poiss_r, n_par.is_dd_local ? 1 : 0, dd.get(), pts.data(), n_pts,
                    s_inf, res.data()),
        "stress");
  for (int j = 0; j < 6; ++j)
    for (il::int_t p = 0; p < n_pts; ++p) out(p, j) = res[(size_t)(p + n_pts * j)];
  return out;
}

// mod_3dbem_system_vc (system_assembly.cpp:560-629): the truncated bordered
// system of the DoF that dof_hndl keeps (dof_h >= 0), from orig_matrix, the
// (orig_ndof + 1)-square matrix make_3dbem_matrix_vc returns for
// orig_dof_hndl.  The corner stays 0 as the reference leaves it; delta_t is
// indexed by the full element-node, the original or the truncated numbering,
// told apart by its size as there; delta_v is the last right-hand side entry.
SAE_T mod_3dbem_system_vc(const il::Array2D<double>& orig_matrix, const DoF_Handle_T& orig_dof_hndl,
                          const DoF_Handle_T& dof_hndl, const il::Array<double>& delta_t, const double delta_v) {
  expect(orig_matrix.size(0) == orig_matrix.size(1), "orig_matrix.size(0) == orig_matrix.size(1)");
  const il::int_t num_of_ele = orig_dof_hndl.dof_h.size(0);
  const il::int_t ndpe = orig_dof_hndl.dof_h.size(1);
  expect(num_of_ele > 0, "num_of_ele > 0");
  const il::int_t full_ndof = num_of_ele * ndpe;
  const il::int_t orig_ndof = orig_dof_hndl.n_dof;
  expect(orig_ndof > 0 && orig_ndof <= full_ndof, "orig_ndof > 0 && orig_ndof <= full_ndof");
  expect(orig_ndof + 1 == orig_matrix.size(0), "orig_matrix is the bordered matrix (orig_ndof + 1 square)");
  const il::int_t used_ndof = dof_hndl.n_dof;
  expect(used_ndof > 0 && used_ndof <= orig_ndof, "used_ndof > 0 && used_ndof <= orig_ndof");
  expect(dof_hndl.dof_h.size(0) == num_of_ele && dof_hndl.dof_h.size(1) == ndpe, "dof_hndl matches orig_dof_hndl");
  const il::int_t tsize = delta_t.size();
  expect(tsize == full_ndof || tsize == orig_ndof || tsize == used_ndof, "delta_t size");
  std::vector<int64_t> keep((size_t)used_ndof, -1);
  SAE_T sys;
  sys.rhs_v = il::Array<double>{used_ndof + 1, 0.0};
  sys.rhs_v[used_ndof] = delta_v;
  for (il::int_t e = 0; e < num_of_ele; ++e)
    for (il::int_t j = 0; j < ndpe; ++j) {
      const il::int_t t = dof_hndl.dof_h(e, j);
      if (t < 0) continue;
      expect(t < used_ndof && keep[(size_t)t] < 0, "each truncated DoF at one element node");
      const il::int_t o = orig_dof_hndl.dof_h(e, j);
      expect(o >= 0 && o < orig_ndof, "a truncated DoF has an original DoF");
      keep[(size_t)t] = o;
      sys.rhs_v[t] = tsize == full_ndof ? delta_t[e * ndpe + j] : (tsize == orig_ndof ? delta_t[o] : delta_t[t]);
    }
  for (int64_t o : keep) expect(o >= 0, "the truncated numbering has no gaps");
  hfpx_matrix *a = nullptr, *t = nullptr;
  check(hfpx_matrix_upload(ctx(), orig_matrix.data(), orig_matrix.size(0), orig_matrix.stride(1), &a),
        "matrix upload");
  const int rc = hfpx_matrix_truncate(ctx(), a, keep.data(), used_ndof, 1, &t);
  hfpx_matrix_destroy(a);
  check(rc, "truncation");
  sys.matrix = il::Array2D<double>{used_ndof + 1, used_ndof + 1};
  const int rc2 = hfpx_matrix_download(ctx(), t, sys.matrix.data(), sys.matrix.stride(1));
  hfpx_matrix_destroy(t);
  check(rc2, "matrix download");
  return sys;
}

}  // namespace hfp3d
