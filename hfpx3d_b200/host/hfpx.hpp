// C++ host layer over the engine's C-ABI (include/hfpx_engine.h), mirroring
// the reference's call surface for the assembly -> solve -> stress path:
// the model structs of src/Core/model_parameters.h and
// src/Core/surface_mesh_utilities.h, and the functions of
// src/Solvers/system_assembly.h:35-71, il::LU (LU.h:46-61), and the IO of
// src/IO/ that main.cpp uses.  Same names and argument meaning; arrays are
// column-major (element (i, j) at data[i + j * size(0)], as il::Array2D).
// Errors throw hfpx::Error (the reference aborts).
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/hfpx_engine.h"

namespace hfpx {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

template <class T>
class Array2D {
 public:
  Array2D() = default;
  Array2D(int64_t n0, int64_t n1, T v = T()) : n0_(n0), n1_(n1), d_((size_t)(n0 * n1), v) {}
  int64_t size(int k) const { return k == 0 ? n0_ : n1_; }
  T& operator()(int64_t i, int64_t j) { return d_[(size_t)(i + n0_ * j)]; }
  const T& operator()(int64_t i, int64_t j) const { return d_[(size_t)(i + n0_ * j)]; }
  T* data() { return d_.data(); }
  const T* data() const { return d_.data(); }

 private:
  int64_t n0_ = 0, n1_ = 0;
  std::vector<T> d_;
};

// src/Core/surface_mesh_utilities.h:25-47
struct Mesh_Geom_T {
  Array2D<double> nods;   // >= 3 x Nn (rows 3,4: tip flags)
  Array2D<int64_t> conn;  // >= 3 x Ne, 0-based
};
struct DoF_Handle_T {
  int64_t n_dof = 0;
  Array2D<int64_t> dof_h;  // Ne x 18, -1 = fixed
};
// surface_mesh_utilities.h:51-62: "damage state" and forces per collocation point
struct Frac_State_T {
  std::vector<double> mr_open, mr_slip;                               // max. relative opening / slip
  std::vector<double> friction_coef, slip_cohesion, open_cohesion;   // instant forces
};
struct Mesh_Data_T {
  Mesh_Geom_T mesh;
  DoF_Handle_T dof_h_dd;
  Array2D<double> dd;      // (6 Ne) x 3
  // the volume-control iteration's state (surface_mesh_utilities.h:66-101),
  // per collocation point (6 el + local node)
  std::vector<int> mat_id;
  std::vector<double> pp;
  Frac_State_T frac_state;
};
// src/Core/model_parameters.h:22-31
struct F_C_Param_T {
  double cr_open = 1.0, peak_ts = 0.0, cr_slip = 1.0, peak_sc = 0.0, peak_sf = 0.0, res_sf = 0.0;
};
// src/Core/model_parameters.h:34-102
struct Properties_T {
  double shear_m = 1.0, poiss_r = 0.0;
  Array2D<int> c_model_id;              // n_surface x 2: cohesion, friction model ids
  std::vector<F_C_Param_T> f_c_param;   // per surface (material) id
};
struct Load_T {
  double s_inf[6] = {0, 0, 0, 0, 0, 0};  // xx, yy, zz, xy, xz, yz (tension positive)
  Array2D<int64_t> inj_loc;              // injection points: (element, local node) rows
};
struct Num_Param_T {
  double beta = 0.125;
  int tip_type = 1;
  bool is_dd_local = false;
};
struct Sim_Param_T {
  bool do_save_matrix = false, do_save_solution = false, do_postprocess = false;
};
struct IO_param_T {
  std::string src_dir, input_dir, output_dir, obs_p_dir;
  std::string conn_f_name, node_f_name, obs_p_f_name;
  std::string in_f_format = "npy32", out_f_format = "csv", obs_p_f_format = "npy32";
  std::string matr_f_name = "test_assembly", out_f_name = "test_solution", strs_f_name = "test_stresses";
  int64_t array_origin = 0;
};
// Settings of this engine, read from an optional [engine] table that the
// reference's parser ignores.
struct Engine_Param_T {
  int device = 0;
  int lu_mode = HFPX_LU_FP64;   // "fp64" | "mixed"
  double refine_tol = 1e-12;
  bool full_precision = false;  // also write %.17g csv copies of the outputs
};

// One GPU context (one stream) shared by the calls below.
hfpx_ctx* context(int device = 0);
void check(int rc);

// surface_mesh_utilities.cpp:28-112, :256-328
DoF_Handle_T make_dof_h_crack(const Mesh_Geom_T& mesh, int ap_order, int tip_type);
void write_dd_vector_to_md(const std::vector<double>& sol, const DoF_Handle_T& dof, Mesh_Data_T& md);

// Device-resident objects.
class DeviceMesh {
 public:
  DeviceMesh(const Mesh_Geom_T& mesh, double beta);
  ~DeviceMesh();
  DeviceMesh(const DeviceMesh&) = delete;
  DeviceMesh& operator=(const DeviceMesh&) = delete;
  hfpx_mesh* get() const { return h_; }

 private:
  hfpx_mesh* h_ = nullptr;
};

class DeviceMatrix {
 public:
  explicit DeviceMatrix(hfpx_matrix* h) : h_(h) {}
  ~DeviceMatrix();
  DeviceMatrix(const DeviceMatrix&) = delete;
  DeviceMatrix& operator=(const DeviceMatrix&) = delete;
  hfpx_matrix* get() const { return h_; }
  int64_t n() const;
  Array2D<double> download() const;

 private:
  hfpx_matrix* h_ = nullptr;
};

// system_assembly.cpp:30-219 (vc = false) and :458-557 (vc = true); the
// matrix stays on the device.
DeviceMatrix* assemble(const DeviceMesh& m, const DoF_Handle_T& dof, double shear_m, double poiss_r,
                       const Num_Param_T& n_par, bool vc);
// Host-returning forms with the reference's signatures.
Array2D<double> make_3dbem_matrix_s(double shear_m, double poiss_r, const Mesh_Geom_T& mesh,
                                    const Num_Param_T& n_par, DoF_Handle_T& dof_hndl);
Array2D<double> make_3dbem_matrix_vc(double shear_m, double poiss_r, const Mesh_Geom_T& mesh,
                                     const Num_Param_T& n_par, DoF_Handle_T& dof_hndl);
// system_assembly.cpp:222-274
void add_s_inf_to_3dbem_rhs(const DeviceMesh& m, const DoF_Handle_T& dof, const Load_T& load,
                            std::vector<double>& rhs);
// system_assembly.cpp:279-455; pts 3 x P -> P x 6
Array2D<double> make_3dbem_stress_f_s(double shear_m, double poiss_r, const DeviceMesh& m, const Mesh_Data_T& md,
                                      const Load_T& load, const Num_Param_T& n_par, const Array2D<double>& pts);

// il::LU<il::Array2D<double>> (LU.h:79-120): factors on construction.
class LU {
 public:
  LU(DeviceMatrix& a, int mode = HFPX_LU_FP64);
  std::vector<double> solve(const std::vector<double>& y, double tol = 1e-12, int max_iter = 30);
  hfpx_solve_info last_info{};

 private:
  DeviceMatrix& a_;
};

// src/Development/cohesion_friction.cpp:22-130, :134-194 (on the device)
void match_f_c(const Properties_T& prop, const std::vector<int>& mat_id, const Array2D<double>& dd,
               bool is_dd_local, Frac_State_T& f_state);
void update_mrd(const Properties_T& prop, const std::vector<int>& mat_id, const Array2D<double>& dd,
                bool is_dd_local, Frac_State_T& f_state);
// src/Development/c_f_iteration.cpp:27-436: one step of the volume-control
// scheme with cohesion and friction on the device-resident bordered matrix of
// orig_dof_h (make_3dbem_matrix_vc; unfactored, or factored with
// HFPX_LU_MIXED).  m_data (dd, pp, frac_state, mat_id) is updated and its
// dof_h_dd set to the step's truncated handle; returns the reference's
// residual (|increments|_1 + |traction adjustments|_1).  cf_flags are
// hfpx_vc_cf_iteration's (bit 0 all traction components, bit 1 the
// releasing sign); 0 reproduces the reference.  m_data_p (the previous time
// step) is unused, as in the reference.
double vc_cf_iteration(const Mesh_Data_T& m_data_p, const DeviceMatrix& orig_vc_sys, const DoF_Handle_T& orig_dof_h,
                       const DeviceMesh& mesh, const Properties_T& prop, const Num_Param_T& n_par, const Load_T& load,
                       double new_vol, Mesh_Data_T& m_data, int cf_flags = 0, hfpx_cf_info* info = nullptr);

// src/IO: config (config_file_io.cpp:56-361), meshes and points
// (mesh_file_io.cpp:28-605), csv output (data_file_io.h:131-168).
void read_config(const std::string& path, Mesh_Data_T& md, Properties_T& props, Load_T& load, Num_Param_T& n_par,
                 Sim_Param_T& sim, IO_param_T& io, Engine_Param_T& eng);
Array2D<double> load_npy_f64(const std::string& path);
Array2D<int64_t> load_npy_int(const std::string& path);
Mesh_Geom_T load_mesh_from_numpy(const std::string& dir, const std::string& conn_f, const std::string& node_f,
                                 int64_t origin);
Mesh_Geom_T load_mesh_from_csv(const std::string& dir, const std::string& conn_f, const std::string& node_f,
                               int64_t origin);
Array2D<double> load_crd_from_csv(const std::string& dir, const std::string& f);
Array2D<double> load_crd_from_numpy(const std::string& dir, const std::string& f);
// precision 0: the reference's default stream precision (6 significant digits)
bool save_data_to_csv(const Array2D<double>& a, const std::string& dir, const std::string& name, int precision = 0);
// NumPy .npy (format 1.0, Fortran order), float32 (bits 32) or float64 (64):
// the npy32/npy64 output formats the reference's driver leaves unwritten
// (main.cpp:131-136, 218-222, 271-275).
bool save_data_to_npy(const Array2D<double>& a, const std::string& dir, const std::string& name, int bits);
// save_data_to_npy for output_format "npy32"/"npy64" (".csv" in name becomes
// ".npy"), else save_data_to_csv; returns the file name written.
std::string save_output(const Array2D<double>& a, const IO_param_T& io, const std::string& name, int precision,
                        bool* ok);

}  // namespace hfpx
