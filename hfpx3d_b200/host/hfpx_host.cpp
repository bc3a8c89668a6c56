// Implementation of the C++ host layer (hfpx.hpp): calls through the C-ABI,
// plus the file formats the reference's driver reads and writes.
#include "hfpx.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>

namespace hfpx {

// ---------------------------------------------------------------- context
static hfpx_ctx* g_ctx = nullptr;

hfpx_ctx* context(int device) {
  if (!g_ctx) {
    const int rc = hfpx_ctx_create(device, &g_ctx);
    if (rc) throw Error(rc, "cannot create an engine context on device " + std::to_string(device));
  }
  return g_ctx;
}

void check(int rc) {
  if (rc) throw Error(rc, hfpx_ctx_last_error(g_ctx));
}

// ------------------------------------------------------------- DoF handle
DoF_Handle_T make_dof_h_crack(const Mesh_Geom_T& mesh, int ap_order, int tip_type) {
  if (ap_order != 2) throw Error(HFPX_ERR_ARG, "only quadratic (order 2) elements are supported");
  DoF_Handle_T d;
  const int64_t ne = mesh.conn.size(1);
  d.dof_h = Array2D<int64_t>(ne, 18);
  d.n_dof = hfpx_dof_handle(mesh.nods.data(), mesh.nods.size(0), mesh.nods.size(1), mesh.conn.data(),
                            mesh.conn.size(0), ne, tip_type, d.dof_h.data());
  if (d.n_dof < 0) throw Error((int)-d.n_dof, "bad mesh for the DoF handle");
  return d;
}

void write_dd_vector_to_md(const std::vector<double>& sol, const DoF_Handle_T& dof, Mesh_Data_T& md) {
  const int64_t ne = dof.dof_h.size(0);
  md.dd = Array2D<double>(6 * ne, 3, 0.0);
  for (int64_t e = 0; e < ne; ++e)
    for (int j = 0; j < 18; ++j) {
      const int64_t g = dof.dof_h(e, j);
      if (g >= 0) md.dd(6 * e + j / 3, j % 3) = sol[(size_t)g];
    }
}

// ---------------------------------------------------------- device objects
DeviceMesh::DeviceMesh(const Mesh_Geom_T& m, double beta) {
  check(hfpx_mesh_create(context(), m.nods.data(), m.nods.size(0), m.nods.size(1), m.conn.data(), m.conn.size(0),
                         m.conn.size(1), beta, &h_));
}
DeviceMesh::~DeviceMesh() { hfpx_mesh_destroy(h_); }

DeviceMatrix::~DeviceMatrix() { hfpx_matrix_destroy(h_); }
int64_t DeviceMatrix::n() const {
  int64_t n = 0, ld = 0;
  hfpx_matrix_dims(h_, &n, &ld);
  return n;
}
Array2D<double> DeviceMatrix::download() const {
  const int64_t m = n();
  Array2D<double> a(m, m);
  check(hfpx_matrix_download(context(), h_, a.data(), m));
  return a;
}

DeviceMatrix* assemble(const DeviceMesh& m, const DoF_Handle_T& dof, double G, double nu, const Num_Param_T& np,
                       bool vc) {
  hfpx_matrix* h = nullptr;
  check(hfpx_assemble(context(), m.get(), dof.dof_h.data(), dof.n_dof, G, nu, np.is_dd_local ? 1 : 0, vc ? 1 : 0, &h));
  return new DeviceMatrix(h);
}

static Array2D<double> host_matrix(double G, double nu, const Mesh_Geom_T& mesh, const Num_Param_T& np,
                                   DoF_Handle_T& dof, bool vc) {
  if (dof.n_dof == 0 || dof.dof_h.size(0) == 0) dof = make_dof_h_crack(mesh, 2, np.tip_type);
  DeviceMesh m(mesh, np.beta);
  DeviceMatrix* a = assemble(m, dof, G, nu, np, vc);
  Array2D<double> out = a->download();
  delete a;
  return out;
}

Array2D<double> make_3dbem_matrix_s(double G, double nu, const Mesh_Geom_T& mesh, const Num_Param_T& np,
                                    DoF_Handle_T& dof) {
  return host_matrix(G, nu, mesh, np, dof, false);
}
Array2D<double> make_3dbem_matrix_vc(double G, double nu, const Mesh_Geom_T& mesh, const Num_Param_T& np,
                                     DoF_Handle_T& dof) {
  return host_matrix(G, nu, mesh, np, dof, true);
}

void add_s_inf_to_3dbem_rhs(const DeviceMesh& m, const DoF_Handle_T& dof, const Load_T& load,
                            std::vector<double>& rhs) {
  if ((int64_t)rhs.size() != dof.n_dof) rhs.assign((size_t)dof.n_dof, 0.0);
  check(hfpx_rhs_sinf(context(), m.get(), dof.dof_h.data(), dof.n_dof, load.s_inf, 1, rhs.data(), dof.n_dof));
}

Array2D<double> make_3dbem_stress_f_s(double G, double nu, const DeviceMesh& m, const Mesh_Data_T& md,
                                      const Load_T& load, const Num_Param_T& np, const Array2D<double>& pts) {
  Array2D<double> out(pts.size(1), 6);
  check(hfpx_stress(context(), m.get(), G, nu, np.is_dd_local ? 1 : 0, md.dd.data(), pts.data(), pts.size(1),
                    load.s_inf, out.data()));
  return out;
}

// ---- the volume-control iteration with cohesion and friction
static std::vector<hfpx_cf_material> cf_materials(const Properties_T& prop) {
  if (prop.f_c_param.empty()) throw Error(HFPX_ERR_ARG, "Properties_T has no contact parameters");
  std::vector<hfpx_cf_material> m(prop.f_c_param.size());
  for (size_t i = 0; i < m.size(); ++i) {
    const F_C_Param_T& p = prop.f_c_param[i];
    m[i] = {p.cr_open, p.peak_ts, p.cr_slip, p.peak_sc, p.peak_sf, p.res_sf, 0, 0};
    if ((int64_t)i < prop.c_model_id.size(0)) {
      m[i].cohesion_model = prop.c_model_id((int64_t)i, 0);
      m[i].friction_model = prop.c_model_id((int64_t)i, 1);
    }
  }
  return m;
}

// Frac_State_T sized for n_cp points (new entries 0)
static void size_state(Frac_State_T& f, size_t n_cp) {
  for (std::vector<double>* v : {&f.mr_open, &f.mr_slip, &f.friction_coef, &f.slip_cohesion, &f.open_cohesion})
    if (v->size() != n_cp) v->resize(n_cp, 0.0);
}

static hfpx_cf_state cf_view(const Array2D<double>& dd, std::vector<double>& pp, Frac_State_T& f,
                             const std::vector<int32_t>& mat_id, int64_t* dof_h) {
  return hfpx_cf_state{const_cast<double*>(dd.data()), pp.data(), f.mr_open.data(), f.mr_slip.data(),
                       f.friction_coef.data(), f.slip_cohesion.data(), f.open_cohesion.data(), mat_id.data(), dof_h};
}

static std::vector<int32_t> mat_ids(const std::vector<int>& mat_id, int64_t n_cp) {
  if ((int64_t)mat_id.size() != n_cp) throw Error(HFPX_ERR_ARG, "mat_id needs one entry per collocation point");
  return std::vector<int32_t>(mat_id.begin(), mat_id.end());
}

void match_f_c(const Properties_T& prop, const std::vector<int>& mat_id, const Array2D<double>& dd, bool,
               Frac_State_T& f_state) {
  const int64_t n_cp = dd.size(0);
  if (dd.size(1) != 3) throw Error(HFPX_ERR_ARG, "dd must be n x 3");
  const std::vector<hfpx_cf_material> m = cf_materials(prop);
  const std::vector<int32_t> id = mat_ids(mat_id, n_cp);
  size_state(f_state, (size_t)n_cp);
  std::vector<double> pp((size_t)n_cp, 0.0);
  hfpx_cf_state st = cf_view(dd, pp, f_state, id, nullptr);
  check(hfpx_cf_match(context(), n_cp, m.data(), (int)m.size(), &st));
}

void update_mrd(const Properties_T& prop, const std::vector<int>& mat_id, const Array2D<double>& dd, bool,
                Frac_State_T& f_state) {
  const int64_t n_cp = dd.size(0);
  if (dd.size(1) != 3) throw Error(HFPX_ERR_ARG, "dd must be n x 3");
  const std::vector<hfpx_cf_material> m = cf_materials(prop);
  const std::vector<int32_t> id = mat_ids(mat_id, n_cp);
  size_state(f_state, (size_t)n_cp);
  std::vector<double> pp((size_t)n_cp, 0.0);
  hfpx_cf_state st = cf_view(dd, pp, f_state, id, nullptr);
  check(hfpx_cf_update_mrd(context(), n_cp, m.data(), (int)m.size(), &st));
}

double vc_cf_iteration(const Mesh_Data_T&, const DeviceMatrix& orig_vc_sys, const DoF_Handle_T& orig_dof_h,
                       const DeviceMesh& mesh, const Properties_T& prop, const Num_Param_T& n_par, const Load_T& load,
                       double new_vol, Mesh_Data_T& m_data, int cf_flags, hfpx_cf_info* info_out) {
  const int64_t n_el = orig_dof_h.dof_h.size(0), n_cp = 6 * n_el;
  if (m_data.dd.size(0) != n_cp || m_data.dd.size(1) != 3) throw Error(HFPX_ERR_ARG, "m_data.dd must be (6 Ne) x 3");
  if ((int64_t)m_data.pp.size() != n_cp) throw Error(HFPX_ERR_ARG, "m_data.pp needs one entry per collocation point");
  if (load.inj_loc.size(0) < 1 || load.inj_loc.size(1) < 2) throw Error(HFPX_ERR_ARG, "load.inj_loc is empty");
  const std::vector<hfpx_cf_material> m = cf_materials(prop);
  const std::vector<int32_t> id = mat_ids(m_data.mat_id, n_cp);
  size_state(m_data.frac_state, (size_t)n_cp);
  Array2D<int64_t> dof_new(n_el, 18, -1);
  hfpx_cf_state st = cf_view(m_data.dd, m_data.pp, m_data.frac_state, id, dof_new.data());
  hfpx_cf_info info{};
  // the injection point inj_loc(0, 0) * 6 + inj_loc(0, 1) (c_f_iteration.cpp:80)
  const int64_t inj = load.inj_loc(0, 0) * 6 + load.inj_loc(0, 1);
  check(hfpx_vc_cf_iteration(context(), mesh.get(), orig_vc_sys.get(), orig_dof_h.dof_h.data(), orig_dof_h.n_dof,
                             m.data(), (int)m.size(), load.s_inf, inj, new_vol, n_par.is_dd_local ? 1 : 0, cf_flags,
                             1e-12, &st, &info));
  m_data.dof_h_dd.dof_h = dof_new;
  m_data.dof_h_dd.n_dof = info.n_dof;
  if (info_out) *info_out = info;
  return info.residual;
}

LU::LU(DeviceMatrix& a, int mode) : a_(a) {
  int64_t info = 0;
  check(hfpx_lu_factor(context(), a.get(), mode, &info));
}

std::vector<double> LU::solve(const std::vector<double>& y, double tol, int max_iter) {
  std::vector<double> x = y;
  check(hfpx_lu_solve(context(), a_.get(), x.data(), 1, (int64_t)x.size(), tol, max_iter, &last_info));
  return x;
}

// ------------------------------------------------------------- TOML subset
// key = value lines (strings, integers, floats, booleans), [table] headers
// and # comments: the part of TOML the reference's config.toml uses.  Types
// are kept apart because the reference only accepts, e.g., a float for
// S_zz or cp_offset and an integer for fix_tip.
struct TomlValue {
  enum Kind { Str, Int, Dbl, Bool } kind = Str;
  std::string s;
  int64_t i = 0;
  double d = 0;
  bool b = false;
};
using Toml = std::map<std::string, TomlValue>;

static std::string trim(const std::string& s) {
  const size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? "" : s.substr(a, b - a + 1);
}

static Toml parse_toml(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw Error(HFPX_ERR_ARG, "cannot open config file " + path);
  Toml t;
  std::string line, table;
  int ln = 0;
  while (std::getline(f, line)) {
    ++ln;
    // strip a comment that is not inside a string
    bool in_str = false;
    for (size_t k = 0; k < line.size(); ++k) {
      if (line[k] == '"') in_str = !in_str;
      if (line[k] == '#' && !in_str) { line.resize(k); break; }
    }
    line = trim(line);
    if (line.empty()) continue;
    if (line.front() == '[') {
      table = trim(line.substr(1, line.find(']') - 1));
      continue;
    }
    const size_t eq = line.find('=');
    if (eq == std::string::npos) throw Error(HFPX_ERR_ARG, path + ":" + std::to_string(ln) + ": expected key = value");
    const std::string key = (table.empty() ? "" : table + ".") + trim(line.substr(0, eq));
    const std::string v = trim(line.substr(eq + 1));
    TomlValue val;
    if (!v.empty() && v.front() == '"') {
      val.kind = TomlValue::Str;
      val.s = v.substr(1, v.rfind('"') - 1);
    } else if (v == "true" || v == "false") {
      val.kind = TomlValue::Bool;
      val.b = v == "true";
    } else if (v.find_first_of(".eE") != std::string::npos || v == "inf" || v == "nan") {
      val.kind = TomlValue::Dbl;
      val.d = std::stod(v);
    } else {
      val.kind = TomlValue::Int;
      val.i = std::stoll(v);
    }
    t[key] = val;
  }
  return t;
}

static const TomlValue* get(const Toml& t, const std::string& k, TomlValue::Kind kind) {
  auto it = t.find(k);
  return it != t.end() && it->second.kind == kind ? &it->second : nullptr;
}

static std::string dir_of(const std::string& p) {
  const size_t s = p.rfind('/');
  return s == std::string::npos ? "." : p.substr(0, s);
}

static std::string join_dir(const std::string& base, const std::string& d) {
  std::string r = (!d.empty() && d[0] == '/') ? d : base + "/" + d;
  if (r.empty() || r.back() != '/') r += '/';
  return r;
}

// config_file_io.cpp:26-54 (defaults), :56-361 (keys).
void read_config(const std::string& path, Mesh_Data_T& md, Properties_T& props, Load_T& load, Num_Param_T& np,
                 Sim_Param_T& sim, IO_param_T& io, Engine_Param_T& eng) {
  const Toml t = parse_toml(path);
  io.src_dir = dir_of(path);
  io.input_dir = io.src_dir + "/Mesh_Files/";
  io.output_dir = io.src_dir + "/Test_Output/";
  if (auto v = get(t, "mesh_input_directory", TomlValue::Str)) io.input_dir = join_dir(io.src_dir, v->s);
  if (auto v = get(t, "mesh_conn_fname", TomlValue::Str)) io.conn_f_name = v->s;
  else throw Error(HFPX_ERR_ARG, "config: mesh_conn_fname missing");
  if (auto v = get(t, "nodes_crd_fname", TomlValue::Str)) io.node_f_name = v->s;
  else throw Error(HFPX_ERR_ARG, "config: nodes_crd_fname missing");
  if (auto v = get(t, "mesh_input_format", TomlValue::Str)) io.in_f_format = v->s;
  if (auto v = get(t, "array_origin", TomlValue::Int)) io.array_origin = v->i;
  if (auto v = get(t, "do_save_matrix", TomlValue::Bool)) sim.do_save_matrix = v->b;
  if (auto v = get(t, "do_save_solution", TomlValue::Bool)) sim.do_save_solution = v->b;
  if (auto v = get(t, "do_postprocess", TomlValue::Bool)) sim.do_postprocess = v->b;
  // elastic properties: a [solid] table or top-level keys
  const std::string pre = t.count("solid.Poisson_ratio") || t.count("solid.Shear_modulus") ||
                                  t.count("solid.Young_modulus")
                              ? "solid."
                              : "";
  props.shear_m = 1.0;
  props.poiss_r = 0.0;
  if (auto v = get(t, pre + "Poisson_ratio", TomlValue::Dbl)) props.poiss_r = v->d;
  if (auto v = get(t, pre + "Shear_modulus", TomlValue::Dbl)) props.shear_m = v->d;
  else if (auto w = get(t, pre + "Young_modulus", TomlValue::Dbl)) props.shear_m = w->d / 2.0 / (1.0 + props.poiss_r);
  np.beta = 0.125;
  np.tip_type = 1;
  np.is_dd_local = false;
  if (auto v = get(t, "cp_offset", TomlValue::Dbl)) np.beta = v->d;
  if (auto v = get(t, "fix_tip", TomlValue::Int)) np.tip_type = (int)v->i;
  if (auto v = get(t, "is_dd_local", TomlValue::Bool)) np.is_dd_local = v->b;
  // in-situ stress: normal components given compression-positive (negated,
  // config_file_io.cpp:250-262), shear components as given
  const char* keys[6] = {"S_xx", "S_yy", "S_zz", "S_xy", "S_xz", "S_yz"};
  for (int k = 0; k < 6; ++k) {
    load.s_inf[k] = 0.0;
    if (auto v = get(t, keys[k], TomlValue::Dbl)) load.s_inf[k] = k < 3 ? -v->d : v->d;
  }
  // observation points
  io.obs_p_dir = io.input_dir;
  if (auto v = get(t, "observ_crd_directory", TomlValue::Str)) io.obs_p_dir = join_dir(io.src_dir, v->s);
  if (auto v = get(t, "observ_crd_fname", TomlValue::Str)) io.obs_p_f_name = v->s;
  else if (sim.do_postprocess) throw Error(HFPX_ERR_ARG, "config: observ_crd_fname missing");
  if (auto v = get(t, "observ_input_format", TomlValue::Str)) io.obs_p_f_format = v->s;
  // outputs
  if (auto v = get(t, "output_directory", TomlValue::Str)) io.output_dir = join_dir(io.src_dir, v->s);
  if (auto v = get(t, "output_signature", TomlValue::Str)) {
    io.matr_f_name += v->s;
    io.out_f_name += v->s;
    io.strs_f_name += v->s;
  }
  if (auto v = get(t, "output_format", TomlValue::Str)) io.out_f_format = v->s;
  io.matr_f_name += ".csv";
  io.out_f_name += ".csv";
  io.strs_f_name += ".csv";
  // this engine's own settings
  if (auto v = get(t, "engine.device", TomlValue::Int)) eng.device = (int)v->i;
  if (auto v = get(t, "engine.precision", TomlValue::Str)) {
    if (v->s == "mixed") eng.lu_mode = HFPX_LU_MIXED;
    else if (v->s == "fp64") eng.lu_mode = HFPX_LU_FP64;
    else throw Error(HFPX_ERR_ARG, "config: engine.precision must be \"fp64\" or \"mixed\"");
  }
  if (auto v = get(t, "engine.refine_tol", TomlValue::Dbl)) eng.refine_tol = v->d;
  if (auto v = get(t, "engine.full_precision_output", TomlValue::Bool)) eng.full_precision = v->b;
  // mesh (config_file_io.cpp:279-291)
  if (io.in_f_format == "csv")
    md.mesh = load_mesh_from_csv(io.input_dir, io.conn_f_name, io.node_f_name, io.array_origin);
  else
    md.mesh = load_mesh_from_numpy(io.input_dir, io.conn_f_name, io.node_f_name, io.array_origin);
}

// ------------------------------------------------------------------- npy
// NumPy .npy reader (format versions 1-3, little-endian f8/i4/i8, C or
// Fortran order).  The reference reads Fortran-order f8/i4 only
// (il/io/numpy/numpy.h:217-276); C order is transposed here.
struct Npy {
  std::string descr;
  bool fortran = false;
  std::vector<int64_t> shape;
  std::vector<char> data;
};

static Npy read_npy(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw Error(HFPX_ERR_ARG, "cannot open " + path);
  char magic[8];
  f.read(magic, 8);
  if (!f || std::memcmp(magic, "\x93NUMPY", 6) != 0) throw Error(HFPX_ERR_ARG, path + ": not a .npy file");
  uint32_t hlen = 0;
  if (magic[6] == 1) {
    uint16_t h16 = 0;
    f.read(reinterpret_cast<char*>(&h16), 2);
    hlen = h16;
  } else {
    f.read(reinterpret_cast<char*>(&hlen), 4);
  }
  std::string hdr(hlen, '\0');
  f.read(&hdr[0], hlen);
  Npy n;
  auto field = [&](const std::string& k) {
    const size_t p = hdr.find("'" + k + "'");
    if (p == std::string::npos) throw Error(HFPX_ERR_ARG, path + ": header lacks " + k);
    return hdr.substr(hdr.find(':', p) + 1);
  };
  std::string d = field("descr");
  n.descr = d.substr(d.find('\'') + 1, d.find('\'', d.find('\'') + 1) - d.find('\'') - 1);
  n.fortran = trim(field("fortran_order")).rfind("True", 0) == 0;
  std::string s = field("shape");
  s = s.substr(s.find('(') + 1, s.find(')') - s.find('(') - 1);
  std::stringstream ss(s);
  std::string tok;
  while (std::getline(ss, tok, ','))
    if (!trim(tok).empty()) n.shape.push_back(std::stoll(trim(tok)));
  if (n.shape.size() == 1) n.shape.push_back(1);
  if (n.shape.size() != 2) throw Error(HFPX_ERR_ARG, path + ": expected a 2-D array");
  const int64_t es = n.descr == "<f8" || n.descr == "<i8" ? 8 : n.descr == "<i4" ? 4 : 0;
  if (!es) throw Error(HFPX_ERR_ARG, path + ": unsupported dtype " + n.descr);
  n.data.resize((size_t)(n.shape[0] * n.shape[1] * es));
  f.read(n.data.data(), (std::streamsize)n.data.size());
  if (!f) throw Error(HFPX_ERR_ARG, path + ": truncated data");
  return n;
}

template <class T, class S>
static Array2D<T> npy_to(const Npy& n) {
  Array2D<T> a(n.shape[0], n.shape[1]);
  const S* src = reinterpret_cast<const S*>(n.data.data());
  for (int64_t i = 0; i < n.shape[0]; ++i)
    for (int64_t j = 0; j < n.shape[1]; ++j)
      a(i, j) = (T)(n.fortran ? src[i + n.shape[0] * j] : src[i * n.shape[1] + j]);
  return a;
}

Array2D<double> load_npy_f64(const std::string& path) {
  Npy n = read_npy(path);
  if (n.descr != "<f8") throw Error(HFPX_ERR_ARG, path + ": expected float64");
  return npy_to<double, double>(n);
}

Array2D<int64_t> load_npy_int(const std::string& path) {
  Npy n = read_npy(path);
  if (n.descr == "<i4") return npy_to<int64_t, int32_t>(n);
  if (n.descr == "<i8") return npy_to<int64_t, int64_t>(n);
  throw Error(HFPX_ERR_ARG, path + ": expected int32 or int64");
}

static void shift_origin(Mesh_Geom_T& m, int64_t origin) {
  if (!origin) return;
  const int64_t nr = m.conn.size(0) >= 3 ? 3 : m.conn.size(0);
  for (int64_t k = 0; k < m.conn.size(1); ++k)
    for (int64_t j = 0; j < nr; ++j) m.conn(j, k) -= origin;
}

// mesh_file_io.cpp:186-340
Mesh_Geom_T load_mesh_from_numpy(const std::string& dir, const std::string& cf, const std::string& nf,
                                 int64_t origin) {
  Mesh_Geom_T m;
  m.conn = load_npy_int(dir + cf);
  m.nods = load_npy_f64(dir + nf);
  shift_origin(m, origin);
  return m;
}

// Comma-separated rows; each row of the file becomes one column
// (mesh_file_io.cpp:28-185, 342-605).
static std::vector<std::vector<double>> read_csv_rows(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw Error(HFPX_ERR_ARG, "cannot open " + path);
  std::vector<std::vector<double>> rows;
  std::string line;
  while (std::getline(f, line)) {
    if (trim(line).empty()) continue;
    std::vector<double> r;
    std::stringstream ls(line);
    std::string cell;
    while (std::getline(ls, cell, ','))
      if (!trim(cell).empty()) r.push_back(std::stod(trim(cell)));
    if (!rows.empty() && r.size() != rows[0].size()) throw Error(HFPX_ERR_ARG, path + ": row size is not constant");
    rows.push_back(r);
  }
  return rows;
}

Array2D<double> load_crd_from_csv(const std::string& dir, const std::string& fn) {
  auto rows = read_csv_rows(dir + fn);
  Array2D<double> a(rows.empty() ? 0 : (int64_t)rows[0].size(), (int64_t)rows.size());
  for (size_t k = 0; k < rows.size(); ++k)
    for (size_t j = 0; j < rows[k].size(); ++j) a((int64_t)j, (int64_t)k) = rows[k][j];
  return a;
}

Array2D<double> load_crd_from_numpy(const std::string& dir, const std::string& fn) { return load_npy_f64(dir + fn); }

Mesh_Geom_T load_mesh_from_csv(const std::string& dir, const std::string& cf, const std::string& nf,
                               int64_t origin) {
  Mesh_Geom_T m;
  auto c = load_crd_from_csv(dir, cf);
  m.conn = Array2D<int64_t>(c.size(0), c.size(1));
  for (int64_t i = 0; i < c.size(0); ++i)
    for (int64_t j = 0; j < c.size(1); ++j) m.conn(i, j) = (int64_t)std::llround(c(i, j));
  m.nods = load_crd_from_csv(dir, nf);
  shift_origin(m, origin);
  return m;
}

// data_file_io.h:131-168: rows of the array, comma separated.
bool save_data_to_csv(const Array2D<double>& a, const std::string& dir, const std::string& name, int precision) {
  std::string p = dir;
  if (p.empty() || p.back() != '/') p += '/';
  p += name;
  std::ofstream o(p);
  if (!o) {
    std::cout << "Can't open the file (" << p << ")" << std::endl;
    return false;
  }
  if (precision > 0) o << std::setprecision(precision);
  for (int64_t i = 0; i < a.size(0); ++i) {
    for (int64_t j = 0; j < a.size(1); ++j) {
      o << a(i, j);
      if (j < a.size(1) - 1) o << ",";
    }
    o << "\n";
  }
  return true;
}

bool save_data_to_npy(const Array2D<double>& a, const std::string& dir, const std::string& name, int bits) {
  std::string p = dir;
  if (p.empty() || p.back() != '/') p += '/';
  p += name;
  std::ofstream o(p, std::ios::binary);
  if (!o) {
    std::cout << "Can't open the file (" << p << ")" << std::endl;
    return false;
  }
  std::string hdr = std::string("{'descr': '") + (bits == 32 ? "<f4" : "<f8") +
                    "', 'fortran_order': True, 'shape': (" + std::to_string(a.size(0)) + ", " +
                    std::to_string(a.size(1)) + "), }";
  // magic (6) + version (2) + length (2) + header, padded with spaces to a
  // multiple of 64 bytes and ended by a newline
  const size_t total = ((10 + hdr.size() + 1 + 63) / 64) * 64;
  hdr.append(total - 10 - hdr.size() - 1, ' ');
  hdr.push_back('\n');
  const uint16_t hlen = (uint16_t)hdr.size();
  o.write("\x93NUMPY\x01\x00", 8);
  o.write(reinterpret_cast<const char*>(&hlen), 2);
  o.write(hdr.data(), (std::streamsize)hdr.size());
  const size_t n = (size_t)(a.size(0) * a.size(1));
  if (bits == 32) {
    std::vector<float> f(n);
    for (size_t i = 0; i < n; ++i) f[i] = (float)a.data()[i];
    o.write(reinterpret_cast<const char*>(f.data()), (std::streamsize)(n * sizeof(float)));
  } else {
    o.write(reinterpret_cast<const char*>(a.data()), (std::streamsize)(n * sizeof(double)));
  }
  return (bool)o;
}

std::string save_output(const Array2D<double>& a, const IO_param_T& io, const std::string& name, int precision,
                        bool* ok) {
  if (io.out_f_format == "npy32" || io.out_f_format == "npy64") {
    std::string f = name;
    if (f.size() >= 4 && f.compare(f.size() - 4, 4, ".csv") == 0) f.replace(f.size() - 4, 4, ".npy");
    *ok = save_data_to_npy(a, io.output_dir, f, io.out_f_format == "npy32" ? 32 : 64);
    return f;
  }
  *ok = save_data_to_csv(a, io.output_dir, name, precision);
  return name;
}

}  // namespace hfpx
