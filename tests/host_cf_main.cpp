// Test program of the C++ host layer's volume-control iteration
// (hfpx::vc_cf_iteration, hfpx::match_f_c, hfpx::update_mrd): reads a case
// written by tests/test_gpu_cf.py as .npy files, assembles the bordered
// matrix of the mesh (tip vertices fixed, DD local), factors it mixed, runs
// `steps` iterations and update_mrd, and writes dd, pp, the truncated handle
// and the last residual back as .npy files.
//   host_cf_main <dir> <steps> <flags>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "hfpx.hpp"

int main(int argc, char** argv) {
  if (argc != 4) {
    std::fprintf(stderr, "usage: host_cf_main <dir> <steps> <flags>\n");
    return 2;
  }
  const std::string dir = argv[1];
  const int steps = std::atoi(argv[2]), flags = std::atoi(argv[3]);
  try {
    hfpx::Mesh_Geom_T mesh;
    mesh.nods = hfpx::load_npy_f64(dir + "/nods.npy");
    mesh.conn = hfpx::load_npy_int(dir + "/conn.npy");
    hfpx::Num_Param_T np;
    np.beta = 0.125;
    np.tip_type = 1;
    np.is_dd_local = true;
    hfpx::DoF_Handle_T dof = hfpx::make_dof_h_crack(mesh, 2, np.tip_type);
    hfpx::Properties_T prop;
    prop.shear_m = 1.0;
    prop.poiss_r = 0.35;
    const hfpx::Array2D<double> mats = hfpx::load_npy_f64(dir + "/mats.npy");  // n_mat x 8
    prop.c_model_id = hfpx::Array2D<int>(mats.size(0), 2);
    for (int64_t m = 0; m < mats.size(0); ++m) {
      prop.f_c_param.push_back({mats(m, 0), mats(m, 1), mats(m, 2), mats(m, 3), mats(m, 4), mats(m, 5)});
      prop.c_model_id(m, 0) = (int)mats(m, 6);
      prop.c_model_id(m, 1) = (int)mats(m, 7);
    }
    const hfpx::Array2D<double> par = hfpx::load_npy_f64(dir + "/params.npy");  // s_inf[6], inj el, inj node, vol
    hfpx::Load_T load;
    for (int k = 0; k < 6; ++k) load.s_inf[k] = par(k, 0);
    load.inj_loc = hfpx::Array2D<int64_t>(1, 2);
    load.inj_loc(0, 0) = (int64_t)par(6, 0);
    load.inj_loc(0, 1) = (int64_t)par(7, 0);
    const double new_vol = par(8, 0);
    hfpx::Mesh_Data_T md;
    md.mesh = mesh;
    md.dd = hfpx::load_npy_f64(dir + "/dd.npy");
    const hfpx::Array2D<double> pp = hfpx::load_npy_f64(dir + "/pp.npy");
    const hfpx::Array2D<double> mro = hfpx::load_npy_f64(dir + "/mr_open.npy");
    const hfpx::Array2D<double> mrs = hfpx::load_npy_f64(dir + "/mr_slip.npy");
    const hfpx::Array2D<int64_t> mid = hfpx::load_npy_int(dir + "/mat_id.npy");
    const int64_t n_cp = md.dd.size(0);
    for (int64_t i = 0; i < n_cp; ++i) {
      md.pp.push_back(pp(i, 0));
      md.frac_state.mr_open.push_back(mro(i, 0));
      md.frac_state.mr_slip.push_back(mrs(i, 0));
      md.mat_id.push_back((int)mid(i, 0));
    }
    hfpx::DeviceMesh dm(mesh, np.beta);
    hfpx::DeviceMatrix* A = hfpx::assemble(dm, dof, prop.shear_m, prop.poiss_r, np, true);
    hfpx::LU lu(*A, HFPX_LU_MIXED);
    double res = 0.0;
    for (int s = 0; s < steps; ++s)
      res = hfpx::vc_cf_iteration(md, *A, dof, dm, prop, np, load, new_vol, md, flags);
    hfpx::update_mrd(prop, md.mat_id, md.dd, np.is_dd_local, md.frac_state);
    hfpx::Array2D<double> out_pp(n_cp, 3), out_dof(dof.dof_h.size(0), 18), out_res(1, 2);
    for (int64_t i = 0; i < n_cp; ++i) {
      out_pp(i, 0) = md.pp[(size_t)i];
      out_pp(i, 1) = md.frac_state.mr_open[(size_t)i];
      out_pp(i, 2) = md.frac_state.mr_slip[(size_t)i];
    }
    for (int64_t e = 0; e < dof.dof_h.size(0); ++e)
      for (int l = 0; l < 18; ++l) out_dof(e, l) = (double)md.dof_h_dd.dof_h(e, l);
    out_res(0, 0) = res;
    out_res(0, 1) = (double)md.dof_h_dd.n_dof;
    bool ok = hfpx::save_data_to_npy(md.dd, dir, "out_dd.npy", 64);
    ok = ok && hfpx::save_data_to_npy(out_pp, dir, "out_pp.npy", 64);
    ok = ok && hfpx::save_data_to_npy(out_dof, dir, "out_dof.npy", 64);
    ok = ok && hfpx::save_data_to_npy(out_res, dir, "out_res.npy", 64);
    delete A;
    return ok ? 0 : 1;
  } catch (const hfpx::Error& e) {
    std::fprintf(stderr, "hfpx::Error %d: %s\n", e.code, e.what());
    return 1;
  }
}
