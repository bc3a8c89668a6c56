// config.toml driver: the reference's main.cpp pipeline (read config ->
// DoF handle -> assemble + in-situ RHS -> LU solve -> nodal DD output ->
// stresses at observation points), with assembly, factorisation, solve and
// stress on the GPU through the engine's C-ABI.  Same console lines and the
// same csv files (main.cpp:66-291).
//
//   hfpx_main [path/to/config.toml]          (default: ./config.toml)
//   hfpx_main --check [path/to/config.toml]  read the config, the mesh and
//       the observation points, print what was read and exit (no GPU use)
//
// An optional [engine] table selects the device (device = 0), the LU mode
// (precision = "fp64" | "mixed"), the refinement tolerance of the mixed mode
// (refine_tol = 1e-12) and csv output with 17 significant digits
// (full_precision_output = true) in place of the reference's 6.
// output_format = "npy32" | "npy64" writes .npy files, which the reference's
// driver leaves unwritten.
#include <chrono>
#include <iostream>

#include "hfpx.hpp"

using namespace hfpx;

namespace {
double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}
}  // namespace

int main(int argc, char* argv[]) {
  int arg = 1;
  const bool check_only = argc > 1 && std::string(argv[1]) == "--check";
  if (check_only) ++arg;
  const std::string cfg = argc > arg ? argv[arg] : "config.toml";
  try {
    Mesh_Data_T md;
    Properties_T props;
    Load_T load;
    Num_Param_T np;
    Sim_Param_T sim;
    IO_param_T io;
    Engine_Param_T eng;
    read_config(cfg, md, props, load, np, sim, io, eng);
    if (check_only) {
      std::cout.precision(17);
      std::cout << "elements " << md.mesh.conn.size(1) << "\nnodes " << md.mesh.nods.size(1) << "\nshear_m "
                << props.shear_m << "\npoiss_r " << props.poiss_r << "\nbeta " << np.beta << "\ntip_type "
                << np.tip_type << "\nis_dd_local " << np.is_dd_local << "\ns_inf";
      for (double s : load.s_inf) std::cout << " " << s;
      std::cout << "\nsave_matrix " << sim.do_save_matrix << "\nsave_solution " << sim.do_save_solution
                << "\npostprocess " << sim.do_postprocess << "\noutput " << io.output_dir << io.out_f_name
                << "\nlu_mode " << eng.lu_mode << "\ndevice " << eng.device << "\n";
      int64_t csum = 0;
      for (int64_t j = 0; j < md.mesh.conn.size(1); ++j)
        for (int k = 0; k < 3; ++k) csum += md.mesh.conn(k, j) * (k + 1);
      double nsum = 0;
      for (int64_t j = 0; j < md.mesh.nods.size(1); ++j)
        for (int k = 0; k < 3; ++k) nsum += md.mesh.nods(k, j) * (k + 1);
      std::cout << "conn_checksum " << csum << "\nnods_checksum " << nsum << "\n";
      if (sim.do_postprocess) {
        const Array2D<double> pts = io.out_f_format == "csv" ? load_crd_from_csv(io.obs_p_dir, io.obs_p_f_name)
                                                             : load_crd_from_numpy(io.obs_p_dir, io.obs_p_f_name);
        std::cout << "points " << pts.size(0) << " x " << pts.size(1) << "\n";
      }
      return 0;
    }
    context(eng.device);
    const int prec = eng.full_precision ? 17 : 0;
    const int64_t ne = md.mesh.conn.size(1);

    std::cout << "Assembly";
    auto t0 = std::chrono::steady_clock::now();
    md.dof_h_dd = make_dof_h_crack(md.mesh, 2, np.tip_type);
    DeviceMesh dmesh(md.mesh, np.beta);
    DeviceMatrix* a = assemble(dmesh, md.dof_h_dd, props.shear_m, props.poiss_r, np, false);
    std::vector<double> rhs((size_t)md.dof_h_dd.n_dof, 0.0);
    add_s_inf_to_3dbem_rhs(dmesh, md.dof_h_dd, load, rhs);
    check(hfpx_ctx_synchronize(context()));
    std::cout << ": " << seconds_since(t0) << "s" << std::endl;
    std::cout << 18 * ne << " DoF Total" << std::endl;
    std::cout << 18 * ne - md.dof_h_dd.n_dof << " Fixed DoF" << std::endl;

    if (sim.do_save_matrix) {
      bool ok = false;
      const std::string f = save_output(a->download(), io, io.matr_f_name, prec, &ok);
      if (ok) std::cout << "Matrix saved to " << io.output_dir << "/" << f << std::endl;
      else std::cout << "Cannot save the matrix" << std::endl;
    }

    std::cout << "Solution";
    t0 = std::chrono::steady_clock::now();
    std::vector<double> dd_v;
    {
      LU lu(*a, eng.lu_mode);
      dd_v = lu.solve(rhs, eng.refine_tol);
    }
    std::cout << ": " << seconds_since(t0) << "s" << std::endl;
    delete a;
    write_dd_vector_to_md(dd_v, md.dof_h_dd, md);

    if (sim.do_save_solution) {
      // nodes (el_cp_uniform with beta 0: vertices, then the midpoint of the
      // edge across each vertex), a zero column, the three DD components
      Array2D<double> out(6 * ne, 7, 0.0);
      for (int64_t j = 0; j < ne; ++j) {
        double v[3][3];
        for (int k = 0; k < 3; ++k)
          for (int l = 0; l < 3; ++l) v[k][l] = md.mesh.nods(l, md.mesh.conn(k, j));
        for (int k = 0; k < 3; ++k) {
          const int m = (k + 1) % 3, q = (m + 1) % 3;
          for (int l = 0; l < 3; ++l) {
            out(6 * j + k, l) = v[k][l];
            out(6 * j + k + 3, l) = 0.5 * (v[m][l] + v[q][l]);
          }
        }
        for (int k = 0; k < 6; ++k)
          for (int l = 0; l < 3; ++l) out(6 * j + k, l + 4) = md.dd(6 * j + k, l);
      }
      bool ok = false;
      const std::string f = save_output(out, io, io.out_f_name, prec, &ok);
      if (ok) std::cout << "Solution (nodes + DD) saved to " << io.output_dir << "/" << f << std::endl;
      else std::cout << "Cannot save the solution" << std::endl;
    }

    if (sim.do_postprocess) {
      // the reference picks the point reader by the OUTPUT format
      // (main.cpp:238-247)
      const Array2D<double> pts = io.out_f_format == "csv" ? load_crd_from_csv(io.obs_p_dir, io.obs_p_f_name)
                                                           : load_crd_from_numpy(io.obs_p_dir, io.obs_p_f_name);
      std::cout << "Postprocessing";
      t0 = std::chrono::steady_clock::now();
      const Array2D<double> s = make_3dbem_stress_f_s(props.shear_m, props.poiss_r, dmesh, md, load, np, pts);
      std::cout << ": " << seconds_since(t0) << "s" << std::endl;
      bool ok = false;
      const std::string f = save_output(s, io, io.strs_f_name, prec, &ok);
      if (ok) std::cout << "Stresses at given points saved to " << io.output_dir << "/" << f << std::endl;
      else std::cout << "Cannot save the stresses" << std::endl;
    }
  } catch (const Error& e) {
    std::cerr << "hfpx_main: " << e.what() << " (status " << e.code << ")" << std::endl;
    return 1;
  } catch (const std::exception& e) {
    std::cerr << "hfpx_main: " << e.what() << std::endl;
    return 1;
  }
  return 0;
}
