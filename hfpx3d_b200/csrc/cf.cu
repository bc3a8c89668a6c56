// The volume-control iteration with cohesion and friction on the device:
// vc_cf_iteration (src/Development/c_f_iteration.cpp:27-436) with match_f_c
// and update_mrd (src/Development/cohesion_friction.cpp:22-130, :134-194).
//
// One step: the fracture state's cohesion and friction (match_kernel), the
// elastic tractions of the current DD and the crack volume (one FP64 product
// with the bordered matrix: rows 0..n-1 are the tractions, row n the volume
// row), per collocation point the traction check and its adjustments
// (point_kernel: full separation, cohesive opening, slip, or intact; intact
// points fix their DoF), the truncated system solved (with the full
// system's mixed factors and a capacitance correction, or by factoring the
// truncated system), then the DD and pressures (update_kernel).  The O(n)
// work per point is a few hundred flops; the step's cost is the product
// (8 n^2 bytes) and the solve.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <vector>
#include "engine_internal.h"
#include "hfpx_device.cuh"

namespace hfpx {
namespace {

// Nodal shape functions of the element at its collocation point `cp`:
// the monomials [1, t, conj t, t^2, conj t^2, t conj t] of the point's local
// complex coordinate t, times the element's shape-function matrix (real
// part), as set_ele_struct forms sf_cp (element_utilities.cpp:455-476).
__device__ void shape_at_cp(const ElemRec& E, int cp, double sf[6]) {
  double d[3];
  for (int k = 0; k < 3; ++k) d[k] = E.cp[3 * cp + k] - E.v0[k];
  const double tr = E.r[0] * d[0] + E.r[1] * d[1] + E.r[2] * d[2];
  const double ti = E.r[3] * d[0] + E.r[4] * d[1] + E.r[5] * d[2];
  // monomials (re, im)
  const double mr[6] = {1.0, tr, tr, tr * tr - ti * ti, tr * tr - ti * ti, tr * tr + ti * ti};
  const double mi[6] = {0.0, ti, -ti, 2.0 * tr * ti, -2.0 * tr * ti, 0.0};
  for (int a = 0; a < 6; ++a) {
    double s = 0.0;
    for (int j = 0; j < 6; ++j) s += E.sfm[2 * (6 * a + j)] * mr[j] - E.sfm[2 * (6 * a + j) + 1] * mi[j];
    sf[a] = s;
  }
}

__device__ __forceinline__ void to_local(const double* r, const double* g, double* l) {
  for (int k = 0; k < 3; ++k) l[k] = r[3 * k] * g[0] + r[3 * k + 1] * g[1] + r[3 * k + 2] * g[2];
}
__device__ __forceinline__ void to_global(const double* r, const double* l, double* g) {
  for (int k = 0; k < 3; ++k) g[k] = r[k] * l[0] + r[3 + k] * l[1] + r[6 + k] * l[2];
}

// match_f_c (cohesion_friction.cpp:22-130), one thread per point.  The
// reference keeps its nodal DD in one array shared by the OpenMP threads;
// here each point has its own.
__global__ void match_kernel(int64_t n_cp, const hfpx_cf_material* __restrict__ mats,
                             const int32_t* __restrict__ mat_id, const double* __restrict__ dd,
                             const double* __restrict__ mr_open, const double* __restrict__ mr_slip,
                             double* __restrict__ fric, double* __restrict__ slip_coh, double* __restrict__ open_coh) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= n_cp) return;
  const hfpx_cf_material p = mats[mat_id[n]];
  const double d0 = dd[n], d1 = dd[n + n_cp], d2 = dd[n + 2 * n_cp];
  const double dl_open = d2 / p.cr_open, pr_open = mr_open[n];
  const double dl_slip = sqrt(d0 * d0 + d1 * d1) / p.cr_slip, pr_slip = mr_slip[n];
  double r_s = 0.0;
  if (dl_open > 0.0 && dl_open < 1.0) {
    if (p.cohesion_model == 1) r_s = 1.0 - dl_open;
    else if (p.cohesion_model == 0) r_s = 1.0;
  }
  if (dl_open > 0.0 && dl_open < pr_open) r_s *= dl_open / pr_open;  // linear unloading
  open_coh[n] = p.peak_ts * r_s;
  slip_coh[n] = p.peak_sc * r_s;
  double r_f = 0.0;  // fully opened: no friction
  if (dl_open < 1.0) {
    r_f = p.res_sf;
    if (p.friction_model == 1) {
      if (dl_slip < 1.0) {
        const double m = dl_slip < pr_slip ? pr_slip : dl_slip;
        r_f = p.res_sf + (p.peak_sf - p.res_sf) * (1.0 - m);
      }
    } else if (p.friction_model == 0) {
      r_f = p.peak_sf;
    }
  }
  fric[n] = r_f;
}

// update_mrd (cohesion_friction.cpp:134-194)
__global__ void mrd_kernel(int64_t n_cp, const hfpx_cf_material* __restrict__ mats,
                           const int32_t* __restrict__ mat_id, const double* __restrict__ dd,
                           double* __restrict__ mr_open, double* __restrict__ mr_slip) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= n_cp) return;
  const hfpx_cf_material p = mats[mat_id[n]];
  const double d0 = dd[n], d1 = dd[n + n_cp], d2 = dd[n + 2 * n_cp];
  const double dl_open = d2 / p.cr_open;
  const double dl_slip = sqrt(d0 * d0 + d1 * d1) / p.cr_slip;
  const double pr_open = mr_open[n], pr_slip = mr_slip[n];
  if (dl_slip > pr_slip) mr_slip[n] = dl_slip;
  if (dl_open >= 1.0) mr_open[n] = 1.0;
  if (dl_open > pr_open) mr_open[n] = dl_open;
}

// x[dof] = dd(point, component) over the original numbering, x[n] = 0 (the
// pressure unknown), as get_dd_vector_from_md (surface_mesh_utilities.cpp:
// 193-240) without the pressure block
__global__ void gather_dd_kernel(int64_t n_el, const int32_t* __restrict__ dof, const double* __restrict__ dd,
                                 int64_t n, double* __restrict__ x) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i == 0) x[n] = 0.0;
  if (i >= 18 * n_el) return;
  const int64_t el = i / 18;
  const int l18 = (int)(i - 18 * el);
  const int32_t d = dof[el + n_el * l18];
  if (d >= 0) x[d] = dd[6 * el + l18 / 3 + 6 * n_el * (l18 % 3)];
}

// The traction check of every collocation point (c_f_iteration.cpp:98-271),
// one thread per point.  r = -A [dd; 0] (the product's sign), so the elastic
// traction of DoF d is -r[d].  Writes the traction adjustments (global
// frame, times sign) into dtrac at the point's DoF for the first ncomp
// components, and fixed[18 el + l] = 1 for the DoF of an intact point.
__global__ void point_kernel(const ElemRec* __restrict__ elems, int64_t n_el, const int32_t* __restrict__ dof,
                             const double* __restrict__ dd, const double* __restrict__ pp,
                             const double* __restrict__ mr_open, const double* __restrict__ mr_slip,
                             const double* __restrict__ fric, const double* __restrict__ slip_coh,
                             const double* __restrict__ open_coh, const double* __restrict__ r,
                             const double* __restrict__ sinf, int ncomp, double sign, double* __restrict__ dtrac,
                             int8_t* __restrict__ fixed) {
  const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (g >= 6 * n_el) return;
  const int64_t el = g / 6;
  const int lnn = (int)(g - 6 * el);
  const ElemRec& E = elems[el];
  // in-situ traction on the element (n . s_inf), in local coordinates
  const double* nv = E.nrm;
  const double tg[3] = {nv[0] * sinf[0] + nv[1] * sinf[3] + nv[2] * sinf[4],
                        nv[0] * sinf[3] + nv[1] * sinf[1] + nv[2] * sinf[5],
                        nv[0] * sinf[4] + nv[1] * sinf[5] + nv[2] * sinf[2]};
  double ti[3];
  to_local(E.r, tg, ti);
  double sf[6];
  shape_at_cp(E, lnn, sf);
  double pr = 0.0;
  for (int a = 0; a < 6; ++a) pr += pp[6 * el + a] * sf[a];
  // elastic traction at the point from its DoF
  double trg[3], tr[3];
  int32_t dl[3];
  for (int i = 0; i < 3; ++i) {
    dl[i] = dof[el + n_el * (3 * lnn + i)];
    trg[i] = dl[i] >= 0 ? -r[dl[i]] : 0.0;
  }
  to_local(E.r, trg, tr);
  const double nt = pr - ti[2] - tr[2];
  const double st[2] = {-ti[0] - tr[0], -ti[1] - tr[1]};
  const double sh = sqrt(st[0] * st[0] + st[1] * st[1]);
  const double adm_nt = open_coh[g];
  const double adm_st = slip_coh[g] - fric[g] * nt;
  const double dir[2] = {sh > 0.0 ? st[0] / sh : 0.0, sh > 0.0 ? st[1] / sh : 0.0};
  const double fr_state = mr_open[g], sl_state = mr_slip[g];
  double dt[3] = {0.0, 0.0, 0.0};
  bool intact = false;
  if (nt > adm_nt) {  // full separation: release the normal and the shear traction
    dt[2] = -nt;
    dt[0] = -st[0];
    dt[1] = -st[1];
  } else {
    if (fr_state < 1.0 && nt > 0.0) dt[2] = adm_nt - nt;  // cohesion
    if (sl_state > 0.0 || sh > adm_st) {                   // slip against cohesion + friction
      dt[0] = adm_st * dir[0] - st[0];
      dt[1] = adm_st * dir[1] - st[1];
    } else if (nt <= 0.0) {
      intact = true;
    }
  }
  double dg[3];
  to_global(E.r, dt, dg);
  for (int i = 0; i < ncomp; ++i)
    if (dl[i] >= 0) dtrac[dl[i]] = sign * dg[i];
  for (int i = 0; i < 3; ++i) fixed[18 * el + 3 * lnn + i] = intact ? 1 : 0;
}

// DD and pressure update (c_f_iteration.cpp:314-427), one thread per element.
// x: the increments over the original numbering (0 at fixed DoF).
__global__ void update_kernel(const ElemRec* __restrict__ elems, int64_t n_el, const int32_t* __restrict__ dof,
                              const double* __restrict__ x, int is_dd_local, const hfpx_cf_material* __restrict__ mats,
                              const int32_t* __restrict__ mat_id, const double* __restrict__ mr_open,
                              double pressure, double* __restrict__ dd, double* __restrict__ pp) {
  const int64_t el = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (el >= n_el) return;
  const ElemRec& E = elems[el];
  const int64_t n_cp = 6 * n_el;
  double ddl[6][3];  // nodal DD in local coordinates
  for (int lnn = 0; lnn < 6; ++lnn) {
    const int64_t g = 6 * el + lnn;
    double v[3], w[3];
    int32_t dl[3];
    for (int i = 0; i < 3; ++i) {
      dl[i] = dof[el + n_el * (3 * lnn + i)];
      v[i] = dd[g + n_cp * i];
      if (dl[i] >= 0) v[i] += x[dl[i]];
    }
    if (!is_dd_local) to_local(E.r, v, w);
    else for (int i = 0; i < 3; ++i) w[i] = v[i];
    if (w[2] < 0.0) w[2] = 0.0;  // no overlap
    for (int i = 0; i < 3; ++i) ddl[lnn][i] = w[i];
    if (!is_dd_local) to_global(E.r, w, v);
    else for (int i = 0; i < 3; ++i) v[i] = w[i];
    for (int i = 0; i < 3; ++i)
      if (dl[i] >= 0) dd[g + n_cp * i] = v[i];
  }
  for (int cpe = 0; cpe < 6; ++cpe) {
    const int64_t g = 6 * el + cpe;
    double sf[6];
    shape_at_cp(E, cpe, sf);
    double open = 0.0;
    for (int a = 0; a < 6; ++a) open += ddl[a][2] * sf[a];
    const double fr_state = mr_open[g];
    double st = open / mats[mat_id[g]].cr_open;
    if (st >= 1.0 || fr_state >= 1.0) st = 1.0;
    if (st >= 1.0 || (st > 0.0 && fr_state >= 1.0)) pp[g] = pressure;
  }
}

struct Buf {
  void* p = nullptr;
  ~Buf() {
    if (p) cudaFree(p);
  }
  template <class T>
  T* as() const { return static_cast<T*>(p); }
};

int alloc(hfpx_ctx* c, Buf& b, size_t bytes, const char* what) {
  return check_cuda(c, cudaMalloc(&b.p, bytes > 0 ? bytes : 8), what);
}
int up(hfpx_ctx* c, void* d, const void* h, size_t bytes) {
  return check_cuda(c, cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, c->stream), "upload");
}
int down(hfpx_ctx* c, void* h, const void* d, size_t bytes) {
  return check_cuda(c, cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, c->stream), "download");
}

int check_materials(hfpx_ctx* c, int64_t n_cp, const hfpx_cf_material* mats, int n_mat, const hfpx_cf_state* st) {
  if (n_cp < 1 || !mats || n_mat < 1 || !st || !st->dd || !st->pp || !st->mr_open || !st->mr_slip ||
      !st->friction_coef || !st->slip_cohesion || !st->open_cohesion || !st->mat_id)
    return set_error(c, HFPX_ERR_ARG, "null or empty cohesion/friction argument");
  for (int m = 0; m < n_mat; ++m)
    if (!(mats[m].cr_open > 0.0) || !(mats[m].cr_slip > 0.0))
      return set_error(c, HFPX_ERR_ARG, "critical opening and slip must be positive");
  for (int64_t i = 0; i < n_cp; ++i)
    if (st->mat_id[i] < 0 || st->mat_id[i] >= n_mat) return set_error(c, HFPX_ERR_ARG, "material id out of range");
  return HFPX_OK;
}

// The state arrays on the device: dd (3 n_cp), pp, mr_open, mr_slip, fric,
// slip_coh, open_coh (n_cp each), materials, material ids.
struct DevState {
  Buf dd, pp, mro, mrs, fr, sc, oc, mats, mid;
  int load(hfpx_ctx* c, int64_t n_cp, const hfpx_cf_material* m, int n_mat, const hfpx_cf_state* st) {
    const size_t b = sizeof(double) * n_cp;
    int rc = alloc(c, dd, 3 * b, "dd");
    if (!rc) rc = alloc(c, pp, b, "pp");
    if (!rc) rc = alloc(c, mro, b, "mr_open");
    if (!rc) rc = alloc(c, mrs, b, "mr_slip");
    if (!rc) rc = alloc(c, fr, b, "friction");
    if (!rc) rc = alloc(c, sc, b, "slip cohesion");
    if (!rc) rc = alloc(c, oc, b, "open cohesion");
    if (!rc) rc = alloc(c, mats, sizeof(hfpx_cf_material) * n_mat, "materials");
    if (!rc) rc = alloc(c, mid, sizeof(int32_t) * n_cp, "material ids");
    if (!rc) rc = up(c, dd.p, st->dd, 3 * b);
    if (!rc) rc = up(c, pp.p, st->pp, b);
    if (!rc) rc = up(c, mro.p, st->mr_open, b);
    if (!rc) rc = up(c, mrs.p, st->mr_slip, b);
    if (!rc) rc = up(c, mats.p, m, sizeof(hfpx_cf_material) * n_mat);
    if (!rc) rc = up(c, mid.p, st->mat_id, sizeof(int32_t) * n_cp);
    return rc;
  }
};

unsigned blocks(int64_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace
}  // namespace hfpx

using namespace hfpx;

extern "C" {

int hfpx_cf_match(hfpx_ctx* c, int64_t n_cp, const hfpx_cf_material* mats, int n_mat, hfpx_cf_state* st) {
  if (!c) return HFPX_ERR_ARG;
  if (int rc = check_materials(c, n_cp, mats, n_mat, st)) return rc;
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  DevState s;
  int rc = s.load(c, n_cp, mats, n_mat, st);
  if (!rc) {
    ++g_launches;
    match_kernel<<<blocks(n_cp, 256), 256, 0, c->stream>>>(n_cp, s.mats.as<hfpx_cf_material>(), s.mid.as<int32_t>(),
                                                           s.dd.as<double>(), s.mro.as<double>(), s.mrs.as<double>(),
                                                           s.fr.as<double>(), s.sc.as<double>(), s.oc.as<double>());
    rc = check_cuda(c, cudaGetLastError(), "match_f_c");
  }
  const size_t b = sizeof(double) * n_cp;
  if (!rc) rc = down(c, st->friction_coef, s.fr.p, b);
  if (!rc) rc = down(c, st->slip_cohesion, s.sc.p, b);
  if (!rc) rc = down(c, st->open_cohesion, s.oc.p, b);
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "match_f_c");
  return rc;
}

int hfpx_cf_update_mrd(hfpx_ctx* c, int64_t n_cp, const hfpx_cf_material* mats, int n_mat, hfpx_cf_state* st) {
  if (!c) return HFPX_ERR_ARG;
  if (int rc = check_materials(c, n_cp, mats, n_mat, st)) return rc;
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  DevState s;
  int rc = s.load(c, n_cp, mats, n_mat, st);
  if (!rc) {
    ++g_launches;
    mrd_kernel<<<blocks(n_cp, 256), 256, 0, c->stream>>>(n_cp, s.mats.as<hfpx_cf_material>(), s.mid.as<int32_t>(),
                                                         s.dd.as<double>(), s.mro.as<double>(), s.mrs.as<double>());
    rc = check_cuda(c, cudaGetLastError(), "update_mrd");
  }
  const size_t b = sizeof(double) * n_cp;
  if (!rc) rc = down(c, st->mr_open, s.mro.p, b);
  if (!rc) rc = down(c, st->mr_slip, s.mrs.p, b);
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "update_mrd");
  return rc;
}

int hfpx_vc_cf_iteration(hfpx_ctx* c, const hfpx_mesh* mesh, const hfpx_matrix* m, const int64_t* orig_dof_h,
                         int64_t n_dof, const hfpx_cf_material* mats, int n_mat, const double* s_inf, int64_t inj_cp,
                         double new_vol, int is_dd_local, int flags, double tol, hfpx_cf_state* st,
                         hfpx_cf_info* info) {
  if (!c) return HFPX_ERR_ARG;
  if (!mesh || !m || !orig_dof_h || !s_inf || !info) return set_error(c, HFPX_ERR_ARG, "null argument");
  const int64_t n_el = mesh->n_el, n_cp = 6 * n_el, n = n_dof;
  if (int rc = check_materials(c, n_cp, mats, n_mat, st)) return rc;
  if (m->op_mixed || !m->d_a) return set_error(c, HFPX_ERR_STATE, "the iteration needs the FP64 bordered matrix");
  if (m->factored == 1) return set_error(c, HFPX_ERR_STATE, "the matrix holds FP64 LU factors, not the operator");
  if (m->n != n + 1) return set_error(c, HFPX_ERR_ARG, "the matrix is not the bordered matrix of n_dof unknowns");
  if (inj_cp < 0 || inj_cp >= n_cp) return set_error(c, HFPX_ERR_ARG, "injection point out of range");
  std::vector<int32_t> dof32((size_t)(18 * n_el));
  {
    std::vector<char> seen((size_t)n, 0);
    for (int64_t i = 0; i < 18 * n_el; ++i) {
      const int64_t d = orig_dof_h[i];
      if (d < -1 || d >= n || (d >= 0 && seen[(size_t)d]))
        return set_error(c, HFPX_ERR_ARG, "DoF handle entries must be -1 or distinct indices below n_dof");
      if (d >= 0) seen[(size_t)d] = 1;
      dof32[(size_t)i] = (int32_t)d;
    }
  }
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  *info = hfpx_cf_info{};
  const ElemRec* elems = static_cast<const ElemRec*>(mesh->d_elem);
  DevState s;
  Buf ddof, dx, dr, dsinf, dtr, dfix;
  int rc = s.load(c, n_cp, mats, n_mat, st);
  if (!rc) rc = alloc(c, ddof, sizeof(int32_t) * 18 * n_el, "dof");
  if (!rc) rc = alloc(c, dx, sizeof(double) * (n + 1), "x");
  if (!rc) rc = alloc(c, dr, sizeof(double) * (n + 1), "tractions");
  if (!rc) rc = alloc(c, dsinf, sizeof(double) * 6, "s_inf");
  if (!rc) rc = alloc(c, dtr, sizeof(double) * (n + 1), "traction adjustments");
  if (!rc) rc = alloc(c, dfix, 18 * n_el, "fixed flags");
  if (!rc) rc = up(c, ddof.p, dof32.data(), sizeof(int32_t) * 18 * n_el);
  if (!rc) rc = up(c, dsinf.p, s_inf, sizeof(double) * 6);
  if (!rc) rc = check_cuda(c, cudaMemsetAsync(dtr.p, 0, sizeof(double) * (n + 1), c->stream), "zero");
  // 1. cohesion and friction of the current state (c_f_iteration.cpp:87-89)
  if (!rc) {
    g_launches += 2;
    match_kernel<<<blocks(n_cp, 256), 256, 0, c->stream>>>(n_cp, s.mats.as<hfpx_cf_material>(), s.mid.as<int32_t>(),
                                                           s.dd.as<double>(), s.mro.as<double>(), s.mrs.as<double>(),
                                                           s.fr.as<double>(), s.sc.as<double>(), s.oc.as<double>());
    gather_dd_kernel<<<blocks(18 * n_el, 256), 256, 0, c->stream>>>(n_el, ddof.as<int32_t>(), s.dd.as<double>(), n,
                                                                    dx.as<double>());
    rc = check_cuda(c, cudaGetLastError(), "match_f_c");
  }
  // 2. r = -A [dd; 0]: the elastic tractions (:65-69) and -volume (:71-77)
  if (!rc) rc = hfpx_residual_device(c, m, dx.as<double>(), nullptr, dr.as<double>());
  // 3. the traction check per point (:98-271)
  if (!rc) {
    ++g_launches;
    point_kernel<<<blocks(n_cp, 128), 128, 0, c->stream>>>(
        elems, n_el, ddof.as<int32_t>(), s.dd.as<double>(), s.pp.as<double>(), s.mro.as<double>(),
        s.mrs.as<double>(), s.fr.as<double>(), s.sc.as<double>(), s.oc.as<double>(), dr.as<double>(),
        dsinf.as<double>(), (flags & 1) ? 3 : 2, (flags & 2) ? -1.0 : 1.0, dtr.as<double>(), dfix.as<int8_t>());
    rc = check_cuda(c, cudaGetLastError(), "traction check");
  }
  std::vector<double> b((size_t)(n + 1));
  std::vector<int8_t> fixed_flag((size_t)(18 * n_el));
  double neg_vol = 0.0, pressure = 0.0;
  if (!rc) rc = down(c, b.data(), dtr.p, sizeof(double) * n);
  if (!rc) rc = down(c, fixed_flag.data(), dfix.p, (size_t)(18 * n_el));
  if (!rc) rc = down(c, &neg_vol, dr.as<double>() + n, sizeof(double));
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "traction check");
  if (rc) return rc;
  pressure = st->pp[inj_cp];
  const double volume = -neg_vol, delta_v = new_vol - volume;
  // 4. the DoF of intact points are fixed; the rest are renumbered in order
  // (the truncated handle, :212-258, without the shared counter's race)
  std::vector<char> is_fixed((size_t)n, 0);
  for (int64_t el = 0; el < n_el; ++el)
    for (int l = 0; l < 18; ++l) {
      const int64_t d = orig_dof_h[el + n_el * l];
      if (d >= 0 && fixed_flag[(size_t)(18 * el + l)]) is_fixed[(size_t)d] = 1;
    }
  std::vector<int64_t> fixed, keep, renum((size_t)n, -1);
  for (int64_t d = 0; d < n; ++d) {
    if (is_fixed[(size_t)d]) {
      fixed.push_back(d);
    } else {
      renum[(size_t)d] = (int64_t)keep.size();
      keep.push_back(d);
    }
  }
  const int64_t k = (int64_t)fixed.size(), n_keep = (int64_t)keep.size();
  double l1_trac = 0.0;
  for (int64_t d = 0; d < n; ++d) l1_trac += std::fabs(b[(size_t)d]);
  b[(size_t)n] = delta_v;
  if (n_keep == 0) return set_error(c, HFPX_ERR_SINGULAR, "every DoF is fixed: the truncated system is singular");
  // 5. the truncated system (mod_3dbem_system_vc, system_assembly.cpp:560-629)
  hfpx_solve_info si{};
  // The full system's factors with the capacitance correction cost k + 1
  // refined solves, about 1.4e-12 s n^2 (k + 1) on a B200 (80 ms for
  // n = 17770, k = 183); factoring the truncated system about 2.7e-14 s
  // n_keep^3 (60 ms for n_keep = 13000).  Take the cheaper one.
  const double nd = (double)n, nk = (double)n_keep;
  const bool capacitance = m->factored == 2 && k <= 4096 &&
                           ((flags & 4) || (double)(k + 1) * nd * nd < 0.02 * nk * nk * nk);
  if (capacitance) {
    std::vector<int64_t> fx(fixed);
    rc = hfpx_lu_solve_fixed(c, m, fx.data(), k, b.data(), tol, &si);
    info->solver = 0;
  } else {
    hfpx_matrix* t = nullptr;
    rc = hfpx_matrix_truncate(c, m, keep.data(), n_keep, 1, &t);
    int64_t linfo = 0;
    if (!rc) rc = hfpx_lu_factor(c, t, HFPX_LU_MIXED, &linfo);
    std::vector<double> bt((size_t)(n_keep + 1));
    for (int64_t i = 0; i < n_keep; ++i) bt[(size_t)i] = b[(size_t)keep[(size_t)i]];
    bt[(size_t)n_keep] = delta_v;
    if (!rc) rc = hfpx_lu_solve(c, t, bt.data(), 1, n_keep + 1, tol, 50, &si);
    if (t) hfpx_matrix_destroy(t);
    if (!rc) {
      std::fill(b.begin(), b.end(), 0.0);
      for (int64_t i = 0; i < n_keep; ++i) b[(size_t)keep[(size_t)i]] = bt[(size_t)i];
      b[(size_t)n] = bt[(size_t)n_keep];
    }
    info->solver = 1;
  }
  if (rc) return rc;
  double l1_x = 0.0;
  for (double v : b) l1_x += std::fabs(v);
  const double delta_p = b[(size_t)n];
  pressure += delta_p;
  // 6. DD and pressures (:314-427)
  rc = up(c, dx.p, b.data(), sizeof(double) * (n + 1));
  if (!rc) {
    ++g_launches;
    update_kernel<<<blocks(n_el, 128), 128, 0, c->stream>>>(elems, n_el, ddof.as<int32_t>(), dx.as<double>(),
                                                            is_dd_local, s.mats.as<hfpx_cf_material>(),
                                                            s.mid.as<int32_t>(), s.mro.as<double>(), pressure,
                                                            s.dd.as<double>(), s.pp.as<double>());
    rc = check_cuda(c, cudaGetLastError(), "update");
  }
  const size_t bb = sizeof(double) * n_cp;
  if (!rc) rc = down(c, st->dd, s.dd.p, 3 * bb);
  if (!rc) rc = down(c, st->pp, s.pp.p, bb);
  if (!rc) rc = down(c, st->friction_coef, s.fr.p, bb);
  if (!rc) rc = down(c, st->slip_cohesion, s.sc.p, bb);
  if (!rc) rc = down(c, st->open_cohesion, s.oc.p, bb);
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "update");
  if (rc) return rc;
  if (st->dof_h)
    for (int64_t i = 0; i < 18 * n_el; ++i) {
      const int64_t d = orig_dof_h[i];
      st->dof_h[i] = d >= 0 ? renum[(size_t)d] : -1;
    }
  info->residual = l1_x + l1_trac;
  info->volume = volume;
  info->pressure = pressure;
  info->delta_p = delta_p;
  info->n_dof = n_keep;
  info->n_fixed = k;
  info->refinement = si.iterations;
  return HFPX_OK;
}

}  // extern "C"
