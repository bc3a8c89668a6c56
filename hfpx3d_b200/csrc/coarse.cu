// Coarse level of the two-level near-field preconditioner for flexible GMRES
// on the dense FP64 operator (the matrix make_3dbem_matrix_s fills,
// src/Solvers/system_assembly.cpp:30-219; the reference itself only solves
// directly, il::LU at il/linear_algebra/dense/factorization/LU.h:79-120).
//
// A near-field preconditioner acts on the element scale only, so the
// smooth, crack-wide DD modes converge slowly and the GMRES step count grows
// with the mesh.  The coarse level removes them: the elements are grouped
// into aggregates of about 30 (k-means of the centroids), and on each
// aggregate the three DD components are represented by linear functions in
// the aggregate's tangent plane (1, xi, eta): P is n x nc, nc = 9
// aggregates.  Each step the assembly's operator gives A P (one pass over the
// matrix, from its FP32 copy when current) and the nc x nc coarse operator
// P^T A P, factored by the engine's FP64 LU and inverted.  The preconditioner
// is then
//   c = (P^T A P)^-1 P^T v,  z = P c + M (v - A P c),
// a coarse correction followed by the near-field M on the residual it leaves
// (the multiplicative two-level form).  Per GMRES step this costs one pass
// over A P (n x nc) and the near-field product; the matrix itself is not
// read again.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>
#include <type_traits>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "engine_internal.h"

namespace hfpx {
namespace {

constexpr int kApThreads = 128;

// A P for the columns of one aggregate (blockIdx.y): each thread R rows,
// 9 accumulators per row (basis m, DD component k at 3 m + k).
template <class T, int R>
__global__ void __launch_bounds__(kApThreads) ap_kernel(const T* __restrict__ A, int64_t lda, int64_t n,
                                                        const int32_t* __restrict__ ptr,
                                                        const int32_t* __restrict__ el,
                                                        const double* __restrict__ w, double* __restrict__ AP) {
  extern __shared__ double s_w[];  // the aggregate's elements x 18 weights, then their ids
  const int a = blockIdx.y;
  const int e0 = ptr[a], cnt = ptr[a + 1] - e0;
  int32_t* s_el = reinterpret_cast<int32_t*>(s_w + 18 * cnt);
  for (int i = threadIdx.x; i < cnt; i += kApThreads) s_el[i] = el[e0 + i];
  __syncthreads();
  for (int i = threadIdx.x; i < 18 * cnt; i += kApThreads) s_w[i] = w[(int64_t)s_el[i / 18] * 18 + i % 18];
  __syncthreads();
  const int64_t r0 = ((int64_t)blockIdx.x * kApThreads + threadIdx.x) * R;
  if (r0 >= n) return;
  double acc[R][9];
#pragma unroll
  for (int i = 0; i < R; ++i)
#pragma unroll
    for (int j = 0; j < 9; ++j) acc[i][j] = 0.0;
  if (r0 + R <= n) {
    // whole rows: each element's 18 column loads issued before their products
    using V = typename std::conditional<R == 4, float4, double2>::type;
    for (int le = 0; le < cnt; ++le) {
      const T* col = A + r0 + lda * (18 * (int64_t)s_el[le]);
      const double* wl = s_w + 18 * le;
#pragma unroll
      for (int half = 0; half < 2; ++half) {  // nodes 0-2, then 3-5: 9 loads in flight
        V q[9];
#pragma unroll
        for (int u = 0; u < 9; ++u) q[u] = __ldcs(reinterpret_cast<const V*>(col + lda * (9 * half + u)));
#pragma unroll
        for (int u = 0; u < 9; ++u) {
          const int k = u % 3, node = 3 * half + u / 3;
          double v[R];
          if constexpr (R == 4) {
            v[0] = q[u].x; v[1] = q[u].y; v[2] = q[u].z; v[3] = q[u].w;
          } else {
            v[0] = q[u].x; v[1] = q[u].y;
          }
          const double w0 = wl[3 * node], w1 = wl[3 * node + 1], w2 = wl[3 * node + 2];
#pragma unroll
          for (int i = 0; i < R; ++i) {
            acc[i][k] = fma(v[i], w0, acc[i][k]);
            acc[i][3 + k] = fma(v[i], w1, acc[i][3 + k]);
            acc[i][6 + k] = fma(v[i], w2, acc[i][6 + k]);
          }
        }
      }
    }
  } else {
    for (int le = 0; le < cnt; ++le) {
      const T* col = A + r0 + lda * (18 * (int64_t)s_el[le]);
      const double* wl = s_w + 18 * le;
#pragma unroll
      for (int cidx = 0; cidx < 18; ++cidx) {
        const int k = cidx % 3, node = cidx / 3;
        const double w0 = wl[3 * node], w1 = wl[3 * node + 1], w2 = wl[3 * node + 2];
#pragma unroll
        for (int i = 0; i < R; ++i)
          if (r0 + i < n) {
            const double v = (double)col[lda * cidx + i];
            acc[i][k] = fma(v, w0, acc[i][k]);
            acc[i][3 + k] = fma(v, w1, acc[i][3 + k]);
            acc[i][6 + k] = fma(v, w2, acc[i][6 + k]);
          }
      }
    }
  }
#pragma unroll
  for (int j = 0; j < 9; ++j)
#pragma unroll
    for (int i = 0; i < R; ++i)
      if (r0 + i < n) AP[(r0 + i) + n * (9 * (int64_t)a + j)] = acc[i][j];
}

// P^T (A P): rows 9 a .. 9 a + 8 (blockIdx.y = a), one column J per thread.
__global__ void coarse_matrix_kernel(const double* __restrict__ AP, int64_t n, int64_t nc,
                                     const int32_t* __restrict__ ptr, const int32_t* __restrict__ el,
                                     const double* __restrict__ w, double* __restrict__ Ac, int64_t ldc) {
  const int a = blockIdx.y;
  const int64_t J = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (J >= nc) return;
  const double* col = AP + n * J;
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = ptr[a]; i < ptr[a + 1]; ++i) {
    const int64_t e = el[i];
    const double* we = w + 18 * e;
#pragma unroll
    for (int node = 0; node < 6; ++node)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double v = col[18 * e + 3 * node + k];
        acc[k] = fma(we[3 * node], v, acc[k]);
        acc[3 + k] = fma(we[3 * node + 1], v, acc[3 + k]);
        acc[6 + k] = fma(we[3 * node + 2], v, acc[6 + k]);
      }
  }
#pragma unroll
  for (int j = 0; j < 9; ++j) Ac[(9 * (int64_t)a + j) + ldc * J] = acc[j];
}

// q = P^T v: one block per aggregate, fixed-order tree reduction.
constexpr int kRThreads = 128;
__global__ void __launch_bounds__(kRThreads) restrict_kernel(const double* __restrict__ v,
                                                             const int32_t* __restrict__ ptr,
                                                             const int32_t* __restrict__ el,
                                                             const double* __restrict__ w, double* __restrict__ q) {
  __shared__ double red[9][kRThreads];
  const int a = blockIdx.x;
  const int e0 = ptr[a], cnt = ptr[a + 1] - e0;
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int idx = threadIdx.x; idx < 6 * cnt; idx += kRThreads) {
    const int64_t e = el[e0 + idx / 6];
    const int node = idx % 6;
    const double* we = w + 18 * e + 3 * node;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double x = v[18 * e + 3 * node + k];
      acc[k] = fma(we[0], x, acc[k]);
      acc[3 + k] = fma(we[1], x, acc[3 + k]);
      acc[6 + k] = fma(we[2], x, acc[6 + k]);
    }
  }
#pragma unroll
  for (int j = 0; j < 9; ++j) red[j][threadIdx.x] = acc[j];
  __syncthreads();
  for (int s = kRThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
#pragma unroll
      for (int j = 0; j < 9; ++j) red[j][threadIdx.x] += red[j][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x < 9) q[9 * a + threadIdx.x] = red[threadIdx.x][0];
}

// z += P c
__global__ void prolong_add_kernel(const double* __restrict__ cc, const int32_t* __restrict__ agg_of,
                                   const double* __restrict__ w, int64_t n, double* __restrict__ z) {
  const int64_t d = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= n) return;
  const int64_t e = d / 18;
  const int r = (int)(d - 18 * e), node = r / 3, k = r % 3;
  const int64_t a = agg_of[e];
  const double* we = w + 18 * e + 3 * node;
  z[d] += we[0] * cc[9 * a + k] + we[1] * cc[9 * a + 3 + k] + we[2] * cc[9 * a + 6 + k];
}

__global__ void identity_kernel(double* X, int64_t nc) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nc) X[i + nc * i] = 1.0;
}

}  // namespace

int env_agg_size() {
  if (const char* e = std::getenv("HFPX_PC_AGG")) {
    const int v = std::atoi(e);
    if (v >= 1 && v <= 100000) return v;
  }
  return 30;
}

// k-means of the element centroids (farthest-point start from element 0,
// Lloyd steps), then per aggregate a tangent frame and the basis values at
// the six element nodes (vertices, then the edge nodes opposite them).
bool build_coarse(const hfpx_mesh* m, int agg_size, CoarseSpace* cs) {
  const int64_t ne = m->n_el;
  if ((int64_t)m->h_vert.size() < 9 * ne) return false;
  const double* V = m->h_vert.data();
  std::vector<double> cen(3 * ne), nrm(3 * ne);
  for (int64_t e = 0; e < ne; ++e) {
    const double* v = V + 9 * e;
    double u[3], t[3];
    for (int k = 0; k < 3; ++k) {
      cen[3 * e + k] = (v[k] + v[3 + k] + v[6 + k]) / 3.0;
      u[k] = v[3 + k] - v[k];
      t[k] = v[6 + k] - v[k];
    }
    nrm[3 * e] = u[1] * t[2] - u[2] * t[1];  // twice the area times the unit normal
    nrm[3 * e + 1] = u[2] * t[0] - u[0] * t[2];
    nrm[3 * e + 2] = u[0] * t[1] - u[1] * t[0];
  }
  int64_t na = std::max<int64_t>(1, (ne + agg_size / 2) / agg_size);
  na = std::min(na, ne);
  auto d2 = [&](int64_t e, const double* c) {
    const double x = cen[3 * e] - c[0], y = cen[3 * e + 1] - c[1], z = cen[3 * e + 2] - c[2];
    return x * x + y * y + z * z;
  };
  std::vector<double> C(3 * na);
  std::vector<double> dmin(ne, 1e300);
  int64_t pick = 0;
  for (int64_t a = 0; a < na; ++a) {
    for (int k = 0; k < 3; ++k) C[3 * a + k] = cen[3 * pick + k];
    double best = -1.0;
    for (int64_t e = 0; e < ne; ++e) {
      dmin[e] = std::min(dmin[e], d2(e, &C[3 * a]));
      if (dmin[e] > best) {
        best = dmin[e];
        pick = e;
      }
    }
  }
  std::vector<int32_t> lab(ne, 0);
  std::vector<double> sum(3 * na);
  std::vector<int64_t> cnt(na);
  std::vector<int32_t> order(na);
  std::vector<double> ox(na);
  for (int it = 0; it < 6; ++it) {  // a few Lloyd steps: the aggregates need to be compact, not optimal
    bool moved = false;
    // The nearest centre of each centroid (the lowest index among equal
    // distances): centres sorted by x and searched outward from the
    // centroid's x, each direction ending where dx^2 alone exceeds the best
    // distance (d2 >= dx^2 in floating point too, so the pruned centres are
    // strictly farther and the choice is the full scan's).
    for (int64_t a = 0; a < na; ++a) order[a] = (int32_t)a;
    std::sort(order.begin(), order.end(), [&](int32_t u, int32_t v) {
      return C[3 * u] < C[3 * v] || (C[3 * u] == C[3 * v] && u < v);
    });
    for (int64_t a = 0; a < na; ++a) ox[a] = C[3 * order[a]];
    for (int64_t e = 0; e < ne; ++e) {
      int32_t best = -1;
      double bd = 1e300;
      auto visit = [&](int64_t q) {
        const int32_t a = order[q];
        const double d = d2(e, &C[3 * a]);
        if (d < bd || (d == bd && a < best)) {
          bd = d;
          best = a;
        }
      };
      const double x = cen[3 * e];
      const int64_t p = std::lower_bound(ox.begin(), ox.end(), x) - ox.begin();
      for (int64_t q = p; q < na; ++q) {
        const double dx = cen[3 * e] - ox[q];
        if (dx * dx > bd) break;
        visit(q);
      }
      for (int64_t q = p - 1; q >= 0; --q) {
        const double dx = cen[3 * e] - ox[q];
        if (dx * dx > bd) break;
        visit(q);
      }
      moved = moved || best != lab[e];
      lab[e] = best;
    }
    if (!moved && it > 0) break;
    std::fill(sum.begin(), sum.end(), 0.0);
    std::fill(cnt.begin(), cnt.end(), 0);
    for (int64_t e = 0; e < ne; ++e) {
      for (int k = 0; k < 3; ++k) sum[3 * lab[e] + k] += cen[3 * e + k];
      ++cnt[lab[e]];
    }
    for (int64_t a = 0; a < na; ++a)
      if (cnt[a])
        for (int k = 0; k < 3; ++k) C[3 * a + k] = sum[3 * a + k] / (double)cnt[a];
  }
  // drop empty aggregates, number the rest in order
  std::fill(cnt.begin(), cnt.end(), 0);
  for (int64_t e = 0; e < ne; ++e) ++cnt[lab[e]];
  std::vector<int32_t> renum(na, -1);
  int64_t used = 0;
  for (int64_t a = 0; a < na; ++a)
    if (cnt[a]) renum[a] = (int32_t)used++;
  cs->n_el = ne;
  cs->agg_size = agg_size;
  cs->n_agg = used;
  cs->nc = 9 * used;
  cs->agg_of.assign(ne, 0);
  cs->ptr.assign(used + 1, 0);
  for (int64_t e = 0; e < ne; ++e) {
    cs->agg_of[e] = renum[lab[e]];
    ++cs->ptr[cs->agg_of[e] + 1];
  }
  for (int64_t a = 0; a < used; ++a) cs->ptr[a + 1] += cs->ptr[a];
  cs->el.assign(ne, 0);
  std::vector<int32_t> fill(cs->ptr.begin(), cs->ptr.end() - 1);
  for (int64_t e = 0; e < ne; ++e) cs->el[fill[cs->agg_of[e]]++] = (int32_t)e;
  cs->max_agg = 0;
  for (int64_t a = 0; a < used; ++a) cs->max_agg = std::max(cs->max_agg, cs->ptr[a + 1] - cs->ptr[a]);
  // frames: centre, summed (area-weighted) normal, two tangents, radius
  cs->w.assign(18 * ne, 0.0);
  for (int64_t a = 0; a < used; ++a) {
    double c[3] = {0, 0, 0}, nn[3] = {0, 0, 0};
    const int32_t b0 = cs->ptr[a], b1 = cs->ptr[a + 1];
    for (int32_t i = b0; i < b1; ++i)
      for (int k = 0; k < 3; ++k) {
        c[k] += cen[3 * cs->el[i] + k] / (double)(b1 - b0);
        nn[k] += nrm[3 * cs->el[i] + k];
      }
    double ln = std::sqrt(nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2]);
    if (!(ln > 0.0)) {
      nn[0] = nn[1] = 0.0;
      nn[2] = ln = 1.0;
    }
    for (double& x : nn) x /= ln;
    // t1: the coordinate axis least parallel to the normal, made orthogonal
    int ax = 0;
    for (int k = 1; k < 3; ++k)
      if (std::fabs(nn[k]) < std::fabs(nn[ax])) ax = k;
    double t1[3] = {0, 0, 0}, t2[3];
    t1[ax] = 1.0;
    const double dp = t1[0] * nn[0] + t1[1] * nn[1] + t1[2] * nn[2];
    for (int k = 0; k < 3; ++k) t1[k] -= dp * nn[k];
    const double l1 = std::sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
    for (double& x : t1) x /= l1;
    t2[0] = nn[1] * t1[2] - nn[2] * t1[1];
    t2[1] = nn[2] * t1[0] - nn[0] * t1[2];
    t2[2] = nn[0] * t1[1] - nn[1] * t1[0];
    double rad = 0.0;
    for (int32_t i = b0; i < b1; ++i)
      for (int j = 0; j < 3; ++j) {
        const double* p = V + 9 * cs->el[i] + 3 * j;
        const double x = p[0] - c[0], y = p[1] - c[1], z = p[2] - c[2];
        rad = std::max(rad, std::sqrt(x * x + y * y + z * z));
      }
    if (!(rad > 0.0)) rad = 1.0;
    for (int32_t i = b0; i < b1; ++i) {
      const int64_t e = cs->el[i];
      const double* v = V + 9 * e;
      for (int node = 0; node < 6; ++node) {
        double p[3];
        for (int k = 0; k < 3; ++k)
          p[k] = node < 3 ? v[3 * node + k] : 0.5 * (v[3 * ((node - 2) % 3) + k] + v[3 * ((node - 1) % 3) + k]);
        const double x = p[0] - c[0], y = p[1] - c[1], z = p[2] - c[2];
        double* we = &cs->w[18 * e + 3 * node];
        we[0] = 1.0;
        we[1] = (x * t1[0] + y * t1[1] + z * t1[2]) / rad;
        we[2] = (x * t2[0] + y * t2[1] + z * t2[2]) / rad;
      }
    }
  }
  return true;
}

namespace {

void free_coarse(CoarseSpace* cs) {
  void* ps[] = {(void*)cs->d_ptr, (void*)cs->d_el, (void*)cs->d_agg_of, (void*)cs->d_w};
  pool_free_many(ps, 4);
  cs->d_ptr = cs->d_el = cs->d_agg_of = nullptr;
  cs->d_w = nullptr;
}

template <class T>
int upload(hfpx_ctx* c, T** d, const std::vector<T>& h, const char* what) {
  int rc = pool_alloc(c, (void**)d, sizeof(T) * std::max<size_t>(1, h.size()), what);
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, c->stream), what);
  return rc;
}

}  // namespace

std::shared_ptr<CoarseSpace> mesh_coarse(hfpx_ctx* c, const hfpx_mesh* mesh, int agg_size) {
  hfpx_mesh* mm = const_cast<hfpx_mesh*>(mesh);
  if (!mm->coarse || mm->coarse->agg_size != agg_size) {
    std::shared_ptr<CoarseSpace> p(new (std::nothrow) CoarseSpace, [](CoarseSpace* q) {
      free_coarse(q);
      delete q;
    });
    if (!p) return nullptr;
    MeshHostSetup* hs = mm->host_setup.get();
    bool ready = false;
    if (hs && agg_size == env_agg_size()) {  // made on the mesh's set-up thread
      const SetupClock::time_point t0 = SetupClock::now();
      hs->wait(2);
      setup_note("coarse aggregates and basis (wait for the set-up thread)", ms_since(t0));
      if (hs->coarse_ok && hs->coarse.agg_size == agg_size) {
        const CoarseSpace& h = hs->coarse;
        p->n_el = h.n_el;
        p->n_agg = h.n_agg;
        p->nc = h.nc;
        p->agg_size = h.agg_size;
        p->max_agg = h.max_agg;
        p->agg_of = h.agg_of;
        p->ptr = h.ptr;
        p->el = h.el;
        p->w = h.w;
        ready = true;
      }
    }
    if (!ready) {
      const SetupClock::time_point t0 = SetupClock::now();
      if (!build_coarse(mesh, agg_size, p.get())) return nullptr;
      setup_note("coarse aggregates and basis", ms_since(t0));
    }
    int rc = upload(c, &p->d_ptr, p->ptr, "coarse space");
    if (!rc) rc = upload(c, &p->d_el, p->el, "coarse space");
    if (!rc) rc = upload(c, &p->d_agg_of, p->agg_of, "coarse space");
    if (!rc) rc = upload(c, &p->d_w, p->w, "coarse space");
    if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "coarse space");
    if (rc) return nullptr;
    mm->coarse = p;
  }
  return mm->coarse;
}

int coarse_alloc(hfpx_ctx* c, hfpx_precond* pc) {
  pc->cs = mesh_coarse(c, pc->mesh, env_agg_size());
  if (!pc->cs) return set_error(c, HFPX_ERR_NOMEM, "coarse space");
  const int64_t n = pc->n, nc = pc->cs->nc;
  if (!c->cusolver) {
    cusolverDnHandle_t h = nullptr;
    if (cusolverDnCreate(&h) != CUSOLVER_STATUS_SUCCESS) return set_error(c, HFPX_ERR_CUDA, "cuSOLVER handle");
    cusolverDnSetStream(h, c->stream);
    c->cusolver = h;
  }
  int lwork = 0;
  if (cusolverDnDgetrf_bufferSize(static_cast<cusolverDnHandle_t>(c->cusolver), (int)nc, (int)nc, nullptr, (int)nc,
                                  &lwork) != CUSOLVER_STATUS_SUCCESS)
    return set_error(c, HFPX_ERR_CUDA, "coarse LU workspace");
  pc->acwork_bytes = sizeof(double) * (size_t)std::max(1, lwork);
  int rc = pool_alloc(c, (void**)&pc->d_ap, sizeof(double) * n * nc, "A P");
  if (!rc) rc = pool_alloc(c, (void**)&pc->d_ac, sizeof(double) * nc * nc, "coarse operator");
  if (!rc) rc = pool_alloc(c, (void**)&pc->d_acpiv, sizeof(int32_t) * nc, "coarse pivots");
  if (!rc) rc = pool_alloc(c, (void**)&pc->d_acinfo, sizeof(int), "coarse status");
  if (!rc) rc = pool_alloc(c, &pc->d_acwork, pc->acwork_bytes, "coarse LU workspace");
  if (!rc) rc = pool_alloc(c, (void**)&pc->d_acinv, sizeof(double) * nc * nc, "coarse inverse");
  if (!rc) rc = pool_alloc(c, (void**)&pc->d_q, sizeof(double) * nc, "coarse vectors");
  if (!rc) rc = pool_alloc(c, (void**)&pc->d_cc, sizeof(double) * nc, "coarse vectors");
  if (!rc) rc = pool_alloc(c, (void**)&pc->d_t, sizeof(double) * n, "coarse vectors");
  return rc;
}

void coarse_free(hfpx_precond* pc) {
  void* ps[] = {(void*)pc->d_ap, (void*)pc->d_ac, (void*)pc->d_acpiv, (void*)pc->d_acinfo, pc->d_acwork,
                (void*)pc->d_acinv, (void*)pc->d_q, (void*)pc->d_cc, (void*)pc->d_t};
  pool_free_many(ps, 9);
  pc->d_ap = pc->d_ac = pc->d_acinv = pc->d_q = pc->d_cc = pc->d_t = nullptr;
  pc->d_acpiv = nullptr;
  pc->d_acinfo = nullptr;
  pc->d_acwork = nullptr;
  pc->cs.reset();
}

// HFPX_PROFILE=1: event times of the coarse set-up's phases to stderr
static bool coarse_profile() {
  static const bool on = [] {
    const char* e = std::getenv("HFPX_PROFILE");
    return e && *e == '1';
  }();
  return on;
}

int coarse_setup(hfpx_ctx* c, hfpx_precond* pc, const hfpx_matrix* m) {
  const CoarseSpace& cs = *pc->cs;
  const size_t smem = sizeof(double) * 18 * cs.max_agg + sizeof(int32_t) * cs.max_agg;
  if (smem > 200 * 1024) return set_error(c, HFPX_ERR_ARG, "an aggregate too large for the coarse pass");
  cudaEvent_t ev[5] = {};
  const bool prof = coarse_profile();
  if (prof)
    for (auto& e : ev) cudaEventCreate(&e);
  auto mark = [&](int i) {
    if (prof) cudaEventRecord(ev[i], c->stream);
  };
  mark(0);
  const int64_t n = pc->n, nc = cs.nc;
  ++g_launches;
  if (m->d_f && m->f32_current) {
    constexpr int R = 4;
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(ap_kernel<float, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const dim3 grid((unsigned)((n + R * kApThreads - 1) / (R * kApThreads)), (unsigned)cs.n_agg);
    ap_kernel<float, R><<<grid, kApThreads, smem, c->stream>>>(m->d_f, m->ld, n, cs.d_ptr, cs.d_el, cs.d_w, pc->d_ap);
  } else {
    constexpr int R = 2;
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(ap_kernel<double, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const dim3 grid((unsigned)((n + R * kApThreads - 1) / (R * kApThreads)), (unsigned)cs.n_agg);
    ap_kernel<double, R><<<grid, kApThreads, smem, c->stream>>>(m->d_a, m->ld, n, cs.d_ptr, cs.d_el, cs.d_w,
                                                                pc->d_ap);
  }
  int rc = check_cuda(c, cudaGetLastError(), "A P");
  mark(1);
  if (!rc) {
    ++g_launches;
    coarse_matrix_kernel<<<dim3((unsigned)((nc + 127) / 128), (unsigned)cs.n_agg), 128, 0, c->stream>>>(
        pc->d_ap, n, nc, cs.d_ptr, cs.d_el, cs.d_w, pc->d_ac, nc);
    rc = check_cuda(c, cudaGetLastError(), "coarse operator");
  }
  mark(2);
  // LU of the coarse operator (cuSOLVER's dense getrf: a library
  // factorisation of an nc x nc matrix that lives in L2), then its explicit
  // inverse by getrs on the identity
  cusolverDnHandle_t hs = static_cast<cusolverDnHandle_t>(c->cusolver);
  cusolverDnSetStream(hs, c->stream);
  if (!rc && cusolverDnDgetrf(hs, (int)nc, (int)nc, pc->d_ac, (int)nc, static_cast<double*>(pc->d_acwork),
                              pc->d_acpiv, pc->d_acinfo) != CUSOLVER_STATUS_SUCCESS)
    rc = set_error(c, HFPX_ERR_CUDA, "coarse LU");
  int hinfo = 0;
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(&hinfo, pc->d_acinfo, sizeof(int), cudaMemcpyDeviceToHost, c->stream),
                           "coarse status");
  if (!rc) rc = check_cuda(c, cudaMemsetAsync(pc->d_acinv, 0, sizeof(double) * nc * nc, c->stream), "coarse inverse");
  if (!rc) {
    ++g_launches;
    identity_kernel<<<(unsigned)((nc + 255) / 256), 256, 0, c->stream>>>(pc->d_acinv, nc);
    rc = check_cuda(c, cudaStreamSynchronize(c->stream), "coarse LU");
  }
  if (!rc && hinfo != 0) rc = set_error(c, HFPX_ERR_SINGULAR, "the coarse operator is singular");
  mark(3);
  if (!rc && cusolverDnDgetrs(hs, CUBLAS_OP_N, (int)nc, (int)nc, pc->d_ac, (int)nc, pc->d_acpiv, pc->d_acinv, (int)nc,
                              pc->d_acinfo) != CUSOLVER_STATUS_SUCCESS)
    rc = set_error(c, HFPX_ERR_CUDA, "coarse inverse");
  mark(4);
  if (prof) {
    cudaEventSynchronize(ev[4]);
    float t[4] = {0, 0, 0, 0};
    for (int i = 0; i < 4; ++i) cudaEventElapsedTime(&t[i], ev[i], ev[i + 1]);
    std::fprintf(stderr, "[hfpx profile] coarse set-up (%lld aggregates, nc %lld): A P %.3f ms, P^T A P %.3f ms, "
                 "LU %.3f ms, inverse %.3f ms\n", (long long)cs.n_agg, (long long)nc, t[0], t[1], t[2], t[3]);
    for (auto& e : ev) cudaEventDestroy(e);
  }
  return rc;
}

int coarse_apply(hfpx_ctx* c, const hfpx_precond* pc, const double* v, double* z) {
  const CoarseSpace& cs = *pc->cs;
  const int64_t n = pc->n, nc = cs.nc;
  cublasHandle_t h = static_cast<cublasHandle_t>(c->cublas);
  const double one = 1.0, zero = 0.0, mone = -1.0;
  ++g_launches;
  restrict_kernel<<<(unsigned)cs.n_agg, kRThreads, 0, c->stream>>>(v, cs.d_ptr, cs.d_el, cs.d_w, pc->d_q);
  int rc = check_cuda(c, cudaGetLastError(), "coarse restriction");
  if (!rc && cublasDgemv(h, CUBLAS_OP_N, (int)nc, (int)nc, &one, pc->d_acinv, (int)nc, pc->d_q, 1, &zero, pc->d_cc,
                         1) != CUBLAS_STATUS_SUCCESS)
    rc = set_error(c, HFPX_ERR_CUDA, "coarse solve");
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(pc->d_t, v, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream), "t");
  if (!rc && cublasDgemv(h, CUBLAS_OP_N, (int)n, (int)nc, &mone, pc->d_ap, (int)n, pc->d_cc, 1, &one, pc->d_t, 1) !=
                 CUBLAS_STATUS_SUCCESS)
    rc = set_error(c, HFPX_ERR_CUDA, "v - A P c");
  if (!rc) rc = precond_apply_near(c, pc, pc->d_t, z);
  if (!rc) {
    ++g_launches;
    prolong_add_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(pc->d_cc, cs.d_agg_of, cs.d_w, n, z);
    rc = check_cuda(c, cudaGetLastError(), "coarse prolongation");
  }
  return rc;
}

}  // namespace hfpx

using namespace hfpx;

extern "C" int hfpx_precond_coarse(hfpx_ctx* c, const hfpx_precond* pc, int64_t* n_agg, int32_t* agg_of_el,
                                   double* weights, double* ap, double* acinv) {
  if (!c) return HFPX_ERR_ARG;
  if (!pc || !n_agg) return set_error(c, HFPX_ERR_ARG, "null preconditioner");
  if (!pc->cs) return set_error(c, HFPX_ERR_STATE, "the preconditioner has no coarse level");
  const CoarseSpace& cs = *pc->cs;
  *n_agg = cs.n_agg;
  if (agg_of_el) std::copy(cs.agg_of.begin(), cs.agg_of.end(), agg_of_el);
  if (weights) std::copy(cs.w.begin(), cs.w.end(), weights);
  if (!ap && !acinv) return HFPX_OK;
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  int rc = 0;
  if (ap)
    rc = check_cuda(c, cudaMemcpyAsync(ap, pc->d_ap, sizeof(double) * pc->n * cs.nc, cudaMemcpyDeviceToHost, c->stream),
                    "A P");
  if (!rc && acinv)
    rc = check_cuda(c, cudaMemcpyAsync(acinv, pc->d_acinv, sizeof(double) * cs.nc * cs.nc, cudaMemcpyDeviceToHost,
                                       c->stream),
                    "coarse inverse");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "coarse download");
  return rc;
}
