// C-ABI of the engine (include/hfpx_engine.h): objects, argument checks,
// host<->device copies around the kernels of assembly.cu and lu.cu.
#include <cublas_v2.h>
#include <cusolverDn.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>
#include "engine_internal.h"

namespace hfpx {

std::atomic<long long> g_launches{0};

bool setup_profile() {
  static const bool on = [] {
    const char* e = std::getenv("HFPX_PROFILE");
    return e && *e == '1';
  }();
  return on;
}

void setup_note(const char* what, double ms) {
  if (setup_profile()) std::fprintf(stderr, "[hfpx profile] %s: %.3f ms (host)\n", what, ms);
}

void* ctx_scratch(hfpx_ctx* c, int slot, size_t bytes) {
  static_assert(kScrCount <= hfpx_ctx::kScratchSlots, "scratch slots");
  if (slot < 0 || slot >= hfpx_ctx::kScratchSlots) return nullptr;
  if (bytes == 0) bytes = 1;
  if (c->scratch[slot] && c->scratch_bytes[slot] >= bytes) return c->scratch[slot];
  if (c->scratch[slot]) {
    // earlier work queued on the context's streams may still read it
    cudaStreamSynchronize(c->stream);
    cudaStreamSynchronize(c->stream_panel);
    cudaStreamSynchronize(c->stream_left);
    cudaFree(c->scratch[slot]);
    c->scratch[slot] = nullptr;
    c->scratch_bytes[slot] = 0;
  }
  void* p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  c->scratch[slot] = p;
  c->scratch_bytes[slot] = bytes;
  return p;
}

int set_error(hfpx_ctx* c, int code, const std::string& msg) {
  if (c) c->last_error = msg;
  return code;
}

int check_cuda(hfpx_ctx* c, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return HFPX_OK;
  return set_error(c, e == cudaErrorMemoryAllocation ? HFPX_ERR_NOMEM : HFPX_ERR_CUDA,
                   std::string(what) + ": " + cudaGetErrorString(e));
}

// RAII device buffer for per-call temporaries.
struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
  cudaError_t alloc(size_t bytes) { return cudaMalloc(&p, bytes ? bytes : 16); }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

// A context scratch buffer with DevBuf's interface: grown on first use and
// kept, so the host-buffer entry points allocate nothing in steady state.
struct ScratchBuf {
  hfpx_ctx* c;
  int slot;
  void* p = nullptr;
  ScratchBuf(hfpx_ctx* ctx, int s) : c(ctx), slot(s) {}
  cudaError_t alloc(size_t bytes) {
    p = ctx_scratch(c, slot, bytes ? bytes : 16);
    return p ? cudaSuccess : cudaErrorMemoryAllocation;
  }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

// dof_h (int64, n_el x 18) to int32 in the context's dof buffer.
static int upload_dof(hfpx_ctx* c, const int64_t* dof_h, int64_t n_el, int64_t n_dof, int32_t** d) {
  std::vector<int32_t> tmp(18 * n_el);
  for (int64_t i = 0; i < 18 * n_el; ++i) {
    const int64_t v = dof_h[i];
    if (v < -1 || v >= n_dof) return set_error(c, HFPX_ERR_ARG, "dof_h entry out of range");
    tmp[i] = (int32_t)v;
  }
  *d = (int32_t*)ctx_scratch(c, kScrDof, sizeof(int32_t) * tmp.size());
  if (!*d) return set_error(c, HFPX_ERR_NOMEM, "dof_h alloc");
  int rc = check_cuda(c, cudaMemcpyAsync(*d, tmp.data(), sizeof(int32_t) * tmp.size(), cudaMemcpyHostToDevice, c->stream), "dof_h copy");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "dof_h copy");
  return rc;
}

static int64_t round_ld(int64_t n) { return ((n + 31) / 32) * 32; }

}  // namespace hfpx

using namespace hfpx;

namespace hfpx {
// The set-up thread of a mesh: pattern, coarse space, network inputs (host),
// each part published as it finishes.  Failures (allocation) leave the part
// to be made where it is needed.
void start_mesh_setup(hfpx_mesh* m) {
  if (m->n_el < kMeshSetupMinElems) return;
  std::unique_ptr<MeshHostSetup> hs(new (std::nothrow) MeshHostSetup);
  if (!hs) return;
  MeshHostSetup* s = hs.get();
  auto publish = [s](int part, bool ok) {
    {
      std::lock_guard<std::mutex> l(s->mu);
      if (part == 1) s->pattern_ok = ok;
      if (part == 2) s->coarse_ok = ok;
      if (part == 3) s->graph_ok = ok;
      s->done = part;
    }
    s->cv.notify_all();
  };
  try {
    s->worker = std::thread([m, s, publish] {
      SetupClock::time_point t0 = SetupClock::now();
      bool ok = false;
      try {
        ok = pattern_host(m, &s->pattern);
      } catch (...) {
        ok = false;
      }
      publish(1, ok);
      setup_note("set-up thread: pattern", ms_since(t0));
      t0 = SetupClock::now();
      const bool pat_ok = ok;
      ok = false;
      try {
        ok = build_coarse(m, env_agg_size(), &s->coarse);
      } catch (...) {
        ok = false;
      }
      publish(2, ok);
      setup_note("set-up thread: coarse space", ms_since(t0));
      t0 = SetupClock::now();
      ok = false;
      try {
        ok = pat_ok && graph_host_inputs(m, s->pattern, &s->graph);
      } catch (...) {
        ok = false;
      }
      publish(3, ok);
      setup_note("set-up thread: network inputs", ms_since(t0));
    });
  } catch (...) {
    return;  // no thread: every part is made where it is needed
  }
  m->host_setup = std::move(hs);
}
}  // namespace hfpx

extern "C" {

int hfpx_ctx_create(int device, hfpx_ctx** out) {
  if (!out) return HFPX_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return HFPX_ERR_CUDA;
  hfpx_ctx* c = new (std::nothrow) hfpx_ctx;
  if (!c) return HFPX_ERR_NOMEM;
  c->device = device;
  int rc = check_cuda(c, cudaSetDevice(device), "cudaSetDevice");
  if (!rc) rc = check_cuda(c, cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device), "SM count");
  if (!rc) rc = check_cuda(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream");
  if (!rc) rc = check_cuda(c, cudaMalloc(&c->d_flags, 16 * sizeof(int)), "flags");
  if (!rc) {
    cublasHandle_t h = nullptr;
    if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) rc = HFPX_ERR_CUDA;
    else {
      cublasSetStream(h, c->stream);
      c->cublas = h;
    }
  }
  if (!rc) {
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    rc = check_cuda(c, cudaStreamCreateWithPriority(&c->stream_panel, cudaStreamNonBlocking, hi), "panel stream");
    if (!rc) rc = check_cuda(c, cudaStreamCreateWithFlags(&c->stream_left, cudaStreamNonBlocking), "swap stream");
    cublasHandle_t h = nullptr;
    if (!rc && cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) rc = HFPX_ERR_CUDA;
    if (!rc) {
      cublasSetStream(h, c->stream_panel);
      c->cublas_panel = h;
    }
  }
  if (rc) {
    hfpx_ctx_destroy(c);
    return rc;
  }
  *out = c;
  return HFPX_OK;
}

int hfpx_ctx_destroy(hfpx_ctx* c) {
  if (!c) return HFPX_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->stream_panel) cudaStreamSynchronize(c->stream_panel);
  if (c->stream_left) cudaStreamSynchronize(c->stream_left);
  if (c->cublas) cublasDestroy(static_cast<cublasHandle_t>(c->cublas));
  if (c->cublas_panel) cublasDestroy(static_cast<cublasHandle_t>(c->cublas_panel));
  if (c->cusolver) cusolverDnDestroy(static_cast<cusolverDnHandle_t>(c->cusolver));
  if (c->d_flags) cudaFree(c->d_flags);
  for (void* p : c->scratch)
    if (p) cudaFree(p);
  if (c->stream_coarse) cudaStreamSynchronize(c->stream_coarse);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->stream_coarse) cudaStreamDestroy(c->stream_coarse);
  if (c->stream) cudaStreamDestroy(c->stream);
  if (c->stream_panel) cudaStreamDestroy(c->stream_panel);
  if (c->stream_left) cudaStreamDestroy(c->stream_left);
  delete c;
  return HFPX_OK;
}

const char* hfpx_ctx_last_error(const hfpx_ctx* c) { return c ? c->last_error.c_str() : "null context"; }

int hfpx_ctx_stream(hfpx_ctx* c, void** stream) {
  if (!c || !stream) return HFPX_ERR_ARG;
  *stream = c->stream;
  return HFPX_OK;
}

int hfpx_ctx_synchronize(hfpx_ctx* c) {
  if (!c) return HFPX_ERR_ARG;
  return check_cuda(c, cudaStreamSynchronize(c->stream), "synchronize");
}

// surface_mesh_utilities.cpp:28-112 (make_dof_h_crack, approximation order 2).
int64_t hfpx_dof_handle(const double* nods, int64_t ld_nods, int64_t n_nodes, const int64_t* conn,
                        int64_t ld_conn, int64_t n_el, int tip_type, int64_t* dof_h) {
  if (!nods || !conn || !dof_h || ld_nods < 3 || ld_conn < 3 || n_el < 1 || n_nodes < 3) return -HFPX_ERR_ARG;
  const bool ext = ld_nods >= 5 && ld_conn >= 5;
  int64_t n_dof = 18 * n_el, dec = 0;
  for (int64_t el = 0; el < n_el; ++el)
    for (int l = 0; l < 18; ++l) dof_h[el + n_el * l] = 18 * el + l;
  for (int64_t el = 0; el < n_el; ++el) {
    bool tip[3] = {false, false, false};
    if (ext && conn[3 + ld_conn * el] == conn[4 + ld_conn * el])
      for (int v = 0; v < 3; ++v) {
        const int64_t n = conn[v + ld_conn * el];
        if (n < 0 || n >= n_nodes) return -HFPX_ERR_ARG;
        tip[v] = nods[3 + ld_nods * n] == 1.0 && nods[4 + ld_nods * n] == 1.0;
      }
    for (int v = 0; v < 6; ++v) {
      // act: 0 shift by the running count, 1 fix, 2 keep (the reference leaves
      // non-tip edge nodes unshifted when tip_type == 2)
      int act = 0;
      if (tip_type >= 1 && v < 3 && tip[v]) act = 1;
      else if (tip_type == 2 && v >= 3) {
        const int a = (v - 3 + 1) % 3, b = (a + 1) % 3;
        act = (tip[a] && tip[b]) ? 1 : 2;
      }
      for (int l = 0; l < 3; ++l) {
        int64_t& d = dof_h[el + n_el * (3 * v + l)];
        if (act == 1) { --n_dof; ++dec; d = -1; }
        else if (act == 0) d -= dec;
      }
    }
  }
  return n_dof;
}

int hfpx_mesh_create(hfpx_ctx* c, const double* nods, int64_t ld_nods, int64_t n_nodes, const int64_t* conn,
                     int64_t ld_conn, int64_t n_el, double beta, hfpx_mesh** out) {
  if (!c || !out) return HFPX_ERR_ARG;
  *out = nullptr;
  if (!nods || !conn || ld_nods < 3 || ld_conn < 3 || n_el < 1 || n_nodes < 3)
    return set_error(c, HFPX_ERR_ARG, "mesh needs >= 3 coordinate rows, >= 3 nodes and >= 1 element");
  for (int64_t e = 0; e < n_el; ++e)
    for (int j = 0; j < 3; ++j) {
      const int64_t n = conn[j + ld_conn * e];
      if (n < 0 || n >= n_nodes) return set_error(c, HFPX_ERR_ARG, "connectivity refers to a missing node");
    }
  for (int64_t n = 0; n < n_nodes; ++n)
    for (int k = 0; k < 3; ++k)
      if (!std::isfinite(nods[k + ld_nods * n])) return set_error(c, HFPX_ERR_ARG, "non-finite node coordinate");
  if (int rc_dev = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc_dev;
  ScratchBuf dn(c, kScrHostNods), dc(c, kScrHostConn);
  int rc = check_cuda(c, dn.alloc(sizeof(double) * ld_nods * n_nodes), "nods alloc");
  if (!rc) rc = check_cuda(c, dc.alloc(sizeof(int64_t) * ld_conn * n_el), "conn alloc");
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(dn.p, nods, sizeof(double) * ld_nods * n_nodes, cudaMemcpyHostToDevice, c->stream), "nods copy");
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(dc.p, conn, sizeof(int64_t) * ld_conn * n_el, cudaMemcpyHostToDevice, c->stream), "conn copy");
  hfpx_mesh* m = new (std::nothrow) hfpx_mesh;
  if (!m) return HFPX_ERR_NOMEM;
  m->n_el = n_el;
  m->h_vid.resize(3 * n_el);
  m->h_vert.resize(9 * n_el);
  for (int64_t e = 0; e < n_el; ++e)
    for (int j = 0; j < 3; ++j) {
      const int64_t v = conn[j + ld_conn * e];
      m->h_vid[3 * e + j] = v;
      for (int k = 0; k < 3; ++k) m->h_vert[9 * e + 3 * j + k] = nods[k + ld_nods * v];
    }
  // the preconditioners' mesh-only set-up runs on a host thread from here on
  if (!rc) start_mesh_setup(m);
  if (!rc) rc = pool_alloc(c, &m->d_elem, elem_record_bytes() * n_el, "element records");
  if (!rc) launch_element_precompute(dn.as<double>(), ld_nods, dc.as<int64_t>(), ld_conn, n_el, beta, m->d_elem, c->stream);
  if (!rc) rc = check_cuda(c, cudaGetLastError(), "element precompute");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "element precompute");
  if (rc) {
    hfpx_mesh_destroy(m);
    return rc;
  }
  *out = m;
  return HFPX_OK;
}

int hfpx_mesh_destroy(hfpx_mesh* m) {
  if (!m) return HFPX_OK;
  if (m->host_setup && m->host_setup->worker.joinable()) m->host_setup->worker.join();
  if (m->gnn_graph) gnn_graph_release(m->gnn_graph);
  m->pattern.reset();
  pool_free(m->d_elem);
  delete m;
  return HFPX_OK;
}

static int new_matrix(hfpx_ctx* c, int64_t n, hfpx_matrix** out) {
  hfpx_matrix* m = new (std::nothrow) hfpx_matrix;
  if (!m) return HFPX_ERR_NOMEM;
  m->n = n;
  m->ld = round_ld(n);
  int rc = check_cuda(c, cudaMalloc(&m->d_a, sizeof(double) * (size_t)m->ld * n), "matrix alloc");
  if (!rc) rc = check_cuda(c, cudaMalloc(&m->d_piv, sizeof(int32_t) * n), "pivot alloc");
  if (rc) {
    hfpx_matrix_destroy(m);
    return rc;
  }
  *out = m;
  return HFPX_OK;
}

static int check_assembly_args(hfpx_ctx* c, const hfpx_mesh* mesh, const int64_t* dof_h, int64_t n_dof, double G,
                               double nu) {
  if (!mesh || !dof_h) return set_error(c, HFPX_ERR_ARG, "null mesh or dof handle");
  if (n_dof < 1 || n_dof > 18 * mesh->n_el) return set_error(c, HFPX_ERR_ARG, "n_dof out of range");
  if (mesh->n_el > 65535) return set_error(c, HFPX_ERR_ARG, "more than 65535 elements (grid limit of the assembly launch)");
  if (!(G > 0) || !(nu > -1.0 && nu < 0.5))
    return set_error(c, HFPX_ERR_ARG, "shear modulus must be > 0 and Poisson ratio in (-1, 0.5)");
  return HFPX_OK;
}

static int assemble_into(hfpx_ctx* c, const hfpx_mesh* mesh, const int64_t* dof_h, int64_t n_dof, double G, double nu,
                         int is_dd_local, int vc_border, hfpx_matrix* m) {
  int32_t* dd = nullptr;
  int rc = upload_dof(c, dof_h, mesh->n_el, n_dof, &dd);
  if (rc) return rc;
  m->factored = 0;
  m->info = 0;
  // a matrix that has an FP32 working copy gets it written in the same pass
  // (not with the volume-control border, which only the FP64 matrix takes)
  float* f = vc_border ? nullptr : m->d_f;
  launch_assemble(mesh->d_elem, mesh->n_el, dd, G, nu, is_dd_local, m->d_a, m->ld, f, c->d_flags, c->stream);
  m->f32_current = f != nullptr;
  if (vc_border) launch_vc_border(mesh->d_elem, mesh->n_el, dd, n_dof, is_dd_local, m->d_a, m->ld, c->stream);
  rc = check_cuda(c, cudaGetLastError(), "assembly launch");
  int flags[2] = {0, 0};
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(flags, c->d_flags, sizeof(flags), cudaMemcpyDeviceToHost, c->stream), "flags");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "assembly");
  if (!rc && (flags[0] & 1)) rc = set_error(c, HFPX_ERR_CUDA, "element staging copy timed out");
  return rc;
}

// Far-field pairs of the mixed-precision operator integrated in FP32 by
// quadrature with HFPX_FAR32=1.  The default evaluates every pair by the
// FP64 closed form and rounds it: the quadrature is the more accurate of the
// two far from the source, but the closed form is the reference's
// discretisation, and the solution's parity with the reference (opening
// within 1e-8) is defined against it (the quadrature moves the opening by
// about 5e-6 at 21 600 unknowns).
static bool far32_enabled() {
  const char* e = std::getenv("HFPX_FAR32");
  return e && std::string(e) == "1";
}

// The mixed-precision operator: every entry in FP32 (no FP64 matrix), the
// near-field blocks' low parts on the mesh's pattern.  The pattern indexes
// blocks by element, so the DoF must be the default numbering of a mesh
// without fixed DoF (18 e + 3 node + component), as for the near-field
// preconditioners.
static int assemble_mixed_into(hfpx_ctx* c, const hfpx_mesh* mesh, const int64_t* dof_h, int64_t n_dof, double G,
                               double nu, int is_dd_local, hfpx_matrix* m) {
  const int64_t ne = mesh->n_el;
  if (n_dof != 18 * ne) return set_error(c, HFPX_ERR_ARG, "the mixed-precision operator needs 18 DoF per element");
  for (int64_t l = 0; l < 18; ++l)
    for (int64_t e = 0; e < ne; ++e)
      if (dof_h[e + ne * l] != 18 * e + l)
        return set_error(c, HFPX_ERR_ARG, "the mixed-precision operator needs the default DoF numbering (no fixed DoF)");
  std::shared_ptr<NearPattern> pat = mesh_pattern(c, mesh);
  if (!pat) return set_error(c, HFPX_ERR_NOMEM, "near-field pattern");
  if (pat->maxdeg > kMaxNearDeg) return set_error(c, HFPX_ERR_ARG, "an element has more than 64 vertex neighbours");
  if (m->lo_blocks != pat->blocks()) {
    if (m->d_lo) cudaFree(m->d_lo);
    m->d_lo = nullptr;
    m->lo_blocks = 0;
    if (int rc = check_cuda(c, cudaMalloc(&m->d_lo, sizeof(float) * 324 * (size_t)pat->blocks()), "near-field low parts"))
      return rc;
    m->lo_blocks = pat->blocks();
  }
  m->pat = pat;
  int32_t* dd = nullptr;
  int rc = upload_dof(c, dof_h, ne, n_dof, &dd);
  if (rc) return rc;
  m->factored = 0;
  m->info = 0;
  m->dinv_valid = 0;
  launch_assemble(mesh->d_elem, ne, dd, G, nu, is_dd_local, nullptr, m->ld, m->d_f, c->d_flags, c->stream, m->d_lo,
                  pat->d_ptr, pat->d_idx, far32_enabled() ? 1 : 0);
  m->f32_current = 1;
  rc = check_cuda(c, cudaGetLastError(), "assembly launch");
  int flags[2] = {0, 0};
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(flags, c->d_flags, sizeof(flags), cudaMemcpyDeviceToHost, c->stream), "flags");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "assembly");
  if (!rc && (flags[0] & 1)) rc = set_error(c, HFPX_ERR_CUDA, "element staging copy timed out");
  return rc;
}

// entries (i0 + r, j0 + q) of a mixed-precision operator, hi + lo, into a
// column-major block (ld_out)
__global__ void compose_block_kernel(const OpView V, int64_t i0, int64_t j0, int64_t rows, int64_t cols,
                                     double* __restrict__ out, int64_t ld_out) {
  const int64_t q = blockIdx.y;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x)
    out[r + ld_out * q] = V.at(i0 + r, j0 + q);
  (void)cols;
}

// a block of a mixed-precision operator to the host, in column chunks of at
// most 32 MB through a context buffer
static int download_mixed(hfpx_ctx* c, const hfpx_matrix* m, int64_t i0, int64_t j0, int64_t rows, int64_t cols,
                          double* a, int64_t ld_host) {
  const int64_t per = std::max<int64_t>(1, std::min<int64_t>(cols, ((int64_t)32 << 20) / (8 * rows)));
  double* buf = (double*)ctx_scratch(c, kScrMixedBlk, sizeof(double) * rows * per);
  if (!buf) return set_error(c, HFPX_ERR_NOMEM, "download buffer");
  const OpView V = op_view(m);
  int rc = 0;
  for (int64_t q0 = 0; !rc && q0 < cols; q0 += per) {
    const int64_t nq = std::min(per, cols - q0);
    ++g_launches;
    compose_block_kernel<<<dim3((unsigned)std::min<int64_t>(64, (rows + 255) / 256), (unsigned)nq), 256, 0, c->stream>>>(
        V, i0, j0 + q0, rows, nq, buf, rows);
    rc = check_cuda(c, cudaGetLastError(), "compose block");
    if (!rc)
      rc = check_cuda(c, cudaMemcpy2DAsync(a + ld_host * q0, ld_host * sizeof(double), buf, rows * sizeof(double),
                                           rows * sizeof(double), nq, cudaMemcpyDeviceToHost, c->stream),
                      "block download");
    if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "block download");
  }
  return rc;
}

int hfpx_assemble(hfpx_ctx* c, const hfpx_mesh* mesh, const int64_t* dof_h, int64_t n_dof, double G, double nu,
                  int is_dd_local, int vc_border, hfpx_matrix** out) {
  if (!c || !out) return HFPX_ERR_ARG;
  *out = nullptr;
  int rc = check_assembly_args(c, mesh, dof_h, n_dof, G, nu);
  if (rc) return rc;
  if (int rc_dev = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc_dev;
  hfpx_matrix* m = nullptr;
  rc = new_matrix(c, n_dof + (vc_border ? 1 : 0), &m);
  if (!rc) rc = assemble_into(c, mesh, dof_h, n_dof, G, nu, is_dd_local, vc_border, m);
  if (rc) {
    hfpx_matrix_destroy(m);
    return rc;
  }
  *out = m;
  return HFPX_OK;
}

int hfpx_assemble_into(hfpx_ctx* c, const hfpx_mesh* mesh, const int64_t* dof_h, int64_t n_dof, double G, double nu,
                       int is_dd_local, int vc_border, hfpx_matrix* m) {
  if (!c) return HFPX_ERR_ARG;
  int rc = check_assembly_args(c, mesh, dof_h, n_dof, G, nu);
  if (rc) return rc;
  if (!m || m->n != n_dof + (vc_border ? 1 : 0)) return set_error(c, HFPX_ERR_ARG, "matrix size does not match n_dof");
  if (int rc_dev = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc_dev;
  if (m->op_mixed) {
    if (vc_border) return set_error(c, HFPX_ERR_ARG, "a mixed-precision operator has no volume-control border");
    return assemble_mixed_into(c, mesh, dof_h, n_dof, G, nu, is_dd_local, m);
  }
  return assemble_into(c, mesh, dof_h, n_dof, G, nu, is_dd_local, vc_border, m);
}

int hfpx_assemble_mixed(hfpx_ctx* c, const hfpx_mesh* mesh, const int64_t* dof_h, int64_t n_dof, double G, double nu,
                        int is_dd_local, hfpx_matrix** out) {
  if (!c || !out) return HFPX_ERR_ARG;
  *out = nullptr;
  int rc = check_assembly_args(c, mesh, dof_h, n_dof, G, nu);
  if (rc) return rc;
  if (int rc_dev = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc_dev;
  hfpx_matrix* m = new (std::nothrow) hfpx_matrix;
  if (!m) return set_error(c, HFPX_ERR_NOMEM, "matrix");
  m->n = n_dof;
  m->ld = round_ld(n_dof);
  m->op_mixed = 1;
  rc = check_cuda(c, cudaMalloc(&m->d_f, sizeof(float) * (size_t)m->ld * n_dof), "matrix alloc");
  if (!rc) rc = assemble_mixed_into(c, mesh, dof_h, n_dof, G, nu, is_dd_local, m);
  if (rc) {
    hfpx_matrix_destroy(m);
    return rc;
  }
  *out = m;
  return HFPX_OK;
}

int hfpx_matrix_is_mixed(const hfpx_matrix* m) { return m && m->op_mixed ? 1 : 0; }

int hfpx_assemble_grow(hfpx_ctx* c, const hfpx_mesh* mesh, int64_t n_el_old, const int64_t* dof_h, int64_t n_dof,
                       double G, double nu, int is_dd_local, const hfpx_matrix* old, hfpx_matrix** out) {
  if (!c || !out) return HFPX_ERR_ARG;
  *out = nullptr;
  int rc = check_assembly_args(c, mesh, dof_h, n_dof, G, nu);
  if (rc) return rc;
  if (!old) return set_error(c, HFPX_ERR_ARG, "null old matrix");
  if (old->op_mixed || !old->d_a) return set_error(c, HFPX_ERR_STATE, "the old matrix must be an FP64 operator");
  if (old->factored == 1) return set_error(c, HFPX_ERR_STATE, "the old matrix holds FP64 LU factors, not the operator");
  const int64_t ne = mesh->n_el, n_old = old->n;
  if (n_el_old < 1 || n_el_old > ne) return set_error(c, HFPX_ERR_ARG, "n_el_old out of range");
  if (n_old > n_dof) return set_error(c, HFPX_ERR_ARG, "the old matrix is larger than the new one");
  // The old block is copied as it is, so the old elements must keep their
  // DoF numbers: exactly the old matrix's n_old DoF belong to them, and the
  // appended elements' DoF come after.
  int64_t free_old = 0;
  for (int64_t l = 0; l < 18; ++l)
    for (int64_t e = 0; e < ne; ++e) {
      const int64_t d = dof_h[e + ne * l];
      if (d < -1 || d >= n_dof) return set_error(c, HFPX_ERR_ARG, "dof_h entry out of range");
      if (d < 0) continue;
      if (e < n_el_old) {
        if (d >= n_old) return set_error(c, HFPX_ERR_ARG, "an old element's DoF is not one of the old matrix's");
        ++free_old;
      } else if (d < n_old) {
        return set_error(c, HFPX_ERR_ARG, "an appended element's DoF falls inside the old matrix");
      }
    }
  if (free_old != n_old) return set_error(c, HFPX_ERR_ARG, "the old elements' DoF do not number the old matrix");
  if (int rc_dev = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc_dev;
  hfpx_matrix* m = nullptr;
  rc = new_matrix(c, n_dof, &m);
  if (rc) return rc;
  // element lists: appended sources (all targets), then old sources with
  // the appended targets
  const int64_t n_new = ne - n_el_old;
  std::vector<int32_t> lists(n_new + n_el_old);
  for (int64_t i = 0; i < n_new; ++i) lists[i] = (int32_t)(n_el_old + i);
  for (int64_t i = 0; i < n_el_old; ++i) lists[n_new + i] = (int32_t)i;
  int32_t* dl = (int32_t*)ctx_scratch(c, kScrGrowList, sizeof(int32_t) * std::max<size_t>(1, lists.size()));
  if (!dl) rc = set_error(c, HFPX_ERR_NOMEM, "element lists");
  if (!rc)
    rc = check_cuda(c, cudaMemcpyAsync(dl, lists.data(), sizeof(int32_t) * lists.size(), cudaMemcpyHostToDevice,
                                       c->stream), "element lists");
  int32_t* dd = nullptr;
  if (!rc) rc = upload_dof(c, dof_h, ne, n_dof, &dd);
  if (!rc)
    rc = check_cuda(c, cudaMemcpy2DAsync(m->d_a, m->ld * sizeof(double), old->d_a, old->ld * sizeof(double),
                                         n_old * sizeof(double), n_old, cudaMemcpyDeviceToDevice, c->stream),
                    "old block");
  if (!rc) {
    launch_assemble_partial(mesh->d_elem, ne, dd, G, nu, is_dd_local, m->d_a, m->ld, c->d_flags, c->stream, dl, n_new,
                            dl + n_new, n_el_old, dl, n_new);
    rc = check_cuda(c, cudaGetLastError(), "assembly launch");
  }
  int flags[2] = {0, 0};
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(flags, c->d_flags, sizeof(flags), cudaMemcpyDeviceToHost, c->stream), "flags");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "assembly");
  if (!rc && (flags[0] & 1)) rc = set_error(c, HFPX_ERR_CUDA, "element staging copy timed out");
  if (rc) {
    hfpx_matrix_destroy(m);
    return rc;
  }
  *out = m;
  return HFPX_OK;
}

int hfpx_matrix_upload(hfpx_ctx* c, const double* a, int64_t n, int64_t ld_host, hfpx_matrix** out) {
  if (!c || !out) return HFPX_ERR_ARG;
  *out = nullptr;
  if (!a || n < 1 || ld_host < n) return set_error(c, HFPX_ERR_ARG, "bad matrix dimensions");
  if (int rc_dev = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc_dev;
  hfpx_matrix* m = nullptr;
  int rc = new_matrix(c, n, &m);
  if (rc) return rc;
  rc = check_cuda(c, cudaMemcpy2DAsync(m->d_a, m->ld * sizeof(double), a, ld_host * sizeof(double), n * sizeof(double), n,
                                       cudaMemcpyHostToDevice, c->stream),
                  "matrix upload");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "matrix upload");
  if (rc) {
    hfpx_matrix_destroy(m);
    return rc;
  }
  *out = m;
  return HFPX_OK;
}

int hfpx_matrix_pivots(hfpx_ctx* c, const hfpx_matrix* m, int32_t* ipiv) {
  if (!c) return HFPX_ERR_ARG;
  if (!m || !ipiv) return set_error(c, HFPX_ERR_ARG, "null argument");
  if (m->factored != 1) return set_error(c, HFPX_ERR_STATE, "no FP64 factorisation");
  if (int rc_dev = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc_dev;
  int rc = check_cuda(c, cudaMemcpyAsync(ipiv, m->d_piv, sizeof(int32_t) * m->n, cudaMemcpyDeviceToHost, c->stream),
                      "pivots");
  return rc ? rc : check_cuda(c, cudaStreamSynchronize(c->stream), "pivots");
}

int hfpx_matrix_upload_lu(hfpx_ctx* c, const double* lu, int64_t n, int64_t ld_host, const int32_t* ipiv,
                          hfpx_matrix** out) {
  if (!c || !out) return HFPX_ERR_ARG;
  *out = nullptr;
  if (!ipiv) return set_error(c, HFPX_ERR_ARG, "null pivots");
  for (int64_t i = 0; i < n; ++i)
    if (ipiv[i] < i || ipiv[i] >= n) return set_error(c, HFPX_ERR_ARG, "pivot out of range");
  hfpx_matrix* m = nullptr;
  int rc = hfpx_matrix_upload(c, lu, n, ld_host, &m);
  if (rc) return rc;
  rc = check_cuda(c, cudaMemcpyAsync(m->d_piv, ipiv, sizeof(int32_t) * n, cudaMemcpyHostToDevice, c->stream), "pivots");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "pivots");
  if (rc) {
    hfpx_matrix_destroy(m);
    return rc;
  }
  m->factored = 1;
  m->info = 0;
  *out = m;
  return HFPX_OK;
}

int hfpx_matrix_dims(const hfpx_matrix* m, int64_t* n, int64_t* ld) {
  if (!m) return HFPX_ERR_ARG;
  if (n) *n = m->n;
  if (ld) *ld = m->ld;
  return HFPX_OK;
}

int hfpx_matrix_download(hfpx_ctx* c, const hfpx_matrix* m, double* a, int64_t ld_host) {
  if (!c || !m || !a || ld_host < m->n) return set_error(c, HFPX_ERR_ARG, "bad download arguments");
  if (int rc_dev = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc_dev;
  if (m->op_mixed) return download_mixed(c, m, 0, 0, m->n, m->n, a, ld_host);
  int rc = check_cuda(c, cudaMemcpy2DAsync(a, ld_host * sizeof(double), m->d_a, m->ld * sizeof(double), m->n * sizeof(double),
                                           m->n, cudaMemcpyDeviceToHost, c->stream),
                      "matrix download");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "matrix download");
  return rc;
}

int hfpx_matrix_download_block(hfpx_ctx* c, const hfpx_matrix* m, int64_t i0, int64_t j0, int64_t rows, int64_t cols,
                               double* a, int64_t ld_host) {
  if (!c) return HFPX_ERR_ARG;
  if (!m || !a || rows < 0 || cols < 0 || i0 < 0 || j0 < 0 || i0 + rows > m->n || j0 + cols > m->n ||
      ld_host < rows)
    return set_error(c, HFPX_ERR_ARG, "bad block download arguments");
  if (rows == 0 || cols == 0) return HFPX_OK;
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  if (m->op_mixed) return download_mixed(c, m, i0, j0, rows, cols, a, ld_host);
  int rc = check_cuda(c, cudaMemcpy2DAsync(a, ld_host * sizeof(double), m->d_a + i0 + m->ld * j0, m->ld * sizeof(double),
                                           rows * sizeof(double), cols, cudaMemcpyDeviceToHost, c->stream),
                      "block download");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "block download");
  return rc;
}

int hfpx_matrix_destroy(hfpx_matrix* m) {
  if (!m) return HFPX_OK;
  if (m->d_a) cudaFree(m->d_a);
  if (m->d_f) cudaFree(m->d_f);
  if (m->d_lo) cudaFree(m->d_lo);
  m->pat.reset();
  if (m->d_dinv) cudaFree(m->d_dinv);
  if (m->d_piv) cudaFree(m->d_piv);
  delete m;
  return HFPX_OK;
}

int hfpx_rhs_sinf(hfpx_ctx* c, const hfpx_mesh* mesh, const int64_t* dof_h, int64_t n_dof, const double* s_inf,
                  int64_t n_rhs, double* rhs, int64_t ld_rhs) {
  if (!c) return HFPX_ERR_ARG;
  if (!mesh || !dof_h || !s_inf || !rhs || n_rhs < 1 || ld_rhs < n_dof || n_dof < 1)
    return set_error(c, HFPX_ERR_ARG, "bad rhs arguments");
  if (int rc_dev = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc_dev;
  ScratchBuf ds(c, kScrHostSinf), dr(c, kScrHostRhs);
  int32_t* dd = nullptr;
  int rc = upload_dof(c, dof_h, mesh->n_el, n_dof, &dd);
  if (!rc) rc = check_cuda(c, ds.alloc(sizeof(double) * 6 * n_rhs), "s_inf alloc");
  if (!rc) rc = check_cuda(c, dr.alloc(sizeof(double) * ld_rhs * n_rhs), "rhs alloc");
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(ds.p, s_inf, sizeof(double) * 6 * n_rhs, cudaMemcpyHostToDevice, c->stream), "s_inf");
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(dr.p, rhs, sizeof(double) * ld_rhs * n_rhs, cudaMemcpyHostToDevice, c->stream), "rhs");
  if (!rc) launch_rhs(mesh->d_elem, mesh->n_el, dd, ds.as<double>(), n_rhs, dr.as<double>(), ld_rhs, c->stream);
  if (!rc) rc = check_cuda(c, cudaGetLastError(), "rhs launch");
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(rhs, dr.p, sizeof(double) * ld_rhs * n_rhs, cudaMemcpyDeviceToHost, c->stream), "rhs back");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "rhs");
  return rc;
}

int hfpx_lu_factor(hfpx_ctx* c, hfpx_matrix* m, int mode, int64_t* info) {
  if (!c) return HFPX_ERR_ARG;
  if (!m) return set_error(c, HFPX_ERR_ARG, "null matrix");
  if (mode != HFPX_LU_FP64 && mode != HFPX_LU_MIXED) return set_error(c, HFPX_ERR_ARG, "unknown LU mode");
  if (m->factored == 1) return set_error(c, HFPX_ERR_STATE, "matrix already factored in place");
  if (m->op_mixed)
    return set_error(c, HFPX_ERR_STATE, "a mixed-precision operator is solved by GMRES (assemble in FP64 to factor)");
  if (int rc_dev = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc_dev;
  int rc = mode == HFPX_LU_FP64 ? lu_factor_fp64(c, m) : lu_factor_fp32(c, m);
  if (info) *info = m->info;
  return rc;
}

int hfpx_lu_solve(hfpx_ctx* c, const hfpx_matrix* m, double* b, int64_t nrhs, int64_t ld_b, double tol, int max_iter,
                  hfpx_solve_info* info) {
  if (!c) return HFPX_ERR_ARG;
  if (!m || !b || nrhs < 1 || ld_b < m->n) return set_error(c, HFPX_ERR_ARG, "bad solve arguments");
  if (m->factored == 0) return set_error(c, HFPX_ERR_STATE, "solve before factor");
  if (m->info != 0) return set_error(c, HFPX_ERR_SINGULAR, "matrix is singular");
  if (int rc_dev = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc_dev;
  ScratchBuf db(c, kScrHostRhs);
  int rc = check_cuda(c, db.alloc(sizeof(double) * m->ld * nrhs), "rhs alloc");
  if (!rc) rc = check_cuda(c, cudaMemcpy2DAsync(db.p, m->ld * sizeof(double), b, ld_b * sizeof(double), m->n * sizeof(double),
                                                nrhs, cudaMemcpyHostToDevice, c->stream),
                           "rhs upload");
  if (!rc) {
    if (m->factored == 1) {
      rc = lu_solve_fp64(c, m, db.as<double>(), nrhs, m->ld);
      if (info) { info->iterations = 0; info->residual = 0.0; info->converged = 1; }
    } else {
      rc = refine_solve(c, m, db.as<double>(), nrhs, m->ld, tol > 0 ? tol : 1e-12, max_iter > 0 ? max_iter : 30, info);
    }
  }
  if (!rc || rc == HFPX_ERR_NOT_CONVERGED) {
    int rc2 = check_cuda(c, cudaMemcpy2DAsync(b, ld_b * sizeof(double), db.p, m->ld * sizeof(double), m->n * sizeof(double),
                                              nrhs, cudaMemcpyDeviceToHost, c->stream),
                         "solution download");
    if (!rc2) rc2 = check_cuda(c, cudaStreamSynchronize(c->stream), "solution download");
    if (rc2) rc = rc2;
  }
  return rc;
}

int hfpx_lu_solve_device(hfpx_ctx* c, const hfpx_matrix* m, double* d_b, int64_t nrhs, int64_t ld_b, double tol,
                         int max_iter, hfpx_solve_info* info) {
  if (!c) return HFPX_ERR_ARG;
  if (!m || !d_b || nrhs < 1 || ld_b < m->n) return set_error(c, HFPX_ERR_ARG, "bad solve arguments");
  if (m->factored == 0) return set_error(c, HFPX_ERR_STATE, "solve before factor");
  if (m->info != 0) return set_error(c, HFPX_ERR_SINGULAR, "matrix is singular");
  if (int rc_dev = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc_dev;
  if (m->factored == 1) {
    if (info) { info->iterations = 0; info->residual = 0.0; info->converged = 1; }
    return lu_solve_fp64(c, m, d_b, nrhs, ld_b);
  }
  return refine_solve(c, m, d_b, nrhs, ld_b, tol > 0 ? tol : 1e-12, max_iter > 0 ? max_iter : 30, info);
}

int hfpx_gmres_device(hfpx_ctx* c, const hfpx_matrix* m, double* d_b, double tol, int restart, int max_iter,
                      hfpx_solve_info* info) {
  if (!c) return HFPX_ERR_ARG;
  if (!m || !d_b) return set_error(c, HFPX_ERR_ARG, "bad GMRES arguments");
  if (m->factored != 2) return set_error(c, HFPX_ERR_STATE, "GMRES needs a mixed factorisation of the matrix");
  if (m->info != 0) return set_error(c, HFPX_ERR_SINGULAR, "matrix is singular");
  if (int rc_dev = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc_dev;
  return gmres_solve(c, m, d_b, tol > 0 ? tol : 1e-12, restart > 0 ? restart : 50, max_iter > 0 ? max_iter : 200,
                     info);
}

int hfpx_gmres(hfpx_ctx* c, const hfpx_matrix* m, double* b, double tol, int restart, int max_iter,
               hfpx_solve_info* info) {
  if (!c) return HFPX_ERR_ARG;
  if (!m || !b) return set_error(c, HFPX_ERR_ARG, "bad GMRES arguments");
  if (m->factored != 2) return set_error(c, HFPX_ERR_STATE, "GMRES needs a mixed factorisation of the matrix");
  if (m->info != 0) return set_error(c, HFPX_ERR_SINGULAR, "matrix is singular");
  if (int rc_dev = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc_dev;
  ScratchBuf db(c, kScrHostRhs);
  int rc = check_cuda(c, db.alloc(sizeof(double) * m->n), "rhs alloc");
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(db.p, b, sizeof(double) * m->n, cudaMemcpyHostToDevice, c->stream), "rhs");
  if (!rc) rc = gmres_solve(c, m, db.as<double>(), tol > 0 ? tol : 1e-12, restart > 0 ? restart : 50,
                            max_iter > 0 ? max_iter : 200, info);
  if (!rc || rc == HFPX_ERR_NOT_CONVERGED) {
    int rc2 = check_cuda(c, cudaMemcpyAsync(b, db.p, sizeof(double) * m->n, cudaMemcpyDeviceToHost, c->stream), "x");
    if (!rc2) rc2 = check_cuda(c, cudaStreamSynchronize(c->stream), "x");
    if (rc2) rc = rc2;
  }
  return rc;
}

int hfpx_gemm_f16_update(hfpx_ctx* c, int64_t m, int64_t n, int64_t k, const void* d_a, int64_t lda_k, const void* d_b,
                         int64_t ldb_k, float* d_c, int64_t ldc, const float* d_alpha) {
  if (!c) return HFPX_ERR_ARG;
  if (!d_a || !d_b || !d_c || !d_alpha || m < 0 || n < 0 || k < 0 || lda_k < k || ldb_k < k || ldc < std::max<int64_t>(m, 1))
    return set_error(c, HFPX_ERR_ARG, "bad update arguments");
  if (!tc_update_supported(lda_k, ldb_k, d_a, d_b))
    return set_error(c, HFPX_ERR_ARG, "update operands need 16-byte aligned bases and row strides (multiples of 8)");
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  int* err = (int*)ctx_scratch(c, kScrTcErr, sizeof(int));
  if (!err) return set_error(c, HFPX_ERR_NOMEM, "update status word");
  int rc = check_cuda(c, cudaMemsetAsync(err, 0, sizeof(int), c->stream), "update status");
  if (!rc) rc = tc_update_f16(c, c->stream, m, n, k, d_a, lda_k, d_b, ldb_k, d_c, ldc, d_alpha, nullptr, err, 0);
  int h_err = 0;
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "update status");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "tensor-core update");
  if (!rc && h_err) rc = set_error(c, HFPX_ERR_CUDA, "tensor-core update: a pipeline wait timed out");
  return rc;
}

int hfpx_residual_device(hfpx_ctx* c, const hfpx_matrix* m, const double* d_x, const double* d_b, double* d_r) {
  if (!c) return HFPX_ERR_ARG;
  if (!m || !d_x || !d_r) return set_error(c, HFPX_ERR_ARG, "null argument");
  if (m->factored == 1) return set_error(c, HFPX_ERR_STATE, "the matrix holds FP64 LU factors, not the operator");
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  const int64_t n = m->n;
  double* part = (double*)ctx_scratch(c, kScrResidPart, sizeof(double) * n * resid_chunks(n));
  unsigned long long* dmax = (unsigned long long*)ctx_scratch(c, kScrResidMax, sizeof(unsigned long long));
  double* zero = nullptr;
  if (!d_b) {
    zero = (double*)ctx_scratch(c, kScrGmresZero, sizeof(double) * n);
    if (zero) cudaMemsetAsync(zero, 0, sizeof(double) * n, c->stream);
  }
  if (!part || !dmax || (!d_b && !zero)) return set_error(c, HFPX_ERR_NOMEM, "residual buffers");
  if (m->op_mixed) return residual_mixed(c, m, d_x, d_b ? d_b : zero, d_r, part, dmax);
  return residual_f64(c, m->d_a, m->ld, n, d_x, d_b ? d_b : zero, d_r, part, dmax);
}

int64_t hfpx_ctx_launch_count(const hfpx_ctx* c) { return c ? (int64_t)g_launches.load() : -1; }

int hfpx_lu_panel_factor_noalloc(hfpx_ctx* c, double* d_a, int64_t lda, int64_t m, int w, int32_t* d_piv,
                                 int64_t* info) {
  if (!c) return HFPX_ERR_ARG;
  if (int rc = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc;
  return lu_panel_factor_noalloc(c, d_a, lda, m, w, d_piv, info);
}

int hfpx_stress(hfpx_ctx* c, const hfpx_mesh* mesh, double G, double nu, int is_dd_local, const double* dd,
                const double* pts, int64_t n_pts, const double* s_inf, double* out) {
  if (!c) return HFPX_ERR_ARG;
  if (!mesh || !dd || !pts || !s_inf || !out || n_pts < 1) return set_error(c, HFPX_ERR_ARG, "bad stress arguments");
  if (!(G > 0) || !(nu > -1.0 && nu < 0.5)) return set_error(c, HFPX_ERR_ARG, "bad elastic constants");
  if (int rc_dev = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc_dev;
  // work buffers kept by the context: a loop of stress evaluations allocates nothing
  ScratchBuf ddd(c, kScrStressDd), dp(c, kScrStressPts), ds(c, kScrStressSinf), dout(c, kScrStressOut);
  const int64_t ne = mesh->n_el;
  int rc = check_cuda(c, ddd.alloc(sizeof(double) * 18 * ne), "dd alloc");
  if (!rc) rc = check_cuda(c, dp.alloc(sizeof(double) * 3 * n_pts), "pts alloc");
  if (!rc) rc = check_cuda(c, ds.alloc(sizeof(double) * 6), "s_inf alloc");
  if (!rc) rc = check_cuda(c, dout.alloc(sizeof(double) * 6 * n_pts), "out alloc");
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(ddd.p, dd, sizeof(double) * 18 * ne, cudaMemcpyHostToDevice, c->stream), "dd");
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(dp.p, pts, sizeof(double) * 3 * n_pts, cudaMemcpyHostToDevice, c->stream), "pts");
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(ds.p, s_inf, sizeof(double) * 6, cudaMemcpyHostToDevice, c->stream), "s_inf");
  if (!rc) launch_stress(mesh->d_elem, ne, G, nu, is_dd_local, ddd.as<double>(), dp.as<double>(), n_pts, ds.as<double>(),
                         dout.as<double>(), c->stream);
  if (!rc) rc = check_cuda(c, cudaGetLastError(), "stress launch");
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(out, dout.p, sizeof(double) * 6 * n_pts, cudaMemcpyDeviceToHost, c->stream), "out");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "stress");
  return rc;
}

int hfpx_stress_batch(hfpx_ctx* c, const hfpx_mesh* mesh, double G, double nu, int is_dd_local, const double* dd,
                      int64_t n_cases, const double* pts, int64_t n_pts, const double* s_inf, double* out) {
  if (!c) return HFPX_ERR_ARG;
  if (!mesh || !dd || !pts || !s_inf || !out || n_pts < 1 || n_cases < 1)
    return set_error(c, HFPX_ERR_ARG, "bad stress arguments");
  if (!(G > 0) || !(nu > -1.0 && nu < 0.5)) return set_error(c, HFPX_ERR_ARG, "bad elastic constants");
  if (n_cases == 1) return hfpx_stress(c, mesh, G, nu, is_dd_local, dd, pts, n_pts, s_inf, out);
  if (int rc_dev = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc_dev;
  const int64_t ne = mesh->n_el, rows = 6 * n_pts, cols = 18 * ne;
  ScratchBuf dm(c, kScrStressInfl), ddd(c, kScrStressDd), dvec(c, kScrStressVec), dp(c, kScrStressPts),
      ds(c, kScrStressSinf), dS(c, kScrStressSum), dout(c, kScrStressOut);
  int rc = check_cuda(c, dm.alloc(sizeof(double) * rows * cols), "influence matrix alloc");
  if (!rc) rc = check_cuda(c, ddd.alloc(sizeof(double) * cols * n_cases), "dd alloc");
  if (!rc) rc = check_cuda(c, dvec.alloc(sizeof(double) * cols * n_cases), "dd vectors alloc");
  if (!rc) rc = check_cuda(c, dp.alloc(sizeof(double) * 3 * n_pts), "pts alloc");
  if (!rc) rc = check_cuda(c, ds.alloc(sizeof(double) * 6 * n_cases), "s_inf alloc");
  if (!rc) rc = check_cuda(c, dS.alloc(sizeof(double) * rows * n_cases), "stress alloc");
  if (!rc) rc = check_cuda(c, dout.alloc(sizeof(double) * rows * n_cases), "out alloc");
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(ddd.p, dd, sizeof(double) * cols * n_cases, cudaMemcpyHostToDevice, c->stream), "dd");
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(dp.p, pts, sizeof(double) * 3 * n_pts, cudaMemcpyHostToDevice, c->stream), "pts");
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(ds.p, s_inf, sizeof(double) * 6 * n_cases, cudaMemcpyHostToDevice, c->stream), "s_inf");
  if (!rc) {
    launch_stress_influence(mesh->d_elem, ne, G, nu, is_dd_local, dp.as<double>(), n_pts, dm.as<double>(), rows,
                            c->stream);
    launch_dd_to_vec(ddd.as<double>(), ne, n_cases, dvec.as<double>(), c->stream);
    cublasHandle_t h = static_cast<cublasHandle_t>(c->cublas);
    cublasSetMathMode(h, CUBLAS_DEFAULT_MATH);
    const double one = 1.0, zero = 0.0;
    if (cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, (int)rows, (int)n_cases, (int)cols, &one, dm.as<double>(), (int)rows,
                    dvec.as<double>(), (int)cols, &zero, dS.as<double>(), (int)rows) != CUBLAS_STATUS_SUCCESS)
      rc = set_error(c, HFPX_ERR_CUDA, "stress GEMM");
  }
  if (!rc) launch_stress_out(dS.as<double>(), n_pts, n_cases, ds.as<double>(), dout.as<double>(), c->stream);
  if (!rc) rc = check_cuda(c, cudaGetLastError(), "stress launch");
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(out, dout.p, sizeof(double) * rows * n_cases, cudaMemcpyDeviceToHost, c->stream), "out");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "stress");
  return rc;
}

int hfpx_local_submatrix(hfpx_ctx* c, double G, double nu, double h, double zr, double zi, const double* tau,
                         const double* sfm, double* out) {
  if (!c) return HFPX_ERR_ARG;
  if (!tau || !sfm || !out) return set_error(c, HFPX_ERR_ARG, "null argument");
  if (int rc_dev = check_cuda(c, cudaSetDevice(c->device), "set device")) return rc_dev;
  DevBuf dt, ds, dout;
  int rc = check_cuda(c, dt.alloc(sizeof(double) * 6), "alloc");
  if (!rc) rc = check_cuda(c, ds.alloc(sizeof(double) * 72), "alloc");
  if (!rc) rc = check_cuda(c, dout.alloc(sizeof(double) * 108), "alloc");
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(dt.p, tau, sizeof(double) * 6, cudaMemcpyHostToDevice, c->stream), "tau");
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(ds.p, sfm, sizeof(double) * 72, cudaMemcpyHostToDevice, c->stream), "sfm");
  if (!rc) launch_local_block(G, nu, h, zr, zi, dt.as<double>(), ds.as<double>(), dout.as<double>(), c->stream);
  if (!rc) rc = check_cuda(c, cudaGetLastError(), "local block launch");
  if (!rc) rc = check_cuda(c, cudaMemcpyAsync(out, dout.p, sizeof(double) * 108, cudaMemcpyDeviceToHost, c->stream), "out");
  if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->stream), "local block");
  return rc;
}

// element_utilities.cpp:62-238 on the host, same arithmetic as the device
// precompute (round-to-nearest, no contraction).
int hfpx_element_frame(const double* vert, double* r, double* tau_out, double* sfm_out) {
  if (!vert || !r || !tau_out || !sfm_out) return HFPX_ERR_ARG;
  typedef std::complex<double> C;
  double v[3][3];
  for (int j = 0; j < 3; ++j)
    for (int k = 0; k < 3; ++k) v[j][k] = vert[k + 3 * j];
  auto dot = [](const double* a, const double* b) {
    volatile double t = a[0] * b[0];
    volatile double u = a[1] * b[1];
    volatile double w = a[2] * b[2];
    double s = t + u;
    return s + w;
  };
  double a1[3], a2[3], e1[3], a3[3], e3[3], a4[3];
  for (int k = 0; k < 3; ++k) { a1[k] = v[1][k] - v[0][k]; a2[k] = v[2][k] - v[0][k]; }
  const double n1 = std::sqrt(dot(a1, a1));
  for (int k = 0; k < 3; ++k) e1[k] = a1[k] / n1;
  a3[0] = e1[1] * a2[2] - e1[2] * a2[1];
  a3[1] = e1[2] * a2[0] - e1[0] * a2[2];
  a3[2] = e1[0] * a2[1] - e1[1] * a2[0];
  const double n3 = std::sqrt(dot(a3, a3));
  for (int k = 0; k < 3; ++k) e3[k] = a3[k] / n3;
  a4[0] = e3[1] * e1[2] - e3[2] * e1[1];
  a4[1] = e3[2] * e1[0] - e3[0] * e1[2];
  a4[2] = e3[0] * e1[1] - e3[1] * e1[0];
  const double n4 = std::sqrt(dot(a4, a4));
  for (int k = 0; k < 3; ++k) { r[k] = e1[k]; r[3 + k] = a4[k] / n4; r[6 + k] = e3[k]; }
  C tau[3];
  for (int j = 0; j < 3; ++j) {
    double b[3];
    for (int k = 0; k < 3; ++k) b[k] = v[j][k] - v[0][k];
    tau[j] = C(dot(r, b), dot(r + 3, b));
    tau_out[2 * j] = tau[j].real();
    tau_out[2 * j + 1] = tau[j].imag();
  }
  const C det = tau[1] * std::conj(tau[2]) - tau[2] * std::conj(tau[1]);
  C L[3][3];
  L[1][0] = 0.0; L[1][1] = std::conj(tau[2]) / det; L[1][2] = -tau[2] / det;
  L[2][0] = 0.0; L[2][1] = -std::conj(tau[1]) / det; L[2][2] = tau[1] / det;
  for (int i = 0; i < 3; ++i) L[0][i] = -(L[1][i] + L[2][i]);
  L[0][0] += 1.0;
  C sf[6][6] = {};
  auto prod = [](C* P, const C* A, const C* B, double s) {
    P[0] += s * (A[0] * B[0]);
    P[1] += s * (A[0] * B[1] + A[1] * B[0]);
    P[2] += s * (A[0] * B[2] + A[2] * B[0]);
    P[3] += s * (A[1] * B[1]);
    P[4] += s * (A[2] * B[2]);
    P[5] += s * (A[1] * B[2] + A[2] * B[1]);
  };
  for (int vx = 0; vx < 3; ++vx) {
    prod(sf[vx], L[vx], L[vx], 2.0);
    for (int i = 0; i < 3; ++i) sf[vx][i] -= L[vx][i];
    prod(sf[3 + vx], L[(vx + 1) % 3], L[(vx + 2) % 3], 4.0);
  }
  for (int a = 0; a < 6; ++a)
    for (int j = 0; j < 6; ++j) {
      sfm_out[2 * (6 * a + j)] = sf[a][j].real();
      sfm_out[2 * (6 * a + j) + 1] = sf[a][j].imag();
    }
  return HFPX_OK;
}

}  // extern "C"
