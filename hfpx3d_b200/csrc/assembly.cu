// Assembly, right-hand side, volume-control border and stress kernels.
//
// Matrix fill (make_3dbem_matrix_s, system_assembly.cpp:30-219): grid
// (tiles of 128 target collocation points) x (source elements).  Each CTA
// stages its source element's record in shared memory with one bulk (TMA)
// copy, each thread evaluates one (collocation point, source element) pair --
// a 3 x 18 block of final matrix entries (global traction at the point due to
// global DD at the element's 6 nodes) -- and the CTA writes its 18 columns x
// 384 rows as contiguous column segments (column-major matrix, each source
// element owns 18 full columns).  No atomics: every entry has one writer.
//
// In-plane pairs (|h| < 2.221e-16, every pair of a planar crack) run the
// closed-form path in assemble_kernel<false>; the rare off-plane pairs are
// skipped there and evaluated by assemble_kernel<true> (quadrature moments),
// which exits at once when the first pass found none.
#include <cuda_runtime.h>
#include <cstdint>
#include <cmath>
#include "hfpx_device.cuh"
#include "engine_internal.h"

namespace hfpx {

__constant__ GL12 c_gl;
static PerDeviceOnce g_gl_ready;

// Far-field quadrature over a source triangle (the mixed-precision
// operator's far pairs): the collapsed (Duffy) product of 4-point
// Gauss-Legendre rules, 16 points, barycentric (l1, l2) and, per node a
// (vertices, then the edge node opposite vertex v), the weight times the
// quadratic shape function: wn[a][q] = w_q N_a(l_q).  Weights sum to 1 over
// the triangle (times its area).
constexpr int kFarQ = 16;
struct FarRule {
  float l1[kFarQ], l2[kFarQ];
  float wn[6][kFarQ];
};
__constant__ FarRule c_far;

// Gauss-Legendre nodes and weights on [-1, 1] (Newton on P_n)
static void gauss_legendre(int n, double* x_out, double* w_out) {
  for (int i = 0; i < n; ++i) {
    double x = std::cos(kPi * (i + 0.75) / (n + 0.5)), dp = 1.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = x;
      for (int k = 2; k <= n; ++k) {
        double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (x * p1 - p0) / (x * x - 1.0);
      double dx = p1 / dp;
      x -= dx;
      if (std::fabs(dx) < 1e-16) break;
    }
    x_out[i] = x;
    w_out[i] = 2.0 / ((1.0 - x * x) * dp * dp);
  }
}

static void gl_host_init(cudaStream_t s) {
  if (!g_gl_ready.pending()) return;
  GL12 g;
  gauss_legendre(12, g.x, g.w);
  // the triangle rule: (u, v) on [0,1]^2 -> l1 = u, l2 = v (1 - u), weight
  // 2 (1 - u) w_u w_v (the reference triangle has area 1/2)
  FarRule fr;
  double x4[4], w4[4];
  gauss_legendre(4, x4, w4);
  for (int iu = 0; iu < 4; ++iu)
    for (int iv = 0; iv < 4; ++iv) {
      const int q = 4 * iu + iv;
      const double u = 0.5 * (x4[iu] + 1.0), v = 0.5 * (x4[iv] + 1.0);
      const double w = 2.0 * (1.0 - u) * (0.5 * w4[iu]) * (0.5 * w4[iv]);
      const double l1 = u, l2 = v * (1.0 - u), l0 = 1.0 - l1 - l2;
      const double lam[3] = {l0, l1, l2};
      fr.l1[q] = (float)l1;
      fr.l2[q] = (float)l2;
      for (int a = 0; a < 3; ++a) fr.wn[a][q] = (float)(w * lam[a] * (2.0 * lam[a] - 1.0));
      for (int a = 0; a < 3; ++a) fr.wn[3 + a][q] = (float)(w * 4.0 * lam[(a + 1) % 3] * lam[(a + 2) % 3]);
    }
  if (cudaMemcpyToSymbolAsync(c_far, &fr, sizeof(fr), 0, cudaMemcpyHostToDevice, s) != cudaSuccess) return;
  if (cudaMemcpyToSymbolAsync(c_gl, &g, sizeof(g), 0, cudaMemcpyHostToDevice, s) == cudaSuccess) g_gl_ready.mark();
}

// ------------------------------------------------------------- bulk copy
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Stage `bytes` (multiple of 16, both addresses 16-byte aligned) from global
// to shared memory with one bulk copy completed on an mbarrier.  The wait is
// bounded; on timeout a status bit is set and false returned.
__device__ bool stage_bulk(void* dst, const void* src, uint32_t bytes, uint64_t* bar,
                           int* status) {
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
  }
  auto wait = [&](int limit) {
    uint32_t done = 0;
    for (int it = 0; it < limit && !done; ++it) {
      asm volatile(
          "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0; selp.u32 %0, 1, 0, p; }"
          : "=r"(done)
          : "r"(smem_u32(bar))
          : "memory");
    }
    return done != 0;
  };
  // every thread agrees on the outcome before anyone leaves
  if (__syncthreads_and(wait(1 << 22))) return true;
  if (threadIdx.x == 0 && status) atomicOr(status, 1);
  wait(1 << 22);  // give a late copy the chance to land before the CTA exits
  return false;
}

// --------------------------------------------------------- geometry (rn)
// Geometry that decides branches (h of a point, collocation points) uses
// round-to-nearest products and sums in the reference's order, so that the
// in-plane test |h| < h_tol sees the same value as the CPU.
__device__ __forceinline__ double dot3_rn(const double* r, const double* b) {
  return __dadd_rn(__dadd_rn(__dmul_rn(r[0], b[0]), __dmul_rn(r[1], b[1])), __dmul_rn(r[2], b[2]));
}

__device__ __forceinline__ void point_hz(const ElemRec& E, const double* pt, double& h, cplx& z) {
  double b[3];
  for (int k = 0; k < 3; ++k) b[k] = __dsub_rn(pt[k], E.v0[k]);
  z = mk(dot3_rn(E.r, b), dot3_rn(E.r + 3, b));
  h = -dot3_rn(E.r + 6, b);
}

__device__ __forceinline__ double norm3_rn(const double* a) {
  return __dsqrt_rn(dot3_rn(a, a));
}

// element_utilities.cpp:62-238, 364-395: frame, tau, shape functions, CPs.
__global__ void element_precompute_kernel(const double* __restrict__ nods, int64_t ld_nods,
                                          const int64_t* __restrict__ conn, int64_t ld_conn,
                                          int64_t n_el, double beta, ElemRec* __restrict__ out) {
  const int64_t el = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (el >= n_el) return;
  double v[3][3];
  for (int j = 0; j < 3; ++j) {
    const int64_t n = conn[j + ld_conn * el];
    for (int k = 0; k < 3; ++k) v[j][k] = nods[k + ld_nods * n];
  }
  ElemRec E;
  double a1[3], a2[3], e1[3], a3[3], e3[3], a4[3];
  for (int k = 0; k < 3; ++k) { a1[k] = __dsub_rn(v[1][k], v[0][k]); a2[k] = __dsub_rn(v[2][k], v[0][k]); }
  const double n1 = norm3_rn(a1);
  for (int k = 0; k < 3; ++k) e1[k] = __ddiv_rn(a1[k], n1);
  a3[0] = __dsub_rn(__dmul_rn(e1[1], a2[2]), __dmul_rn(e1[2], a2[1]));
  a3[1] = __dsub_rn(__dmul_rn(e1[2], a2[0]), __dmul_rn(e1[0], a2[2]));
  a3[2] = __dsub_rn(__dmul_rn(e1[0], a2[1]), __dmul_rn(e1[1], a2[0]));
  const double n3 = norm3_rn(a3);
  for (int k = 0; k < 3; ++k) e3[k] = __ddiv_rn(a3[k], n3);
  a4[0] = __dsub_rn(__dmul_rn(e3[1], e1[2]), __dmul_rn(e3[2], e1[1]));
  a4[1] = __dsub_rn(__dmul_rn(e3[2], e1[0]), __dmul_rn(e3[0], e1[2]));
  a4[2] = __dsub_rn(__dmul_rn(e3[0], e1[1]), __dmul_rn(e3[1], e1[0]));
  const double n4 = norm3_rn(a4);
  for (int k = 0; k < 3; ++k) {
    E.v0[k] = v[0][k];
    E.r[k] = e1[k];
    E.r[3 + k] = __ddiv_rn(a4[k], n4);
    E.r[6 + k] = e3[k];
    E.nrm[k] = -e3[k];
  }
  cplx tau[3];
  for (int j = 0; j < 3; ++j) {
    double b[3];
    for (int k = 0; k < 3; ++k) b[k] = __dsub_rn(v[j][k], v[0][k]);
    tau[j] = mk(dot3_rn(E.r, b), dot3_rn(E.r + 3, b));
    E.tau[2 * j] = tau[j].re;
    E.tau[2 * j + 1] = tau[j].im;
  }
  // quadratic Lagrange shape functions in monomials [1, t, tc, t^2, tc^2, t tc]
  const cplx det = tau[1] * conj(tau[2]) - tau[2] * conj(tau[1]);
  const double dn = det.re * det.re + det.im * det.im;
  const cplx idet = mk(det.re / dn, -det.im / dn);
  cplx L[3][3];
  L[1][0] = mk(0.0); L[1][1] = conj(tau[2]) * idet; L[1][2] = -(tau[2] * idet);
  L[2][0] = mk(0.0); L[2][1] = -(conj(tau[1]) * idet); L[2][2] = tau[1] * idet;
  for (int i = 0; i < 3; ++i) L[0][i] = -(L[1][i] + L[2][i]);
  L[0][0] = L[0][0] + mk(1.0);
  cplx sf[6][6];
  for (int a = 0; a < 6; ++a)
    for (int j = 0; j < 6; ++j) sf[a][j] = mk(0.0);
  auto prod = [](cplx* P, const cplx* A, const cplx* B, double s) {
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
      E.sfm[2 * (6 * a + j)] = sf[a][j].re;
      E.sfm[2 * (6 * a + j) + 1] = sf[a][j].im;
    }
  // collocation points, reference order of operations (element_utilities.cpp:364-395)
  double c[3];
  for (int k = 0; k < 3; ++k)
    c[k] = __dadd_rn(__dadd_rn(__ddiv_rn(v[0][k], 3.0), __ddiv_rn(v[1][k], 3.0)), __ddiv_rn(v[2][k], 3.0));
  const double omb = 1.0 - beta;
  for (int vx = 0; vx < 3; ++vx) {
    const int m = (vx + 1) % 3, l = (m + 1) % 3;
    for (int k = 0; k < 3; ++k) {
      E.cp[3 * vx + k] = __dadd_rn(__dmul_rn(omb, v[vx][k]), __dmul_rn(beta, c[k]));
      E.cp[3 * (vx + 3) + k] =
          __dadd_rn(__dmul_rn(__dmul_rn(0.5, omb), __dadd_rn(v[m][k], v[l][k])), __dmul_rn(beta, c[k]));
    }
  }
  E.area = 0.5 * norm3_rn(a3) * n1;
  edge_directions(E.tau, E.nt2);
  out[el] = E;
}

// -------------------------------------------------------------- pair math
// Local 6x(3 per node) stress of the in-plane closed form, contracted per node.
struct InPlaneBlock {
  cplx Ps[6], Qs[6];  // shifted moments: shift(z) applied on the monomial side
};

__device__ __forceinline__ void inplane_moments(const ElemRec& S, cplx z, cplx* P, cplx* Q) {
  EdgeSet E;
  edge_setup(S.tau, S.nt2, z, E);
  for (int j = 0; j < 6; ++j) { P[j] = mk(0.0); Q[j] = mk(0.0); }
  for (int m = 0; m < 3; ++m)
    if (E.use[m]) lim_moments_diff(E.chi[0][m], E.chi[1][m], E.d[m], P, Q);
}

// sink(a, S[6][3]) receives the local stress columns of node a.
template <class F>
__device__ __forceinline__ void inplane_nodes(const ElemRec& S, cplx z, const cplx* P,
                                              const cplx* Q, double nu, double scale, F&& sink) {
  const cplx zc = conj(z), z2 = z * z, zc2 = zc * zc, zz = z * zc;
  const double ca = -0.5 * (1.0 + 2.0 * nu), cb = -1.5 * (1.0 - 2.0 * nu);
  const double cp_ = 0.25 * (2.0 - nu), cq = 0.75 * nu;
  for (int a = 0; a < 6; ++a) {
    const cplx* sr = reinterpret_cast<const cplx*>(S.sfm) + 6 * a;
    cplx sz[6];
    sz[0] = sr[0] + sr[1] * z + sr[2] * zc + sr[3] * z2 + sr[4] * zc2 + sr[5] * zz;
    sz[1] = sr[1] + 2.0 * (sr[3] * z) + sr[5] * zc;
    sz[2] = sr[2] + 2.0 * (sr[4] * zc) + sr[5] * z;
    sz[3] = sr[3];
    sz[4] = sr[4];
    sz[5] = sr[5];
    cplx p = mk(0.0), q = mk(0.0);
#pragma unroll
    for (int j = 0; j < 6; ++j) { p += sz[j] * P[j]; q += sz[j] * Q[j]; }
    const cplx s0 = ca * p, s1 = cb * q, s3 = -p;
    const cplx t0 = -(cp_ * p + cq * q);
    const cplx t1 = -mul_i(cp_ * p - cq * q);
    double Sx[6][3];
    Sx[0][2] = scale * (s0.re + s1.re);
    Sx[1][2] = scale * (s0.re - s1.re);
    Sx[2][2] = scale * s3.re;
    Sx[3][2] = scale * s1.im;
    Sx[4][2] = 0.0;
    Sx[5][2] = 0.0;
    Sx[0][0] = Sx[1][0] = Sx[2][0] = Sx[3][0] = 0.0;
    Sx[4][0] = scale * 2.0 * t0.re;
    Sx[5][0] = scale * 2.0 * t0.im;
    Sx[0][1] = Sx[1][1] = Sx[2][1] = Sx[3][1] = 0.0;
    Sx[4][1] = scale * 2.0 * t1.re;
    Sx[5][1] = scale * 2.0 * t1.im;
    sink(a, Sx);
  }
}

// The far field in FP32: the in-plane (h = 0) stress of each node's shape
// function at z by the 16-point triangle rule, for a target at least
// kFarRatio element sizes from the source (there the rule's error is below
// 1e-7 of the block and the FP32 sums keep the block to about 2e-7).  The
// point kernel of a DD on the plane x3 = 0, at r = (r1, r2, 0) from the
// source point, is K = P(r1, r2) / R^7 with P of degree 4 (Kelvin's solution
// differentiated through Volterra's formula); only eight (stress, DD
// component) pairs are non-zero in the plane.  sink(a, S[6][3]) as for
// inplane_nodes.
constexpr double kFarRatio = 8.0;

__device__ __forceinline__ bool far_pair(const ElemRec& S, const double* pt) {
  // the source centroid is the mean of its three vertex collocation points
  double d2 = 0.0;
  for (int k = 0; k < 3; ++k) {
    const double c = (S.cp[k] + S.cp[3 + k] + S.cp[6 + k]) * (1.0 / 3.0);
    d2 += (pt[k] - c) * (pt[k] - c);
  }
  // largest edge (tau of vertex j at tau[2 j], tau[2 j + 1]; vertex 0 is the origin)
  const double e1 = S.tau[2] * S.tau[2] + S.tau[3] * S.tau[3];
  const double e2 = S.tau[4] * S.tau[4] + S.tau[5] * S.tau[5];
  const double dx = S.tau[4] - S.tau[2], dy = S.tau[5] - S.tau[3];
  const double e3 = dx * dx + dy * dy;
  const double L2 = fmax(e1, fmax(e2, e3));
  return d2 >= kFarRatio * kFarRatio * L2;
}

template <class F>
__device__ __forceinline__ void quad_nodes(const ElemRec& S, cplx z, double nu, double G, F&& sink) {
  const float zr = (float)z.re, zi = (float)z.im;
  const float t1r = (float)S.tau[2], t1i = (float)S.tau[3], t2r = (float)S.tau[4], t2i = (float)S.tau[5];
  const float fn = (float)nu;
  const float a11 = 2.f - 2.f * fn, b11 = 2.f * fn + 1.f, c11 = 4.f * fn - 1.f;   // S11 (normal DD)
  const float c12 = 3.f - 6.f * fn;                                               // S12 (normal DD)
  const float a13 = 1.f + fn, b13 = 2.f - fn, c13 = 1.f - 2.f * fn;               // S13 (DD 0), S23 (DD 1) mirrored
  const float d13 = 3.f * fn;                                                     // S13 (DD 1), S23 (DD 0)
  const double scale = G / (4.0 * kPi * (1.0 - nu)) * S.area;
  for (int a = 0; a < 6; ++a) {
    float s11 = 0.f, s22 = 0.f, s33 = 0.f, s12 = 0.f, s13_0 = 0.f, s13_1 = 0.f, s23_0 = 0.f, s23_1 = 0.f;
#pragma unroll 4
    for (int q = 0; q < kFarQ; ++q) {
      const float l1 = c_far.l1[q], l2 = c_far.l2[q];
      const float r1 = zr - (l1 * t1r + l2 * t2r), r2 = zi - (l1 * t1i + l2 * t2i);
      const float u = r1 * r1, v = r2 * r2, w = r1 * r2, R2 = u + v;
      const float ri = rsqrtf(R2), ri2 = ri * ri, ri3 = ri2 * ri, ri5 = ri3 * ri2, ri7 = ri5 * ri2;
      const float c = c_far.wn[a][q];
      const float cu = c * ri7;
      s11 = fmaf(cu, fmaf(a11, u * u, fmaf(b11, u * v, c11 * v * v)), s11);
      s22 = fmaf(cu, fmaf(c11, u * u, fmaf(b11, u * v, a11 * v * v)), s22);
      s33 = fmaf(c, ri3, s33);
      const float cw = c * w * ri5;
      s12 = fmaf(c12, cw, s12);
      s13_0 = fmaf(cu, fmaf(a13, u * u, fmaf(b13, u * v, c13 * v * v)), s13_0);
      s13_1 = fmaf(d13, cw, s13_1);
      s23_0 = fmaf(d13, cw, s23_0);
      s23_1 = fmaf(cu, fmaf(c13, u * u, fmaf(b13, u * v, a13 * v * v)), s23_1);
    }
    double Sx[6][3];
    for (int k = 0; k < 6; ++k) Sx[k][0] = Sx[k][1] = Sx[k][2] = 0.0;
    Sx[0][2] = scale * s11;
    Sx[1][2] = scale * s22;
    Sx[2][2] = scale * s33;
    Sx[3][2] = scale * s12;
    Sx[4][0] = scale * s13_0;
    Sx[4][1] = scale * s13_1;
    Sx[5][0] = scale * s23_0;
    Sx[5][1] = scale * s23_1;
    sink(a, Sx);
  }
}

// Off-plane monomial tensor (6x4x3) from the quadrature moments.
__device__ __noinline__ void offplane_smon(const ElemRec& S, cplx z, double h, double nu,
                                           cplx* smon) {
  EdgeSet E;
  edge_setup(S.tau, S.nt2, z, E);
  // Points below the element's span integrate the regular parts F_p and add
  // the h-singular lower-limit parts in closed form (exact vertex cancellation
  // around the contour); points higher up integrate I_p directly.
  const bool upper = fabs(h) < 0.05 * E.span;
  cplx W[HFPX_N_MOMENTS];
  for (int m = 0; m < HFPX_N_MOMENTS; ++m) W[m] = mk(0.0);
  int vcount[3] = {0, 0, 0};
  double angle = 0.0;
  for (int m = 0; m < 3; ++m)
    if (E.use[m]) {
      gen_moments_edge(E.chi[0][m], E.chi[1][m], E.d[m], h, upper, c_gl, W);
      vcount[(m + 1) % 3] += 1;
      vcount[m] -= 1;
      angle += E.chi[1][m] - E.chi[0][m];
    }
  for (int i = 0; i < 72; ++i) smon[i] = mk(0.0);
  double hq[5] = {1.0, h, h * h, h * h * h, h * h * h * h};
  for (int t = 0; t < HFPX_N_TERMS; ++t) {
    const hfpx_term_t tm = hfpx_terms[t];
    const cplx coef = mk(tm.cr0 + nu * tm.cr1, tm.ci0 + nu * tm.ci1);
    smon[tm.jck] -= (hq[tm.q] * coef) * W[tm.moment];
  }
  if (upper) {
    const double ah = fabs(h), lg = log(ah), sg = h > 0 ? 1.0 : -1.0;
    for (int t = 0; t < HFPX_N_LOWER; ++t) {
      const hfpx_lower_t lw = hfpx_lower[t];
      cplx A = mk(0.0);
      if (lw.sigma == 0) {
        A = mk(angle);
      } else {
        for (int v = 0; v < 3; ++v)
          if (vcount[v]) {
            double sn, cs;
            sincos(lw.sigma * E.phi[v], &sn, &cs);
            // e^{i s phi} / (i s) = (sin - i cos) / s
            A += (vcount[v] / (double)lw.sigma) * mk(sn, -cs);
          }
      }
      const double f = (lw.esg ? sg : 1.0) * (lw.ea == 1 ? ah : (lw.ea == -1 ? 1.0 / ah : 1.0)) *
                       (lw.elog ? lg : 1.0);
      const cplx coef = mk(lw.cr0 + nu * lw.cr1, lw.ci0 + nu * lw.ci1);
      smon[lw.jck] -= (f * coef) * A;
    }
  }
}

// Traction block rows for node a: 3x3 (traction comp, DD comp) in global
// coordinates, from local stress columns Sx (system_assembly.cpp:138-185).
__device__ __forceinline__ void traction_3x3(const double* r, const double* nl, const double Sx[6][3],
                                             int is_dd_local, double B[3][3]) {
  double tl[3][3], tg[3][3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    tl[0][k] = nl[0] * Sx[0][k] + nl[1] * Sx[3][k] + nl[2] * Sx[4][k];
    tl[1][k] = nl[1] * Sx[1][k] + nl[0] * Sx[3][k] + nl[2] * Sx[5][k];
    tl[2][k] = nl[2] * Sx[2][k] + nl[0] * Sx[4][k] + nl[1] * Sx[5][k];
  }
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int k = 0; k < 3; ++k) tg[a][k] = r[a] * tl[0][k] + r[3 + a] * tl[1][k] + r[6 + a] * tl[2][k];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      B[a][j] = is_dd_local ? tg[a][j] : tg[a][0] * r[j] + tg[a][1] * r[3 + j] + tg[a][2] * r[6 + j];
}

// ------------------------------------------------------------ assembly
constexpr int kTile = 128;
constexpr int kStageRows = 3 * kTile;

// The in-plane pass writes each matrix column segment straight from the
// warp: the 96 rows of a warp (3 per collocation point) go through a
// 768-byte per-warp buffer so that every lane stores 3 consecutive-row values
// (coalesced), instead of staging the CTA's whole 18-column block (55 KB of
// shared memory, 3 CTAs per SM) behind a CTA barrier.
struct AsmSmem {
  ElemRec src;
  uint64_t bar;
  int32_t cols[18];
  int32_t rows[kStageRows];
  double wbuf[kTile / 32][96];
  // mixed-precision operator: the source element's near-field column (its
  // neighbours, sorted, and the index of its self block)
  int32_t nb[kMaxNearDeg];
  int32_t ndeg;
  int64_t nbase;
};

// Block index of (target t, source s) in the near-field block store, or -1
// for a far pair (self block s + ptr[s], neighbour k at s + ptr[s] + 1 + k).
__device__ __forceinline__ int64_t near_block(const AsmSmem& sm, int64_t t, int64_t s) {
  if (t == s) return sm.nbase;
  for (int k = 0; k < sm.ndeg; ++k)
    if (sm.nb[k] == t) return sm.nbase + 1 + k;
  return -1;
}

// The low part of a near-field entry: what rounding v to FP32 lost, itself
// rounded to FP32 (hi + lo carries about 48 bits of v).
__device__ __forceinline__ float low_part(double v) { return (float)(v - (double)(float)v); }

// One CTA's work: source element s against the targets of tile bx (all
// n_t targets, or those listed in tlist).  A (FP64) and the FP32 arrays Af,
// Af2 (any may be null) receive every entry; lo the near-field low parts.
template <bool GENERAL>
__device__ __forceinline__ void assemble_body(AsmSmem& sm, const ElemRec* __restrict__ elems, int64_t n_el,
                                              const int32_t* __restrict__ dof, double G, double nu,
                                              int is_dd_local, double* __restrict__ A, int64_t ld,
                                              float* __restrict__ Af, float* __restrict__ Af2,
                                              int* __restrict__ status, float* __restrict__ lo,
                                              const int32_t* __restrict__ np_ptr,
                                              const int32_t* __restrict__ np_idx, int64_t s, int64_t bx,
                                              const int32_t* __restrict__ tlist, int64_t n_t, bool far32) {
  const int tid = threadIdx.x;
  if (!stage_bulk(&sm.src, elems + s, sizeof(ElemRec), &sm.bar, status)) return;
  if (tid < 18) sm.cols[tid] = dof[s + n_el * tid];
  if (lo) {
    const int32_t p0 = np_ptr[s], deg = min(np_ptr[s + 1] - p0, kMaxNearDeg);
    for (int k = tid; k < deg; k += kTile) sm.nb[k] = np_idx[p0 + k];
    if (tid == 0) {
      sm.ndeg = deg;
      sm.nbase = s + p0;
    }
  }
  const int64_t g = bx * kTile + tid;
  const bool valid = g < 6 * n_t;
  const int64_t tg = valid ? g / 6 : 0;
  const int nt = (int)(g - 6 * tg);
  const int64_t t = tlist ? tlist[tg] : tg;
  double pt[3] = {0.0, 0.0, 0.0}, nrm[3] = {0.0, 0.0, 0.0};
  if (valid) {
    const ElemRec* T = elems + t;
    for (int k = 0; k < 3; ++k) { pt[k] = T->cp[3 * nt + k]; nrm[k] = T->nrm[k]; }
  }
  const ElemRec& S = sm.src;
  double h;
  cplx z;
  point_hz(S, pt, h, z);
  const bool inplane = fabs(h) < kHTol;
  const double scale = -G / (4.0 * kPi * (1.0 - nu));
  double nl[3];
  for (int i = 0; i < 3; ++i) nl[i] = S.r[3 * i] * nrm[0] + S.r[3 * i + 1] * nrm[1] + S.r[3 * i + 2] * nrm[2];

  if (!GENERAL) {
    const bool mine = valid && inplane;
    const int lane = tid & 31, warp = tid >> 5;
    for (int k = 0; k < 3; ++k)
      sm.rows[3 * tid + k] = mine ? dof[t + n_el * (3 * nt + k)] : -1;
    const unsigned off = __ballot_sync(0xffffffffu, valid && !inplane);
    if (off && lane == 0) atomicAdd(status + 1, __popc(off));
    __syncthreads();  // sm.cols and every lane's rows
    // the rows this lane stores: warp rows lane, lane + 32, lane + 64
    int32_t trow[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) trow[q] = sm.rows[96 * warp + lane + 32 * q];
    double* wb = sm.wbuf[warp];
    // mixed-precision operator: this lane's block in the near-field store
    // (the sm.nb list was staged before the barrier above)
    const int64_t blk = (lo && mine) ? near_block(sm, t, s) : -1;
    float* lob = blk >= 0 ? lo + blk * 324 + 3 * nt : nullptr;
    // every lane runs the same form (the warp stays converged for the
    // per-warp transpose); rows of lanes that are not in-plane pairs are -1.
    // With far32 a warp whose pairs are all far from the source (and none
    // in its near-field pattern) takes the FP32 quadrature instead of the
    // closed form.
    const bool lane_far = !mine || (far32 && blk < 0 && far_pair(S, pt));
    const bool warp_far = far32 && __all_sync(0xffffffffu, lane_far) && __any_sync(0xffffffffu, mine);
    auto sink = [&](int a, const double Sx[6][3]) {
      double B[3][3];
      traction_3x3(S.r, nl, Sx, is_dd_local, B);
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const int32_t col = sm.cols[3 * a + j];
#pragma unroll
        for (int i = 0; i < 3; ++i) wb[3 * lane + i] = B[i][j];
        if (lob) {
#pragma unroll
          for (int i = 0; i < 3; ++i) lob[18 * (3 * a + j) + i] = low_part(B[i][j]);
        }
        __syncwarp();
        if (col >= 0) {
          if (A) {
            double* colp = A + (int64_t)col * ld;
#pragma unroll
            for (int q = 0; q < 3; ++q)
              if (trow[q] >= 0) colp[trow[q]] = wb[lane + 32 * q];
          }
          if (Af) {
            float* colf = Af + (int64_t)col * ld;
#pragma unroll
            for (int q = 0; q < 3; ++q)
              if (trow[q] >= 0) colf[trow[q]] = (float)wb[lane + 32 * q];
          }
          if (Af2) {
            float* colf = Af2 + (int64_t)col * ld;
#pragma unroll
            for (int q = 0; q < 3; ++q)
              if (trow[q] >= 0) colf[trow[q]] = (float)wb[lane + 32 * q];
          }
        }
        __syncwarp();
      }
    };
    if (warp_far) {
      quad_nodes(S, z, nu, G, sink);
    } else {
      cplx P[6], Q[6];
      inplane_moments(S, z, P, Q);
      inplane_nodes(S, z, P, Q, nu, scale, sink);
    }
  } else {
    __syncthreads();
    if (!(valid && !inplane)) return;
    cplx smon[72];
    offplane_smon(S, z, h, nu, smon);
    int32_t rows[3];
    for (int k = 0; k < 3; ++k) rows[k] = dof[t + n_el * (3 * nt + k)];
    const int64_t blk = lo ? near_block(sm, t, s) : -1;
    float* lob = blk >= 0 ? lo + blk * 324 + 3 * nt : nullptr;
    contract_nodes(S.sfm, z, smon, scale, [&](int a, const double Sx[6][3]) {
      double B[3][3];
      traction_3x3(S.r, nl, Sx, is_dd_local, B);
      for (int j = 0; j < 3; ++j) {
        if (lob)
          for (int i = 0; i < 3; ++i) lob[18 * (3 * a + j) + i] = low_part(B[i][j]);
        const int32_t col = sm.cols[3 * a + j];
        if (col < 0) continue;
        for (int i = 0; i < 3; ++i)
          if (rows[i] >= 0) {
            if (A) A[(int64_t)col * ld + rows[i]] = B[i][j];
            if (Af) Af[(int64_t)col * ld + rows[i]] = (float)B[i][j];
            if (Af2) Af2[(int64_t)col * ld + rows[i]] = (float)B[i][j];
          }
      }
    });
  }
}

template <bool GENERAL>
__global__ void __launch_bounds__(kTile, GENERAL ? 1 : 4) assemble_kernel(const ElemRec* __restrict__ elems,
                                                         int64_t n_el,
                                                         const int32_t* __restrict__ dof,
                                                         double G, double nu, int is_dd_local,
                                                         double* __restrict__ A, int64_t ld,
                                                         float* __restrict__ Af,
                                                         int* __restrict__ status,
                                                         float* __restrict__ lo,
                                                         const int32_t* __restrict__ np_ptr,
                                                         const int32_t* __restrict__ np_idx,
                                                         const int32_t* __restrict__ slist,
                                                         const int32_t* __restrict__ tlist, int64_t n_t,
                                                         int far32) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  AsmSmem& sm = *reinterpret_cast<AsmSmem*>(smem_raw);
  if (GENERAL && status[1] == 0) return;  // first pass met no off-plane pair
  // source element of this CTA and the target elements of the grid's x
  // range: all of them, or the lists of a partial (incremental) assembly
  const int64_t s = slist ? slist[blockIdx.y] : blockIdx.y;
  assemble_body<GENERAL>(sm, elems, n_el, dof, G, nu, is_dd_local, A, ld, Af, nullptr, status, lo, np_ptr, np_idx, s,
                         blockIdx.x, tlist, n_t, far32 != 0);
}

// Many meshes in one launch: CTA i takes task i = (mesh, source element,
// target tile) and writes that mesh's mixed-precision operator (FP32
// entries and near-field low parts) and its FP32 copy for the factorisation.
__global__ void __launch_bounds__(kTile, 4) batch_assemble_kernel(const BatchAsmMesh* __restrict__ meshes,
                                                                  const int4* __restrict__ tasks, double G,
                                                                  double nu, int* __restrict__ status, int far32) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  AsmSmem& sm = *reinterpret_cast<AsmSmem*>(smem_raw);
  const int4 tk = tasks[blockIdx.x];
  const BatchAsmMesh M = meshes[tk.x];
  assemble_body<false>(sm, static_cast<const ElemRec*>(M.elems), M.n_el, M.dof, G, nu, 0, nullptr, M.ld, M.A, M.F, status, M.lo, M.np_ptr,
                       M.np_idx, tk.y, tk.z, nullptr, M.n_el, far32 != 0);
}
__global__ void __launch_bounds__(kTile, 1) batch_assemble_general_kernel(const BatchAsmMesh* __restrict__ meshes,
                                                                          const int4* __restrict__ tasks, double G,
                                                                          double nu, int* __restrict__ status) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  AsmSmem& sm = *reinterpret_cast<AsmSmem*>(smem_raw);
  if (status[1] == 0) return;  // the in-plane pass met no off-plane pair
  const int4 tk = tasks[blockIdx.x];
  const BatchAsmMesh M = meshes[tk.x];
  assemble_body<true>(sm, static_cast<const ElemRec*>(M.elems), M.n_el, M.dof, G, nu, 0, nullptr, M.ld, M.A, M.F, status, M.lo, M.np_ptr,
                      M.np_idx, tk.y, tk.z, nullptr, M.n_el, false);
}

// set-up of the batched assembly kernels on the current device (before a
// stream capture records their launches)
static PerDeviceOnce g_batch_attr0, g_batch_attr1;
int batch_assemble_setup(cudaStream_t s) {
  gl_host_init(s);
  const size_t smem = sizeof(AsmSmem);
  cudaError_t e = smem_attr_once(g_batch_attr0, batch_assemble_kernel, (int)smem);
  if (e == cudaSuccess) e = smem_attr_once(g_batch_attr1, batch_assemble_general_kernel, (int)smem);
  return e == cudaSuccess ? 0 : 1;
}

void launch_batch_assemble(const BatchAsmMesh* d_meshes, const void* d_tasks, int64_t n_tasks, double G, double nu,
                           int* d_status, cudaStream_t s, int far32) {
  const size_t smem = sizeof(AsmSmem);
  cudaMemsetAsync(d_status, 0, 2 * sizeof(int), s);
  const int4* t = static_cast<const int4*>(d_tasks);
  ++g_launches;
  batch_assemble_kernel<<<(unsigned)n_tasks, kTile, smem, s>>>(d_meshes, t, G, nu, d_status, far32);
  ++g_launches;
  batch_assemble_general_kernel<<<(unsigned)n_tasks, kTile, smem, s>>>(d_meshes, t, G, nu, d_status);
}

size_t elem_record_bytes() { return sizeof(ElemRec); }

void launch_element_precompute(const double* d_nods, int64_t ld_nods, const int64_t* d_conn,
                               int64_t ld_conn, int64_t n_el, double beta, void* d_elem,
                               cudaStream_t s) {
  gl_host_init(s);
  const int bs = 128;
  ++g_launches;
  element_precompute_kernel<<<(unsigned)((n_el + bs - 1) / bs), bs, 0, s>>>(
      d_nods, ld_nods, d_conn, ld_conn, n_el, beta, static_cast<ElemRec*>(d_elem));
}

static void launch_assemble_pairs(const void* d_elem, int64_t n_el, const int32_t* d_dof, double G, double nu,
                                  int is_dd_local, double* d_a, int64_t ld, float* d_f, int* d_status, cudaStream_t s,
                                  float* d_lo, const int32_t* np_ptr, const int32_t* np_idx, const int32_t* slist,
                                  int64_t n_s, const int32_t* tlist, int64_t n_t, int far32) {
  gl_host_init(s);
  const size_t smem = sizeof(AsmSmem);
  static PerDeviceOnce attr0, attr1;
  smem_attr_once(attr0, assemble_kernel<false>, (int)smem);
  smem_attr_once(attr1, assemble_kernel<true>, (int)smem);
  cudaMemsetAsync(d_status, 0, 2 * sizeof(int), s);
  if (n_s <= 0 || n_t <= 0) return;
  const dim3 grid((unsigned)((6 * n_t + kTile - 1) / kTile), (unsigned)n_s);
  const ElemRec* e = static_cast<const ElemRec*>(d_elem);
  ++g_launches;
  assemble_kernel<false><<<grid, kTile, smem, s>>>(e, n_el, d_dof, G, nu, is_dd_local, d_a, ld, d_f, d_status, d_lo,
                                                   np_ptr, np_idx, slist, tlist, n_t, far32);
  ++g_launches;
  assemble_kernel<true><<<grid, kTile, smem, s>>>(e, n_el, d_dof, G, nu, is_dd_local, d_a, ld, d_f, d_status, d_lo,
                                                  np_ptr, np_idx, slist, tlist, n_t, 0);
}

void launch_assemble(const void* d_elem, int64_t n_el, const int32_t* d_dof, double G, double nu,
                     int is_dd_local, double* d_a, int64_t ld, float* d_f, int* d_status, cudaStream_t s,
                     float* d_lo, const int32_t* np_ptr, const int32_t* np_idx, int far32) {
  launch_assemble_pairs(d_elem, n_el, d_dof, G, nu, is_dd_local, d_a, ld, d_f, d_status, s, d_lo, np_ptr, np_idx,
                        nullptr, n_el, nullptr, n_el, far32);
}

// The pairs of an incremental assembly: every target of the sources in
// slist (n_s), then the targets in tlist (n_t) of the sources in slist2
// (n_s2).  The status words are cleared once; the off-plane passes run when
// either in-plane pass met an off-plane pair.
void launch_assemble_partial(const void* d_elem, int64_t n_el, const int32_t* d_dof, double G, double nu,
                             int is_dd_local, double* d_a, int64_t ld, int* d_status, cudaStream_t s,
                             const int32_t* slist, int64_t n_s, const int32_t* slist2, int64_t n_s2,
                             const int32_t* tlist, int64_t n_t) {
  gl_host_init(s);
  const size_t smem = sizeof(AsmSmem);
  static PerDeviceOnce attr0, attr1;
  smem_attr_once(attr0, assemble_kernel<false>, (int)smem);
  smem_attr_once(attr1, assemble_kernel<true>, (int)smem);
  cudaMemsetAsync(d_status, 0, 2 * sizeof(int), s);
  const ElemRec* e = static_cast<const ElemRec*>(d_elem);
  for (int pass = 0; pass < 2; ++pass) {
    const int32_t* sl = pass == 0 ? slist : slist2;
    const int64_t ns = pass == 0 ? n_s : n_s2;
    const int32_t* tl = pass == 0 ? nullptr : tlist;
    const int64_t nt = pass == 0 ? n_el : n_t;
    if (ns <= 0 || nt <= 0) continue;
    const dim3 grid((unsigned)((6 * nt + kTile - 1) / kTile), (unsigned)ns);
    ++g_launches;
    assemble_kernel<false><<<grid, kTile, smem, s>>>(e, n_el, d_dof, G, nu, is_dd_local, d_a, ld, nullptr, d_status,
                                                     nullptr, nullptr, nullptr, sl, tl, nt, 0);
  }
  for (int pass = 0; pass < 2; ++pass) {
    const int32_t* sl = pass == 0 ? slist : slist2;
    const int64_t ns = pass == 0 ? n_s : n_s2;
    const int32_t* tl = pass == 0 ? nullptr : tlist;
    const int64_t nt = pass == 0 ? n_el : n_t;
    if (ns <= 0 || nt <= 0) continue;
    const dim3 grid((unsigned)((6 * nt + kTile - 1) / kTile), (unsigned)ns);
    ++g_launches;
    assemble_kernel<true><<<grid, kTile, smem, s>>>(e, n_el, d_dof, G, nu, is_dd_local, d_a, ld, nullptr, d_status,
                                                    nullptr, nullptr, nullptr, sl, tl, nt, 0);
  }
}

// ----------------------------------------------------------- VC border
// system_assembly.cpp:495-555: volume row (shape-function integral x normal
// component, or x e3 for local DD) and pressure column (-normal).  The
// integrals of quadratic Lagrange shape functions over a flat triangle are 0
// for vertex nodes and area/3 for edge nodes.
__global__ void vc_border_kernel(const ElemRec* __restrict__ elems, int64_t n_el,
                                 const int32_t* __restrict__ dof, int64_t n_dof, int is_dd_local,
                                 double* __restrict__ A, int64_t ld) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i == 0) A[n_dof + ld * n_dof] = 0.0;
  if (i >= 18 * n_el) return;
  const int64_t el = i / 18;
  const int l = (int)(i - 18 * el), ns = l / 3, j = l % 3;
  const int32_t sd = dof[el + n_el * l];
  if (sd < 0) return;
  const ElemRec& E = elems[el];
  const double sfi = ns < 3 ? 0.0 : E.area / 3.0;
  A[n_dof + ld * (int64_t)sd] = is_dd_local ? (j == 2 ? sfi : 0.0) : sfi * E.r[6 + j];
  A[sd + ld * n_dof] = -E.r[6 + j];
}

void launch_vc_border(const void* d_elem, int64_t n_el, const int32_t* d_dof, int64_t n_dof,
                      int is_dd_local, double* d_a, int64_t ld, cudaStream_t s) {
  const int bs = 256;
  ++g_launches;
  vc_border_kernel<<<(unsigned)((18 * n_el + bs - 1) / bs), bs, 0, s>>>(
      static_cast<const ElemRec*>(d_elem), n_el, d_dof, n_dof, is_dd_local, d_a, ld);
}

// ------------------------------------------------------------------ RHS
// system_assembly.cpp:222-274: rhs[dof] -= (n . s_inf)_l, per load case.
__global__ void rhs_kernel(const ElemRec* __restrict__ elems, int64_t n_el,
                           const int32_t* __restrict__ dof, const double* __restrict__ sinf,
                           int64_t n_rhs, double* __restrict__ rhs, int64_t ld) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= 18 * n_el * n_rhs) return;
  const int64_t c = i / (18 * n_el), rem = i - c * 18 * n_el;
  const int64_t el = rem / 18;
  const int l18 = (int)(rem - 18 * el), l = l18 % 3;
  const int32_t d = dof[el + n_el * l18];
  if (d < 0) return;
  const double* n = elems[el].nrm;
  const double* si = sinf + 6 * c;
  double t;
  if (l == 0) t = n[0] * si[0] + n[1] * si[3] + n[2] * si[4];
  else if (l == 1) t = n[1] * si[1] + n[0] * si[3] + n[2] * si[5];
  else t = n[2] * si[2] + n[0] * si[4] + n[1] * si[5];
  rhs[d + ld * c] -= t;
}

// The right-hand sides of the 6 unit in-situ stress states of many meshes
// without fixed DoF (rhs = -(n . e_c) per collocation point and component,
// DoF 18 e + 3 node + l): block y is mesh y, its n x 6 block at B + boff[y].
__global__ void batch_basis_rhs_kernel(const BatchAsmMesh* __restrict__ meshes, double* __restrict__ B,
                                       const int64_t* __restrict__ boff) {
  const BatchAsmMesh M = meshes[blockIdx.y];
  const ElemRec* E = static_cast<const ElemRec*>(M.elems);
  const int64_t n = 18 * M.n_el;
  double* b = B + boff[blockIdx.y];
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 6 * n; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = t / n, d = t - c * n, el = d / 18;
    const int l = (int)(d % 3);
    const double* nr = E[el].nrm;
    double si[6] = {0, 0, 0, 0, 0, 0};
    si[c] = 1.0;
    double v;
    if (l == 0) v = nr[0] * si[0] + nr[1] * si[3] + nr[2] * si[4];
    else if (l == 1) v = nr[1] * si[1] + nr[0] * si[3] + nr[2] * si[5];
    else v = nr[2] * si[2] + nr[0] * si[4] + nr[1] * si[5];
    b[t] = -v;
  }
}

void launch_batch_basis_rhs(const BatchAsmMesh* d_meshes, int64_t n_mesh, double* d_B, const int64_t* d_boff,
                            cudaStream_t s) {
  ++g_launches;
  batch_basis_rhs_kernel<<<dim3(64, (unsigned)n_mesh), 256, 0, s>>>(d_meshes, d_B, d_boff);
}

void launch_rhs(const void* d_elem, int64_t n_el, const int32_t* d_dof, const double* d_sinf,
                int64_t n_rhs, double* d_rhs, int64_t ld_rhs, cudaStream_t s) {
  const int bs = 256;
  const int64_t n = 18 * n_el * n_rhs;
  ++g_launches;
  rhs_kernel<<<(unsigned)((n + bs - 1) / bs), bs, 0, s>>>(static_cast<const ElemRec*>(d_elem), n_el,
                                                        d_dof, d_sinf, n_rhs, d_rhs, ld_rhs);
}

// --------------------------------------------------------------- stress
// system_assembly.cpp:279-455: one CTA per observation point, threads over
// source elements, fixed-order tree reduction (deterministic).
constexpr int kStressThreads = 128;

__global__ void __launch_bounds__(kStressThreads) stress_kernel(
    const ElemRec* __restrict__ elems, int64_t n_el, double G, double nu, int is_dd_local,
    const double* __restrict__ dd, const double* __restrict__ pts, int64_t n_pts,
    const double* __restrict__ sinf, double* __restrict__ out) {
  __shared__ double red[6][kStressThreads];
  const int64_t p = blockIdx.x;
  const int tid = threadIdx.x;
  const double pt[3] = {pts[3 * p], pts[3 * p + 1], pts[3 * p + 2]};
  const double scale = -G / (4.0 * kPi * (1.0 - nu));
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int64_t s = tid; s < n_el; s += kStressThreads) {
    const ElemRec& S = elems[s];
    double h;
    cplx z;
    point_hz(S, pt, h, z);
    const double* r = S.r;
    auto sink = [&](int a, const double Sx[6][3]) {
      // rotate_sim (tensor_utilities.cpp:57-91): sigma_g = R^T sigma R per DD column
      double Sg[6][3];
      for (int k = 0; k < 3; ++k) {
        const double m[3][3] = {{Sx[0][k], Sx[3][k], Sx[4][k]},
                                {Sx[3][k], Sx[1][k], Sx[5][k]},
                                {Sx[4][k], Sx[5][k], Sx[2][k]}};
        double tt[3][3], gg[3][3];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) tt[i][j] = m[i][0] * r[j] + m[i][1] * r[3 + j] + m[i][2] * r[6 + j];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) gg[i][j] = r[i] * tt[0][j] + r[3 + i] * tt[1][j] + r[6 + i] * tt[2][j];
        Sg[0][k] = gg[0][0]; Sg[1][k] = gg[1][1]; Sg[2][k] = gg[2][2];
        Sg[3][k] = gg[0][1]; Sg[4][k] = gg[0][2]; Sg[5][k] = gg[1][2];
      }
      double ddv[3];
      for (int j = 0; j < 3; ++j) ddv[j] = dd[(6 * s + a) + 6 * n_el * j];
      for (int c = 0; c < 6; ++c) {
        double w0 = Sg[c][0], w1 = Sg[c][1], w2 = Sg[c][2];
        if (!is_dd_local) {
          const double g0 = w0 * r[0] + w1 * r[3] + w2 * r[6];
          const double g1 = w0 * r[1] + w1 * r[4] + w2 * r[7];
          const double g2 = w0 * r[2] + w1 * r[5] + w2 * r[8];
          w0 = g0; w1 = g1; w2 = g2;
        }
        acc[c] += w0 * ddv[0] + w1 * ddv[1] + w2 * ddv[2];
      }
    };
    if (fabs(h) < kHTol) {
      cplx P[6], Q[6];
      inplane_moments(S, z, P, Q);
      inplane_nodes(S, z, P, Q, nu, scale, sink);
    } else {
      cplx smon[72];
      offplane_smon(S, z, h, nu, smon);
      contract_nodes(S.sfm, z, smon, scale, sink);
    }
  }
  for (int c = 0; c < 6; ++c) red[c][tid] = acc[c];
  __syncthreads();
  for (int w = kStressThreads / 2; w > 0; w >>= 1) {
    if (tid < w)
      for (int c = 0; c < 6; ++c) red[c][tid] += red[c][tid + w];
    __syncthreads();
  }
  if (tid < 6) out[p + n_pts * tid] = red[tid][0] + sinf[tid];
}

void launch_stress(const void* d_elem, int64_t n_el, double G, double nu, int is_dd_local,
                   const double* d_dd, const double* d_pts, int64_t n_pts, const double* d_sinf,
                   double* d_out, cudaStream_t s) {
  gl_host_init(s);
  ++g_launches;
  stress_kernel<<<(unsigned)n_pts, kStressThreads, 0, s>>>(static_cast<const ElemRec*>(d_elem), n_el, G,
                                                          nu, is_dd_local, d_dd, d_pts, n_pts, d_sinf,
                                                          d_out);
}

// ----------------------------------------------------- stress influence
// The same per-(point, element) blocks as stress_kernel, stored instead of
// summed: M (6 n_pts x 18 n_el, column-major, ldm) with row 6 p + c (stress
// component c at point p) and column 18 s + 3 a + j (DD component j of node
// a of element s).  Threads run over points for one element, so each column
// segment is written contiguously.
__global__ void __launch_bounds__(kStressThreads) stress_influence_kernel(
    const ElemRec* __restrict__ elems, int64_t n_el, double G, double nu, int is_dd_local,
    const double* __restrict__ pts, int64_t n_pts, double* __restrict__ M, int64_t ldm) {
  const int64_t s = blockIdx.y;
  const int64_t p = (int64_t)blockIdx.x * kStressThreads + threadIdx.x;
  if (p >= n_pts) return;
  const double pt[3] = {pts[3 * p], pts[3 * p + 1], pts[3 * p + 2]};
  const double scale = -G / (4.0 * kPi * (1.0 - nu));
  const ElemRec& S = elems[s];
  double h;
  cplx z;
  point_hz(S, pt, h, z);
  const double* r = S.r;
  auto sink = [&](int a, const double Sx[6][3]) {
    double Sg[6][3];
    for (int k = 0; k < 3; ++k) {
      const double m[3][3] = {{Sx[0][k], Sx[3][k], Sx[4][k]},
                              {Sx[3][k], Sx[1][k], Sx[5][k]},
                              {Sx[4][k], Sx[5][k], Sx[2][k]}};
      double tt[3][3], gg[3][3];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) tt[i][j] = m[i][0] * r[j] + m[i][1] * r[3 + j] + m[i][2] * r[6 + j];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) gg[i][j] = r[i] * tt[0][j] + r[3 + i] * tt[1][j] + r[6 + i] * tt[2][j];
      Sg[0][k] = gg[0][0]; Sg[1][k] = gg[1][1]; Sg[2][k] = gg[2][2];
      Sg[3][k] = gg[0][1]; Sg[4][k] = gg[0][2]; Sg[5][k] = gg[1][2];
    }
    for (int c = 0; c < 6; ++c) {
      double w0 = Sg[c][0], w1 = Sg[c][1], w2 = Sg[c][2];
      if (!is_dd_local) {
        const double g0 = w0 * r[0] + w1 * r[3] + w2 * r[6];
        const double g1 = w0 * r[1] + w1 * r[4] + w2 * r[7];
        const double g2 = w0 * r[2] + w1 * r[5] + w2 * r[8];
        w0 = g0; w1 = g1; w2 = g2;
      }
      double* col = M + (6 * p + c) + ldm * (18 * s + 3 * a);
      col[0] = w0;
      col[ldm] = w1;
      col[2 * ldm] = w2;
    }
  };
  if (fabs(h) < kHTol) {
    cplx P[6], Q[6];
    inplane_moments(S, z, P, Q);
    inplane_nodes(S, z, P, Q, nu, scale, sink);
  } else {
    cplx smon[72];
    offplane_smon(S, z, h, nu, smon);
    contract_nodes(S.sfm, z, smon, scale, sink);
  }
}

// DD of n_cases load cases, (6 n_el) x 3 each, to the vectors of the
// influence matrix's columns: D[18 s + 3 a + j, case].
__global__ void dd_to_vec_kernel(const double* __restrict__ dd, int64_t n_el, int64_t n_cases,
                                 double* __restrict__ D) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= 18 * n_el * n_cases) return;
  const int64_t cs = i / (18 * n_el), e = i - cs * 18 * n_el;
  const int64_t s = e / 18, a = (e % 18) / 3, j = e % 3;
  D[i] = dd[cs * 18 * n_el + (6 * s + a) + 6 * n_el * j];
}

// S (6 n_pts x n_cases) + s_inf to out: n_cases blocks of n_pts x 6.
__global__ void stress_out_kernel(const double* __restrict__ S, int64_t n_pts, int64_t n_cases,
                                  const double* __restrict__ sinf, double* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= 6 * n_pts * n_cases) return;
  const int64_t cs = i / (6 * n_pts), e = i - cs * 6 * n_pts;
  const int64_t c = e / n_pts, p = e - c * n_pts;
  out[i] = S[(6 * p + c) + 6 * n_pts * cs] + sinf[c + 6 * cs];
}

void launch_stress_influence(const void* d_elem, int64_t n_el, double G, double nu, int is_dd_local,
                             const double* d_pts, int64_t n_pts, double* d_M, int64_t ldm, cudaStream_t s) {
  gl_host_init(s);
  ++g_launches;
  stress_influence_kernel<<<dim3((unsigned)((n_pts + kStressThreads - 1) / kStressThreads), (unsigned)n_el),
                            kStressThreads, 0, s>>>(static_cast<const ElemRec*>(d_elem), n_el, G, nu, is_dd_local,
                                                    d_pts, n_pts, d_M, ldm);
}

void launch_dd_to_vec(const double* d_dd, int64_t n_el, int64_t n_cases, double* d_D, cudaStream_t s) {
  const int64_t tot = 18 * n_el * n_cases;
  ++g_launches;
  dd_to_vec_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(d_dd, n_el, n_cases, d_D);
}

void launch_stress_out(const double* d_S, int64_t n_pts, int64_t n_cases, const double* d_sinf, double* d_out,
                       cudaStream_t s) {
  const int64_t tot = 6 * n_pts * n_cases;
  ++g_launches;
  stress_out_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(d_S, n_pts, n_cases, d_sinf, d_out);
}

// --------------------------------------------------------- single block
__global__ void local_block_kernel(double G, double nu, double h, double zr, double zi,
                                   const double* __restrict__ tau, const double* __restrict__ sfm,
                                   double* __restrict__ out) {
  ElemRec S;
  for (int i = 0; i < 6; ++i) S.tau[i] = tau[i];
  for (int i = 0; i < 72; ++i) S.sfm[i] = sfm[i];
  edge_directions(S.tau, S.nt2);
  const cplx z = mk(zr, zi);
  const double scale = -G / (4.0 * kPi * (1.0 - nu));
  auto sink = [&](int a, const double Sx[6][3]) {
    for (int c = 0; c < 6; ++c)
      for (int k = 0; k < 3; ++k) out[18 * c + 3 * a + k] = Sx[c][k];
  };
  if (fabs(h) < kHTol) {
    cplx P[6], Q[6];
    inplane_moments(S, z, P, Q);
    inplane_nodes(S, z, P, Q, nu, scale, sink);
  } else {
    cplx smon[72];
    offplane_smon(S, z, h, nu, smon);
    contract_nodes(S.sfm, z, smon, scale, sink);
  }
}

void launch_local_block(double G, double nu, double h, double zr, double zi, const double* d_tau,
                        const double* d_sfm, double* d_out, cudaStream_t s) {
  gl_host_init(s);
  ++g_launches;
  local_block_kernel<<<1, 1, 0, s>>>(G, nu, h, zr, zi, d_tau, d_sfm, d_out);
}

// ------------------------------------------------------- FP64 -> FP32 copy
// Whole columns (ld entries each, padding rows included) as a flat range.
// FP64 -> FP32 copy, one fixed 2048-element chunk per CTA (16-byte loads and
// stores; the ragged tail element by element).  Short-lived CTAs let a
// higher-priority stream's kernels take SMs as they free up while a large
// conversion runs beside them.
constexpr int kConvThreads = 256;
constexpr int kConvPer = 8;  // elements per thread
__global__ void __launch_bounds__(kConvThreads) convert_f32_kernel(const double* __restrict__ a, int64_t total,
                                                                    float* __restrict__ f) {
  const int64_t i0 = ((int64_t)blockIdx.x * kConvThreads + threadIdx.x) * kConvPer;
  if (i0 + kConvPer <= total) {
    const double2* src = reinterpret_cast<const double2*>(a + i0);
    const double2 v0 = src[0], v1 = src[1], v2 = src[2], v3 = src[3];
    float4* dst = reinterpret_cast<float4*>(f + i0);
    dst[0] = make_float4((float)v0.x, (float)v0.y, (float)v1.x, (float)v1.y);
    dst[1] = make_float4((float)v2.x, (float)v2.y, (float)v3.x, (float)v3.y);
  } else {
    for (int64_t i = i0; i < total; ++i) f[i] = (float)a[i];
  }
}

// ld x n elements; both pointers 16-byte aligned (column offsets of a
// cudaMalloc'd matrix whose ld is a multiple of 32).
void launch_convert_f32(const double* d_a, int64_t ld, int64_t n, float* d_f, cudaStream_t s) {
  const int64_t total = ld * n;
  const int64_t per_cta = (int64_t)kConvThreads * kConvPer;
  if (total <= 0) return;
  ++g_launches;
  convert_f32_kernel<<<(unsigned)((total + per_cta - 1) / per_cta), kConvThreads, 0, s>>>(d_a, total, d_f);
}

}  // namespace hfpx
