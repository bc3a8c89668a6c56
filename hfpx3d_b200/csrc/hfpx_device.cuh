// Device-side building blocks of the HFPx3D engine: complex arithmetic, the
// per-element record, and the DD -> stress influence of one source element at
// one point (the work of make_local_3dbem_submatrix,
// elasticity_kernel_integration.cpp:34-205, in this engine's own formulation).
//
// In-plane points (|h| < 2.221e-16) use closed-form sector moments
//   P_j = FP int m_j(w) rho^-3 dA,  Q_j = FP int m_j(w) e^{2i theta} rho^-3 dA
// (6 complex each, m_j = [1, w, conj w, w^2, conj w^2, |w|^2]); off-plane
// points use 23 sector moments W[sigma,p] from a radial closed form and
// Gauss-Legendre in t = asinh(a/|d|) along each edge, combined through the
// generated term table dd_terms.h.  Branch decisions (tolerances, skipped
// edges, angle wrapping) are those of the reference.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define HFPX_TABLE_QUAL static __device__ __constant__ const
#include "dd_terms.h"
#include "dd_lower.h"

namespace hfpx {

constexpr double kPi = 3.1415926535897932385;
constexpr double kHTol = 2.221e-16;   // constants.h:20
constexpr double kATol = 1.825e-8;    // constants.h:21

struct cplx {
  double re, im;
};
__host__ __device__ __forceinline__ cplx mk(double r, double i = 0.0) { return {r, i}; }
__host__ __device__ __forceinline__ cplx operator+(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__host__ __device__ __forceinline__ cplx operator-(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
__host__ __device__ __forceinline__ cplx operator-(cplx a) { return {-a.re, -a.im}; }
__host__ __device__ __forceinline__ cplx operator*(cplx a, cplx b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__host__ __device__ __forceinline__ cplx operator*(double s, cplx a) { return {s * a.re, s * a.im}; }
__host__ __device__ __forceinline__ cplx operator*(cplx a, double s) { return {s * a.re, s * a.im}; }
__host__ __device__ __forceinline__ cplx conj(cplx a) { return {a.re, -a.im}; }
__host__ __device__ __forceinline__ cplx& operator+=(cplx& a, cplx b) { a.re += b.re; a.im += b.im; return a; }
__host__ __device__ __forceinline__ cplx& operator-=(cplx& a, cplx b) { a.re -= b.re; a.im -= b.im; return a; }
__host__ __device__ __forceinline__ cplx mul_i(cplx a) { return {-a.im, a.re}; }
__device__ __forceinline__ double cabs_(cplx a) { return hypot(a.re, a.im); }
__device__ __forceinline__ double carg_(cplx a) { return atan2(a.im, a.re); }

// Per-element record in HBM (one per element, 1 KiB aligned slot so one bulk
// copy stages it in shared memory).  Everything the pair kernel needs about a
// source element: vertex 0, frame rows, tau of vertices 1,2, shape functions,
// and, as a target, its 6 collocation points and normal.
struct alignas(16) ElemRec {
  double v0[3];
  double r[9];          // rows e1, e2, e3 (element_utilities.cpp:62-87)
  double tau[6];        // vertices in local complex coords (re,im); tau[0] = 0
  double sfm[72];       // 6x6 complex shape-function matrix, row-major (re,im)
  double cp[18];        // collocation points (6 x xyz)
  double nrm[3];        // target normal -e3
  double area;          // element area
  double nt2[6];        // per edge j (tau_j -> tau_j+1): dt / conj(dt), the edge's doubled-angle
                        // direction that reflects z across the edge line (re,im), by Smith's quotient
};
static_assert(sizeof(ElemRec) % 16 == 0, "bulk copy size");

// ------------------------------------------------------------ in-plane path
// Per edge-end antiderivatives; vertex-only terms in Q_1, Q_2 kept as the
// reference's s_ij_lim_h (h_potential.cpp:1180-1232) carries them.
__device__ __forceinline__ void lim_moments_diff(double chi_m, double chi_n, cplx d,
                                                 cplx* P, cplx* Q) {
  const double D = cabs_(d);
  const double iD = 1.0 / D;
  // e^{i arg d} = d / |d| (the unit foot direction; no angle round trip)
  const cplx e = mk(d.re * iD, d.im * iD), e2 = e * e, e3 = e2 * e, e4 = e2 * e2;
  const cplx ec = conj(e), e2c = conj(e2);
  // Both ends go through the same code into separate arrays and are
  // subtracted explicitly: for an edge whose two ends are seen under the same
  // angle (the point on the edge line) the terms, of size 1/|d|, cancel
  // exactly instead of leaving a contraction residue.
  cplx E[2][12];
#pragma unroll 1
  for (int side = 0; side < 2; ++side) {  // one instruction sequence for both ends
    const double chi = side ? chi_n : chi_m;
    double s, c;
    sincos(chi, &s, &c);
    const cplx u = mk(c, s), u3 = u * u * u;
    const double at = atanh(s);
    const cplx iu = mul_i(u), iu3 = mul_i(u3);
    cplx* V = E[side];
    V[0] = mk(-s * iD);
    V[1] = -at * e;
    V[2] = -at * ec;
    V[3] = -D * (e2 * (mk(at) + 2.0 * iu));
    V[4] = -D * (e2c * (mk(at) - 2.0 * mul_i(conj(u))));
    V[5] = mk(D * at);
    V[6] = (iD / 6.0) * mul_i(e2 * (u3 + 3.0 * u));
    V[7] = e3 * (mk(at / 3.0) + (2.0 / 3.0) * iu + iu3 * (1.0 / 12.0));
    V[8] = -(e * (mk(at) + (5.0 / 12.0) * iu));
    V[9] = D * (e4 * (mk(at) + 2.0 * iu - (2.0 / 3.0) * iu3));
    V[10] = mk(D * at);
    V[11] = -D * (e2 * (mk(at) + 2.0 * iu));
  }
#pragma unroll
  for (int j = 0; j < 12; ++j) {
    const cplx dlt = mk(__dsub_rn(E[1][j].re, E[0][j].re), __dsub_rn(E[1][j].im, E[0][j].im));
    cplx& T = j < 6 ? P[j] : Q[j - 6];
    T = mk(__dadd_rn(T.re, dlt.re), __dadd_rn(T.im, dlt.im));
  }
}

// ----------------------------------------------------------- off-plane path
struct GL12 {
  double x[12], w[12];
};

// I_p(X) = int_0^X rho^p (rho^2+h^2)^(-7/2) d rho, p = 1..7, stable for X << |h|.
__device__ __forceinline__ void radial_I(double X, double h, double* I) {
  h = fabs(h);
  const double R = hypot(X, h), s = X / R, dl = X * X / (R * (R + h));
  const double s2 = s * s, s3 = s2 * s, s5 = s3 * s2;
  const double d2 = dl * dl, d3 = d2 * dl, d4 = d2 * d2, d5 = d4 * dl, d6 = d3 * d3;
  const double ih = 1.0 / h, ih2 = ih * ih, ih3 = ih2 * ih, ih4 = ih2 * ih2, ih5 = ih4 * ih;
  I[1] = dl * (5.0 - 10.0 * dl + 10.0 * d2 - 5.0 * d3 + d4) * 0.2 * ih5;
  I[2] = (s3 / 3.0 - s5 * 0.2) * ih4;
  I[3] = (d2 - 5.0 * d3 / 3.0 + d4 - d5 * 0.2) * ih3;
  I[4] = s5 * 0.2 * ih2;
  I[5] = (4.0 * d3 / 3.0 - d4 + d5 * 0.2) * ih;
  if (s < 0.6) {
    double acc = 0.0, t = s5 * s2;
    for (int k = 3; k < 200; ++k) {
      const double term = t / (2 * k + 1);
      acc += term;
      if (term <= 1e-17 * acc) break;
      t *= s2;
    }
    I[6] = acc;
  } else {
    I[6] = atanh(s) - s - s3 / 3.0 - s5 * 0.2;
  }
  I[7] = R * (2.0 * d4 - 1.2 * d5 + 0.2 * d6);
}

// F_p(X) = I_p(X) - C_p(|h|): the radial integrals without their h-singular
// lower-limit constants, finite as h -> 0 (e = 1 - X/R, ee = e / h^2).
__device__ __forceinline__ void radial_F(double X, double h, double* F) {
  h = fabs(h);
  const double R = hypot(X, h), s = X / R, ee = 1.0 / (R * (R + X)), e = h * h * ee;
  const double iR = 1.0 / R, iR2 = iR * iR, iR3 = iR2 * iR, iR5 = iR3 * iR2, h2 = h * h;
  F[1] = -0.2 * iR5;
  F[2] = -ee * ee * (1.0 - 5.0 * e / 3.0 + e * e - 0.2 * e * e * e);
  F[3] = -(iR3 / 3.0 - 0.2 * h2 * iR5);
  F[4] = -ee * (5.0 - 10.0 * e + 10.0 * e * e - 5.0 * e * e * e + e * e * e * e) * 0.2;
  F[5] = -(iR - 2.0 * h2 * iR3 / 3.0 + 0.2 * h2 * h2 * iR5);
  F[6] = log((1.0 + s) * R) - s - s * s * s / 3.0 - 0.2 * s * s * s * s * s;
  F[7] = R + 3.0 * h2 * iR - h2 * h2 * iR3 + 0.2 * h2 * h2 * h2 * iR5;
}

// Sector moments W[sigma,p] of one edge (foot d, angles chi_m -> chi_n) by
// Gauss-Legendre in t = asinh(a/|d|); upper integrates F_p instead of I_p.
__device__ inline void gen_moments_edge(double chi_m, double chi_n, cplx d, double h, bool upper,
                                        const GL12& gl, cplx* W) {
  const double D = cabs_(d);
  const cplx e = mk(d.re / D, d.im / D);  // e^{i arg d}
  const double tm = asinh(tan(chi_m)), tn = asinh(tan(chi_n));
  int npan = (int)ceil(fabs(tn - tm) / 1.5);
  npan = npan < 1 ? 1 : (npan > 64 ? 64 : npan);
  for (int ip = 0; ip < npan; ++ip) {
    const double a0 = tm + (tn - tm) * ip / npan, a1 = tm + (tn - tm) * (ip + 1) / npan;
    const double hw = 0.5 * (a1 - a0), mid = 0.5 * (a0 + a1);
    for (int g = 0; g < 12; ++g) {
      const double t = mid + hw * gl.x[g];
      const double ch = cosh(t), sh = sinh(t);
      const double wt = hw * gl.w[g] / ch;
      double I[8];
      if (upper) radial_F(D * ch, h, I);
      else radial_I(D * ch, h, I);
      const cplx eth = (1.0 / ch) * (e * mk(1.0, sh));
      constexpr int S = HFPX_SIGMA_MAX;
      cplx pw[2 * S + 1];  // e^{i s theta}, s = -S..S
      pw[S] = mk(1.0);
#pragma unroll
      for (int s = 1; s <= S; ++s) pw[S + s] = pw[S + s - 1] * eth;
#pragma unroll
      for (int s = 1; s <= S; ++s) pw[S - s] = conj(pw[S + s]);
#pragma unroll
      for (int m = 0; m < HFPX_N_MOMENTS; ++m)
        W[m] += (wt * I[hfpx_moments[m].p]) * pw[S + hfpx_moments[m].sigma];
    }
  }
}

// Edge geometry and the reference's branch decisions for one point.
struct EdgeSet {
  cplx d[3];
  double chi[2][3];
  double phi[3];     // absolute angle of each vertex seen from z
  double span;       // largest vertex distance from z
  bool use[3];
};

// Complex product and quotient without fused multiply-adds (round-to-nearest
// products and sums in the order of the textbook formulas).  The quotient is
// Smith's algorithm (Smith 1962, CACM Algorithm 116).  Foot vectors of points
// that lie exactly on an edge line come out as rounding noise whose size
// decides the |d| < 2.221e-16 branch, so this arithmetic is kept identical to
// an IEEE-double host computation of the same formulas.
__device__ __forceinline__ cplx mul_rn(cplx x, cplx y) {
  return {__dsub_rn(__dmul_rn(x.re, y.re), __dmul_rn(x.im, y.im)),
          __dadd_rn(__dmul_rn(x.re, y.im), __dmul_rn(x.im, y.re))};
}

__device__ __forceinline__ cplx div_smith(cplx x, cplx y) {
  const double a = x.re, b = x.im, c = y.re, d = y.im;
  if (fabs(c) < fabs(d)) {
    const double r = __ddiv_rn(c, d), den = __dadd_rn(__dmul_rn(c, r), d);
    return {__ddiv_rn(__dadd_rn(__dmul_rn(a, r), b), den), __ddiv_rn(__dsub_rn(__dmul_rn(b, r), a), den)};
  }
  const double r = __ddiv_rn(d, c), den = __dadd_rn(__dmul_rn(d, r), c);
  if (fabs(r) > 2.2250738585072014e-308)
    return {__ddiv_rn(__dadd_rn(__dmul_rn(b, r), a), den), __ddiv_rn(__dsub_rn(b, __dmul_rn(a, r)), den)};
  // r underflowed (d == 0): divide b and a by c first
  return {__ddiv_rn(__dadd_rn(a, __dmul_rn(d, __ddiv_rn(b, c))), den),
          __ddiv_rn(__dsub_rn(b, __dmul_rn(d, __ddiv_rn(a, c))), den)};
}

// dt / conj(dt) of each edge (tau_j -> tau_j+1): a property of the element,
// made once per element with the same arithmetic the point loop used
__device__ __forceinline__ void edge_directions(const double* tau6, double* nt2_6) {
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const int q = (j + 1) % 3;
    const cplx tj = mk(tau6[2 * j], tau6[2 * j + 1]), tq = mk(tau6[2 * q], tau6[2 * q + 1]);
    const cplx dt = mk(__dsub_rn(tq.re, tj.re), __dsub_rn(tq.im, tj.im));
    const cplx nt2 = div_smith(dt, conj(dt));
    nt2_6[2 * j] = nt2.re;
    nt2_6[2 * j + 1] = nt2.im;
  }
}

__device__ __forceinline__ void edge_setup(const double* tau6, const double* nt2_6, cplx z, EdgeSet& E) {
  cplx tz[3];
  double phi[3], psi[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const cplx tj = mk(tau6[2 * j], tau6[2 * j + 1]);
    tz[j] = mk(__dsub_rn(tj.re, z.re), __dsub_rn(tj.im, z.im));
    const cplx nt2 = mk(nt2_6[2 * j], nt2_6[2 * j + 1]);
    const cplx pr = mul_rn(nt2, conj(tz[j]));
    E.d[j] = mk(__dmul_rn(0.5, __dsub_rn(tz[j].re, pr.re)), __dmul_rn(0.5, __dsub_rn(tz[j].im, pr.im)));
  }
  E.span = 0.0;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    phi[j] = carg_(tz[j]);
    psi[j] = carg_(E.d[j]);
    E.phi[j] = phi[j];
    E.span = fmax(E.span, cabs_(tz[j]));
  }
  bool is90[2][3];
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      double c = phi[(j + k) % 3] - psi[j];
      if (c <= -kPi) { while (c <= -kPi) c += 2.0 * kPi; }
      else if (c > kPi) { while (c > kPi) c -= 2.0 * kPi; }
      E.chi[k][j] = c;
      is90[k][j] = fabs(0.5 * kPi - fabs(c)) < kATol;
    }
#pragma unroll
  for (int m = 0; m < 3; ++m) E.use[m] = cabs_(E.d[m]) >= kHTol && !is90[0][m] && !is90[1][m];
}

// Contraction with the shifted shape functions and re-shaping
// (elasticity_kernel_integration.cpp:180-203): local stress S[6][18] columns
// for node a are produced by the callback as the 3 DD components k.
// smon is the 6x4x3 monomial tensor, index (j*4+c)*3+k.
template <class F>
__device__ __forceinline__ void contract_nodes(const double* sfm, cplx z, const cplx* smon,
                                               double scale, F&& sink) {
  // row a of sfm . shift(z): shape functions re-expanded in monomials of w = tau - z
  // (element_utilities.cpp:339-360)
  const cplx zc = conj(z), z2 = z * z, zc2 = zc * zc, zz = z * zc;
  for (int a = 0; a < 6; ++a) {
    const cplx* sr = reinterpret_cast<const cplx*>(sfm) + 6 * a;
    cplx sz[6];
    sz[0] = sr[0] + sr[1] * z + sr[2] * zc + sr[3] * z2 + sr[4] * zc2 + sr[5] * zz;
    sz[1] = sr[1] + 2.0 * (sr[3] * z) + sr[5] * zc;
    sz[2] = sr[2] + 2.0 * (sr[4] * zc) + sr[5] * z;
    sz[3] = sr[3];
    sz[4] = sr[4];
    sz[5] = sr[5];
    double S[6][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      cplx s[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        cplx acc = mk(0.0);
#pragma unroll
        for (int j = 0; j < 6; ++j) acc += sz[j] * smon[(j * 4 + c) * 3 + k];
        s[c] = acc;
      }
      S[0][k] = scale * (s[0].re + s[1].re);
      S[1][k] = scale * (s[0].re - s[1].re);
      S[2][k] = scale * s[3].re;
      S[3][k] = scale * s[1].im;
      S[4][k] = scale * 2.0 * s[2].re;
      S[5][k] = scale * 2.0 * s[2].im;
    }
    sink(a, S);
  }
}

}  // namespace hfpx
