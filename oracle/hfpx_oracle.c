/* Test infrastructure: CPU oracle (plain C restatement) for the HFPx3D
 * assembly -> solve -> stress path.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg call it, as the checker.  See hfpx_oracle.h.
 *
 * Reference files cited below are paths inside the HFPx3D project.
 * Closed forms of the sector integrals are this project's own derivation
 * (hfpx3d_b200/codegen/derive_dd_kernel.py): in-plane sector moments in closed
 * form, off-plane moments by a radial closed form plus Gauss-Legendre in
 * t = asinh(a/|d|) along each edge.  The branch decisions (tolerances, skipped
 * edges, angle wrapping) follow the reference exactly.
 */
#include "hfpx_oracle.h"
#include "dd_terms.h"
#include "dd_lower.h"
#include <complex.h>
#include <math.h>
#include <string.h>

typedef double complex cplx;

/* constants.h:17-21 */
static const double PI = 3.1415926535897932385;
static const double H_TOL = 2.221e-16;
static const double A_TOL = 1.825e-8;

/* ---------------------------------------------------------------- geometry */

static void get_vert(const double *nods, int64_t ld_nods, const int64_t *conn,
                     int64_t ld_conn, int64_t el, double *v) {
  for (int j = 0; j < 3; ++j) {
    int64_t n = conn[j + ld_conn * el];
    for (int k = 0; k < 3; ++k) v[k + 3 * j] = nods[k + ld_nods * n];
  }
}

static double norm3(const double *a) { return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

static void cross3(const double *a, const double *b, double *c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

/* element_utilities.cpp:62-87 (make_el_r_tensor): rows e1, e2, e3. */
static void frame(const double *v, double *r) {
  double a1[3], a2[3], e1[3], a3[3], e3[3], a4[3];
  for (int k = 0; k < 3; ++k) { a1[k] = v[k + 3] - v[k]; a2[k] = v[k + 6] - v[k]; }
  double n1 = norm3(a1);
  for (int k = 0; k < 3; ++k) e1[k] = a1[k] / n1;
  cross3(e1, a2, a3);
  double n3 = norm3(a3);
  for (int k = 0; k < 3; ++k) e3[k] = a3[k] / n3;
  cross3(e3, e1, a4);
  double n4 = norm3(a4);
  for (int k = 0; k < 3; ++k) { r[k] = e1[k]; r[3 + k] = a4[k] / n4; r[6 + k] = e3[k]; }
}

/* element_utilities.cpp:89-118 (tau of the vertices), :120-146 and :170-238
 * (quadratic shape functions in the monomials [1, t, tc, t^2, tc^2, t tc]).
 * Node order: vertices 0..2, then node 3+v on the edge opposite vertex v. */
void ora_element_frame(const double *v, double *r, double *tau_out, double *sfm_out) {
  frame(v, r);
  cplx tau[3];
  for (int j = 0; j < 3; ++j) {
    double b[3];
    for (int k = 0; k < 3; ++k) b[k] = v[k + 3 * j] - v[k];
    double x = r[0] * b[0] + r[1] * b[1] + r[2] * b[2];
    double y = r[3] * b[0] + r[4] * b[1] + r[5] * b[2];
    tau[j] = x + I * y;
  }
  /* barycentric forms L = c + a t + b tc from t = x t1 + y t2 */
  cplx det = tau[1] * conj(tau[2]) - tau[2] * conj(tau[1]);
  cplx lx[3] = {0.0, conj(tau[2]) / det, -tau[2] / det};
  cplx ly[3] = {0.0, -conj(tau[1]) / det, tau[1] / det};
  cplx L[3][3];
  for (int i = 0; i < 3; ++i) { L[1][i] = lx[i]; L[2][i] = ly[i]; L[0][i] = -lx[i] - ly[i]; }
  L[0][0] += 1.0;
  cplx sf[6][6];
  memset(sf, 0, sizeof(sf));
  /* quadratic coefficients of the product of two linear forms */
#define PROD(P, A, B, S)                                  \
  do {                                                    \
    (P)[0] += (S) * (A)[0] * (B)[0];                      \
    (P)[1] += (S) * ((A)[0] * (B)[1] + (A)[1] * (B)[0]);  \
    (P)[2] += (S) * ((A)[0] * (B)[2] + (A)[2] * (B)[0]);  \
    (P)[3] += (S) * (A)[1] * (B)[1];                      \
    (P)[4] += (S) * (A)[2] * (B)[2];                      \
    (P)[5] += (S) * ((A)[1] * (B)[2] + (A)[2] * (B)[1]);  \
  } while (0)
  for (int vx = 0; vx < 3; ++vx) {
    PROD(sf[vx], L[vx], L[vx], 2.0);            /* L (2L - 1) */
    for (int i = 0; i < 3; ++i) sf[vx][i] -= L[vx][i];
    int a = (vx + 1) % 3, b = (vx + 2) % 3;     /* edge opposite vertex vx */
    PROD(sf[3 + vx], L[a], L[b], 4.0);
  }
#undef PROD
  for (int j = 0; j < 3; ++j) { tau_out[2 * j] = creal(tau[j]); tau_out[2 * j + 1] = cimag(tau[j]); }
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      sfm_out[2 * (6 * i + j)] = creal(sf[i][j]);
      sfm_out[2 * (6 * i + j) + 1] = cimag(sf[i][j]);
    }
}

/* element_utilities.cpp:148-166: h is minus the local x3 of the point. */
static void pt_hz(const double *v, const double *r, const double *pt, double *h, cplx *z) {
  double b[3];
  for (int k = 0; k < 3; ++k) b[k] = pt[k] - v[k];
  double x = r[0] * b[0] + r[1] * b[1] + r[2] * b[2];
  double y = r[3] * b[0] + r[4] * b[1] + r[5] * b[2];
  double w = r[6] * b[0] + r[7] * b[1] + r[8] * b[2];
  *h = -w;
  *z = x + I * y;
}

void ora_pt_hz(const double *vert, const double *pt, double *h, double *zr, double *zi) {
  double r[9];
  cplx z;
  frame(vert, r);
  pt_hz(vert, r, pt, h, &z);
  *zr = creal(z);
  *zi = cimag(z);
}

/* element_utilities.cpp:364-395 (el_cp_uniform). */
static void cp_uniform(const double *v, double beta, double cp[6][3]) {
  double c[3];
  for (int k = 0; k < 3; ++k) c[k] = v[k] / 3.0 + v[k + 3] / 3.0 + v[k + 6] / 3.0;
  for (int vx = 0; vx < 3; ++vx) {
    int m = (vx + 1) % 3, l = (m + 1) % 3;
    for (int k = 0; k < 3; ++k) {
      cp[vx][k] = (1.0 - beta) * v[k + 3 * vx] + beta * c[k];
      cp[vx + 3][k] = 0.5 * (1.0 - beta) * (v[k + 3 * m] + v[k + 3 * l]) + beta * c[k];
    }
  }
}

/* ------------------------------------------------------ in-plane moments */
/* Per edge-end antiderivatives of the in-plane finite-part moments
 *   P_j = FP int m_j(w) rho^-3 dA,  Q_j = FP int m_j(w) e^{2 i theta} rho^-3 dA
 * over the sector from z to the edge (d = |d| e, u = e^{i chi}).  Two
 * vertex-only terms (in Q_1 and Q_2) that cancel around a closed contour are
 * kept in the form h_potential.cpp:1180-1232 (s_ij_lim_h) has them, so that
 * skipped edges give the reference's values. */
static void lim_moments(double chi, cplx d, cplx *P, cplx *Q) {
  double D = cabs(d);
  double ad = carg(d);
  cplx e = cos(ad) + I * sin(ad);
  cplx u = cos(chi) + I * sin(chi);
  double s = sin(chi);
  double at = atanh(s);
  cplx e2 = e * e, u3 = u * u * u;
  P[0] = -s / D;
  P[1] = -e * at;
  P[2] = -conj(e) * at;
  P[3] = -e2 * D * (at + 2.0 * I * u);
  P[4] = -conj(e2) * D * (at - 2.0 * I * conj(u));
  P[5] = D * at;
  Q[0] = I * e2 / (6.0 * D) * (u3 + 3.0 * u);
  Q[1] = e2 * e * (at / 3.0 + (2.0 / 3.0) * I * u + I * u3 / 12.0);
  Q[2] = -e * (at + (5.0 / 12.0) * I * u);
  Q[3] = e2 * e2 * D * (at + 2.0 * I * u - (2.0 / 3.0) * I * u3);
  Q[4] = D * at;
  Q[5] = -e2 * D * (at + 2.0 * I * u);
}

/* ----------------------------------------------------- off-plane moments */
/* I_p(X) = int_0^X rho^p (rho^2+h^2)^(-7/2) d rho in forms that stay accurate
 * for X << |h| (delta = 1 - |h|/R). */
static void radial(double X, double h, double *Ip) {
  h = fabs(h);
  double R = hypot(X, h), s = X / R, dl = X * X / (R * (R + h));
  double s3 = s * s * s, s5 = s3 * s * s;
  double d2 = dl * dl, d3 = d2 * dl, d4 = d2 * d2, d5 = d4 * dl, d6 = d3 * d3;
  double h2 = h * h, h3 = h2 * h, h4 = h2 * h2, h5 = h4 * h;
  Ip[1] = dl * (5.0 - 10.0 * dl + 10.0 * d2 - 5.0 * d3 + d4) / (5.0 * h5);
  Ip[2] = (s3 / 3.0 - s5 / 5.0) / h4;
  Ip[3] = (d2 - 5.0 * d3 / 3.0 + d4 - d5 / 5.0) / h3;
  Ip[4] = s5 / (5.0 * h2);
  Ip[5] = (4.0 * d3 / 3.0 - d4 + d5 / 5.0) / h;
  if (s < 0.6) {
    double acc = 0.0, t = s5 * s * s, s2 = s * s;
    for (int k = 3; k < 200; ++k) {
      double term = t / (2 * k + 1);
      acc += term;
      if (term <= 1e-17 * acc) break;
      t *= s2;
    }
    Ip[6] = acc;
  } else {
    Ip[6] = atanh(s) - s - s3 / 3.0 - s5 / 5.0;
  }
  Ip[7] = R * (2.0 * d4 - 1.2 * d5 + 0.2 * d6);
}

static double gl_x[12], gl_w[12];
static int gl_ready = 0;

static void gl_init(void) {
  const int n = 12;
  for (int i = 0; i < n; ++i) {
    double x = cos(PI * (i + 0.75) / (n + 0.5)), dp = 1.0;
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
      if (fabs(dx) < 1e-16) break;
    }
    gl_x[i] = x;
    gl_w[i] = 2.0 / ((1.0 - x * x) * dp * dp);
  }
  gl_ready = 1;
}

/* Radial integrals without their h-singular lower-limit constants:
 * F_p(X) = I_p(X) - C_p(|h|), finite as h -> 0 (e = 1 - X/R, ee = e / h^2). */
static void radial_upper(double X, double h, double *F) {
  h = fabs(h);
  double R = hypot(X, h), s = X / R, ee = 1.0 / (R * (R + X)), e = h * h * ee;
  double iR = 1.0 / R, iR2 = iR * iR, iR3 = iR2 * iR, iR5 = iR3 * iR2, h2 = h * h;
  F[1] = -0.2 * iR5;
  F[2] = -ee * ee * (1.0 - 5.0 * e / 3.0 + e * e - 0.2 * e * e * e);
  F[3] = -(iR3 / 3.0 - 0.2 * h2 * iR5);
  F[4] = -ee * (5.0 - 10.0 * e + 10.0 * e * e - 5.0 * e * e * e + e * e * e * e) * 0.2;
  F[5] = -(iR - 2.0 * h2 * iR3 / 3.0 + 0.2 * h2 * h2 * iR5);
  F[6] = log((1.0 + s) * R) - s - s * s * s / 3.0 - 0.2 * s * s * s * s * s;
  F[7] = R + 3.0 * h2 * iR - h2 * h2 * iR3 + 0.2 * h2 * h2 * h2 * iR5;
}

/* Sector moments W[sigma,p] for the edge with foot d, from angle chi_m to chi_n:
 * along the edge a = |d| tan(chi) = |d| sinh(t); d theta = dt / cosh t.
 * upper != 0 integrates F_p (near-plane form) instead of I_p. */
static void gen_moments(double chi_m, double chi_n, cplx d, double h, int upper, cplx *Wm) {
  if (!gl_ready) gl_init();
  double D = cabs(d), ad = carg(d);
  cplx e = cos(ad) + I * sin(ad);
  double tm = asinh(tan(chi_m)), tn = asinh(tan(chi_n));
  int npan = (int)ceil(fabs(tn - tm) / 1.5);
  if (npan < 1) npan = 1;
  if (npan > 64) npan = 64;
  for (int ip = 0; ip < npan; ++ip) {
    double a0 = tm + (tn - tm) * ip / npan, a1 = tm + (tn - tm) * (ip + 1) / npan;
    double hw = 0.5 * (a1 - a0), mid = 0.5 * (a0 + a1);
    for (int g = 0; g < 12; ++g) {
      double t = mid + hw * gl_x[g];
      double ch = cosh(t), sh = sinh(t);
      double wt = hw * gl_w[g] / ch;
      double Ip[8];
      if (upper) radial_upper(D * ch, h, Ip);
      else radial(D * ch, h, Ip);
      cplx eth = e * (1.0 + I * sh) / ch;
      enum { S = HFPX_SIGMA_MAX };
      cplx pw[2 * S + 1];  /* e^{i s theta}, s = -S..S */
      pw[S] = 1.0;
      for (int s = 1; s <= S; ++s) pw[S + s] = pw[S + s - 1] * eth;
      for (int s = 1; s <= S; ++s) pw[S - s] = conj(pw[S + s]);
      for (int m = 0; m < HFPX_N_MOMENTS; ++m)
        Wm[m] += wt * pw[S + hfpx_moments[m].sigma] * Ip[hfpx_moments[m].p];
    }
  }
}

/* --------------------------------------------------------- local block */
/* elasticity_kernel_integration.cpp:34-205 (make_local_3dbem_submatrix). */
static void local_block(double G, double nu, double h, cplx z, const cplx *tau,
                        const cplx sfm[6][6], double out[6][18]) {
  cplx tz[3], d[3];
  for (int j = 0; j < 3; ++j) {
    int q = (j + 1) % 3;
    tz[j] = tau[j] - z;
    cplx dt = tau[q] - tau[j];
    cplx nt2 = dt / conj(dt);
    d[j] = 0.5 * (tz[j] - nt2 * conj(tz[j]));
  }
  double phi[3], psi[3], chi[2][3];
  int is90[2][3] = {{0}};
  for (int j = 0; j < 3; ++j) { phi[j] = carg(tz[j]); psi[j] = carg(d[j]); }
  for (int j = 0; j < 3; ++j)
    for (int k = 0; k < 2; ++k) {
      double c = phi[(j + k) % 3] - psi[j];
      if (c <= -PI) { while (c <= -PI) c += 2.0 * PI; }
      else if (c > PI) { while (c > PI) c -= 2.0 * PI; }
      chi[k][j] = c;
      if (fabs(0.5 * PI - fabs(c)) < A_TOL) is90[k][j] = 1;
    }
  cplx smon[6][4][3];
  memset(smon, 0, sizeof(smon));
  const int in_plane = fabs(h) < H_TOL;
  /* Off-plane points below the element's span (|h| < largest vertex distance
   * in the plane) integrate the regular parts F_p and add the h-singular
   * lower-limit parts in closed form; points above it integrate I_p as is. */
  double span = 0.0;
  for (int j = 0; j < 3; ++j) if (cabs(tz[j]) > span) span = cabs(tz[j]);
  const int upper = !in_plane && fabs(h) < 0.05 * span;
  cplx P[6] = {0}, Q[6] = {0}, Wm[HFPX_N_MOMENTS];
  memset(Wm, 0, sizeof(Wm));
  int vcount[3] = {0, 0, 0};
  double angle = 0.0;
  for (int m = 0; m < 3; ++m) {
    if (!(cabs(d[m]) >= H_TOL && !is90[0][m] && !is90[1][m])) continue;
    if (in_plane) {
      cplx Pn[6], Qn[6], Pm[6], Qm[6];
      lim_moments(chi[1][m], d[m], Pn, Qn);
      lim_moments(chi[0][m], d[m], Pm, Qm);
      for (int j = 0; j < 6; ++j) { P[j] += Pn[j] - Pm[j]; Q[j] += Qn[j] - Qm[j]; }
    } else {
      gen_moments(chi[0][m], chi[1][m], d[m], h, upper, Wm);
      vcount[(m + 1) % 3] += 1;
      vcount[m] -= 1;
      angle += chi[1][m] - chi[0][m];
    }
  }
  if (in_plane) {
    for (int j = 0; j < 6; ++j) {
      smon[j][0][2] = -0.5 * (1.0 + 2.0 * nu) * P[j];
      smon[j][1][2] = -1.5 * (1.0 - 2.0 * nu) * Q[j];
      smon[j][3][2] = -P[j];
      smon[j][2][0] = -(0.25 * (2.0 - nu) * P[j] + 0.75 * nu * Q[j]);
      smon[j][2][1] = -I * (0.25 * (2.0 - nu) * P[j] - 0.75 * nu * Q[j]);
    }
  } else {
    double hq[5] = {1.0, h, h * h, h * h * h, h * h * h * h};
    for (int t = 0; t < HFPX_N_TERMS; ++t) {
      const hfpx_term_t *tm = &hfpx_terms[t];
      int jck = tm->jck, j = jck / 12, c = (jck / 3) % 4, k = jck % 3;
      cplx coef = (tm->cr0 + nu * tm->cr1) + I * (tm->ci0 + nu * tm->ci1);
      smon[j][c][k] -= coef * hq[tm->q] * Wm[tm->moment];
    }
    if (upper) {
      /* A_sigma: vertex terms e^{i sigma phi_v} / (i sigma) weighted by how
       * often the kept edges end (+1) or start (-1) at vertex v, which is
       * exactly zero for a closed contour; A_0 is the subtended angle. */
      const double ah = fabs(h), lg = log(ah), sg = h > 0 ? 1.0 : -1.0;
      for (int t = 0; t < HFPX_N_LOWER; ++t) {
        const hfpx_lower_t *lw = &hfpx_lower[t];
        cplx A = 0.0;
        if (lw->sigma == 0) A = angle;
        else
          for (int v = 0; v < 3; ++v)
            if (vcount[v]) A += vcount[v] * cexp(I * (lw->sigma * phi[v])) / (I * lw->sigma);
        double f = (lw->esg ? sg : 1.0) * (lw->ea == 1 ? ah : (lw->ea == -1 ? 1.0 / ah : 1.0)) *
                   (lw->elog ? lg : 1.0);
        cplx coef = (lw->cr0 + nu * lw->cr1) + I * (lw->ci0 + nu * lw->ci1);
        int jck = lw->jck;
        smon[jck / 12][(jck / 3) % 4][jck % 3] -= coef * f * A;
      }
    }
  }
  /* shifted shape functions sfm . shift(z) (element_utilities.cpp:339-360) */
  cplx zc = conj(z), sh[6][6];
  memset(sh, 0, sizeof(sh));
  sh[0][0] = 1; sh[1][0] = z; sh[1][1] = 1; sh[2][0] = zc; sh[2][2] = 1;
  sh[3][0] = z * z; sh[3][1] = 2.0 * z; sh[3][3] = 1;
  sh[4][0] = zc * zc; sh[4][2] = 2.0 * zc; sh[4][4] = 1;
  sh[5][0] = z * zc; sh[5][1] = zc; sh[5][2] = z; sh[5][5] = 1;
  double scale = -G / (4.0 * PI * (1.0 - nu));
  for (int a = 0; a < 6; ++a) {
    cplx sz[6];
    for (int j = 0; j < 6; ++j) {
      sz[j] = 0;
      for (int l = 0; l < 6; ++l) sz[j] += sfm[a][l] * sh[l][j];
    }
    for (int k = 0; k < 3; ++k) {
      cplx s[4];
      for (int c = 0; c < 4; ++c) {
        s[c] = 0;
        for (int j = 0; j < 6; ++j) s[c] += sz[j] * smon[j][c][k];
      }
      int q = 3 * a + k;
      out[0][q] = scale * (creal(s[0]) + creal(s[1]));
      out[1][q] = scale * (creal(s[0]) - creal(s[1]));
      out[2][q] = scale * creal(s[3]);
      out[3][q] = scale * cimag(s[1]);
      out[4][q] = scale * 2.0 * creal(s[2]);
      out[5][q] = scale * 2.0 * cimag(s[2]);
    }
  }
}

static void unpack(const double *tau, const double *sfm, cplx *t, cplx s[6][6]) {
  for (int j = 0; j < 3; ++j) t[j] = tau[2 * j] + I * tau[2 * j + 1];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) s[i][j] = sfm[2 * (6 * i + j)] + I * sfm[2 * (6 * i + j) + 1];
}

void ora_local_block(double G, double nu, double h, double zr, double zi,
                     const double *tau, const double *sfm, double *out) {
  cplx t[3], s[6][6];
  unpack(tau, sfm, t, s);
  local_block(G, nu, h, zr + I * zi, t, s, (double(*)[18])out);
}

/* ------------------------------------------------------------ DoF handle */
/* surface_mesh_utilities.cpp:28-112 (make_dof_h_crack, order 2). */
int64_t ora_dof_handle(const double *nods, int64_t ld_nods, int64_t n_nodes,
                       const int64_t *conn, int64_t ld_conn, int64_t n_el,
                       int tip_type, int64_t *dof_h) {
  (void)n_nodes;
  const int ext = ld_nods >= 5 && ld_conn >= 5;
  int64_t n_dof = 18 * n_el, dec = 0;
  for (int64_t el = 0; el < n_el; ++el)
    for (int l = 0; l < 18; ++l) dof_h[el + n_el * l] = 18 * el + l;
  for (int64_t el = 0; el < n_el; ++el) {
    int tip[3] = {0, 0, 0};
    if (ext && conn[3 + ld_conn * el] == conn[4 + ld_conn * el])
      for (int v = 0; v < 3; ++v) {
        int64_t n = conn[v + ld_conn * el];
        if (nods[3 + ld_nods * n] == 1.0 && nods[4 + ld_nods * n] == 1.0) tip[v] = 1;
      }
    for (int v = 0; v < 6; ++v) {
      /* 0: shift by the running count, 1: fix, 2: leave as is (the reference
       * does not shift non-tip edge nodes when tip_type == 2) */
      int act = 0;
      if (tip_type >= 1 && v < 3 && tip[v]) act = 1;
      else if (tip_type == 2 && v >= 3) {
        int a = (v - 3 + 1) % 3, b = (a + 1) % 3;
        act = (tip[a] && tip[b]) ? 1 : 2;
      }
      for (int l = 0; l < 3; ++l) {
        int64_t *p = &dof_h[el + n_el * (3 * v + l)];
        if (act == 1) { --n_dof; ++dec; *p = -1; }
        else if (act == 0) *p -= dec;
      }
    }
  }
  return n_dof;
}

/* -------------------------------------------------------------- assembly */
typedef struct {
  double v[9], r[9];
  cplx tau[3], sfm[6][6];
} elem_t;

static void make_elem(const double *nods, int64_t ld_nods, const int64_t *conn,
                      int64_t ld_conn, int64_t el, elem_t *E) {
  double tau[6], sfm[72];
  get_vert(nods, ld_nods, conn, ld_conn, el, E->v);
  ora_element_frame(E->v, E->r, tau, sfm);
  unpack(tau, sfm, E->tau, E->sfm);
}

/* traction block (3x18) at a point with global normal n due to global (or
 * local) DD of source element E: system_assembly.cpp:117-196. */
static void traction_block(double G, double nu, const elem_t *E, const double *pt,
                           const double *n, int is_dd_local, double blk[3][18]) {
  double h, S[6][18];
  cplx z;
  pt_hz(E->v, E->r, pt, &h, &z);
  local_block(G, nu, h, z, E->tau, E->sfm, S);
  const double *r = E->r;
  double nl[3];
  for (int i = 0; i < 3; ++i) nl[i] = r[3 * i] * n[0] + r[3 * i + 1] * n[1] + r[3 * i + 2] * n[2];
  double tl[3][18], tg[3][18];
  for (int q = 0; q < 18; ++q) {
    tl[0][q] = nl[0] * S[0][q] + nl[1] * S[3][q] + nl[2] * S[4][q];
    tl[1][q] = nl[1] * S[1][q] + nl[0] * S[3][q] + nl[2] * S[5][q];
    tl[2][q] = nl[2] * S[2][q] + nl[0] * S[4][q] + nl[1] * S[5][q];
  }
  for (int a = 0; a < 3; ++a)
    for (int q = 0; q < 18; ++q) tg[a][q] = r[a] * tl[0][q] + r[3 + a] * tl[1][q] + r[6 + a] * tl[2][q];
  if (is_dd_local) { memcpy(blk, tg, sizeof(tg)); return; }
  for (int ns = 0; ns < 6; ++ns)
    for (int a = 0; a < 3; ++a)
      for (int j = 0; j < 3; ++j)
        blk[a][3 * ns + j] = tg[a][3 * ns] * r[j] + tg[a][3 * ns + 1] * r[3 + j] + tg[a][3 * ns + 2] * r[6 + j];
}

static int assemble_range(const double *nods, int64_t ld_nods, const int64_t *conn,
                          int64_t ld_conn, int64_t n_el, const int64_t *dof_h,
                          double G, double nu, double beta, int is_dd_local,
                          int64_t t0, int64_t t1, double *out, int64_t ld) {
  for (int64_t s = 0; s < n_el; ++s) {
    elem_t S;
    make_elem(nods, ld_nods, conn, ld_conn, s, &S);
    for (int64_t t = t0; t < t1; ++t) {
      double vt[9], rt[9], cp[6][3], n[3];
      get_vert(nods, ld_nods, conn, ld_conn, t, vt);
      frame(vt, rt);
      for (int k = 0; k < 3; ++k) n[k] = -rt[6 + k];
      cp_uniform(vt, beta, cp);
      for (int nt = 0; nt < 6; ++nt) {
        double blk[3][18];
        traction_block(G, nu, &S, cp[nt], n, is_dd_local, blk);
        for (int i1 = 0; i1 < 18; ++i1) {
          int64_t c = dof_h[s + n_el * i1];
          if (c < 0) continue;
          for (int k = 0; k < 3; ++k) {
            int64_t rr = dof_h[t + n_el * (3 * nt + k)];
            if (rr >= 0) out[rr + ld * c] += blk[k][i1];
          }
        }
      }
    }
  }
  return 0;
}

int ora_assemble_rows(const double *nods, int64_t ld_nods, int64_t n_nodes,
                      const int64_t *conn, int64_t ld_conn, int64_t n_el,
                      const int64_t *dof_h, int64_t n_dof,
                      double G, double nu, double beta, int is_dd_local,
                      int64_t t0, int64_t t1, double *out, int64_t ld) {
  (void)n_nodes; (void)n_dof;
  return assemble_range(nods, ld_nods, conn, ld_conn, n_el, dof_h, G, nu, beta, is_dd_local,
                        t0, t1, out, ld);
}

/* system_assembly.cpp:30-219 and, for vc, :458-557.  The shape-function
 * integrals of a flat quadratic triangle are 0 (vertex nodes) and A/3 (edge
 * nodes); the reference evaluates the same integrals by contour integration
 * (element_utilities.cpp:484-510, 573-595). */
int ora_assemble(const double *nods, int64_t ld_nods, int64_t n_nodes,
                 const int64_t *conn, int64_t ld_conn, int64_t n_el,
                 const int64_t *dof_h, int64_t n_dof,
                 double G, double nu, double beta, int is_dd_local, int vc,
                 double *out, int64_t ld) {
  (void)n_nodes;
  int64_t n = n_dof + (vc ? 1 : 0);
  for (int64_t j = 0; j < n; ++j) memset(out + ld * j, 0, sizeof(double) * n);
  assemble_range(nods, ld_nods, conn, ld_conn, n_el, dof_h, G, nu, beta, is_dd_local,
                 0, n_el, out, ld);
  if (!vc) return 0;
  for (int64_t s = 0; s < n_el; ++s) {
    double v[9], r[9], a1[3], a2[3], c[3];
    get_vert(nods, ld_nods, conn, ld_conn, s, v);
    frame(v, r);
    for (int k = 0; k < 3; ++k) { a1[k] = v[k + 3] - v[k]; a2[k] = v[k + 6] - v[k]; }
    cross3(a1, a2, c);
    double area = 0.5 * norm3(c);
    for (int ns = 0; ns < 6; ++ns) {
      double sfi = ns < 3 ? 0.0 : area / 3.0;
      for (int j = 0; j < 3; ++j) {
        int64_t sd = dof_h[s + n_el * (3 * ns + j)];
        if (sd < 0) continue;
        out[n_dof + ld * sd] = is_dd_local ? (j == 2 ? sfi : 0.0) : sfi * r[6 + j];
        out[sd + ld * n_dof] = -r[6 + j];
      }
    }
  }
  out[n_dof + ld * n_dof] = 0.0;
  return 0;
}

/* system_assembly.cpp:222-274 (add_s_inf_to_3dbem_rhs). */
void ora_rhs(const double *nods, int64_t ld_nods, const int64_t *conn, int64_t ld_conn,
             int64_t n_el, const int64_t *dof_h, const double *si, double *rhs) {
  for (int64_t el = 0; el < n_el; ++el) {
    double v[9], r[9], n[3];
    get_vert(nods, ld_nods, conn, ld_conn, el, v);
    frame(v, r);
    for (int k = 0; k < 3; ++k) n[k] = -r[6 + k];
    double t[3] = {n[0] * si[0] + n[1] * si[3] + n[2] * si[4],
                   n[1] * si[1] + n[0] * si[3] + n[2] * si[5],
                   n[2] * si[2] + n[0] * si[4] + n[1] * si[5]};
    for (int ln = 0; ln < 6; ++ln)
      for (int l = 0; l < 3; ++l) {
        int64_t dof = dof_h[el + n_el * (3 * ln + l)];
        if (dof != -1) rhs[dof] -= t[l];
      }
  }
}

/* system_assembly.cpp:279-455 (make_3dbem_stress_f_s), single-threaded. */
void ora_stress(const double *nods, int64_t ld_nods, const int64_t *conn, int64_t ld_conn,
                int64_t n_el, double G, double nu, int is_dd_local, const double *dd,
                const double *pts, int64_t n_pts, const double *si, double *out) {
  for (int64_t i = 0; i < 6 * n_pts; ++i) out[i] = 0.0;
  for (int64_t s = 0; s < n_el; ++s) {
    elem_t E;
    make_elem(nods, ld_nods, conn, ld_conn, s, &E);
    const double *r = E.r;
    for (int64_t p = 0; p < n_pts; ++p) {
      double h, S[6][18], Sg[6][18];
      cplx z;
      pt_hz(E.v, E.r, pts + 3 * p, &h, &z);
      local_block(G, nu, h, z, E.tau, E.sfm, S);
      /* tensor_utilities.cpp:57-91 (rotate_sim): sigma_g = R^T sigma R */
      for (int q = 0; q < 18; ++q) {
        double m[3][3] = {{S[0][q], S[3][q], S[4][q]},
                          {S[3][q], S[1][q], S[5][q]},
                          {S[4][q], S[5][q], S[2][q]}};
        double t[3][3], g[3][3];
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) t[a][b] = m[a][0] * r[b] + m[a][1] * r[3 + b] + m[a][2] * r[6 + b];
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) g[a][b] = r[a] * t[0][b] + r[3 + a] * t[1][b] + r[6 + a] * t[2][b];
        Sg[0][q] = g[0][0]; Sg[1][q] = g[1][1]; Sg[2][q] = g[2][2];
        Sg[3][q] = g[0][1]; Sg[4][q] = g[0][2]; Sg[5][q] = g[1][2];
      }
      if (!is_dd_local) {
        for (int ns = 0; ns < 6; ++ns)
          for (int a = 0; a < 6; ++a) {
            double b0 = Sg[a][3 * ns], b1 = Sg[a][3 * ns + 1], b2 = Sg[a][3 * ns + 2];
            for (int j = 0; j < 3; ++j) Sg[a][3 * ns + j] = b0 * r[j] + b1 * r[3 + j] + b2 * r[6 + j];
          }
      }
      for (int a = 0; a < 6; ++a) {
        double acc = 0.0;
        for (int k = 0; k < 6; ++k)
          for (int j = 0; j < 3; ++j) acc += Sg[a][3 * k + j] * dd[(6 * s + k) + 6 * n_el * j];
        out[p + n_pts * a] += acc;
      }
    }
  }
  for (int64_t p = 0; p < n_pts; ++p)
    for (int a = 0; a < 6; ++a) out[p + n_pts * a] += si[a];
}

/* surface_mesh_utilities.cpp:256-328 (write_dd_vector_to_md). */
void ora_dd_from_solution(const double *sol, const int64_t *dof_h, int64_t n_el, double *dd) {
  for (int64_t el = 0; el < n_el; ++el)
    for (int en = 0; en < 6; ++en)
      for (int i = 0; i < 3; ++i) {
        int64_t g = dof_h[el + n_el * (3 * en + i)];
        dd[(6 * el + en) + 6 * n_el * i] = g >= 0 ? sol[g] : 0.0;
      }
}

/* --------------------------------------------------------------- Sneddon */
/* test_radial_crack_static.cpp:316-337 */
void ora_sneddon_dd(double G, double nu, double a, double p, const double *x, double *dd) {
  double sc = 4.0 * (1.0 - nu) * a * p / (G * PI);
  double r2 = x[0] * x[0] + x[1] * x[1];
  dd[0] = dd[1] = 0.0;
  dd[2] = r2 / (a * a) < 1.0 ? sc * sqrt(1.0 - r2 / (a * a)) : 0.0;
}

/* test_radial_crack_static.cpp:340-401: stress of a pressurised penny crack
 * (Sneddon) through the potential derivatives F_ij, F_ijz. */
void ora_sneddon_stress(double G, double nu, double a, double p, const double *x, double *sv) {
  double sc = p / G, fac = 2.0 / PI, a2 = a * a;
  double x2 = x[0] * x[0], y2 = x[1] * x[1], xy = x[0] * x[1];
  double r = sqrt(x2 + y2), r2 = r * r, r3 = r * r2;
  double z = fabs(x[2]), z2 = z * z;
  double sp = sqrt((a + r) * (a + r) + z2), sm = sqrt((a - r) * (a - r) + z2);
  double L1 = 0.5 * (sp - sm), L2 = 0.5 * (sp + sm);
  double g0 = asin(L1 / r), g1 = L1 / L2, L14 = L1 * L1 * L1 * L1;
  double g2 = L2 * L2 - L1 * L1, g23 = g2 * g2 * g2;
  double g3 = sqrt(a2 - L1 * L1), g4 = sqrt(L2 * L2 - a2), g5 = sqrt(r2 - L1 * L1);
  double Fr = 0.5 * r * g0 - 0.5 * g1 * g4;
  double Frr = 0.5 * g0 - 0.5 * a * (1.0 + g1 * g1) * g4 / g2;
  double Fxx = x2 / r2 * Frr + y2 / r3 * Fr, Fyy = y2 / r2 * Frr + x2 / r3 * Fr;
  double Fxy = xy / r2 * Frr - xy / r3 * Fr;
  double Fzz = -g0 + a * g4 / g2, Frz = -a * g1 * g3 / g2;
  double Frrz = a2 * z / (L2 * L2) / g4 * (4.0 * r2 * g4 / g23 - (a2 + z2) / (g2 * g2));
  double Fxxz = x2 / r2 * Frrz + y2 / r3 * Frz, Fyyz = y2 / r2 * Frrz + x2 / r3 * Frz;
  double Fxyz = xy / r2 * Frrz - xy / r3 * Frz;
  double Frzz = a / L2 * g5 / g23 * (a2 * (4.0 * L2 * L2 - 5.0 * r2) + L14);
  double Fxzz = x[0] / r * Frzz, Fyzz = x[1] / r * Frzz;
  double Fzzz = g3 / g23 * (L14 + a2 * (2.0 * a2 + 2.0 * z2 - 3.0 * r2));
  sv[0] = -sc * fac * (z * Fxxz + Fxx + 2.0 * nu * Fyy);
  sv[1] = -sc * fac * (z * Fyyz + Fyy + 2.0 * nu * Fxx);
  sv[2] = sc * (1.0 - fac * (z * Fzzz - Fzz));
  sv[3] = -sc * fac * (z * Fxyz + (1.0 - 2.0 * nu) * Fxy);
  sv[4] = -sc * fac * (z * Fxzz);
  sv[5] = -sc * fac * (z * Fyzz);
}
