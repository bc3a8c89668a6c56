"""Derivation of the displacement-discontinuity (DD) -> stress kernel tables.

Run:  python -m hfpx3d_b200.codegen.derive_dd_kernel
Writes hfpx3d_b200/csrc/dd_terms.h (product) and oracle/dd_terms.h (oracle copy).

Method (own derivation, checked numerically against the reference's
make_local_3dbem_submatrix, elasticity_kernel_integration.cpp:34-205):

1. Kelvin's point-force solution U_km(r) = [(3-4nu) d_km + r_k r_m / R^2] / (16 pi G (1-nu) R).
2. Volterra's formula for a DD b on a plane with normal e3, differentiated once
   more for the stress:  sigma_pq(x) = -C_pqmn C_i3kl d_l d_n U_km (x - xi) b_i.
   K = sigma * 4 pi (1-nu) / G is homogeneous of degree -3 in r = x - xi.
3. Stress combinations used by the reference's 6x4x3 monomial tensor
   (elasticity_kernel_integration.cpp:107-110, 186-203):
       c0 = (S11+S22)/2,  c1 = (S11-S22)/2 + i S12,  c2 = (S13 + i S23)/2,  c3 = S33.
4. In the element's local frame a point of the element is xi = z + w, w = rho e^{i theta},
   and the reference's h is minus the local x3 of the observation point, so
   r1 + i r2 = -w and r3 = -h.  The product monomial_j(w) * K_{c,k} is a sum of terms
       coef(nu) * h^q * rho^(p-1) * e^{i sigma theta} / R^7,   R^2 = rho^2 + h^2,
   so every entry of the monomial tensor is a linear combination of the 23
   sector moments  W[sigma,p] = int_sector e^{i sigma theta} rho^(p-1) R^-7 dA.
   The reference stores the negated integral (its scale carries the sign).
"""
import os
import pickle
import sympy as sp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def derive():
    r1, r2, r3 = sp.symbols('r1 r2 r3', real=True)
    nu, G = sp.symbols('nu G', positive=True)
    r = [r1, r2, r3]
    R = sp.sqrt(r1**2 + r2**2 + r3**2)
    kd = lambda a, b: 1 if a == b else 0
    U = [[((3 - 4*nu)*kd(k, m) + r[k]*r[m]/R**2) / (16*sp.pi*G*(1 - nu)*R)
          for m in range(3)] for k in range(3)]
    lam = 2*G*nu/(1 - 2*nu)
    C = lambda p, q, m, n: lam*kd(p, q)*kd(m, n) + G*(kd(p, m)*kd(q, n) + kd(p, n)*kd(q, m))
    d2U = {(k, m, l, n): sp.diff(U[k][m], r[l], r[n])
           for k in range(3) for m in range(3) for l in range(3) for n in range(3)}

    def K(p, q, i):
        s = 0
        for m in range(3):
            for n in range(3):
                cpq = C(p, q, m, n)
                if cpq == 0:
                    continue
                for k in range(3):
                    for l in range(3):
                        ci = C(i, 2, k, l)
                        if ci != 0:
                            s += cpq*ci*d2U[(k, m, l, n)]
        return sp.simplify(-s*4*sp.pi*(1 - nu)/G)

    W, Wb = sp.symbols('W Wb')
    h = sp.symbols('h', real=True)
    I = sp.I
    combos = {}
    for k in range(3):
        Kk = {pq: K(pq[0], pq[1], k) for pq in [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]}
        cs = ((Kk[(0, 0)] + Kk[(1, 1)])/2,
              (Kk[(0, 0)] - Kk[(1, 1)])/2 + I*Kk[(0, 1)],
              (Kk[(0, 2)] + I*Kk[(1, 2)])/2,
              Kk[(2, 2)])
        for c, e in enumerate(cs):
            e2 = e.subs({r1: -(W + Wb)/2, r2: -(W - Wb)/(2*I), r3: -h})
            combos[(c, k)] = sp.expand(sp.simplify(e2*(W*Wb + h**2)**sp.Rational(7, 2)))
    monomials = [1, W, Wb, W**2, Wb**2, W*Wb]
    terms = []
    for j, mono in enumerate(monomials):
        for c in range(4):
            for k in range(3):
                poly = sp.Poly(sp.expand(mono*combos[(c, k)]), W, Wb, h)
                for (a, b, q), coef in poly.terms():
                    coef = sp.expand(sp.nsimplify(sp.simplify(coef)))
                    re0 = sp.re(coef.subs(nu, 0)); im0 = sp.im(coef.subs(nu, 0))
                    lin = sp.expand(coef - coef.subs(nu, 0))
                    re1 = sp.re(sp.expand(lin/nu)); im1 = sp.im(sp.expand(lin/nu))
                    assert sp.simplify(coef - (re0 + I*im0 + nu*(re1 + I*im1))) == 0
                    terms.append((j, c, k, a - b, a + b + 1, q,
                                  float(re0), float(im0), float(re1), float(im1)))
    return terms


def emit(terms, path, guard, comment):
    moments = sorted({(t[3], t[4]) for t in terms})
    mid = {m: i for i, m in enumerate(moments)}
    lines = [f'// {comment}',
             '// Generated by hfpx3d_b200/codegen/derive_dd_kernel.py -- do not edit.',
             '// Off-plane DD->stress kernel as sector moments W[sigma,p] =',
             '//   int_sector e^{i sigma theta} rho^(p-1) (rho^2+h^2)^(-7/2) dA.',
             '// Entry (j,c,k) of the monomial tensor (monomial j of w = xi - z,',
             '// stress combination c, DD component k) is',
             '//   -sum_terms (cr0 + nu cr1 + i (ci0 + nu ci1)) h^q W[moment].',
             f'#ifndef {guard}', f'#define {guard}',
             f'#define HFPX_N_MOMENTS {len(moments)}',
             f'#define HFPX_SIGMA_MAX {max(abs(s) for s, _ in moments)}  /* |sigma| bound of the moments */',
             f'#define HFPX_N_TERMS {len(terms)}',
             'typedef struct { signed char sigma, p; } hfpx_moment_t;',
             'typedef struct { unsigned char jck, moment, q, pad; double cr0, cr1, ci0, ci1; } hfpx_term_t;',
             '#ifndef HFPX_TABLE_QUAL', '#define HFPX_TABLE_QUAL static const', '#endif',
             'HFPX_TABLE_QUAL hfpx_moment_t hfpx_moments[HFPX_N_MOMENTS] = {']
    lines += [f'  {{{s}, {p}}},' for (s, p) in moments]
    lines += ['};', 'HFPX_TABLE_QUAL hfpx_term_t hfpx_terms[HFPX_N_TERMS] = {']
    for (j, c, k, s, p, q, a0, b0, a1, b1) in sorted(terms):
        lines.append(f'  {{{(j*4 + c)*3 + k}, {mid[(s, p)]}, {q}, 0, {a0!r}, {a1!r}, {b0!r}, {b1!r}}},')
    lines += ['};', f'#endif  // {guard}', '']
    with open(path, 'w') as f:
        f.write('\n'.join(lines))




# ---------------------------------------------------------------------------
# Split of the radial integrals for points near the element plane.
#
#   I_p(X) = int_0^X rho^p R^-7 d rho = F_p(X) + C_p(|h|)
#
# F_p is finite as h -> 0 and C_p(a) = c_p a^(p-6) (p <= 5), -log a (p = 6),
# -16 a / 5 (p = 7).  Summed with the kernel coefficients, the C parts of one
# (j, c, k) entry group by sigma into B[j,c,k,sigma](h); they multiply the
# exact angle integral int_sector e^{i sigma theta} d theta (vertex terms for
# sigma != 0, which cancel around a closed contour; the subtended angle for
# sigma = 0).  Exact cancellations happen here, in the algebra.
C_CONST = {1: (1, 5), 2: (2, 15), 3: (2, 15), 4: (1, 5), 5: (8, 15)}


def lower_limit_table(terms):
    nu = sp.symbols('nu', positive=True)
    a = sp.symbols('a', positive=True)
    sg, L = sp.symbols('sg L')
    Cp = {p: sp.Rational(*C_CONST[p]) / a**(6 - p) for p in C_CONST}
    Cp[6] = -L
    Cp[7] = -sp.Rational(16, 5)*a
    acc = {}
    for (j, c, k, s, p, q, a0, b0, a1, b1) in terms:
        coef = sp.nsimplify(a0) + sp.I*sp.nsimplify(b0) + nu*(sp.nsimplify(a1) + sp.I*sp.nsimplify(b1))
        acc[(j, c, k, s)] = acc.get((j, c, k, s), 0) + coef*(sg*a)**q*Cp[p]
    rows = []
    for (j, c, k, s), v in sorted(acc.items()):
        v = sp.expand(sp.simplify(sp.expand(v)))
        v = sp.expand(v.subs({sg**4: 1, sg**3: sg, sg**2: 1}))
        if v == 0:
            continue
        poly = sp.Poly(v, sg, a, 1/a, L)
        for (esg, ea, eia, eL), cf in poly.terms():
            cf = sp.expand(cf)
            re0, im0 = sp.re(cf.subs(nu, 0)), sp.im(cf.subs(nu, 0))
            lin = sp.expand((cf - cf.subs(nu, 0))/nu)
            rows.append(((j*4 + c)*3 + k, s, esg, ea - eia, eL,
                         float(re0), float(sp.re(lin)), float(im0), float(sp.im(lin))))
    return rows


def emit_lower(rows, path, guard):
    lines = ['// Generated by hfpx3d_b200/codegen/derive_dd_kernel.py -- do not edit.',
             '// Near-plane lower-limit terms: entry jck of the monomial tensor gains',
             '//   -sum (cr0 + nu cr1 + i (ci0 + nu ci1)) sgn(h)^esg |h|^ea log|h|^eL A_sigma,',
             '// A_sigma = int_sector e^{i sigma theta} d theta over the non-skipped edges.',
             f'#ifndef {guard}', f'#define {guard}', f'#define HFPX_N_LOWER {len(rows)}',
             'typedef struct { unsigned char jck; signed char sigma, esg, ea, elog, pad[3];',
             '                 double cr0, cr1, ci0, ci1; } hfpx_lower_t;',
             'HFPX_TABLE_QUAL hfpx_lower_t hfpx_lower[HFPX_N_LOWER] = {']
    for (jck, s, esg, ea, eL, a0, a1, b0, b1) in rows:
        lines.append(f'  {{{jck}, {s}, {esg}, {ea}, {eL}, {{0, 0, 0}}, {a0!r}, {a1!r}, {b0!r}, {b1!r}}},')
    lines += ['};', f'#endif  // {guard}', '']
    with open(path, 'w') as f:
        f.write('\n'.join(lines))


def main():
    terms = derive()
    emit(terms, os.path.join(ROOT, 'hfpx3d_b200', 'csrc', 'dd_terms.h'), 'HFPX_DD_TERMS_H',
         'Kernel tables for the CUDA engine.')
    emit(terms, os.path.join(ROOT, 'oracle', 'dd_terms.h'), 'HFPX_ORACLE_DD_TERMS_H',
         'Test infrastructure: kernel tables for the CPU oracle.')
    rows = lower_limit_table(terms)
    emit_lower(rows, os.path.join(ROOT, 'hfpx3d_b200', 'csrc', 'dd_lower.h'), 'HFPX_DD_LOWER_H')
    emit_lower(rows, os.path.join(ROOT, 'oracle', 'dd_lower.h'), 'HFPX_ORACLE_DD_LOWER_H')
    print(f'{len(terms)} terms, {len({(t[3], t[4]) for t in terms})} moments, {len(rows)} lower-limit terms')


if __name__ == '__main__':
    main()
