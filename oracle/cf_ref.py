"""Test infrastructure: a CPU restatement of the reference's volume-control
iteration with cohesion and friction, the checker of hfpx_cf_match,
hfpx_cf_update_mrd and hfpx_vc_cf_iteration.  It is not used by the
product.

It follows, statement by statement:
* match_f_c  (src/Development/cohesion_friction.cpp:22-130),
* update_mrd (src/Development/cohesion_friction.cpp:134-194),
* vc_cf_iteration (src/Development/c_f_iteration.cpp:27-436), with the
  truncated system of mod_3dbem_system_vc (src/Solvers/system_assembly.cpp:
  560-629) taken from vc_ref.py and solved by numpy (il::linearSolve, LAPACK
  dgesv, in the reference).

Where the reference's statements disagree with each other, this restatement
(and the engine) takes one reading, each listed here:
1. DoF renumbering in element and node order: the reference decrements a
   counter shared by the threads of an OpenMP loop (c_f_iteration.cpp:
   93-95, 212-256), so its numbering depends on thread timing;
2. a DoF that no branch renumbers stays active with the next number (the
   reference leaves its entry of dof_h_dd as it was before the step);
3. the intact point's DoF that the original handle already fixes (-1) are
   not counted in the decrement (the reference counts them);
4. tractions and volume come from the current DD over the original
   numbering with the pressure unknown 0 (the reference gathers dd_v by the
   truncated handle, :65, and multiplies by the original matrix, :69);
5. the volume row is the bordered matrix's own last row (the reference reads
   row orig_ndof of a matrix it requires to be orig_ndof square, :58, :74);
6. the traction of a point DoF the original handle fixes is 0 (the
   reference leaves it uninitialised, :157-164);
7. after the clamp the element DD are local; the reference rotates them once
   more when is_dd_local is false (:392-395);
8. match_f_c and update_mrd per point (the reference's nodal DD array is
   shared by the OpenMP threads, cohesion_friction.cpp:41-42, 150).
The traction adjustments enter the right-hand side for components 0 and 1,
as the reference's loop does (:262-268); all_components=True adds all three.
They enter with the reference's sign: the system A d(dd) = dt with dt =
-(excess traction) raises the traction A dd that the check subtracts by dt,
so the excess doubles and the iteration grows; release_sign=True takes the
opposite sign, with which the iteration settles.

Parity: unpinned against a run of the reference, whose iteration cannot run
as written (mod_3dbem_system_vc reads past its matrix; the caller passes the
bordered matrix its checks reject).  Pinned on the loops restated here.
"""
import os
import sys
from types import SimpleNamespace

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import vc_ref  # noqa: E402


def element_data(ora, nods, conn, beta):
    """Per element: the frame r (rows e1, e2, e3), the normal -e3 and sf_cp
    (6 x 6, row = collocation point, column = node), as set_ele_struct forms
    them (element_utilities.cpp:433-480)."""
    out = []
    for el in range(conn.shape[1]):
        vert = nods[:3, conn[:3, el]]
        r, tau, sfm = ora.element_frame(vert)
        sfm = (sfm[0::2] + 1j * sfm[1::2]).reshape(6, 6)
        c = vert[:, 0] / 3.0 + vert[:, 1] / 3.0 + vert[:, 2] / 3.0
        cps = []
        for vx in range(3):
            cps.append((1.0 - beta) * vert[:, vx] + beta * c)
        for vx in range(3):
            m, l = (vx + 1) % 3, (vx + 2) % 3
            cps.append(0.5 * (1.0 - beta) * (vert[:, m] + vert[:, l]) + beta * c)
        sf = np.empty((6, 6))
        for n, p in enumerate(cps):
            _, z = ora.pt_hz(vert, p)
            tv = np.array([1.0, z, np.conj(z), z * z, np.conj(z) ** 2, z * np.conj(z)])
            sf[n] = np.real(sfm @ tv)
        out.append(SimpleNamespace(r=r, nrm=-r[2], sf=sf))
    return out


def match_f_c(mats, mat_id, dd, mr_open, mr_slip):
    """cohesion_friction.cpp:22-130 -> (friction_coef, slip_cohesion, open_cohesion)."""
    n_cp = dd.shape[0]
    fric, sc, oc = np.zeros(n_cp), np.zeros(n_cp), np.zeros(n_cp)
    for n in range(n_cp):
        p = mats[mat_id[n]]
        dl_open = dd[n, 2] / p['cr_open']
        pr_open = mr_open[n]
        dl_slip = np.sqrt(dd[n, 0] ** 2 + dd[n, 1] ** 2) / p['cr_slip']
        pr_slip = mr_slip[n]
        r_s = 0.0
        if 0.0 < dl_open < 1.0:
            if p['cohesion_model'] == 1:
                r_s = 1.0 - dl_open
            elif p['cohesion_model'] == 0:
                r_s = 1.0
        if 0.0 < dl_open < pr_open:
            r_s *= dl_open / pr_open
        oc[n] = p['peak_ts'] * r_s
        sc[n] = p['peak_sc'] * r_s
        r_f = 0.0
        if dl_open < 1.0:
            r_f = p['res_sf']
            if p['friction_model'] == 1:
                if dl_slip < 1.0:
                    m = pr_slip if dl_slip < pr_slip else dl_slip
                    r_f = p['res_sf'] + (p['peak_sf'] - p['res_sf']) * (1.0 - m)
            elif p['friction_model'] == 0:
                r_f = p['peak_sf']
        fric[n] = r_f
    return fric, sc, oc


def update_mrd(mats, mat_id, dd, mr_open, mr_slip):
    """cohesion_friction.cpp:134-194 -> (mr_open, mr_slip) updated copies."""
    mo, ms = np.array(mr_open, dtype=np.float64), np.array(mr_slip, dtype=np.float64)
    for n in range(dd.shape[0]):
        p = mats[mat_id[n]]
        dl_open = dd[n, 2] / p['cr_open']
        dl_slip = np.sqrt(dd[n, 0] ** 2 + dd[n, 1] ** 2) / p['cr_slip']
        pr_open, pr_slip = mo[n], ms[n]
        if dl_slip > pr_slip:
            ms[n] = dl_slip
        if dl_open >= 1.0:
            mo[n] = 1.0
        if dl_open > pr_open:
            mo[n] = dl_open
    return mo, ms


def vc_cf_iteration(elems, A, orig_dof_h, mats, st, s_inf, inj_cp, new_vol, is_dd_local=False,
                    all_components=False, release_sign=False):
    """c_f_iteration.cpp:27-436.  elems: element_data(); A: the bordered
    matrix (n + 1 square) of orig_dof_h (n_el x 18); st: namespace with dd
    (n_cp x 3), pp, mr_open, mr_slip, mat_id (not modified).  Returns the
    new state (dd, pp, friction_coef, slip_cohesion, open_cohesion, dof_h,
    n_dof) and info (residual, volume, pressure, delta_p, n_fixed, the
    count of points in each branch)."""
    od = np.asarray(orig_dof_h, dtype=np.int64)
    n_el = od.shape[0]
    n = A.shape[0] - 1
    dd = np.array(st.dd, dtype=np.float64)
    pp = np.array(st.pp, dtype=np.float64)
    # the fracture state's cohesion and friction (:87-89)
    fric, sc, oc = match_f_c(mats, st.mat_id, dd, st.mr_open, st.mr_slip)
    # dd over the original numbering, the elastic tractions and the volume (:65-77)
    x = np.zeros(n + 1)
    for el in range(n_el):
        for l in range(18):
            if od[el, l] >= 0:
                x[od[el, l]] = dd[6 * el + l // 3, l % 3]
    e_t = A[:n] @ x
    volume = float(A[n] @ x)
    delta_v = new_vol - volume
    pressure = pp[inj_cp]
    s = np.asarray(s_inf, dtype=np.float64)
    sig = np.array([[s[0], s[3], s[4]], [s[3], s[1], s[5]], [s[4], s[5], s[2]]])
    delta_trac = np.zeros(n)
    fixed = np.zeros((n_el, 18), dtype=bool)
    counts = dict(separation=0, cohesion=0, slip=0, intact=0)
    ncomp = 3 if all_components else 2
    for el in range(n_el):
        E = elems[el]
        ti = E.r @ (sig @ E.nrm)
        pr_el = pp[6 * el:6 * el + 6]
        for lnn in range(6):
            g = 6 * el + lnn
            tr = np.zeros(3)
            for i in range(3):
                d = od[el, 3 * lnn + i]
                if d >= 0:
                    tr[i] = e_t[d]
            tr = E.r @ tr
            pr_cp = pr_el @ E.sf[lnn]
            nt = pr_cp - ti[2] - tr[2]
            stc = np.array([-ti[0] - tr[0], -ti[1] - tr[1]])
            sh = np.sqrt(stc[0] ** 2 + stc[1] ** 2)
            adm_nt = oc[g]
            adm_st = sc[g] - fric[g] * nt
            sh_dir = stc / sh if sh > 0 else np.zeros(2)
            dt = np.zeros(3)
            if nt > adm_nt:
                dt[2] = -nt
                dt[:2] = -stc
                counts['separation'] += 1
            else:
                if st.mr_open[g] < 1.0 and nt > 0.0:
                    dt[2] = adm_nt - nt
                    counts['cohesion'] += 1
                if st.mr_slip[g] > 0 or sh > adm_st:
                    dt[:2] = adm_st * sh_dir - stc
                    counts['slip'] += 1
                elif nt <= 0.0:
                    fixed[el, 3 * lnn:3 * lnn + 3] = True
                    counts['intact'] += 1
            dt = E.r.T @ dt
            if release_sign:
                dt = -dt
            for i in range(ncomp):
                d = od[el, 3 * lnn + i]
                if d >= 0:
                    delta_trac[d] = dt[i]
    # the truncated handle: walk the element nodes in order (:212-258)
    td = vc_ref.truncate_handle(od, fixed)
    n_fixed = int(np.count_nonzero(fixed & (od >= 0)))
    mat, rhs = vc_ref.mod_3dbem_system_vc(A, od, td, delta_trac, delta_v)
    incr = np.linalg.solve(mat, rhs)
    used = mat.shape[0] - 1
    delta_p = incr[used]
    pressure += delta_p
    # DD, clamp, pressures (:314-427)
    for el in range(n_el):
        E = elems[el]
        dd_el = np.zeros((6, 3))
        for lnn in range(6):
            g = 6 * el + lnn
            dn = dd[g].copy()
            for i in range(3):
                if od[el, 3 * lnn + i] >= 0 and td[el, 3 * lnn + i] >= 0:
                    dn[i] += incr[td[el, 3 * lnn + i]]
            if not is_dd_local:
                dn = E.r @ dn
            if dn[2] < 0.0:
                dn[2] = 0.0
            dd_el[lnn] = dn
            if not is_dd_local:
                dn = E.r.T @ dn
            for i in range(3):
                if od[el, 3 * lnn + i] >= 0:
                    dd[g, i] = dn[i]
        for cpe in range(6):
            g = 6 * el + cpe
            open_cp = dd_el[:, 2] @ E.sf[cpe]
            fr = st.mr_open[g]
            op = open_cp / mats[st.mat_id[g]]['cr_open']
            if op >= 1.0 or fr >= 1.0:
                op = 1.0
            if op >= 1.0 or (op > 0.0 and fr >= 1.0):
                pp[g] = pressure
    residual = float(np.abs(incr).sum() + np.abs(delta_trac).sum())
    new = SimpleNamespace(dd=dd, pp=pp, friction_coef=fric, slip_cohesion=sc, open_cohesion=oc, dof_h=td,
                          n_dof=used)
    info = dict(residual=residual, volume=volume, pressure=pressure, delta_p=delta_p, n_fixed=n_fixed,
                counts=counts, increments=incr, delta_trac=delta_trac)
    return new, info
