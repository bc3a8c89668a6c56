"""High-precision (mpmath, 40 digits) values of element-to-point stress blocks
for near-plane configurations, where the reference's closed form loses
accuracy through cancellation (observation point close to an element's plane
but far from the element).  The integrals are the exact sector integrals of
the DD -> stress kernel, evaluated by adaptive quadrature in extended
precision from the term table in hfpx3d_b200/csrc/dd_terms.h.

    python tests/golden/make_truth.py      # -> tests/golden/truth_blocks.npz
(the reference build oracle/_ref is used only to record its own values)
"""
import os
import re
import sys

import mpmath as mp
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle_lib import Oracle, dp, ref, ref_available  # noqa: E402
from conftest import golden  # noqa: E402

mp.mp.dps = 40
G, NU = 1.0, 0.35


def load_terms():
    txt = open(os.path.join(ROOT, 'hfpx3d_b200', 'csrc', 'dd_terms.h')).read()
    head, body = txt.split('hfpx_terms[HFPX_N_TERMS]')
    moms = [(int(a), int(b)) for a, b in re.findall(r'\{(-?\d+), (-?\d+)\},', head.split('hfpx_moments')[-1])]
    rows = re.findall(r'\{(\d+), (\d+), (\d+), 0, ([-\deE.+]+), ([-\deE.+]+), ([-\deE.+]+), ([-\deE.+]+)\}', body)
    return moms, [(int(j), int(m), int(q), float(a0), float(a1), float(b0), float(b1))
                  for j, m, q, a0, a1, b0, b1 in rows]


def mp_block(h, z, tau, sfm):
    moms, rows = load_terms()
    h = mp.mpf(h)
    z = mp.mpc(z.real, z.imag)
    tau = [mp.mpc(t.real, t.imag) for t in tau]
    tz = [t - z for t in tau]
    d = []
    for j in range(3):
        dt = tau[(j + 1) % 3] - tau[j]
        d.append((tz[j] - dt / mp.conj(dt) * mp.conj(tz[j])) / 2)
    phi = [mp.arg(t) for t in tz]
    W = [mp.mpc(0)] * len(moms)
    for m in range(3):
        psi = mp.arg(d[m])
        D = abs(d[m])
        chis = []
        for idx in (m, (m + 1) % 3):
            c = phi[idx] - psi
            while c <= -mp.pi:
                c += 2 * mp.pi
            while c > mp.pi:
                c -= 2 * mp.pi
            chis.append(c)
        pts = [chis[0], 0, chis[1]] if chis[0] * chis[1] < 0 else [chis[0], chis[1]]
        for i, (s, p) in enumerate(moms):
            f = lambda th: mp.exp(1j * s * (psi + th)) * mp.quad(
                lambda r: r ** p / (r * r + h * h) ** mp.mpf(3.5), [0, D / mp.cos(th)])
            W[i] += mp.quad(f, pts)
    smon = [mp.mpc(0)] * 72
    for (jck, mi, q, a0, a1, b0, b1) in rows:
        coef = mp.mpc(a0 + NU * a1, b0 + NU * b1)
        smon[jck] -= coef * h ** q * W[mi]
    zc = mp.conj(z)
    scale = -G / (4 * mp.pi * (1 - NU))
    out = np.zeros((6, 18))
    for a in range(6):
        sr = [mp.mpc(sfm[a, j].real, sfm[a, j].imag) for j in range(6)]
        sz = [sr[0] + sr[1] * z + sr[2] * zc + sr[3] * z * z + sr[4] * zc * zc + sr[5] * z * zc,
              sr[1] + 2 * sr[3] * z + sr[5] * zc, sr[2] + 2 * sr[4] * zc + sr[5] * z, sr[3], sr[4], sr[5]]
        for k in range(3):
            s = [sum(sz[j] * smon[(j * 4 + c) * 3 + k] for j in range(6)) for c in range(4)]
            q = 3 * a + k
            out[:, q] = [float(scale * (s[0].real + s[1].real)), float(scale * (s[0].real - s[1].real)),
                         float(scale * s[3].real), float(scale * s[1].imag), float(scale * 2 * s[2].real),
                         float(scale * 2 * s[2].imag)]
    return out


def cp_of(nods, conn, t, nt, beta=0.125):
    vt = nods[:3, conn[:3, t]]
    c = vt.mean(axis=1)
    if nt < 3:
        return (1 - beta) * vt[:, nt] + beta * c
    m = (nt - 3 + 1) % 3
    l = (m + 1) % 3
    return 0.5 * (1 - beta) * (vt[:, m] + vt[:, l]) + beta * c


def main():
    o = Oracle()
    cases = []
    g = golden('ref_p121')
    for e in (69, 66, 41):
        cases.append((g['nods'][:3, g['conn'][:3, e]], g['pts'][:, 76]))
    w = golden('ref_wavy48')
    cases.append((w['nods'][:3, w['conn'][:3, 7]], cp_of(w['nods'], w['conn'], 5, 3)))
    tri = np.array([[0.0, 0.1, 0.0], [1.8, 0.0, 0.0], [1.2, 1.8, 0.0]]).T
    cases.append((tri, np.array([3.5, 0.4, 2e-3])))
    out = {k: [] for k in ('vert', 'pt', 'h', 'z', 'tau', 'sfm', 'truth', 'ref')}
    for vert, pt in cases:
        r, tau, sfm = o.element_frame(vert)
        h, z = o.pt_hz(vert, pt)
        tc = tau[0::2] + 1j * tau[1::2]
        sc = (sfm[0::2] + 1j * sfm[1::2]).reshape(6, 6)
        out['vert'].append(vert)
        out['pt'].append(pt)
        out['h'].append(h)
        out['z'].append(z)
        out['tau'].append(tau)
        out['sfm'].append(sfm)
        out['truth'].append(mp_block(h, z, tc, sc))
        r2 = np.empty(108)
        if ref_available():
            ref().ref_local_submatrix(G, NU, h, z.real, z.imag, dp(np.ascontiguousarray(tau)),
                                      dp(np.ascontiguousarray(sfm)), dp(r2))
        out['ref'].append(r2.reshape(6, 18))
        print(len(out['truth']), 'done', flush=True)
    np.savez_compressed(os.path.join(HERE, 'truth_blocks.npz'), **{k: np.array(v) for k, v in out.items()})


if __name__ == '__main__':
    main()
