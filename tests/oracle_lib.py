"""Test infrastructure: ctypes bindings of the CPU oracle (oracle/libhfpx_oracle.so)
and of the reference build (oracle/_ref/libhfpx_ref.so, present only where the
reference sources were available to compile).  Only tests, smoke() and the
bench's CPU-baseline leg use these, as checkers."""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, 'oracle', 'libhfpx_oracle.so')
REF_SO = os.path.join(ROOT, 'oracle', '_ref', 'libhfpx_ref.so')

_D = ctypes.POINTER(ctypes.c_double)
_L = ctypes.POINTER(ctypes.c_int64)
_i64, _f64, _int = ctypes.c_int64, ctypes.c_double, ctypes.c_int

_ORACLE_SIG = {
    'ora_element_frame': (None, [_D, _D, _D, _D]),
    'ora_pt_hz': (None, [_D, _D, _D, _D, _D]),
    'ora_local_block': (None, [_f64, _f64, _f64, _f64, _f64, _D, _D, _D]),
    'ora_dof_handle': (_i64, [_D, _i64, _i64, _L, _i64, _i64, _int, _L]),
    'ora_assemble': (_int, [_D, _i64, _i64, _L, _i64, _i64, _L, _i64, _f64, _f64, _f64, _int, _int, _D, _i64]),
    'ora_assemble_rows': (_int, [_D, _i64, _i64, _L, _i64, _i64, _L, _i64, _f64, _f64, _f64, _int, _i64, _i64,
                                 _D, _i64]),
    'ora_rhs': (None, [_D, _i64, _L, _i64, _i64, _L, _D, _D]),
    'ora_stress': (None, [_D, _i64, _L, _i64, _i64, _f64, _f64, _int, _D, _D, _i64, _D, _D]),
    'ora_dd_from_solution': (None, [_D, _L, _i64, _D]),
    'ora_sneddon_dd': (None, [_f64, _f64, _f64, _f64, _D, _D]),
    'ora_sneddon_stress': (None, [_f64, _f64, _f64, _f64, _D, _D]),
}

_REF_SIG = {
    'ref_element_frame': (_int, [_D, _D, _D, _D]),
    'ref_pt_hz': (_int, [_D, _D, _D, _D, _D]),
    'ref_local_submatrix': (_int, [_f64, _f64, _f64, _f64, _f64, _D, _D, _D]),
    'ref_s_ij_lim': (_int, [_f64, _f64, _f64, _f64, _f64, _D]),
    'ref_dof_handle': (_i64, [_D, _i64, _i64, _L, _i64, _i64, _int, _L]),
    'ref_assemble': (_int, [_D, _i64, _i64, _L, _i64, _i64, _f64, _f64, _f64, _int, _int, _int, _D, _L, _L]),
    'ref_rhs': (_int, [_D, _i64, _i64, _L, _i64, _i64, _int, _D, _D]),
    'ref_stress': (_int, [_D, _i64, _i64, _L, _i64, _i64, _f64, _f64, _int, _D, _D, _i64, _D, _D]),
}


def _bind(path, sig):
    lib = ctypes.CDLL(path)
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


def dp(a):
    return a.ctypes.data_as(_D)


def lp(a):
    return a.ctypes.data_as(_L)


_oracle = None


def oracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO) or \
                os.path.getmtime(ORACLE_SO) < os.path.getmtime(os.path.join(ROOT, 'oracle', 'hfpx_oracle.c')):
            subprocess.run(['make', '-s', '-C', os.path.join(ROOT, 'oracle')], check=True)
        _oracle = _bind(ORACLE_SO, _ORACLE_SIG)
    return _oracle


def ref_available():
    return os.path.exists(REF_SO)


_ref = None


def ref():
    global _ref
    if _ref is None:
        _ref = _bind(REF_SO, _REF_SIG)
    return _ref


class Oracle:
    """Convenience wrappers (column-major numpy in, numpy out)."""

    def __init__(self):
        self.L = oracle()

    @staticmethod
    def _m(nods, conn):
        return np.asfortranarray(nods, dtype=np.float64), np.asfortranarray(conn, dtype=np.int64)

    def element_frame(self, vert3x3):
        v = np.ascontiguousarray(np.asarray(vert3x3, dtype=np.float64).T)
        r, tau, sfm = np.empty(9), np.empty(6), np.empty(72)
        self.L.ora_element_frame(dp(v), dp(r), dp(tau), dp(sfm))
        return r.reshape(3, 3), tau, sfm

    def pt_hz(self, vert3x3, pt):
        v = np.ascontiguousarray(np.asarray(vert3x3, dtype=np.float64).T)
        p = np.ascontiguousarray(pt, dtype=np.float64)
        h, zr, zi = _f64(), _f64(), _f64()
        self.L.ora_pt_hz(dp(v), dp(p), ctypes.byref(h), ctypes.byref(zr), ctypes.byref(zi))
        return h.value, complex(zr.value, zi.value)

    def local_block(self, G, nu, h, z, tau, sfm):
        out = np.empty(108)
        tau = np.ascontiguousarray(tau, dtype=np.float64)
        sfm = np.ascontiguousarray(sfm, dtype=np.float64)
        self.L.ora_local_block(G, nu, h, z.real, z.imag, dp(tau), dp(sfm), dp(out))
        return out.reshape(6, 18)

    def dof_handle(self, nods, conn, tip_type):
        nods, conn = self._m(nods, conn)
        ne = conn.shape[1]
        d = np.zeros((ne, 18), dtype=np.int64, order='F')
        n = self.L.ora_dof_handle(dp(nods), nods.shape[0], nods.shape[1], lp(conn), conn.shape[0], ne, tip_type,
                                  lp(d))
        return d, int(n)

    def assemble(self, nods, conn, dof, n_dof, G=1.0, nu=0.35, beta=0.125, is_dd_local=0, vc=0):
        nods, conn = self._m(nods, conn)
        dof = np.asfortranarray(dof, dtype=np.int64)
        n = n_dof + (1 if vc else 0)
        A = np.zeros((n, n), order='F')
        self.L.ora_assemble(dp(nods), nods.shape[0], nods.shape[1], lp(conn), conn.shape[0], conn.shape[1], lp(dof),
                            n_dof, G, nu, beta, int(is_dd_local), int(vc), dp(A), n)
        return A

    def assemble_rows(self, nods, conn, dof, n_dof, t0, t1, G=1.0, nu=0.35, beta=0.125, is_dd_local=0):
        """Rows of target elements [t0, t1) only, as a dense (rows x n_dof) block."""
        nods, conn = self._m(nods, conn)
        dof = np.asfortranarray(dof, dtype=np.int64)
        rows = dof[t0:t1].reshape(-1)
        rows = np.sort(rows[rows >= 0])
        lo, hi = rows[0], rows[-1] + 1
        buf = np.zeros((hi - lo, n_dof), order='F')
        # ora_assemble_rows writes at absolute row indices; shift the base pointer
        base = buf.ctypes.data - int(lo) * 8
        self.L.ora_assemble_rows(dp(nods), nods.shape[0], nods.shape[1], lp(conn), conn.shape[0], conn.shape[1],
                                 lp(dof), n_dof, G, nu, beta, int(is_dd_local), t0, t1,
                                 ctypes.cast(base, _D), hi - lo)
        return lo, buf

    def rhs(self, nods, conn, dof, n_dof, s_inf):
        nods, conn = self._m(nods, conn)
        dof = np.asfortranarray(dof, dtype=np.int64)
        r = np.zeros(n_dof)
        s = np.ascontiguousarray(s_inf, dtype=np.float64)
        self.L.ora_rhs(dp(nods), nods.shape[0], lp(conn), conn.shape[0], conn.shape[1], lp(dof), dp(s), dp(r))
        return r

    def stress(self, nods, conn, dd, pts, s_inf, G=1.0, nu=0.35, is_dd_local=0):
        nods, conn = self._m(nods, conn)
        dd = np.asfortranarray(dd, dtype=np.float64)
        pts = np.asfortranarray(pts, dtype=np.float64)
        s = np.ascontiguousarray(s_inf, dtype=np.float64)
        out = np.zeros((pts.shape[1], 6), order='F')
        self.L.ora_stress(dp(nods), nods.shape[0], lp(conn), conn.shape[0], conn.shape[1], G, nu, int(is_dd_local),
                          dp(dd), dp(pts), pts.shape[1], dp(s), dp(out))
        return out

    def dd_from_solution(self, sol, dof, n_el):
        dof = np.asfortranarray(dof, dtype=np.int64)
        dd = np.zeros((6 * n_el, 3), order='F')
        sol = np.ascontiguousarray(sol, dtype=np.float64)
        self.L.ora_dd_from_solution(dp(sol), lp(dof), n_el, dp(dd))
        return dd

    def sneddon_dd(self, G, nu, a, p, x):
        out = np.empty(3)
        self.L.ora_sneddon_dd(G, nu, a, p, dp(np.ascontiguousarray(x, dtype=np.float64)), dp(out))
        return out

    def sneddon_stress(self, G, nu, a, p, x):
        out = np.empty(6)
        self.L.ora_sneddon_stress(G, nu, a, p, dp(np.ascontiguousarray(x, dtype=np.float64)), dp(out))
        return out
