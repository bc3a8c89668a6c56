"""Reference-pinned fixtures for the two large configurations (run in the
container that has the reference tree; commits only the .npz outputs and this
script):

    HFPX_REFERENCE=<reference tree> make -C oracle ref
    HFPX_REFERENCE=<reference tree> python tests/golden/make_configs.py

ref_c2.npz -- the volume-control 2:1 ellipse of 1025 triangles (18 450 DoF
  + 1 pressure unknown): the reference's make_3dbem_matrix_vc
  (src/Solvers/system_assembly.cpp:458-557, the never-written corner set to
  0) summarised by A w and w^T A for a seeded weight vector w, its volume row,
  seeded entry samples and its diagonal; the right-hand side of a seeded
  Haar-rotated in-situ stress with injected volume 1
  (add_s_inf_to_3dbem_rhs, :222-274, plus V); and the LAPACK solution of the
  reference's own bordered matrix (dgesv, the algorithm il::LU calls at
  il/linear_algebra/dense/factorization/LU.h:87, 115).

ref_c3.npz -- the 4000-triangle penny (72 000 DoF) the headline step runs
  on.  Its 41.5 GB matrix is not formed here: every entry depends only on its
  (target element, source element) pair (system_assembly.cpp:63-215), so the
  reference assembles sub-meshes made of a seeded sample T of elements plus a
  chunk of the others, and the blocks (t, s) and (s, t), t in T, are the
  full-mesh matrix's rows and columns of T exactly.  Stored: those rows and
  columns summarised by seeded weight vectors (rows A[T,:] W, columns
  W^T A[:,T]), the full 18 x 18 blocks of each sampled element with itself
  and its nearest neighbours, and seeded entry samples.

Both meshes come from hfpx3d_b200.meshgen with fixed seeds; a checksum of the
mesh arrays is stored so that the tests notice a changed generator.
"""
import ctypes
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))
from oracle_lib import _REF_SIG, _bind, dp, lp  # noqa: E402
from hfpx3d_b200 import meshgen  # noqa: E402

G, NU, BETA = 1.0, 0.35, 0.125
# the OpenMP build of the reference (same arithmetic per entry; parallel over
# source elements only)
REF_OMP = os.path.join(ROOT, 'oracle', '_ref', 'libhfpx_ref_omp.so')

C2_SEED, C2_NEL = 1025, 1025
C3_SEED, C3_NEL = 2026, 4000          # the bench's workload: meshgen.penny(4000, seed=2026)
C3_SAMPLE = 11                        # sampled elements: 198 rows and 198 columns
C3_NEAR = 6                           # full blocks with the 6 nearest source elements (self included)


def mesh_digest(nods, conn):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(nods, dtype=np.float64).tobytes())
    h.update(np.ascontiguousarray(conn, dtype=np.int64).tobytes())
    return h.hexdigest()


def weights(seed, n, k):
    """The seeded weight vectors the summaries use (n x k, uniform in [-1, 1])."""
    return np.random.default_rng(int(seed)).uniform(-1.0, 1.0, (n, k))


def haar_sinf(rng):
    """Q diag(lam) Q^T, lam ~ U[-1, 0], Q Haar, as Voigt [xx, yy, zz, xy, xz, yz]."""
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))
    s = q @ np.diag(rng.uniform(-1.0, 0.0, 3)) @ q.T
    return np.array([s[0, 0], s[1, 1], s[2, 2], s[0, 1], s[0, 2], s[1, 2]])


class Ref:
    def __init__(self):
        if not os.path.exists(REF_OMP):
            sys.exit('build the reference first: make -C oracle ref')
        self.L = _bind(REF_OMP, _REF_SIG)

    def dof(self, nods, conn, tip=0):
        ne = conn.shape[1]
        d = np.zeros((ne, 18), dtype=np.int64, order='F')
        n = self.L.ref_dof_handle(dp(nods), nods.shape[0], nods.shape[1], lp(conn), conn.shape[0], ne, tip, lp(d))
        return d, int(n)

    def assemble(self, nods, conn, vc=0):
        nods, conn = np.asfortranarray(nods), np.asfortranarray(conn, dtype=np.int64)
        ne = conn.shape[1]
        d, n = self.dof(nods, conn)
        m = n + (1 if vc else 0)
        A = np.zeros((m, m), order='F')
        dd = np.zeros((ne, 18), dtype=np.int64, order='F')
        nd = ctypes.c_int64()
        self.L.ref_assemble(dp(nods), nods.shape[0], nods.shape[1], lp(conn), conn.shape[0], ne, G, NU, BETA, 0, 0,
                            vc, dp(A), lp(dd), ctypes.byref(nd))
        return A, d, n

    def rhs(self, nods, conn, s_inf):
        ne = conn.shape[1]
        _, n = self.dof(nods, conn)
        r = np.zeros(n)
        self.L.ref_rhs(dp(nods), nods.shape[0], nods.shape[1], lp(conn), conn.shape[0], ne, 0,
                       dp(np.ascontiguousarray(s_inf, dtype=np.float64)), dp(r))
        return r


def make_c2(R):
    nods, conn = meshgen.ellipse(C2_NEL, seed=C2_SEED)
    rng = np.random.default_rng(C2_SEED)
    s_inf = haar_sinf(rng)
    t = time.time()
    A, dof, n = R.assemble(nods, conn, vc=1)
    print(f'C2 reference VC assembly: {A.shape[0]} unknowns, {time.time() - t:.1f} s')
    assert np.array_equal(dof, 18 * np.arange(C2_NEL)[:, None] + np.arange(18))    # tip_type 0: no fixed DoF
    rhs = np.concatenate([R.rhs(nods, conn, s_inf), [1.0]])
    w = weights(C2_SEED + 1, A.shape[0], 1)[:, 0]
    ii = rng.integers(0, A.shape[0], 4000)
    jj = rng.integers(0, A.shape[0], 4000)
    t = time.time()
    x = np.linalg.solve(A, rhs)
    print(f'C2 LAPACK solve: {time.time() - t:.1f} s, residual '
          f'{np.abs(A @ x - rhs).max() / np.abs(rhs).max():.2e}')
    return dict(mesh_digest=mesh_digest(nods, conn), n_dof=n, s_inf=s_inf, rhs=rhs, w_seed=C2_SEED + 1,
                Aw=A @ w, wA=w @ A, abs_Aw=np.abs(A) @ np.abs(w), vc_row=A[n, :].copy(), vc_col=A[:, n].copy(),
                diag=np.diag(A).copy(), sample_i=ii, sample_j=jj, sample_v=A[ii, jj], x=x)


def submesh(nods, conn, elems):
    sub = conn[:, elems]
    uniq, inv = np.unique(sub[:3], return_inverse=True)
    c = np.asfortranarray(sub.copy())
    c[:3] = inv.reshape(3, -1)
    return np.asfortranarray(nods[:, uniq]), c


def make_c3(R):
    nods, conn = meshgen.penny(C3_NEL, seed=C3_SEED)
    ne = conn.shape[1]
    n = 18 * ne
    rng = np.random.default_rng(C3_SEED)
    cent = nods[:3, conn[:3]].mean(axis=1)            # 3 x ne centroids
    rad = np.hypot(cent[0], cent[1])
    # the sample: the element nearest the centre, the outermost element (a
    # tip element), and seeded others
    T = [int(np.argmin(rad)), int(np.argmax(rad))]
    while len(T) < C3_SAMPLE:
        e = int(rng.integers(0, ne))
        if e not in T:
            T.append(e)
    T = np.array(T)
    rows = (18 * T[:, None] + np.arange(18)).reshape(-1)     # tip_type 0: dof(e, k) = 18 e + k
    Arow = np.zeros((len(rows), n))                    # A[rows, :]
    Acol = np.zeros((n, len(rows)))                    # A[:, rows]
    others = np.setdiff1d(np.arange(ne), T)
    chunk = 189
    t = time.time()
    for c0 in range(0, len(others) + 1, chunk):
        S = others[c0:c0 + chunk]
        elems = np.concatenate([T, S])
        sn, sc = submesh(nods, conn, elems)
        A, dof, nsub = R.assemble(sn, sc)
        assert nsub == 18 * len(elems)
        assert np.array_equal(dof, 18 * np.arange(len(elems))[:, None] + np.arange(18))
        # sub-mesh element p <-> mesh element elems[p]; sub dof 18 p + k
        sub_rows = np.arange(18 * len(T))
        gcols = (18 * elems[:, None] + np.arange(18)).reshape(-1)
        Arow[:, gcols] = A[sub_rows, :]
        Acol[gcols, :] = A[:, sub_rows]
    print(f'C3 reference rows/columns of {len(T)} elements by sub-meshes: {time.time() - t:.1f} s')
    W = weights(C3_SEED + 1, n, 3)
    near = np.argsort(((cent[:, :, None] - cent[:, None, T]) ** 2).sum(axis=0), axis=0)[:C3_NEAR].T   # len(T) x 6
    blocks = np.stack([np.stack([Arow[18 * i:18 * i + 18, 18 * s:18 * s + 18] for s in near[i]])
                       for i in range(len(T))])
    ri = rng.integers(0, len(rows), 3000)
    rj = rng.integers(0, n, 3000)
    ci = rng.integers(0, n, 3000)
    cj = rng.integers(0, len(rows), 3000)
    return dict(mesh_digest=mesh_digest(nods, conn), n_dof=n, elems=T, rows=rows,
                row_w=Arow @ W, row_abs=np.abs(Arow) @ np.abs(W), col_w=W.T @ Acol, col_abs=np.abs(W).T @ np.abs(Acol),
                near=near, near_blocks=blocks, row_si=ri, row_sj=rj, row_sv=Arow[ri, rj], col_si=ci, col_sj=cj,
                col_sv=Acol[ci, cj], w_seed=C3_SEED + 1)


def main():
    R = Ref()
    which = sys.argv[1:] or ['c2', 'c3']
    if 'c2' in which:
        np.savez_compressed(os.path.join(HERE, 'ref_c2.npz'), **make_c2(R))
    if 'c3' in which:
        np.savez_compressed(os.path.join(HERE, 'ref_c3.npz'), **make_c3(R))


if __name__ == '__main__':
    main()
