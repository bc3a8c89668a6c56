"""Generate the golden fixtures in tests/golden/ (run in the container that has
the reference tree; commits only the .npz outputs and this script).

    make -C oracle ref && python tests/golden/make_golden.py

Sources:
  * the reference's own golden vectors (MATLAB-generated csv of
    src/Elasticity/_test/integration_test_triangle_pt{1,2,3}.csv and
    src/Solvers/_test/assembly_test_{triangle,bitriangle,radial_crack_24el}.csv,
    read by the tests at src/Elasticity/_test/kernel_integration_test.cpp:28-296
    and src/Solvers/_test/matrix_assembly_test.cpp:25-308), with the meshes
    and points those tests use;
  * the reference's shipped meshes (Mesh_Files/*pennymesh{24,121}el_32.npy);
  * full-precision outputs of the reference itself, compiled from its sources
    by oracle/Makefile into oracle/_ref/libhfpx_ref.so: local blocks,
    DoF handles, assembled matrices (full for small meshes, row/column sums and
    seeded entry samples for larger ones), right-hand sides, stresses;
  * LAPACK dgesv (numpy) solutions of the reference's matrices, the
    third-party algorithm il::LU calls (LU.h:87, 115).
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))
from oracle_lib import dp, lp, ref  # noqa: E402
from hfpx3d_b200 import meshgen  # noqa: E402

REF = os.environ.get('HFPX_REFERENCE', '')
if not os.path.isdir(REF):
    sys.exit('set HFPX_REFERENCE to the reference tree')
G, NU, BETA = 1.0, 0.35, 0.125


def csv(rel):
    return np.loadtxt(os.path.join(REF, rel), delimiter=',')


def ref_mesh(name):
    E = np.load(os.path.join(REF, 'Mesh_Files', f'Elems_{name}_32.npy')).astype(np.int64)
    N = np.load(os.path.join(REF, 'Mesh_Files', f'Nodes_{name}_32.npy')).astype(np.float64)
    conn = np.asfortranarray(E)
    conn[:3] -= 1
    return np.asfortranarray(N), conn


def test_mesh(name):
    E = np.load(os.path.join(REF, 'src', 'Solvers', '_test', f'Elems_{name}_32.npy')).astype(np.int64)
    N = np.load(os.path.join(REF, 'src', 'Solvers', '_test', f'Nodes_{name}_32.npy')).astype(np.float64)
    conn = np.asfortranarray(E)
    conn[:3] -= 1
    return np.asfortranarray(N), conn


TRI = np.array([[0.0, 0.1, 0.0], [1.8, 0.0, 0.0], [1.2, 1.8, 0.0]]).T        # column j = vertex j
QUAD_EXTRA = np.array([2.2, 1.72, -1.21])                                   # 4th node of the bitriangle


def R():
    return ref()


def ref_frame(vert):
    v = np.ascontiguousarray(vert.T)
    r, tau, sfm = np.empty(9), np.empty(6), np.empty(72)
    R().ref_element_frame(dp(v), dp(r), dp(tau), dp(sfm))
    return r, tau, sfm


def ref_block(vert, pt):
    v = np.ascontiguousarray(vert.T)
    p = np.ascontiguousarray(pt, dtype=np.float64)
    h, zr, zi = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    R().ref_pt_hz(dp(v), dp(p), ctypes.byref(h), ctypes.byref(zr), ctypes.byref(zi))
    _, tau, sfm = ref_frame(vert)
    out = np.empty(108)
    R().ref_local_submatrix(G, NU, h, zr, zi, dp(tau), dp(sfm), dp(out))
    return h.value, zr.value, zi.value, out.reshape(6, 18)


def ref_dof(nods, conn, tip):
    ne = conn.shape[1]
    d = np.zeros((ne, 18), dtype=np.int64, order='F')
    n = R().ref_dof_handle(dp(nods), nods.shape[0], nods.shape[1], lp(conn), conn.shape[0], ne, tip, lp(d))
    return d, int(n)


def ref_assemble(nods, conn, tip=0, vc=0, local=0):
    ne = conn.shape[1]
    d, n = ref_dof(nods, conn, tip)
    m = n + (1 if vc else 0)
    A = np.zeros((m, m), order='F')
    dd = np.zeros((ne, 18), dtype=np.int64, order='F')
    nd = ctypes.c_int64()
    R().ref_assemble(dp(nods), nods.shape[0], nods.shape[1], lp(conn), conn.shape[0], ne, G, NU, BETA, tip, local,
                     vc, dp(A), lp(dd), ctypes.byref(nd))
    return A, d, n


def ref_rhs(nods, conn, tip, s_inf):
    ne = conn.shape[1]
    _, n = ref_dof(nods, conn, tip)
    r = np.zeros(n)
    s = np.ascontiguousarray(s_inf, dtype=np.float64)
    R().ref_rhs(dp(nods), nods.shape[0], nods.shape[1], lp(conn), conn.shape[0], ne, tip, dp(s), dp(r))
    return r


def ref_stress(nods, conn, dd, pts, s_inf, local=0):
    ne = conn.shape[1]
    out = np.zeros((pts.shape[1], 6), order='F')
    s = np.ascontiguousarray(s_inf, dtype=np.float64)
    R().ref_stress(dp(nods), nods.shape[0], nods.shape[1], lp(conn), conn.shape[0], ne, G, NU, local,
                   dp(np.asfortranarray(dd)), dp(np.asfortranarray(pts)), pts.shape[1], dp(s), dp(out))
    return out


def dd_from_solution(x, dof, ne):
    dd = np.zeros((6 * ne, 3), order='F')
    for j in range(18):
        g = dof[:, j]
        ok = g >= 0
        dd[(6 * np.arange(ne) + j // 3)[ok], j % 3] = x[g[ok]]
    return dd


def summarize(A, seed, n_sample=20000):
    rng = np.random.default_rng(seed)
    n = A.shape[0]
    ii = rng.integers(0, n, n_sample)
    jj = rng.integers(0, n, n_sample)
    return dict(row_sum=A.sum(axis=1), col_sum=A.sum(axis=0), abs_col_sum=np.abs(A).sum(axis=0),
                sample_i=ii, sample_j=jj, sample_v=A[ii, jj], diag=np.diag(A).copy())


def case(nods, conn, tip, s_inf, pts, seed, full=False, vc=False):
    A, dof, n = ref_assemble(nods, conn, tip)
    rhs = ref_rhs(nods, conn, tip, s_inf)
    x = np.linalg.solve(A, rhs)
    ne = conn.shape[1]
    dd = dd_from_solution(x, dof, ne)
    st = ref_stress(nods, conn, dd, pts, s_inf)
    out = dict(nods=nods, conn=conn, tip=tip, s_inf=np.asarray(s_inf, dtype=np.float64), dof=dof, n_dof=n, rhs=rhs,
               x=x, dd=dd, pts=pts, stress=st)
    if full:
        out['A'] = A
    else:
        out.update({'A_' + k: v for k, v in summarize(A, seed).items()})
    if vc:
        Av, _, _ = ref_assemble(nods, conn, tip, vc=1)
        out['vc_row'] = Av[n, :].copy()
        out['vc_col'] = Av[:, n].copy()
    return out


def main():
    os.makedirs(HERE, exist_ok=True)
    # 1. the reference's MATLAB goldens, with the inputs of its tests
    np.savez_compressed(os.path.join(HERE, 'matlab_kernel.npz'), vert=TRI,
                        pts=np.array([[1.0, 1.0, 0.0], [1.2, 1.8, -1.21], [1.0, 1.0, -1.21]]),
                        pt1=csv('src/Elasticity/_test/integration_test_triangle_pt1.csv'),
                        pt2=csv('src/Elasticity/_test/integration_test_triangle_pt2.csv'),
                        pt3=csv('src/Elasticity/_test/integration_test_triangle_pt3.csv'))
    n24, c24 = test_mesh('pennymesh24el')
    bit_nods = np.asfortranarray(np.column_stack([TRI, QUAD_EXTRA]))
    bit_conn = np.asfortranarray(np.array([[0, 1, 2], [1, 2, 3]]).T.astype(np.int64))
    np.savez_compressed(os.path.join(HERE, 'matlab_assembly.npz'),
                        tri_nods=np.asfortranarray(TRI), tri_conn=np.asfortranarray(np.array([[0], [1], [2]], np.int64)),
                        bit_nods=bit_nods, bit_conn=bit_conn, p24_nods=n24, p24_conn=c24,
                        triangle=csv('src/Solvers/_test/assembly_test_triangle.csv'),
                        bitriangle=csv('src/Solvers/_test/assembly_test_bitriangle.csv'),
                        radial24=csv('src/Solvers/_test/assembly_test_radial_crack_24el.csv'))
    # 2. reference local blocks at seeded points around the test triangle
    rng = np.random.default_rng(7)
    pts = [[1.0, 1.0, 0.0], [1.2, 1.8, 0.0], [1.8, 0.0, 0.0], [0.9, 0.05, 0.0], [3.0, 3.0, 0.0],
           [2.4, -1.8, 0.0], [1.2, 1.8, -1.21], [1.0, 1.0, -1.21], [0.5, 0.2, 0.01], [1.0, 1.0, 1e-3],
           [1.5, 0.5, -0.05], [3.0, 2.0, 1.0], [0.6, 1.2, 0.4]]
    pts += [list(rng.uniform(-1, 3, 2)) + [0.0] for _ in range(25)]
    pts += [list(rng.uniform(-1, 3, 3)) for _ in range(25)]
    pts = np.array(pts)
    blocks = [ref_block(TRI, p) for p in pts]
    r, tau, sfm = ref_frame(TRI)
    np.savez_compressed(os.path.join(HERE, 'ref_kernel_points.npz'), vert=TRI, pts=pts,
                        h=np.array([b[0] for b in blocks]), z=np.array([b[1] + 1j * b[2] for b in blocks]),
                        out=np.array([b[3] for b in blocks]), r=r.reshape(3, 3), tau=tau, sfm=sfm)
    # 3. reference meshes and their DoF handles
    n121, c121 = ref_mesh('pennymesh121el')
    dofs = {}
    for name, (nn, cc) in (('p24', (n24, c24)), ('p121', (n121, c121))):
        for tip in (0, 1, 2):
            d, n = ref_dof(nn, cc, tip)
            dofs[f'{name}_tip{tip}'] = d
            dofs[f'{name}_tip{tip}_n'] = np.array(n)
    np.savez_compressed(os.path.join(HERE, 'ref_dof.npz'), p24_nods=n24, p24_conn=c24, p121_nods=n121,
                        p121_conn=c121, **dofs)
    # 4. full cases: 24 el (full matrices), bitriangle (non-planar), 121 el, seeded C1 penny
    s_zz = [0.0, 0.0, 1.0, 0.0, 0.0, 0.0]
    pts24 = meshgen.observation_points(20, seed=11, nods=n24, conn=c24)
    np.savez_compressed(os.path.join(HERE, 'ref_p24.npz'), **case(n24, c24, 0, s_zz, pts24, 1, full=True, vc=True))
    A1, d1, nd1 = ref_assemble(n24, c24, tip=1)
    np.savez_compressed(os.path.join(HERE, 'ref_p24_tip1.npz'), A=A1, dof=d1, n_dof=nd1,
                        rhs=ref_rhs(n24, c24, 1, s_zz))
    s_gen = [0.3, -0.2, 1.0, 0.1, -0.15, 0.05]
    ptsb = meshgen.observation_points(12, seed=12, box=2.5, nods=bit_nods, conn=bit_conn, r_tol=0.05)
    np.savez_compressed(os.path.join(HERE, 'ref_bitriangle.npz'),
                        **case(bit_nods, bit_conn, 0, s_gen, ptsb, 2, full=True, vc=True))
    pts121 = meshgen.observation_points(100, seed=13, nods=n121, conn=c121)
    np.savez_compressed(os.path.join(HERE, 'ref_p121.npz'), **case(n121, c121, 0, s_zz, pts121, 3, vc=True))
    nc1, cc1 = meshgen.penny(121, seed=2024)
    ptsc1 = meshgen.observation_points(100, seed=2025, nods=nc1, conn=cc1)
    np.savez_compressed(os.path.join(HERE, 'ref_c1.npz'), **case(nc1, cc1, 0, s_zz, ptsc1, 4, vc=True))
    # non-planar seeded wavy crack (general path everywhere)
    nw, cw = meshgen.wavy(48, aspect=1.5, amp=0.15, k=2.0, seed=5)
    ptsw = meshgen.observation_points(20, seed=14, nods=nw, conn=cw)
    np.savez_compressed(os.path.join(HERE, 'ref_wavy48.npz'),
                        **case(nw, cw, 0, s_gen, ptsw, 5, full=False, vc=True))
    for f in sorted(os.listdir(HERE)):
        if f.endswith('.npz'):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == '__main__':
    main()
