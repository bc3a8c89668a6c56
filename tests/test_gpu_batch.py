"""Many load cases at once (the batched workload: seeded penny/ellipse meshes
of 24-550 elements, each with many load cases) and the VC ellipse with a
random in-situ stress (the C2 loading): right-hand sides for all cases in one
call, one factorisation, all cases solved together, stresses of all cases
from one influence matrix and one GEMM; checked against the oracle (pinned to
the reference by the golden fixtures) and LAPACK."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
G, NU, BETA = 1.0, 0.35, 0.125


def haar_sinf(rng, n):
    """n in-situ stresses Q diag(lam) Q^T, lam ~ U[-1, 0], Q Haar (seeded), as
    Voigt [xx, yy, zz, xy, xz, yz] columns."""
    out = np.empty((6, n))
    for k in range(n):
        q, r = np.linalg.qr(rng.standard_normal((3, 3)))
        q = q * np.sign(np.diag(r))
        s = q @ np.diag(rng.uniform(-1.0, 0.0, 3)) @ q.T
        out[:, k] = [s[0, 0], s[1, 1], s[2, 2], s[0, 1], s[0, 2], s[1, 2]]
    return out


def load_cases(rng, n):
    """Uniform pressures U[0.5, 2] (s_zz) and random stresses, alternating."""
    S = haar_sinf(rng, n)
    for k in range(0, n, 2):
        S[:, k] = [0, 0, rng.uniform(0.5, 2.0), 0, 0, 0]
    return S


@pytest.mark.parametrize('kind,n_el,seed', [('penny', 24, 1), ('ellipse', 124, 2), ('penny', 550, 3)])
def test_many_load_cases(ctx, ora, kind, n_el, seed):
    from hfpx3d_b200 import engine, meshgen
    rng = np.random.default_rng(seed)
    nods, conn = (meshgen.penny if kind == 'penny' else meshgen.ellipse)(n_el, seed=seed)
    mesh = engine.MeshGeom(nods, conn)
    dof, n = engine.make_dof_h_crack(mesh, 0)
    dm = engine.DeviceMesh(ctx, mesh, BETA)
    nc = 16
    S = load_cases(rng, nc)
    R = engine.add_s_inf_to_3dbem_rhs(ctx, dm, dof, n, S)
    for k in (0, 1, nc - 1):
        assert np.abs(R[:, k] - ora.rhs(nods, conn, dof, n, S[:, k])).max() <= 1e-14 * max(1.0, np.abs(R[:, k]).max())
    A = engine.assemble(ctx, dm, dof, n, G, NU)
    Ah = A.download()
    X_ref = np.linalg.solve(Ah, R)
    for mode, tol in ((engine.HFPX_LU_MIXED, 1e-10), (engine.HFPX_LU_FP64, 1e-12)):
        M = engine.DeviceMatrix.upload(ctx, Ah)
        X = engine.LU(ctx, M, mode).solve(R, tol=1e-12)
        assert np.abs(X - X_ref).max() <= tol * np.abs(X_ref).max()
    dd = np.stack([engine.write_dd_vector_to_md(X_ref[:, k], dof, mesh.n_el) for k in range(nc)])
    pts = meshgen.observation_points(40, seed, nods=nods, conn=conn, box=2.2 if kind == 'ellipse' else 1.5)
    St = engine.make_3dbem_stress_f_s_batch(ctx, dm, G, NU, dd, pts, S)
    for k in range(nc):
        one = engine.make_3dbem_stress_f_s(ctx, dm, G, NU, dd[k], pts, S[:, k])
        assert np.abs(St[k] - one).max() <= 1e-11 * max(1.0, np.abs(one).max())
    for k in (0, nc - 1):
        o = ora.stress(nods, conn, dd[k], pts, S[:, k])
        assert np.abs(St[k] - o).max() <= 1e-10 * max(1.0, np.abs(o).max())


def test_vc_ellipse_random_stress(ctx, ora):
    # the C2 loading on a smaller 2:1 ellipse: bordered system with injected
    # volume V = 1 and a Haar-rotated in-situ stress; both LU modes against
    # LAPACK on the device-assembled matrix, which matches the oracle
    from hfpx3d_b200 import engine, meshgen
    rng = np.random.default_rng(11)
    nods, conn = meshgen.ellipse(240, seed=11)
    mesh = engine.MeshGeom(nods, conn)
    dof, n = engine.make_dof_h_crack(mesh, 0)
    dm = engine.DeviceMesh(ctx, mesh, BETA)
    s = haar_sinf(rng, 1)[:, 0]
    rhs = np.concatenate([engine.add_s_inf_to_3dbem_rhs(ctx, dm, dof, n, s), [1.0]])
    A = engine.assemble(ctx, dm, dof, n, G, NU, vc=True)
    Ah = A.download()
    Ao = ora.assemble(nods, conn, dof, n, vc=1)
    # a few far-field pairs of this mesh put the collocation point ~0.003 off
    # the line of one of the source element's edges at ~2.2 from the element:
    # the closed form cancels there, and both the reference (the oracle follows
    # it to 1e-11) and this engine miss a direct-quadrature value by up to
    # 7e-5 of those small entries, in different directions.  At the matrix
    # scale that is 4.3e-11, hence 1e-10 here.
    assert np.abs(Ah - Ao).max() <= 1e-10 * np.abs(Ao).max()
    x_ref = np.linalg.solve(Ah, rhs)
    for mode, tol in ((engine.HFPX_LU_MIXED, 1e-9), (engine.HFPX_LU_FP64, 1e-12)):
        M = engine.DeviceMatrix.upload(ctx, Ah)
        x = engine.LU(ctx, M, mode).solve(rhs, tol=1e-12)
        assert np.abs(x - x_ref).max() <= tol * np.abs(x_ref).max()
    # the volume row holds the injected volume
    assert abs(Ah[n, :n] @ x_ref[:n] - 1.0) < 1e-10
