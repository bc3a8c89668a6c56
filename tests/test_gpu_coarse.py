"""The coarse level of the two-level preconditioner (HFPX_PC_COARSE): no
counterpart in the reference, which solves directly (il::LU,
il/linear_algebra/dense/factorization/LU.h:79-120); the operator is
make_3dbem_matrix_s's (src/Solvers/system_assembly.cpp:30-219).

* aggregates cover every element once, of about the requested size;
* A P from the FP64 matrix against numpy's A @ P (1e-12 of |A| |P|), and from
  the FP32 copy against the FP32-rounded matrix times P;
* the coarse inverse times numpy's P^T A P is the identity (1e-8);
* GMRES with the two-level forms reaches the LU solution in fewer steps than
  the near-field forms alone, on an unseen 900-element crack;
* an update in place equals a fresh two-level preconditioner."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
G, NU, BETA = 1.0, 0.35, 0.125


def setup(ctx, n_tri, seed, **kw):
    from hfpx3d_b200 import engine, meshgen
    nods, conn = meshgen.wavy(n_tri, seed=seed, **kw)
    mesh = engine.MeshGeom(nods, conn)
    dof, n = engine.make_dof_h_crack(mesh, 0)
    dm = engine.DeviceMesh(ctx, mesh, BETA)
    A = engine.assemble(ctx, dm, dof, n, G, NU)
    rhs = engine.add_s_inf_to_3dbem_rhs(ctx, dm, dof, n, [0, 0, 1.0, 0, 0, 0])
    return dm, dof, n, A, rhs


def dense_P(agg, w):
    ne = agg.size
    na = int(agg.max()) + 1
    P = np.zeros((18 * ne, 9 * na))
    for e in range(ne):
        for node in range(6):
            for k in range(3):
                for m in range(3):
                    P[18 * e + 3 * node + k, 9 * agg[e] + 3 * m + k] = w[e, node, m]
    return P


def test_coarse_quantities_match_numpy(ctx, monkeypatch):
    from hfpx3d_b200 import engine
    monkeypatch.setenv('HFPX_PC_AGG', '12')
    dm, dof, n, A, rhs = setup(ctx, 300, 11, aspect=1.5, amp=0.15)
    Ah = A.download()
    pc = engine.Precond(ctx, dm, A, engine.HFPX_PC_NEUMANN | engine.HFPX_PC_COARSE)
    agg, w, AP, inv = pc.coarse(with_ap=True)
    ne = agg.size
    sizes = np.bincount(agg)
    assert sizes.sum() == ne and sizes.min() >= 1 and 6 <= sizes.mean() <= 24
    assert np.all(w[:, :, 0] == 1.0) and np.abs(w[:, :, 1:]).max() <= 1.0 + 1e-12
    P = dense_P(agg, w)
    scale = np.abs(Ah) @ np.abs(P)
    assert np.abs(AP - Ah @ P).max() <= 1e-12 * scale.max()
    Ac = P.T @ Ah @ P
    assert np.abs(inv @ Ac - np.eye(Ac.shape[0])).max() <= 1e-8
    # the FP32 copy (written by a re-assembly once the matrix holds one)
    engine.gmres(ctx, A, rhs, pc, tol=1e-10)               # makes the copy
    engine.assemble_into(ctx, dm, dof, n, G, NU, A)          # writes FP64 and FP32
    pc.update(A)
    _, _, AP32, _ = pc.coarse(with_ap=True)
    A32 = Ah.astype(np.float32).astype(np.float64)
    assert np.abs(AP32 - A32 @ P).max() <= 1e-12 * scale.max()
    assert np.abs(AP32 - Ah @ P).max() <= 1e-6 * scale.max()


def test_two_level_gmres_fewer_steps(ctx):
    from hfpx3d_b200 import engine
    dm, dof, n, A, rhs = setup(ctx, 900, 900123, aspect=2.0, amp=0.12)
    x_ref = engine.LU(ctx, engine.DeviceMatrix.upload(ctx, A.download())).solve(rhs)
    net = engine.Gnn(ctx, path=engine.WEIGHTS_PATH)
    steps = {}
    for name, kind in (('neumann', engine.HFPX_PC_NEUMANN), ('learned', engine.HFPX_PC_LEARNED)):
        for two in (False, True):
            k = kind | (engine.HFPX_PC_COARSE if two else 0)
            pc = engine.Precond(ctx, dm, A, k, net=net if kind == engine.HFPX_PC_LEARNED else None, shear_m=G)
            x, info = engine.gmres(ctx, A, rhs, pc, tol=1e-10)
            assert info.converged, (name, two)
            assert np.abs(x - x_ref).max() <= 1e-8 * np.abs(x_ref).max(), (name, two)
            steps[(name, two)] = info.iterations
            pc.close()
    print('GMRES(50) steps', steps)
    assert steps[('neumann', True)] < 0.8 * steps[('neumann', False)]
    assert steps[('learned', True)] < 0.8 * steps[('learned', False)]
    assert steps[('learned', True)] <= steps[('neumann', True)]


def test_two_level_update_equals_fresh(ctx):
    from hfpx3d_b200 import engine
    dm, dof, n, A1, rhs = setup(ctx, 200, 5)
    A2 = engine.assemble(ctx, dm, dof, n, 2.0 * G, 0.2)
    for kind in (engine.HFPX_PC_NEUMANN, engine.HFPX_PC_LOCAL_INVERSE):
        k = kind | engine.HFPX_PC_COARSE
        pc = engine.Precond(ctx, dm, A1, k)
        pc.update(A2)
        fresh = engine.Precond(ctx, dm, A2, k)
        a1, w1, ap1, inv1 = pc.coarse(with_ap=True)
        a2, w2, ap2, inv2 = fresh.coarse(with_ap=True)
        assert np.array_equal(a1, a2) and np.array_equal(w1, w2)
        assert np.array_equal(ap1, ap2) and np.array_equal(inv1, inv2)
        assert np.array_equal(pc.blocks()[2], fresh.blocks()[2])
        x1, _ = engine.gmres(ctx, A2, rhs, pc, tol=1e-10)
        x2, _ = engine.gmres(ctx, A2, rhs, fresh, tol=1e-10)
        assert np.array_equal(x1, x2)
        pc.close()
        fresh.close()
