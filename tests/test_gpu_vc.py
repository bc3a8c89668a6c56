"""Volume-control truncation on the device (hfpx_matrix_truncate, the gather
of mod_3dbem_system_vc, src/Solvers/system_assembly.cpp:560-629) and the
truncated system solved with the factors of the full one
(hfpx_lu_solve_fixed); the in-place preconditioner update
(hfpx_precond_update) beside them, since a contact/cohesion loop that
truncates also re-assembles.

* truncated bordered matrix of a penny crack's VC system (make_3dbem_matrix_vc,
  :458-557) against the loop restatement oracle/vc_ref.py on the downloaded
  matrix, bit for bit (a gather); rhs likewise;
* an unordered kept set without the border against a numpy index gather;
* x from the full FP64 and mixed factorisations against numpy's solve of the
  truncated system: kept entries within 1e-9 of |x|, dropped entries 0
  exactly; no dropped DoF gives the plain solve;
* bad arguments fail with the engine's error, not a fault;
* a preconditioner updated from a second matrix equals one made from it."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
G, NU, BETA = 1.0, 0.35, 0.125
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, 'oracle'))


def vc_system(ctx, n_tri=40, seed=0):
    from hfpx3d_b200 import engine, meshgen
    nods, conn = meshgen.penny(n_tri, seed=seed)
    mesh = engine.MeshGeom(nods, conn)
    dof, n = engine.make_dof_h_crack(mesh, 0)
    dm = engine.DeviceMesh(ctx, mesh, BETA)
    A = engine.assemble(ctx, dm, dof, n, G, NU, vc=True)
    return dm, dof, n, A


def test_truncate_matches_restatement(ctx):
    import vc_ref
    from hfpx3d_b200 import engine
    dm, dof, n, A = vc_system(ctx)
    Ah = A.download()
    rng = np.random.default_rng(5)
    td = vc_ref.truncate_handle(dof, rng.random(dof.shape) < 0.2)
    dv = 0.3
    for size in (n, int(td.max()) + 1):
        dt = rng.standard_normal(size)
        T, rhs = engine.mod_3dbem_system_vc(ctx, A, dof, td, dt, dv)
        M, r = vc_ref.mod_3dbem_system_vc(Ah, dof, td, dt, dv)
        assert T.n == M.shape[0]
        assert np.array_equal(T.download(), M)
        assert np.array_equal(rhs, r)
        T.close()


def test_truncate_unordered_without_border(ctx):
    from hfpx3d_b200 import engine
    dm, dof, n, A = vc_system(ctx, 24, 1)
    Ah = A.download()
    keep = np.random.default_rng(6).permutation(n)[: n // 2]
    T = engine.truncate(ctx, A, keep, keep_border=False)
    assert np.array_equal(T.download(), Ah[np.ix_(keep, keep)])
    T2 = engine.truncate(ctx, A, keep, keep_border=True)
    idx = np.append(keep, n)
    assert np.array_equal(T2.download(), Ah[np.ix_(idx, idx)])


@pytest.mark.parametrize('mode', ['fp64', 'mixed'])
def test_solve_fixed_matches_truncated_solve(ctx, mode):
    import vc_ref
    from hfpx3d_b200 import engine
    dm, dof, n, A = vc_system(ctx, 60, 2)
    Ah = A.download()
    rng = np.random.default_rng(7)
    drop = rng.random(dof.shape) < 0.15
    td = vc_ref.truncate_handle(dof, drop)
    keep = engine.vc_truncation_map(dof, td)
    fixed = np.setdiff1d(np.arange(n), keep)
    b = rng.standard_normal(n + 1)
    idx = np.append(keep, n)
    want = np.linalg.solve(Ah[np.ix_(idx, idx)], b[idx])
    lu = engine.LU(ctx, A, engine.HFPX_LU_MIXED if mode == 'mixed' else engine.HFPX_LU_FP64)
    x = lu.solve_fixed(b, fixed, tol=1e-13)
    assert np.all(x[fixed] == 0.0)
    assert np.abs(x[idx] - want).max() <= 1e-9 * np.abs(want).max()
    # nothing dropped: the plain solve
    x0 = lu.solve_fixed(b, [], tol=1e-13)
    assert np.abs(x0 - np.linalg.solve(Ah, b)).max() <= 1e-9 * np.abs(x0).max()


def test_bad_arguments(ctx):
    from hfpx3d_b200 import engine
    dm, dof, n, A = vc_system(ctx, 24, 3)
    with pytest.raises(engine.EngineError):
        engine.truncate(ctx, A, [0, 5, 5])           # repeated
    with pytest.raises(engine.EngineError):
        engine.truncate(ctx, A, [0, n])               # the border is not a DD unknown
    lu = engine.LU(ctx, A, engine.HFPX_LU_FP64)
    with pytest.raises(engine.EngineError):
        lu.solve_fixed(np.ones(n + 1), [3, 3])
    with pytest.raises(engine.EngineError):
        lu.solve_fixed(np.ones(n + 1), [n + 1])
    with pytest.raises(engine.EngineError):
        engine.truncate(ctx, A, [0, 1])               # holds FP64 factors now


def test_precond_update_equals_fresh(ctx):
    from hfpx3d_b200 import engine, meshgen
    nods, conn = meshgen.wavy(120, aspect=1.5, amp=0.1, seed=4)
    mesh = engine.MeshGeom(nods, conn)
    dof, n = engine.make_dof_h_crack(mesh, 0)
    dm = engine.DeviceMesh(ctx, mesh, BETA)
    A1 = engine.assemble(ctx, dm, dof, n, G, NU)
    A2 = engine.assemble(ctx, dm, dof, n, 2.0 * G, 0.2)
    net = engine.Gnn(ctx, path=engine.WEIGHTS_PATH)
    for kind in (engine.HFPX_PC_NEUMANN, engine.HFPX_PC_LOCAL_INVERSE, engine.HFPX_PC_LEARNED):
        kw = dict(net=net, shear_m=2.0 * G) if kind == engine.HFPX_PC_LEARNED else {}
        pc = engine.Precond(ctx, dm, A1, kind, **({'net': net} if kind == engine.HFPX_PC_LEARNED else {}))
        pc.update(A2, **kw)
        fresh = engine.Precond(ctx, dm, A2, kind, **kw)
        assert np.array_equal(pc.blocks()[2], fresh.blocks()[2])
        pc.close()
        fresh.close()
    # a matrix of another mesh is refused
    other = engine.MeshGeom(*meshgen.wavy(60, seed=1))
    dof_o, n_o = engine.make_dof_h_crack(other, 0)
    A3 = engine.assemble(ctx, engine.DeviceMesh(ctx, other, BETA), dof_o, n_o, G, NU)
    pc = engine.Precond(ctx, dm, A1, engine.HFPX_PC_NEUMANN)
    with pytest.raises(engine.EngineError):
        pc.update(A3)
