"""Dense LU (il::LU / LAPACK dgetrf+dgetrs semantics) on the GPU: FP64 and mixed
(FP32 factorisation whose trailing updates run in FP16 with FP32 accumulation
on the engine's own tcgen05 kernel, L21 and U12 scaled by powers of two, plus
FP64 refinement), against LAPACK (numpy)."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def test_fp64_solution_matches_lapack(ctx):
    from hfpx3d_b200 import engine
    g = golden('ref_p24')
    m = engine.DeviceMatrix.upload(ctx, g['A'])
    lu = engine.LU(ctx, m, engine.HFPX_LU_FP64)
    x = lu.solve(g['rhs'])
    assert np.abs(x - g['x']).max() / np.abs(g['x']).max() < 1e-12


@pytest.mark.parametrize('n', [300, 1000, 2500])
def test_fp64_random_and_factors(ctx, n):
    from hfpx3d_b200 import engine
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n)) + n ** 0.5 * np.eye(n)
    B = rng.standard_normal((n, 3))
    m = engine.DeviceMatrix.upload(ctx, A)
    lu = engine.LU(ctx, m)
    X = lu.solve(B)
    assert np.abs(A @ X - B).max() < 1e-10 * np.abs(B).max()
    # factors reproduce A under the row permutation LAPACK-style
    F = m.download()
    L = np.tril(F, -1) + np.eye(n)
    U = np.triu(F)
    PA = L @ U
    assert np.abs(np.sort(PA, axis=None) - np.sort(A, axis=None)).max() < 1e-9 * np.abs(A).max()


def test_mixed_refinement_reaches_fp64(ctx):
    from hfpx3d_b200 import engine
    g = golden('ref_c1')
    from hfpx3d_b200 import meshgen  # noqa: F401
    mesh = engine.MeshGeom(g['nods'], g['conn'])
    dof, n = engine.make_dof_h_crack(mesh, 0)
    dm = engine.DeviceMesh(ctx, mesh)
    A = engine.assemble(ctx, dm, dof, n, 1.0, 0.35)
    lu = engine.LU(ctx, A, engine.HFPX_LU_MIXED)
    x = lu.solve(g['rhs'], tol=1e-12, max_iter=30)
    assert lu.last_info.converged and lu.last_info.residual <= 1e-12
    assert np.abs(x - g['x']).max() / np.abs(g['x']).max() < 1e-9


def test_vc_bordered_system(ctx, ora):
    from hfpx3d_b200 import engine
    g = golden('ref_c1')
    mesh = engine.MeshGeom(g['nods'], g['conn'])
    dof, n = engine.make_dof_h_crack(mesh, 0)
    dm = engine.DeviceMesh(ctx, mesh)
    A = engine.assemble(ctx, dm, dof, n, 1.0, 0.35, vc=True)
    Ah = A.download()
    rhs = np.concatenate([g['rhs'], [1.0]])
    x_ref = np.linalg.solve(Ah, rhs)
    for mode in (engine.HFPX_LU_FP64, engine.HFPX_LU_MIXED):
        A2 = engine.DeviceMatrix.upload(ctx, Ah)
        x = engine.LU(ctx, A2, mode).solve(rhs, tol=1e-12)
        assert np.abs(x - x_ref).max() / np.abs(x_ref).max() < 1e-9


def test_singular_matrix_reports_column(ctx):
    from hfpx3d_b200 import engine
    A = np.eye(50)
    A[:, 17] = 0.0
    m = engine.DeviceMatrix.upload(ctx, A)
    with pytest.raises(engine.EngineError) as e:
        engine.LU(ctx, m)
    assert e.value.code == engine.HFPX_ERR_SINGULAR
    b = np.ones(50)
    with pytest.raises(engine.EngineError):
        engine.lib()  # library still usable
        engine.LU.solve(type('X', (), {'ctx': ctx, 'matrix': m})(), b)


def test_solve_before_factor_is_refused(ctx):
    from hfpx3d_b200 import engine
    m = engine.DeviceMatrix.upload(ctx, np.eye(10))
    b = np.ones((10, 1), order='F')
    rc = engine.lib().hfpx_lu_solve(ctx.h, m.h, engine._dp(b), 1, 10, 0.0, 0, None)
    assert rc == engine.HFPX_ERR_STATE


_PANEL_RUN = r'''
import sys
import numpy as np
from hfpx3d_b200 import engine, meshgen
ctx = engine.Context(0)
nods, conn = meshgen.penny(int(sys.argv[1]), seed=3)
mesh = engine.MeshGeom(nods, conn)
dof, n = engine.make_dof_h_crack(mesh, 1)
dm = engine.DeviceMesh(ctx, mesh)
A = engine.assemble(ctx, dm, dof, n, 1.0, 0.35)
rhs = engine.add_s_inf_to_3dbem_rhs(ctx, dm, dof, n, [0, 0, 1.0, 0, 0, 0])
lu = engine.LU(ctx, A, engine.HFPX_LU_MIXED)
x = lu.solve(rhs, tol=1e-12)
np.save(sys.argv[2], np.concatenate([x, [lu.last_info.iterations, lu.last_info.residual]]))
'''


# a strongly diagonal matrix with its rows shuffled: partial pivoting
# interchanges rows at nearly every column (it undoes the shuffle), in every
# base panel and across block panels, and the system stays well conditioned
def _shuffled_system(n):
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n)) + 3.0 * n ** 0.5 * np.eye(n)
    return A[rng.permutation(n)], rng.standard_normal(n)


_RANDOM_RUN = r'''
import sys
import numpy as np
from hfpx3d_b200 import engine
ctx = engine.Context(0)
n = int(sys.argv[1])
rng = np.random.default_rng(n)
A = rng.standard_normal((n, n)) + 3.0 * n ** 0.5 * np.eye(n)
A = A[rng.permutation(n)]
b = rng.standard_normal(n)
lu = engine.LU(ctx, engine.DeviceMatrix.upload(ctx, A), engine.HFPX_LU_MIXED)
x = lu.solve(b, tol=1e-12, max_iter=60)
np.save(sys.argv[2], np.concatenate([x, [lu.last_info.iterations, lu.last_info.residual]]))
'''


def _panel_runs(tmp_path, n_el, kinds, script=_PANEL_RUN):
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = {}
    for kind in kinds:
        env = dict(os.environ, HFPX_LU_PANEL=kind, PYTHONPATH=root)
        f = tmp_path / ('x_%s.npy' % (kind or 'default'))
        r = subprocess.run([sys.executable, '-c', script, str(n_el), str(f)], env=env, cwd=root,
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        out[kind] = np.load(f)
    return out


@pytest.mark.parametrize('n_el', [300, 1200])
def test_fp32_panel_kernels_agree_bitwise(tmp_path, n_el):
    # the register-resident FP32 panel with partial pivoting (L2 word exchange
    # per column) and the shared-memory panel (grid barrier per column) take
    # the same pivots and do the same arithmetic per element: the mixed
    # solutions match bit for bit.  1200 elements (21 600 rows) spread the
    # first panels over 15 CTAs.
    out = _panel_runs(tmp_path, n_el, ('ll', 'smem'))
    assert np.array_equal(out['ll'], out['smem'])
    assert out['ll'][-1] <= 1e-12


def test_fp32_panel_kernels_agree_bitwise_with_interchanges(tmp_path):
    # 4500 rows: three block panels, rows interchanged at nearly every column,
    # so the register panel's row moves (and the compacted row-swap plans of
    # the block steps) carry the factorisation; the shared-memory panel swaps
    # by plans inside the recursion.  Same pivots, same bits, and the solution
    # meets the Gaussian system.
    n = 4500
    out = _panel_runs(tmp_path, n, ('ll', 'smem'), script=_RANDOM_RUN)
    assert np.array_equal(out['ll'], out['smem'])
    A, b = _shuffled_system(n)
    x = out['ll'][:n]
    assert out['ll'][-1] <= 1e-12
    assert np.abs(A @ x - b).max() <= 1e-10 * np.abs(A).max() * np.abs(x).max()
    assert np.abs(x - np.linalg.solve(A, b)).max() <= 1e-10 * np.abs(x).max()


@pytest.mark.parametrize('n_el', [300, 1200, 2500])
def test_tournament_panel_reaches_the_same_solution(tmp_path, n_el):
    # HFPX_LU_PANEL=tslu pivots the mixed factorisation by tournament (one
    # exchange per 32 columns instead of one per column); its pivots differ
    # from partial pivoting's, and the refinement against the FP64 matrix
    # brings both to the same solution.  2500 elements (45 000 rows) spread
    # the first panels over 30 CTAs, 960 tournament candidates.
    out = _panel_runs(tmp_path, n_el, ('tslu', ''))
    x0, x1 = out[''][:-2], out['tslu'][:-2]
    assert out['tslu'][-1] <= 1e-12
    assert out['tslu'][-2] <= out[''][-2] + 2     # refinement iterations
    assert np.abs(x1 - x0).max() <= 1e-10 * np.abs(x0).max()


def test_mixed_singular_reports_column(ctx):
    from hfpx3d_b200 import engine
    for n, col in ((50, 17), (3000, 1234)):
        A = np.eye(n) + 0.01 * np.random.default_rng(n).standard_normal((n, n))
        A[:, col] = 0.0
        m = engine.DeviceMatrix.upload(ctx, A)
        with pytest.raises(engine.EngineError) as e:
            engine.LU(ctx, m, engine.HFPX_LU_MIXED)
        assert e.value.code == engine.HFPX_ERR_SINGULAR
        assert str(col + 1) in str(e.value)


def test_tile_sweep_triangular_solves(tmp_path):
    # the engine's tile-sweep triangular solves (default) and cuBLAS's
    # (HFPX_TRSV=cublas) reach the same refined solution
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = {}
    for kind in ('', 'cublas'):
        env = dict(os.environ, HFPX_TRSV=kind, PYTHONPATH=root)
        f = tmp_path / ('x_%s.npy' % (kind or 'own'))
        r = subprocess.run([sys.executable, '-c', _PANEL_RUN, '700', str(f)], env=env, cwd=root,
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        out[kind] = np.load(f)
    x0, x1 = out['cublas'][:-2], out[''][:-2]
    assert out[''][-1] <= 1e-12
    assert np.abs(x1 - x0).max() <= 1e-10 * np.abs(x0).max()


def test_gmres_matches_the_reference_solution(ctx):
    # flexible GMRES on the FP64 matrix, preconditioned by the mixed FP32
    # factors (hfpx_gmres), against the reference's own LAPACK solution
    from hfpx3d_b200 import engine
    g = golden('ref_c1')
    mesh = engine.MeshGeom(g['nods'], g['conn'])
    dof, n = engine.make_dof_h_crack(mesh, 0)
    dm = engine.DeviceMesh(ctx, mesh)
    A = engine.assemble(ctx, dm, dof, n, 1.0, 0.35)
    lu = engine.LU(ctx, A, engine.HFPX_LU_MIXED)
    x = lu.gmres(g['rhs'], tol=1e-12)
    assert lu.last_info.converged and lu.last_info.residual <= 1e-12
    assert 1 <= lu.last_info.iterations <= 10
    assert np.abs(x - g['x']).max() / np.abs(g['x']).max() < 1e-9
    # a second call on the same factors gives the same bits
    x2 = lu.gmres(g['rhs'], tol=1e-12)
    assert np.array_equal(x, x2)


def test_gmres_against_refinement_and_states(ctx):
    from hfpx3d_b200 import engine, meshgen
    nods, conn = meshgen.penny(1200, seed=3)
    mesh = engine.MeshGeom(nods, conn)
    dof, n = engine.make_dof_h_crack(mesh, 1)
    dm = engine.DeviceMesh(ctx, mesh)
    rhs = engine.add_s_inf_to_3dbem_rhs(ctx, dm, dof, n, [0, 0, 1.0, 0, 0, 0])
    A = engine.assemble(ctx, dm, dof, n, 1.0, 0.35)
    lu = engine.LU(ctx, A, engine.HFPX_LU_MIXED)
    xr = lu.solve(rhs, tol=1e-12)
    it_refine = lu.last_info.iterations
    xg = lu.gmres(rhs, tol=1e-12, restart=2)     # restarts: cycles of two steps
    assert lu.last_info.converged and lu.last_info.iterations <= 2 * it_refine
    assert np.abs(xg - xr).max() <= 1e-10 * np.abs(xr).max()
    # GMRES needs the FP64 matrix beside FP32 factors: an FP64 factorisation is refused
    A64 = engine.assemble(ctx, dm, dof, n, 1.0, 0.35)
    lu64 = engine.LU(ctx, A64, engine.HFPX_LU_FP64)
    with pytest.raises(engine.EngineError) as e:
        lu64.gmres(rhs)
    assert e.value.code == engine.HFPX_ERR_STATE
