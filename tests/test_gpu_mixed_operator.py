"""The mixed-precision operator (hfpx_assemble_mixed): the matrix of
make_3dbem_matrix_s (src/Solvers/system_assembly.cpp:30-219) held as FP32
entries, with the near-field blocks (each element with itself and with the
elements sharing a vertex) kept to ~2^-48 by FP32 low parts.

* entries against the FP64 assembly of the same kernel: far entries are
  exactly the FP32 rounding of the FP64 entries, near entries within 1e-14
  relative, on a planar penny (in-plane path) and a wavy crack (off-plane
  path);
* its product r = b - A x against numpy with the composed matrix (1e-13);
* GMRES on it (near-field and learned two-level preconditioners) against the
  FP64 LU solution of the FP64 matrix: the opening within 1e-8 of the
  opening's scale (the metric's accuracy bound), the solution's residual on
  the FP64 matrix within 1e-7 of |b|;
* the operations it does not support report HFPX_ERR_STATE."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
G, NU, BETA = 1.0, 0.35, 0.125


def near_mask(conn):
    ne = conn.shape[1]
    v2e = {}
    for e in range(ne):
        for v in conn[:3, e]:
            v2e.setdefault(int(v), set()).add(e)
    m = np.zeros((ne, ne), dtype=bool)
    for e in range(ne):
        for i in set().union(*[v2e[int(v)] for v in conn[:3, e]]):
            m[i, e] = True
    return np.kron(m, np.ones((18, 18), dtype=bool))


def build(ctx, kind, args, kwargs):
    from hfpx3d_b200 import engine, meshgen
    nods, conn = getattr(meshgen, kind)(*args, **kwargs)
    mesh = engine.MeshGeom(nods, conn)
    dof, n = engine.make_dof_h_crack(mesh, 0)
    dm = engine.DeviceMesh(ctx, mesh, BETA)
    return nods, conn, dm, dof, n


@pytest.mark.parametrize('kind,args,kwargs', [('penny', (200,), dict(seed=11)),
                                              ('wavy', (120,), dict(aspect=1.5, amp=0.15, seed=12))])
def test_entries_are_the_fp64_entries_rounded(ctx, kind, args, kwargs):
    from hfpx3d_b200 import engine
    nods, conn, dm, dof, n = build(ctx, kind, args, kwargs)
    A64 = engine.assemble(ctx, dm, dof, n, G, NU).download()
    Am = engine.assemble_mixed(ctx, dm, dof, n, G, NU)
    assert Am.mixed
    M = Am.download()
    near = near_mask(conn)
    far = ~near
    assert np.array_equal(M[far], A64[far].astype(np.float32).astype(np.float64))
    rel = np.abs(M[near] - A64[near]) / np.maximum(np.abs(A64[near]), 1e-300)
    assert rel.max() <= 1e-14, rel.max()
    # the near entries carry more than the FP32 rounding alone would
    assert np.abs(M[near] - A64[near]).max() < 1e-3 * np.abs(A64[near].astype(np.float32) - A64[near]).max()
    # a block of the same, and re-assembly into it
    blk = Am.block(18 * 5, 18 * 7, 40, 30)
    assert np.array_equal(blk, M[90:130, 126:156])
    engine.assemble_into(ctx, dm, dof, n, G, NU, Am)
    assert np.array_equal(Am.download(), M)


def test_product_matches_numpy(ctx):
    import torch
    from hfpx3d_b200 import engine
    nods, conn, dm, dof, n = build(ctx, 'penny', (300,), dict(seed=13))
    Am = engine.assemble_mixed(ctx, dm, dof, n, G, NU)
    M = Am.download()
    rng = np.random.default_rng(3)
    x = rng.standard_normal(n)
    b = rng.standard_normal(n)
    dx = torch.tensor(x, device='cuda')
    db = torch.tensor(b, device='cuda')
    dr = torch.empty(n, dtype=torch.float64, device='cuda')
    torch.cuda.synchronize()
    lib = engine.lib()
    ctx.check(lib.hfpx_residual_device(ctx.h, Am.h, ctypes.c_void_p(dx.data_ptr()), ctypes.c_void_p(db.data_ptr()),
                                       ctypes.c_void_p(dr.data_ptr())))
    ctx.synchronize()
    r_ref = b - M @ x
    scale = np.abs(M).max() * np.abs(x).sum() / np.sqrt(n)
    assert np.abs(dr.cpu().numpy() - r_ref).max() <= 1e-13 * scale


@pytest.mark.parametrize('kind,args,kwargs,pc', [
    ('penny', (1200,), dict(seed=14), 'learned+coarse'),
    ('wavy', (600,), dict(aspect=2.0, amp=0.15, seed=15), 'neumann')])
def test_gmres_on_the_mixed_operator_matches_the_fp64_solution(ctx, kind, args, kwargs, pc):
    from hfpx3d_b200 import engine
    nods, conn, dm, dof, n = build(ctx, kind, args, kwargs)
    A64 = engine.assemble(ctx, dm, dof, n, G, NU)
    rhs = engine.add_s_inf_to_3dbem_rhs(ctx, dm, dof, n, [0, 0, 1.0, 0, 0, 0])
    Ah = A64.download()
    x64 = engine.LU(ctx, A64, engine.HFPX_LU_FP64).solve(rhs)
    Am = engine.assemble_mixed(ctx, dm, dof, n, G, NU)
    if pc == 'learned+coarse':
        net = engine.Gnn(ctx, path=engine.WEIGHTS_PATH)
        P = engine.Precond(ctx, dm, Am, engine.HFPX_PC_LEARNED | engine.HFPX_PC_COARSE, net=net, shear_m=G)
    else:
        P = engine.Precond(ctx, dm, Am, engine.HFPX_PC_NEUMANN)
    x, info = engine.gmres(ctx, Am, rhs, P, tol=1e-10, restart=50, max_iter=500)
    assert info.converged, info.residual
    w, w64 = x[2::3], x64[2::3]
    err = np.abs(w - w64).max() / np.abs(w64).max()
    print(f'{kind} N={n}: opening error of the mixed-precision operator vs FP64: {err:.2e}, '
          f'{info.iterations} GMRES steps')
    assert err <= 1e-8, err
    res = np.abs(rhs - Ah @ x).max() / np.abs(rhs).max()
    assert res <= 1e-7, res


def test_unsupported_operations_report_state(ctx):
    from hfpx3d_b200 import engine
    nods, conn, dm, dof, n = build(ctx, 'penny', (60,), dict(seed=16))
    Am = engine.assemble_mixed(ctx, dm, dof, n, G, NU)
    lib = engine.lib()
    info = ctypes.c_int64()
    assert lib.hfpx_lu_factor(ctx.h, Am.h, engine.HFPX_LU_MIXED, ctypes.byref(info)) == engine.HFPX_ERR_STATE
    out = ctypes.c_void_p()
    keep = np.arange(10, dtype=np.int64)
    assert lib.hfpx_matrix_truncate(ctx.h, Am.h, keep.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), 10, 0,
                                    ctypes.byref(out)) == engine.HFPX_ERR_STATE
    # fixed DoF (tip type 1) are not supported by the mixed form
    mesh = engine.MeshGeom(nods, conn)
    dof1, n1 = engine.make_dof_h_crack(mesh, 1)
    if n1 < n:
        with pytest.raises(engine.EngineError):
            engine.assemble_mixed(ctx, dm, dof1, n1, G, NU)
