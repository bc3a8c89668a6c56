"""Incremental assembly of a growing crack (hfpx_assemble_grow): the step the
reference leaves as "todo: growing mesh" (src/Development/c_f_iteration.cpp:289)
around its full re-assembly (make_3dbem_matrix_s,
src/Solvers/system_assembly.cpp:30-219).

* a crack grown by appending elements: the old block copied and only the new
  rows and columns assembled equals the full assembly of the grown mesh bit
  for bit (the same kernel evaluates every pair), on a planar penny grown
  ring by ring and on a non-planar wavy crack (off-plane pairs);
* the grown operator's solution matches the oracle's (1e-10);
* removing elements again (hfpx_matrix_truncate on the remaining elements'
  DoF) gives the old operator;
* DoF numberings that do not keep the old elements' numbers are refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
G, NU, BETA = 1.0, 0.35, 0.125


def meshes(kind, n_tri, n_old, **kw):
    from hfpx3d_b200 import engine, meshgen
    nods, conn = getattr(meshgen, kind)(n_tri, **kw)
    old = engine.MeshGeom(nods, np.asfortranarray(conn[:, :n_old]))
    new = engine.MeshGeom(nods, conn)
    return nods, conn, old, new


@pytest.mark.parametrize('kind,n_tri,n_old,kw', [('penny', 400, 250, dict(seed=21)),
                                                 ('wavy', 200, 120, dict(aspect=1.5, amp=0.15, seed=22))])
def test_grown_operator_equals_the_full_assembly(ctx, kind, n_tri, n_old, kw):
    from hfpx3d_b200 import engine
    nods, conn, old, new = meshes(kind, n_tri, n_old, **kw)
    dof_o, n_o = engine.make_dof_h_crack(old, 0)
    dof_n, n_n = engine.make_dof_h_crack(new, 0)
    dm_o = engine.DeviceMesh(ctx, old, BETA)
    dm_n = engine.DeviceMesh(ctx, new, BETA)
    A_old = engine.assemble(ctx, dm_o, dof_o, n_o, G, NU)
    A_grown = engine.assemble_grow(ctx, dm_n, n_old, dof_n, n_n, G, NU, A_old)
    A_full = engine.assemble(ctx, dm_n, dof_n, n_n, G, NU).download()
    Ag = A_grown.download()
    assert np.array_equal(Ag, A_full)
    # removing the appended elements again: the old operator
    T = engine.truncate(ctx, A_grown, np.arange(n_o, dtype=np.int64), keep_border=False)
    assert np.array_equal(T.download(), A_old.download())


def test_grown_solution_matches_the_oracle(ctx, ora):
    from hfpx3d_b200 import engine
    nods, conn, old, new = meshes('penny', 150, 90, seed=23)
    dof_o, n_o = engine.make_dof_h_crack(old, 0)
    dof_n, n_n = engine.make_dof_h_crack(new, 0)
    A_old = engine.assemble(ctx, engine.DeviceMesh(ctx, old, BETA), dof_o, n_o, G, NU)
    dm_n = engine.DeviceMesh(ctx, new, BETA)
    A = engine.assemble_grow(ctx, dm_n, 90, dof_n, n_n, G, NU, A_old)
    rhs = engine.add_s_inf_to_3dbem_rhs(ctx, dm_n, dof_n, n_n, [0, 0, 1.0, 0, 0, 0])
    x = engine.LU(ctx, A, engine.HFPX_LU_FP64).solve(rhs)
    Ao = ora.assemble(nods, conn, dof_n, n_n)
    xo = np.linalg.solve(Ao, ora.rhs(nods, conn, dof_n, n_n, [0, 0, 1.0, 0, 0, 0]))
    assert np.abs(x - xo).max() <= 1e-10 * np.abs(xo).max()


def test_numbering_that_moves_old_dof_is_refused(ctx):
    from hfpx3d_b200 import engine
    nods, conn, old, new = meshes('penny', 120, 60, seed=24)
    dof_o, n_o = engine.make_dof_h_crack(old, 0)
    dof_n, n_n = engine.make_dof_h_crack(new, 0)
    A_old = engine.assemble(ctx, engine.DeviceMesh(ctx, old, BETA), dof_o, n_o, G, NU)
    dm_n = engine.DeviceMesh(ctx, new, BETA)
    # appended elements numbered first
    perm = np.concatenate([np.arange(60, 120), np.arange(60)])
    bad = np.asfortranarray(dof_n[perm])
    with pytest.raises(engine.EngineError):
        engine.assemble_grow(ctx, dm_n, 60, bad, n_n, G, NU, A_old)
