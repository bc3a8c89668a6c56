"""The batched workload (hfpx_batch_*): many meshes of uneven sizes, each with
many load cases, assembled, factored and solved in one CUDA-graph launch.
Per mesh and load case this is the reference's make_3dbem_matrix_s
(src/Solvers/system_assembly.cpp:30-219), add_s_inf_to_3dbem_rhs (:222-274)
and il::LU factor + solve (il/linear_algebra/dense/factorization/LU.h:79-120).

* every mesh's load-case solutions against the FP64 LU solution of the FP64
  matrix of the same mesh (engine path pinned to the reference elsewhere):
  within 1e-8 of each case's largest DD (the operator's far field is held in
  FP32, as hfpx_assemble_mixed's), with the refinement residual <= 1e-10;
* one mesh against the CPU oracle's LAPACK solution;
* the block size / leaf-row tile choices give the same solutions;
* a replayed run (the captured graph) reproduces the first run bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
G, NU, BETA = 1.0, 0.35, 0.125


def load_cases(rng, n_cases):
    """Uniform pressures in [0.5, 2] and random in-situ stress tensors
    (principal values in [-1, 0], Haar rotation), Voigt, tension positive."""
    out = np.zeros((6, n_cases))
    for j in range(n_cases):
        if j % 2 == 0:
            out[2, j] = rng.uniform(0.5, 2.0)
        else:
            q, r = np.linalg.qr(rng.standard_normal((3, 3)))
            q = q * np.sign(np.diag(r))
            s = q @ np.diag(rng.uniform(-1, 0, 3)) @ q.T
            out[:, j] = [s[0, 0], s[1, 1], s[2, 2], s[0, 1], s[0, 2], s[1, 2]]
    return out


def make_batch_meshes(seed, sizes):
    from hfpx3d_b200 import meshgen
    out = []
    for k, ne in enumerate(sizes):
        if k % 2 == 0:
            out.append(meshgen.penny(ne, seed=seed + k))
        else:
            out.append(meshgen.ellipse(ne, seed=seed + k))
    return out


def fp64_solutions(ctx, nods, conn, S):
    from hfpx3d_b200 import engine
    mesh = engine.MeshGeom(nods, conn)
    dof, n = engine.make_dof_h_crack(mesh, 0)
    dm = engine.DeviceMesh(ctx, mesh, BETA)
    A = engine.assemble(ctx, dm, dof, n, G, NU)
    rhs = np.stack([engine.add_s_inf_to_3dbem_rhs(ctx, dm, dof, n, S[:, j]) for j in range(S.shape[1])], axis=1)
    return engine.LU(ctx, A, engine.HFPX_LU_FP64).solve(np.asfortranarray(rhs))


@pytest.fixture(scope='module')
def small_batch(ctx):
    from hfpx3d_b200 import engine
    sizes = [24, 150, 60, 121, 300, 90, 200, 45]
    meshes = make_batch_meshes(500, sizes)
    rng = np.random.default_rng(7)
    S = np.stack([load_cases(rng, 8) for _ in sizes])
    dms = [engine.DeviceMesh(ctx, engine.MeshGeom(nods, conn), BETA) for nods, conn in meshes]
    return meshes, S, dms


@pytest.mark.parametrize('nb,leaf', [(128, 512), (64, 256)])
def test_batch_matches_fp64_solutions(ctx, small_batch, nb, leaf):
    from hfpx3d_b200 import engine
    meshes, S, dms = small_batch
    B = engine.Batch(ctx, dms, G, NU, nb=nb, leaf_rows=leaf)
    B.set_loads(S)
    info = B.run(tol=1e-10)
    assert info.converged, info.residual
    assert info.singular_mesh == -1
    assert np.all(B.residuals() <= 1e-10)
    worst = 0.0
    for m, (nods, conn) in enumerate(meshes):
        x = B.solution(m)
        x64 = fp64_solutions(ctx, nods, conn, S[m])
        err = np.abs(x - x64).max(axis=0) / np.abs(x64).max(axis=0)
        worst = max(worst, err.max())
        assert err.max() <= 1e-8, (m, err.max())
    print(f'batch nb={nb} leaf={leaf}: worst case error vs FP64 LU {worst:.2e}, residual {info.residual:.2e}')
    # the captured graph replayed: the same bits
    x0 = B.solution(4)
    info2 = B.run(tol=1e-10)
    assert info2.converged
    assert np.array_equal(B.solution(4), x0)
    B.close()


def test_batch_mesh_matches_the_oracle(ctx, ora):
    from hfpx3d_b200 import engine
    nods, conn = make_batch_meshes(900, [60])[0]
    S = load_cases(np.random.default_rng(3), 4)
    dm = engine.DeviceMesh(ctx, engine.MeshGeom(nods, conn), BETA)
    B = engine.Batch(ctx, [dm], G, NU)
    B.set_loads(S[None])
    assert B.run(tol=1e-11).converged
    x = B.solution(0)
    mesh = engine.MeshGeom(nods, conn)
    dof, n = engine.make_dof_h_crack(mesh, 0)
    Ao = ora.assemble(nods, conn, dof, n)
    for j in range(S.shape[1]):
        xo = np.linalg.solve(Ao, ora.rhs(nods, conn, dof, n, S[:, j]))
        assert np.abs(x[:, j] - xo).max() <= 1e-8 * np.abs(xo).max(), j
    B.close()


def test_unit_states_without_load_cases(ctx, small_batch):
    """Without load cases the solutions are the 6 unit in-situ stress states'."""
    from hfpx3d_b200 import engine
    meshes, S, dms = small_batch
    B = engine.Batch(ctx, dms[:3], G, NU)
    assert B.run(tol=1e-10).converged
    x6 = B.solution(1)
    x64 = fp64_solutions(ctx, *meshes[1], np.eye(6))
    assert np.abs(x6 - x64).max() <= 1e-8 * np.abs(x64).max()
    B.close()
