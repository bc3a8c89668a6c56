"""Matrix assembly, volume-control border, right-hand side and stress on the
GPU through the C-ABI, against the CPU oracle (pinned to the reference by the
golden fixtures) and the reference's own outputs."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu
G, NU, BETA = 1.0, 0.35, 0.125


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def device_case(ctx, nods, conn, tip=0, vc=False, local=False):
    from hfpx3d_b200 import engine
    mesh = engine.MeshGeom(nods, conn)
    dof, n = engine.make_dof_h_crack(mesh, tip)
    dm = engine.DeviceMesh(ctx, mesh, BETA)
    A = engine.assemble(ctx, dm, dof, n, G, NU, is_dd_local=local, vc=vc).download()
    return mesh, dm, dof, n, A


@pytest.mark.parametrize('name', ['triangle', 'bitriangle', 'radial24'])
def test_matlab_full_matrices(ctx, name):
    g = golden('matlab_assembly')
    key = {'triangle': 'tri', 'bitriangle': 'bit', 'radial24': 'p24'}[name]
    _, _, _, _, A = device_case(ctx, g[key + '_nods'], g[key + '_conn'])
    assert np.abs(A - g[name]).max() < 5e-7 * max(1.0, np.abs(g[name]).max())


@pytest.mark.parametrize('case,tol', [('ref_p24', 1e-11), ('ref_bitriangle', 1e-11)])
def test_full_matrix_vs_reference(ctx, ora, case, tol):
    g = golden(case)
    mesh, dm, dof, n, A = device_case(ctx, g['nods'], g['conn'], int(g['tip']))
    assert (dof == g['dof']).all() and n == int(g['n_dof'])
    assert rel(A, g['A']) < tol
    assert rel(A, ora.assemble(g['nods'], g['conn'], dof, n)) < 1e-12


def test_tip_fixed_matrix(ctx):
    g = golden('ref_p24_tip1')
    m = golden('ref_dof')
    _, _, dof, n, A = device_case(ctx, m['p24_nods'], m['p24_conn'], tip=1)
    assert n == int(g['n_dof']) and rel(A, g['A']) < 1e-11


@pytest.mark.parametrize('case,tol', [('ref_p121', 1e-11), ('ref_c1', 1e-11), ('ref_wavy48', 1e-9)])
def test_summarized_vs_reference_and_oracle(ctx, ora, case, tol):
    # wavy48: tilted neighbours put collocation points near other elements'
    # planes, where the reference's closed form loses up to ~1e-7 per block
    # (truth_blocks.npz); 1e-9 of the matrix scale covers that, and the
    # oracle comparison below stays tight.
    g = golden(case)
    mesh, dm, dof, n, A = device_case(ctx, g['nods'], g['conn'], int(g['tip']))
    scale = np.abs(g['A_sample_v']).max()
    assert np.abs(A[g['A_sample_i'], g['A_sample_j']] - g['A_sample_v']).max() < tol * scale
    assert np.abs(A.sum(axis=0) - g['A_col_sum']).max() < 10 * tol * np.abs(g['A_abs_col_sum']).max()
    # far-field entries come from sums that cancel to ~1e-4 of their terms, so
    # FMA-vs-CPU rounding shows up at a few 1e-12 of the matrix scale
    Ao = ora.assemble(g['nods'], g['conn'], dof, n)
    assert rel(A, Ao) < 1e-11


@pytest.mark.parametrize('case', ['ref_p24', 'ref_bitriangle', 'ref_c1'])
def test_vc_border(ctx, case):
    g = golden(case)
    _, _, dof, n, Av = device_case(ctx, g['nods'], g['conn'], int(g['tip']), vc=True)
    assert rel(Av[n, :], g['vc_row']) < 1e-13 and rel(Av[:, n], g['vc_col']) < 1e-15
    assert Av[n, n] == 0.0


@pytest.mark.parametrize('case', ['ref_p24', 'ref_c1', 'ref_bitriangle'])
def test_rhs(ctx, case):
    from hfpx3d_b200 import engine
    g = golden(case)
    mesh = engine.MeshGeom(g['nods'], g['conn'])
    dof, n = engine.make_dof_h_crack(mesh, int(g['tip']))
    dm = engine.DeviceMesh(ctx, mesh, BETA)
    rhs = engine.add_s_inf_to_3dbem_rhs(ctx, dm, dof, n, g['s_inf'])
    assert np.abs(rhs - g['rhs']).max() <= 1e-15
    # several load cases at once
    S = np.column_stack([g['s_inf'], 2 * g['s_inf'], -g['s_inf']])
    R = engine.add_s_inf_to_3dbem_rhs(ctx, dm, dof, n, S)
    assert np.abs(R - np.column_stack([g['rhs'], 2 * g['rhs'], -g['rhs']])).max() <= 1e-14


@pytest.mark.parametrize('case,tol', [('ref_p24', 1e-10), ('ref_bitriangle', 1e-10), ('ref_c1', 1e-10),
                                      ('ref_p121', 1e-8), ('ref_wavy48', 1e-8)])
def test_stress(ctx, ora, case, tol):
    # ref_p121 point 76 sits 0.005 off the crack plane and 0.6 away in-plane:
    # the reference's own value there is off by ~4e-9 (truth_blocks.npz), so
    # the reference comparison uses 1e-8 and the oracle comparison 1e-11
    from hfpx3d_b200 import engine
    g = golden(case)
    mesh = engine.MeshGeom(g['nods'], g['conn'])
    dm = engine.DeviceMesh(ctx, mesh, BETA)
    st = engine.make_3dbem_stress_f_s(ctx, dm, G, NU, g['dd'], g['pts'], g['s_inf'])
    assert rel(st, g['stress']) < tol
    assert rel(st, ora.stress(g['nods'], g['conn'], g['dd'], g['pts'], g['s_inf'])) < 1e-11


def test_local_dd_variant(ctx, ora):
    g = golden('ref_bitriangle')
    _, _, dof, n, A = device_case(ctx, g['nods'], g['conn'], local=True)
    assert rel(A, ora.assemble(g['nods'], g['conn'], dof, n, is_dd_local=1)) < 1e-12


def test_assembly_is_deterministic(ctx):
    from hfpx3d_b200 import engine, meshgen
    nods, conn = meshgen.penny(300, seed=9)
    mesh = engine.MeshGeom(nods, conn)
    dof, n = engine.make_dof_h_crack(mesh, 0)
    dm = engine.DeviceMesh(ctx, mesh)
    A1 = engine.assemble(ctx, dm, dof, n, G, NU).download()
    A2 = engine.assemble(ctx, dm, dof, n, G, NU).download()
    assert np.array_equal(A1, A2)


def test_bad_inputs_report_errors(ctx):
    from hfpx3d_b200 import engine
    nods, conn = golden('ref_p24')['nods'], golden('ref_p24')['conn']
    bad = np.array(nods, copy=True, order='F')
    bad[0, 3] = np.nan
    with pytest.raises(engine.EngineError) as e:
        engine.DeviceMesh(ctx, engine.MeshGeom(bad, conn))
    assert e.value.code == engine.HFPX_ERR_ARG
    badc = np.array(conn, copy=True, order='F')
    badc[0, 0] = 10_000
    with pytest.raises(engine.EngineError):
        engine.DeviceMesh(ctx, engine.MeshGeom(nods, badc))
    mesh = engine.MeshGeom(nods, conn)
    dm = engine.DeviceMesh(ctx, mesh)
    dof, n = engine.make_dof_h_crack(mesh, 0)
    with pytest.raises(engine.EngineError):
        engine.assemble(ctx, dm, dof, n, -1.0, NU)
    dof2 = dof.copy(order='F')
    dof2[0, 0] = 10 ** 9
    with pytest.raises(engine.EngineError):
        engine.assemble(ctx, dm, dof2, n, G, NU)
