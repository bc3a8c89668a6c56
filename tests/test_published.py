"""The reference's published driver outputs (Test_Output/test_{solution,stresses}_<sig>.csv
for five shipped meshes, written by main.cpp with the shipped config.toml and packed
into tests/golden/ref_published.npz by tests/golden/make_published.py) reproduced
  * by the CPU oracle (pins the oracle to the reference's own known answers),
  * by this engine's driver hfpx3d_b200/bin/hfpx_main, FP64 and mixed precision,
  * by the reference's own main.cpp, compiled unchanged with the engine's
    system_assembly and LAPACKE libraries in place of its assembly and OpenBLAS
    (oracle/_ref/HFPx3D_engine, built where the reference tree is).

The csv values carry 6 significant digits, so agreement is to that precision:
|published - ours| <= 5e-6 |published| + 1e-6 max|published|.  One entry set is
looser: psc_1025 at the first observation point (0, 1.001, 0.001), 0.001 from the
crack front, where the published run differs from the reference's own code as
compiled here by up to 3e-4 (Sxy -0.10855 published, -0.1085783 from
system_assembly.cpp:279-455 here); the oracle and the engine agree with the latter.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_MAIN = os.path.join(ROOT, 'oracle', '_ref', 'HFPx3D_engine')
MESHES = {'psc_24': 'pennymesh24el', 'psc_121': 'pennymesh121el', 'psc_1025': 'pennymesh1025el',
          'elc_124': 'elliptical_124_el', 'elc_550': 'elliptical_550_el'}
G, NU, S_INF = 1.0, 0.35, [0.0, 0.0, 1.0, 0.0, 0.0, 0.0]

# the keys of the shipped config.toml that the driver reads, with its values
CONFIG = '''mesh_input_directory = "Mesh_Files"
mesh_conn_fname = "Elems_{mesh}_32.npy"
nodes_crd_fname = "Nodes_{mesh}_32.npy"
output_signature = "_{sig}_ele"
mesh_input_format = "npy32"
do_save_matrix = false
do_save_solution = true
do_postprocess = true
output_directory = "Test_Output"
output_format = "csv"
observ_crd_directory = "Test_Output"
observ_crd_fname = "observation_points.csv"
observ_input_format = "csv"
array_origin = 1
cp_offset = 0.125
fix_tip = 1
is_dd_local = false
is_tr_local = false
S_xx = 0
S_yy = 0
S_zz = -1.0
S_xy = 0
S_xz = 0
S_yz = 0
Shear_modulus = 1.0
Poisson_ratio = 3.5e-1
'''


@pytest.fixture(scope='module')
def pub():
    return golden('ref_published')


def write_run_dir(d, pub, sig, extra=''):
    """config.toml, Mesh_Files/ (the shipped .npy files) and
    Test_Output/observation_points.csv, laid out as in the reference tree."""
    mesh = MESHES[sig]
    (d / 'Mesh_Files').mkdir(parents=True, exist_ok=True)
    (d / 'Test_Output').mkdir(exist_ok=True)
    np.save(d / 'Mesh_Files' / f'Elems_{mesh}_32.npy', pub[f'{sig}_conn'])
    np.save(d / 'Mesh_Files' / f'Nodes_{mesh}_32.npy', pub[f'{sig}_nods'])
    (d / 'Test_Output' / 'observation_points.csv').write_text(
        '\n'.join(','.join(repr(float(v)) for v in row) for row in pub['pts']))
    (d / 'config.toml').write_text(CONFIG.format(mesh=mesh, sig=sig) + extra)
    return d / 'config.toml'


def assert_print_precision(ours, published, looser_rows=()):
    ours = np.asarray(ours, dtype=np.float64)
    assert ours.shape == published.shape
    tol = 5e-6 * np.abs(published) + 1e-6 * np.abs(published).max()
    for r in looser_rows:
        tol[r] = 3e-4 * np.abs(published[r]) + 1e-6 * np.abs(published).max()
    bad = np.abs(ours - published) > tol
    assert not bad.any(), (np.argwhere(bad)[:5], ours[bad][:5], published[bad][:5])


def looser(sig):
    return (0,) if sig == 'psc_1025' else ()


def node_points(pub, sig):
    """Columns 0-3 of the solution file: the 6 nodal points of each element
    (vertices, then the midpoint of the edge opposite each vertex) and a 0."""
    conn = pub[f'{sig}_conn'][:3].astype(np.int64) - 1
    nods = pub[f'{sig}_nods'][:3]
    v = nods[:, conn]
    mid = 0.5 * (v[:, [1, 2, 0]] + v[:, [2, 0, 1]])
    xyz = np.concatenate([v, mid], axis=1).transpose(2, 1, 0).reshape(-1, 3)
    return np.concatenate([xyz, np.zeros((xyz.shape[0], 1))], axis=1)


@pytest.mark.parametrize('sig', ['psc_24', 'psc_121', 'elc_124'])
def test_oracle_reproduces_published(ora, pub, sig):
    conn = np.asfortranarray(pub[f'{sig}_conn'].astype(np.int64))
    conn[:3] -= 1
    nods = np.asfortranarray(pub[f'{sig}_nods'])
    dof, n = ora.dof_handle(nods, conn, 1)
    A = ora.assemble(nods, conn, dof, n, G, NU, beta=0.125)
    x = np.linalg.solve(A, ora.rhs(nods, conn, dof, n, S_INF))
    dd = ora.dd_from_solution(x, dof, conn.shape[1])
    sol = pub[f'{sig}_solution']
    assert_print_precision(node_points(pub, sig), sol[:, :4])
    assert_print_precision(dd, sol[:, 4:])
    st = ora.stress(nods, conn, dd, np.asfortranarray(pub['pts'].T), S_INF, G, NU)
    assert_print_precision(st, pub[f'{sig}_stresses'])


def check_outputs(d, pub, sig):
    out = d / 'Test_Output'
    sol = np.loadtxt(out / f'test_solution_{sig}_ele.csv', delimiter=',')
    st = np.loadtxt(out / f'test_stresses_{sig}_ele.csv', delimiter=',')
    assert_print_precision(sol, pub[f'{sig}_solution'])
    assert_print_precision(st, pub[f'{sig}_stresses'], looser(sig))


@pytest.fixture(scope='module')
def driver():
    from hfpx3d_b200 import build
    build.build()
    return build.MAIN


def test_driver_reads_the_shipped_config(tmp_path, pub, driver):
    cfg = write_run_dir(tmp_path, pub, 'elc_550')
    r = subprocess.run([driver, '--check', str(cfg)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    o = dict(line.partition(' ')[::2] for line in r.stdout.splitlines())
    assert int(o['elements']) == 550 and int(o['tip_type']) == 1 and float(o['beta']) == 0.125
    assert [float(v) for v in o['s_inf'].split()] == S_INF
    assert o['points'] == '3 x 11'
    assert o['output'].endswith('/Test_Output/test_solution_elc_550_ele.csv')


@pytest.mark.gpu
@pytest.mark.parametrize('sig,precision', [('psc_24', 'fp64'), ('psc_121', 'fp64'), ('elc_124', 'fp64'),
                                           ('elc_550', 'fp64'), ('elc_550', 'mixed'), ('psc_1025', 'fp64'),
                                           ('psc_1025', 'mixed')])
def test_engine_driver_reproduces_published(tmp_path, pub, driver, sig, precision):
    cfg = write_run_dir(tmp_path, pub, sig, '[engine]\nprecision = "%s"\n' % precision)
    r = subprocess.run([driver, str(cfg)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    n_el = pub[f'{sig}_conn'].shape[1]
    assert '%d DoF Total' % (18 * n_el) in r.stdout
    check_outputs(tmp_path, pub, sig)


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF_MAIN), reason='oracle/_ref/HFPx3D_engine is built where the reference tree is')
@pytest.mark.parametrize('sig', ['psc_24', 'psc_121', 'elc_550'])
def test_reference_main_on_the_engine(tmp_path, pub, sig):
    # the reference's driver reads ./config.toml and writes under ./Test_Output
    write_run_dir(tmp_path, pub, sig)
    r = subprocess.run([REF_MAIN], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.splitlines()
    n_el = pub[f'{sig}_conn'].shape[1]
    assert lines[0].startswith('Assembly: ') and lines[1] == '%d DoF Total' % (18 * n_el)
    assert any(s.startswith('Solution: ') for s in lines) and any(s.startswith('Postprocessing: ') for s in lines)
    check_outputs(tmp_path, pub, sig)
