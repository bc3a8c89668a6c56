"""The C++ host layer and its config.toml driver (hfpx3d_b200/bin/hfpx_main),
which replaces the reference's main.cpp: config parsing
(src/IO/config_file_io.cpp:56-361), mesh / point readers
(src/IO/mesh_file_io.cpp), csv output (src/IO/data_file_io.h:131-168) on the
CPU; the whole pipeline on the GPU against the reference's outputs."""
import os
import subprocess

import numpy as np
import pytest

from conftest import golden

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope='module')
def driver():
    from hfpx3d_b200 import build
    build.build()
    return build.MAIN


def write_npy(path, a, fortran=True):
    a = np.asfortranarray(a) if fortran else np.ascontiguousarray(a)
    np.save(path, a)


def write_case(tmp, nods, conn, extra='', conn_dtype=np.int32, origin=0, fortran=True, fmt='npy32',
               pts=None, s_cfg=None):
    mesh = tmp / 'Mesh_Files'
    mesh.mkdir(exist_ok=True)
    conn = np.asarray(conn)[:3].astype(conn_dtype) + origin
    if fmt == 'csv':
        np.savetxt(mesh / 'conn.csv', conn.T, fmt='%d', delimiter=',')
        np.savetxt(mesh / 'nods.csv', np.asarray(nods)[:3].T, fmt='%.17g', delimiter=',')
        names = ('conn.csv', 'nods.csv')
    else:
        write_npy(mesh / 'conn.npy', conn, fortran)
        write_npy(mesh / 'nods.npy', np.asarray(nods, dtype=np.float64), fortran)
        names = ('conn.npy', 'nods.npy')
    lines = [f'mesh_input_directory = "Mesh_Files"',
             f'mesh_conn_fname = "{names[0]}"',
             f'nodes_crd_fname = "{names[1]}"',
             f'mesh_input_format = "{fmt}"',
             f'array_origin = {origin}',
             'output_directory = "Out"']
    (tmp / 'Out').mkdir(exist_ok=True)
    if pts is not None:
        np.savetxt(mesh / 'pts.csv', np.asarray(pts).T, fmt='%.17g', delimiter=',')
        lines += ['do_postprocess = true', 'observ_crd_fname = "pts.csv"']
    if s_cfg is not None:
        for k, v in s_cfg.items():
            lines.append(f'{k} = {v!r}')
    cfg = tmp / 'config.toml'
    cfg.write_text('\n'.join(lines) + '\n' + extra)
    return cfg


def check(driver, cfg):
    r = subprocess.run([driver, '--check', str(cfg)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    out = {}
    for line in r.stdout.splitlines():
        k, _, v = line.partition(' ')
        out[k] = v
    return out


def checksums(nods, conn):
    c = np.asarray(conn)[:3].astype(np.int64)
    n = np.asarray(nods)[:3]
    w = np.arange(1, 4)[:, None]
    return int((c * w).sum()), float((n * w).sum())


@pytest.mark.parametrize('fortran,dtype,origin', [(True, np.int32, 0), (False, np.int64, 1), (True, np.int64, 1)])
def test_config_and_numpy_mesh(tmp_path, driver, fortran, dtype, origin):
    g = golden('ref_p24')
    extra = ('cp_offset = 0.25\nfix_tip = 0\nis_dd_local = true\n'
             'S_xx = 1.5\nS_yy = -2.0\nS_zz = 3.0\nS_xy = 0.5\nS_xz = -0.25\nS_yz = 0.125\n'
             '[solid]\nYoung_modulus = 2.6\nPoisson_ratio = 0.3\n'
             '[engine]\nprecision = "mixed"\ndevice = 0\n')
    cfg = write_case(tmp_path, g['nods'], g['conn'], extra, dtype, origin, fortran)
    o = check(driver, cfg)
    assert int(o['elements']) == 24 and int(o['nodes']) == 19
    assert float(o['shear_m']) == 2.6 / 2.0 / 1.3 and float(o['poiss_r']) == 0.3
    assert float(o['beta']) == 0.25 and int(o['tip_type']) == 0 and o['is_dd_local'] == '1'
    # normal in-situ stresses are given compression-positive and negated
    assert [float(v) for v in o['s_inf'].split()] == [-1.5, 2.0, -3.0, 0.5, -0.25, 0.125]
    assert int(o['lu_mode']) == 1
    cs, ns = checksums(g['nods'], g['conn'])
    assert int(o['conn_checksum']) == cs
    assert float(o['nods_checksum']) == pytest.approx(ns, rel=1e-15)


def test_config_defaults_and_csv_mesh(tmp_path, driver):
    g = golden('ref_p24')
    pts = g['pts']
    cfg = write_case(tmp_path, g['nods'], g['conn'], 'Shear_modulus = 3.0\n', fmt='csv', pts=pts,
                     origin=1)
    o = check(driver, cfg)
    assert float(o['shear_m']) == 3.0 and float(o['poiss_r']) == 0.0
    assert float(o['beta']) == 0.125 and int(o['tip_type']) == 1 and o['is_dd_local'] == '0'
    assert [float(v) for v in o['s_inf'].split()] == [0.0] * 6
    assert int(o['lu_mode']) == 0
    assert o['points'] == '3 x 20'
    cs, ns = checksums(g['nods'], g['conn'])
    assert int(o['conn_checksum']) == cs
    assert float(o['nods_checksum']) == pytest.approx(ns, rel=1e-14)
    assert o['output'].endswith('/Out/test_solution.csv')


@pytest.mark.parametrize('extra,msg', [('', 'observ_crd_fname'),
                                       ('observ_crd_fname = "p.csv"\n[engine]\nprecision = "half"\n',
                                        'precision')])
def test_config_errors(tmp_path, driver, extra, msg):
    g = golden('ref_p24')
    cfg = write_case(tmp_path, g['nods'], g['conn'], 'do_postprocess = true\n' + extra)
    r = subprocess.run([driver, '--check', str(cfg)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and msg in r.stderr


def test_missing_mesh_key(tmp_path, driver):
    cfg = tmp_path / 'config.toml'
    cfg.write_text('nodes_crd_fname = "n.npy"\n')
    r = subprocess.run([driver, '--check', str(cfg)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and 'mesh_conn_fname' in r.stderr


def s_config(s_inf):
    """config.toml in-situ stress entries that give the internal s_inf."""
    s = np.asarray(s_inf, dtype=np.float64)
    return {'S_xx': float(-s[0]), 'S_yy': float(-s[1]), 'S_zz': float(-s[2]),
            'S_xy': float(s[3]), 'S_xz': float(s[4]), 'S_yz': float(s[5])}


@pytest.mark.gpu
@pytest.mark.parametrize('precision', ['fp64', 'mixed'])
def test_driver_matches_reference(tmp_path, driver, precision):
    g = golden('ref_p24')
    extra = ('do_save_solution = true\ndo_save_matrix = true\nfix_tip = %d\n'
             '[solid]\nShear_modulus = 1.0\nPoisson_ratio = 0.35\n'
             '[engine]\nprecision = "%s"\nfull_precision_output = true\n' % (int(g['tip']), precision))
    cfg = write_case(tmp_path, g['nods'], g['conn'], extra, pts=g['pts'], s_cfg=s_config(g['s_inf']))
    r = subprocess.run([driver, str(cfg)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    assert lines[0].startswith('Assembly: ') and lines[1] == '432 DoF Total'
    assert lines[2] == '%d Fixed DoF' % (432 - int(g['n_dof']))
    assert any(s.startswith('Solution: ') for s in lines)
    out = tmp_path / 'Out'
    A = np.loadtxt(out / 'test_assembly.csv', delimiter=',')
    assert np.abs(A - g['A']).max() / np.abs(g['A']).max() < 1e-11
    sol = np.loadtxt(out / 'test_solution.csv', delimiter=',')
    assert sol.shape == (144, 7) and (sol[:, 3] == 0).all()
    assert np.abs(sol[:, 4:] - g['dd']).max() / np.abs(g['dd']).max() < 1e-10
    # node coordinates: vertices, then the midpoint of the edge across each
    conn, nods = g['conn'][:3].astype(int), g['nods'][:3]
    v = nods[:, conn]                                    # 3 x 3 x Ne
    mid = 0.5 * (v[:, [1, 2, 0]] + v[:, [2, 0, 1]])
    want = np.concatenate([v, mid], axis=1).transpose(2, 1, 0).reshape(-1, 3)
    assert np.array_equal(sol[:, :3], want)
    st = np.loadtxt(out / 'test_stresses.csv', delimiter=',')
    assert np.abs(st - g['stress']).max() / np.abs(g['stress']).max() < 1e-9


@pytest.mark.gpu
def test_driver_default_output_precision(tmp_path, driver):
    # the reference writes csv with the stream's default 6 significant digits
    g = golden('ref_p24')
    extra = 'do_save_solution = true\nfix_tip = %d\nPoisson_ratio = 0.35\n' % int(g['tip'])
    cfg = write_case(tmp_path, g['nods'], g['conn'], extra, s_cfg=s_config(g['s_inf']))
    r = subprocess.run([driver, str(cfg)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    text = (tmp_path / 'Out' / 'test_solution.csv').read_text().splitlines()
    digits = [c.lstrip('-').split('e')[0].replace('.', '').lstrip('0') for line in text for c in line.split(',')]
    assert max(len(d) for d in digits) == 6
    sol = np.loadtxt(tmp_path / 'Out' / 'test_solution.csv', delimiter=',')
    assert np.abs(sol[:, 4:] - g['dd']).max() / np.abs(g['dd']).max() < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize('fmt,tol', [('npy64', 1e-10), ('npy32', 1e-6)])
def test_driver_npy_output(tmp_path, driver, fmt, tol):
    # npy32/npy64 outputs (left unwritten by the reference's driver); with
    # these formats the observation points are read as .npy, as there
    g = golden('ref_p24')
    extra = ('do_save_solution = true\ndo_postprocess = true\nobserv_crd_fname = "pts.npy"\n'
             'output_format = "%s"\nfix_tip = %d\nPoisson_ratio = 0.35\n' % (fmt, int(g['tip'])))
    cfg = write_case(tmp_path, g['nods'], g['conn'], extra, s_cfg=s_config(g['s_inf']))
    np.save(tmp_path / 'Mesh_Files' / 'pts.npy', np.asfortranarray(g['pts']))
    r = subprocess.run([driver, str(cfg)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert 'test_solution.npy' in r.stdout and 'test_stresses.npy' in r.stdout
    sol = np.load(tmp_path / 'Out' / 'test_solution.npy')
    assert sol.dtype == (np.float32 if fmt == 'npy32' else np.float64) and sol.shape == (144, 7)
    assert np.abs(sol[:, 4:] - g['dd']).max() / np.abs(g['dd']).max() < tol
    st = np.load(tmp_path / 'Out' / 'test_stresses.npy')
    assert np.abs(st - g['stress']).max() / np.abs(g['stress']).max() < max(tol, 1e-9)
