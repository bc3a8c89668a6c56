"""The volume-control iteration with cohesion and friction
(hfpx_vc_cf_iteration, hfpx_cf_match, hfpx_cf_update_mrd): the reference's
vc_cf_iteration (src/Development/c_f_iteration.cpp:27-436), match_f_c and
update_mrd (src/Development/cohesion_friction.cpp:22-194), against the loop
restatement oracle/cf_ref.py.

CPU (the oracle itself):
* match_f_c and update_mrd on hand-worked points of every model branch;
* one step on a small penny: the truncated system's kept rows, the volume
  row (the injected volume), zero increments at fixed DoF, the renumbered
  handle; the step visits every branch of the traction check;
* with the reference's sign the iteration grows; with the releasing sign it
  settles.
GPU, three steps each from the device's own state (a penny crack of 40
elements, tip-vertex DoF fixed, DD in local coordinates, two materials):
* every step against the oracle from the same state: the truncated handle
  and the fixed count exactly, DD, pressures, cohesion and friction within
  1e-9 of their scale, residual, volume and pressure increment;
* with the reference's right-hand side (components 0 and 1) on the full
  system's mixed factors, all three components on them, and all three with
  the releasing sign on the truncated system factored anew;
* update_mrd after the steps;
* bad arguments and a matrix holding FP64 factors fail with the engine's
  error."""
import os
import sys
from types import SimpleNamespace

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, 'oracle'))
G, NU, BETA = 1.0, 0.35, 0.125
MATS = [dict(cr_open=0.02, peak_ts=0.8, cr_slip=0.02, peak_sc=0.2, peak_sf=0.6, res_sf=0.3, cohesion_model=1,
             friction_model=1),
        dict(cr_open=0.03, peak_ts=1.2, cr_slip=0.03, peak_sc=0.1, peak_sf=0.5, res_sf=0.5, cohesion_model=0,
             friction_model=0)]
S_INF = np.array([-1.0, -0.9, -1.0, 0.05, 0.35, -0.2])


def point_positions(nods, conn):
    ne = conn.shape[1]
    pos = np.zeros((6 * ne, 3))
    for el in range(ne):
        v = nods[:3, conn[:3, el]]
        for a in range(3):
            pos[6 * el + a] = v[:, a]
            pos[6 * el + 3 + a] = 0.5 * (v[:, (a + 1) % 3] + v[:, (a + 2) % 3])
    return pos


def scenario(n_tri=40, seed=11):
    """A penny crack opened in its centre (Sneddon-like opening within r <
    0.7, fully opened within 0.35, partly within 0.6, earlier slip in a ring
    0.6-0.75), pressure 1.5 within 0.45, compressive in-situ stress with
    shear, two materials."""
    from hfpx3d_b200 import meshgen
    nods, conn = meshgen.penny(n_tri, seed=seed)
    ne = conn.shape[1]
    r = np.hypot(*point_positions(nods, conn)[:, :2].T)
    rng = np.random.default_rng(5)
    dd = np.zeros((6 * ne, 3))
    dd[:, 2] = 0.03 * np.sqrt(np.clip(1 - (r / 0.7) ** 2, 0, None))
    dd[:, 0] = 0.002 * rng.standard_normal(6 * ne) * (r < 0.8)
    dd[:, 1] = 0.002 * rng.standard_normal(6 * ne) * (r < 0.8)
    st = SimpleNamespace(dd=dd, pp=np.where(r < 0.45, 1.5, 0.0),
                         mr_open=np.where(r < 0.35, 1.0, np.where(r < 0.6, 0.5, 0.0)),
                         mr_slip=np.where((r > 0.6) & (r < 0.75), 0.3, 0.0),
                         mat_id=(rng.random(6 * ne) < 0.3).astype(np.int32))
    return nods, conn, st, int(np.argmin(r))


def dd_vector(dd, dof, n):
    x = np.zeros(n + 1)
    for el in range(dof.shape[0]):
        for l in range(18):
            if dof[el, l] >= 0:
                x[dof[el, l]] = dd[6 * el + l // 3, l % 3]
    return x


# ---------------------------------------------------------------- CPU: the oracle

def test_oracle_match_and_mrd_cases():
    import cf_ref
    box = dict(cr_open=0.1, peak_ts=2.0, cr_slip=0.2, peak_sc=1.0, peak_sf=0.8, res_sf=0.2, cohesion_model=0,
               friction_model=1)
    lin = dict(box, cohesion_model=1, friction_model=0)
    mats = [box, lin]
    # points: (dd, mr_open, mr_slip, material)
    pts = [((0, 0, 0.05), 0.0, 0.0, 0),    # box, half open: full cohesion
           ((0, 0, 0.05), 0.0, 0.0, 1),    # linear: half the peak
           ((0, 0, 0.05), 0.8, 0.0, 0),    # unloading from 0.8: scaled by 0.5 / 0.8
           ((0, 0, 0.15), 0.0, 0.0, 0),    # fully open: no cohesion, no friction
           ((0.1, 0, 0.0), 0.0, 0.75, 0),  # slip 0.5 below the reached 0.75: weakening by 0.75
           ((0.1, 0, 0.0), 0.0, 0.25, 0),  # slip 0.5 above the reached 0.25
           ((0.3, 0, 0.0), 0.0, 0.0, 0),   # slip past critical: residual friction
           ((0.3, 0, 0.0), 0.0, 0.0, 1)]   # constant friction: the peak
    dd = np.array([p[0] for p in pts], dtype=float)
    mo = np.array([p[1] for p in pts])
    ms = np.array([p[2] for p in pts])
    mid = np.array([p[3] for p in pts])
    fric, sc, oc = cf_ref.match_f_c(mats, mid, dd, mo, ms)
    np.testing.assert_allclose(oc, [2.0, 1.0, 2.0 * 0.5 / 0.8, 0, 0, 0, 0, 0], rtol=1e-15)
    np.testing.assert_allclose(sc, oc / 2.0, rtol=1e-15)
    np.testing.assert_allclose(fric, [0.8, 0.8, 0.8, 0.0, 0.2 + 0.6 * 0.25,
                                      0.2 + 0.6 * 0.5, 0.2, 0.8], rtol=1e-15)
    mo2, ms2 = cf_ref.update_mrd(mats, mid, dd, mo, ms)
    np.testing.assert_allclose(mo2, [0.5, 0.5, 0.8, 1.5, 0, 0, 0, 0], rtol=1e-15)
    np.testing.assert_allclose(ms2, [0, 0, 0, 0, 0.75, 0.5, 1.5, 1.5], rtol=1e-15)


@pytest.mark.parametrize('is_dd_local', [True, False])
def test_oracle_step_properties(ora, is_dd_local):
    import cf_ref
    nods, conn, st, inj = scenario(24, seed=3)
    dof, n = ora.dof_handle(nods, conn, 1)
    A = ora.assemble(nods, conn, dof, n, G, NU, BETA, is_dd_local=int(is_dd_local), vc=1)
    elems = cf_ref.element_data(ora, nods, conn, BETA)
    vol = A[n] @ dd_vector(st.dd, dof, n)
    new, info = cf_ref.vc_cf_iteration(elems, A, dof, MATS, st, S_INF, inj, 1.1 * vol, is_dd_local=is_dd_local,
                                       all_components=True)
    assert all(v > 0 for v in info['counts'].values()), info['counts']
    assert abs(info['volume'] - vol) <= 1e-15 * abs(vol)
    td = new.dof_h
    kept = td >= 0
    # the truncated numbering is 0 .. n_dof - 1, in the original order
    assert np.array_equal(np.sort(td[kept]), np.arange(new.n_dof))
    assert new.n_dof == n - info['n_fixed']
    order = np.argsort(dof[kept])
    assert np.all(np.diff(td[kept][order]) > 0)
    # kept rows of the truncated system, volume row: the injected volume
    incr = info['increments']
    x = np.zeros(n + 1)
    x[dof[kept]] = incr[td[kept]]
    x[n] = incr[-1]
    rows = dof[kept]
    res = A[rows] @ x - info['delta_trac'][rows]
    assert np.abs(res).max() <= 1e-10 * np.abs(A).max() * np.abs(x).max()
    assert abs(A[n] @ x - 0.1 * vol) <= 1e-12 * vol
    # fixed DoF keep their DD unless the clamp acts on the opening (in
    # global DD the round trip through the element frame may move the last bit,
    # and a clamped opening moves every global component)
    if is_dd_local:
        fixed = (dof >= 0) & ~kept
        for el, l in zip(*np.nonzero(fixed)):
            if l % 3 != 2:
                assert new.dd[6 * el + l // 3, l % 3] == st.dd[6 * el + l // 3, l % 3]


def test_oracle_sign_of_the_adjustments(ora):
    """The reference's sign doubles the excess traction (the residual
    grows); the opposite sign removes it (the residual falls)."""
    import cf_ref
    nods, conn, st0, inj = scenario(24, seed=3)
    dof, n = ora.dof_handle(nods, conn, 1)
    A = ora.assemble(nods, conn, dof, n, G, NU, BETA, is_dd_local=1, vc=1)
    elems = cf_ref.element_data(ora, nods, conn, BETA)
    vol = A[n] @ dd_vector(st0.dd, dof, n)
    res = {}
    for release in (False, True):
        st = st0
        r = []
        for _ in range(5):
            new, info = cf_ref.vc_cf_iteration(elems, A, dof, MATS, st, S_INF, inj, 1.1 * vol, is_dd_local=True,
                                               all_components=True, release_sign=release)
            r.append(info['residual'])
            st = SimpleNamespace(dd=new.dd, pp=new.pp, mr_open=st0.mr_open, mr_slip=st0.mr_slip,
                                 mat_id=st0.mat_id)
        res[release] = r
    print('residuals, reference sign:', ['%.3g' % v for v in res[False]],
          'releasing sign:', ['%.3g' % v for v in res[True]])
    assert res[False][-1] > 2 * res[False][0]
    assert res[True][-1] < 0.2 * res[True][0]


# ---------------------------------------------------------------- GPU

@pytest.fixture(scope='module')
def cf_case(ctx, ora):
    import cf_ref
    from hfpx3d_b200 import engine
    nods, conn, st, inj = scenario()
    mesh = engine.MeshGeom(nods, conn)
    dof, n = engine.make_dof_h_crack(mesh, 1)
    dm = engine.DeviceMesh(ctx, mesh, BETA)
    elems = cf_ref.element_data(ora, nods, conn, BETA)
    return dict(nods=nods, conn=conn, st=st, inj=inj, dof=dof, n=n, dm=dm, elems=elems)


@pytest.mark.gpu
def test_match_and_mrd_vs_oracle(ctx, cf_case):
    import cf_ref
    from hfpx3d_b200 import engine
    rng = np.random.default_rng(2)
    ne = cf_case['conn'].shape[1]
    st = engine.CfState(ne, dd=rng.uniform(-0.03, 0.05, (6 * ne, 3)), mr_open=rng.uniform(0, 1.3, 6 * ne),
                        mr_slip=rng.uniform(0, 1.3, 6 * ne), mat_id=rng.integers(0, 2, 6 * ne))
    engine.match_f_c(ctx, MATS, st)
    fric, sc, oc = cf_ref.match_f_c(MATS, st.mat_id, st.dd, st.mr_open, st.mr_slip)
    np.testing.assert_allclose(st.friction_coef, fric, rtol=1e-14, atol=1e-16)
    np.testing.assert_allclose(st.slip_cohesion, sc, rtol=1e-14, atol=1e-16)
    np.testing.assert_allclose(st.open_cohesion, oc, rtol=1e-14, atol=1e-16)
    mo, ms = cf_ref.update_mrd(MATS, st.mat_id, st.dd, st.mr_open, st.mr_slip)
    engine.update_mrd(ctx, MATS, st)
    np.testing.assert_allclose(st.mr_open, mo, rtol=1e-14)
    np.testing.assert_allclose(st.mr_slip, ms, rtol=1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize('all_components,release,factored', [(False, False, True), (True, False, True),
                                                              (True, True, False)])
def test_iteration_vs_oracle(ctx, cf_case, all_components, release, factored):
    import cf_ref
    from hfpx3d_b200 import engine
    c = cf_case
    dof, n, dm, st0, inj = c['dof'], c['n'], c['dm'], c['st'], c['inj']
    A = engine.assemble(ctx, dm, dof, n, G, NU, is_dd_local=True, vc=True)
    Ah = A.download()
    lu = engine.LU(ctx, A, engine.HFPX_LU_MIXED) if factored else None
    ne = c['conn'].shape[1]
    gs = engine.CfState(ne, dd=st0.dd, pp=st0.pp, mr_open=st0.mr_open, mr_slip=st0.mr_slip, mat_id=st0.mat_id)
    vol = Ah[n] @ dd_vector(st0.dd, dof, n)
    for step in range(3):
        pre = SimpleNamespace(dd=gs.dd.copy(), pp=gs.pp.copy(), mr_open=gs.mr_open, mr_slip=gs.mr_slip,
                              mat_id=gs.mat_id)
        info = engine.vc_cf_iteration(ctx, dm, A, dof, n, MATS, gs, S_INF, inj, 1.1 * vol, is_dd_local=True,
                                      all_components=all_components, release_sign=release, reuse_factors=factored)
        new, oi = cf_ref.vc_cf_iteration(c['elems'], Ah, dof, MATS, pre, S_INF, inj, 1.1 * vol, is_dd_local=True,
                                         all_components=all_components, release_sign=release)
        if step == 0:
            assert all(v > 0 for k, v in oi['counts'].items() if k != 'cohesion'), oi['counts']
        assert info.solver == (0 if factored else 1)
        assert info.n_fixed == oi['n_fixed'] and info.n_dof == new.n_dof == gs.n_dof
        assert np.array_equal(gs.dof_h, new.dof_h)
        ddscale = np.abs(new.dd).max()
        errs = dict(dd=np.abs(gs.dd - new.dd).max() / ddscale,
                    pp=np.abs(gs.pp - new.pp).max() / np.abs(new.pp).max(),
                    coh=max(np.abs(gs.open_cohesion - new.open_cohesion).max(),
                            np.abs(gs.slip_cohesion - new.slip_cohesion).max(),
                            np.abs(gs.friction_coef - new.friction_coef).max()),
                    residual=abs(info.residual - oi['residual']) / oi['residual'],
                    volume=abs(info.volume - oi['volume']) / abs(oi['volume']),
                    delta_p=abs(info.delta_p - oi['delta_p']) / max(abs(oi['pressure']), 1.0))
        print(f'step {step} (components {3 if all_components else 2}, release {release}, '
              f'{"full factors" if factored else "truncated system"}): fixed {info.n_fixed}, '
              f'residual {info.residual:.4g}, ' + ', '.join(f'{k} {v:.1e}' for k, v in errs.items()))
        assert errs['dd'] <= 1e-9 and errs['pp'] <= 1e-9 and errs['coh'] <= 1e-12
        assert errs['residual'] <= 1e-9 and errs['volume'] <= 1e-12 and errs['delta_p'] <= 1e-9
    mo, ms = cf_ref.update_mrd(MATS, gs.mat_id, gs.dd, gs.mr_open, gs.mr_slip)
    engine.update_mrd(ctx, MATS, gs)
    np.testing.assert_allclose(gs.mr_open, mo, rtol=1e-14)
    np.testing.assert_allclose(gs.mr_slip, ms, rtol=1e-14)
    del lu
    A.close()


@pytest.mark.gpu
def test_iteration_errors(ctx, cf_case):
    from hfpx3d_b200 import engine
    c = cf_case
    dof, n, dm, st0, inj = c['dof'], c['n'], c['dm'], c['st'], c['inj']
    ne = c['conn'].shape[1]
    A = engine.assemble(ctx, dm, dof, n, G, NU, is_dd_local=True, vc=True)
    gs = engine.CfState(ne, dd=st0.dd, pp=st0.pp, mr_open=st0.mr_open, mr_slip=st0.mr_slip, mat_id=st0.mat_id)
    bad = gs.copy()
    bad.mat_id[3] = 7
    with pytest.raises(engine.EngineError) as e:
        engine.vc_cf_iteration(ctx, dm, A, dof, n, MATS, bad, S_INF, inj, 0.1, is_dd_local=True)
    assert e.value.code == engine.HFPX_ERR_ARG
    with pytest.raises(engine.EngineError) as e:
        engine.vc_cf_iteration(ctx, dm, A, dof, n, MATS, gs, S_INF, 6 * ne, 0.1, is_dd_local=True)
    assert e.value.code == engine.HFPX_ERR_ARG
    with pytest.raises(engine.EngineError) as e:
        engine.vc_cf_iteration(ctx, dm, A, dof, n - 1, MATS, gs, S_INF, inj, 0.1, is_dd_local=True)
    assert e.value.code == engine.HFPX_ERR_ARG
    zero = [dict(MATS[0], cr_open=0.0), MATS[1]]
    with pytest.raises(engine.EngineError) as e:
        engine.match_f_c(ctx, zero, gs)
    assert e.value.code == engine.HFPX_ERR_ARG
    lu = engine.LU(ctx, A, engine.HFPX_LU_FP64)   # FP64 factors replace the operator
    with pytest.raises(engine.EngineError) as e:
        engine.vc_cf_iteration(ctx, dm, A, dof, n, MATS, gs, S_INF, inj, 0.1, is_dd_local=True)
    assert e.value.code == engine.HFPX_ERR_STATE
    assert np.array_equal(gs.dd, st0.dd)
    del lu
    A.close()


@pytest.mark.gpu
def test_cpp_host_layer_matches_python(ctx, cf_case, tmp_path):
    """hfpx::vc_cf_iteration / hfpx::update_mrd (the C++ host layer,
    hfpx3d_b200/host) against the Python mirror on the same case, two steps
    with all components and the releasing sign: both call the same C-ABI
    (each its own mixed factorisation, refined to 1e-12)."""
    import subprocess
    from hfpx3d_b200 import build, engine
    c = cf_case
    nods, conn, st0, inj = c['nods'], c['conn'], c['st'], c['inj']
    dof, n, dm = c['dof'], c['n'], c['dm']
    ne = conn.shape[1]
    exe = str(tmp_path / 'host_cf_main')
    subprocess.run(['g++', '-O2', '-std=c++17', '-I' + os.path.join(ROOT, 'include'), '-I' + build.HOST,
                    os.path.join(ROOT, 'tests', 'host_cf_main.cpp'), '-o', exe, '-L' + build.HERE, '-lhfpx_host',
                    '-lhfpx_engine', '-Wl,-rpath,' + build.HERE], check=True, timeout=300)
    A = engine.assemble(ctx, dm, dof, n, G, NU, is_dd_local=True, vc=True)
    vol = 1.1 * float(A.block(n, 0, 1, n + 1)[0] @ dd_vector(st0.dd, dof, n))
    keys = ['cr_open', 'peak_ts', 'cr_slip', 'peak_sc', 'peak_sf', 'res_sf', 'cohesion_model', 'friction_model']
    np.save(tmp_path / 'mats.npy', np.array([[float(m[k]) for k in keys] for m in MATS]))
    np.save(tmp_path / 'params.npy', np.concatenate([S_INF, [inj // 6, inj % 6, vol]])[:, None])
    np.save(tmp_path / 'nods.npy', np.asfortranarray(nods, dtype=np.float64))
    np.save(tmp_path / 'conn.npy', np.asfortranarray(conn, dtype=np.int64))
    np.save(tmp_path / 'dd.npy', np.asfortranarray(st0.dd))
    for k in ('pp', 'mr_open', 'mr_slip'):
        np.save(tmp_path / f'{k}.npy', np.asarray(getattr(st0, k), dtype=np.float64)[:, None])
    np.save(tmp_path / 'mat_id.npy', np.asarray(st0.mat_id, dtype=np.int64)[:, None])
    flags = 3
    r = subprocess.run([exe, str(tmp_path), '2', str(flags)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lu = engine.LU(ctx, A, engine.HFPX_LU_MIXED)
    gs = engine.CfState(ne, dd=st0.dd, pp=st0.pp, mr_open=st0.mr_open, mr_slip=st0.mr_slip, mat_id=st0.mat_id)
    for _ in range(2):
        info = engine.vc_cf_iteration(ctx, dm, A, dof, n, MATS, gs, S_INF, inj, vol, is_dd_local=True,
                                      all_components=True, release_sign=True)
    engine.update_mrd(ctx, MATS, gs)
    out_pp = np.load(tmp_path / 'out_pp.npy')
    res = np.load(tmp_path / 'out_res.npy')
    out_dd = np.load(tmp_path / 'out_dd.npy')
    assert np.abs(out_dd - gs.dd).max() <= 1e-12 * np.abs(gs.dd).max()
    assert np.abs(out_pp[:, 0] - gs.pp).max() <= 1e-12 * np.abs(gs.pp).max()
    np.testing.assert_allclose(out_pp[:, 1], gs.mr_open, rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(out_pp[:, 2], gs.mr_slip, rtol=1e-10, atol=1e-14)
    assert np.array_equal(np.load(tmp_path / 'out_dof.npy').astype(np.int64), gs.dof_h)
    assert abs(res[0, 0] - info.residual) <= 1e-10 * info.residual and int(res[0, 1]) == info.n_dof
    del lu
    A.close()
