"""The C-ABI library builds, loads and exports every function include/hfpx_engine.h
declares; host-only entry points run without a GPU."""
import ctypes
import os
import re

import numpy as np

from conftest import ROOT, golden


def header_functions():
    txt = open(os.path.join(ROOT, 'include', 'hfpx_engine.h')).read()
    txt = re.sub(r'/\*.*?\*/', '', txt, flags=re.S)
    return sorted(set(re.findall(r'\b(hfpx_[a-z0-9_]+)\s*\(', txt)))


def test_exports_every_declared_symbol():
    from hfpx3d_b200 import build, engine
    build.build()
    lib = ctypes.CDLL(engine.LIB_PATH)
    names = header_functions()
    assert len(names) >= 18
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(engine.SIGNATURES), set(names) ^ set(engine.SIGNATURES)


def test_host_dof_handle_matches_reference():
    from hfpx3d_b200 import engine
    g = golden('ref_dof')
    for name in ('p24', 'p121'):
        mesh = engine.MeshGeom(g[name + '_nods'], g[name + '_conn'])
        for tip in (0, 1, 2):
            d, n = engine.make_dof_h_crack(mesh, tip)
            assert n == int(g[f'{name}_tip{tip}_n'])
            assert (d == g[f'{name}_tip{tip}']).all()


def test_host_element_frame_matches_oracle(ora):
    from hfpx3d_b200 import engine
    g = golden('ref_kernel_points')
    r, tau, sfm = engine.element_frame(g['vert'])
    np.testing.assert_array_equal(r, g['r'])
    np.testing.assert_allclose(tau, g['tau'][0::2] + 1j * g['tau'][1::2], rtol=0, atol=1e-15)
    np.testing.assert_allclose(sfm.reshape(-1), g['sfm'][0::2] + 1j * g['sfm'][1::2], rtol=0, atol=1e-13)


def test_bad_arguments_are_rejected():
    from hfpx3d_b200 import engine
    L = engine.lib()
    nods = np.zeros((3, 2), order='F')
    conn = np.zeros((3, 1), dtype=np.int64, order='F')
    dof = np.zeros((1, 18), dtype=np.int64, order='F')
    n = L.hfpx_dof_handle(engine._dp(nods), 3, 2, engine._lp(conn), 3, 1, 0, engine._lp(dof))
    assert n == -engine.HFPX_ERR_ARG
    assert L.hfpx_element_frame(None, None, None, None) == engine.HFPX_ERR_ARG
    h = ctypes.c_void_p()
    rc = L.hfpx_ctx_create(-1, ctypes.byref(h))
    assert rc != engine.HFPX_OK and not h.value
