"""The CPU oracle against the reference-pinned fixtures of the two large
configurations (tests/golden/ref_c2.npz, ref_c3.npz, made from oracle/_ref
by tests/golden/make_configs.py): rows of sampled elements of the 1025-element
VC ellipse and of the 4000-element penny, the right-hand side exactly, and
the mesh generator's output by checksum.  The same fixtures pin the GPU path
(tests/test_gpu_configs.py); tolerances are explained there."""
import hashlib
import os
import sys

import numpy as np

from conftest import golden

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden'))
G, NU = 1.0, 0.35


def digest(nods, conn):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(nods, dtype=np.float64).tobytes())
    h.update(np.ascontiguousarray(conn, dtype=np.int64).tobytes())
    return h.hexdigest()


def test_c3_oracle_rows(ora):
    from hfpx3d_b200 import meshgen
    z = golden('ref_c3')
    nods, conn = meshgen.penny(4000, seed=2026)
    assert digest(nods, conn) == str(z['mesh_digest'])
    dof, n = ora.dof_handle(nods, conn, 0)
    W = np.random.default_rng(int(z['w_seed'])).uniform(-1.0, 1.0, (n, 3))
    rows = []
    for t in z['elems']:
        lo, buf = ora.assemble_rows(nods, conn, dof, n, int(t), int(t) + 1)
        assert lo == 18 * int(t)
        rows.append(buf)
    rows = np.concatenate(rows)
    e_rows = float((np.abs(rows @ W - z['row_w']) / z['row_abs']).max())
    e_samp = np.abs(rows[z['row_si'], z['row_sj']] - z['row_sv']).max() / np.abs(rows).max()
    near = np.stack([np.stack([rows[18 * i:18 * i + 18, 18 * s:18 * s + 18] for s in z['near'][i]])
                     for i in range(len(z['elems']))])
    e_near = np.abs(near - z['near_blocks']).max() / np.abs(z['near_blocks']).max()
    print(f'oracle C3 rows vs reference: weighted {e_rows:.1e}, samples {e_samp:.1e}, near blocks {e_near:.1e}')
    assert e_rows <= 1e-10 and e_samp <= 1e-10 and e_near <= 1e-12


def test_c2_oracle_rows_and_rhs(ora):
    from hfpx3d_b200 import meshgen
    z = golden('ref_c2')
    nods, conn = meshgen.ellipse(1025, seed=1025)
    assert digest(nods, conn) == str(z['mesh_digest'])
    dof, n = ora.dof_handle(nods, conn, 0)
    rhs = np.concatenate([ora.rhs(nods, conn, dof, n, z['s_inf']), [1.0]])
    assert np.array_equal(rhs, z['rhs'])
    w = np.random.default_rng(int(z['w_seed'])).uniform(-1.0, 1.0, (n + 1, 1))[:, 0]
    # element 767 holds the largest closed-form disagreement with the reference
    for t in (0, 300, 767, 1024):
        lo, buf = ora.assemble_rows(nods, conn, dof, n, t, t + 1)
        r = slice(lo, lo + 18)
        # the border column is -e3 of the row's element (the reference's, exactly)
        aw = buf @ w[:n] + z['vc_col'][r] * w[n]
        e = float((np.abs(aw - z['Aw'][r]) / z['abs_Aw'][r]).max())
        assert e <= 2e-9, (t, e)
