"""Host side of the volume-control truncation (mod_3dbem_system_vc,
src/Solvers/system_assembly.cpp:560-629): the truncated-to-original DoF map
and the right-hand-side gather of hfpx3d_b200.engine, against the loop
restatement oracle/vc_ref.py; and that restatement against a numpy index
gather of the bordered matrix.  CPU only."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, 'oracle'))


def handles(n_el, seed, frac=0.25):
    rng = np.random.default_rng(seed)
    orig = np.arange(n_el * 18, dtype=np.int64).reshape(n_el, 18)
    drop = rng.random((n_el, 18)) < frac
    import vc_ref
    return orig, vc_ref.truncate_handle(orig, drop), drop


def test_truncation_map_and_restatement():
    import vc_ref
    from hfpx3d_b200 import engine
    orig, td, drop = handles(5, 1)
    keep = engine.vc_truncation_map(orig, td)
    assert np.array_equal(keep, orig.reshape(-1)[~drop.reshape(-1)])
    n = orig.size
    rng = np.random.default_rng(2)
    A = rng.standard_normal((n + 1, n + 1))
    A[n, n] = 0.0
    dv = 0.25
    for size in (orig.size, n, keep.size):  # full == original here: both read the same way
        dt = rng.standard_normal(size)
        M, r = vc_ref.mod_3dbem_system_vc(A, orig, td, dt, dv)
        idx = np.append(keep, n)
        want = A[np.ix_(idx, idx)].copy()
        want[-1, -1] = 0.0  # the reference never writes the corner
        assert np.array_equal(M, want)
        assert np.array_equal(engine.vc_rhs(orig, td, dt, dv, n), r)


def test_rhs_by_original_numbering_with_fixed_dof():
    """An original handle with fixed DoF (-1), so that the full element-node
    numbering and the original DoF numbering differ in length."""
    import vc_ref
    from hfpx3d_b200 import engine
    n_el = 4
    orig = np.full((n_el, 18), -1, dtype=np.int64)
    rng = np.random.default_rng(3)
    free = rng.random((n_el, 18)) > 0.2
    orig[free] = np.arange(int(free.sum()))
    n = int(free.sum())
    drop = rng.random((n_el, 18)) < 0.3
    td = vc_ref.truncate_handle(orig, drop)
    A = rng.standard_normal((n + 1, n + 1))
    for size in (n_el * 18, n, int(td.max()) + 1):
        dt = rng.standard_normal(size)
        M, r = vc_ref.mod_3dbem_system_vc(A, orig, td, dt, -1.5)
        assert np.array_equal(engine.vc_rhs(orig, td, dt, -1.5, n), r)
        keep = engine.vc_truncation_map(orig, td)
        idx = np.append(keep, n)
        want = A[np.ix_(idx, idx)].copy()
        want[-1, -1] = 0.0
        assert np.array_equal(M, want)


def test_bad_handles_and_sizes():
    from hfpx3d_b200 import engine
    orig, td, _ = handles(3, 4)
    bad = td.copy()
    k = np.argwhere(bad >= 0)
    bad[tuple(k[1])] = bad[tuple(k[0])]
    with pytest.raises(ValueError):
        engine.vc_truncation_map(orig, bad)
    with pytest.raises(ValueError):
        engine.vc_rhs(orig, td, np.zeros(7), 0.0, orig.size)
