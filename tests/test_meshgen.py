from collections import Counter

import numpy as np
import pytest

from hfpx3d_b200 import meshgen


@pytest.mark.parametrize('n', [3, 24, 121, 1025, 4000])
def test_penny_counts_and_topology(n):
    nods, conn = meshgen.penny(n, seed=1)
    assert conn.shape == (5, n) and nods.shape[0] == 6
    p, c = nods[:2], conn[:3]
    a1, a2 = p[:, c[1]] - p[:, c[0]], p[:, c[2]] - p[:, c[0]]
    area = 0.5 * (a1[0] * a2[1] - a1[1] * a2[0])
    assert (area > 0).all()
    edges = Counter()
    for e in c.T:
        for i in range(3):
            edges[tuple(sorted((e[i], e[(i + 1) % 3])))] += 1
    assert set(edges.values()) <= {1, 2}
    tips = nods[4] == 1
    assert np.allclose(np.hypot(nods[0, tips], nods[1, tips]), 1.0)
    assert (np.hypot(nods[0, ~tips], nods[1, ~tips]) < 1.0).all()


def test_seeded_reproducible():
    a = meshgen.penny(121, seed=5)
    b = meshgen.penny(121, seed=5)
    assert all((x == y).all() for x, y in zip(a, b))
    c = meshgen.penny(121, seed=6)
    assert not np.array_equal(a[0], c[0])


def test_ellipse_and_wavy():
    nods, conn = meshgen.ellipse(1025, 2.0, 1.0, seed=3)
    tips = nods[4] == 1
    assert conn.shape[1] == 1025
    assert np.allclose((nods[0, tips] / 2.0) ** 2 + nods[1, tips] ** 2, 1.0)
    nw, cw = meshgen.wavy(200, aspect=2.0, amp=0.2, k=np.pi, seed=3)
    assert np.abs(nw[2]).max() > 0.1


def test_batch_workload_is_seeded_and_uneven():
    from hfpx3d_b200 import meshgen
    m1, S1 = meshgen.batch_workload(16, 8, seed=5)
    m2, S2 = meshgen.batch_workload(16, 8, seed=5)
    assert len(m1) == 16 and S1.shape == (16, 6, 8)
    assert all(np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) for a, b in zip(m1, m2))
    assert np.array_equal(S1, S2)
    sizes = [c.shape[1] for _, c in m1]
    assert min(sizes) >= 24 and max(sizes) <= 550 and len(set(sizes)) > 8
    # even cases: uniform pressure in [0.5, 2] (sigma_zz only); odd: in-situ
    # stress tensors with principal values in [-1, 0]
    assert np.all((S1[:, 2, 0::2] >= 0.5) & (S1[:, 2, 0::2] <= 2.0))
    assert np.all(S1[:, [0, 1, 3, 4, 5]][:, :, 0::2] == 0.0)
    for m in range(16):
        s = S1[m, :, 1]
        T = np.array([[s[0], s[3], s[4]], [s[3], s[1], s[5]], [s[4], s[5], s[2]]])
        ev = np.linalg.eigvalsh(T)
        assert np.all(ev >= -1 - 1e-12) and np.all(ev <= 1e-12)


def test_batch_tile_table_is_read():
    from hfpx3d_b200 import engine
    nb, leaf = engine.batch_tiles()
    assert nb % 32 == 0 and leaf in (256, 512)
