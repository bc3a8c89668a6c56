"""Seeded crack meshes of 3-node triangles in the reference's file layout.

The reference ships no mesher (its meshes come from MATLAB .mat files,
Mesh_Files/).  This one builds concentric-ring triangulations of the unit
disk with an exact element count, optional in-plane node jitter, and maps
them to ellipses or wavy (non-planar) surfaces.

Layout (same as Mesh_Files/*_32.npy, read by load_mesh_from_numpy_32,
src/IO/mesh_file_io.cpp:186-226): nods 6 x Nn float64 (rows x, y, z, 1,
tip flag, 0), conn 5 x Ne (rows: 3 vertex indices, 1, 1); counter-clockwise
elements (normal +z); boundary nodes carry tip flag 1.
"""
from __future__ import annotations

import numpy as np


def _ring_counts(n_tri: int):
    """Node counts n_1..n_K of K rings with 2*sum(n) - n_K == n_tri."""
    if n_tri < 3:
        raise ValueError('need at least 3 triangles')
    K = max(1, int(round(np.sqrt(n_tri / 6.0))))
    while True:
        if K == 1:
            return [n_tri]
        nK = max(3, int(round(n_tri / (2.0 * K - 1.0) * (2.0 * K) / (K + 1.0))))
        if (n_tri + nK) % 2:
            nK += 1
        S = (n_tri + nK) // 2
        rest = S - nK
        w = np.arange(1, K, dtype=np.float64)
        target = rest * w / w.sum()
        counts = np.floor(target).astype(int)
        left = rest - counts.sum()
        order = np.argsort(-(target - counts), kind='stable')
        counts[order[:left]] += 1
        counts = list(counts) + [nK]
        if min(counts) >= 3 and all(counts[i] <= counts[i + 1] for i in range(len(counts) - 1)):
            return counts
        K -= 1


def penny(n_tri: int, seed: int | None = 0, jitter: float = 0.05, radius: float = 1.0):
    """Unit-disk crack (scaled by radius) with exactly n_tri triangles.

    jitter: in-plane node displacement bound as a fraction of the ring
    spacing (interior nodes); boundary nodes move only along the circle.
    Returns (nods 6 x Nn, conn 5 x Ne), both Fortran-ordered."""
    counts = _ring_counts(n_tri)
    K = len(counts)
    rng = np.random.default_rng(seed) if seed is not None else None
    xs, ys, tip, rings = [0.0], [0.0], [0.0], [[0]]
    for k, n in enumerate(counts, start=1):
        r = k / K
        off = 0.5 * (k % 2) * 2 * np.pi / n
        ids = []
        for i in range(n):
            th = off + 2 * np.pi * i / n
            ids.append(len(xs))
            xs.append(r * np.cos(th))
            ys.append(r * np.sin(th))
            tip.append(1.0 if k == K else 0.0)
        rings.append(ids)
    xs, ys = np.array(xs), np.array(ys)
    ang = np.arctan2(ys, xs)
    tris = []
    # fan around the centre
    r1 = rings[1]
    for i in range(len(r1)):
        tris.append((0, r1[i], r1[(i + 1) % len(r1)]))
    # zipper between consecutive rings, by angle
    for k in range(1, K):
        a, b = rings[k], rings[k + 1]
        ta = np.mod(ang[a] - ang[a[0]], 2 * np.pi)
        tb = np.mod(ang[b] - ang[a[0]], 2 * np.pi)
        ib = int(np.argmin(tb))
        b = b[ib:] + b[:ib]
        tb = np.mod(ang[b] - ang[a[0]], 2 * np.pi)
        i = j = 0
        na, nb = len(a), len(b)
        while i < na or j < nb:
            ta_next = ta[i + 1] if i + 1 < na else 2 * np.pi + ta[0]
            tb_next = tb[j + 1] if j + 1 < nb else 2 * np.pi + tb[0]
            ca, cb = a[i % na], b[j % nb]
            if (j >= nb) or (i < na and ta_next <= tb_next):
                tris.append((ca, cb, a[(i + 1) % na]))
                i += 1
            else:
                tris.append((ca, cb, b[(j + 1) % nb]))
                j += 1
    conn = np.array(tris, dtype=np.int64).T
    # orient counter-clockwise
    p = np.stack([xs, ys])
    a1 = p[:, conn[1]] - p[:, conn[0]]
    a2 = p[:, conn[2]] - p[:, conn[0]]
    flip = (a1[0] * a2[1] - a1[1] * a2[0]) < 0
    c1 = conn[1].copy()
    conn[1, flip] = conn[2, flip]
    conn[2, flip] = c1[flip]
    if rng is not None and jitter > 0:
        h = 1.0 / K
        n_int = len(xs)
        interior = np.array(tip) == 0
        interior[0] = True
        rad = jitter * h * np.sqrt(rng.uniform(0, 1, n_int))
        phi = rng.uniform(0, 2 * np.pi, n_int)
        dth = rng.uniform(-1, 1, n_int) * jitter * 2 * np.pi / counts[-1]
        for i in range(n_int):
            if interior[i]:
                xs[i] += rad[i] * np.cos(phi[i])
                ys[i] += rad[i] * np.sin(phi[i])
            else:
                th = np.arctan2(ys[i], xs[i]) + dth[i]
                xs[i], ys[i] = np.cos(th), np.sin(th)
    nods = np.zeros((6, len(xs)), order='F')
    nods[0], nods[1] = radius * xs, radius * ys
    nods[3] = 1.0
    nods[4] = tip
    conn5 = np.ones((5, conn.shape[1]), dtype=np.int64, order='F')
    conn5[:3] = conn
    assert conn5.shape[1] == n_tri, (conn5.shape, n_tri)
    return nods, conn5


def ellipse(n_tri: int, a: float = 2.0, b: float = 1.0, seed: int | None = 0, jitter: float = 0.05):
    """Planar elliptical crack with semi-axes a (x) and b (y)."""
    nods, conn = penny(n_tri, seed, jitter)
    nods[0] *= a
    nods[1] *= b
    return nods, conn


def wavy(n_tri: int, aspect: float = 1.0, amp: float = 0.1, k: float = np.pi, phase: float = 0.0,
         seed: int | None = 0, jitter: float = 0.05):
    """Non-planar crack z = amp * sin(k x + phase) over an ellipse (aspect:1)."""
    nods, conn = penny(n_tri, seed, jitter)
    nods[0] *= aspect
    nods[2] = amp * np.sin(k * nods[0] + phase)
    return nods, conn


def observation_points(n: int, seed: int, box: float = 1.5, nods=None, conn=None, r_tol: float | None = None):
    """n seeded points uniform in [-box, box]^3 (3 x n, Fortran order), rejecting
    points closer than r_tol to any mesh vertex as the reference's
    postprocessing test does (test_radial_crack_static.cpp:237-269)."""
    rng = np.random.default_rng(seed)
    pts = []
    verts = None if nods is None else np.asarray(nods)[:3].T
    if r_tol is None and conn is not None:
        r_tol = 0.2 * np.sqrt(np.pi / conn.shape[1] / np.sqrt(3.0))
    while len(pts) < n:
        p = rng.uniform(-box, box, 3)
        if verts is not None and np.min(np.linalg.norm(verts - p, axis=1)) < r_tol:
            continue
        pts.append(p)
    return np.asfortranarray(np.array(pts).T)


def in_situ_stress(rng, lo: float = -1.0, hi: float = 0.0):
    """A random in-situ stress tensor (Voigt xx, yy, zz, xy, xz, yz): principal
    values uniform in [lo, hi], Haar-random principal axes."""
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))
    s = q @ np.diag(rng.uniform(lo, hi, 3)) @ q.T
    return np.array([s[0, 0], s[1, 1], s[2, 2], s[0, 1], s[0, 2], s[1, 2]])


def batch_workload(n_mesh: int = 256, n_cases: int = 64, seed: int = 2027, el_min: int = 24, el_max: int = 550):
    """The batched workload: n_mesh seeded penny or 2:1 elliptical cracks of
    uneven sizes (elements uniform in [el_min, el_max]), each with n_cases
    load cases: uniform pressures in [0.5, 2] (sigma_zz, even cases) and random
    in-situ stress tensors (odd cases).  Returns ([(nods, conn)], S) with S
    of shape (n_mesh, 6, n_cases)."""
    rng = np.random.default_rng(seed)
    meshes = []
    S = np.zeros((n_mesh, 6, n_cases))
    for m in range(n_mesh):
        ne = int(rng.integers(el_min, el_max + 1))
        if rng.random() < 0.5:
            meshes.append(penny(ne, seed=seed + 1 + m))
        else:
            meshes.append(ellipse(ne, seed=seed + 1 + m))
        for j in range(n_cases):
            if j % 2 == 0:
                S[m, 2, j] = rng.uniform(0.5, 2.0)
            else:
                S[m, :, j] = in_situ_stress(rng)
    return meshes, S
