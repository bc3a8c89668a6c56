"""The CPU restatement of the learned preconditioner's network
(oracle/gnn_ref.py) checked on its own: its backward pass against central
finite differences of its forward pass (FP64, BF16 rounding switched off),
on a small random graph.  The GPU kernels are then checked against it
(tests/test_gpu_gnn.py)."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'oracle'))
import gnn_ref  # noqa: E402


def small_graph(rng, n=7):
    # a ring with chords: symmetric adjacency, edges grouped by destination
    adj = {j: sorted({(j - 1) % n, (j + 1) % n, (j + 3) % n, (j - 3) % n} - {j}) for j in range(n)}
    src = np.array([i for j in range(n) for i in adj[j]], dtype=np.int64)
    dst = np.array([j for j in range(n) for _ in adj[j]], dtype=np.int64)
    xn = rng.standard_normal((n, gnn_ref.FN)) * 0.3
    xe = rng.standard_normal((len(src), gnn_ref.FE)) * 0.3
    tn = rng.standard_normal((n, gnn_ref.OUT)) * 0.1
    te = rng.standard_normal((len(src), gnn_ref.OUT)) * 0.1
    return xn, xe, src, dst, tn, te


def test_backward_matches_finite_differences(monkeypatch):
    monkeypatch.setattr(gnn_ref, 'bf16', lambda x: np.asarray(x, dtype=np.float64))
    rng = np.random.default_rng(0)
    xn, xe, src, dst, tn, te = small_graph(rng)
    p = np.concatenate([np.concatenate([rng.standard_normal(r * c) * np.sqrt(2.0 / r), rng.standard_normal(c) * 0.1])
                        for r, c in gnn_ref.shapes()])
    loss, g = gnn_ref.loss_and_gradients(p, xn, xe, src, dst, tn, te)
    # one probe entry in every weight and bias tensor, plus random others
    offs, o = [], 0
    for r, c in gnn_ref.shapes():
        offs += [o + rng.integers(r * c), o + r * c + rng.integers(c)]
        o += r * c + c
    offs += list(rng.integers(0, len(p), 20))
    eps = 1e-6
    for k in offs:
        q = p.copy()
        q[k] += eps
        lp, _ = gnn_ref.loss_and_gradients(q, xn, xe, src, dst, tn, te)
        q[k] -= 2 * eps
        lm, _ = gnn_ref.loss_and_gradients(q, xn, xe, src, dst, tn, te)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9 * np.abs(g).max(), (k, fd, g[k])


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 0.0, 3.0e38])
    r = gnn_ref.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == 1.0
    assert r[4] == -2.5 and r[5] == 0.0 and np.isfinite(r[6])
