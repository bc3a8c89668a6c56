"""Test infrastructure: a CPU restatement of the learned preconditioner's graph
network (hfpx3d_b200/csrc/gnn.cu) in numpy FP64, forward and backward, the
checker of the GPU kernels' loss and gradients.  It is not used by the product.

The GPU stores weights and activations in BF16 and accumulates every product
in FP32; this restatement rounds to BF16 at the same points (weights, every
hidden activation, the mean-aggregated messages) and accumulates in FP64, so
that the two differ only by accumulation order (and the rare BF16 rounding
that order flips).

Layout of the parameter vector (as hfpx_gnn_get_params returns it): for each
tensor in the order Wn, We, (Wm, Wu) x 4 layers, Woe, Won, the weight
row-major (inputs x outputs), then its bias.
"""
import numpy as np

H, LAYERS, FN, FE, OUT = 64, 4, 336, 336, 324


def shapes():
    s = [(FN, H), (FE, H)]
    for _ in range(LAYERS):
        s += [(3 * H, H), (2 * H, H)]
    s += [(3 * H, OUT), (H, OUT)]
    return s


def unpack(p):
    """List of (W, b) in FP64 from the flat parameter vector."""
    out, off = [], 0
    for r, c in shapes():
        W = np.asarray(p[off:off + r * c], dtype=np.float64).reshape(r, c)
        off += r * c
        b = np.asarray(p[off:off + c], dtype=np.float64)
        off += c
        out.append((W, b))
    assert off == len(p)
    return out


def pack(tensors):
    return np.concatenate([np.concatenate([W.reshape(-1), b]) for W, b in tensors])


def bf16(x):
    """Round to the nearest BF16 (ties to even), via FP32 like the GPU's
    __float2bfloat16_rn of an FP32 value."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def relu(x):
    return np.maximum(x, 0.0)


def forward(p, xn, xe, src, dst):
    T = [(bf16(W), b) for W, b in unpack(p)]
    n, E = xn.shape[0], xe.shape[0]
    deg = np.bincount(dst, minlength=n).astype(np.float64)
    h = bf16(relu(xn @ T[0][0] + T[0][1]))
    z = bf16(relu(xe @ T[1][0] + T[1][1]))
    act = dict(h=[h], cm=[], m=[], cu=[], u=[], z=z, deg=deg)
    for l in range(LAYERS):
        Wm, bm = T[2 + 2 * l]
        Wu, bu = T[3 + 2 * l]
        cm = np.concatenate([h[src], h[dst], z], axis=1)
        m = bf16(relu(cm @ Wm + bm))
        s = np.zeros((n, H))
        np.add.at(s, dst, m)
        agg = bf16(np.where(deg[:, None] > 0, s / np.maximum(deg, 1)[:, None], 0.0))
        cu = np.concatenate([h, agg], axis=1)
        u = bf16(relu(cu @ Wu + bu))
        h = bf16(h + u)
        act['cm'].append(cm)
        act['m'].append(m)
        act['cu'].append(cu)
        act['u'].append(u)
        act['h'].append(h)
    ce = np.concatenate([h[src], h[dst], z], axis=1)
    oe = ce @ T[-2][0] + T[-2][1]
    on = h @ T[-1][0] + T[-1][1]
    act['ce'] = ce
    return oe, on, act, T


def loss_and_gradients(p, xn, xe, src, dst, tn, te):
    """(loss, flat gradient) of the mean squared error over all outputs."""
    oe, on, a, T = forward(p, xn, xe, src, dst)
    n, E = xn.shape[0], xe.shape[0]
    cnt = (n + E) * OUT
    loss = (np.sum((oe - te) ** 2) + np.sum((on - tn) ** 2)) / cnt
    doe = 2.0 * (oe - te) / cnt
    don = 2.0 * (on - tn) / cnt
    grads = [None] * len(T)
    grads[-2] = (a['ce'].T @ doe, doe.sum(axis=0))
    dce = doe @ T[-2][0].T
    h = a['h'][-1]
    grads[-1] = (h.T @ don, don.sum(axis=0))
    dh = don @ T[-1][0].T
    np.add.at(dh, src, dce[:, :H])
    np.add.at(dh, dst, dce[:, H:2 * H])
    dz = dce[:, 2 * H:].copy()
    deg = a['deg']
    for l in reversed(range(LAYERS)):
        Wm, _ = T[2 + 2 * l]
        Wu, _ = T[3 + 2 * l]
        du = dh * (a['u'][l] > 0)
        grads[3 + 2 * l] = (a['cu'][l].T @ du, du.sum(axis=0))
        dcu = du @ Wu.T
        dh2 = dh + dcu[:, :H]
        dm = dcu[dst, H:] / deg[dst][:, None]
        dm = dm * (a['m'][l] > 0)
        grads[2 + 2 * l] = (a['cm'][l].T @ dm, dm.sum(axis=0))
        dcm = dm @ Wm.T
        np.add.at(dh2, src, dcm[:, :H])
        np.add.at(dh2, dst, dcm[:, H:2 * H])
        dz += dcm[:, 2 * H:]
        dh = dh2
    dh = dh * (a['h'][0] > 0)
    grads[0] = (xn.T @ dh, dh.sum(axis=0))
    dz = dz * (a['z'] > 0)
    grads[1] = (xe.T @ dz, dz.sum(axis=0))
    return loss, pack(grads)
