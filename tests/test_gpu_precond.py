"""Near-field preconditioners and flexible GMRES on the dense FP64 operator
(hfpx_precond_*, hfpx_gmres_precond), and the learned preconditioner's graph
network (hfpx_gnn_*): no counterpart in the reference, which solves directly
(il::LU, il/linear_algebra/dense/factorization/LU.h:79-120); the operator is
make_3dbem_matrix_s's (src/Solvers/system_assembly.cpp:30-219).

* blocks of block-Jacobi, Neumann and the exact local inverse against numpy
  on the downloaded matrix (1e-10 of the block scale);
* GMRES with each reaches the LU solution;
* the network's loss and gradients (BF16 storage, FP32 accumulation) against
  the CPU FP64 restatement oracle/gnn_ref.py rounding to BF16 at the same
  points: loss within 1e-3, every tensor's gradient within 2 % of its largest
  entry (accumulation order can flip a BF16 rounding);
* Adam training on the GPU reduces the loss;
* the trained network (hfpx3d_b200/data/pc_gnn.bin) on an unseen crack: its
  GMRES(50) iterations against no preconditioner, block-Jacobi and Neumann."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
G, NU, BETA = 1.0, 0.35, 0.125
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, 'oracle'))


def setup(ctx, mesh_args, kind='wavy'):
    from hfpx3d_b200 import engine, meshgen
    nods, conn = getattr(meshgen, kind)(*mesh_args[0], **mesh_args[1])
    mesh = engine.MeshGeom(nods, conn)
    dof, n = engine.make_dof_h_crack(mesh, 0)
    dm = engine.DeviceMesh(ctx, mesh, BETA)
    A = engine.assemble(ctx, dm, dof, n, G, NU)
    rhs = engine.add_s_inf_to_3dbem_rhs(ctx, dm, dof, n, [0, 0, 1.0, 0, 0, 0])
    return nods, conn, dm, A, rhs, n


def neighbours(conn):
    ne = conn.shape[1]
    v2e = {}
    for e in range(ne):
        for v in conn[:3, e]:
            v2e.setdefault(int(v), set()).add(e)
    return [sorted(set().union(*[v2e[int(v)] for v in conn[:3, e]]) - {e}) for e in range(ne)]


def test_blocks_match_numpy(ctx):
    from hfpx3d_b200 import engine
    nods, conn, dm, A, rhs, n = setup(ctx, ((80,), dict(aspect=1.5, amp=0.15, seed=2)))
    Ah = A.download()
    ne = conn.shape[1]
    nb = neighbours(conn)
    blk = lambda i, j: Ah[18 * i:18 * i + 18, 18 * j:18 * j + 18]
    Dinv = [np.linalg.inv(blk(j, j)) for j in range(ne)]
    scale = max(np.abs(d).max() for d in Dinv)
    for kind in (engine.HFPX_PC_BLOCK_JACOBI, engine.HFPX_PC_NEUMANN, engine.HFPX_PC_LOCAL_INVERSE):
        pc = engine.Precond(ctx, dm, A, kind)
        rows, cols, B = pc.blocks()
        assert len(rows) == ne + sum(len(x) for x in nb)
        ref = {}
        for j in range(ne):
            if kind == engine.HFPX_PC_LOCAL_INVERSE:
                P = [j] + nb[j]
                idx = np.concatenate([np.arange(18) + 18 * p for p in P])
                E = np.zeros((len(idx), 18))
                E[:18] = np.eye(18)
                m = np.linalg.solve(Ah[np.ix_(idx, idx)], E)
                for k, p in enumerate(P):
                    ref[(p, j)] = m[18 * k:18 * k + 18]
            else:
                ref[(j, j)] = Dinv[j]
                for i in nb[j]:
                    ref[(i, j)] = -Dinv[i] @ blk(i, j) @ Dinv[j] if kind == engine.HFPX_PC_NEUMANN else 0 * Dinv[i]
        err = max(np.abs(B[k] - ref[(int(rows[k]), int(cols[k]))]).max() for k in range(len(rows)))
        assert err <= 1e-10 * scale, (kind, err / scale)
        pc.close()


def test_gmres_with_each_preconditioner_reaches_the_lu_solution(ctx):
    from hfpx3d_b200 import engine
    nods, conn, dm, A, rhs, n = setup(ctx, ((300,), dict(aspect=2.0, amp=0.15, seed=3)))
    x_lu = engine.LU(ctx, engine.DeviceMatrix.upload(ctx, A.download()), engine.HFPX_LU_FP64).solve(rhs)
    iters = {}
    for name, kind in (('none', None), ('jacobi', engine.HFPX_PC_BLOCK_JACOBI), ('neumann', engine.HFPX_PC_NEUMANN),
                       ('local', engine.HFPX_PC_LOCAL_INVERSE)):
        pc = engine.Precond(ctx, dm, A, kind) if kind is not None else None
        x, info = engine.gmres(ctx, A, rhs, pc, tol=1e-11, restart=50, max_iter=2000)
        assert info.converged, name
        assert np.abs(x - x_lu).max() <= 1e-8 * np.abs(x_lu).max(), name
        iters[name] = info.iterations
    print('GMRES(50) iterations to 1e-11:', iters)
    assert iters['local'] <= iters['neumann'] < iters['jacobi'] < iters['none']


def test_network_gradients_match_cpu_restatement(ctx):
    import gnn_ref
    from hfpx3d_b200 import engine
    nods, conn, dm, A, rhs, n = setup(ctx, ((40,), dict(aspect=1.2, amp=0.1, seed=5)))
    net = engine.Gnn(ctx, seed=7)
    p = net.params()
    # give the (zero-initialised) output heads random values so that every
    # tensor receives a gradient
    rng = np.random.default_rng(1)
    off = 0
    for t, (r, c) in enumerate(gnn_ref.shapes()):
        if t >= len(gnn_ref.shapes()) - 2:
            p[off:off + r * c + c] = rng.standard_normal(r * c + c).astype(np.float32) * 0.05
        off += r * c + c
    net.set_params(p)
    graph = engine.GnnGraph(ctx, dm, A, G, targets=True)
    d = graph.data()
    loss_gpu, g_gpu = net.gradients(graph)
    loss_cpu, g_cpu = gnn_ref.loss_and_gradients(p.astype(np.float64), d['xn'].astype(np.float64),
                                                 d['xe'].astype(np.float64), d['src'], d['dst'],
                                                 d['tn'].astype(np.float64), d['te'].astype(np.float64))
    assert abs(loss_gpu - loss_cpu) <= 1e-3 * loss_cpu, (loss_gpu, loss_cpu)
    off = 0
    for t, (r, c) in enumerate(gnn_ref.shapes()):
        for a, b in ((off, off + r * c), (off + r * c, off + r * c + c)):
            gc, gg = g_cpu[a:b], g_gpu[a:b].astype(np.float64)
            scale = np.abs(gc).max()
            assert scale > 0, t
            assert np.abs(gg - gc).max() <= 2e-2 * scale, (t, np.abs(gg - gc).max() / scale)
        off += r * c + c


def test_training_reduces_the_loss(ctx):
    from hfpx3d_b200 import engine
    nods, conn, dm, A, rhs, n = setup(ctx, ((150,), dict(aspect=2.0, amp=0.1, seed=6)))
    net = engine.Gnn(ctx, seed=3)
    graph = engine.GnnGraph(ctx, dm, A, G, targets=True)
    losses = net.train(graph, 60, 1e-3)
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.5 * losses[0], (losses[0], losses[-1])


def test_learned_preconditioner_gain_on_an_unseen_crack(ctx):
    from hfpx3d_b200 import engine
    assert os.path.exists(engine.WEIGHTS_PATH), 'trained weights missing (python -m hfpx3d_b200.train_pc)'
    net = engine.Gnn(ctx, path=engine.WEIGHTS_PATH)
    # an unseen seed, outside the training seeds
    nods, conn, dm, A, rhs, n = setup(ctx, ((900,), dict(aspect=2.5, amp=0.12, k=np.pi, phase=0.7, seed=90001)))
    x_lu = engine.LU(ctx, engine.DeviceMatrix.upload(ctx, A.download()), engine.HFPX_LU_FP64).solve(rhs)
    iters = {}
    for name, kind in (('none', None), ('jacobi', engine.HFPX_PC_BLOCK_JACOBI), ('neumann', engine.HFPX_PC_NEUMANN),
                       ('learned', engine.HFPX_PC_LEARNED), ('local', engine.HFPX_PC_LOCAL_INVERSE)):
        pc = engine.Precond(ctx, dm, A, kind, net=net if kind == engine.HFPX_PC_LEARNED else None, shear_m=G) \
            if kind is not None else None
        x, info = engine.gmres(ctx, A, rhs, pc, tol=1e-8, restart=50, max_iter=3000)
        assert info.converged, name
        assert np.abs(x - x_lu).max() <= 1e-5 * np.abs(x_lu).max(), name
        iters[name] = info.iterations
    print('GMRES(50) iterations to 1e-8 on an unseen 900-element wavy crack:', iters)
    assert iters['learned'] < iters['neumann'] < iters['jacobi'] < iters['none']
