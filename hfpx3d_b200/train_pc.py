"""Train the learned preconditioner's graph network on the GPU.

    python -m hfpx3d_b200.train_pc [--meshes 500] [--out hfpx3d_b200/data/pc_gnn.bin]

Training set: seeded non-planar cracks from hfpx3d_b200.meshgen.wavy -- an
ellipse of aspect U[1, 4] (semi-axes aspect x 1) with out-of-plane waviness
z = amp sin(k x + phase), amp U[0, 0.2] (of the unit semi-axis), k U[pi/2,
2 pi], phase U[0, 2 pi), 500-2000 elements.  For each mesh the engine
assembles the FP64 matrix (hfpx_assemble), builds the network's graph with
its targets (hfpx_gnn_graph_create: the exact local inverse's corrections to
the Neumann blocks) and takes a few Adam steps on it (hfpx_gnn_train, the
engine's own BF16 forward and backward kernels).  A held-out set of meshes
(other seeds) gives the validation loss.  Writes the weights and a short
JSON log (per-mesh loss) beside them.
"""
import argparse
import json
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

G, NU, BETA = 1.0, 0.35, 0.125


def crack(seed, n_min=500, n_max=2000):
    """The seeded training/evaluation crack of a seed: (nods, conn, params)."""
    from hfpx3d_b200 import meshgen
    rng = np.random.default_rng(seed)
    n_tri = int(rng.integers(n_min, n_max + 1))
    aspect = float(rng.uniform(1.0, 4.0))
    amp = float(rng.uniform(0.0, 0.2))
    k = float(rng.uniform(0.5 * np.pi, 2.0 * np.pi))
    phase = float(rng.uniform(0.0, 2.0 * np.pi))
    nods, conn = meshgen.wavy(n_tri, aspect=aspect, amp=amp, k=k, phase=phase, seed=seed)
    return nods, conn, dict(seed=seed, n_tri=n_tri, aspect=aspect, amp=amp, k=k, phase=phase)


def graph_of(ctx, nods, conn, targets=True):
    from hfpx3d_b200 import engine
    mesh = engine.MeshGeom(nods, conn)
    dof, n = engine.make_dof_h_crack(mesh, 0)
    dm = engine.DeviceMesh(ctx, mesh, BETA)
    A = engine.assemble(ctx, dm, dof, n, G, NU)
    graph = engine.GnnGraph(ctx, dm, A, G, targets=targets)
    return dm, A, graph


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument('--meshes', type=int, default=500)
    ap.add_argument('--steps', type=int, default=8, help='Adam steps per mesh')
    ap.add_argument('--epochs', type=int, default=1)
    ap.add_argument('--lr', type=float, default=1e-3)
    ap.add_argument('--lr-min', type=float, default=1e-4)
    ap.add_argument('--val', type=int, default=8, help='held-out meshes')
    ap.add_argument('--seed', type=int, default=0)
    ap.add_argument('--n-min', type=int, default=500)
    ap.add_argument('--n-max', type=int, default=2000)
    ap.add_argument('--out', default=os.path.join(HERE, 'data', 'pc_gnn.bin'))
    ap.add_argument('--max-seconds', type=float, default=0.0,
                    help='stop taking new training meshes after this long (0: no limit)')
    args = ap.parse_args(argv)
    from hfpx3d_b200 import build, engine
    build.build()
    ctx = engine.Context(0)
    net = engine.Gnn(ctx, seed=args.seed)
    train_seeds = [1000 + k for k in range(args.meshes)]
    val_seeds = [900000 + k for k in range(args.val)]
    total = args.epochs * len(train_seeds) * args.steps
    log = dict(meshes=args.meshes, steps_per_mesh=args.steps, epochs=args.epochs, lr=args.lr, lr_min=args.lr_min,
               n_params=net.n_params, train=[], val=[])

    def validate():
        out = []
        for s in val_seeds:
            nods, conn, prm = crack(s, args.n_min, args.n_max)
            dm, A, graph = graph_of(ctx, nods, conn)
            loss, _ = net.gradients(graph)
            out.append(loss)
            graph.close(); A.close(); dm.close()
        return float(np.mean(out))

    v0 = validate()
    log['val'].append(dict(step=0, loss=v0))
    print(f'validation loss before training {v0:.4e}', flush=True)
    t0 = time.time()
    done = 0
    stopped = False
    for ep in range(args.epochs):
        for s in train_seeds:
            if args.max_seconds > 0 and time.time() - t0 > args.max_seconds:
                stopped = True
                break
            nods, conn, prm = crack(s, args.n_min, args.n_max)
            dm, A, graph = graph_of(ctx, nods, conn)
            # cosine schedule over all steps
            lr = args.lr_min + 0.5 * (args.lr - args.lr_min) * (1 + math.cos(math.pi * done / max(1, total)))
            losses = net.train(graph, args.steps, lr)
            done += args.steps
            log['train'].append(dict(seed=s, n_el=int(conn.shape[1]), first=float(losses[0]), last=float(losses[-1])))
            graph.close(); A.close(); dm.close()
            if len(log['train']) % 50 == 0:
                print(f'{len(log["train"])} meshes, {time.time() - t0:.0f} s, loss {losses[-1]:.4e}', flush=True)
        if stopped:
            break
    log['meshes_trained'] = len(log['train'])
    v1 = validate()
    log['val'].append(dict(step=done, loss=v1))
    log['train_seconds'] = time.time() - t0
    print(f'validation loss after training {v1:.4e} ({log["train_seconds"]:.0f} s)', flush=True)
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    net.save(args.out)
    with open(os.path.splitext(args.out)[0] + '_train.json', 'w') as f:
        json.dump(log, f, indent=1)
    return log


if __name__ == '__main__':
    main()
