"""Autotuner of the batched factorisation's tiles (hfpx_batch_create's block
size nb and leaf rows): times every candidate on a workload of the batched
form and writes the fastest to hfpx3d_b200/data/batch_tiles.json, which
engine.Batch reads for its defaults.

    python -m hfpx3d_b200.batch_tune [--n-mesh 256] [--reps 2]

Each candidate's time is the best of `reps` replays of the captured run
(assembly, factorisation, solves and refinement of every mesh) after one
warm-up run that also captures the graph."""
import argparse
import json
import os
import time

import numpy as np

from hfpx3d_b200 import engine, meshgen

CANDIDATES = [(nb, leaf) for nb in (64, 128, 256) for leaf in (256, 512)]
G, NU, BETA = 1.0, 0.35, 0.125


def time_candidates(ctx, dms, S, candidates=CANDIDATES, reps=2, tol=1e-10):
    out = {}
    for nb, leaf in candidates:
        B = engine.Batch(ctx, dms, G, NU, nb=nb, leaf_rows=leaf)
        B.set_loads(S)
        info = B.run(tol=tol)
        best = float('inf')
        for _ in range(reps):
            t0 = time.perf_counter()
            info = B.run(tol=tol)
            best = min(best, time.perf_counter() - t0)
        out[f'{nb}x{leaf}'] = {'nb': nb, 'leaf_rows': leaf, 'seconds': best, 'residual': info.residual,
                               'converged': bool(info.converged), 'launches': B.launches}
        B.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--n-mesh', type=int, default=256)
    ap.add_argument('--n-cases', type=int, default=64)
    ap.add_argument('--reps', type=int, default=2)
    ap.add_argument('--out', default=engine.BATCH_TILES_PATH)
    ap.add_argument('--candidates', default='', help='comma-separated NBxLEAF (default: all)')
    args = ap.parse_args()
    cands = CANDIDATES
    if args.candidates:
        cands = [tuple(int(v) for v in c.split('x')) for c in args.candidates.split(',')]
    ctx = engine.Context(0)
    meshes, S = meshgen.batch_workload(args.n_mesh, args.n_cases)
    dms = [engine.DeviceMesh(ctx, engine.MeshGeom(n, c), BETA) for n, c in meshes]
    res = time_candidates(ctx, dms, S, candidates=cands, reps=args.reps)
    ok = {k: v for k, v in res.items() if v['converged']}
    best = min(ok.values(), key=lambda v: v['seconds'])
    table = {'workload': f'{args.n_mesh} seeded penny/2:1 ellipse meshes, 24-550 elements, {args.n_cases} load cases '
                         'each (meshgen.batch_workload)',
             'trailing_update': 'SIMT FP32' if os.environ.get('HFPX_BATCH_TC') == '0' else 'tcgen05 FP16 grouped (nb a multiple of 64)',
             'candidates': res, 'best': {'nb': best['nb'], 'leaf_rows': best['leaf_rows']}}
    with open(args.out, 'w') as f:
        json.dump(table, f, indent=1)
    print(json.dumps(table))


if __name__ == '__main__':
    main()
