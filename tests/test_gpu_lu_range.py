"""The mixed LU's FP16 trailing update on a strongly pivoting matrix.

The update multiplies FP16 copies of L21 and U12 (FP32 accumulation).  Under
partial pivoting |l| <= 1, so multipliers below 6.1e-5 would fall into FP16's
subnormal range (and below 6e-8 to zero); the engine therefore scales each
row of L21 by a power of two into [2^14, 2^15) and its own tcgen05 kernel
undoes the scale per row in the epilogue (U12 is scaled as a whole).  This
test factors a non-planar (wavy) crack matrix of 10 800 unknowns whose rows
are randomly permuted, so that every panel pivots, with the default update,
with the TF32 update (HFPX_LU_UPDATE=tf32) and with the unscaled cuBLAS FP16
update (HFPX_LU_GEMM=cublas), each in its own process (the switches are read
at start-up), and checks that the refined solutions agree with LAPACK's
(dgesv, the algorithm il::LU calls, il/linear_algebra/dense/factorization/LU.h:87)
to 1e-10 and that the default needs no more refinement steps than TF32."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from hfpx3d_b200 import engine, meshgen
nods, conn = meshgen.wavy(600, aspect=2.0, amp=0.2, k=2 * np.pi, seed=21)
ctx = engine.Context(0)
mesh = engine.MeshGeom(nods, conn)
dof, n = engine.make_dof_h_crack(mesh, 0)
dm = engine.DeviceMesh(ctx, mesh, 0.125)
A = engine.assemble(ctx, dm, dof, n, 1.0, 0.35).download()
b = engine.add_s_inf_to_3dbem_rhs(ctx, dm, dof, n, [0.3, -0.2, 1.0, 0.1, 0.0, 0.2])
perm = np.random.default_rng(5).permutation(n)
M = engine.DeviceMatrix.upload(ctx, A[perm])
lu = engine.LU(ctx, M, engine.HFPX_LU_MIXED)
x = lu.solve(b[perm], tol=1e-13, max_iter=30)
np.save(sys.argv[2], x)
print(json.dumps({'iterations': lu.last_info.iterations, 'residual': lu.last_info.residual, 'n': n}))
'''


def run(env_extra, tmp_path, tag):
    env = dict(os.environ, **env_extra)
    out = str(tmp_path / f'x_{tag}.npy')
    r = subprocess.run([sys.executable, '-c', CHILD, ROOT, out], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    info = json.loads([l for l in r.stdout.splitlines() if l.startswith('{')][-1])
    return info, np.load(out)


def test_pivoting_matrix_fp16_update_matches_lapack(tmp_path):
    from hfpx3d_b200 import engine, meshgen
    nods, conn = meshgen.wavy(600, aspect=2.0, amp=0.2, k=2 * np.pi, seed=21)
    ctx = engine.Context(0)
    mesh = engine.MeshGeom(nods, conn)
    dof, n = engine.make_dof_h_crack(mesh, 0)
    dm = engine.DeviceMesh(ctx, mesh, 0.125)
    A = engine.assemble(ctx, dm, dof, n, 1.0, 0.35).download()
    b = engine.add_s_inf_to_3dbem_rhs(ctx, dm, dof, n, [0.3, -0.2, 1.0, 0.1, 0.0, 0.2])
    ctx.close()
    assert n >= 10000
    x_ref = np.linalg.solve(A, b)
    res = {}
    for tag, env in (('default', {}), ('tf32', {'HFPX_LU_UPDATE': 'tf32'}), ('cublas', {'HFPX_LU_GEMM': 'cublas'})):
        info, x = run(env, tmp_path, tag)
        err = float(np.abs(x - x_ref).max() / np.abs(x_ref).max())
        res[tag] = (info['iterations'], err)
        assert err <= 1e-10, (tag, err)
    print('refinement steps and error vs LAPACK:', res)
    assert res['default'][0] <= res['tf32'][0]
