"""Device kernel of make_local_3dbem_submatrix (elasticity_kernel_integration.cpp:34-205)
through the C-ABI, against the reference's MATLAB goldens, the reference's own
outputs and 40-digit values."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu
G, NU = 1.0, 0.35


def block(ctx, h, z, tau, sfm):
    from hfpx3d_b200 import engine
    tc = tau[0::2] + 1j * tau[1::2]
    sc = (sfm[0::2] + 1j * sfm[1::2]).reshape(6, 6)
    return engine.make_local_3dbem_submatrix(ctx, G, NU, h, z, tc, sc)


@pytest.mark.parametrize('k', [1, 2, 3])
def test_matlab_goldens(ctx, ora, k):
    g = golden('matlab_kernel')
    r, tau, sfm = ora.element_frame(g['vert'])
    h, z = ora.pt_hz(g['vert'], g['pts'][k - 1])
    assert np.abs(block(ctx, h, z, tau, sfm) - g[f'pt{k}']).max() < 5e-8


def test_reference_points_and_oracle(ctx, ora):
    g = golden('ref_kernel_points')
    r, tau, sfm = ora.element_frame(g['vert'])
    for i, pt in enumerate(g['pts']):
        h, z = ora.pt_hz(g['vert'], pt)
        out = block(ctx, h, z, tau, sfm)
        ref = g['out'][i]
        scale = np.abs(ref).max()
        assert np.abs(out - ref).max() < 1e-10 * scale, i            # vs the reference
        assert np.abs(out - ora.local_block(G, NU, h, z, tau, sfm)).max() < 1e-12 * scale, i  # vs oracle


def test_near_plane_truth(ctx):
    g = golden('truth_blocks')
    for i in range(len(g['h'])):
        out = block(ctx, g['h'][i], g['z'][i], g['tau'][i], g['sfm'][i])
        assert np.abs(out - g['truth'][i]).max() < 1e-10 * np.abs(g['truth'][i]).max(), i
