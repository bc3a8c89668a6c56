"""The engine's own tcgen05 tensor-core kernels (the 2-SM pair and the 1-SM
kernel) for the mixed LU's trailing update (hfpx_gemm_f16_update; the GEMM of LAPACK dgetrf's blocked loop,
A22 -= L21 U12, that il::LU reaches at
il/linear_algebra/dense/factorization/LU.h:87), against a plain PyTorch FP32
reference of the same operation on the same FP16 operands.

FP16 x FP16 products are exact in FP32, so the kernel and the reference
differ only by the order of the FP32 accumulation over k: the bound is
2e-6 of sum_l |alpha a_il b_jl| + |c_ij| per entry (k <= 2048 terms, FP32
unit round-off 6e-8)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(params=['2sm', '1sm'])
def variant(request, monkeypatch):
    """Both kernels: the 2-SM pair (cta_group::2, the default) and the 1-SM
    kernel (HFPX_TC_2SM=0), chosen per call from the environment."""
    monkeypatch.setenv('HFPX_TC_2SM', '1' if request.param == '2sm' else '0')
    return request.param


def run_update(ctx, m, n, k, lda_k=None, ldb_k=None, ldc=None, alpha=-0.75, seed=0, lu_like=False):
    import torch
    from hfpx3d_b200 import engine
    lda_k = lda_k or ((k + 7) // 8 * 8)
    ldb_k = ldb_k or ((k + 7) // 8 * 8)
    ldc = ldc or m
    g = torch.Generator(device='cuda').manual_seed(seed)
    dev = 'cuda:0'
    A = torch.randn(m, lda_k, generator=g, device=dev).to(torch.float16)
    B = torch.randn(n, ldb_k, generator=g, device=dev).to(torch.float16)
    if lu_like:
        # L21 multipliers in [-1, 1]; U12 scaled into [2^14, 2^15) as the LU does
        A = (torch.rand(m, lda_k, generator=g, device=dev) * 2 - 1).to(torch.float16)
        B = (torch.randn(n, ldb_k, generator=g, device=dev) * 4096).to(torch.float16)
        alpha = -2.0 ** -12
    # padding beyond k must not be read: fill it with NaN
    if lda_k > k:
        A[:, k:] = float('nan')
    if ldb_k > k:
        B[:, k:] = float('nan')
    Cbuf = torch.randn(n, ldc, generator=g, device=dev)          # column-major m x n with ldc
    if ldc > m:
        Cbuf[:, m:] = 12345.0                                   # rows below m must stay untouched
    C0 = Cbuf.clone()
    a = torch.tensor([alpha], dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    rc = engine.lib().hfpx_gemm_f16_update(ctx.h, m, n, k, ctypes.c_void_p(A.data_ptr()), lda_k,
                                           ctypes.c_void_p(B.data_ptr()), ldb_k, ctypes.c_void_p(Cbuf.data_ptr()),
                                           ldc, ctypes.c_void_p(a.data_ptr()))
    ctx.check(rc)
    torch.cuda.synchronize()
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        Af, Bf = A[:, :k].float(), B[:, :k].float()
        ref = C0[:, :m].T + alpha * (Af @ Bf.T)                     # m x n, FP32
        bound = 2e-6 * (abs(alpha) * (Af.abs() @ Bf.abs().T) + C0[:, :m].T.abs())
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    out = Cbuf[:, :m].T
    err = ((out - ref).abs() / bound.clamp_min(1e-30)).max().item()
    untouched = bool((Cbuf[:, m:] == C0[:, m:]).all().item()) if ldc > m else True
    return err, untouched


@pytest.mark.parametrize('m,n,k', [(128, 256, 64), (1, 1, 8), (1000, 700, 2048), (5000, 300, 320),
                                   (333, 1027, 136), (129, 257, 72)])
def test_update_matches_fp32_reference(ctx, variant, m, n, k):
    err, untouched = run_update(ctx, m, n, k)
    assert err <= 1.0 and untouched, err


def test_padded_strides_and_ldc(ctx, variant):
    # K strides beyond k (padding filled with NaN) and C with ldc > m
    err, untouched = run_update(ctx, 700, 513, 200, lda_k=208, ldb_k=256, ldc=800)
    assert err <= 1.0 and untouched, err


@pytest.mark.parametrize('m,n', [(20000, 2048), (8000, 8000)])
def test_lu_shaped_update(ctx, variant, m, n):
    # tall-skinny L21 (m x 2048) times scaled U12 (2048 x n), as one LU step
    err, untouched = run_update(ctx, m, n, 2048, lu_like=True, seed=m)
    assert err <= 1.0 and untouched, err


def test_rejects_unaligned_strides(ctx):
    import torch
    from hfpx3d_b200 import engine
    A = torch.zeros(64 * 64, dtype=torch.float16, device='cuda:0')
    C = torch.zeros(64 * 64, dtype=torch.float32, device='cuda:0')
    a = torch.ones(1, dtype=torch.float32, device='cuda:0')
    rc = engine.lib().hfpx_gemm_f16_update(ctx.h, 8, 8, 12, ctypes.c_void_p(A.data_ptr()), 12,
                                           ctypes.c_void_p(A.data_ptr()), 12, ctypes.c_void_p(C.data_ptr()), 8,
                                           ctypes.c_void_p(a.data_ptr()))
    assert rc == engine.HFPX_ERR_ARG
