"""The allocation-free panel LU (hfpx_lu_panel_factor_noalloc) through the C-ABI.

It is for callers that cannot allocate device memory: hosts whose device
memory all belongs to an arena of their own, and real-time loops that forbid
allocation after start-up (cudaMalloc can synchronise the device and take
unbounded time).  The caller passes device buffers (made here with torch); the
entry point itself allocates nothing and keeps its pivot-search scratch in one
static device array.  Its results are checked against the existing entry
point (hfpx_lu_factor), within the tolerance the other LU tests use, on two
calls in a row, and the device's free memory is checked to stay the same
across warmed-up calls."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def factor_existing(ctx, A):
    from hfpx3d_b200 import engine
    m = engine.DeviceMatrix.upload(ctx, A)
    info = ctypes.c_int64()
    ctx.check(engine.lib().hfpx_lu_factor(ctx.h, m.h, engine.HFPX_LU_FP64, ctypes.byref(info)))
    return m.download(), m


def factor_noalloc(ctx, A):
    import torch
    from hfpx3d_b200 import engine
    m, w = A.shape
    # a (w, m) row-major tensor is the (m, w) column-major panel, lda = m
    d = torch.from_numpy(np.ascontiguousarray(A.T)).to('cuda:0')
    piv = torch.full((w,), -7, dtype=torch.int32, device='cuda:0')
    info = ctypes.c_int64(-1)
    torch.cuda.synchronize()
    rc = engine.lib().hfpx_lu_panel_factor_noalloc(ctx.h, ctypes.c_void_p(d.data_ptr()), m, m, w,
                                                   ctypes.c_void_p(piv.data_ptr()), ctypes.byref(info))
    torch.cuda.synchronize()
    return rc, d.cpu().numpy().T.copy(), piv.cpu().numpy(), info.value


def apply_pivots(A, piv):
    P = A.copy()
    for i, p in enumerate(piv):
        P[[i, p]] = P[[p, i]]
    return P


@pytest.mark.parametrize('n', [5, 17, 32])
def test_matches_existing_entry_point_on_two_calls(ctx, n):
    from hfpx3d_b200 import engine
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n))
    F_ref, m = factor_existing(ctx, A)
    b = rng.standard_normal(n)
    x_ref = engine.LU.solve(type('L', (), {'ctx': ctx, 'matrix': m, 'mode': 0})(), b)
    for _ in range(2):
        rc, F, piv, info = factor_noalloc(ctx, A)
        assert rc == engine.HFPX_OK and info == 0
        assert np.abs(F - F_ref).max() <= 1e-12 * np.abs(F_ref).max()
        L = np.tril(F, -1) + np.eye(n)
        U = np.triu(F)
        y = np.linalg.solve(L, apply_pivots(b[:, None], piv)[:, 0])
        x = np.linalg.solve(U, y)
        assert np.abs(x - x_ref).max() <= 1e-10 * np.abs(x_ref).max()


def test_tall_panel_two_calls(ctx):
    from hfpx3d_b200 import engine
    rng = np.random.default_rng(3)
    A = rng.standard_normal((6000, 32))
    out = [factor_noalloc(ctx, A) for _ in range(2)]
    for rc, F, piv, info in out:
        assert rc == engine.HFPX_OK and info == 0
        L = np.tril(F, -1)
        L[:32] += np.eye(32)
        U = np.triu(F[:32])
        assert np.abs(L @ U - apply_pivots(A, piv)).max() <= 1e-12 * np.abs(A).max()
        assert np.abs(L).max() <= 1.0 + 1e-15     # partial pivoting bound
    assert np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][2], out[1][2])


def test_rejects_sizes_beyond_the_limit(ctx):
    import torch
    from hfpx3d_b200 import engine
    d = torch.zeros(64, dtype=torch.float64, device='cuda:0')
    piv = torch.zeros(64, dtype=torch.int32, device='cuda:0')
    info = ctypes.c_int64()
    L = engine.lib()
    for m, w in ((64, 33), (10, 32), (1_000_000, 32)):
        rc = L.hfpx_lu_panel_factor_noalloc(ctx.h, ctypes.c_void_p(d.data_ptr()), m, m, w,
                                            ctypes.c_void_p(piv.data_ptr()), ctypes.byref(info))
        assert rc == engine.HFPX_ERR_ARG, (m, w)


def test_zero_pivot_reported(ctx):
    from hfpx3d_b200 import engine
    A = np.random.default_rng(4).standard_normal((300, 12))
    A[:, 7] = 0.0
    rc, F, piv, info = factor_noalloc(ctx, A)
    assert rc == engine.HFPX_ERR_SINGULAR and info == 8
    rc, F, piv, info = factor_noalloc(ctx, np.eye(40, 20))   # scratch reused: info cleared again
    assert rc == engine.HFPX_OK and info == 0


def test_allocates_nothing(ctx):
    import torch
    from hfpx3d_b200 import engine
    rng = np.random.default_rng(5)
    A = rng.standard_normal((20000, 32))
    d = torch.from_numpy(np.ascontiguousarray(A.T)).to('cuda:0')
    piv = torch.zeros(32, dtype=torch.int32, device='cuda:0')
    info = ctypes.c_int64(-1)
    L = engine.lib()

    def call():
        d.copy_(torch.from_numpy(np.ascontiguousarray(A.T)))
        torch.cuda.synchronize()
        rc = L.hfpx_lu_panel_factor_noalloc(ctx.h, ctypes.c_void_p(d.data_ptr()), 20000, 20000, 32,
                                            ctypes.c_void_p(piv.data_ptr()), ctypes.byref(info))
        torch.cuda.synchronize()
        assert rc == engine.HFPX_OK and info.value == 0

    call()                                   # first call on the device: address look-up
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(3):
        call()
    # any cudaMalloc inside the call would take at least one 2 MiB page
    assert torch.cuda.mem_get_info(0)[0] == free0


def test_captured_into_a_graph(ctx):
    """The call inside a stream capture of the context's stream: the capture
    ends cleanly (no host read, no synchronisation inside it), and each
    replay of the graph factors the panel as a direct call does."""
    import torch
    from cuda.bindings import driver as cu
    from hfpx3d_b200 import engine
    rng = np.random.default_rng(6)
    A = rng.standard_normal((3000, 24))
    rc, F_ref, piv_ref, info_ref = factor_noalloc(ctx, A)   # also the first call on the device
    assert rc == engine.HFPX_OK and info_ref == 0
    d = torch.from_numpy(np.ascontiguousarray(A.T)).to('cuda:0')
    piv = torch.full((24,), -7, dtype=torch.int32, device='cuda:0')
    stream = ctypes.c_void_p()
    ctx.check(engine.lib().hfpx_ctx_stream(ctx.h, ctypes.byref(stream)))
    hs = cu.CUstream(stream.value)
    torch.cuda.synchronize()

    def ok(res):
        err = res[0] if isinstance(res, tuple) else res
        assert err == cu.CUresult.CUDA_SUCCESS, err
        return res[1] if isinstance(res, tuple) and len(res) > 1 else None
    ok(cu.cuStreamBeginCapture(hs, cu.CUstreamCaptureMode.CU_STREAM_CAPTURE_MODE_THREAD_LOCAL))
    info = ctypes.c_int64(-1)
    rc = engine.lib().hfpx_lu_panel_factor_noalloc(ctx.h, ctypes.c_void_p(d.data_ptr()), 3000, 3000, 24,
                                                   ctypes.c_void_p(piv.data_ptr()), ctypes.byref(info))
    graph = ok(cu.cuStreamEndCapture(hs))
    assert rc == engine.HFPX_OK and info.value == 0
    gexec = ok(cu.cuGraphInstantiate(graph, 0))
    for _ in range(2):
        d.copy_(torch.from_numpy(np.ascontiguousarray(A.T)))
        piv.fill_(-7)
        torch.cuda.synchronize()
        ok(cu.cuGraphLaunch(gexec, hs))
        ok(cu.cuStreamSynchronize(hs))
        assert np.array_equal(d.cpu().numpy().T, F_ref) and np.array_equal(piv.cpu().numpy(), piv_ref)
    ok(cu.cuGraphExecDestroy(gexec))
    ok(cu.cuGraphDestroy(graph))
