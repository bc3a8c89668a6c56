"""The link-level drop-in of the LU: libhfpx_lapacke.so implements
LAPACKE_dgetrf/LAPACKE_dgetrs on the engine, and the reference's own il::LU
(il/linear_algebra/dense/factorization/LU.h:79-120), compiled from the
reference tree against it (oracle/_ref/lu_dropin), factors and solves on the
GPU with LAPACK's results."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, 'hfpx3d_b200', 'libhfpx_lapacke.so')
DROPIN = os.path.join(ROOT, 'oracle', '_ref', 'lu_dropin')
_I = ctypes.c_int
_D = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)


def shim():
    from hfpx3d_b200 import build
    build.build()
    lib = ctypes.CDLL(SHIM)
    lib.LAPACKE_dgetrf.argtypes = [_I, _I, _I, _D, _I, _IP]
    lib.LAPACKE_dgetrf.restype = _I
    lib.LAPACKE_dgetrs.argtypes = [_I, ctypes.c_char, _I, _I, _D, _I, _IP, _D, _I]
    lib.LAPACKE_dgetrs.restype = _I
    lib.LAPACKE_dgesv.argtypes = [_I, _I, _I, _D, _I, _IP, _D, _I]
    lib.LAPACKE_dgesv.restype = _I
    return lib


def dp(a):
    return a.ctypes.data_as(_D)


def test_exports_and_argument_checks():
    # no GPU needed: LAPACK's illegal-argument codes come back before the engine
    lib = shim()
    a = np.zeros((4, 4), order='F')
    ip = np.zeros(4, dtype=np.int32)
    ipp = ip.ctypes.data_as(_IP)
    assert lib.LAPACKE_dgetrf(101, 4, 4, dp(a), 4, ipp) == -1       # row-major
    assert lib.LAPACKE_dgetrf(102, 4, 3, dp(a), 4, ipp) == -3       # not square
    assert lib.LAPACKE_dgetrf(102, 4, 4, dp(a), 2, ipp) == -5       # lda < m
    b = np.zeros(4)
    assert lib.LAPACKE_dgetrs(102, b'T', 4, 1, dp(a), 4, ipp, dp(b), 4) == -2   # transposed
    assert lib.LAPACKE_dgetrs(102, b'N', 4, 1, dp(a), 4, ipp, dp(b), 2) == -9   # ldb < n
    assert lib.LAPACKE_dgesv(100, 4, 1, dp(a), 4, ipp, dp(b), 4) == -1          # unknown layout
    assert lib.LAPACKE_dgesv(102, 4, -1, dp(a), 4, ipp, dp(b), 4) == -3
    assert lib.LAPACKE_dgesv(102, 4, 1, dp(a), 3, ipp, dp(b), 4) == -5
    assert lib.LAPACKE_dgesv(102, 4, 1, dp(a), 4, ipp, dp(b), 3) == -8          # col-major: ldb < n
    assert lib.LAPACKE_dgesv(101, 4, 2, dp(a), 4, ipp, dp(b), 1) == -8          # row-major: ldb < nrhs


@pytest.mark.gpu
@pytest.mark.parametrize('layout', [102, 101])
def test_dgesv_matches_lapack(layout):
    # il::linearSolve (linearSolve.h:28-76): column-major Array2D, row-major Array2C
    import scipy.linalg as sl
    lib = shim()
    rng = np.random.default_rng(5)
    n, nrhs = 300, 2
    A = rng.standard_normal((n, n)) + np.diag(np.linspace(1, 3, n))
    B = rng.standard_normal((n, nrhs))
    order = 'F' if layout == 102 else 'C'
    a, b = np.array(A, order=order), np.array(B, order=order)
    ip = np.zeros(n, dtype=np.int32)
    ld_b = n if layout == 102 else nrhs
    assert lib.LAPACKE_dgesv(layout, n, nrhs, dp(a), n, ip.ctypes.data_as(_IP), dp(b), ld_b) == 0
    lu, piv = sl.lu_factor(A)
    assert np.array_equal(ip - 1, piv)
    assert np.abs(a - lu).max() <= 1e-12 * np.abs(lu).max()
    assert np.abs(b - np.linalg.solve(A, B)).max() <= 1e-11 * np.abs(b).max()
    # a zero column: info = its 1-based index, B untouched
    A[:, 7] = 0.0
    a, b = np.array(A, order=order), np.array(B, order=order)
    assert lib.LAPACKE_dgesv(layout, n, nrhs, dp(a), n, ip.ctypes.data_as(_IP), dp(b), ld_b) == 8
    assert np.array_equal(b, B)


@pytest.mark.gpu
def test_dgetrf_matches_lapack():
    import scipy.linalg as sl
    lib = shim()
    rng = np.random.default_rng(4)
    n = 700
    A = rng.standard_normal((n, n)) + np.diag(np.linspace(1, 3, n))
    a = np.asfortranarray(A.copy())
    ip = np.zeros(n, dtype=np.int32)
    assert lib.LAPACKE_dgetrf(102, n, n, dp(a), n, ip.ctypes.data_as(_IP)) == 0
    lu, piv = sl.lu_factor(A)
    assert np.array_equal(ip - 1, piv)                       # the same interchanges
    assert np.abs(a - lu).max() <= 1e-12 * np.abs(lu).max()  # the same factors up to rounding
    B = np.asfortranarray(rng.standard_normal((n, 3)))
    X = B.copy(order='F')
    assert lib.LAPACKE_dgetrs(102, b'N', n, 3, dp(a), n, ip.ctypes.data_as(_IP), dp(X), n) == 0
    assert np.abs(A @ X - B).max() <= 1e-11 * np.abs(B).max()


def run_dropin(tmp_path, A, B):
    n, nrhs = A.shape[0], B.shape[1]
    fi, fo = tmp_path / 'in.bin', tmp_path / 'out.bin'
    with open(fi, 'wb') as f:
        np.array([n, nrhs], dtype=np.int64).tofile(f)
        np.asfortranarray(A).reshape(-1, order='F').tofile(f)
        np.asfortranarray(B).reshape(-1, order='F').tofile(f)
    r = subprocess.run([DROPIN, str(fi), str(fo)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    raw = np.fromfile(fo, dtype=np.int64, count=1)
    X = np.fromfile(fo, dtype=np.float64, offset=8).reshape(n, nrhs, order='F')
    return int(raw[0]), X


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(DROPIN), reason='oracle/_ref/lu_dropin is built where the reference tree is')
def test_reference_il_lu_on_the_engine(tmp_path):
    g = golden('ref_p24')
    st, X = run_dropin(tmp_path, g['A'], g['rhs'].reshape(-1, 1))
    assert st == 0
    assert np.abs(X[:, 0] - g['x']).max() <= 1e-12 * np.abs(g['x']).max()
    # a singular matrix: il::Status MatrixSingular with LAPACK's rank info
    A = np.eye(60) + 0.01 * np.random.default_rng(2).standard_normal((60, 60))
    A[:, 23] = 0.0
    st, _ = run_dropin(tmp_path, A, np.ones((60, 1)))
    assert st == 24
