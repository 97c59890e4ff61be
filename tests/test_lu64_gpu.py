"""Binary64 LU solves with inverted diagonal blocks (the correction solves
of the mixed-precision LU solver) against the row-by-row binary64 getrs and a
numpy solve: shapes around the 128-row block, one and many right-hand
sides, repeated solves with one prepared workspace."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _factor(mf, A):
    n = A.shape[0]
    lib, h, s = mf._native.load(), mf._handle(0), torch.cuda.current_stream().cuda_stream
    LU = mf.MFMatrix.from_numpy(A[None])
    ipiv = torch.arange(1, n + 1, dtype=torch.int64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.mflab_getrf(h, s, 1, n, n, LU.ptr(), LU.ld, LU.ls, ipiv.data_ptr(), 12,
                           info.data_ptr()) == 0
    assert int(info.item()) == 0
    wb = C.c_size_t()
    assert lib.mflab_lu64_work_bytes(n, C.byref(wb)) == 0
    work = torch.empty(wb.value, dtype=torch.uint8, device="cuda")
    assert lib.mflab_lu64_prepare(h, s, n, LU.ptr(), LU.ld, ipiv.data_ptr(), work.data_ptr()) == 0
    return LU, ipiv, work


@pytest.mark.parametrize("n,nrhs", [(1, 1), (100, 3), (128, 16), (129, 1), (300, 17),
                                    (1000, 16), (2100, 40)])
def test_lu64_solve_matches_getrs(mf, n, nrhs):
    rng = np.random.default_rng(n + nrhs)
    A = rng.standard_normal((n, n)) + 3 * np.eye(n)
    B = rng.standard_normal((n, nrhs))
    LU, ipiv, work = _factor(mf, A)
    lib, h, s = mf._native.load(), mf._handle(0), torch.cuda.current_stream().cuda_stream
    X1 = mf.MFMatrix.from_numpy(B[None])
    assert lib.mflab_lu64_solve(h, s, n, nrhs, LU.ptr(), LU.ld, work.data_ptr(), X1.ptr(),
                                X1.ld) == 0
    X2 = mf.MFMatrix.from_numpy(B[None])
    assert lib.mflab_getrs(h, s, 1, n, nrhs, LU.ptr(), LU.ld, LU.ls, ipiv.data_ptr(), X2.ptr(),
                           X2.ld, X2.ls) == 0
    x1, x2 = X1.to_numpy()[0], X2.to_numpy()[0]
    ref = np.linalg.solve(A, B)
    scale = np.abs(ref).max()
    assert np.abs(x1 - x2).max() <= 1e-10 * scale
    # the backward error of the new solves is at the binary64 level
    r = B - A @ x1
    be = np.abs(r).max(axis=0) / (np.abs(A).sum(axis=1).max() * np.abs(x1).max(axis=0) +
                                  np.abs(B).max(axis=0))
    assert be.max() <= 64 * n * 2.0 ** -53


def test_lu64_prepared_workspace_is_reused(mf):
    n = 700
    rng = np.random.default_rng(1)
    A = rng.standard_normal((n, n)) + 3 * np.eye(n)
    LU, ipiv, work = _factor(mf, A)
    lib, h, s = mf._native.load(), mf._handle(0), torch.cuda.current_stream().cuda_stream
    first = None
    for _ in range(3):
        B = rng.standard_normal((n, 5))
        X = mf.MFMatrix.from_numpy(B[None])
        assert lib.mflab_lu64_solve(h, s, n, 5, LU.ptr(), LU.ld, work.data_ptr(), X.ptr(),
                                    X.ld) == 0
        assert np.allclose(X.to_numpy()[0], np.linalg.solve(A, B), rtol=1e-9, atol=1e-9)


def test_lu64_arguments(mf):
    lib, h, s = mf._native.load(), mf._handle(0), torch.cuda.current_stream().cuda_stream
    wb = C.c_size_t()
    assert lib.mflab_lu64_work_bytes(-1, C.byref(wb)) == mf._native.MFLAB_ERR_ARG
    assert lib.mflab_lu64_solve(h, s, 10, 1, None, 10, None, None, 10) == mf._native.MFLAB_ERR_ARG
    assert lib.mflab_lu64_solve(h, s, 0, 1, None, 0, None, None, 0) == 0


@pytest.mark.parametrize("m,n,nb", [(4096, 4096, 32), (3000, 2000, 32), (600, 900, 17),
                                    (7000, 300, 32), (45, 45, 32), (1, 1, 32)])
def test_binary64_getrf_cluster_panel_matches_lapack(mf, m, n, nb):
    """the binary64 LU (panels in a cluster's shared memory when they fit,
    streamed through one CTA when taller than about 6000 rows) against
    LAPACK's partial pivoting: the same interchanges, factors within binary64
    rounding"""
    import scipy.linalg as sl
    rng = np.random.default_rng(m + n)
    A = rng.standard_normal((m, n))
    lib, h, s = mf._native.load(), mf._handle(0), torch.cuda.current_stream().cuda_stream
    LU = mf.MFMatrix.from_numpy(A[None])
    k = min(m, n)
    ipiv = torch.zeros(k, dtype=torch.int64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.mflab_getrf(h, s, 1, m, n, LU.ptr(), LU.ld, LU.ls, ipiv.data_ptr(), nb,
                           info.data_ptr()) == 0
    assert int(info.item()) == 0
    lu, piv = sl.lu_factor(A, check_finite=False)
    assert np.array_equal(ipiv.cpu().numpy(), piv + 1)
    got = LU.to_numpy()[0]
    assert np.abs(got - lu).max() <= 1e-9 * max(1.0, np.abs(lu).max())


def test_binary64_getrf_singular_reports_first_zero_pivot(mf):
    n = 300
    A = np.random.default_rng(3).standard_normal((n, n))
    A[:, 100] = 0.0  # column 100 is zero below and above: pivot 101 is zero
    lib, h, s = mf._native.load(), mf._handle(0), torch.cuda.current_stream().cuda_stream
    LU = mf.MFMatrix.from_numpy(A[None])
    ipiv = torch.zeros(n, dtype=torch.int64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.mflab_getrf(h, s, 1, n, n, LU.ptr(), LU.ld, LU.ls, ipiv.data_ptr(), 32,
                           info.data_ptr()) == 0
    assert int(info.item()) == 101
