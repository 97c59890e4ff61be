"""Single right-hand-side solves on the device: trsv! (trsv.jl:19-73) and the
vector ldiv!/solve methods of Cholesky, LU and LDLT (solve.jl:23-52,
115-147, 299-335), bitwise against the oracle's one-column solves (trsv!
keeps trsm!'s per-row ascending chains, trsv.jl:47-70), plus the option-code
errors of the C ABI (ArgumentError, as trsv.jl:32-34)."""
import ctypes as C

import numpy as np
import pytest

from conftest import assert_bitwise
from test_oracle import syn

pytestmark = pytest.mark.gpu


def _tri(rng, N, n, uplo):
    A = syn.randn_mf(rng, N, n, n)
    A[0] += 4.0 * np.eye(n)  # well-conditioned triangle
    other = np.triu_indices(n, 1) if uplo == "lower" else np.tril_indices(n, -1)
    A[:, other[0], other[1]] = np.nan  # the other triangle is never read
    return A


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("uplo", ["lower", "upper"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("diag", ["nonunit", "unit"])
@pytest.mark.parametrize("n", [1, 37, 300])
def test_trsv_matches_oracle(mf, ref, rng, N, uplo, trans, diag, n):
    A = _tri(rng, N, n, uplo)
    b = syn.randn_mf(rng, N, n, 1)
    alpha = syn.randn_mf(rng, N, 1, 1)[:, 0, 0]
    for a in (1.0, alpha):
        xd = mf.MFMatrix.from_numpy(b[:, :, 0])
        assert xd.is_vector
        mf.trsv_(xd, mf.MFMatrix.from_numpy(A), a, uplo=uplo, trans=trans, diag=diag)
        want = ref.trsm(b.copy(), A, a, "left", uplo, trans, diag)[:, :, 0]
        assert_bitwise(xd.to_numpy(), want, f"trsv {uplo} {trans} {diag}")


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("n", [1, 29, 200])
def test_cholesky_vector_solve(mf, ref, rng, N, n):
    S = syn.spd_matrix(rng, N, n, ref.gemm)
    Sd = mf.MFMatrix.from_numpy(S)
    F = mf.cholesky_(Sd)
    L, info = ref.potrf(S)
    assert info == 0
    b = syn.randn_mf(rng, N, n, 1)
    bd = mf.MFMatrix.from_numpy(b[:, :, 0])
    x = mf.solve(F, bd)
    assert x.is_vector and x.shape == (n,)
    want = ref.potrs(L, b)[:, :, 0]
    assert_bitwise(x.to_numpy(), want, "cholesky vector solve")
    # ldiv!(x, F, b): b is copied into x first, b itself is untouched
    xd = mf.MFMatrix.zeros(N, n)
    mf.ldiv_(xd, F, bd)
    assert_bitwise(xd.to_numpy(), want, "cholesky ldiv!(x, F, b)")
    assert_bitwise(bd.to_numpy(), b[:, :, 0], "source unchanged")
    assert np.all(ref.backward_error(S, want[:, :, None], b) < 4096 * n * 2.0 ** (-52 * N))


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("n", [1, 45, 160])
def test_lu_vector_solve(mf, ref, rng, N, n):
    A = syn.randn_mf(rng, N, n, n)
    Ad = mf.MFMatrix.from_numpy(A)
    F = mf.lu_(Ad)
    LU, piv, info = ref.getrf(A)
    assert info == 0
    b = syn.randn_mf(rng, N, n, 1)
    x = mf.solve(F, mf.MFMatrix.from_numpy(b[:, :, 0]))
    assert x.is_vector
    assert_bitwise(x.to_numpy(), ref.getrs(LU, piv, b)[:, :, 0], "lu vector solve")


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("n,blocked,block", [(1, False, 1), (40, False, 1), (90, True, 8)])
def test_ldlt_vector_solve(mf, ref, rng, N, n, blocked, block):
    X = syn.randn_mf(rng, N, n, n)
    S = np.tril(X) + np.transpose(np.tril(X, -1), (0, 2, 1))
    cfg = mf.KernelConfig(ldlt_strategy="blocked" if blocked else "unblocked",
                          ldlt_block=block, ldlt_blocked_crossover=1)
    Sd = mf.MFMatrix.from_numpy(S)
    F = mf.ldlt_(Sd, config=cfg)
    Fr, dsr, pvr, blr, info = ref.sytrf(S, blocked=blocked, block=block)
    assert info == 0
    b = syn.randn_mf(rng, N, n, 1)
    x = mf.solve(F, mf.MFMatrix.from_numpy(b[:, :, 0]), config=cfg)
    Xr, rc = ref.sytrs(Fr, dsr, pvr, blr, b)
    assert rc == 0 and x.is_vector
    assert_bitwise(x.to_numpy(), Xr[:, :, 0], "ldlt vector solve")


@pytest.mark.parametrize("N", [2, 4])
def test_vector_solve_dimension_errors(mf, ref, rng, N):
    n = 12
    S = syn.spd_matrix(rng, N, n, ref.gemm)
    F = mf.cholesky_(mf.MFMatrix.from_numpy(S))
    with pytest.raises(mf.DimensionMismatch):
        mf.solve(F, mf.MFMatrix.zeros(N, n + 1))
    A = mf.MFMatrix.from_numpy(_tri(rng, N, n, "lower"))
    with pytest.raises(mf.DimensionMismatch):
        mf.trsv_(mf.MFMatrix.zeros(N, n - 1), A)
    with pytest.raises(mf.ArgumentError):
        mf.trsv_(mf.MFMatrix.zeros(N, n), A, uplo="middle")
    with pytest.raises(mf.ArgumentError):
        mf.trsv_(mf.MFMatrix.zeros(N, n), A, trans="C")


def test_option_codes_are_argument_errors(mf):
    """the C ABI returns MFLAB_ERR_FLAG for an option code outside its range
    and MFLAB_ERR_ARG for a bad size; the host maps them to ArgumentError and
    DimensionMismatch"""
    lib = mf._native.load()
    h = mf._handle(0)
    x = mf.MFMatrix.zeros(2, 8, 8)
    one = (C.c_double * 4)(1.0)
    args = (8, 8, x.ptr(), x.ld, x.ls, x.ptr(), x.ld, x.ls, one)
    assert lib.mflab_trsm(h, None, 2, 2, 0, 0, 0, *args) == mf._native.MFLAB_ERR_FLAG
    assert lib.mflab_trsm(h, None, 2, 0, 0, 5, 0, *args) == mf._native.MFLAB_ERR_FLAG
    assert lib.mflab_trsm(h, None, 2, 0, 0, 0, 0, -1, 8, *args[2:]) == mf._native.MFLAB_ERR_ARG
    assert lib.mflab_set_solve_order(h, 9) == mf._native.MFLAB_ERR_FLAG
    with pytest.raises(mf.ArgumentError):
        mf._check(mf._native.MFLAB_ERR_FLAG, "trsm!")
    with pytest.raises(mf.DimensionMismatch):
        mf._check(mf._native.MFLAB_ERR_ARG, "trsm!")
