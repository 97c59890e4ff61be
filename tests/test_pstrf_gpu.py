"""Pivoted Cholesky on the device against the oracle, bit for bit (the whole
factor array, permutation, rank and status), on full-rank and rank-deficient
inputs, the reference's known answers, failures and argument errors."""
import numpy as np
import pytest

from conftest import assert_bitwise
from test_oracle import syn
from test_pstrf_oracle import kat_matrix

pytestmark = pytest.mark.gpu


def _run(mf, A, tol=0.0, check=False):
    Ad = mf.MFMatrix.from_numpy(A)
    F = mf.cholesky_pivoted_(Ad, tol=tol, check=check)
    return F, Ad.to_numpy()


def _psd(ref, rng, N, n, r):
    R = syn.randn_mf(rng, N, n, r)
    return ref.gemm(R, np.ascontiguousarray(R.transpose(0, 2, 1)))


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("n,r,tol", [(1, 1, 0.0), (100, 100, 0.0), (300, 300, 0.0),
                                     (200, 50, 1e-12), (257, 256, 1e-12), (130, 20, 0.0)],
                         ids=str)
def test_pstrf_matches_oracle(mf, ref, rng, N, n, r, tol):
    A = _psd(ref, rng, N, n, r)
    if r == n:
        A[0][np.diag_indices(n)] += n  # well conditioned, as S = R R^T + n I
    F, got = _run(mf, A, tol)
    want, perm, rank, info = ref.pstrf(A, tol)
    assert (F.rank, F.info) == (rank, info)
    assert np.array_equal(mf.factor_permutation(F), perm)
    assert_bitwise(got, want, "pstrf factor")
    if tol > 0:
        assert rank == r


@pytest.mark.parametrize("N", [2, 4])
def test_pstrf_reference_known_answers(mf, ref, N):
    """test/cholesky_pivoted.jl:36-83"""
    A = kat_matrix(N)
    F, got = _run(mf, A, 1e-12, check=True)
    assert mf.factor_kind(F) == "cholesky_pivoted" and mf.factor_status(F) == 0
    assert mf.issuccess(F) and F.rank == 3
    perm = mf.factor_permutation(F)
    assert sorted(perm) == list(range(1, 8)) and perm[0] == 4
    d = mf.factor_diagnostics(F)
    assert d["kind"] == "cholesky_pivoted" and d["rank"] == 3
    assert np.array_equal(d["permutation"], perm)
    assert np.all(mf.factor_rdiag(F)[0, :3] > 0)
    want, wperm, _, _ = ref.pstrf(A, 1e-12)
    assert_bitwise(got, want, "known-answer factor")
    with pytest.raises(mf.ArgumentError):
        mf.cholesky_pivoted_(mf.MFMatrix.from_numpy(A), tol=-1.0, check=False)
    with pytest.raises(mf.ArgumentError):
        mf.cholesky_pivoted_(mf.MFMatrix.from_numpy(A), tol=np.inf, check=False)
    # only the lower triangle is authoritative
    Au = A.copy()
    for c in range(7):
        for r in range(c):
            Au[0, r, c] = 17 + (r + 1) + 3 * (c + 1)
    Fu, gotu = _run(mf, Au, 1e-12, check=True)
    assert Fu.rank == 3 and np.array_equal(mf.factor_permutation(Fu), perm)
    assert_bitwise(gotu, want, "upper triangle replaced")


@pytest.mark.parametrize("N", [2, 3])
def test_pstrf_failures(mf, ref, N):
    A = np.zeros((N, 7, 7))
    A[0] = -np.eye(7)
    F, _ = _run(mf, A)
    assert mf.factor_status(F) > 0 and not mf.issuccess(F) and F.rank == 0
    assert mf.factor_state(F) == "not_posdef"
    with pytest.raises(mf.PosDefException):
        mf.cholesky_pivoted_(mf.MFMatrix.from_numpy(A))
    # a negative pivot later on is reported at its step, as by the oracle
    B = _psd(ref, np.random.default_rng(5), N, 60, 60)
    B[0][np.diag_indices(60)] += 60
    B[0, 45, 45] = -1e6
    F, got = _run(mf, B)
    want, perm, rank, info = ref.pstrf(B)
    assert (F.rank, F.info) == (rank, info) and info > 0
    assert_bitwise(got, want, "failed factor")
    # non-finite lower triangle: status -1, matrix and permutation untouched
    C = kat_matrix(N)
    C[0, 5, 2] = np.inf
    F, got = _run(mf, C)
    assert F.info == -1 and F.rank == 0 and mf.factor_state(F) == "nonfinite_input"
    assert np.array_equal(mf.factor_permutation(F), np.arange(1, 8))
    assert np.array_equal(got.view(np.uint64), C.view(np.uint64))
    with pytest.raises(mf.DomainError):
        mf.cholesky_pivoted_(mf.MFMatrix.from_numpy(C))
    with pytest.raises(mf.DimensionMismatch):
        mf.cholesky_pivoted_(mf.MFMatrix.zeros(N, 5, 4))
    F = mf.cholesky_pivoted_(mf.MFMatrix.zeros(N, 0, 0))
    assert F.rank == 0 and F.info == 0
