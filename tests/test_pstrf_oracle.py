"""The oracle's pivoted Cholesky (cholesky_pivoted.jl:65-175) on the CPU,
pinned by the reference's own known answers (test/cholesky_pivoted.jl): the
7 x 7 rank-3 matrix must pivot row 4 first, reveal rank 3 and reproduce
A[p, p]; a negative definite matrix fails at the first pivot; the upper
triangle is not read; non-finite input is returned unchanged."""
import numpy as np
import pytest

from test_oracle import syn


def kat_matrix(N):
    """test/cholesky_pivoted.jl:18-35: original = B B^T, B 7 x 3 integers"""
    B = np.zeros((7, 3))
    B[0, 0], B[1, 1], B[2, 2] = 1, 4, 2
    B[3], B[4], B[5], B[6] = [2, 4, 1], [-1, 1, 3], [3, -2, 1], [1, 2, -2]
    A = np.zeros((N, 7, 7))
    A[0] = B @ B.T  # small integers: exact
    return A


@pytest.mark.parametrize("N", [2, 3, 4])
def test_oracle_pstrf_reference_known_answers(ref, N):
    A = kat_matrix(N)
    F, perm, rank, info = ref.pstrf(A, tol=1e-12, nthreads=1)
    assert info == 0 and rank == 3
    assert sorted(perm) == list(range(1, 8)) and perm[0] == 4
    L = np.tril(F)[:, :, :rank]
    LLt = ref.gemm(L, np.ascontiguousarray(L.transpose(0, 2, 1)), nthreads=1)
    p = perm - 1
    err = np.max(np.abs(ref.to_double(LLt - A[:, p][:, :, p])))
    assert err <= 1e-20 * max(1.0, np.max(np.abs(A[0])))
    assert np.all(F[0][np.arange(rank), np.arange(rank)] > 0)
    # only the lower triangle is authoritative
    Au = A.copy()
    for c in range(7):
        for r in range(c):
            Au[0, r, c] = 17 + (r + 1) + 3 * (c + 1)
    F2, perm2, rank2, info2 = ref.pstrf(Au, tol=1e-12, nthreads=1)
    assert rank2 == 3 and np.array_equal(perm2, perm) and info2 == 0
    assert np.array_equal(np.tril(F2).view(np.uint64), np.tril(F).view(np.uint64))


@pytest.mark.parametrize("N", [2, 4])
def test_oracle_pstrf_failures(ref, N):
    A = np.zeros((N, 7, 7))
    A[0] = -np.eye(7)
    _, _, rank, info = ref.pstrf(A, nthreads=1)
    assert info > 0 and rank == 0
    A = kat_matrix(N)
    A[0, 5, 2] = np.nan
    F, perm, rank, info = ref.pstrf(A, nthreads=1)
    assert info == -1 and rank == 0 and list(perm) == list(range(1, 8))
    assert np.array_equal(np.isnan(F), np.isnan(A)) and np.array_equal(F[~np.isnan(F)],
                                                                        A[~np.isnan(A)])


@pytest.mark.parametrize("N", [2, 3])
def test_oracle_pstrf_rank_deficient(ref, N):
    """a rank-r PSD matrix: zero tolerance ends on a non-positive roundoff
    pivot at or after r (status), a relative tolerance reveals rank r"""
    rng = np.random.default_rng(11)
    n, r = 40, 12
    R = syn.randn_mf(rng, N, n, r)
    A = ref.gemm(R, np.ascontiguousarray(R.transpose(0, 2, 1)), nthreads=1)
    _, _, rank, info = ref.pstrf(A, tol=1e-12, nthreads=1)
    assert rank == r and info == 0
    _, _, rank0, info0 = ref.pstrf(A, nthreads=1)
    assert rank0 >= r and (info0 == 0 or info0 == rank0 + 1)
