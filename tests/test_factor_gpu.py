"""Device Cholesky / LU and solves against the oracle (bitwise in the matched
order), failure statuses and diagnostics known answers."""
import numpy as np
import pytest

from conftest import assert_bitwise
from test_oracle import syn

pytestmark = pytest.mark.gpu


def _spd(ref, rng, N, n):
    S = syn.spd_matrix(rng, N, n, ref.gemm)
    return np.tril(S) + np.transpose(np.tril(S, -1), (0, 2, 1))


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("n,block", [(1, 16), (13, 16), (37, 16), (100, 16), (150, 32), (50, 4)])
def test_cholesky_and_solve_match_oracle(mf, ref, rng, N, n, block):
    S = _spd(ref, rng, N, n)
    S_in = S.copy()
    S_in[:, np.triu_indices(n, 1)[0], np.triu_indices(n, 1)[1]] = np.nan  # upper never read
    Sd = mf.MFMatrix.from_numpy(S_in)
    F = mf.cholesky_(Sd, config=mf.KernelConfig(cholesky_block=block))
    L, info = ref.potrf(S_in, block=block)
    assert mf.factor_status(F) == info == 0
    assert_bitwise(np.tril(Sd.to_numpy()), np.tril(L), "cholesky factor")
    B = syn.randn_mf(rng, N, n, 5)
    X = mf.solve(F, mf.MFMatrix.from_numpy(B)).to_numpy()
    assert_bitwise(X, ref.potrs(L, B), "cholesky solve")
    be = ref.backward_error(S, X, B)
    assert np.all(be < 4096 * n * 2.0 ** (-52 * N))


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("m,n,block", [(1, 1, 16), (20, 20, 16), (70, 70, 16), (90, 60, 16),
                                       (60, 90, 16), (45, 45, 5)])
def test_lu_and_solve_match_oracle(mf, ref, rng, N, m, n, block):
    A = syn.randn_mf(rng, N, m, n)
    Ad = mf.MFMatrix.from_numpy(A)
    F = mf.lu_(Ad, config=mf.KernelConfig(lu_block=block))
    LU, piv, info = ref.getrf(A, block=block)
    assert mf.factor_status(F) == info == 0
    assert np.array_equal(mf.factor_pivots(F), piv)
    assert_bitwise(Ad.to_numpy(), LU, "lu factor")
    if m == n:
        B = syn.randn_mf(rng, N, n, 4)
        X = mf.solve(F, mf.MFMatrix.from_numpy(B)).to_numpy()
        assert_bitwise(X, ref.getrs(LU, piv, B), "lu solve")


@pytest.mark.parametrize("N", [2, 3, 4])
def test_cholesky_failure_status(mf, N):
    """adversarial.jl:76-92: the Schur complement fails at pivot 2"""
    delta = 16 * 2.0 ** (-52 * N)
    A = np.zeros((N, 2, 2))
    A[0] = [[1, np.nan], [1, 1]]
    A[1, 1, 1] = -delta if N >= 2 else 0
    F = mf.cholesky_(mf.MFMatrix.from_numpy(A), check=False,
                     config=mf.KernelConfig(cholesky_block=2))
    assert mf.factor_status(F) == 2
    assert mf.factor_state(F) == "not_posdef"
    assert mf.factor_diagnostics(F)["failure_location"] == 2
    with pytest.raises(mf.PosDefException):
        mf.cholesky_(mf.MFMatrix.from_numpy(A), config=mf.KernelConfig(cholesky_block=2))
    with pytest.raises(mf.PosDefException):
        mf.solve(F, mf.MFMatrix.from_numpy(np.ones((N, 2))))


@pytest.mark.parametrize("N", [2, 4])
def test_nonfinite_inputs(mf, rng, N):
    A = syn.randn_mf(rng, N, 6, 6)
    A[0, 4, 1] = np.nan
    F = mf.cholesky_(mf.MFMatrix.from_numpy(A), check=False)
    assert mf.factor_status(F) == -1 and mf.factor_state(F) == "nonfinite_input"
    with pytest.raises(mf.DomainError):
        mf.cholesky_(mf.MFMatrix.from_numpy(A))
    G = mf.lu_(mf.MFMatrix.from_numpy(A), check=False)
    assert mf.factor_status(G) == -1
    with pytest.raises(mf.DomainError):
        mf.lu_(mf.MFMatrix.from_numpy(A))


@pytest.mark.parametrize("N", [2, 3, 4])
def test_lu_zero_pivot(mf, N):
    A = np.zeros((N, 3, 3))
    A[0] = [[1, 2, 3], [2, 4, 6], [1, 1, 1]]
    F = mf.lu_(mf.MFMatrix.from_numpy(A), check=False)
    assert mf.factor_status(F) > 0 and mf.factor_state(F) == "singular"
    with pytest.raises(mf.SingularException):
        mf.lu_(mf.MFMatrix.from_numpy(A))


@pytest.mark.parametrize("N", [2, 3, 4])
def test_kat_diagonal_spread(mf, ref, N):
    """adversarial.jl:37-52: exact solve and diagonal_spread == 2^300"""
    ex = [-300, -150, 0, 150, 300]
    S = np.zeros((N, 5, 5))
    for i, e in enumerate(ex):
        S[0, i, i] = 2.0 ** e
    truth = np.zeros((N, 5, 1))
    truth[0, :, 0] = [1, -2, 3, -4, 5]
    rhs = ref.gemm(S, truth)
    F = mf.cholesky_(mf.MFMatrix.from_numpy(S), config=mf.KernelConfig(cholesky_block=2))
    X = mf.solve(F, mf.MFMatrix.from_numpy(rhs)).to_numpy()
    assert_bitwise(X, truth)
    d = mf.factor_diagnostics(F)
    assert d["diagonal_spread"][0] == 2.0 ** 300 and not np.any(d["diagonal_spread"][1:])
    assert d["finite"] and d["accepted_pivots"] == 5


@pytest.mark.parametrize("N", [2, 3, 4])
def test_kat_wilkinson_growth(mf, N):
    """adversarial.jl:148-171: pivot growth 128 exactly"""
    n = 8
    W = np.zeros((N, n, n))
    for r in range(n):
        W[0, r, r] = 1.0
        W[0, r, n - 1] = 1.0
        W[0, r, :r] = -1.0
    F = mf.lu_(mf.MFMatrix.from_numpy(W), config=mf.KernelConfig(lu_block=2))
    d = mf.factor_diagnostics(F)
    assert d["pivot_growth"][0] == 128.0 and not np.any(d["pivot_growth"][1:])
    assert d["maximum_u"][0] == 128.0


@pytest.mark.parametrize("N", [2, 3, 4])
def test_kat_tiny_first_pivot(mf, N):
    """adversarial.jl:119-130: the 2^-300 leading entry is not the pivot"""
    A = np.zeros((N, 2, 2))
    A[0] = [[2.0 ** -300, 1], [1, 1]]
    F = mf.lu_(mf.MFMatrix.from_numpy(A), config=mf.KernelConfig(lu_block=2))
    assert mf.factor_diagnostics(F)["pivots"][0] == 2


@pytest.mark.parametrize("N", [2, 4])
@pytest.mark.parametrize("kind", ["cholesky", "lu", "ldlt"])
def test_fast_solve_order(mf, ref, rng, N, kind):
    """solve_order="fast" (wavefront backward substitution): deterministic and
    within the reference tolerance, not bitwise the matched order"""
    n = 130
    S = _spd(ref, rng, N, n)
    B = syn.randn_mf(rng, N, n, 4)
    fac = {"cholesky": mf.cholesky_, "lu": mf.lu_, "ldlt": mf.ldlt_}[kind]
    F = fac(mf.MFMatrix.from_numpy(S))
    fast = mf.KernelConfig(solve_order="fast")
    X1 = mf.solve(F, mf.MFMatrix.from_numpy(B), config=fast).to_numpy()
    X2 = mf.solve(F, mf.MFMatrix.from_numpy(B), config=fast).to_numpy()
    assert np.array_equal(X1.view(np.uint64), X2.view(np.uint64))
    assert np.all(ref.backward_error(S, X1, B) < 4096 * n * 2.0 ** (-52 * N))
    # the handle returns to the matched order afterwards
    Xm = mf.solve(F, mf.MFMatrix.from_numpy(B)).to_numpy()
    if kind == "cholesky":
        L, _ = ref.potrf(S)
        assert_bitwise(Xm, ref.potrs(L, B))
