"""Device residual, mixed residual, normwise backward error and refinement
correction (src/residual.jl) against the oracle."""
import numpy as np
import pytest

from conftest import assert_bitwise
from test_oracle import syn

pytestmark = pytest.mark.gpu


def _mirror(S, uplo):
    """full symmetric matrix from the authoritative triangle"""
    if uplo == "lower":
        return np.tril(S) + np.transpose(np.tril(S, -1), (0, 2, 1))
    return np.triu(S) + np.transpose(np.triu(S, 1), (0, 2, 1))


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("uplo", ["general", "lower", "upper"])
@pytest.mark.parametrize("vector", [False, True])
def test_residual_matches_oracle(mf, ref, rng, N, uplo, vector):
    n, nrhs = 37, (1 if vector else 5)
    A = syn.randn_mf(rng, N, n, n)
    X, B = syn.randn_mf(rng, N, n, nrhs), syn.randn_mf(rng, N, n, nrhs)
    A_in = A.copy()
    if uplo == "lower":
        iu = np.triu_indices(n, 1)
        A_in[:, iu[0], iu[1]] = np.nan
    elif uplo == "upper":
        il = np.tril_indices(n, -1)
        A_in[:, il[0], il[1]] = np.nan
    Ad = mf.MFMatrix.from_numpy(A_in)
    if vector:
        Xd, Bd = mf.MFMatrix.from_numpy(X[:, :, 0]), mf.MFMatrix.from_numpy(B[:, :, 0])
        Rd = mf.MFMatrix.zeros(N, n)
    else:
        Xd, Bd = mf.MFMatrix.from_numpy(X), mf.MFMatrix.from_numpy(B)
        Rd = mf.MFMatrix.zeros(N, n, nrhs)
    mf.residual_(Rd, Ad, Xd, Bd, uplo=uplo)
    Afull = A if uplo == "general" else _mirror(A_in, uplo)
    fused = uplo == "general" and not vector
    want = ref.gemm(Afull, X, B, -1.0, 1.0, x3_fused=fused)
    got = Rd.to_numpy()
    assert_bitwise(got[:, :, None] if vector else got, want, "residual")
    # r may be b itself
    mf.residual_(Bd, Ad, Xd, Bd, uplo=uplo)
    assert_bitwise(Bd.to_numpy(), got)


@pytest.mark.parametrize("src,res", [(1, 2), (1, 4), (2, 3), (2, 4), (3, 4)])
@pytest.mark.parametrize("uplo", ["general", "lower"])
def test_residual_mixed_matches_oracle(mf, ref, rng, src, res, uplo):
    n, nrhs = 29, 3
    A = syn.randn_mf(rng, max(src, 1), n, n)[:src]
    X = syn.randn_mf(rng, max(src, 1), n, nrhs)[:src]
    B = syn.randn_mf(rng, max(src, 1), n, nrhs)[:src]
    Rd = mf.MFMatrix.zeros(res, n, nrhs)
    mf.residual_mixed_(Rd, mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(X),
                       mf.MFMatrix.from_numpy(B), uplo=uplo)
    assert_bitwise(Rd.to_numpy(), ref.residual_mixed(A, X, B, res, uplo), "residual_mixed")


@pytest.mark.parametrize("N", [2, 4])
def test_backward_error_value_and_edge_cases(mf, ref, rng, N):
    n = 30
    A = syn.randn_mf(rng, N, n, n)
    X, B = syn.randn_mf(rng, N, n, 2), syn.randn_mf(rng, N, n, 2)
    R = ref.gemm(A, X, B, -1.0, 1.0)
    Ad, Xd, Bd, Rd = (mf.MFMatrix.from_numpy(M) for M in (A, X, B, R))
    vals = mf.normwise_backward_error(Ad, Xd, Bd, Rd)
    Ad0, Xd0, Bd0, Rd0 = (ref.to_double(M) for M in (A, X, B, R))
    an = np.max(np.sum(np.abs(Ad0), axis=1))
    for j in range(2):
        want = np.max(np.abs(Rd0[:, j])) / (an * np.max(np.abs(Xd0[:, j])) + np.max(np.abs(Bd0[:, j])))
        assert abs(vals[j][0] - want) <= 1e-12 * want
    Z = mf.MFMatrix.zeros(N, n, 1)
    assert mf.normwise_backward_error(mf.MFMatrix.zeros(N, n, n), Z, Z, Z)[0][0] == 0.0
    R1 = np.zeros((N, n, 1))
    R1[0, 0, 0] = 1.0
    v = mf.normwise_backward_error(mf.MFMatrix.zeros(N, n, n), Z, Z, mf.MFMatrix.from_numpy(R1))
    assert v[0][0] == np.inf
    Xn = X[:, :, :1].copy()
    Xn[0, 3, 0] = np.nan
    v = mf.normwise_backward_error(Ad, mf.MFMatrix.from_numpy(Xn), mf.MFMatrix.from_numpy(B[:, :, :1]),
                                   mf.MFMatrix.from_numpy(R[:, :, :1]))
    assert np.isnan(v[0][0])


@pytest.mark.parametrize("N", [2, 3])
def test_kat_badly_scaled_lu_backward_error(mf, ref, N):
    """adversarial.jl:94-117: row/column scales span 2^600, backward error
    <= 4096 eps(T)"""
    core = np.array([[4.0, 1, 0, 1], [2, 5, 1, 0], [0, 2, 6, 1], [1, 0, 1, 7]])
    rs = 2.0 ** np.array([-200, -60, 60, 200])
    cs = 2.0 ** np.array([100, 30, -30, -100])
    A = np.zeros((N, 4, 4))
    A[0] = rs[:, None] * core * cs[None, :]
    truth = np.zeros((N, 4, 1))
    truth[0, :, 0] = [1, -2, 3, -1]
    rhs = ref.gemm(A, truth)
    Ad = mf.MFMatrix.from_numpy(A)
    F = mf.lu_(Ad.copy(), config=mf.KernelConfig(lu_block=2))
    Xd = mf.solve(F, mf.MFMatrix.from_numpy(rhs[:, :, 0]))
    Bd = mf.MFMatrix.from_numpy(rhs[:, :, 0])
    Rd = mf.MFMatrix.zeros(N, 4)
    mf.residual_(Rd, Ad, Xd, Bd)
    be = mf.normwise_backward_error(Ad, Xd, Bd, Rd)
    assert be[0] <= 4096 * 2.0 ** (-52 * N)


@pytest.mark.parametrize("N", [2, 4])
def test_refinement_correction(mf, ref, rng, N):
    n = 25
    S = syn.spd_matrix(rng, N, n, ref.gemm)
    S = np.tril(S) + np.transpose(np.tril(S, -1), (0, 2, 1))
    F = mf.cholesky_(mf.MFMatrix.from_numpy(S))
    r = syn.randn_mf(rng, N, n, 2)
    d = mf.MFMatrix.zeros(N, n, 2)
    mf.refinement_correction_(d, F, mf.MFMatrix.from_numpy(r))
    L, _ = ref.potrf(S)
    assert_bitwise(d.to_numpy(), ref.potrs(L, r))
