"""gemv!, symv! and mfdot on the device against the oracle's GEMM in the
same ascending order (plain network): bit for bit, with alpha/beta, both
transposes and triangles, views and edge cases."""
import numpy as np
import pytest

from conftest import assert_bitwise
from test_oracle import syn

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("m,n", [(1, 1), (37, 90), (300, 129)], ids=str)
def test_gemv_matches_oracle(mf, ref, rng, N, trans, m, n):
    A = syn.randn_mf(rng, N, m, n)
    lx, ly = (n, m) if trans == "N" else (m, n)
    x, y0 = syn.randn_mf(rng, N, lx, 1), syn.randn_mf(rng, N, ly, 1)
    alpha, beta = syn.randn_mf(rng, N, 1, 1)[:, 0, 0], syn.randn_mf(rng, N, 1, 1)[:, 0, 0]
    Aop = A if trans == "N" else np.ascontiguousarray(A.transpose(0, 2, 1))
    for a, b in ((1.0, 0.0), (alpha, beta)):
        yd = mf.MFMatrix.from_numpy(y0[:, :, 0])
        mf.gemv_(yd, mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(x[:, :, 0]), a, b,
                 trans=trans)
        want = ref.gemm(Aop, x, y0.copy(), a, b, x3_fused=False)[:, :, 0]
        assert_bitwise(yd.to_numpy(), want, f"gemv {trans}")


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("uplo", ["lower", "upper"])
def test_symv_reads_one_triangle(mf, ref, rng, N, uplo):
    n = 150
    S = syn.randn_mf(rng, N, n, n)
    Sfull = np.tril(S) + np.transpose(np.tril(S, -1), (0, 2, 1)) if uplo == "lower" else \
        np.triu(S) + np.transpose(np.triu(S, 1), (0, 2, 1))
    Sin = S.copy()
    other = np.triu_indices(n, 1) if uplo == "lower" else np.tril_indices(n, -1)
    Sin[:, other[0], other[1]] = np.nan  # the other triangle is never read
    x = syn.randn_mf(rng, N, n, 1)
    yd = mf.MFMatrix.zeros(N, n)
    mf.symv_(yd, mf.MFMatrix.from_numpy(Sin), mf.MFMatrix.from_numpy(x[:, :, 0]), uplo=uplo)
    assert_bitwise(yd.to_numpy(), ref.gemm(Sfull, x, x3_fused=False)[:, :, 0], "symv")


@pytest.mark.parametrize("N", [2, 3, 4])
def test_mfdot_vectors_and_matrices(mf, ref, rng, N):
    x, y = syn.randn_mf(rng, N, 500, 1), syn.randn_mf(rng, N, 500, 1)
    got = mf.mfdot(mf.MFMatrix.from_numpy(x[:, :, 0]), mf.MFMatrix.from_numpy(y[:, :, 0]))
    want = ref.gemm(np.ascontiguousarray(x.transpose(0, 2, 1)), y, x3_fused=False)[:, 0, 0]
    assert_bitwise(got, want, "mfdot vector")
    # Frobenius product of views (ld > rows): column-major order
    X, Y = syn.randn_mf(rng, N, 40, 30), syn.randn_mf(rng, N, 40, 30)
    Xv = mf.MFMatrix.from_numpy(X).view(slice(3, 20), slice(2, 25))
    Yv = mf.MFMatrix.from_numpy(Y).view(slice(10, 27), slice(4, 27))
    xs = X[:, 3:20, 2:25].transpose(0, 2, 1).reshape(N, 1, -1)
    ys = Y[:, 10:27, 4:27].transpose(0, 2, 1).reshape(N, -1, 1)
    assert_bitwise(mf.mfdot(Xv, Yv), ref.gemm(np.ascontiguousarray(xs), np.ascontiguousarray(ys),
                                               x3_fused=False)[:, 0, 0], "mfdot matrix")


def test_vector_kernel_errors(mf, rng):
    N = 2
    A = mf.MFMatrix.from_numpy(syn.randn_mf(rng, N, 5, 4))
    with pytest.raises(mf.DimensionMismatch):
        mf.gemv_(mf.MFMatrix.zeros(N, 5), A, mf.MFMatrix.zeros(N, 5))
    with pytest.raises(mf.ArgumentError):
        mf.gemv_(mf.MFMatrix.zeros(N, 5), A, mf.MFMatrix.zeros(N, 4), trans="C")
    with pytest.raises(mf.DimensionMismatch):
        mf.symv_(mf.MFMatrix.zeros(N, 5), A, mf.MFMatrix.zeros(N, 4))
    with pytest.raises(mf.DimensionMismatch):
        mf.mfdot(mf.MFMatrix.zeros(N, 5), mf.MFMatrix.zeros(N, 4))
    assert np.all(mf.mfdot(mf.MFMatrix.zeros(N, 0), mf.MFMatrix.zeros(N, 0)) == 0)
