"""Device GEMM / SYRK / GEMMT / TRSM against the oracle: bitwise equal in the
matched reduction order, plus semantics (beta == 0 does not read C, inactive
triangles preserved, aliasing and shape errors)."""
import numpy as np
import pytest

from conftest import assert_bitwise
from test_oracle import syn

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1, 1), (5, 3, 7), (23, 25, 17), (64, 64, 64), (67, 130, 45), (129, 17, 200)]


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("shape", SHAPES, ids=str)
def test_gemm_matches_oracle(mf, ref, rng, N, shape):
    m, k, n = shape
    A, B, C0 = syn.randn_mf(rng, N, m, k), syn.randn_mf(rng, N, k, n), syn.randn_mf(rng, N, m, n)
    alpha = syn.randn_mf(rng, N, 1, 1)[:, 0, 0]
    beta = syn.randn_mf(rng, N, 1, 1)[:, 0, 0]
    for strategy, fused in (("auto", True), ("direct", False)):
        cfg = mf.KernelConfig(gemm_strategy=strategy)
        Cd = mf.MFMatrix.from_numpy(C0)
        mf.gemm_(Cd, mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B), alpha, beta, cfg)
        assert_bitwise(Cd.to_numpy(), ref.gemm(A, B, C0, alpha, beta, x3_fused=fused), f"gemm {strategy}")


@pytest.mark.parametrize("N", [2, 3, 4])
def test_gemm_beta_zero_does_not_read_c(mf, ref, rng, N):
    """runtests.jl:315-396: NaN-poisoned destination with beta == 0"""
    A, B = syn.randn_mf(rng, N, 33, 20), syn.randn_mf(rng, N, 20, 31)
    C0 = np.full((N, 33, 31), np.nan)
    Cd = mf.MFMatrix.from_numpy(C0)
    mf.gemm_(Cd, mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B))
    got = Cd.to_numpy()
    assert np.all(np.isfinite(got))
    assert_bitwise(got, ref.gemm(A, B))


@pytest.mark.parametrize("N", [2, 3, 4])
def test_gemm_error_vs_exact(mf, ref, rng, N):
    m, k, n = 96, 300, 80
    A, B = syn.randn_mf(rng, N, m, k, spread=20), syn.randn_mf(rng, N, k, n, spread=20)
    Cd = mf.MFMatrix.zeros(N, m, n)
    mf.gemm_(Cd, mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B))
    rows = rng.integers(0, m, 200)
    cols = rng.integers(0, n, 200)
    err, scale, _ = ref.exact_gemm_check(A, B, Cd.to_numpy(), rows, cols)
    assert np.all(err <= 4096 * k * 2.0 ** (-52 * N) * scale)


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("n,k", [(1, 1), (7, 3), (70, 16), (131, 40)])
def test_syrk_lower_matches_oracle(mf, ref, rng, N, n, k):
    P = syn.randn_mf(rng, N, k, n)
    C0 = syn.randn_mf(rng, N, n, n)
    C0[:, np.triu_indices(n, 1)[0], np.triu_indices(n, 1)[1]] = np.nan  # inactive triangle
    Cd = mf.MFMatrix.from_numpy(C0)
    mf.syrk_(Cd, mf.MFMatrix.from_numpy(P), -1.0, 1.0)
    got = Cd.to_numpy()
    want = ref.syrk_lower(P, C0, -1.0, 1.0)
    assert_bitwise(got, want, "syrk")
    assert np.all(np.isnan(got[:, np.triu_indices(n, 1)[0], np.triu_indices(n, 1)[1]]))


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("n,k", [(5, 2), (70, 17), (100, 64)])
def test_gemmt_lower_matches_oracle(mf, ref, rng, N, n, k):
    A, B = syn.randn_mf(rng, N, n, k), syn.randn_mf(rng, N, n, k)
    C0 = syn.randn_mf(rng, N, n, n)
    Cd = mf.MFMatrix.from_numpy(C0)
    mf.gemmt_(Cd, mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B), 1.0, 0.0)
    assert_bitwise(Cd.to_numpy(), ref.gemmt_lower(A, B, C0, 1.0, 0.0), "gemmt")


def _tri(rng, N, n, lower, unit_scale=True):
    T = syn.randn_mf(rng, N, n, n)
    for i in range(n):
        T[0, i, i] += 4.0 if unit_scale else 0.0
    mask = np.tril(np.ones((n, n), bool)) if lower else np.triu(np.ones((n, n), bool))
    T[:, ~mask] = np.nan  # the inactive triangle is never read
    return T


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("side", ["left", "right"])
@pytest.mark.parametrize("uplo", ["lower", "upper"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("diag", ["nonunit", "unit"])
def test_trsm_matches_oracle(mf, ref, rng, N, side, uplo, trans, diag):
    m, n = (90, 7) if side == "left" else (9, 40)
    na = m if side == "left" else n
    T = _tri(rng, N, na, uplo == "lower")
    B = syn.randn_mf(rng, N, m, n)
    alpha = 1.0 if diag == "unit" else 0.75
    Bd = mf.MFMatrix.from_numpy(B)
    mf.trsm_(Bd, mf.MFMatrix.from_numpy(T), alpha, side, uplo, trans, diag)
    assert_bitwise(Bd.to_numpy(), ref.trsm(B, T, alpha, side, uplo, trans, diag), "trsm")


@pytest.mark.parametrize("N", [2, 4])
@pytest.mark.parametrize("m,n", [(300, 5), (2100, 3), (40, 300)])
def test_trsm_left_kernel_variants(mf, ref, rng, N, m, n):
    """exercises the CTA-per-column (with 8 and 16 rows per thread) and the
    thread-per-column left kernels"""
    T = _tri(rng, N, m, True)
    B = syn.randn_mf(rng, N, m, n)
    Bd = mf.MFMatrix.from_numpy(B)
    mf.trsm_(Bd, mf.MFMatrix.from_numpy(T), 1.0, "left", "lower", "T", "nonunit")
    assert_bitwise(Bd.to_numpy(), ref.trsm(B, T, 1.0, "left", "lower", "T", "nonunit"))


def test_errors(mf, rng):
    A = mf.MFMatrix.from_numpy(syn.randn_mf(rng, 2, 4, 5))
    B = mf.MFMatrix.from_numpy(syn.randn_mf(rng, 2, 6, 3))
    C = mf.MFMatrix.zeros(2, 4, 3)
    with pytest.raises(mf.DimensionMismatch):
        mf.gemm_(C, A, B)
    with pytest.raises(mf.ArgumentError):
        mf.gemm_(A, A, mf.MFMatrix.from_numpy(syn.randn_mf(rng, 2, 5, 5)))
    X = mf.MFMatrix.from_numpy(syn.randn_mf(rng, 3, 4, 4))
    with pytest.raises(mf.ArgumentError):
        mf.gemm_(C, A, X)
    with pytest.raises(mf.ArgumentError):
        mf.syrk_(C, A, uplo="upper")


def test_views_of_one_matrix_do_not_alias(mf, ref, rng):
    """disjoint blocks of one matrix are accepted (as in the reference's
    factorization views), overlapping ones are rejected"""
    N = 2
    M = syn.randn_mf(rng, N, 40, 40)
    Md = mf.MFMatrix.from_numpy(M)
    A21 = Md.view(slice(20, 40), slice(0, 10))
    U12 = Md.view(slice(0, 10), slice(20, 40))
    A22 = Md.view(slice(20, 40), slice(20, 40))
    mf.gemm_(A22, A21, U12, -1.0, 1.0)
    want = M.copy()
    want[:, 20:, 20:] = ref.gemm(M[:, 20:, :10], M[:, :10, 20:], M[:, 20:, 20:], -1.0, 1.0)
    assert_bitwise(Md.to_numpy(), want)
    with pytest.raises(mf.ArgumentError):
        mf.gemm_(Md.view(slice(0, 20), slice(0, 20)), Md.view(slice(10, 30), slice(0, 20)),
                 Md.view(slice(0, 20), slice(20, 40)))
