"""trmm! and syrk_packed! on the device against the oracle, bit for bit:
every side / triangle / transpose / diagonal combination with NaN and Inf in
the entries that must not be read, views, reduction bounds, stale packed
storage under beta = 0, and the argument errors of the reference's tests."""
import numpy as np
import pytest

from conftest import assert_bitwise
from test_oracle import syn
from test_trmm_packed_oracle import COMBOS, _triangular

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("side,uplo,trans,diag", COMBOS)
@pytest.mark.parametrize("order,rhs", [(7, 5), (150, 90)], ids=str)
def test_trmm_matches_oracle(mf, ref, rng, N, side, uplo, trans, diag, order, rhs):
    A = _triangular(rng, N, order, uplo, diag == "unit")
    B = syn.randn_mf(rng, N, order, rhs) if side == "left" else syn.randn_mf(rng, N, rhs, order)
    alpha = syn.randn_mf(rng, N, 1, 1)[:, 0, 0]
    Bd = mf.MFMatrix.from_numpy(B)
    mf.trmm_(Bd, mf.MFMatrix.from_numpy(A), alpha, side=side, uplo=uplo, trans=trans, diag=diag)
    want = ref.trmm(B, A, alpha, side, uplo, trans, diag)
    got = Bd.to_numpy()
    assert np.all(np.isfinite(got))
    assert_bitwise(got, want, f"trmm {side} {uplo} {trans} {diag}")


def test_trmm_views(mf, ref, rng):
    """B and A as sub-matrix views of larger storage; the rest is untouched"""
    N = 3
    M = syn.randn_mf(rng, N, 300, 260)
    Md = mf.MFMatrix.from_numpy(M)
    Bv = Md.view(slice(5, 135), slice(7, 77))      # 130 x 70
    Av = Md.view(slice(140, 270), slice(100, 230))  # 130 x 130
    mf.trmm_(Bv, Av, 1.0, side="left", uplo="upper", trans="T")
    want = M.copy()
    want[:, 5:135, 7:77] = ref.trmm(M[:, 5:135, 7:77], M[:, 140:270, 100:230], 1.0, "left",
                                    "upper", "T")
    assert_bitwise(Md.to_numpy(), want, "trmm views")


def test_trmm_errors(mf):
    N, order = 2, 7
    sq = mf.MFMatrix.zeros(N, order, order)
    with pytest.raises(mf.DimensionMismatch):
        mf.trmm_(mf.MFMatrix.zeros(N, order - 1, 2), sq, side="left")
    with pytest.raises(mf.DimensionMismatch):
        mf.trmm_(mf.MFMatrix.zeros(N, 2, order - 1), sq, side="right")
    with pytest.raises(mf.DimensionMismatch):
        mf.trmm_(mf.MFMatrix.zeros(N, order, 2), mf.MFMatrix.zeros(N, order, order - 1))
    for kw in ("side", "uplo", "trans", "diag"):
        with pytest.raises(mf.ArgumentError):
            mf.trmm_(mf.MFMatrix.zeros(N, order, 2), sq, **{kw: "bad"})
    with pytest.raises(mf.ArgumentError):
        mf.trmm_(sq, sq)
    Bz = mf.MFMatrix.zeros(N, order, 0)
    mf.trmm_(Bz, sq)  # empty B: nothing to do


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("kp,n,rf,rl", [(11, 9, 2, 10), (300, 200, 17, 250), (64, 1, 1, 64),
                                        (5, 70, 3, 3)], ids=str)
def test_syrk_packed_matches_oracle(mf, ref, rng, N, kp, n, rf, rl):
    P = syn.randn_mf(rng, N, kp, n)
    L = n * (n + 1) // 2
    init = syn.randn_mf(rng, N, L, 1)[:, :, 0]
    alpha, beta = syn.randn_mf(rng, N, 1, 1)[:, 0, 0], syn.randn_mf(rng, N, 1, 1)[:, 0, 0]
    out = mf.MFMatrix.from_numpy(init)
    mf.syrk_packed_(out, mf.MFMatrix.from_numpy(P), alpha, beta, reduction_first=rf,
                    reduction_last=rl)
    want = ref.syrk_packed(init, P, alpha, beta, reduction_first=rf, reduction_last=rl)
    assert_bitwise(out.to_numpy(), want, "syrk_packed")
    # beta = 0 never reads the destination
    stale = mf.MFMatrix.from_numpy(np.full((N, L), np.nan))
    clean = mf.MFMatrix.zeros(N, L)
    mf.syrk_packed_(stale, mf.MFMatrix.from_numpy(P))
    mf.syrk_packed_(clean, mf.MFMatrix.from_numpy(P))
    assert_bitwise(stale.to_numpy(), clean.to_numpy(), "stale")
    assert_bitwise(clean.to_numpy(), ref.syrk_packed(np.zeros((N, L)), P), "beta 0")


def test_syrk_packed_errors(mf):
    N = 2
    P = mf.MFMatrix.zeros(N, 11, 9)
    with pytest.raises(mf.DimensionMismatch):
        mf.syrk_packed_(mf.MFMatrix.zeros(N, 44), P)
    with pytest.raises(mf.BoundsError):
        mf.syrk_packed_(mf.MFMatrix.zeros(N, 45), P, reduction_first=0, reduction_last=10)
    with pytest.raises(mf.BoundsError):
        mf.syrk_packed_(mf.MFMatrix.zeros(N, 45), P, reduction_first=2, reduction_last=12)
    with pytest.raises(mf.BoundsError):
        mf.syrk_packed_(mf.MFMatrix.zeros(N, 45), P, reduction_first=5, reduction_last=4)
