"""Householder QR, rank-revealing QR (both of the reference's routes),
apply_q!, solve_r!, numerical_rank and the square QR solve on the device,
bit for bit against the oracle, plus the reference's known answers."""
import numpy as np
import pytest

from conftest import assert_bitwise
from test_oracle import syn
from test_qr_oracle import mf_of, sincos_panel

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1), (15, 7), (7, 15), (9, 9), (40, 30), (100, 100), (20, 900), (300, 200),
          (64, 300)]


def _dev_qr(mf, A, pivoted):
    Ad = mf.MFMatrix.from_numpy(A)
    F = (mf.rrqr_ if pivoted else mf.qr_)(Ad, check=False)
    return F, Ad.to_numpy(), F.tau.cpu().numpy(), mf.factor_permutation(F)


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("shape", SHAPES, ids=str)
@pytest.mark.parametrize("pivoted", [False, True], ids=["qr", "rrqr"])
def test_qr_matches_oracle(mf, ref, rng, N, shape, pivoted):
    m, n = shape
    A = syn.randn_mf(rng, N, m, n, spread=4)
    F, got, tau, perm = _dev_qr(mf, A, pivoted)
    want, wtau, wperm, info = (ref.rrqr if pivoted else ref.qr)(A)
    assert F.info == info == 0
    assert np.array_equal(perm, wperm)
    assert_bitwise(tau, wtau, "tau")
    assert_bitwise(got, want, "factors")
    assert mf.numerical_rank(F) == ref.qr_numerical_rank(want)
    assert mf.numerical_rank(F, rtol=1e-20) == ref.qr_numerical_rank(want, rtol=1e-20)


@pytest.mark.parametrize("N", [2, 4])
def test_rrqr_reference_known_answers(mf, ref, N):
    """runtests.jl:829-870 and qr_delayed_norm.jl: panel breaks, re-entering
    columns and delayed norm rebuilds on the blocked route"""
    A = sincos_panel(N)
    F, got, tau, perm = _dev_qr(mf, A, True)
    want, wtau, wperm, _ = ref.rrqr(A)
    assert np.array_equal(perm, wperm)
    assert_bitwise(got, want, "sin/cos panel")
    assert mf.numerical_rank(F, rtol=1e-12) == 31
    if N == 4:
        assert mf.numerical_rank(F, rtol=1e-30) == 40
        r = np.arange(1, 257)[:, None].astype(float)
        c = np.arange(1, 31)[None, :].astype(float)
        core = np.sin(0.013 * r + 0.23 * c) + 0.21 * np.cos(0.005 * r * c)
        D = np.zeros((256, 64))
        D[:, :30] = core
        D[:, 30:40] = core[:, 1:11]
        Fd, gotd, _, permd = _dev_qr(mf, mf_of(D, N), True)
        wd, _, wpd, _ = ref.rrqr(mf_of(D, N))
        assert np.array_equal(permd, wpd)
        assert_bitwise(gotd, wd, "duplicated columns")
        assert mf.numerical_rank(Fd, rtol=2.0 ** -104) == 30
    E = mf_of(np.eye(8)[:, :4], N)
    assert list(_dev_qr(mf, E, True)[3]) == [1, 2, 3, 4]
    S = np.random.default_rng(3).standard_normal((10, 4)) * np.array([1e-100, 1e100, 1e-40, 1e40])
    Fs, _, _, ps = _dev_qr(mf, mf_of(S, N), True)
    assert ps[0] == 2 and mf.numerical_rank(Fs) == 4
    assert mf.numerical_rank(mf.rrqr_(mf.MFMatrix.zeros(N, 5, 8))) == 0


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("trans", ["N", "T"])
def test_apply_q_matches_oracle(mf, ref, rng, N, trans):
    for m, n in ((40, 30), (30, 40), (300, 200)):
        A = syn.randn_mf(rng, N, m, n)
        F = mf.rrqr_(mf.MFMatrix.from_numpy(A))
        D = syn.randn_mf(rng, N, m, 5)
        Dd = mf.MFMatrix.from_numpy(D)
        mf.apply_q_(Dd, F, trans=trans)
        want = ref.apply_q(F.factors.to_numpy(), F.tau.cpu().numpy(), D, trans)
        assert_bitwise(Dd.to_numpy(), want, f"apply_q {trans}")
        v = syn.randn_mf(rng, N, m, 1)[:, :, 0]
        vd = mf.MFMatrix.from_numpy(v)
        mf.apply_q_(vd, F, trans=trans)
        wantv = ref.apply_q(F.factors.to_numpy(), F.tau.cpu().numpy(), v[:, :, None], trans)
        assert_bitwise(vd.to_numpy(), wantv[:, :, 0], "apply_q vector")


@pytest.mark.parametrize("N", [2, 4])
def test_qr_solves(mf, ref, rng, N):
    n = 60
    A = syn.randn_mf(rng, N, n, n)
    F = mf.rrqr_(mf.MFMatrix.from_numpy(A))
    Fn, taun, permn = F.factors.to_numpy(), F.tau.cpu().numpy(), mf.factor_permutation(F)
    B = syn.randn_mf(rng, N, n, 3)
    X = mf.ldiv_(mf.MFMatrix.from_numpy(B), F).to_numpy()
    Y = ref.apply_q(Fn, taun, B, "T")
    Y = ref.trsm(Y, np.triu(Fn), 1.0, "left", "upper", "N", "nonunit")
    want = np.empty_like(Y)
    want[:, permn - 1, :] = Y
    assert_bitwise(X, want, "square QR solve")
    be = ref.backward_error(A, X, B)
    assert np.all(be < 4096 * n * 2.0 ** (-52 * N))
    # solve_r! with a caller rank, both transposes
    for trans in ("N", "T"):
        Bk = syn.randn_mf(rng, N, 20, 2)
        got = mf.solve_r_(mf.MFMatrix.from_numpy(Bk), F, 20, trans=trans).to_numpy()
        wantk = ref.trsm(Bk, np.ascontiguousarray(np.triu(Fn)[:, :20, :20]), 1.0, "left", "upper",
                         trans, "nonunit")
        assert_bitwise(got, wantk, f"solve_r {trans}")
    with pytest.raises(mf.ArgumentError):
        mf.solve_r_(mf.MFMatrix.zeros(N, 3, 1), F, n + 1)
    with pytest.raises(mf.DimensionMismatch):
        mf.solve_r_(mf.MFMatrix.zeros(N, 3, 1), F, 4)
    Z = np.zeros((N, 6, 6))
    Z[0] = np.diag([1.0, 2.0, 0.0, 4.0, 5.0, 6.0])
    Fz = mf.qr_(mf.MFMatrix.from_numpy(Z))
    with pytest.raises(mf.SingularException):
        mf.solve_r_(mf.MFMatrix.zeros(N, 4, 1), Fz, 4)
    with pytest.raises(mf.SingularException):
        mf.ldiv_(mf.MFMatrix.zeros(N, 6, 1), Fz)
    with pytest.raises(mf.DimensionMismatch):
        mf.ldiv_(mf.MFMatrix.zeros(N, 7, 1), mf.rrqr_(mf.MFMatrix.from_numpy(
            syn.randn_mf(rng, N, 7, 5))))


@pytest.mark.parametrize("N", [2, 3])
def test_qr_fixed_permutation(mf, ref, rng, N):
    """qr_fixed_permutation.jl: the caller's order equals an explicit reorder"""
    m, n = 20, 12
    A = syn.randn_mf(rng, N, m, n)
    perm = np.array([3, 1, 12, 5, 7, 2, 4, 6, 8, 9, 11, 10])
    F1 = mf.qr_(mf.MFMatrix.from_numpy(A), perm)
    want, wtau, _, _ = ref.qr(np.ascontiguousarray(A[:, :, perm - 1]))
    assert_bitwise(F1.factors.to_numpy(), want, "fixed order")
    assert np.array_equal(mf.factor_permutation(F1), perm)
    with pytest.raises(mf.DimensionMismatch):
        mf.qr_(mf.MFMatrix.from_numpy(A), np.ones(n + 1, dtype=int))
    with pytest.raises(mf.ArgumentError):
        mf.qr_(mf.MFMatrix.from_numpy(A), np.r_[1, 1, np.arange(3, n + 1)])
    with pytest.raises(mf.ArgumentError):
        mf.qr_(mf.MFMatrix.from_numpy(A), np.r_[0, np.arange(2, n + 1)])


def test_qr_nonfinite_and_diagnostics(mf, ref, rng):
    N = 2
    A = syn.randn_mf(rng, N, 9, 7)
    A[1, 4, 2] = np.nan
    for fn in (mf.qr_, mf.rrqr_):
        Ad = mf.MFMatrix.from_numpy(A)
        F = fn(Ad, check=False)
        assert F.info == -1 and mf.factor_state(F) == "nonfinite_input"
        assert np.all(F.tau.cpu().numpy() == 0)
        assert np.array_equal(mf.factor_permutation(F), np.arange(1, 8))
        got = Ad.to_numpy()
        assert np.array_equal(np.isnan(got), np.isnan(A))
        with pytest.raises(mf.DomainError):
            fn(mf.MFMatrix.from_numpy(A))
        with pytest.raises(mf.ArgumentError):
            mf.apply_q_(mf.MFMatrix.zeros(N, 9, 1), F)
    B = syn.randn_mf(rng, N, 12, 5)
    F = mf.rrqr_(mf.MFMatrix.from_numpy(B))
    d = mf.factor_diagnostics(F, rtol=1e-20)
    assert d["kind"] == "qr" and d["success"] and d["rank_at_threshold"] == 5
    assert np.array_equal(d["permutation"], mf.factor_permutation(F))
    assert d["finite"] and d["rdiag"].shape == (N, 5)
    with pytest.raises(mf.ArgumentError):
        mf.numerical_rank(F, rtol=-1.0)
