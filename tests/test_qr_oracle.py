"""The oracle's Householder QR and rank-revealing QR (qr.jl) on the CPU,
pinned by the reference's own deterministic known answers (test/runtests.jl
rank-revealing QR block, test/qr_delayed_norm.jl): revealed ranks of the
sin/cos panels (which exercise the blocked DLAQPS path with panel breaks and
delayed norm rebuilds), tie and scale rules of the pivot choice, exact-zero
and near-dependent columns, and Q R = A[:, p] reconstructions."""
import numpy as np
import pytest

from test_oracle import syn


def mf_of(X, N):
    A = np.zeros((N,) + X.shape)
    A[0] = X
    return A


def sincos_panel(N, rows=500, cols=40):
    r = np.arange(1, rows + 1)[:, None].astype(float)
    c = np.arange(1, cols + 1)[None, :].astype(float)
    return mf_of(np.sin(r * 0.01 + c * 0.7) + 0.1 * np.cos(r * 0.003 * c), N)


def explicit_r(F):
    N, m, n = F.shape
    R = np.triu(F)[:, :min(m, n), :]
    return R


def q_matrix(ref, F, tau):
    N, m, _ = F.shape
    Q = np.zeros((N, m, m))
    Q[0] = np.eye(m)
    return ref.apply_q(F, tau, Q, "N")


def rel_err(ref, X, Y):
    d = np.abs(ref.to_double(X - Y))
    return np.max(d) / max(np.max(np.abs(ref.to_double(Y))), 1.0)


@pytest.mark.parametrize("N", [2, 4])
def test_oracle_rrqr_blocked_panel_known_ranks(ref, N):
    A = sincos_panel(N)
    F, tau, perm, info = ref.rrqr(A)
    assert info == 0 and sorted(perm) == list(range(1, 41))
    assert ref.qr_numerical_rank(F, rtol=1e-12) == 31
    if N == 4:
        assert ref.qr_numerical_rank(F, rtol=1e-30) == 40
    T = ref.apply_q(F, tau, np.ascontiguousarray(A[:, :, perm - 1]), "T")
    lower = np.abs(ref.to_double(np.tril(T[:, :40, :], -1)))
    assert np.max(lower) <= (1e-50 if N == 4 else 4096 * 512 * 500 * 2.0 ** -104)


def test_oracle_rrqr_delayed_norm_rank_reveal(ref):
    """qr_delayed_norm.jl:71-95: duplicated columns, true rank 30"""
    N = 4
    r = np.arange(1, 257)[:, None].astype(float)
    c = np.arange(1, 31)[None, :].astype(float)
    core = np.sin(0.013 * r + 0.23 * c) + 0.21 * np.cos(0.005 * r * c)
    D = np.zeros((256, 64))
    D[:, :30] = core
    D[:, 30:40] = core[:, 1:11]
    A = mf_of(D, N)
    F, tau, perm, info = ref.rrqr(A)
    assert ref.qr_numerical_rank(F, rtol=2.0 ** -104) == 30
    T = ref.apply_q(F, tau, np.ascontiguousarray(A[:, :, perm - 1]), "T")
    assert np.max(np.abs(ref.to_double(np.tril(T[:, :64, :], -1)))) <= 1e-50


@pytest.mark.parametrize("N", [2, 3, 4])
def test_oracle_rrqr_pivot_rules(ref, N):
    rng = np.random.default_rng(3)
    # equal exact norms keep the original order
    E = mf_of(np.eye(8)[:, :4], N)
    assert list(ref.rrqr(E)[2]) == [1, 2, 3, 4]
    # scale-safe norms: the 1e100 column is the first pivot
    S = rng.standard_normal((10, 4)) * np.array([1e-100, 1e100, 1e-40, 1e40])
    F, tau, perm, _ = ref.rrqr(mf_of(S, N))
    assert perm[0] == 2 and ref.qr_numerical_rank(F) == 4
    # exact zero and duplicate columns are rank decisions of the caller
    src = rng.standard_normal((13, 4))
    Dm = np.hstack([src, src[:, 1:2], np.zeros((13, 1))])
    F, tau, perm, _ = ref.rrqr(mf_of(Dm, N))
    assert ref.qr_numerical_rank(F, rtol=2.0 ** (-26 * N)) == 4
    assert ref.qr_numerical_rank(ref.rrqr(np.zeros((N, 5, 8)))[0]) == 0
    # a perturbation near sqrt(eps) is visible only under the exact test
    Nr = mf_of(rng.standard_normal((12, 5)), N)
    Nr[:, :, 4] = Nr[:, :, 0]
    Nr[:, 0, 4] = ref.add(Nr[:, 0, 4], ref._scalar(N, 2.0 ** (-26 * N) / 4))
    F = ref.rrqr(Nr)[0]
    assert ref.qr_numerical_rank(F) == 5
    assert ref.qr_numerical_rank(F, rtol=2.0 ** (-26 * N)) == 4


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("shape", [(15, 7), (7, 15), (9, 9), (40, 30)], ids=str)
@pytest.mark.parametrize("pivoted", [True, False])
def test_oracle_qr_reconstruction(ref, rng, N, shape, pivoted):
    m, n = shape
    A = syn.randn_mf(rng, N, m, n)
    F, tau, perm, info = (ref.rrqr if pivoted else ref.qr)(A)
    assert info == 0
    if not pivoted:
        assert list(perm) == list(range(1, n + 1))
    Q = q_matrix(ref, F, tau)
    QR = ref.gemm(Q[:, :, :min(m, n)], explicit_r(F))
    assert rel_err(ref, QR, np.ascontiguousarray(A[:, :, perm - 1])) <= \
        4096 * 64 * max(m, n) * 2.0 ** (-52 * N)
    QtQ = ref.gemm(np.ascontiguousarray(Q.transpose(0, 2, 1)), Q)
    assert rel_err(ref, QtQ, mf_of(np.eye(m), N)) <= 4096 * 64 * m * 2.0 ** (-52 * N)
    assert ref.qr_numerical_rank(F) == min(m, n)
    V = syn.randn_mf(rng, N, m, 3)
    back = ref.apply_q(F, tau, ref.apply_q(F, tau, V, "T"), "N")
    assert rel_err(ref, back, V) <= 4096 * 64 * m * 2.0 ** (-52 * N)


def test_oracle_qr_nonfinite(ref):
    A = np.zeros((2, 6, 5))
    A[0] = np.arange(30).reshape(6, 5)
    A[1, 2, 3] = np.nan
    for fn in (ref.qr, ref.rrqr):
        F, tau, perm, info = fn(A)
        assert info == -1 and np.all(tau == 0) and list(perm) == [1, 2, 3, 4, 5]
        assert np.array_equal(np.isnan(F), np.isnan(A))
