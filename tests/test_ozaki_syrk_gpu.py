"""INT8 (modular) SYRK and the Cholesky factorization with INT8 trailing
updates: componentwise error of the lower triangle against the exact
superaccumulator oracle, the strict upper triangle untouched, both product
forms and both int8 engines bit for bit, backward errors and failure
statuses of the factorization."""
import numpy as np
import pytest

from conftest import assert_bitwise
from test_oracle import syn

pytestmark = pytest.mark.gpu

LOWER = dict(gemm_strategy="ozaki", ozaki_scheme="modular")


def _lower_err(ref, P, C, rng, samples=300):
    """max componentwise error of sampled lower entries of C = P^T P"""
    n = C.shape[1]
    i, j = rng.integers(0, n, samples), rng.integers(0, n, samples)
    rows, cols = np.maximum(i, j), np.minimum(i, j)
    PT = np.ascontiguousarray(P.transpose(0, 2, 1))
    err, scale, _ = ref.exact_gemm_check(PT, P, C, rows, cols)
    return np.max(err / np.maximum(scale, 1e-300))


def _spd(ref, rng, N, n):
    S = syn.spd_matrix(rng, N, n, ref.gemm)
    return np.tril(S) + np.transpose(np.tril(S, -1), (0, 2, 1))


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("n,k", [(1, 1), (70, 45), (300, 130), (513, 257)], ids=str)
def test_syrk_ozaki_matches_plain_accuracy(mf, ref, rng, N, n, k):
    P = syn.randn_mf(rng, N, k, n, spread=15)
    Pd = mf.MFMatrix.from_numpy(P)
    sentinel = np.full((N, n, n), 7.0)
    Cp, Co = mf.MFMatrix.from_numpy(sentinel), mf.MFMatrix.from_numpy(sentinel)
    mf.syrk_(Cp, Pd)
    mf.syrk_(Co, Pd, config=mf.KernelConfig(**LOWER))
    got = Co.to_numpy()
    iu = np.triu_indices(n, 1)
    assert np.all(got[:, iu[0], iu[1]] == 7.0), "strict upper triangle written"
    ep = _lower_err(ref, P, Cp.to_numpy(), np.random.default_rng(1))
    eo = _lower_err(ref, P, got, np.random.default_rng(1))
    assert eo <= 4096 * k * 2.0 ** (-52 * N)
    assert eo <= 2 * ep + 2.0 ** (-53 * N), (eo, ep, mf.ozaki_last_moduli())


@pytest.mark.parametrize("N", [2, 4])
def test_syrk_ozaki_alpha_beta(mf, ref, rng, N):
    n, k = 90, 70
    P, C0 = syn.randn_mf(rng, N, k, n), syn.randn_mf(rng, N, n, n)
    alpha, beta = syn.randn_mf(rng, N, 1, 1)[:, 0, 0], syn.randn_mf(rng, N, 1, 1)[:, 0, 0]
    Co = mf.MFMatrix.from_numpy(C0)
    mf.syrk_(Co, mf.MFMatrix.from_numpy(P), alpha, beta, config=mf.KernelConfig(**LOWER))
    want = ref.syrk_lower(P, C0, alpha, beta)
    got = Co.to_numpy()
    scale = (np.abs(P[0]).T @ np.abs(P[0])) * abs(alpha[0]) + np.abs(beta[0] * C0[0])
    il = np.tril_indices(n)
    diff = np.abs(ref.to_double(got - want))[il]
    assert np.all(diff <= 4096 * k * 2.0 ** (-52 * N) * scale[il] + 1e-300)
    iu = np.triu_indices(n, 1)
    assert np.array_equal(got[:, iu[0], iu[1]], C0[:, iu[0], iu[1]])


@pytest.mark.parametrize("N", [2, 3])
def test_syrk_ozaki_forms_and_engines_bitwise(mf, rng, N):
    """A A^T (trans 0) on A = P^T equals P^T P (trans 1) bit for bit (same
    digits, same products), and the tcgen05 triangle-tile GEMM equals the
    library's whole products on the lower triangle"""
    import torch
    n, k = 300, 200
    P = syn.randn_mf(rng, N, k, n, spread=10)
    AT = np.ascontiguousarray(P.transpose(0, 2, 1))
    outs = []
    for engine in ("tcgen05", "library"):
        Co = mf.MFMatrix.zeros(N, n, n)
        mf.syrk_(Co, mf.MFMatrix.from_numpy(P), config=mf.KernelConfig(ozaki_engine=engine,
                                                                        **LOWER))
        outs.append(np.tril(Co.to_numpy()))
    assert_bitwise(outs[0], outs[1], "tcgen05 vs library")
    lib = mf._native.load()
    h = mf._handle(0)
    Ad, Ct = mf.MFMatrix.from_numpy(AT), mf.MFMatrix.zeros(N, n, n)
    one, zero = mf._scalar(N, 1.0), mf._scalar(N, 0.0)
    rc = lib.mflab_syrk_lower_ozaki(h, torch.cuda.current_stream().cuda_stream, N, 0, 0, n, k,
                                    Ad.ptr(), Ad.ld, Ad.ls, Ct.ptr(), Ct.ld, Ct.ls, one, zero)
    assert rc == 0
    assert_bitwise(np.tril(Ct.to_numpy()), outs[0], "A A^T vs P^T P")
    assert mf.device_status() == 0


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("n,nb", [(40, 256), (300, 128), (600, 256)], ids=str)
def test_cholesky_int8_trailing_backward_error(mf, ref, rng, N, n, nb):
    S = _spd(ref, rng, N, n)
    Sd = mf.MFMatrix.from_numpy(S)
    cfg = mf.KernelConfig(ozaki_block=nb, **LOWER)
    F = mf.cholesky_(Sd, config=cfg)
    assert mf.factor_status(F) == 0
    B = syn.randn_mf(rng, N, n, 3)
    X = mf.solve(F, mf.MFMatrix.from_numpy(B)).to_numpy()
    be = ref.backward_error(S, X, B)
    assert np.all(be < 4096 * n * 2.0 ** (-52 * N)), be
    # the first panel is the matched-order factorization itself
    L, info = ref.potrf(S)
    w = min(nb, n)
    assert_bitwise(np.tril(Sd.to_numpy())[:, :, :w], np.tril(L)[:, :, :w], "first panel")


@pytest.mark.parametrize("N", [2, 4])
def test_cholesky_int8_trailing_failure(mf, ref, rng, N):
    """a pivot that turns negative in the second panel is reported at the
    same position as by the matched factorization"""
    n = 400
    S = _spd(ref, rng, N, n)
    S[:, 300, 300] = 0.0
    S[0, 300, 300] = -1.0
    Fm = mf.cholesky_(mf.MFMatrix.from_numpy(S), check=False)
    Fo = mf.cholesky_(mf.MFMatrix.from_numpy(S), check=False,
                      config=mf.KernelConfig(ozaki_block=256, **LOWER))
    assert mf.factor_status(Fo) == mf.factor_status(Fm) == 301
    with pytest.raises(mf.PosDefException):
        mf.cholesky_(mf.MFMatrix.from_numpy(S), config=mf.KernelConfig(**LOWER))
    S[0, 5, 2] = np.inf
    with pytest.raises(mf.DomainError):
        mf.cholesky_(mf.MFMatrix.from_numpy(S), config=mf.KernelConfig(**LOWER))


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("m,n,nb", [(40, 40, 256), (300, 300, 128), (520, 400, 256),
                                    (300, 520, 128)], ids=str)
def test_lu_int8_trailing(mf, ref, rng, N, m, n, nb):
    """LU with INT8 trailing updates: the first panel (pivots and factors)
    equals the matched factorization bit for bit; square systems solve to the
    backward error of the matched LU"""
    A = syn.randn_mf(rng, N, m, n)
    Ad = mf.MFMatrix.from_numpy(A)
    F = mf.lu_(Ad, config=mf.KernelConfig(ozaki_block=nb, **LOWER))
    LU, piv, info = ref.getrf(A)
    assert mf.factor_status(F) == info == 0
    w = min(nb, m, n)
    assert np.array_equal(mf.factor_pivots(F)[:w], piv[:w])
    assert_bitwise(Ad.to_numpy()[:, :, :w], LU[:, :, :w], "first panel")
    if m == n:
        B = syn.randn_mf(rng, N, n, 3)
        X = mf.solve(F, mf.MFMatrix.from_numpy(B)).to_numpy()
        be = ref.backward_error(A, X, B)
        assert np.all(be < 4096 * n * 2.0 ** (-52 * N)), be


@pytest.mark.parametrize("N", [2, 4])
def test_lu_int8_trailing_singular(mf, rng, N):
    """a zero pivot in the second panel is reported at the matched position"""
    n = 400
    A = syn.randn_mf(rng, N, n, n)
    A[:, :, 300] = 0.0  # an exactly zero column stays zero through the updates
    Fm = mf.lu_(mf.MFMatrix.from_numpy(A), check=False)
    Fo = mf.lu_(mf.MFMatrix.from_numpy(A), check=False,
                config=mf.KernelConfig(ozaki_block=256, **LOWER))
    assert mf.factor_status(Fm) == 301
    assert mf.factor_status(Fo) == mf.factor_status(Fm)
