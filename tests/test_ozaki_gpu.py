"""INT8-slice (Ozaki) GEMM route: componentwise error against the exact
superaccumulator oracle, compared with the plain FP64 route on the same
inputs, plus the alpha/beta epilogue and non-finite propagation."""
import numpy as np
import pytest

from test_oracle import syn

pytestmark = pytest.mark.gpu


def _err(ref, A, B, C, rng, samples=300):
    m, n = C.shape[1], C.shape[2]
    rows, cols = rng.integers(0, m, samples), rng.integers(0, n, samples)
    err, scale, _ = ref.exact_gemm_check(A, B, C, rows, cols)
    return np.max(err / scale)


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("shape", [(1, 1, 1), (33, 70, 45), (200, 513, 130)], ids=str)
def test_ozaki_default_slices_match_plain_accuracy(mf, ref, rng, N, shape):
    """with the default slice count the Ozaki error is no worse than twice the
    plain matched-order kernel's error (and within 4096 k eps(T))"""
    m, k, n = shape
    A, B = syn.randn_mf(rng, N, m, k, spread=20), syn.randn_mf(rng, N, k, n, spread=20)
    Ad, Bd = mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B)
    Cp, Co = mf.MFMatrix.zeros(N, m, n), mf.MFMatrix.zeros(N, m, n)
    mf.gemm_(Cp, Ad, Bd)
    mf.gemm_(Co, Ad, Bd, config=mf.KernelConfig(gemm_strategy="ozaki", ozaki_scheme="slices"))
    ep = _err(ref, A, B, Cp.to_numpy(), np.random.default_rng(1))
    eo = _err(ref, A, B, Co.to_numpy(), np.random.default_rng(1))
    assert eo <= 4096 * k * 2.0 ** (-52 * N)
    assert eo <= 2 * ep + 2.0 ** (-53 * N), (eo, ep, mf.ozaki_last_slices())


@pytest.mark.parametrize("N", [2, 4])
def test_ozaki_error_decreases_with_slices(mf, ref, rng, N):
    m, k, n = 64, 256, 48
    A, B = syn.randn_mf(rng, N, m, k, spread=20), syn.randn_mf(rng, N, k, n, spread=20)
    Ad, Bd = mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B)
    errs = []
    base = mf.ozaki_default_slices(N, k)
    for S in (base - 8, base - 4, base):
        Co = mf.MFMatrix.zeros(N, m, n)
        mf.gemm_(Co, Ad, Bd, config=mf.KernelConfig(gemm_strategy="ozaki", ozaki_slices=S))
        errs.append(_err(ref, A, B, Co.to_numpy(), np.random.default_rng(2)))
    assert errs[0] > errs[1] > 0 and errs[1] >= errs[2]
    # each extra slice buys about 7 bits while truncation dominates
    assert errs[0] / max(errs[1], 1e-300) > 2.0 ** 20


@pytest.mark.parametrize("N", [2, 3])
def test_ozaki_alpha_beta(mf, ref, rng, N):
    m, k, n = 40, 60, 30
    A, B, C0 = (syn.randn_mf(rng, N, m, k), syn.randn_mf(rng, N, k, n),
                syn.randn_mf(rng, N, m, n))
    alpha, beta = syn.randn_mf(rng, N, 1, 1)[:, 0, 0], syn.randn_mf(rng, N, 1, 1)[:, 0, 0]
    Co = mf.MFMatrix.from_numpy(C0)
    mf.gemm_(Co, mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B), alpha, beta,
             config=mf.KernelConfig(gemm_strategy="ozaki", ozaki_scheme="slices"))
    want = ref.gemm(A, B, C0, alpha, beta)
    got = Co.to_numpy()
    scale = (np.abs(A[0]) @ np.abs(B[0])) * abs(alpha[0]) + np.abs(beta[0] * C0[0])
    assert np.all(np.abs(ref.to_double(got - want)) <= 4096 * k * 2.0 ** (-52 * N) * scale + 1e-300)


def test_ozaki_nonfinite_rows_give_nan(mf, rng):
    N = 2
    A, B = syn.randn_mf(rng, N, 8, 8), syn.randn_mf(rng, N, 8, 8)
    A[0, 3, 5] = np.inf
    Co = mf.MFMatrix.zeros(N, 8, 8)
    mf.gemm_(Co, mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B),
             config=mf.KernelConfig(gemm_strategy="ozaki", ozaki_scheme="slices"))
    got = Co.to_numpy()
    assert np.all(np.isnan(got[0, 3, :]))
    assert np.all(np.isfinite(np.delete(got[0], 3, axis=0)))


def test_ozaki_zero_matrix(mf):
    N = 2
    Co = mf.MFMatrix.zeros(N, 5, 7)
    mf.gemm_(Co, mf.MFMatrix.zeros(N, 5, 9), mf.MFMatrix.zeros(N, 9, 7),
             config=mf.KernelConfig(gemm_strategy="ozaki", ozaki_scheme="slices"))
    assert np.all(Co.to_numpy() == 0)
