"""Modular (CRT) INT8 GEMM route on the device: exact results for operands
that fit the digit width, componentwise error against the exact
superaccumulator oracle compared with the plain FP64 route, the modulus
knob, both int8 engines bit for bit, epilogue, views and edge cases."""
from fractions import Fraction

import numpy as np
import pytest

from test_oracle import syn

pytestmark = pytest.mark.gpu


def _cfg(mf, **kw):
    return mf.KernelConfig(gemm_strategy="ozaki", ozaki_scheme="modular", **kw)


def _err(ref, A, B, C, rng, samples=300):
    m, n = C.shape[1], C.shape[2]
    rows, cols = rng.integers(0, m, samples), rng.integers(0, n, samples)
    err, scale, _ = ref.exact_gemm_check(A, B, C, rows, cols)
    return np.max(err / scale)


def _exact_value(X, i, j):
    return sum(Fraction(float(X[l, i, j])) for l in range(X.shape[0]))


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("shape", [(1, 1, 1), (33, 70, 45), (200, 513, 130)], ids=str)
def test_modular_matches_plain_accuracy(mf, ref, rng, N, shape):
    m, k, n = shape
    A, B = syn.randn_mf(rng, N, m, k, spread=20), syn.randn_mf(rng, N, k, n, spread=20)
    Ad, Bd = mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B)
    Cp, Co = mf.MFMatrix.zeros(N, m, n), mf.MFMatrix.zeros(N, m, n)
    mf.gemm_(Cp, Ad, Bd)
    mf.gemm_(Co, Ad, Bd, config=_cfg(mf))
    T = mf.ozaki_last_moduli()
    assert 1 <= T <= 49
    ep = _err(ref, A, B, Cp.to_numpy(), np.random.default_rng(1))
    eo = _err(ref, A, B, Co.to_numpy(), np.random.default_rng(1))
    assert eo <= 4096 * k * 2.0 ** (-52 * N)
    assert eo <= 2 * ep + 2.0 ** (-53 * N), (eo, ep, T)


@pytest.mark.parametrize("N", [2, 3, 4])
def test_modular_exact_for_representable_operands(mf, rng, N):
    """entries that fit the digit width multiply exactly: the result equals
    the exact integer product (checked with Python big integers)"""
    m, k, n = 37, 300, 41
    A = np.zeros((N, m, k))
    B = np.zeros((N, k, n))
    A[0] = rng.integers(-2 ** 20, 2 ** 20, (m, k)).astype(np.float64)
    B[0] = rng.integers(-2 ** 20, 2 ** 20, (k, n)).astype(np.float64)
    if N >= 3:
        # two limbs per entry: a0 * 2^40 + a1 (exact integers, 61 bits)
        A[0] *= 2.0 ** 40
        A[1] = rng.integers(-2 ** 20, 2 ** 20, (m, k)).astype(np.float64)
    C = mf.MFMatrix.zeros(N, m, n)
    mf.gemm_(C, mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B), config=_cfg(mf))
    got = C.to_numpy()
    Ai = [[int(A[0, i, kk]) + (int(A[1, i, kk]) if N >= 3 else 0) for kk in range(k)]
          for i in range(m)]
    Bi = [[int(B[0, kk, j]) for j in range(n)] for kk in range(k)]
    for i in range(0, m, 5):
        for j in range(0, n, 4):
            exact = sum(Ai[i][kk] * Bi[kk][j] for kk in range(k))
            assert _exact_value(got, i, j) == exact, (i, j)


@pytest.mark.parametrize("N", [2, 4])
def test_modular_error_decreases_with_moduli(mf, ref, rng, N):
    m, k, n = 64, 256, 48
    A, B = syn.randn_mf(rng, N, m, k, spread=20), syn.randn_mf(rng, N, k, n, spread=20)
    Ad, Bd = mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B)
    Co = mf.MFMatrix.zeros(N, m, n)
    mf.gemm_(Co, Ad, Bd, config=_cfg(mf))
    base = mf.ozaki_last_moduli()
    errs = []
    for T in (base - 12, base - 8, base):
        mf.gemm_(Co, Ad, Bd, config=_cfg(mf, ozaki_moduli=T))
        assert mf.ozaki_last_moduli() == T
        errs.append(_err(ref, A, B, Co.to_numpy(), np.random.default_rng(2)))
    assert errs[0] > errs[1] > 0 and errs[1] >= errs[2]
    # four moduli widen the digits by about 15 bits (one digit) / 7 bits per
    # digit (two), while truncation dominates the error
    assert errs[0] / max(errs[1], 1e-300) > 2.0 ** 6


@pytest.mark.parametrize("N", [2, 3, 4])
def test_modular_engines_bitwise_equal(mf, rng, N):
    """the tcgen05 kernel and the library GEMM give identical residues, so
    the route's results agree bit for bit"""
    from conftest import assert_bitwise
    m, k, n = 130, 300, 260
    A, B = syn.randn_mf(rng, N, m, k, spread=10), syn.randn_mf(rng, N, k, n, spread=10)
    Ad, Bd = mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B)
    C1, C2 = mf.MFMatrix.zeros(N, m, n), mf.MFMatrix.zeros(N, m, n)
    mf.gemm_(C1, Ad, Bd, config=_cfg(mf, ozaki_engine="tcgen05"))
    mf.gemm_(C2, Ad, Bd, config=_cfg(mf, ozaki_engine="library"))
    assert_bitwise(C1.to_numpy(), C2.to_numpy(), "tcgen05 vs library")
    assert mf.device_status() == 0


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("T", [8, 30, 36, 49])
@pytest.mark.parametrize("shape", [(129, 200, 257), (256, 130, 256), (1, 64, 3), (300, 33, 1)],
                         ids=str)
def test_reconstruction_engines_bitwise(mf, rng, N, T, shape):
    """the tensor-core reconstruction (tcgen05 engines: byte sums of the
    residues by an int8 MMA) and the CUDA-core one (library engine) give the
    same bits for every word count of the CRT sum (T = 8, 30: 8 words; 36:
    10; 49: 12), ragged shapes (rows past a 128-row block, an odd column past
    a column pair) and a general alpha/beta epilogue"""
    from conftest import assert_bitwise
    m, k, n = shape
    A, B = syn.randn_mf(rng, N, m, k, spread=12), syn.randn_mf(rng, N, k, n, spread=12)
    C0 = syn.randn_mf(rng, N, m, n)
    alpha, beta = syn.randn_mf(rng, N, 1, 1)[:, 0, 0], syn.randn_mf(rng, N, 1, 1)[:, 0, 0]
    Ad, Bd = mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B)
    out = []
    for engine in ("tcgen05", "tcgen05_pair", "library"):
        Cd = mf.MFMatrix.from_numpy(C0)
        mf.gemm_(Cd, Ad, Bd, alpha, beta, config=_cfg(mf, ozaki_moduli=T, ozaki_engine=engine))
        out.append(Cd.to_numpy())
    assert_bitwise(out[0], out[2], "tensor-core vs CUDA-core reconstruction")
    assert_bitwise(out[1], out[2], "pair engine vs CUDA-core reconstruction")
    assert mf.device_status() == 0


def test_reconstruction_nonfinite_rows_and_columns(mf, rng):
    """a row of A or a column of B with a non-finite entry gives NaN in its
    row / column of C on both reconstructions, the rest is unchanged"""
    from conftest import assert_bitwise
    N, m, k, n = 2, 140, 50, 9
    A, B = syn.randn_mf(rng, N, m, k), syn.randn_mf(rng, N, k, n)
    A[0, 5, 7] = np.inf
    B[0, 3, 4] = np.nan
    Ad, Bd = mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B)
    out = []
    for engine in ("tcgen05", "library"):
        Cd = mf.MFMatrix.zeros(N, m, n)
        mf.gemm_(Cd, Ad, Bd, config=_cfg(mf, ozaki_moduli=20, ozaki_engine=engine))
        out.append(Cd.to_numpy())
    assert np.all(np.isnan(out[0][0, 5, :])) and np.all(np.isnan(out[0][0, :, 4]))
    assert np.all(np.isfinite(np.delete(np.delete(out[0][0], 5, 0), 4, 1)))
    assert_bitwise(out[0], out[1], "non-finite")


@pytest.mark.parametrize("N", [2, 4])
def test_modular_alpha_beta(mf, ref, rng, N):
    m, k, n = 40, 60, 30
    A, B, C0 = (syn.randn_mf(rng, N, m, k), syn.randn_mf(rng, N, k, n),
                syn.randn_mf(rng, N, m, n))
    alpha, beta = syn.randn_mf(rng, N, 1, 1)[:, 0, 0], syn.randn_mf(rng, N, 1, 1)[:, 0, 0]
    Co = mf.MFMatrix.from_numpy(C0)
    mf.gemm_(Co, mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B), alpha, beta,
             config=_cfg(mf))
    want = ref.gemm(A, B, C0, alpha, beta)
    got = Co.to_numpy()
    scale = (np.abs(A[0]) @ np.abs(B[0])) * abs(alpha[0]) + np.abs(beta[0] * C0[0])
    assert np.all(np.abs(ref.to_double(got - want)) <= 4096 * k * 2.0 ** (-52 * N) * scale + 1e-300)


def test_modular_views(mf, ref, rng):
    """operands and result as sub-matrix views (ld > rows, offsets)"""
    N = 2
    M = syn.randn_mf(rng, N, 90, 80, spread=5)
    Md = mf.MFMatrix.from_numpy(M)
    A = Md.view(slice(3, 40), slice(5, 50))     # 37 x 45
    B = Md.view(slice(41, 86), slice(2, 33))    # 45 x 31
    Cbig = mf.MFMatrix.zeros(N, 60, 40)
    Cv = Cbig.view(slice(7, 44), slice(4, 35))  # 37 x 31
    mf.gemm_(Cv, A, B, config=_cfg(mf))
    An, Bn = M[:, 3:40, 5:50].copy(), M[:, 41:86, 2:33].copy()
    got = Cbig.to_numpy()
    e = _err(ref, An, Bn, np.ascontiguousarray(got[:, 7:44, 4:35]), np.random.default_rng(3))
    assert e <= 4096 * 45 * 2.0 ** -104
    assert np.all(got[:, :7, :] == 0) and np.all(got[:, :, :4] == 0)
    assert np.all(got[:, 44:, :] == 0) and np.all(got[:, :, 35:] == 0)


def test_modular_long_reduction(mf, ref, rng):
    """k = 40000: beyond what the slice route can keep exact in int32 at the
    slice counts Float64x2 needs"""
    N, m, k, n = 2, 24, 40000, 20
    A, B = syn.randn_mf(rng, N, m, k, spread=3), syn.randn_mf(rng, N, k, n, spread=3)
    Ad, Bd = mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B)
    Cp, Co = mf.MFMatrix.zeros(N, m, n), mf.MFMatrix.zeros(N, m, n)
    mf.gemm_(Cp, Ad, Bd)
    mf.gemm_(Co, Ad, Bd, config=_cfg(mf))
    ep = _err(ref, A, B, Cp.to_numpy(), np.random.default_rng(4), samples=60)
    eo = _err(ref, A, B, Co.to_numpy(), np.random.default_rng(4), samples=60)
    assert eo <= 2 * ep + 2.0 ** -106, (eo, ep)


def test_modular_nonfinite_rows_give_nan(mf, rng):
    N = 2
    A, B = syn.randn_mf(rng, N, 8, 8), syn.randn_mf(rng, N, 8, 8)
    A[0, 3, 5] = np.nan
    B[1, 2, 6] = np.inf
    Co = mf.MFMatrix.zeros(N, 8, 8)
    mf.gemm_(Co, mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B), config=_cfg(mf))
    got = Co.to_numpy()
    assert np.all(np.isnan(got[0, 3, :])) and np.all(np.isnan(got[0, :, 6]))
    keep = np.delete(np.delete(got[0], 3, axis=0), 6, axis=1)
    assert np.all(np.isfinite(keep))


def test_modular_zero_and_empty(mf):
    N = 3
    Co = mf.MFMatrix.zeros(N, 5, 7)
    mf.gemm_(Co, mf.MFMatrix.zeros(N, 5, 9), mf.MFMatrix.zeros(N, 9, 7), config=_cfg(mf))
    assert np.all(Co.to_numpy() == 0)
    # k = 0: C = beta * C
    C0 = np.zeros((N, 4, 3))
    C0[0] = 1.0
    Cd = mf.MFMatrix.from_numpy(C0)
    mf.gemm_(Cd, mf.MFMatrix.zeros(N, 4, 0), mf.MFMatrix.zeros(N, 0, 3), 1.0, 2.0,
             config=_cfg(mf))
    assert np.all(Cd.to_numpy()[0] == 2.0) and np.all(Cd.to_numpy()[1:] == 0)
