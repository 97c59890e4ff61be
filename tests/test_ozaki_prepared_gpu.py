"""Prepared left operand of the modular INT8 route (the residuals of
iterative refinement): a product through the prepared residues equals the
unprepared product with the same modulus count bit for bit, for every limb
count, views, epilogues, both int8 engines and repeated use; the argument
checks; the mixed-precision LU solve that uses it still converges."""
import numpy as np
import pytest

from conftest import assert_bitwise
from test_oracle import syn

pytestmark = pytest.mark.gpu


def _cfg(mf, **kw):
    return mf.KernelConfig(gemm_strategy="ozaki", ozaki_scheme="modular", **kw)


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("shape", [(1, 1, 1), (33, 70, 45), (200, 513, 130), (300, 257, 1)],
                         ids=str)
@pytest.mark.parametrize("T", [8, 17])
def test_prepared_equals_unprepared(mf, rng, N, shape, T):
    m, k, n = shape
    A, B = syn.randn_mf(rng, N, m, k, spread=20), syn.randn_mf(rng, N, k, n, spread=20)
    C0 = syn.randn_mf(rng, N, m, n)
    Ad, Bd = mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B)
    C1, C2 = mf.MFMatrix.from_numpy(C0), mf.MFMatrix.from_numpy(C0)
    mf.gemm_(C1, Ad, Bd, -1.0, 1.0, config=_cfg(mf, ozaki_moduli=T))
    P = mf.PreparedInt8Operand(Ad, T)
    mf.gemm_prepared_(C2, P, Bd, -1.0, 1.0)
    assert_bitwise(C2.to_numpy(), C1.to_numpy(), "prepared")


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("shape,spread", [((33, 70, 45), 0), ((200, 513, 130), 20),
                                          ((300, 1100, 16), 10)], ids=str)
def test_tune_only_matches_tuned_product(mf, ref, rng, N, shape, spread):
    """ozaki_crt_tune_moduli picks the count the tuned product picks on the same
    operands; the prepared product at that count equals the fixed-count
    product bit for bit, and its error against the exact product is at most
    the tuned product's (wider digits; the mixed solve's first residual)"""
    m, k, n = shape
    A, B = syn.randn_mf(rng, N, m, k, spread=spread), syn.randn_mf(rng, N, k, n, spread=spread)
    Ad, Bd = mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B)
    T = mf.ozaki_crt_tune_moduli(Ad, Bd)
    C1, C2, C3 = (mf.MFMatrix.zeros(N, m, n) for _ in range(3))
    mf.gemm_(C1, Ad, Bd, config=_cfg(mf))
    assert mf.ozaki_last_moduli() == T
    mf.gemm_prepared_(C2, mf.PreparedInt8Operand(Ad, T), Bd)
    mf.gemm_(C3, Ad, Bd, config=_cfg(mf, ozaki_moduli=T))
    assert_bitwise(C2.to_numpy(), C3.to_numpy(), "prepared at the tuned count")
    rows, cols = (a.ravel() for a in np.meshgrid(np.arange(m), np.arange(n), indexing="ij"))
    err1, scale, _ = ref.exact_gemm_check(A, B, C1.to_numpy(), rows, cols)
    err2, _, _ = ref.exact_gemm_check(A, B, C2.to_numpy(), rows, cols)
    floor = 2.0 ** (-53 * N) * scale.max()
    assert err2.max() <= 1.01 * max(err1.max(), floor)


def test_tune_only_argument_checks(mf, rng):
    A = mf.MFMatrix.from_numpy(syn.randn_mf(rng, 2, 10, 12))
    with pytest.raises(mf.DimensionMismatch):
        mf.ozaki_crt_tune_moduli(A, mf.MFMatrix.from_numpy(syn.randn_mf(rng, 2, 11, 3)))
    with pytest.raises(mf.ArgumentError):
        mf.ozaki_crt_tune_moduli(A, mf.MFMatrix.from_numpy(syn.randn_mf(rng, 3, 12, 3)))


@pytest.mark.parametrize("engine", ["tcgen05", "tcgen05_pair", "library"])
def test_prepared_engines_and_reuse(mf, rng, engine):
    N, m, k, n, T = 2, 260, 700, 140, 20
    A = syn.randn_mf(rng, N, m, k, spread=10)
    Ad = mf.MFMatrix.from_numpy(A)
    P = mf.PreparedInt8Operand(Ad, T)
    cfg = _cfg(mf, ozaki_moduli=T, ozaki_engine=engine)
    for rep in range(3):
        B = syn.randn_mf(rng, N, k, n, spread=10 * rep)
        Bd = mf.MFMatrix.from_numpy(B)
        C1, C2 = mf.MFMatrix.zeros(N, m, n), mf.MFMatrix.zeros(N, m, n)
        mf.gemm_(C1, Ad, Bd, 2.0, 0.0, config=cfg)
        mf.gemm_prepared_(C2, P, Bd, 2.0, 0.0, config=cfg)
        assert_bitwise(C2.to_numpy(), C1.to_numpy(), f"rep {rep}")


def test_prepared_views(mf, rng):
    N, T = 3, 12
    A = syn.randn_mf(rng, N, 90, 120)
    B = syn.randn_mf(rng, N, 130, 70)
    Ad, Bd = mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B)
    Av, Bv = Ad.view(slice(5, 85), slice(7, 107)), Bd.view(slice(3, 103), slice(10, 60))
    Cd = mf.MFMatrix.zeros(N, 100, 90)
    C1 = mf.MFMatrix.zeros(N, 100, 90)
    mf.gemm_(C1.view(slice(10, 90), slice(20, 70)), Av, Bv, config=_cfg(mf, ozaki_moduli=T))
    mf.gemm_prepared_(Cd.view(slice(10, 90), slice(20, 70)), mf.PreparedInt8Operand(Av, T), Bv)
    assert_bitwise(Cd.to_numpy(), C1.to_numpy(), "views")


def test_prepared_argument_checks(mf, rng):
    N = 2
    Ad = mf.MFMatrix.from_numpy(syn.randn_mf(rng, N, 20, 30))
    P = mf.PreparedInt8Operand(Ad, 5)
    with pytest.raises(mf.DimensionMismatch):
        mf.gemm_prepared_(mf.MFMatrix.zeros(N, 20, 4), P, mf.MFMatrix.zeros(N, 31, 4))
    with pytest.raises(mf.DimensionMismatch):
        mf.gemm_prepared_(mf.MFMatrix.zeros(N, 21, 4), P, mf.MFMatrix.zeros(N, 30, 4))
    with pytest.raises(mf.ArgumentError):
        mf.gemm_prepared_(mf.MFMatrix.zeros(3, 20, 4), P, mf.MFMatrix.zeros(3, 30, 4))
    with pytest.raises(mf.ArgumentError):
        mf.PreparedInt8Operand(Ad, 0)
    with pytest.raises(mf.ArgumentError):
        mf.PreparedInt8Operand(Ad, 50)
    # too few moduli for any digit width: refused like the unprepared route
    with pytest.raises(mf.ArgumentError):
        mf.PreparedInt8Operand(mf.MFMatrix.from_numpy(syn.randn_mf(rng, 3, 20, 30)), 3)


def test_mixed_lu_with_prepared_residuals_converges(mf):
    N, n = 4, 900
    rng = np.random.default_rng(5)
    A = syn.randn_mf(rng, N, n, n)
    A[0] += 4 * np.sqrt(n) * np.eye(n)
    X0 = syn.randn_mf(rng, N, n, 1)
    Ad = mf.MFMatrix.from_numpy(A)
    B = mf.MFMatrix.zeros(N, n, 1)
    mf.gemm_(B, Ad, mf.MFMatrix.from_numpy(X0))
    X, rep = mf.solve_mixed_lu(Ad, B)
    assert rep["converged"], rep
    assert rep["backward_error"] <= 2.0 ** (-52 * N) * 64
