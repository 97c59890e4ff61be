"""Device Bunch-Kaufman LDL^T against the oracle (bitwise, unblocked and lazy
blocked routes) and the reference's LDLT known answers (adversarial.jl:172-309)."""
import numpy as np
import pytest

from conftest import assert_bitwise
from test_oracle import syn

pytestmark = pytest.mark.gpu


def _sym(rng, N, n, scale=1.0):
    X = syn.randn_mf(rng, N, n, n, scale=scale)
    return np.tril(X) + np.transpose(np.tril(X, -1), (0, 2, 1))


def _run(mf, S, blocked, block):
    cfg = mf.KernelConfig(ldlt_strategy="blocked" if blocked else "unblocked",
                          ldlt_block=block, ldlt_blocked_crossover=1)
    Sd = mf.MFMatrix.from_numpy(S)
    F = mf.ldlt_(Sd, check=False, config=cfg)
    return F, Sd, cfg


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("n,blocked,block", [(1, False, 1), (2, False, 1), (5, False, 1),
                                             (33, False, 1), (70, False, 1), (40, True, 4),
                                             (70, True, 5), (90, True, 16)])
def test_ldlt_matches_oracle(mf, ref, rng, N, n, blocked, block):
    S = _sym(rng, N, n)
    S_in = S.copy()
    iu = np.triu_indices(n, 1)
    S_in[:, iu[0], iu[1]] = np.nan  # the upper triangle is never read
    F, Sd, cfg = _run(mf, S_in, blocked, block)
    Fr, dsr, pvr, blr, info = ref.sytrf(S_in, blocked=blocked, block=block)
    assert mf.factor_status(F) == info == 0
    assert np.array_equal(mf.factor_pivots(F), pvr)
    assert np.array_equal(mf.factor_blocks(F), blr)
    assert_bitwise(F.dsub.cpu().numpy(), dsr, "dsub")
    assert_bitwise(Sd.to_numpy(), Fr, "factor")
    B = syn.randn_mf(rng, N, n, 3)
    X = mf.solve(F, mf.MFMatrix.from_numpy(B), config=cfg).to_numpy()
    Xr, rc = ref.sytrs(Fr, dsr, pvr, blr, B)
    assert rc == 0
    assert_bitwise(X, Xr, "ldlt solve")
    assert np.all(ref.backward_error(S, X, B) < 4096 * n * 2.0 ** (-52 * N))


@pytest.mark.parametrize("N", [2, 4])
def test_ldlt_default_blocked_route(mf, ref, rng, N):
    """n >= 512 takes the lazy blocked route by default (16/8 columns)"""
    n = 520
    S = _sym(rng, N, n)
    assert mf.ldlt_plan(N, n)["strategy"] == "blocked"
    Sd = mf.MFMatrix.from_numpy(S)
    F = mf.ldlt_(Sd)
    Fr, dsr, pvr, blr, info = ref.sytrf(S)
    assert info == 0
    assert np.array_equal(mf.factor_pivots(F), pvr)
    assert_bitwise(Sd.to_numpy(), Fr, "factor")


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("strategy", ["unblocked", "blocked"])
def test_kat_kkt_inertia(mf, ref, N, strategy):
    """adversarial.jl:172-217: saddle point with inertia (4, 2, 0), NaN upper"""
    H = np.diag([4.0, 5, 6, 7])
    Cn = np.array([[1.0, 2, 0, 1], [0, 1, 1, -1]])
    K = np.block([[H, Cn.T], [Cn, np.zeros((2, 2))]])
    clean = np.zeros((N, 6, 6))
    clean[0] = K
    truth = np.zeros((N, 6, 1))
    truth[0, :, 0] = [1, -2, 3, -1, 2, -3]
    rhs = ref.gemm(clean, truth)
    kkt = clean.copy()
    iu = np.triu_indices(6, 1)
    kkt[:, iu[0], iu[1]] = np.nan
    cfg = mf.KernelConfig(ldlt_strategy=strategy, ldlt_block=3, ldlt_blocked_crossover=1)
    F = mf.ldlt_(mf.MFMatrix.from_numpy(kkt), config=cfg)
    assert mf.factor_inertia(F) == {"positive": 4, "negative": 2, "zero": 0}
    X = mf.solve(F, mf.MFMatrix.from_numpy(rhs), config=cfg).to_numpy()
    assert np.all(ref.backward_error(clean, X, rhs) <= 4096 * 2.0 ** (-52 * N))


@pytest.mark.parametrize("N", [2, 3, 4])
def test_kat_tiny_diagonal(mf, ref, N):
    """adversarial.jl:219-240"""
    vals = [2.0 ** -300, -2.0 ** -100, 2.0 ** 100, -2.0 ** 300]
    D = np.zeros((N, 4, 4))
    D[0] = np.diag(vals)
    cfg = mf.KernelConfig(ldlt_strategy="unblocked")
    F = mf.ldlt_(mf.MFMatrix.from_numpy(D), config=cfg)
    d = mf.factor_diagnostics(F)
    assert d["one_by_one_pivots"] == 4
    assert d["inertia"] == {"positive": 2, "negative": 2, "zero": 0}
    assert d["minimum_block_eigenvalue_magnitude"][0] == 2.0 ** -300
    truth = np.zeros((N, 4, 1))
    truth[0, :, 0] = [1, -2, 3, -4]
    X = mf.solve(F, mf.MFMatrix.from_numpy(ref.gemm(D, truth)), config=cfg).to_numpy()
    assert_bitwise(X, truth)


@pytest.mark.parametrize("N", [2, 3, 4])
def test_kat_scaled_two_by_two(mf, ref, N):
    """adversarial.jl:242-266: four coupled 2x2 blocks at 2^-300..2^300"""
    couplings = [2.0 ** -300, 2.0 ** -100, 2.0 ** 100, 2.0 ** 300]
    A = np.zeros((N, 8, 8))
    for b, c in enumerate(couplings):
        f = 2 * b
        A[0, f + 1, f] = c
        A[:, f, f + 1] = np.nan
    cfg = mf.KernelConfig(ldlt_strategy="unblocked")
    F = mf.ldlt_(mf.MFMatrix.from_numpy(A), config=cfg)
    d = mf.factor_diagnostics(F)
    assert d["two_by_two_pivots"] == 4
    assert d["inertia"] == {"positive": 4, "negative": 4, "zero": 0}
    assert d["minimum_block_eigenvalue_magnitude"][0] == 2.0 ** -300
    truth = np.arange(1.0, 9.0)
    rhs = np.zeros((N, 8, 1))
    for b, c in enumerate(couplings):
        f = 2 * b
        rhs[0, f, 0] = c * truth[f + 1]
        rhs[0, f + 1, 0] = c * truth[f]
    X = mf.solve(F, mf.MFMatrix.from_numpy(rhs), config=cfg).to_numpy()
    want = np.zeros((N, 8, 1))
    want[0, :, 0] = truth
    assert_bitwise(X, want)


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("strategy", ["unblocked", "blocked"])
@pytest.mark.parametrize("exponent", [-600, 600])
def test_kat_extreme_2x2(mf, ref, N, strategy, exponent):
    """adversarial.jl:268-302: det(D) would over/underflow"""
    c = 2.0 ** exponent
    E = np.zeros((N, 4, 4))
    for f in (0, 2):
        E[0, f + 1, f] = c
        E[0, f, f + 1] = c
    cfg = mf.KernelConfig(ldlt_strategy=strategy, ldlt_block=2, ldlt_blocked_crossover=1)
    F = mf.ldlt_(mf.MFMatrix.from_numpy(E), config=cfg)
    assert mf.issuccess(F)
    assert mf.factor_inertia(F) == {"positive": 2, "negative": 2, "zero": 0}
    truth = np.zeros((N, 4, 2))
    truth[0, :, 0] = [1, -2, 3, -4]
    truth[0, :, 1] = [-1, 2, -3, 4]
    rhs = ref.gemm(E, truth)
    X = mf.solve(F, mf.MFMatrix.from_numpy(rhs), config=cfg).to_numpy()
    err = np.abs(ref.to_double(X - truth))
    assert np.max(err) <= 32 * 2.0 ** (-52 * N) * 4


@pytest.mark.parametrize("N", [2, 3, 4])
def test_kat_singular(mf, N):
    """adversarial.jl:304-309"""
    A = np.zeros((N, 2, 2))
    A[0] = [[1, 1], [1, 1]]
    F = mf.ldlt_(mf.MFMatrix.from_numpy(A), check=False,
                 config=mf.KernelConfig(ldlt_strategy="unblocked"))
    assert mf.factor_status(F) == 2
    assert mf.factor_state(F) == "singular"
    assert mf.factor_diagnostics(F)["failure_location"] == 2
    with pytest.raises(mf.SingularException):
        mf.ldlt_(mf.MFMatrix.from_numpy(A), config=mf.KernelConfig(ldlt_strategy="unblocked"))


def test_ldlt_nonfinite(mf, rng):
    A = _sym(rng, 2, 5)
    A[0, 3, 1] = np.inf
    F = mf.ldlt_(mf.MFMatrix.from_numpy(A), check=False)
    assert mf.factor_status(F) == -1
    with pytest.raises(mf.DomainError):
        mf.ldlt_(mf.MFMatrix.from_numpy(A))
