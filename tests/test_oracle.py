"""CPU tests of the oracle against the reference's golden vectors and exact
arithmetic (no GPU)."""
import json
import os

import numpy as np
import pytest

from conftest import assert_bitwise

HERE = os.path.dirname(os.path.abspath(__file__))


def _f(bits):
    return np.array([int(b, 16) for b in bits], dtype=np.uint64).view(np.float64)


def _cases():
    with open(os.path.join(HERE, "golden", "mulacc_x3_proof_vectors.json")) as f:
        return json.load(f)["cases"]


def _gen():
    import importlib.util
    p = os.path.join(os.path.dirname(HERE), "multifloatlinearalgebra.jl_b200", "synthetic.py")
    spec = importlib.util.spec_from_file_location("synthetic_cpu", p)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


syn = _gen()


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c["name"])
def test_mulacc_x3_proof_vectors(ref, case):
    """test/mulacc_x3_proof_vectors.jl: fused and standard x3 networks give the
    committed output bits."""
    acc, x, y, out = _f(case["acc"]), _f(case["x"]), _f(case["y"]), _f(case["output"])
    assert_bitwise(ref.mulacc_x3(acc, x, y), out, "fused mulacc_x3")
    assert_bitwise(ref.add(acc, ref.mul(x, y)), out, "acc + x*y")


def test_proof_vector_lane_permutation(ref):
    """lanes are independent: the (4,2,1,3) permutation permutes outputs"""
    cases = _cases()
    for first in range(0, len(cases), 4):
        group = cases[first:first + 4]
        perm = [3, 1, 0, 2]
        for lane, src in enumerate(perm):
            c = group[src]
            assert_bitwise(ref.mulacc_x3(_f(c["acc"]), _f(c["x"]), _f(c["y"])), _f(c["output"]))


@pytest.mark.parametrize("N", [2, 3, 4])
def test_gemm_error_vs_exact(ref, rng, N):
    """componentwise error <= 4096*k*eps(T) * sum|a||b| (runtests.jl:25-29)"""
    m, k, n = 23, 41, 19
    A, B = syn.randn_mf(rng, N, m, k), syn.randn_mf(rng, N, k, n)
    C = ref.gemm(A, B)
    rows, cols = np.meshgrid(np.arange(m), np.arange(n), indexing="ij")
    err, scale, _ = ref.exact_gemm_check(A, B, C, rows.ravel(), cols.ravel())
    eps = 2.0 ** (-52 * N)
    assert np.all(err <= 4096 * k * eps * scale)
    # and much tighter in practice: a few units of 2^(-53N+1)
    assert np.max(err / scale) < 64 * 2.0 ** (-53 * N) * k


@pytest.mark.parametrize("N", [2, 3, 4])
def test_div_sqrt_accuracy(ref, rng, N):
    for _ in range(50):
        x = syn.randn_mf(rng, N, 1, 1)[:, 0, 0]
        y = syn.randn_mf(rng, N, 1, 1)[:, 0, 0]
        q = ref.div(x, y)
        # q*y - x exactly small
        r = ref.add(ref.mul(q, y), -x)
        assert abs(r[0]) <= 2.0 ** (-53 * N + 4) * abs(x[0])
        ax = x * np.sign(x[0])
        s = ref.sqrt(ax)
        r2 = ref.add(ref.mul(s, s), -ax)
        assert abs(r2[0]) <= 2.0 ** (-53 * N + 4) * abs(ax[0])


def test_x3_fused_equals_standard_gemm_on_random(ref, rng):
    """the reference reports the fused route bitwise equal to the standard
    one on its suites; the same holds on these random inputs"""
    A, B = syn.randn_mf(rng, 3, 17, 33), syn.randn_mf(rng, 3, 33, 13)
    assert_bitwise(ref.gemm(A, B, x3_fused=True), ref.gemm(A, B, x3_fused=False))


@pytest.mark.parametrize("N", [2, 3, 4])
def test_factorizations_backward_error(ref, rng, N):
    n = 50
    S = syn.spd_matrix(rng, N, n, ref.gemm)
    S = np.tril(S) + np.transpose(np.tril(S, -1), (0, 2, 1))  # exactly symmetric
    Bm = syn.randn_mf(rng, N, n, 3)
    tol = 4096 * n * 2.0 ** (-52 * N)
    L, info = ref.potrf(S)
    assert info == 0
    assert np.all(ref.backward_error(S, ref.potrs(L, Bm), Bm) < tol)
    LU, piv, info = ref.getrf(S)
    assert info == 0
    assert np.all(ref.backward_error(S, ref.getrs(LU, piv, Bm), Bm) < tol)
    for blocked in (False, True):
        F, ds, pv, bl, info = ref.sytrf(S, blocked=blocked, block=4)
        assert info == 0
        X, rc = ref.sytrs(F, ds, pv, bl, Bm)
        assert rc == 0
        assert np.all(ref.backward_error(S, X, Bm) < tol)


@pytest.mark.parametrize("N", [2, 3, 4])
def test_kat_diagonal_spd_exact(ref, N):
    """adversarial.jl:37-52: diag(2^-300..2^300) solves exactly"""
    ex = [-300, -150, 0, 150, 300]
    S = np.zeros((N, 5, 5))
    for i, e in enumerate(ex):
        S[0, i, i] = 2.0 ** e
    truth = np.zeros((N, 5, 1))
    truth[0, :, 0] = [1, -2, 3, -4, 5]
    rhs = ref.gemm(S, truth)
    L, info = ref.potrf(S, block=2)
    assert info == 0
    X = ref.potrs(L, rhs)
    assert_bitwise(X, truth)


@pytest.mark.parametrize("N", [2, 3, 4])
def test_kat_wilkinson_growth(ref, N):
    """adversarial.jl:148-171: Wilkinson's matrix has pivot growth 2^(n-1)"""
    n = 8
    W = np.zeros((N, n, n))
    for r in range(n):
        W[0, r, r] = 1.0
        W[0, r, n - 1] = 1.0
        W[0, r, :r] = -1.0
    LU, piv, info = ref.getrf(W, block=2)
    assert info == 0
    U = np.triu(LU[0])
    assert np.max(np.abs(U)) / 1.0 == 128.0
