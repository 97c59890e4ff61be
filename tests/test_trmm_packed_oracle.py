"""The oracle's trmm! and syrk_packed! restatements on the CPU: bit for bit
against element-wise loops written like the reference's own test models
(test/runtests.jl:48-75 trmm_reference, :493-520 the packed expected values)
on the oracle's scalar networks, exact integer products, and the packed
storage order."""
import itertools

import numpy as np
import pytest

from conftest import assert_bitwise
from test_oracle import syn

COMBOS = list(itertools.product(("left", "right"), ("lower", "upper"), ("N", "T"),
                                ("unit", "nonunit")))


def _triangular(rng, N, n, uplo, unit):
    """a triangular test matrix whose inactive triangle (and declared unit
    diagonal) hold NaN / Inf, which no chain may read"""
    A = syn.randn_mf(rng, N, n, n)
    for l in range(N):
        if uplo == "lower":
            A[l][np.triu_indices(n, 1)] = np.nan
        else:
            A[l][np.tril_indices(n, -1)] = np.inf
        if unit:
            A[l][np.diag_indices(n)] = np.nan
    A[0][np.diag_indices(n)] += 0 if unit else 3.0
    return A


def _trmm_model(ref, B, A, alpha, side, uplo, trans, diag):
    """test/runtests.jl:48-75, element by element on the oracle's networks"""
    N, m, n = B.shape
    al = ref._scalar(N, alpha)
    one = ref._scalar(N, 1.0)
    eff_lower = (uplo == "lower") == (trans == "N")
    unit = diag == "unit"
    out = np.empty_like(B)
    coef = (lambda r, c: A[:, r, c]) if trans == "N" else (lambda r, c: A[:, c, r])
    for i in range(m):
        for j in range(n):
            acc = np.zeros(N)
            if side == "left":
                ks = range(0, i + 1) if eff_lower else range(i, m)
                for k in ks:
                    c = one if (k == i and unit) else coef(i, k)
                    acc = ref.add(acc, ref.mul(c, B[:, k, j]))
            else:
                ks = range(j, n) if eff_lower else range(0, j + 1)
                for k in ks:
                    c = one if (k == j and unit) else coef(k, j)
                    acc = ref.add(acc, ref.mul(B[:, i, k], c))
            out[:, i, j] = ref.mul(al, acc)
    return out


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("side,uplo,trans,diag", COMBOS)
def test_oracle_trmm_matches_reference_model(ref, rng, N, side, uplo, trans, diag):
    order = 7
    A = _triangular(rng, N, order, uplo, diag == "unit")
    B = syn.randn_mf(rng, N, order, 5) if side == "left" else syn.randn_mf(rng, N, 5, order)
    alpha = ref._scalar(N, -2.0)
    got = ref.trmm(B, A, alpha, side, uplo, trans, diag, nthreads=1)
    assert np.all(np.isfinite(got))
    assert_bitwise(got, _trmm_model(ref, B, A, alpha, side, uplo, trans, diag), "trmm")


@pytest.mark.parametrize("side,uplo,trans,diag", COMBOS)
def test_oracle_trmm_exact_integers(ref, rng, side, uplo, trans, diag):
    """small integer entries multiply exactly: the product equals numpy's"""
    N, order = 2, 9
    T = np.zeros((N, order, order))
    T[0] = rng.integers(-50, 50, (order, order))
    T[0] = np.tril(T[0]) if uplo == "lower" else np.triu(T[0])
    if diag == "unit":
        np.fill_diagonal(T[0], 1.0)
    B = np.zeros((N, order, 4) if side == "left" else (N, 4, order))
    B[0] = rng.integers(-50, 50, B.shape[1:])
    op = T[0] if trans == "N" else T[0].T
    want = 3.0 * (op @ B[0] if side == "left" else B[0] @ op)
    got = ref.trmm(B, T, 3.0, side, uplo, trans, diag, nthreads=1)
    assert np.array_equal(got[0], want) and np.all(got[1] == 0)


@pytest.mark.parametrize("N", [2, 3, 4])
def test_oracle_syrk_packed_matches_reference_model(ref, rng, N):
    """runtests.jl:493-520: 11 x 9 panel, rows 2..10, alpha 2, beta -3"""
    P = syn.randn_mf(rng, N, 11, 9)
    init = syn.randn_mf(rng, N, 45, 1)[:, :, 0]
    al, be = ref._scalar(N, 2.0), ref._scalar(N, -3.0)
    want = np.empty_like(init)
    idx = 0
    for col in range(9):
        for row in range(col, 9):
            acc = np.zeros(N)
            for k in range(1, 10):
                acc = ref.add(acc, ref.mul(P[:, k, row], P[:, k, col]))
            want[:, idx] = ref.add(ref.mul(al, acc), ref.mul(be, init[:, idx]))
            idx += 1
    got = ref.syrk_packed(init, P, al, be, reduction_first=2, reduction_last=10, nthreads=1)
    assert_bitwise(got, want, "packed")
    # beta = 0 never reads the destination; the packed order is the lower triangle's
    stale = ref.syrk_packed(np.full((N, 45), np.nan), P, nthreads=1)
    clean = ref.syrk_packed(np.zeros((N, 45)), P, nthreads=1)
    assert_bitwise(stale, clean, "stale")
    full = ref.syrk_lower(P, np.zeros((N, 9, 9)), nthreads=1)
    il = np.tril_indices(9)
    order = np.lexsort((il[0], il[1]))  # column-major over the lower triangle
    assert_bitwise(clean, full[:, il[0][order], il[1][order]], "packed order")
