"""Parity at the benchmark workloads' own sizes, on their own input
distributions, against the oracle:

* plain Float64x2 GEMM, n = 256 (bitwise against the reference-order GEMM);
* Cholesky + 64-RHS solve, n = 2048, Float64x2/x3/x4 (bitwise factor and
  solve; exact backward error from the superaccumulator residual);
* INT8 modular GEMM against the plain kernel, m = n = k = 8192, Float64x2/x4,
  entries randn 2^U(-20,20) (componentwise error on sampled entries);
* mixed-precision LU solve, n = 4096, 16 RHS (exact backward error <= 1e-60);
* 10,000 batched Float64x2 SPD blocks, sizes U{8..256} (sampled blocks
  bitwise against the oracle's per-block Cholesky and solve).

Tolerances: bitwise where the order is the reference's; otherwise the
reference's 4096 k eps(T) (runtests.jl:25-29) and twice the plain kernel's
sampled error for the INT8 route."""
import numpy as np
import pytest
import torch

from conftest import assert_bitwise
from test_oracle import syn

pytestmark = pytest.mark.gpu


def _dsyn(mf):
    from importlib import import_module
    return import_module("mflab200.synthetic")


def test_gemm_x2_n256(mf, ref):
    """the plain Float64x2 GEMM workload: limb 0 randn, limb 1 randn 2^-53
    |limb 0| (renormalised), C zero-initialised, seed 1"""
    rng = np.random.default_rng(1)
    n = 256
    A, B = syn.randn_mf(rng, 2, n, n), syn.randn_mf(rng, 2, n, n)
    Cd = mf.MFMatrix.zeros(2, n, n)
    mf.gemm_(Cd, mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B))
    C = Cd.to_numpy()
    assert_bitwise(C, ref.gemm(A, B), "gemm x2 n=256")
    rows, cols = np.divmod(np.arange(0, n * n, 97), n)
    err, scale, _ = ref.exact_gemm_check(A, B, C, rows, cols)
    assert np.max(err / scale) <= 4096 * n * 2.0 ** -104


@pytest.mark.parametrize("N", [2, 3, 4])
def test_cholesky_n2048_rhs64(mf, ref, N):
    n, nrhs = 2048, 64
    dsyn = _dsyn(mf)
    S = dsyn.spd_matrix_device(mf, 70 + N, N, n)
    Sn = S.to_numpy()
    B = syn.randn_mf(np.random.default_rng(80 + N), N, n, nrhs)
    Sw = S.copy()
    F = mf.cholesky_(Sw)
    L, info = ref.potrf(Sn)
    assert info == 0 and mf.factor_status(F) == 0
    assert_bitwise(np.tril(Sw.to_numpy()), np.tril(L), f"cholesky x{N} n=2048")
    X = mf.solve(F, mf.MFMatrix.from_numpy(B)).to_numpy()
    Xr = ref.potrs(L, B)
    assert_bitwise(X, Xr, f"cholesky solve x{N} n=2048, 64 RHS")
    cols = [0, 21, 42, 63]  # exact residuals of four columns
    be = ref.backward_error(Sn, X[:, :, cols], B[:, :, cols])
    assert np.all(be <= 4096 * n * 2.0 ** (-52 * N)), be


def _sampled_error(ref, A, B, C, rows, cols):
    """componentwise error of C[rows[j], cols[j]] from the sampled rows of A
    and columns of B only"""
    As = A.planes()[:, :, rows].cpu().numpy().transpose(0, 2, 1)       # (N, s, k)
    Bs = B.planes()[:, cols, :].cpu().numpy().transpose(0, 2, 1)       # (N, k, s)
    Cs = C.planes()[:, cols, rows].cpu().numpy()                       # (N, s)
    s = len(rows)
    Cm = np.zeros((C.N, s, s))
    Cm[:, np.arange(s), np.arange(s)] = Cs
    err, scale, _ = ref.exact_gemm_check(np.ascontiguousarray(As), np.ascontiguousarray(Bs), Cm,
                                         np.arange(s), np.arange(s))
    return float(np.max(err / scale))


@pytest.mark.parametrize("N", [2, 4])
def test_int8_modular_vs_plain_n8192(mf, ref, N):
    n = 8192
    dsyn = _dsyn(mf)
    A = mf.MFMatrix.from_tensor(dsyn.randn_mf_device(1000, N, n, n, spread=20))
    B = mf.MFMatrix.from_tensor(dsyn.randn_mf_device(2000, N, n, n, spread=20))
    rs = np.random.default_rng(5)
    rows, cols = rs.integers(0, n, 256), rs.integers(0, n, 256)
    C = mf.MFMatrix.zeros(N, n, n)
    mf.gemm_(C, A, B)
    e_plain = _sampled_error(ref, A, B, C, rows, cols)
    mf.gemm_(C, A, B, config=mf.KernelConfig(gemm_strategy="ozaki", ozaki_scheme="modular"))
    assert mf.device_status() == 0
    e_int8 = _sampled_error(ref, A, B, C, rows, cols)
    assert e_plain <= 4096 * n * 2.0 ** (-52 * N)
    assert e_int8 <= 4096 * n * 2.0 ** (-52 * N)
    assert e_int8 <= 2 * e_plain + 2.0 ** (-53 * N), (e_int8, e_plain, mf.ozaki_last_moduli())


def test_mixed_lu_n4096_rhs16(mf, ref):
    dsyn = _dsyn(mf)
    A, B = dsyn.mixed_lu_problem(mf, 4096, 16, seed=4)
    X, rep = mf.solve_mixed_lu(A, B, tol=1e-60)
    assert rep["converged"] and rep["backward_error"] <= 1e-60
    cols = [0, 5, 10, 15]
    An = A.to_numpy()
    be = ref.backward_error(An, X.to_numpy()[:, :, cols], B.to_numpy()[:, :, cols])
    assert np.all(be <= 1e-60), be


def test_batched_spd_10000_blocks(mf, ref):
    rng = np.random.default_rng(5)
    sizes = rng.integers(8, 257, 10000)
    batch = mf.batched.SPDBatch(2, sizes)
    _dsyn(mf).spd_batch_fill(mf, batch, seed=5)
    S0, X0 = batch.S.clone(), batch.X.clone()
    graph = mf.batched.BatchedSPDGraph(batch, tuning="auto")
    batch.S.copy_(S0)
    batch.X.copy_(X0)
    graph.replay()
    torch.cuda.synchronize()
    assert not np.any(batch.info[:batch.nblocks].cpu().numpy())
    picks = np.concatenate([np.argsort(-sizes)[:4], np.argsort(sizes)[:4],
                            np.random.default_rng(9).choice(10000, 8, replace=False)])
    for i in picks:
        Si, bi = batch.block(i, S0), batch.rhs(i, X0)
        L, info = ref.potrf(Si)
        x = ref.potrs(L, bi[:, :, None])
        assert info == 0
        assert_bitwise(np.tril(batch.block(i)), np.tril(L), f"block {i} factor")
        assert_bitwise(batch.rhs(i), x[:, :, 0], f"block {i} solve")
    # the graph replays the same bits
    L1, X1 = batch.S.clone(), batch.X.clone()
    batch.S.copy_(S0)
    batch.X.copy_(X0)
    graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(batch.S, L1) and torch.equal(batch.X, X1)
