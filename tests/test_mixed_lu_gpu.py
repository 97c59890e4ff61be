"""FP64-factor / Float64xN-refinement LU solver: the binary64 LU instance and
the refinement loop reach the Float64xN backward error."""
import numpy as np
import pytest
import torch

from test_oracle import syn

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N", [2, 4])
@pytest.mark.parametrize("n", [7, 64, 150])
def test_mixed_lu_converges(mf, ref, rng, N, n):
    A = syn.randn_mf(rng, N, n, n)
    B = syn.randn_mf(rng, N, n, 3)
    X, rep = mf.solve_mixed_lu(mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B))
    assert rep["converged"], rep
    be = ref.backward_error(A, X.to_numpy(), B)
    assert np.all(be <= 4 * 2.0 ** (-53 * N)), be


def test_mixed_lu_ill_conditioned(mf, ref):
    """A = U diag(sigma) V^T, sigma from 1 to 1e-12 (the mixed-LU workload
    shape), refinement to a Float64x4 backward error below 1e-60"""
    from mflab200 import synthetic
    A, B = synthetic.mixed_lu_problem(mf, 128, 4, seed=1)
    X, rep = mf.solve_mixed_lu(A, B, tol=1e-60)
    assert rep["converged"] and rep["backward_error"] <= 1e-60, rep
    be = ref.backward_error(A.to_numpy(), X.to_numpy(), B.to_numpy())
    assert np.all(be <= 1e-60)


def test_binary64_lu_factor(mf, rng):
    """limbs = 1 LU: P A = L U to binary64 backward accuracy"""
    n = 90
    A = rng.standard_normal((n, n))
    Ad = mf.MFMatrix(torch.tensor(A.T.copy()[None], device="cuda"))
    lib, h, s = mf._lib_h(Ad)
    ipiv = torch.arange(1, n + 1, dtype=torch.int64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.mflab_getrf(h, s, 1, n, n, Ad.ptr(), Ad.ld, Ad.ls, ipiv.data_ptr(), 16,
                           info.data_ptr()) == 0
    assert int(info.item()) == 0
    LU = Ad.storage[0].cpu().numpy().T
    L = np.tril(LU, -1) + np.eye(n)
    U = np.triu(LU)
    PA = A.copy()
    for k, p in enumerate(ipiv.cpu().numpy()):
        PA[[k, p - 1]] = PA[[p - 1, k]]
    assert np.max(np.abs(PA - L @ U)) <= 1e-12 * np.max(np.abs(A)) * n


@pytest.mark.parametrize("n,nrhs", [(129, 3), (300, 16), (1000, 5)])
def test_binary64_getrs_blocked(mf, rng, n, nrhs):
    """limbs = 1 solve (blocked 64 x 64 diagonal solves + FP64 GEMM updates):
    P A X = B to binary64 backward accuracy"""
    A = rng.standard_normal((n, n)) + n ** 0.5 * np.eye(n)
    B = rng.standard_normal((n, nrhs))
    Ad = mf.MFMatrix(torch.tensor(A.T.copy()[None], device="cuda"))
    Bd = mf.MFMatrix(torch.tensor(B.T.copy()[None], device="cuda"))
    lib, h, s = mf._lib_h(Ad)
    ipiv = torch.arange(1, n + 1, dtype=torch.int64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.mflab_getrf(h, s, 1, n, n, Ad.ptr(), Ad.ld, Ad.ls, ipiv.data_ptr(), 16,
                           info.data_ptr()) == 0
    assert lib.mflab_getrs(h, s, 1, n, nrhs, Ad.ptr(), Ad.ld, Ad.ls, ipiv.data_ptr(), Bd.ptr(),
                           Bd.ld, Bd.ls) == 0
    X = Bd.storage[0].cpu().numpy().T
    r = B - A @ X
    be = np.max(np.abs(r)) / (np.max(np.sum(np.abs(A), 1)) * np.max(np.abs(X)) + np.max(np.abs(B)))
    assert be <= 64 * n * 2.0 ** -53, be


@pytest.mark.parametrize("N", [2, 4])
def test_mixed_lu_residual_routes(mf, ref, rng, N):
    """the INT8 residual and the reference-order residual both refine to the
    Float64xN backward error"""
    n = 200
    A = syn.randn_mf(rng, N, n, n)
    B = syn.randn_mf(rng, N, n, 4)
    for route in ("int8", "matched"):
        X, rep = mf.solve_mixed_lu(mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B),
                                   residual=route)
        assert rep["converged"], (route, rep)
        be = ref.backward_error(A, X.to_numpy(), B)
        assert np.all(be <= 4 * 2.0 ** (-53 * N)), (route, be)


@pytest.mark.parametrize("N", [2, 3, 4])
def test_backward_error_with_cached_norm(mf, rng, N):
    """normwise_backward_error with an OpNormInf equals the one-call form bit for bit"""
    n, k = 120, 6
    A, X, B, R = (syn.randn_mf(rng, N, n, n), syn.randn_mf(rng, N, n, k),
                  syn.randn_mf(rng, N, n, k), syn.randn_mf(rng, N, n, k))
    Ad, Xd, Bd, Rd = (mf.MFMatrix.from_numpy(v) for v in (A, X, B, R))
    a = mf.normwise_backward_error(Ad, Xd, Bd, Rd)
    b = mf.normwise_backward_error(Ad, Xd, Bd, Rd, anorm=mf.OpNormInf(Ad))
    assert np.array_equal(np.array(a).view(np.uint64), np.array(b).view(np.uint64))
    # the norm formed on a side stream with a handle of its own (as the mixed
    # solve does while its factor runs) is the same value
    side, h2 = torch.cuda.Stream(), mf.create_handle()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        an2 = mf.OpNormInf(Ad, handle=h2)
    torch.cuda.current_stream().wait_stream(side)
    c = mf.normwise_backward_error(Ad, Xd, Bd, Rd, anorm=an2)
    torch.cuda.synchronize()
    mf.destroy_handle(h2)
    assert np.array_equal(np.array(a).view(np.uint64), np.array(c).view(np.uint64))


@pytest.mark.parametrize("m,n", [(300, 300), (257, 130), (130, 257)])
def test_binary64_lu_panels(mf, rng, m, n):
    """the 32-column panel binary64 LU: P A = L U for square and rectangular
    shapes, and a zero column reported at its index"""
    A = rng.standard_normal((m, n))
    Ad = mf.MFMatrix(torch.tensor(A.T.copy()[None], device="cuda"))
    lib, h, s = mf._lib_h(Ad)
    kmax = min(m, n)
    ipiv = torch.arange(1, kmax + 1, dtype=torch.int64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.mflab_getrf(h, s, 1, m, n, Ad.ptr(), Ad.ld, Ad.ls, ipiv.data_ptr(), 16,
                           info.data_ptr()) == 0
    assert int(info.item()) == 0
    LU = Ad.storage[0].cpu().numpy().T
    L = np.tril(LU, -1)[:, :kmax] + np.eye(m, kmax)
    U = np.triu(LU)[:kmax, :]
    PA = A.copy()
    for k, p in enumerate(ipiv.cpu().numpy()):
        PA[[k, p - 1]] = PA[[p - 1, k]]
    assert np.max(np.abs(PA - L @ U)) <= 1e-12 * np.max(np.abs(A)) * max(m, n)
    Z = A.copy()
    Z[:, 57] = 0.0
    Zd = mf.MFMatrix(torch.tensor(Z.T.copy()[None], device="cuda"))
    assert lib.mflab_getrf(h, s, 1, m, n, Zd.ptr(), Zd.ld, Zd.ls, ipiv.data_ptr(), 16,
                           info.data_ptr()) == 0
    assert int(info.item()) == 58
