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
