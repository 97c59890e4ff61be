"""The allocation-free reduction entry point against the handle-based one.

mflab_max_abs_noalloc exists for callers that cannot let the library
allocate device memory (their device memory belongs to their own pool
allocator, or they cannot take the implicit synchronisation of
cudaMalloc/cudaFree mid-pipeline).  It keeps its partial results in a fixed
device array instead of handle scratch.  This file is collected last so that a
failure here does not stop a `-x` run before the other tests have run.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from test_oracle import syn

pytestmark = pytest.mark.gpu


def _with_handle(mf, A, region):
    lib = mf._native.load()
    out = torch.full((A.N + 1,), -7.0, dtype=torch.float64, device=A.storage.device)
    rc = lib.mflab_max_abs(mf._handle(A.device), mf._stream(A.device), A.N, A.m, A.n, A.ptr(),
                           A.ld, A.ls, region, out.data_ptr())
    assert rc == 0
    return out.cpu().numpy()


def _no_alloc(mf, A, region):
    lib = mf._native.load()
    out = torch.full((A.N + 1,), -7.0, dtype=torch.float64, device=A.storage.device)
    rc = lib.mflab_max_abs_noalloc(mf._stream(A.device), A.N, A.m, A.n, A.ptr(), A.ld, A.ls,
                                   region, out.data_ptr())
    assert rc == 0, lib.mflab_last_error()
    return out.cpu().numpy()


@pytest.mark.parametrize("N", [2, 3, 4])
def test_noalloc_matches_handle_version_on_consecutive_calls(mf, N):
    """two calls in a row: the second has fewer columns and smaller entries, so
    records left over from the first call would show up in its result"""
    rng = np.random.default_rng(99)
    cases = [(300, 200, 1e10, False), (150, 90, 1.0, True)]
    for m, n, scale, with_nan in cases:
        X = syn.randn_mf(rng, N, m, n, scale=scale)
        if with_nan:
            X[0, m - 1, 0] = np.nan  # only in the lower triangle
        A = mf.MFMatrix.from_numpy(X)
        for region in (0, 1, 2):
            got = _no_alloc(mf, A, region)
            want = _with_handle(mf, A, region)
            # the maximum of absolute values is exact: bitwise equality
            assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), (m, n, region)
        torch.cuda.synchronize()


def test_noalloc_rejects_more_columns_than_its_scratch(mf):
    lib = mf._native.load()
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    A = mf.MFMatrix.zeros(2, 1, 16385)
    rc = lib.mflab_max_abs_noalloc(mf._stream(A.device), 2, A.m, A.n, A.ptr(), A.ld, A.ls, 0,
                                   out.data_ptr())
    assert rc == mf._native.MFLAB_ERR_UNSUPPORTED
    assert b"16384" in lib.mflab_last_error()
