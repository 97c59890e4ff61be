"""Interleaved Float64xN storage (a Julia Matrix{MultiFloat{Float64,N}}:
the N limbs of an element side by side, gemm.jl:747-755) to limb planes and
back through the C ABI, bit for bit against a numpy transpose: host and
device forms, padded leading dimensions, views, chunked staging, odd
alignment and empty shapes."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import assert_bitwise
from test_oracle import syn

pytestmark = pytest.mark.gpu


def _interleaved(X, ld=None):
    """(N, m, n) limb-major -> (n, ld, N) interleaved host array"""
    N, m, n = X.shape
    out = np.full((n, ld or m, N), np.nan)
    out[:, :m, :] = X.transpose(2, 1, 0)
    return out


@pytest.mark.parametrize("N", [1, 2, 3, 4])
@pytest.mark.parametrize("m,n,pad", [(1, 1, 0), (37, 20, 0), (300, 129, 5), (1000, 33, 1)])
def test_roundtrip_host(mf, rng, N, m, n, pad):
    X = syn.randn_mf(rng, N, m, n)
    H = _interleaved(X, m + pad)
    M = mf.MFMatrix.from_interleaved(H, m=m)
    assert (M.N, M.m, M.n) == (N, m, n)
    assert_bitwise(M.to_numpy(), X, "h2d")
    assert_bitwise(M.to_interleaved(), X.transpose(2, 1, 0), "d2h")


@pytest.mark.parametrize("N", [2, 4])
def test_pinned_and_view_destination(mf, rng, N):
    m, n = 200, 150
    X = syn.randn_mf(rng, N, m, n)
    H = torch.from_numpy(_interleaved(X)).pin_memory()
    big = mf.MFMatrix.zeros(N, m + 30, n + 20)
    V = big.view(slice(10, 10 + m), slice(7, 7 + n))
    V.copy_from_interleaved_(H)
    out = torch.empty((n, m, N), dtype=torch.float64).pin_memory()
    V.copy_to_interleaved_(out)
    torch.cuda.synchronize()
    assert_bitwise(V.to_numpy(), X, "h2d into a view")
    assert_bitwise(out.numpy(), X.transpose(2, 1, 0), "d2h from a view")
    rest = big.to_numpy()
    rest[:, 10:10 + m, 7:7 + n] = 0
    assert not np.any(rest), "a view upload wrote outside the view"


@pytest.mark.parametrize("N,m,n", [(4, 1000, 5000), (2, 2100000, 2)])
def test_chunked_staging(mf, N, m, n):
    """more than one 32 MiB staging chunk: whole-column chunks, and row
    chunks of single columns taller than a chunk"""
    g = np.random.default_rng(3)
    X = g.standard_normal((N, m, n))
    M = mf.MFMatrix.from_interleaved(np.ascontiguousarray(X.transpose(2, 1, 0)))
    assert_bitwise(M.to_numpy(), X, "h2d chunked")
    assert_bitwise(M.to_interleaved(), X.transpose(2, 1, 0), "d2h chunked")


@pytest.mark.parametrize("N", [1, 2, 3, 4])
@pytest.mark.parametrize("offset", [0, 1])
def test_device_forms(mf, rng, N, offset):
    """device interleaved <-> planes, also from a base that is only 8-byte
    aligned (the scalar path)"""
    m, n = 77, 45
    X = syn.randn_mf(rng, N, m, n)
    Hd = torch.zeros(n * m * N + offset, dtype=torch.float64, device="cuda")
    Hd[offset:] = torch.from_numpy(X.transpose(2, 1, 0).reshape(-1)).cuda()
    P = mf.MFMatrix.empty(N, m, n)
    lib, h, s = mf._lib_h(P)
    base = Hd.data_ptr() + 8 * offset
    assert lib.mflab_interleaved_to_planes(h, s, N, m, n, base, m, P.ptr(), P.ld, P.ls) == 0
    assert_bitwise(P.to_numpy(), X, "device to planes")
    Hd.zero_()
    assert lib.mflab_planes_to_interleaved(h, s, N, m, n, P.ptr(), P.ld, P.ls, base, m) == 0
    got = Hd[offset:].cpu().numpy().reshape(n, m, N)
    assert_bitwise(got, X.transpose(2, 1, 0), "planes to device")


def test_empty_and_errors(mf):
    E = mf.MFMatrix.from_interleaved(np.zeros((0, 5, 2)), m=5)
    assert E.shape == (5, 0)
    assert mf.MFMatrix.zeros(2, 0, 3).to_interleaved().shape == (3, 0, 2)
    M = mf.MFMatrix.zeros(2, 10, 4)
    with pytest.raises(mf.DimensionMismatch):
        M.copy_from_interleaved_(np.zeros((4, 9, 2)))   # ld < m
    with pytest.raises(mf.DimensionMismatch):
        M.copy_from_interleaved_(np.zeros((4, 10, 3)))  # limb count
    lib, h, s = mf._lib_h(M)
    buf = np.zeros((4, 10, 2))
    assert lib.mflab_h2d_interleaved(h, s, 2, 10, 4, buf.ctypes.data, 9, M.ptr(), M.ld,
                                     M.ls) == mf._native.MFLAB_ERR_ARG
    assert lib.mflab_h2d_interleaved(h, s, 5, 10, 4, buf.ctypes.data, 10, M.ptr(), M.ld,
                                     M.ls) == mf._native.MFLAB_ERR_UNSUPPORTED
