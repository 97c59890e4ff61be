"""The SM-pair tcgen05 int8 GEMM (cta_group::2, two CTAs per 256 x 256
tile) against exact integer products, the one-SM kernel and the library,
alone and inside both INT8 routes (stacked residue problems, the
lower-triangle tiles of the Gram form, m % 256 == 128 row tiles); and the
timeout path of both tcgen05 kernels: an injected wait runs out, the status
word reports it, and the next launch on the same handle is correct."""
import numpy as np
import pytest
import torch

from conftest import assert_bitwise
from test_oracle import syn

pytestmark = pytest.mark.gpu

ONE_SM, LIBRARY, PAIR = 0, 1, 2


def _run(mf, engine, A, B, K, b_xoff, mp, np_, check_err=True):
    lib = mf._native.load()
    h = mf._handle(0)
    Cd = torch.full((np_, mp), -1, dtype=torch.int32, device="cuda")  # column-major mp x np
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.mflab_int8_gemm_tn(h, torch.cuda.current_stream().cuda_stream, engine, mp, np_, K,
                                A.data_ptr(), A.shape[1], A.shape[1], B.data_ptr(), B.shape[1],
                                B.shape[1], b_xoff, Cd.data_ptr(), mp, err.data_ptr())
    assert rc == 0, lib.mflab_last_error()
    torch.cuda.synchronize()
    if check_err:
        assert int(err.item()) == 0
    return Cd.cpu().numpy().T, int(err.item())


def _operands(mp, np_, K, b_xoff, lo=-128, hi=127):
    rng = np.random.default_rng(mp * 7 + np_ * 3 + K)
    A = rng.integers(lo, hi + 1, (mp, K), dtype=np.int8)
    B = rng.integers(lo, hi + 1, (np_, K + b_xoff), dtype=np.int8)
    want = A.astype(np.int64) @ B[:, b_xoff:b_xoff + K].astype(np.int64).T
    return torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda(), want


@pytest.mark.parametrize("mp,np_,K,b_xoff", [(128, 256, 128, 0), (256, 256, 128, 0),
                                             (384, 512, 1024, 256), (640, 768, 640, 128),
                                             (1024, 1024, 4096, 0), (2176, 2304, 256, 0)])
def test_pair_kernel_exact_and_equal_to_other_engines(mf, mp, np_, K, b_xoff):
    A, B, want = _operands(mp, np_, K, b_xoff)
    got, _ = _run(mf, PAIR, A, B, K, b_xoff, mp, np_)
    assert np.array_equal(got.astype(np.int64), want)
    one, _ = _run(mf, ONE_SM, A, B, K, b_xoff, mp, np_)
    lib, _ = _run(mf, LIBRARY, A, B, K, b_xoff, mp, np_)
    assert np.array_equal(one, got) and np.array_equal(lib, got)


def test_pair_kernel_many_tiles_per_pair(mf):
    """more tiles than pairs: each pair walks several tiles, so both
    accumulators alternate and the epilogue overlaps the next tile"""
    mp, np_, K = 4096, 4096, 512
    A, B, want = _operands(mp, np_, K, 0)
    got, _ = _run(mf, PAIR, A, B, K, 0, mp, np_)
    assert np.array_equal(got.astype(np.int64), want)


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("shape", [(100, 300, 200), (260, 129, 513), (300, 1000, 600)], ids=str)
def test_modular_route_pair_equals_one_sm(mf, rng, N, shape):
    m, k, n = shape
    A, B = syn.randn_mf(rng, N, m, k, spread=20), syn.randn_mf(rng, N, k, n, spread=20)
    Ad, Bd = mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B)
    out = []
    for engine in ("tcgen05_pair", "tcgen05_1sm", "library"):
        Cd = mf.MFMatrix.zeros(N, m, n)
        mf.gemm_(Cd, Ad, Bd, config=mf.KernelConfig(gemm_strategy="ozaki", ozaki_scheme="modular",
                                                    ozaki_engine=engine))
        out.append(Cd.to_numpy())
    assert mf.device_status() == 0
    assert_bitwise(out[0], out[1], "pair vs one-SM")
    assert_bitwise(out[0], out[2], "pair vs library")


@pytest.mark.parametrize("N", [2, 4])
def test_slice_route_and_gram_pair_equals_one_sm(mf, rng, N):
    m, k, n = 300, 400, 520
    A, B = syn.randn_mf(rng, N, m, k, spread=10), syn.randn_mf(rng, N, k, n, spread=10)
    Ad, Bd = mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B)
    out = []
    for engine in ("tcgen05_pair", "tcgen05_1sm"):
        Cd = mf.MFMatrix.zeros(N, m, n)
        mf.gemm_(Cd, Ad, Bd, config=mf.KernelConfig(gemm_strategy="ozaki", ozaki_scheme="slices",
                                                    ozaki_slices=9, ozaki_engine=engine))
        out.append(Cd.to_numpy())
    assert_bitwise(out[0], out[1], "slices: pair vs one-SM")
    P = mf.MFMatrix.from_numpy(syn.randn_mf(rng, N, 700, 600, spread=10))
    gram = []
    for engine in ("tcgen05_pair", "tcgen05_1sm"):
        Cd = mf.MFMatrix.from_numpy(np.full((N, 600, 600), np.nan))
        mf.syrk_(Cd, P, config=mf.KernelConfig(gemm_strategy="ozaki", ozaki_scheme="modular",
                                               ozaki_engine=engine))
        gram.append(np.tril(Cd.to_numpy()))
    assert mf.device_status() == 0
    assert_bitwise(gram[0], gram[1], "syrk lower tiles: pair vs one-SM")


@pytest.mark.parametrize("engine", [ONE_SM, PAIR])
def test_injected_timeout_is_reported_and_recovers(mf, engine):
    """an injected wait that nothing completes runs out: the kernel reports
    the MMA issuer's timeout (2) with its copies still in flight, drains and
    returns; the same handle then multiplies correctly"""
    lib = mf._native.load()
    h = mf._handle(0)
    mp, np_, K = 512, 512, 2048
    A, B, want = _operands(mp, np_, K, 0)
    assert lib.mflab_set_tc_debug(h, 0, 1) == 0
    try:
        _, err = _run(mf, engine, A, B, K, 0, mp, np_, check_err=False)
    finally:
        assert lib.mflab_set_tc_debug(h, 0, 0) == 0
    assert err == 2
    for _ in range(2):
        got, err = _run(mf, engine, A, B, K, 0, mp, np_)
        assert err == 0 and np.array_equal(got.astype(np.int64), want)


def test_debug_hook_arguments(mf):
    lib = mf._native.load()
    h = mf._handle(0)
    assert lib.mflab_set_tc_debug(h, -1, 0) == mf._native.MFLAB_ERR_ARG
    assert lib.mflab_set_tc_debug(h, 0, 3) == mf._native.MFLAB_ERR_FLAG
    assert lib.mflab_set_tc_debug(h, 0, 0) == 0
