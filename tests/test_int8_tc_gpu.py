"""The hand-written tcgen05 int8 GEMM (TMA + TMEM) against exact integer
products and against the library engine, alone and inside the INT8-slice
multi-double route."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import assert_bitwise
from test_oracle import syn

pytestmark = pytest.mark.gpu


def _run(mf, engine, A, B, K, b_xoff, mp, np_):
    lib = mf._native.load()
    h = mf._handle(0)
    Cd = torch.full((np_, mp), -1, dtype=torch.int32, device="cuda")  # column-major mp x np
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.mflab_int8_gemm_tn(h, torch.cuda.current_stream().cuda_stream, engine, mp, np_, K,
                                A.data_ptr(), A.shape[1], A.shape[1], B.data_ptr(), B.shape[1],
                                B.shape[1], b_xoff, Cd.data_ptr(), mp, err.data_ptr())
    assert rc == 0, lib.mflab_last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return Cd.cpu().numpy().T  # (mp, np)


@pytest.mark.parametrize("mp,np_,K,b_xoff", [(128, 256, 128, 0), (256, 512, 1024, 0),
                                             (384, 256, 640, 256), (128, 768, 2048, 128)])
def test_tcgen05_int8_gemm_exact(mf, mp, np_, K, b_xoff):
    rng = np.random.default_rng(mp + np_ + K)
    a_cols, b_cols = K, K + b_xoff
    A = rng.integers(-64, 65, (mp, a_cols), dtype=np.int8)
    B = rng.integers(-64, 65, (np_, b_cols), dtype=np.int8)
    want = A[:, :K].astype(np.int64) @ B[:, b_xoff:b_xoff + K].astype(np.int64).T
    Ad, Bd = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    got = _run(mf, 0, Ad, Bd, K, b_xoff, mp, np_)
    assert np.array_equal(got.astype(np.int64), want)
    lib_got = _run(mf, 1, Ad, Bd, K, b_xoff, mp, np_)
    assert np.array_equal(lib_got, got)


@pytest.mark.parametrize("N", [2, 4])
@pytest.mark.parametrize("shape", [(100, 300, 200), (260, 129, 513)], ids=str)
def test_ozaki_route_engines_agree_bitwise(mf, rng, N, shape):
    m, k, n = shape
    A, B = syn.randn_mf(rng, N, m, k, spread=20), syn.randn_mf(rng, N, k, n, spread=20)
    Ad, Bd = mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B)
    out = []
    for engine in ("tcgen05", "library"):
        Cd = mf.MFMatrix.zeros(N, m, n)
        mf.gemm_(Cd, Ad, Bd, config=mf.KernelConfig(gemm_strategy="ozaki", ozaki_slices=12,
                                                    ozaki_engine=engine))
        out.append(Cd.to_numpy())
    assert mf.device_status() == 0
    assert_bitwise(out[0], out[1], "tcgen05 vs library")
