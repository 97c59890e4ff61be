"""The device data path of the 2-D GEMM split on one GPU (the scatter and
gather degenerate to copies): the tile product through the device GEMM is
bitwise the single-call result, plain and INT8 routes, with beta."""
import numpy as np
import pytest

from conftest import assert_bitwise
from test_oracle import syn

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N", [2, 4])
@pytest.mark.parametrize("route", ["plain", "modular"])
def test_sharded_gemm_device_path_one_rank(mf, rng, N, route):
    from mflab200 import sharding
    m, k, n = 300, 257, 190
    A, B = syn.randn_mf(rng, N, m, k, spread=8), syn.randn_mf(rng, N, k, n, spread=8)
    C0 = syn.randn_mf(rng, N, m, n)
    cfg = mf.KernelConfig() if route == "plain" else \
        mf.KernelConfig(gemm_strategy="ozaki", ozaki_scheme="modular", ozaki_moduli=20)
    Ad, Bd = mf.MFMatrix.from_numpy(A), mf.MFMatrix.from_numpy(B)
    want = mf.MFMatrix.from_numpy(C0)
    mf.gemm_(want, Ad, Bd, 1.0, 0.5, config=cfg)
    Cd = mf.MFMatrix.from_numpy(C0)
    out = sharding.gemm_sharded_(Cd.storage, Ad.storage, Bd.storage, 1.0, 0.5, config=cfg)
    assert out is Cd.storage
    assert_bitwise(Cd.to_numpy(), want.to_numpy(), "sharded vs single call")
