"""The debug build (libmflab200_debug.so, -DMFLAB_DEBUG: device index checks
that record a violation instead of trapping) runs the hot paths with no
recorded violation and the same bits as the release build: the modular INT8
GEMM on both tcgen05 engines and the library, the matched GEMM, Cholesky,
the binary64 LU with its prepared solves, and the interleaved copies."""
import ctypes as C
import os

import numpy as np
import pytest
import torch

from conftest import assert_bitwise
from test_oracle import syn

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def libs(mf):
    nat = mf._native
    if not os.path.exists(nat.DEBUG_LIB_PATH):
        pytest.fail("debug library not built (build() builds it beside the release one)")
    rel, dbg = nat.load(), nat.load_library(nat.DEBUG_LIB_PATH)
    out = {}
    for name, lib in (("release", rel), ("debug", dbg)):
        h = C.c_void_p()
        assert lib.mflab_create(C.byref(h), 0) == 0
        out[name] = (lib, h)
    zero = (C.c_longlong * 4)()
    assert dbg.mflab_debug_violations(zero, 1) == 0
    yield out
    for lib, h in out.values():
        lib.mflab_destroy(h)


def _violations(libs):
    lib, _ = libs["debug"]
    v = (C.c_longlong * 4)()
    assert lib.mflab_debug_violations(v, 1) == 0
    return list(v)


def _stream():
    return torch.cuda.current_stream().cuda_stream


def _run_both(libs, fn):
    res = {}
    for name, (lib, h) in libs.items():
        res[name] = fn(lib, h)
    torch.cuda.synchronize()
    return res


def _planes(X):
    return torch.tensor(np.ascontiguousarray(np.transpose(X, (0, 2, 1))), device="cuda")


def _numpy(T):
    return np.transpose(T.cpu().numpy(), (0, 2, 1))


@pytest.mark.parametrize("engine", [0, 1, 2])
@pytest.mark.parametrize("N", [2, 4])
def test_modular_gemm(mf, libs, rng, N, engine):
    m, k, n, T = 300, 513, 260, 20
    A, B = syn.randn_mf(rng, N, m, k, spread=10), syn.randn_mf(rng, N, k, n, spread=10)
    one, zero = (C.c_double * 4)(1.0), (C.c_double * 4)()

    def run(lib, h):
        Ad, Bd = _planes(A), _planes(B)
        Cd = torch.zeros((N, n, m), dtype=torch.float64, device="cuda")
        assert lib.mflab_set_int8_engine(h, engine) == 0
        rc = lib.mflab_gemm_ozaki_crt(h, _stream(), N, T, m, n, k, Ad.data_ptr(), m, m * k,
                                      Bd.data_ptr(), k, k * n, Cd.data_ptr(), m, m * n, one, zero)
        assert rc == 0, (rc, lib.mflab_last_error())
        return _numpy(Cd)

    r = _run_both(libs, run)
    assert_bitwise(r["debug"], r["release"], "modular GEMM")
    assert _violations(libs)[0] == 0


def test_matched_gemm_and_cholesky(mf, libs, rng):
    N, m, k, n = 2, 130, 70, 90
    A, B = syn.randn_mf(rng, N, m, k), syn.randn_mf(rng, N, k, n)
    one, zero = (C.c_double * 4)(1.0), (C.c_double * 4)()
    R = syn.randn_mf(rng, N, 200, 200)
    S = np.zeros_like(R)
    S[0] = R[0] @ R[0].T + 200 * np.eye(200)

    def run(lib, h):
        Ad, Bd = _planes(A), _planes(B)
        Cd = torch.zeros((N, n, m), dtype=torch.float64, device="cuda")
        assert lib.mflab_gemm(h, _stream(), N, 0, m, n, k, Ad.data_ptr(), m, m * k, Bd.data_ptr(),
                              k, k * n, Cd.data_ptr(), m, m * n, one, zero) == 0
        Sd = _planes(S)
        info = torch.zeros(1, dtype=torch.int32, device="cuda")
        assert lib.mflab_potrf(h, _stream(), N, 200, Sd.data_ptr(), 200, 200 * 200, 16,
                               info.data_ptr()) == 0
        return _numpy(Cd), _numpy(Sd), int(info.item())

    r = _run_both(libs, run)
    assert_bitwise(r["debug"][0], r["release"][0], "matched GEMM")
    assert_bitwise(np.tril(r["debug"][1][0]), np.tril(r["release"][1][0]), "Cholesky")
    assert r["debug"][2] == r["release"][2] == 0
    assert _violations(libs)[0] == 0


def test_binary64_lu_and_prepared_solves(mf, libs, rng):
    n, nrhs = 700, 5
    A = rng.standard_normal((n, n)) + 3 * np.eye(n)
    Bm = rng.standard_normal((n, nrhs))

    def run(lib, h):
        LU = torch.tensor(A.T.copy(), device="cuda")
        ipiv = torch.zeros(n, dtype=torch.int64, device="cuda")
        info = torch.zeros(1, dtype=torch.int32, device="cuda")
        assert lib.mflab_getrf(h, _stream(), 1, n, n, LU.data_ptr(), n, n * n, ipiv.data_ptr(), 32,
                               info.data_ptr()) == 0
        wb = C.c_size_t()
        assert lib.mflab_lu64_work_bytes(n, C.byref(wb)) == 0
        work = torch.empty(wb.value, dtype=torch.uint8, device="cuda")
        assert lib.mflab_lu64_prepare(h, _stream(), n, LU.data_ptr(), n, ipiv.data_ptr(),
                                      work.data_ptr()) == 0
        X = torch.tensor(Bm.T.copy(), device="cuda")
        assert lib.mflab_lu64_solve(h, _stream(), n, nrhs, LU.data_ptr(), n, work.data_ptr(),
                                    X.data_ptr(), n) == 0
        return LU.cpu().numpy(), ipiv.cpu().numpy(), X.cpu().numpy()

    r = _run_both(libs, run)
    for a, b in zip(r["debug"], r["release"]):
        assert np.array_equal(a, b)
    assert _violations(libs)[0] == 0


def test_interleaved_copies(mf, libs, rng):
    N, m, n = 3, 77, 41
    X = syn.randn_mf(rng, N, m, n)
    host = torch.tensor(np.ascontiguousarray(np.transpose(X, (2, 1, 0))))  # (n, m, N) interleaved
    host = host.pin_memory()

    def run(lib, h):
        P = torch.zeros((N, n, m), dtype=torch.float64, device="cuda")
        assert lib.mflab_h2d_interleaved(h, _stream(), N, m, n, host.data_ptr(), m, P.data_ptr(),
                                         m, m * n) == 0
        back = torch.zeros_like(host).pin_memory()
        assert lib.mflab_d2h_interleaved(h, _stream(), N, m, n, P.data_ptr(), m, m * n,
                                         back.data_ptr(), m) == 0
        torch.cuda.synchronize()
        return _numpy(P), back.numpy().copy()

    r = _run_both(libs, run)
    assert_bitwise(r["debug"][0], X, "to planes")
    assert np.array_equal(r["debug"][1], host.numpy())
    assert_bitwise(r["release"][0], X, "to planes (release)")
    assert _violations(libs)[0] == 0
