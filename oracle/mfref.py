"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle restates MultiFloatLinearAlgebra.jl's loop orders and multi-double
networks on the CPU (oracle/mfref.cc).  Only the test-suite, the smoke check
and the CPU-baseline leg of bench.py load it, as the checker.  The product
(the CUDA library and its Python host layer) never imports this module.

Interchange format: a Float64xN matrix with m rows and n columns is a numpy
float64 array of shape (N, m, n); limb l of element (i, j) is X[l, i, j].
Internally the oracle uses N column-major planes, exactly like the device.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None

_d = C.POINTER(C.c_double)
_i64 = C.c_int64
_pi64 = C.POINTER(C.c_int64)
_pu8 = C.POINTER(C.c_uint8)


def _cpu_has(*flags: str) -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            text = f.read()
    except OSError:
        return False
    for line in text.splitlines():
        if line.startswith("flags"):
            have = set(line.split(":", 1)[1].split())
            return all(fl in have for fl in flags)
    return False


def build(quiet: bool = True) -> None:
    """Compile the oracle libraries in place (make -C oracle)."""
    out = subprocess.run(["make", "-C", _HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    name = "libmfref_avx2.so" if _cpu_has("avx2", "fma") else "libmfref.so"
    path = os.path.join(_HERE, name)
    if not os.path.exists(path):
        build()
    L = C.CDLL(path)
    sig = {
        "mfr_add": [C.c_int, _d, _d, _d],
        "mfr_sub": [C.c_int, _d, _d, _d],
        "mfr_mul": [C.c_int, _d, _d, _d],
        "mfr_div": [C.c_int, _d, _d, _d],
        "mfr_sqrt": [C.c_int, _d, _d],
        "mfr_inv": [C.c_int, _d, _d],
        "mfr_mulacc_x3": [_d, _d, _d, _d],
        "mfr_add_n": [C.c_int, _i64, _d, _d, _d, _i64],
        "mfr_mul_n": [C.c_int, _i64, _d, _d, _d, _i64],
        "mfr_gemm": [C.c_int, _i64, _i64, _i64, _d, _i64, _i64, _d, _i64, _i64, _d, _i64, _i64,
                     _d, _d, C.c_int, C.c_int],
        "mfr_syrk_lower": [C.c_int, _i64, _i64, _d, _i64, _i64, _d, _i64, _i64, _d, _d, C.c_int],
        "mfr_gemmt_lower": [C.c_int, _i64, _i64, _d, _i64, _i64, _d, _i64, _i64, _d, _i64, _i64,
                            _d, _d, C.c_int],
        "mfr_trsm": [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _i64, _i64, _d, _i64, _i64, _d,
                     _i64, _i64, _d, C.c_int],
        "mfr_trmm": [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _i64, _i64, _d, _i64, _i64, _d,
                     _i64, _i64, _d, C.c_int],
        "mfr_syrk_packed": [C.c_int, _i64, _i64, _i64, _d, _i64, _i64, _d, _i64, _d, _d, C.c_int],
        "mfr_potrf": [C.c_int, _i64, _d, _i64, _i64, _i64, C.c_int],
        "mfr_pstrf": [C.c_int, _i64, _d, _i64, _i64, _d, _pi64, _pi64, C.c_int],
        "mfr_qr": [C.c_int, _i64, _i64, _d, _i64, _i64, _d, _pi64, _pi64, C.c_int],
        "mfr_rrqr": [C.c_int, _i64, _i64, _d, _i64, _i64, _d, _pi64, _pi64, C.c_int],
        "mfr_apply_q": [C.c_int, _i64, _i64, _d, _i64, _i64, _d, _d, _i64, _i64, _i64, C.c_int,
                        C.c_int],
        "mfr_qr_numerical_rank": [C.c_int, _i64, _i64, _d, _i64, _i64, _d, _d],
        "mfr_potrs": [C.c_int, _i64, _i64, _d, _i64, _i64, _d, _i64, _i64, C.c_int],
        "mfr_getrf": [C.c_int, _i64, _i64, _d, _i64, _i64, _pi64, _i64, C.c_int],
        "mfr_getrs": [C.c_int, _i64, _i64, _d, _i64, _i64, _pi64, _d, _i64, _i64, C.c_int],
        "mfr_sytrf": [C.c_int, _i64, _d, _i64, _i64, _d, _i64, _pi64, _pu8, C.c_int, _i64, C.c_int],
        "mfr_sytrs": [C.c_int, _i64, _i64, _d, _i64, _i64, _d, _i64, _pi64, _pu8, _d, _i64, _i64,
                      C.c_int],
        "mfr_exact_gemm_check": [C.c_int, _i64, _d, _i64, _i64, _d, _i64, _i64, _d, _i64, _i64,
                                 _i64, _pi64, _pi64, _d, _d, _d, C.c_int],
        "mfr_exact_residual": [C.c_int, _i64, _i64, _d, _i64, _i64, _d, _i64, _i64, _d, _i64, _i64,
                               _d, _i64, C.c_int],
        "mfr_to_double": [C.c_int, _i64, _d, _i64, _d],
        "mfr_residual_mixed": [C.c_int, C.c_int, C.c_int, _i64, _i64, _i64, _d, _i64, _i64, _d,
                               _i64, _i64, _d, _i64, _i64, _d, _i64, _i64],
        "mfr_max_threads": [],
    }
    for name_, args in sig.items():
        fn = getattr(L, name_)
        fn.argtypes = args
        fn.restype = C.c_int64 if name_ == "mfr_qr_numerical_rank" else None if name_ in ("mfr_add", "mfr_sub", "mfr_mul", "mfr_div", "mfr_sqrt",
                                       "mfr_inv", "mfr_mulacc_x3", "mfr_add_n", "mfr_mul_n",
                                       "mfr_to_double") else C.c_int
    _lib = L
    return L


def threads() -> int:
    return int(lib().mfr_max_threads())


# ------------------------------------------------------------ layout ----
class Planes:
    """N column-major planes of an (m x n) multi-double matrix, owned numpy."""

    def __init__(self, X: np.ndarray):
        X = np.asarray(X, dtype=np.float64)
        if X.ndim == 2:
            X = X[:, :, None]
        self.N, self.m, self.n = X.shape
        self.buf = np.array(X.transpose(0, 2, 1), order="C", copy=True)  # (N, n, m), owned
        self.ld = max(self.m, 1)
        self.ls = self.n * self.m

    def ptr(self, row: int = 0, col: int = 0):
        base = self.buf.ctypes.data + 8 * (col * self.ld + row)
        return C.cast(C.c_void_p(base), _d)

    def array(self) -> np.ndarray:
        return np.ascontiguousarray(self.buf.transpose(0, 2, 1))


def _scalar(N: int, v) -> np.ndarray:
    out = np.zeros(N, dtype=np.float64)
    v = np.atleast_1d(np.asarray(v, dtype=np.float64))
    out[: len(v)] = v
    return out


def _p(a: np.ndarray):
    return a.ctypes.data_as(_d)


# ------------------------------------------------------------ scalars ---
def add(x, y):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    z = np.empty_like(x)
    lib().mfr_add(len(x), _p(x), _p(y), _p(z))
    return z


def mul(x, y):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    z = np.empty_like(x)
    lib().mfr_mul(len(x), _p(x), _p(y), _p(z))
    return z


def div(x, y):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    z = np.empty_like(x)
    lib().mfr_div(len(x), _p(x), _p(y), _p(z))
    return z


def sqrt(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    z = np.empty_like(x)
    lib().mfr_sqrt(len(x), _p(x), _p(z))
    return z


def mulacc_x3(acc, x, y):
    a = np.ascontiguousarray(acc, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    z = np.empty(3, dtype=np.float64)
    lib().mfr_mulacc_x3(_p(a), _p(x), _p(y), _p(z))
    return z


def add_n(X, Y):
    """elementwise add of arrays shaped (N, ...)"""
    X = np.ascontiguousarray(X, dtype=np.float64)
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    N = X.shape[0]
    cnt = X.size // N
    Z = np.empty_like(X)
    lib().mfr_add_n(N, cnt, _p(X), _p(Y), _p(Z), cnt)
    return Z


def mul_n(X, Y):
    X = np.ascontiguousarray(X, dtype=np.float64)
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    N = X.shape[0]
    cnt = X.size // N
    Z = np.empty_like(X)
    lib().mfr_mul_n(N, cnt, _p(X), _p(Y), _p(Z), cnt)
    return Z


# ------------------------------------------------------------ BLAS ------
def gemm(A, B, C=None, alpha=1.0, beta=0.0, x3_fused=True, nthreads=None):
    """C = alpha*A*B + beta*C (gemm.jl:747-774); returns the new C array."""
    A, B = Planes(A), Planes(B)
    N = A.N
    Cp = Planes(np.zeros((N, A.m, B.n)) if C is None else C)
    al, be = _scalar(N, alpha), _scalar(N, beta)
    rc = lib().mfr_gemm(N, A.m, B.n, A.n, A.ptr(), A.ld, A.ls, B.ptr(), B.ld, B.ls, Cp.ptr(),
                        Cp.ld, Cp.ls, _p(al), _p(be), int(x3_fused), nthreads or threads())
    assert rc == 0
    return Cp.array()


def syrk_lower(P, C, alpha=1.0, beta=0.0, nthreads=None):
    """lower(C) = alpha * P^T P + beta * C (syrk.jl:67-108); P is k x n."""
    Pp, Cp = Planes(P), Planes(C)
    N = Pp.N
    al, be = _scalar(N, alpha), _scalar(N, beta)
    lib().mfr_syrk_lower(N, Pp.n, Pp.m, Pp.ptr(), Pp.ld, Pp.ls, Cp.ptr(), Cp.ld, Cp.ls, _p(al),
                         _p(be), nthreads or threads())
    return Cp.array()


def gemmt_lower(A, B, C, alpha=1.0, beta=0.0, nthreads=None):
    """lower(C) = alpha * A B^T + beta * C (gemmt.jl:69-108)."""
    Ap, Bp, Cp = Planes(A), Planes(B), Planes(C)
    N = Ap.N
    al, be = _scalar(N, alpha), _scalar(N, beta)
    lib().mfr_gemmt_lower(N, Ap.m, Ap.n, Ap.ptr(), Ap.ld, Ap.ls, Bp.ptr(), Bp.ld, Bp.ls, Cp.ptr(),
                          Cp.ld, Cp.ls, _p(al), _p(be), nthreads or threads())
    return Cp.array()


_SIDE = {"left": 0, "right": 1}
_UPLO = {"lower": 0, "upper": 1}
_TRANS = {"N": 0, "T": 1}
_DIAG = {"nonunit": 0, "unit": 1}


def trsm(B, A, alpha=1.0, side="left", uplo="lower", trans="N", diag="nonunit", nthreads=None):
    """trsm.jl:224-302; returns the solved B."""
    Bp, Ap = Planes(B), Planes(A)
    N = Bp.N
    al = _scalar(N, alpha)
    lib().mfr_trsm(N, _SIDE[side], _UPLO[uplo], _TRANS[trans], _DIAG[diag], Bp.m, Bp.n, Ap.ptr(),
                   Ap.ld, Ap.ls, Bp.ptr(), Bp.ld, Bp.ls, _p(al), nthreads or threads())
    return Bp.array()


def trmm(B, A, alpha=1.0, side="left", uplo="lower", trans="N", diag="nonunit", nthreads=None):
    """trmm.jl:82-131; returns the product that overwrites B."""
    Bp, Ap = Planes(B), Planes(A)
    N = Bp.N
    al = _scalar(N, alpha)
    lib().mfr_trmm(N, _SIDE[side], _UPLO[uplo], _TRANS[trans], _DIAG[diag], Bp.m, Bp.n, Ap.ptr(),
                   Ap.ld, Ap.ls, Bp.ptr(), Bp.ld, Bp.ls, _p(al), nthreads or threads())
    return Bp.array()


def syrk_packed(packed, P, alpha=1.0, beta=0.0, reduction_first=1, reduction_last=None,
                nthreads=None):
    """syrk.jl:173-254: packed (N, n(n+1)/2) lower triangle of
    alpha * P[rf:rl,:]^T P[rf:rl,:] + beta * packed, 1-based inclusive bounds."""
    Pp = Planes(P)
    N, n = Pp.N, Pp.n
    rl = Pp.m if reduction_last is None else reduction_last
    out = np.ascontiguousarray(np.asarray(packed, dtype=np.float64).reshape(N, -1).copy())
    assert out.shape[1] == n * (n + 1) // 2 and 1 <= reduction_first <= rl <= Pp.m
    al, be = _scalar(N, alpha), _scalar(N, beta)
    lib().mfr_syrk_packed(N, n, reduction_first - 1, rl, Pp.ptr(), Pp.ld, Pp.ls,
                          out.ctypes.data_as(C.POINTER(C.c_double)), out.shape[1], _p(al), _p(be),
                          nthreads or threads())
    return out


# ------------------------------------------------------- factorizations --
def potrf(A, block=16, nthreads=None):
    """cholesky.jl:68-107 -> (factor array, info)"""
    Ap = Planes(A)
    info = lib().mfr_potrf(Ap.N, Ap.m, Ap.ptr(), Ap.ld, Ap.ls, block, nthreads or threads())
    return Ap.array(), int(info)


def pstrf(A, tol=0.0, nthreads=None):
    """cholesky_pivoted.jl:65-175 -> (factor array, 1-based permutation, rank, info)"""
    Ap = Planes(A)
    N, n = Ap.N, Ap.m
    perm = np.zeros(max(n, 1), dtype=np.int64)
    out = np.zeros(2, dtype=np.int64)
    t = _scalar(N, tol)
    lib().mfr_pstrf(N, n, Ap.ptr(), Ap.ld, Ap.ls, _p(t), perm.ctypes.data_as(_pi64),
                    out.ctypes.data_as(_pi64), nthreads or threads())
    return Ap.array(), perm[:n], int(out[0]), int(out[1])


def _qr_run(fn, A, nthreads):
    Ap = Planes(A)
    N, m, n = Ap.N, Ap.m, Ap.n
    r = min(m, n)
    tau = np.zeros(max(N * r, 1))
    perm = np.zeros(max(n, 1), dtype=np.int64)
    info = np.zeros(1, dtype=np.int64)
    fn(N, m, n, Ap.ptr(), Ap.ld, Ap.ls, _p(tau), perm.ctypes.data_as(_pi64),
       info.ctypes.data_as(_pi64), nthreads or threads())
    return Ap.array(), tau[:N * r].reshape(N, r).copy(), perm[:n], int(info[0])


def qr(A, nthreads=None):
    """qr.jl:763-811 -> (factors, tau (N, r), 1-based permutation, info)"""
    return _qr_run(lib().mfr_qr, A, nthreads)


def rrqr(A, nthreads=None):
    """qr.jl:692-761 (unblocked hybrid or blocked DLAQPS path) -> (factors,
    tau (N, r), 1-based permutation, info)"""
    return _qr_run(lib().mfr_rrqr, A, nthreads)


def apply_q(F, tau, D, trans="N", nthreads=None):
    """qr.jl:890-956: Q D (trans N) or Q^T D (trans T) from the compact factor"""
    Fp, Dp = Planes(F), Planes(D)
    N, r = Fp.N, min(Fp.m, Fp.n)
    t = np.ascontiguousarray(np.asarray(tau, dtype=np.float64).reshape(N, r))
    lib().mfr_apply_q(N, Fp.m, r, Fp.ptr(), Fp.ld, Fp.ls, _p(t), Dp.ptr(), Dp.ld, Dp.ls, Dp.n,
                      1 if trans == "T" else 0, nthreads or threads())
    return Dp.array()


def qr_numerical_rank(F, atol=0.0, rtol=0.0):
    """qr.jl:863-888"""
    Fp = Planes(F)
    N = Fp.N
    return int(lib().mfr_qr_numerical_rank(N, Fp.m, Fp.n, Fp.ptr(), Fp.ld, Fp.ls,
                                           _p(_scalar(N, atol)), _p(_scalar(N, rtol))))


def potrs(L, B, nthreads=None):
    Lp, Bp = Planes(L), Planes(B)
    lib().mfr_potrs(Lp.N, Lp.m, Bp.n, Lp.ptr(), Lp.ld, Lp.ls, Bp.ptr(), Bp.ld, Bp.ls,
                    nthreads or threads())
    return Bp.array()


def getrf(A, block=16, nthreads=None):
    """lu.jl:128-195 -> (factor, ipiv (1-based), info)"""
    Ap = Planes(A)
    kmax = min(Ap.m, Ap.n)
    ipiv = np.zeros(max(kmax, 1), dtype=np.int64)
    info = lib().mfr_getrf(Ap.N, Ap.m, Ap.n, Ap.ptr(), Ap.ld, Ap.ls,
                           ipiv.ctypes.data_as(_pi64), block, nthreads or threads())
    return Ap.array(), ipiv[:kmax], int(info)


def getrs(LU, ipiv, B, nthreads=None):
    Lp, Bp = Planes(LU), Planes(B)
    piv = np.ascontiguousarray(ipiv, dtype=np.int64)
    lib().mfr_getrs(Lp.N, Lp.m, Bp.n, Lp.ptr(), Lp.ld, Lp.ls, piv.ctypes.data_as(_pi64),
                    Bp.ptr(), Bp.ld, Bp.ls, nthreads or threads())
    return Bp.array()


def ldlt_block_default(N: int) -> int:
    """ldlt_tuning.jl:9-15"""
    return 16 if N <= 2 else 12 if N == 3 else 8


def sytrf(A, blocked=None, block=None, crossover=512, nthreads=None):
    """ldlt.jl:654-717 -> (factor, dsub (N, n), pivots (1-based), blocks, info)"""
    Ap = Planes(A)
    N, n = Ap.N, Ap.m
    if block is None:
        block = ldlt_block_default(N)
    if blocked is None:
        blocked = block > 1 and n >= max(crossover, 1)
    dsub = np.zeros((N, max(n, 1)))
    piv = np.zeros(max(n, 1), dtype=np.int64)
    blk = np.zeros(max(n, 1), dtype=np.uint8)
    info = lib().mfr_sytrf(N, n, Ap.ptr(), Ap.ld, Ap.ls, _p(dsub), dsub.shape[1],
                           piv.ctypes.data_as(_pi64), blk.ctypes.data_as(_pu8), int(blocked), block,
                           nthreads or threads())
    return Ap.array(), dsub[:, :n].copy(), piv[:n].copy(), blk[:n].copy(), int(info)


def sytrs(F, dsub, pivots, blocks, B, nthreads=None):
    Fp, Bp = Planes(F), Planes(B)
    ds = np.ascontiguousarray(dsub, dtype=np.float64)
    piv = np.ascontiguousarray(pivots, dtype=np.int64)
    blk = np.ascontiguousarray(blocks, dtype=np.uint8)
    rc = lib().mfr_sytrs(Fp.N, Fp.m, Bp.n, Fp.ptr(), Fp.ld, Fp.ls, _p(ds), ds.shape[1],
                         piv.ctypes.data_as(_pi64), blk.ctypes.data_as(_pu8), Bp.ptr(), Bp.ld,
                         Bp.ls, nthreads or threads())
    return Bp.array(), int(rc)


# ------------------------------------------------------------- exact -----
def exact_gemm_check(A, B, Cmat, rows, cols, nthreads=None):
    """Exact (superaccumulator) check of sampled entries of C = A*B.

    Returns (err, scale, exact): |C_hat - C| rounded, sum_k |a_ik||b_kj|
    (leading limbs) and the exact value rounded to binary64."""
    Ap, Bp, Cp = Planes(A), Planes(B), Planes(Cmat)
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    cols = np.ascontiguousarray(cols, dtype=np.int64)
    ns = len(rows)
    err, scale, exact = np.zeros(ns), np.zeros(ns), np.zeros(ns)
    lib().mfr_exact_gemm_check(Ap.N, Ap.n, Ap.ptr(), Ap.ld, Ap.ls, Bp.ptr(), Bp.ld, Bp.ls,
                               Cp.ptr(), Cp.ld, Cp.ls, ns, rows.ctypes.data_as(_pi64),
                               cols.ctypes.data_as(_pi64), _p(err), _p(scale), _p(exact),
                               nthreads or threads())
    return err, scale, exact


def exact_residual(A, X, B, nthreads=None):
    """R = B - A X exactly, rounded to binary64 (shape (n, nrhs))."""
    Ap, Xp, Bp = Planes(A), Planes(X), Planes(B)
    n, nrhs = Ap.m, Xp.n
    R = np.zeros((nrhs, n))
    lib().mfr_exact_residual(Ap.N, n, nrhs, Ap.ptr(), Ap.ld, Ap.ls, Xp.ptr(), Xp.ld, Xp.ls,
                             Bp.ptr(), Bp.ld, Bp.ls, _p(R), n, nthreads or threads())
    return R.T.copy()


def residual_mixed(A, X, B, res_limbs, uplo="general"):
    """residual.jl:431-496 restated: R = B - A X widened to res_limbs limbs"""
    Ap, Xp, Bp = Planes(A), Planes(X), Planes(B)
    Rp = Planes(np.zeros((res_limbs, Bp.m, Bp.n)))
    up = {"general": 0, "lower": 1, "upper": 2}[uplo]
    lib().mfr_residual_mixed(Ap.N, res_limbs, up, Ap.m, Ap.n, Xp.n, Ap.ptr(), Ap.ld, Ap.ls,
                             Xp.ptr(), Xp.ld, Xp.ls, Bp.ptr(), Bp.ld, Bp.ls, Rp.ptr(), Rp.ld, Rp.ls)
    return Rp.array()


def to_double(X):
    """exact limb sum of each value, rounded to binary64"""
    X = np.ascontiguousarray(X, dtype=np.float64)
    N = X.shape[0]
    cnt = X.size // N
    out = np.zeros(cnt)
    lib().mfr_to_double(N, cnt, _p(X), cnt, _p(out))
    return out.reshape(X.shape[1:])


def backward_error(A, X, B, nthreads=None):
    """normwise ||B - A X||_inf / (||A||_inf ||X||_inf + ||B||_inf) per column,
    from the exact residual (residual.jl:178-200 formula, binary64 norms)."""
    R = exact_residual(A, X, B, nthreads)
    Ad = to_double(A)
    Xd = to_double(X)
    Bd = to_double(B)
    an = np.max(np.sum(np.abs(Ad), axis=1))
    xn = np.max(np.abs(Xd), axis=0)
    bn = np.max(np.abs(Bd), axis=0)
    rn = np.max(np.abs(R), axis=0)
    return rn / (an * xn + bn)
