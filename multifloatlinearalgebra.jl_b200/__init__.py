"""B200 multi-double dense linear algebra with MultiFloatLinearAlgebra.jl's API.

Host-side mirror of the reference's public surface
(src/MultiFloatLinearAlgebra.jl:34-49) over the mflab200 C ABI.  Julia's
mutating `name!` functions are spelled `name_` here (gemm_, cholesky_, ldiv_,
...); argument meaning, defaults and failure behaviour follow the reference:

* DimensionMismatch / ArgumentError for bad shapes, options and aliasing;
* cholesky_/lu_/ldlt_ with check=True raise PosDefException /
  SingularException / DomainError, with check=False return a factor whose
  factor_status is the reference's info code (0, -1, k);
* beta == 0 never reads the destination; only the authoritative triangle is
  read or written by syrk_/gemmt_/cholesky_/ldlt_.

Matrices live on the GPU as MFMatrix: N column-major float64 limb planes in a
torch tensor (PyTorch provides device memory and the current stream only).
Every numerical operation runs in the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import threading
from typing import Optional, Sequence, Union

import numpy as np
import torch

from . import _native

__all__ = [
    "MFMatrix", "KernelConfig", "DimensionMismatch", "ArgumentError", "DomainError",
    "PosDefException", "SingularException", "MFLABError",
    "gemm_", "syrk_", "gemmt_", "trsm_", "trsv_", "gemm_plan", "OpNormInf", "gemv_", "symv_",
    "mfdot", "syrk_packed_", "trmm_", "BoundsError", "cholesky_pivoted_", "MFCholeskyPivoted",
    "factor_rdiag", "MFQR", "qr_", "rrqr_", "apply_q_", "solve_r_", "numerical_rank",
    "cholesky_", "lu_", "ldiv_", "solve", "issuccess",
    "factor_status", "factor_state", "factor_kind", "factor_matrix", "factor_precision",
    "factor_provider", "factor_pivots", "factor_diagnostics",
    "MFCholesky", "MFLU", "capabilities", "limb_type_name",
    "ldlt_", "ldlt_plan", "MFLDLT", "factor_blocks", "factor_permutation", "factor_inertia",
    "residual_", "residual_mixed_", "normwise_backward_error", "refinement_correction_",
    "solve_mixed_lu", "batched", "tuning", "create_handle", "destroy_handle",
    "PreparedInt8Operand", "gemm_prepared_",
]


# ------------------------------------------------------------- errors ----
class DimensionMismatch(ValueError):
    """Julia's DimensionMismatch."""


class ArgumentError(ValueError):
    """Julia's ArgumentError."""


class BoundsError(IndexError):
    """Julia's BoundsError (an index range outside the operand)."""


class DomainError(ValueError):
    """Julia's DomainError (non-finite factorization input with check=true)."""


class PosDefException(Exception):
    """LinearAlgebra.PosDefException(info)."""

    def __init__(self, info: int):
        super().__init__(f"matrix is not positive definite; factorization failed at {info}")
        self.info = info


class SingularException(Exception):
    """LinearAlgebra.SingularException(info)."""

    def __init__(self, info: int):
        super().__init__(f"matrix is singular; factorization failed at {info}")
        self.info = info


class MFLABError(RuntimeError):
    """A CUDA failure, timeout or resource error reported by the library."""


def _check(rc: int, what: str) -> None:
    if rc == _native.MFLAB_OK:
        return
    lib = _native.load()
    msg = f"{what}: {lib.mflab_status_string(rc).decode()}"
    detail = lib.mflab_last_error().decode()
    if detail:
        msg += f" ({detail})"
    if rc == _native.MFLAB_ERR_ARG:
        raise DimensionMismatch(msg)
    if rc == _native.MFLAB_ERR_FLAG:
        raise ArgumentError(msg)
    if rc == _native.MFLAB_ERR_ALIAS:
        raise ArgumentError(f"{what} does not support output/input aliasing")
    if rc == _native.MFLAB_ERR_UNSUPPORTED:
        raise ArgumentError(msg)
    raise MFLABError(msg)


# ------------------------------------------------------------ handles ----
_handles: dict = {}
_handles_lock = threading.Lock()


def _handle(device: int):
    key = (device, threading.get_ident())
    with _handles_lock:
        h = _handles.get(key)
        if h is None:
            lib = _native.load()
            out = C.c_void_p()
            _check(lib.mflab_create(C.byref(out), device), "mflab_create")
            h = out
            _handles[key] = h
        return h


def create_handle(device: Optional[int] = None) -> C.c_void_p:
    """A new library handle (its own scratch and staging buffers) for work
    issued on a stream of its own; the default per-thread handle serves
    everything else.  Release it with destroy_handle."""
    dev = torch.cuda.current_device() if device is None else device
    out = C.c_void_p()
    _check(_native.load().mflab_create(C.byref(out), dev), "mflab_create")
    return out


_side_handles: dict = {}


def _side_handle(device: int):
    """a second per-thread handle (its own scratch) for work that runs on a
    side stream concurrently with the default handle's"""
    key = (device, threading.get_ident())
    with _handles_lock:
        h = _side_handles.get(key)
        if h is None:
            out = C.c_void_p()
            _check(_native.load().mflab_create(C.byref(out), device), "mflab_create")
            h = out
            _side_handles[key] = h
        return h


def destroy_handle(h: C.c_void_p) -> None:
    _check(_native.load().mflab_destroy(h), "mflab_destroy")


def _stream(device: int) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def limb_type_name(N: int) -> str:
    return f"Float64x{N}"


# ------------------------------------------------------------- config ----
@dataclasses.dataclass(frozen=True)
class KernelConfig:
    """Route and block configuration (src/types.jl:13-27).  Fields without a
    GPU meaning (thread_count, reduction_tile, column_tile, packed-GEMM
    tuning) are kept for signature compatibility and ignored."""

    reduction_tile: int = 64
    column_tile: int = 16
    cholesky_block: int = 16
    lu_block: int = 16
    ldlt_block: int = 0
    ldlt_strategy: str = "auto"
    ldlt_blocked_crossover: int = 512
    thread_count: int = 1
    gemm_strategy: str = "auto"
    gemm_packed_crossover: int = 2**63 - 1
    gemm_panel_columns: int = 0
    gemm_micro_columns: int = 0
    ozaki_slices: int = 0
    ozaki_engine: str = "tcgen05"
    ozaki_scheme: str = "auto"
    ozaki_moduli: int = 0
    ozaki_block: int = 256
    solve_order: str = "matched"


_DEFAULT = KernelConfig()
_ROUTES = {"auto": 0, "direct": 1, "fused": 0, "ozaki": 2}


def gemm_plan(N: int, m: int, k: int, n: int, config: KernelConfig = _DEFAULT) -> dict:
    """Resolve the GEMM route (src/kernels/gemm.jl:44-136) for the device."""
    if not 1 <= N <= 4:
        raise ArgumentError("only 1-4 limb MultiFloats are supported")
    s = config.gemm_strategy
    if s not in ("auto", "direct", "packed", "fused", "ozaki"):
        raise ArgumentError("gemm_strategy must be :auto, :direct, :packed, :fused or :ozaki")
    if s == "fused" and N != 3:
        raise ArgumentError("gemm_strategy=:fused is only available for Float64x3")
    if s == "packed":
        s = "direct"  # packing is a CPU cache device; the device mainloop stages tiles itself
    if s == "auto":
        strategy, reason = ("fused", "auto_fused_direct") if N == 3 else ("direct", "auto_direct")
    else:
        strategy, reason = s, f"forced_{s}"
    return {"strategy": strategy, "reason": reason}


# ------------------------------------------------------------- matrix ----
class MFMatrix:
    """A Float64xN matrix (or vector) as N column-major limb planes on a GPU.

    storage: torch.float64 CUDA tensor of shape (N, ncols, ld); limb l of
    element (r, c) of this view is storage[l, c0 + c, r0 + r]."""

    __slots__ = ("storage", "r0", "c0", "m", "n", "is_vector")

    def __init__(self, storage: torch.Tensor, r0: int = 0, c0: int = 0, m: Optional[int] = None,
                 n: Optional[int] = None, is_vector: bool = False):
        if storage.dtype != torch.float64 or storage.dim() != 3:
            raise ArgumentError("MFMatrix storage must be a (N, ncols, ld) float64 tensor")
        if not storage.is_cuda:
            raise ArgumentError("MFMatrix storage must live on a CUDA device")
        if storage.shape[2] > 1 and storage.stride(2) != 1:
            raise ArgumentError("limb planes must be column-major (unit row stride)")
        self.storage = storage
        self.r0, self.c0 = r0, c0
        self.m = storage.shape[2] - r0 if m is None else m
        self.n = storage.shape[1] - c0 if n is None else n
        self.is_vector = is_vector

    # geometry
    @property
    def N(self) -> int:
        return self.storage.shape[0]

    @property
    def shape(self):
        return (self.m,) if self.is_vector else (self.m, self.n)

    @property
    def ld(self) -> int:
        st = self.storage
        # torch reports an arbitrary stride for a size-1 dimension
        return st.stride(1) if st.shape[1] > 1 else max(st.shape[2], 1)

    @property
    def ls(self) -> int:
        st = self.storage
        return st.stride(0) if st.shape[0] > 1 else st.shape[1] * max(st.shape[2], 1)

    @property
    def device(self) -> int:
        return self.storage.device.index

    def ptr(self) -> int:
        return self.storage.data_ptr() + 8 * (self.c0 * self.ld + self.r0)

    def __len__(self):
        return self.m

    def __repr__(self):
        kind = "vector" if self.is_vector else "matrix"
        return f"MFMatrix({limb_type_name(self.N)} {kind} {self.shape} on cuda:{self.device})"

    # construction
    @classmethod
    def empty(cls, N: int, m: int, n: Optional[int] = None, device=None) -> "MFMatrix":
        vec = n is None
        n = 1 if vec else n
        if isinstance(device, torch.device):
            device = device.index
        dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        st = torch.empty((N, max(n, 0), max(m, 1)), dtype=torch.float64, device=dev)
        return cls(st, 0, 0, m, n, vec)

    @classmethod
    def zeros(cls, N: int, m: int, n: Optional[int] = None, device=None) -> "MFMatrix":
        x = cls.empty(N, m, n, device)
        x.storage.zero_()
        return x

    @classmethod
    def from_numpy(cls, X: np.ndarray, device=None) -> "MFMatrix":
        """X shaped (N, m, n) (matrix) or (N, m) (vector), limb-major."""
        X = np.asarray(X, dtype=np.float64)
        vec = X.ndim == 2
        if vec:
            X = X[:, :, None]
        if X.ndim != 3:
            raise ArgumentError("expected an (N, m, n) or (N, m) limb array")
        if isinstance(device, torch.device):
            device = device.index
        dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        st = torch.from_numpy(np.ascontiguousarray(X.transpose(0, 2, 1))).to(dev)
        if st.shape[2] == 0:
            st = torch.zeros((X.shape[0], X.shape[2], 1), dtype=torch.float64, device=dev)
        return cls(st, 0, 0, X.shape[1], X.shape[2], vec)

    @classmethod
    def from_tensor(cls, planes: torch.Tensor, is_vector: bool = False) -> "MFMatrix":
        """planes shaped (N, n, m): used as storage without a copy."""
        return cls(planes, 0, 0, planes.shape[2], planes.shape[1], is_vector)

    # Interleaved storage is the memory order of a Julia
    # Matrix{MultiFloat{Float64,N}} (the reference's operand type,
    # gemm.jl:747-755): limb l of element (r, c) at X[(c*ld + r)*N + l],
    # i.e. a C-contiguous host array of shape (n, ld, N).
    @staticmethod
    def _host_ptr(X) -> tuple:
        """(address, shape, pinned) of a C-contiguous float64 host array"""
        if isinstance(X, torch.Tensor):
            if X.is_cuda or X.dtype != torch.float64 or not X.is_contiguous():
                raise ArgumentError("interleaved host data must be a contiguous float64 CPU tensor")
            return X.data_ptr(), tuple(X.shape), X.is_pinned()
        if not isinstance(X, np.ndarray) or X.dtype != np.float64 or \
                not X.flags["C_CONTIGUOUS"]:
            raise ArgumentError("interleaved host data must be a C-contiguous float64 array")
        return X.ctypes.data, X.shape, False

    def copy_from_interleaved_(self, X, stream=None, handle=None) -> "MFMatrix":
        """Upload interleaved host data of shape (n, ld, N) (ld >= m) into
        this matrix (mflab_h2d_interleaved).  Stream-ordered and not
        synchronised: a pinned X must stay alive until `stream` (default:
        the current stream) has passed this point.  `handle` (a raw
        mflab_handle) lets concurrent streams use their own staging."""
        ptr, shape, _ = self._host_ptr(X)
        if len(shape) != 3 or shape[0] != self.n or shape[1] < self.m or shape[2] != self.N:
            raise DimensionMismatch(f"interleaved data of shape {shape} does not hold a "
                                    f"{self.m}x{self.n} {limb_type_name(self.N)} matrix")
        lib = _native.load()
        h = handle or _handle(self.device)
        s = _stream(self.device) if stream is None else stream.cuda_stream
        _check(lib.mflab_h2d_interleaved(h, s, self.N, self.m, self.n, ptr, shape[1], self.ptr(),
                                         self.ld, self.ls), "h2d_interleaved")
        return self

    def copy_to_interleaved_(self, X, stream=None, handle=None):
        """Download this matrix into interleaved host data of shape (n, ld, N)
        (mflab_d2h_interleaved); not synchronised."""
        ptr, shape, _ = self._host_ptr(X)
        if len(shape) != 3 or shape[0] != self.n or shape[1] < self.m or shape[2] != self.N:
            raise DimensionMismatch(f"interleaved data of shape {shape} cannot take a "
                                    f"{self.m}x{self.n} {limb_type_name(self.N)} matrix")
        lib = _native.load()
        h = handle or _handle(self.device)
        s = _stream(self.device) if stream is None else stream.cuda_stream
        _check(lib.mflab_d2h_interleaved(h, s, self.N, self.m, self.n, self.ptr(), self.ld,
                                         self.ls, ptr, shape[1]), "d2h_interleaved")
        return X

    @classmethod
    def from_interleaved(cls, X, m: Optional[int] = None, device=None) -> "MFMatrix":
        """A new device matrix from interleaved host data (n, ld, N): the
        first m (default ld) rows of each column.  Returns after the copy."""
        _, shape, _ = cls._host_ptr(X)
        if len(shape) != 3 or not 1 <= shape[2] <= 4:
            raise ArgumentError("interleaved data must have shape (n, ld, N), N in 1..4")
        n, ld, N = shape
        M = cls.empty(N, ld if m is None else m, n, device)
        M.copy_from_interleaved_(X)
        torch.cuda.current_stream(M.device).synchronize()
        return M

    def to_interleaved(self) -> np.ndarray:
        """This matrix as an interleaved host array of shape (n, m, N)."""
        out = np.empty((self.n, self.m, self.N), dtype=np.float64)
        if out.size:
            self.copy_to_interleaved_(out)
            torch.cuda.current_stream(self.device).synchronize()
        return out

    def planes(self) -> torch.Tensor:
        """(N, n, m) torch view of this matrix's elements."""
        return self.storage[:, self.c0:self.c0 + self.n, self.r0:self.r0 + self.m]

    def to_numpy(self) -> np.ndarray:
        a = self.planes().cpu().numpy().transpose(0, 2, 1)
        return np.ascontiguousarray(a[:, :, 0] if self.is_vector else a)

    def copy(self) -> "MFMatrix":
        st = self.planes().contiguous().clone()
        if st.shape[2] == 0:
            st = torch.zeros((self.N, self.n, 1), dtype=torch.float64, device=self.storage.device)
        return MFMatrix(st, 0, 0, self.m, self.n, self.is_vector)

    def copy_(self, other: "MFMatrix") -> "MFMatrix":
        if (other.N, other.m, other.n) != (self.N, self.m, self.n):
            raise DimensionMismatch("copy source and destination dimensions differ")
        self.planes().copy_(other.planes())
        return self

    def view(self, rows: slice, cols: slice = slice(None)) -> "MFMatrix":
        r = range(self.m)[rows]
        c = range(self.n)[cols]
        if r.step != 1 or c.step != 1:
            raise ArgumentError("only unit-stride views are supported")
        return MFMatrix(self.storage, self.r0 + r.start, self.c0 + c.start, len(r), len(c), False)


# ------------------------------------------------------------ helpers ----
def _scalar(N: int, v) -> "C.Array":
    arr = (C.c_double * 4)()
    if isinstance(v, (int, float)):
        arr[0] = float(v)
    else:
        vals = np.asarray(v, dtype=np.float64).ravel()
        if len(vals) > N:
            raise ArgumentError("scalar has more limbs than the matrix type")
        for i, x in enumerate(vals):
            arr[i] = float(x)
    return arr


def _same_type(*mats: MFMatrix) -> int:
    N = mats[0].N
    for x in mats:
        if not isinstance(x, MFMatrix):
            raise ArgumentError("expected MFMatrix operands")
        if x.N != N:
            raise ArgumentError("operands have different limb counts")
        if x.device != mats[0].device:
            raise ArgumentError("operands live on different devices")
    if not 1 <= N <= 4:
        raise ArgumentError("only 1-4 limb MultiFloats are supported")
    if N == 1:
        raise ArgumentError("Float64x1 is plain Float64; use a Float64 BLAS")
    return N


def _mightalias(a: MFMatrix, b: MFMatrix) -> bool:
    """2-D index-range overlap of two views (Base.mightalias on views)."""
    if a.storage.data_ptr() != b.storage.data_ptr():
        sa, ea = a.storage.data_ptr(), a.storage.data_ptr() + 8 * a.storage.numel()
        sb, eb = b.storage.data_ptr(), b.storage.data_ptr() + 8 * b.storage.numel()
        return sa < eb and sb < ea
    rows = a.r0 < b.r0 + b.m and b.r0 < a.r0 + a.m
    cols = a.c0 < b.c0 + b.n and b.c0 < a.c0 + a.n
    return rows and cols and a.m > 0 and b.m > 0 and a.n > 0 and b.n > 0


def _no_alias(op: str, dest: MFMatrix, src: MFMatrix) -> None:
    if _mightalias(dest, src):
        raise ArgumentError(f"{op} does not support output/input aliasing")


def _lib_h(x: MFMatrix):
    return _native.load(), _handle(x.device), _stream(x.device)


_ORDERS = {"matched": 0, "fast": 1}


class _solve_order:
    """sets the handle's triangular-solve order for the duration of a call"""

    def __init__(self, x: MFMatrix, config: "KernelConfig"):
        if config.solve_order not in _ORDERS:
            raise ArgumentError("solve_order must be :matched or :fast")
        self.h = _handle(x.device)
        self.order = _ORDERS[config.solve_order]

    def __enter__(self):
        _native.load().mflab_set_solve_order(self.h, self.order)

    def __exit__(self, *exc):
        _native.load().mflab_set_solve_order(self.h, 0)


# --------------------------------------------------------------- BLAS ----
def gemm_(C_: MFMatrix, A: MFMatrix, B: MFMatrix, alpha=1.0, beta=0.0,
          config: KernelConfig = _DEFAULT, workspace=None) -> MFMatrix:
    """C = alpha*A*B + beta*C (src/kernels/gemm.jl:747-774)."""
    N = _same_type(C_, A, B)
    m, k = A.m, A.n
    if B.m != k:
        raise DimensionMismatch("gemm! inner dimensions differ")
    n = B.n
    if (C_.m, C_.n) != (m, n):
        raise DimensionMismatch("gemm! output dimensions differ")
    _no_alias("gemm!", C_, A)
    _no_alias("gemm!", C_, B)
    plan = gemm_plan(N, m, k, n, config)
    route = _ROUTES[plan["strategy"]]
    lib, h, s = _lib_h(C_)
    if route == 2:
        rc = _gemm_ozaki(lib, h, s, N, C_, A, B, alpha, beta, config)
    else:
        rc = lib.mflab_gemm(h, s, N, route, m, n, k, A.ptr(), A.ld, A.ls, B.ptr(), B.ld, B.ls,
                            C_.ptr(), C_.ld, C_.ls, _scalar(N, alpha), _scalar(N, beta))
    _check(rc, "gemm!")
    return C_


def ozaki_scheme(config: KernelConfig = _DEFAULT) -> str:
    """The INT8 scheme a gemm_strategy=:ozaki call runs first: :slices when
    ozaki_slices is set, :modular when ozaki_moduli is set, else
    ozaki_scheme (:auto = :modular, with :slices when the modulus table
    cannot reach the tuned requirement)."""
    sch = config.ozaki_scheme
    if sch not in ("auto", "slices", "modular"):
        raise ArgumentError("ozaki_scheme must be :auto, :slices or :modular")
    if sch == "auto":
        if config.ozaki_slices > 0:
            return "slices"
        return "modular"
    return sch


# int8 engines: the library's own tcgen05 kernels (one CTA per SM, or CTA
# pairs with cta_group::2) and cuBLASLt; :tcgen05 is the default kernel
_TC_DEFAULT = 0
_ENGINES = {"tcgen05": _TC_DEFAULT, "tcgen05_1sm": 0, "tcgen05_pair": 2, "library": 1}


def _int8_engine(config: KernelConfig) -> int:
    engines = _ENGINES
    if config.ozaki_engine not in engines:
        raise ArgumentError("ozaki_engine must be :tcgen05, :tcgen05_1sm, :tcgen05_pair or "
                            ":library")
    if config.ozaki_slices < 0 or config.ozaki_moduli < 0:
        raise ArgumentError("ozaki_slices and ozaki_moduli must be >= 0")
    return engines[config.ozaki_engine]


def _gemm_ozaki(lib, h, s, N, C_, A, B, alpha, beta, config):
    _check(lib.mflab_set_int8_engine(h, _int8_engine(config)), "gemm!")
    m, k, n = A.m, A.n, B.n
    args = (m, n, k, A.ptr(), A.ld, A.ls, B.ptr(), B.ld, B.ls, C_.ptr(), C_.ld, C_.ls,
            _scalar(N, alpha), _scalar(N, beta))
    scheme = ozaki_scheme(config)
    if scheme == "modular":
        rc = lib.mflab_gemm_ozaki_crt(h, s, N, int(config.ozaki_moduli), *args)
        if rc != _native.MFLAB_ERR_UNSUPPORTED or config.ozaki_scheme == "modular" \
                or config.ozaki_moduli > 0:
            return rc
    return lib.mflab_gemm_ozaki(h, s, N, int(config.ozaki_slices), *args)


def ozaki_crt_plan(N: int, k: int, moduli: int = 0, gap_bits: float = 0.0) -> dict:
    """Digit count Q, digit width h and modulus count T of the modular INT8
    route for depth k: for `moduli` > 0 that count, else the tuner's choice
    for a sampled scale gap of `gap_bits` (host-only, no device work)."""
    Q, hh, T = C.c_int(), C.c_int(), C.c_int()
    rc = _native.load().mflab_ozaki_crt_plan(N, k, moduli, int(round(8 * gap_bits)),
                                             C.byref(Q), C.byref(hh), C.byref(T))
    _check(rc, "ozaki_crt_plan")
    return {"digits": Q.value, "digit_bits": hh.value, "moduli": T.value}


def ozaki_crt_moduli() -> list:
    """The modulus table of the modular INT8 route."""
    lib = _native.load()
    return [int(lib.mflab_ozaki_crt_modulus(t)) for t in range(lib.mflab_ozaki_crt_modulus(-1))]


def ozaki_crt_tune_moduli(A: MFMatrix, B: MFMatrix) -> int:
    """The modulus count gemm_(C, A, B) on the modular INT8 route would pick
    with ozaki_moduli = 0 (the sampled scale gap; one stream
    synchronisation), without forming the product.  A product at that fixed
    count takes digits as wide as the count allows, at least as wide as the
    tuned call's, so its error is at most the tuned call's."""
    N = _same_type(A, B)
    if A.n != B.m:
        raise DimensionMismatch("gemm! inner dimensions differ")
    lib, h, s = _lib_h(A)
    T = C.c_int()
    _check(lib.mflab_ozaki_crt_tune(h, s, N, A.m, B.n, A.n, A.ptr(), A.ld, A.ls, B.ptr(), B.ld,
                                    B.ls, C.byref(T)), "ozaki tune")
    return int(T.value)


def ozaki_last_moduli(device: Optional[int] = None) -> int:
    """Modulus count chosen by the last modular INT8 GEMM issued from this thread."""
    dev = torch.cuda.current_device() if device is None else device
    return int(_native.load().mflab_ozaki_last_moduli(_handle(dev)))


class PreparedInt8Operand:
    """A Float64xN matrix prepared once as the left operand of many modular
    INT8 products with a fixed modulus count (mflab_ozaki_crt_prepare): its
    row scales and residue planes live in a device buffer of this object.
    gemm_prepared_(C, P, B) equals gemm_(C, A, B) with ozaki_moduli =
    P.moduli, bit for bit, without reading or splitting A again."""

    def __init__(self, A: MFMatrix, moduli: int):
        N = _same_type(A)
        if A.n < 1:
            raise DimensionMismatch("a prepared operand needs at least one column")
        nbytes = C.c_size_t()
        lib, h, s = _lib_h(A)
        _check(lib.mflab_ozaki_crt_prepare_bytes(N, int(moduli), A.m, A.n, C.byref(nbytes)),
               "ozaki prepare")
        self.N, self.m, self.k, self.moduli = N, A.m, A.n, int(moduli)
        self.device = A.device
        self.buffer = torch.empty(max(nbytes.value, 1), dtype=torch.uint8,
                                  device=A.storage.device)
        _check(lib.mflab_ozaki_crt_prepare(h, s, N, self.moduli, A.m, A.n, A.ptr(), A.ld, A.ls,
                                           self.buffer.data_ptr()), "ozaki prepare")


def gemm_prepared_(C_: MFMatrix, P: PreparedInt8Operand, B: MFMatrix, alpha=1.0, beta=0.0,
                   config: KernelConfig = _DEFAULT) -> MFMatrix:
    """C = alpha*A*B + beta*C with A prepared (PreparedInt8Operand) on the
    modular INT8 route."""
    N = _same_type(C_, B)
    if N != P.N or C_.device != P.device:
        raise ArgumentError("prepared operand of another type or device")
    if B.m != P.k:
        raise DimensionMismatch("gemm! inner dimensions differ")
    if (C_.m, C_.n) != (P.m, B.n):
        raise DimensionMismatch("gemm! output dimensions differ")
    _no_alias("gemm!", C_, B)
    lib, h, s = _lib_h(C_)
    _check(lib.mflab_set_int8_engine(h, _int8_engine(config)), "gemm!")
    _check(lib.mflab_gemm_ozaki_crt_prepared(h, s, N, P.moduli, P.m, B.n, P.k,
                                             P.buffer.data_ptr(), B.ptr(), B.ld, B.ls, C_.ptr(),
                                             C_.ld, C_.ls, _scalar(N, alpha), _scalar(N, beta)),
           "gemm!")
    return C_


def ozaki_default_slices(N: int, k: int) -> int:
    """Digit slices per operand of the INT8 route when KernelConfig.ozaki_slices == 0."""
    return int(_native.load().mflab_ozaki_default_slices(N, k))


def ozaki_last_slices(device: Optional[int] = None) -> int:
    """Slice count chosen by the last INT8-slice GEMM issued from this thread."""
    dev = torch.cuda.current_device() if device is None else device
    return int(_native.load().mflab_ozaki_last_slices(_handle(dev)))


def device_status(device: Optional[int] = None) -> int:
    """0, or the status code a tcgen05 kernel of this thread's handle left
    after a bounded wait ran out (1 producer, 2 MMA issuer, 3 epilogue, 4
    drain); reading resets it (synchronises)"""
    dev = torch.cuda.current_device() if device is None else device
    v = C.c_int()
    _check(_native.load().mflab_device_status(_handle(dev), C.byref(v)), "device_status")
    return int(v.value)


def ozaki_available() -> bool:
    return hasattr(_native.load(), "mflab_gemm_ozaki")


def _vec_len(v: MFMatrix, what: str) -> int:
    if v.n != 1:
        raise DimensionMismatch(f"{what} must be a vector")
    return v.m


def gemv_(y: MFMatrix, A: MFMatrix, x: MFMatrix, alpha=1.0, beta=0.0, trans: str = "N",
          config: KernelConfig = _DEFAULT) -> MFMatrix:
    """y = alpha*op(A)*x + beta*y (src/kernels/gemv.jl:99-167)."""
    if trans not in ("N", "T"):
        raise ArgumentError("trans must be :N or :T")
    N = _same_type(y, A, x)
    m, n = A.m, A.n
    lx, ly = _vec_len(x, "gemv! input"), _vec_len(y, "gemv! output")
    if lx != (n if trans == "N" else m):
        raise DimensionMismatch("gemv! input length differs")
    if ly != (m if trans == "N" else n):
        raise DimensionMismatch("gemv! output length differs")
    _no_alias("gemv!", y, A)
    _no_alias("gemv!", y, x)
    lib, h, s = _lib_h(y)
    _check(lib.mflab_gemv(h, s, N, 0 if trans == "N" else 1, m, n, A.ptr(), A.ld, A.ls, x.ptr(),
                          x.ls, y.ptr(), y.ls, _scalar(N, alpha), _scalar(N, beta)), "gemv!")
    return y


def symv_(y: MFMatrix, A: MFMatrix, x: MFMatrix, alpha=1.0, beta=0.0, uplo: str = "lower",
          config: KernelConfig = _DEFAULT) -> MFMatrix:
    """y = alpha*A*x + beta*y, A symmetric from its uplo triangle
    (src/kernels/symv.jl:43-89)."""
    if uplo not in ("lower", "upper"):
        raise ArgumentError("uplo must be :lower or :upper")
    N = _same_type(y, A, x)
    n = A.m
    if A.n != n:
        raise DimensionMismatch("symv! requires a square matrix")
    if _vec_len(x, "symv! input") != n:
        raise DimensionMismatch("symv! input length differs")
    if _vec_len(y, "symv! output") != n:
        raise DimensionMismatch("symv! output length differs")
    _no_alias("symv!", y, A)
    _no_alias("symv!", y, x)
    lib, h, s = _lib_h(y)
    _check(lib.mflab_symv(h, s, N, 0 if uplo == "lower" else 1, n, A.ptr(), A.ld, A.ls, x.ptr(),
                          x.ls, y.ptr(), y.ls, _scalar(N, alpha), _scalar(N, beta)), "symv!")
    return y


def mfdot(x: MFMatrix, y: MFMatrix) -> np.ndarray:
    """Inner product over the column-major index, one ascending chain
    (src/kernels/dot.jl:1-22); returns the N limbs."""
    N = _same_type(x, y)
    if (x.m, x.n) != (y.m, y.n):
        raise DimensionMismatch("dot product shapes differ")
    out = torch.zeros(N, dtype=torch.float64, device=x.storage.device)
    lib, h, s = _lib_h(x)
    _check(lib.mflab_dot(h, s, N, x.m, x.n, x.ptr(), x.ld, x.ls, y.ptr(), y.ld, y.ls,
                         out.data_ptr()), "mfdot")
    return out.cpu().numpy()


def syrk_packed_(packed: MFMatrix, panel: MFMatrix, alpha=1.0, beta=0.0, reduction_first: int = 1,
                 reduction_last: Optional[int] = None,
                 config: KernelConfig = _DEFAULT) -> MFMatrix:
    """Packed lower triangle (column-major packed, (1,1),(2,1)..(n,1),(2,2)..)
    = alpha * panel[rf:rl, :]^T panel[rf:rl, :] + beta * packed, with the
    inclusive 1-based reduction bounds of src/kernels/syrk.jl:173-254."""
    N = _same_type(packed, panel)
    n, kp = panel.n, panel.m
    if reduction_last is None:
        reduction_last = kp
    if packed.n != 1 or packed.m != n * (n + 1) // 2:
        raise DimensionMismatch("syrk_packed! output length differs")
    if not 1 <= reduction_first <= reduction_last <= kp:
        raise BoundsError(f"reduction range {reduction_first}:{reduction_last} outside 1:{kp}")
    _no_alias("syrk_packed!", packed, panel)
    lib, h, s = _lib_h(packed)
    _check(lib.mflab_syrk_packed(h, s, N, n, kp, reduction_first - 1, reduction_last, panel.ptr(),
                                 panel.ld, panel.ls, packed.ptr(), packed.ls, _scalar(N, alpha),
                                 _scalar(N, beta)), "syrk_packed!")
    return packed


def syrk_(C_: MFMatrix, P: MFMatrix, alpha=1.0, beta=0.0, uplo: str = "lower",
          config: KernelConfig = _DEFAULT) -> MFMatrix:
    """lower(C) = alpha*P^T*P + beta*C (src/kernels/syrk.jl:67-108)."""
    if uplo not in ("lower", "L"):
        raise ArgumentError("syrk! currently supports only uplo=:lower or :L")
    N = _same_type(C_, P)
    n, k = P.n, P.m
    if (C_.m, C_.n) != (n, n):
        raise DimensionMismatch("syrk! output dimensions differ")
    _no_alias("syrk!", C_, P)
    lib, h, s = _lib_h(C_)
    if config.gemm_strategy == "ozaki":
        _check(lib.mflab_set_int8_engine(h, _int8_engine(config)), "syrk!")
        if ozaki_scheme(config) != "modular":
            raise ArgumentError("the INT8 syrk! route uses the modular scheme (ozaki_moduli)")
        rc = lib.mflab_syrk_lower_ozaki(h, s, N, int(config.ozaki_moduli), 1, n, k, P.ptr(), P.ld,
                                        P.ls, C_.ptr(), C_.ld, C_.ls, _scalar(N, alpha),
                                        _scalar(N, beta))
    else:
        rc = lib.mflab_syrk_lower(h, s, N, n, k, P.ptr(), P.ld, P.ls, C_.ptr(), C_.ld, C_.ls,
                                  _scalar(N, alpha), _scalar(N, beta))
    _check(rc, "syrk!")
    return C_


def gemmt_(C_: MFMatrix, A: MFMatrix, B: MFMatrix, alpha=1.0, beta=0.0,
           config: KernelConfig = _DEFAULT) -> MFMatrix:
    """lower(C) = alpha*A*B^T + beta*C (src/kernels/gemmt.jl:69-108)."""
    N = _same_type(C_, A, B)
    rows, k = A.m, A.n
    if (B.m, B.n) != (rows, k):
        raise DimensionMismatch("gemmt! input dimensions differ")
    if (C_.m, C_.n) != (rows, rows):
        raise DimensionMismatch("gemmt! output dimensions differ")
    _no_alias("gemmt!", C_, A)
    _no_alias("gemmt!", C_, B)
    lib, h, s = _lib_h(C_)
    rc = lib.mflab_gemmt_lower(h, s, N, rows, k, A.ptr(), A.ld, A.ls, B.ptr(), B.ld, B.ls,
                               C_.ptr(), C_.ld, C_.ls, _scalar(N, alpha), _scalar(N, beta))
    _check(rc, "gemmt!")
    return C_


_SIDE = {"left": 0, "right": 1}
_UPLO = {"lower": 0, "upper": 1}
_TRANS = {"N": 0, "T": 1}
_DIAG = {"nonunit": 0, "unit": 1}


def trsm_(B: MFMatrix, A: MFMatrix, alpha=1.0, side: str = "left", uplo: str = "lower",
          trans: str = "N", diag: str = "nonunit", config: KernelConfig = _DEFAULT) -> MFMatrix:
    """op(A) X = alpha B or X op(A) = alpha B in place (src/kernels/trsm.jl:224-302)."""
    N = _same_type(B, A)
    if A.m != A.n:
        raise DimensionMismatch("trsm! requires a square triangular matrix")
    if side not in _SIDE:
        raise ArgumentError("side must be :left or :right")
    if uplo not in _UPLO:
        raise ArgumentError("uplo must be :lower or :upper")
    if trans not in _TRANS:
        raise ArgumentError("trans must be :N or :T")
    if diag not in _DIAG:
        raise ArgumentError("diag must be :unit or :nonunit")
    if side == "left" and B.m != A.m:
        raise DimensionMismatch("trsm! left dimensions differ")
    if side == "right" and B.n != A.m:
        raise DimensionMismatch("trsm! right dimensions differ")
    _no_alias("trsm!", B, A)
    lib, h, s = _lib_h(B)
    with _solve_order(B, config):
        rc = lib.mflab_trsm(h, s, N, _SIDE[side], _UPLO[uplo], _TRANS[trans], _DIAG[diag], B.m,
                            B.n, A.ptr(), A.ld, A.ls, B.ptr(), B.ld, B.ls, _scalar(N, alpha))
    _check(rc, "trsm!")
    return B


def trmm_(B: MFMatrix, A: MFMatrix, alpha=1.0, side: str = "left", uplo: str = "lower",
          trans: str = "N", diag: str = "nonunit", config: KernelConfig = _DEFAULT) -> MFMatrix:
    """B = alpha op(A) B or alpha B op(A) in place, reading only the uplo
    triangle of A (src/kernels/trmm.jl:82-131)."""
    N = _same_type(B, A)
    if A.m != A.n:
        raise DimensionMismatch("trmm! requires a square triangular matrix")
    if side not in _SIDE:
        raise ArgumentError("side must be :left or :right")
    if uplo not in _UPLO:
        raise ArgumentError("uplo must be :lower or :upper")
    if trans not in _TRANS:
        raise ArgumentError("trans must be :N or :T")
    if diag not in _DIAG:
        raise ArgumentError("diag must be :unit or :nonunit")
    if side == "left" and B.m != A.m:
        raise DimensionMismatch("trmm! left dimensions differ")
    if side == "right" and B.n != A.m:
        raise DimensionMismatch("trmm! right dimensions differ")
    _no_alias("trmm!", B, A)
    lib, h, s = _lib_h(B)
    _check(lib.mflab_trmm(h, s, N, _SIDE[side], _UPLO[uplo], _TRANS[trans], _DIAG[diag], B.m, B.n,
                          A.ptr(), A.ld, A.ls, B.ptr(), B.ld, B.ls, _scalar(N, alpha)), "trmm!")
    return B


def trsv_(x: MFMatrix, A: MFMatrix, alpha=1.0, uplo: str = "lower", trans: str = "N",
          diag: str = "nonunit", config: KernelConfig = _DEFAULT) -> MFMatrix:
    """op(A) x = alpha b in place (src/kernels/trsv.jl:19-73)."""
    if A.m != A.n:
        raise DimensionMismatch("trsv! requires a square triangular matrix")
    if x.m != A.m or x.n != 1:
        raise DimensionMismatch("trsv! right-hand side length differs")
    return trsm_(x, A, alpha, "left", uplo, trans, diag, config)


# ------------------------------------------------------- factorizations ----
class _Factor:
    kind = "abstract"

    def __init__(self, factors: MFMatrix, info: int):
        self.factors = factors
        self.info = int(info)

    @property
    def N(self) -> int:
        return self.factors.N

    def __repr__(self):
        return (f"MF{self.kind.upper()}({limb_type_name(self.N)}, {self.factors.m}x"
                f"{self.factors.n}, status={self.info})")


class MFCholesky(_Factor):
    """Lower Cholesky factor (src/factorizations/cholesky.jl:1-8)."""
    kind = "cholesky"


class MFCholeskyPivoted(_Factor):
    """Rank-revealing pivoted Cholesky: the lower triangle of factors holds L,
    A[p, p] ~ L[:, :rank] L[:, :rank]^T (src/factorizations/cholesky_pivoted.jl:1-22)."""
    kind = "cholesky_pivoted"

    def __init__(self, factors: MFMatrix, permutation: torch.Tensor, rank: int, info: int):
        super().__init__(factors, info)
        self.permutation = permutation
        self.rank = int(rank)


class MFQR(_Factor):
    """Compact Householder QR: reflectors below the diagonal of factors, R on
    and above it, A[:, permutation] = Q R (src/factorizations/qr.jl:1-16)."""
    kind = "qr"

    def __init__(self, factors: MFMatrix, tau: torch.Tensor, permutation: torch.Tensor,
                 info: int):
        super().__init__(factors, info)
        self.tau = tau
        self.permutation = permutation


class MFLU(_Factor):
    """Partial-pivoting LU factor (src/factorizations/lu.jl:1-14)."""
    kind = "lu"

    def __init__(self, factors, ipiv: torch.Tensor, info, original_maximum: torch.Tensor):
        super().__init__(factors, info)
        self.ipiv = ipiv
        self.original_maximum = original_maximum


class MFLDLT(_Factor):
    """Bunch-Kaufman LDL^T factor (src/factorizations/ldlt.jl:1-63)."""
    kind = "ldlt"

    def __init__(self, factors, dsub: torch.Tensor, pivots: torch.Tensor, blocks: torch.Tensor,
                 info, original_maximum: torch.Tensor):
        super().__init__(factors, info)
        self.dsub = dsub          # (N, n) float64 limb planes
        self.pivots = pivots      # int64, 1-based
        self.blocks = blocks      # uint8: 1 / 2 block start, 0 continuation
        self.original_maximum = original_maximum


def _read_info(dev_info: torch.Tensor) -> int:
    return int(dev_info.item())


def _finite_region(A: MFMatrix, region: int) -> bool:
    out = torch.empty(A.N + 1, dtype=torch.float64, device=A.storage.device)
    lib, h, s = _lib_h(A)
    _check(lib.mflab_max_abs(h, s, A.N, A.m, A.n, A.ptr(), A.ld, A.ls, region, out.data_ptr()),
           "max_abs")
    return bool(out[A.N].item() == 1.0)


def cholesky_(A: MFMatrix, check: bool = True, config: KernelConfig = _DEFAULT) -> MFCholesky:
    """Blocked lower Cholesky in place (src/factorizations/cholesky.jl:68-107)."""
    N = _same_type(A)
    if A.m != A.n:
        raise DimensionMismatch("cholesky! requires a square matrix")
    info = torch.zeros(1, dtype=torch.int32, device=A.storage.device)
    block = max(config.cholesky_block, 1)
    lib, h, s = _lib_h(A)
    if config.gemm_strategy == "ozaki":
        # INT8 trailing updates between panels of ozaki_block columns
        if ozaki_scheme(config) != "modular":
            raise ArgumentError("the INT8 trailing update uses the modular scheme (ozaki_moduli)")
        _check(lib.mflab_set_int8_engine(h, _int8_engine(config)), "cholesky!")
        _check(lib.mflab_potrf_ozaki(h, s, N, int(config.ozaki_moduli), A.m, A.ptr(), A.ld, A.ls,
                                     max(int(config.ozaki_block), block), block,
                                     info.data_ptr()), "cholesky!")
    else:
        _check(lib.mflab_potrf(h, s, N, A.m, A.ptr(), A.ld, A.ls, block, info.data_ptr()),
               "cholesky!")
    st = _read_info(info)
    if st == -1 and check:
        raise DomainError("cholesky!: input matrix contains non-finite entries")
    if st > 0 and check:
        raise PosDefException(st)
    return MFCholesky(A, st)


def cholesky_pivoted_(A: MFMatrix, tol=0.0, check: bool = True,
                      config: KernelConfig = _DEFAULT) -> MFCholeskyPivoted:
    """Rank-revealing pivoted Cholesky in place; tol is the relative pivot
    threshold, a tolerance stop is reported by rank, not by the status
    (src/factorizations/cholesky_pivoted.jl:65-175)."""
    N = _same_type(A)
    n = A.m
    if A.n != n:
        raise DimensionMismatch("cholesky_pivoted! requires a square matrix")
    t = np.zeros(N)
    tv = np.atleast_1d(np.asarray(tol, dtype=np.float64)).ravel()
    if len(tv) > N:
        raise ArgumentError("tol has more limbs than the matrix type")
    t[:len(tv)] = tv
    if not np.all(np.isfinite(t)) or t[0] < 0 or (t[0] == 0 and np.any(t[1:] < 0)):
        raise ArgumentError("tol must be finite and nonnegative")
    dev = A.storage.device
    perm = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    rank_info = torch.zeros(2, dtype=torch.int64, device=dev)
    lib, h, s = _lib_h(A)
    _check(lib.mflab_pstrf(h, s, N, n, A.ptr(), A.ld, A.ls, _scalar(N, t), perm.data_ptr(),
                           rank_info.data_ptr()), "cholesky_pivoted!")
    rank, info = (int(v) for v in rank_info.cpu().tolist())
    if info == -1 and check:
        raise DomainError("cholesky_pivoted!: input matrix contains non-finite entries")
    if info > 0 and check:
        raise PosDefException(info)
    return MFCholeskyPivoted(A, perm[:n], rank, info)


def _qr_run(A: MFMatrix, pivoted: int, check: bool, what: str) -> MFQR:
    N = _same_type(A)
    m, n = A.m, A.n
    r = min(m, n)
    dev = A.storage.device
    tau = torch.zeros((N, max(r, 1)), dtype=torch.float64, device=dev)
    perm = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    lib, h, s = _lib_h(A)
    _check(lib.mflab_qr(h, s, N, pivoted, m, n, A.ptr(), A.ld, A.ls, tau.data_ptr(), tau.stride(0),
                        perm.data_ptr(), info.data_ptr()), what)
    st = _read_info(info)
    if st == -1 and check:
        raise DomainError(f"{what}: input matrix contains non-finite entries")
    return MFQR(A, tau[:, :r], perm[:n], st)


def rrqr_(A: MFMatrix, check: bool = True, config: KernelConfig = _DEFAULT) -> MFQR:
    """Deterministic column-pivoted Householder QR in place
    (src/factorizations/qr.jl:692-761)."""
    return _qr_run(A, 1, check, "rrqr!")


def qr_(A: MFMatrix, permutation=None, check: bool = True,
        config: KernelConfig = _DEFAULT) -> MFQR:
    """Unpivoted Householder QR in place (src/factorizations/qr.jl:763-811);
    with a permutation the columns are first reordered physically and the
    factor records the caller's order (qr.jl:813-861)."""
    if permutation is None:
        return _qr_run(A, 0, check, "qr!")
    p = np.asarray(permutation).astype(np.int64).ravel()
    n = A.n
    if len(p) != n:
        raise DimensionMismatch(f"permutation length {len(p)} does not match {n} columns")
    seen = np.zeros(n, dtype=bool)
    for c in p:
        if not 1 <= c <= n:
            raise ArgumentError(f"permutation entry {c} is outside 1:{n}")
        if seen[c - 1]:
            raise ArgumentError(f"permutation repeats column {c}")
        seen[c - 1] = True
    view = A.storage[:, A.c0:A.c0 + n, A.r0:A.r0 + A.m]
    idx = torch.as_tensor(p - 1, device=A.storage.device)
    view.copy_(view.index_select(1, idx))
    F = _qr_run(A, 0, check, "qr!")
    F.permutation = torch.as_tensor(p, device=A.storage.device)
    return F


def _qr_ok(F: MFQR, what: str) -> None:
    if not issuccess(F):
        raise ArgumentError(f"{what} requires a successful QR factorization")


def apply_q_(B: MFMatrix, F: MFQR, trans: str = "N") -> MFMatrix:
    """B = Q B (trans N) or Q^T B (trans T) from the compact reflectors
    (src/factorizations/qr.jl:938-956)."""
    _qr_ok(F, "apply_q!")
    if trans not in ("N", "T"):
        raise ArgumentError("trans must be :N or :T")
    N = _same_type(B, F.factors)
    if B.m != F.factors.m:
        raise DimensionMismatch("apply_q! destination row count differs")
    if _mightalias(B, F.factors):
        raise ArgumentError("apply_q! destination must not alias QR storage")
    Fm = F.factors
    r = min(Fm.m, Fm.n)
    lib, h, s = _lib_h(B)
    _check(lib.mflab_apply_q(h, s, N, 1 if trans == "T" else 0, Fm.m, r, Fm.ptr(), Fm.ld, Fm.ls,
                             F.tau.data_ptr(), F.tau.stride(0), B.ptr(), B.ld, B.ls, B.n),
           "apply_q!")
    return B


def solve_r_(B: MFMatrix, F: MFQR, rank: int, trans: str = "N",
             config: KernelConfig = _DEFAULT) -> MFMatrix:
    """Solve the leading rank x rank block of R (or its transpose) in place
    (src/factorizations/qr.jl:958-1014)."""
    _qr_ok(F, "solve_r!")
    if trans not in ("N", "T"):
        raise ArgumentError("trans must be :N or :T")
    kmax = min(F.factors.m, F.factors.n)
    rank = int(rank)
    if not 0 <= rank <= kmax:
        raise ArgumentError(f"rank must be between zero and {kmax}")
    if B.m != rank:
        raise DimensionMismatch("solve_r! destination row count must equal rank")
    d = factor_rdiag(F)
    for i in range(rank):
        if np.all(d[:, i] == 0):
            raise SingularException(i + 1)
    if rank == 0:
        return B
    lead = F.factors.view(slice(0, rank), slice(0, rank))
    return trsm_(B, lead, 1.0, side="left", uplo="upper", trans=trans, diag="nonunit",
                 config=config)


def _mf_tol(N: int, v, what: str) -> np.ndarray:
    t = np.zeros(N)
    tv = np.atleast_1d(np.asarray(v, dtype=np.float64)).ravel()
    if len(tv) > N:
        raise ArgumentError(f"{what} has more limbs than the matrix type")
    t[:len(tv)] = tv
    nz = t[t != 0]
    if not np.all(np.isfinite(t)) or (len(nz) and nz[0] < 0):
        raise ArgumentError(f"{what} must be finite and nonnegative")
    return t


def numerical_rank(F: MFQR, atol=0.0, rtol=0.0) -> int:
    """Leading count of |R[i,i]| > max(atol, rtol * max |R[i,i]|)
    (src/factorizations/qr.jl:863-888)."""
    _qr_ok(F, "numerical_rank")
    N = F.N
    a, r = _mf_tol(N, atol, "atol"), _mf_tol(N, rtol, "rtol")
    out = torch.zeros(1, dtype=torch.int64, device=F.factors.storage.device)
    Fm = F.factors
    lib, h, s = _lib_h(Fm)
    _check(lib.mflab_qr_numerical_rank(h, s, N, Fm.m, Fm.n, Fm.ptr(), Fm.ld, Fm.ls,
                                       _scalar(N, a), _scalar(N, r), out.data_ptr()),
           "numerical_rank")
    return int(out.item())


def _ldiv_qr(dest: MFMatrix, F: MFQR, source: Optional[MFMatrix], config) -> MFMatrix:
    """square pivoted-QR solve: Q^T, leading R, column permutation
    (src/solve.jl:425-545)"""
    if not issuccess(F):
        raise ArgumentError("ldiv! requires a successful QR factorization")
    n = F.factors.m
    if F.factors.n != n:
        raise DimensionMismatch("QR ldiv! is defined only for square factors; use apply_q! and "
                                "solve_r! for caller-selected rectangular/rank routes")
    if dest.m != n:
        raise DimensionMismatch("right-hand side dimensions differ")
    d = factor_rdiag(F)
    for i in range(n):
        if np.all(d[:, i] == 0):
            raise SingularException(i + 1)
    if source is not None:
        if (source.m, source.n) != (dest.m, dest.n):
            raise DimensionMismatch("right-hand side length differs")
    _no_alias("ldiv!", dest, F.factors)
    if source is not None and source is not dest:
        if _mightalias(dest, source):
            raise ArgumentError("ldiv! does not support partially overlapping right-hand sides")
        dest.copy_(source)
    apply_q_(dest, F, trans="T")
    solve_r_(dest, F, n, config=config)
    view = dest.storage[:, dest.c0:dest.c0 + dest.n, dest.r0:dest.r0 + dest.m]
    tmp = view.clone()
    view.index_copy_(2, F.permutation.to(torch.int64) - 1, tmp)
    return dest


def factor_rdiag(F: _Factor) -> np.ndarray:
    """copy of the stored diagonal pivots, (N, min(m, n)) limbs
    (src/factorizations/cholesky_pivoted.jl:40-48)"""
    A = F.factors
    view = A.storage[:, A.c0:A.c0 + A.n, A.r0:A.r0 + A.m]
    return torch.diagonal(view, dim1=1, dim2=2).cpu().numpy().copy()


def lu_(A: MFMatrix, check: bool = True, config: KernelConfig = _DEFAULT,
        workspace=None) -> MFLU:
    """Blocked partial-pivoting LU in place (src/factorizations/lu.jl:128-195)."""
    N = _same_type(A)
    m, n = A.m, A.n
    kmax = min(m, n)
    dev = A.storage.device
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    ipiv = torch.arange(1, kmax + 1, dtype=torch.int64, device=dev)
    omax = torch.zeros(N + 1, dtype=torch.float64, device=dev)
    lib, h, s = _lib_h(A)
    if m > 0 and n > 0:
        _check(lib.mflab_max_abs(h, s, N, m, n, A.ptr(), A.ld, A.ls, 0, omax.data_ptr()), "lu!")
    block = max(config.lu_block, 1)
    if config.gemm_strategy == "ozaki":
        # INT8 trailing updates between panels of ozaki_block columns
        if ozaki_scheme(config) != "modular":
            raise ArgumentError("the INT8 trailing update uses the modular scheme (ozaki_moduli)")
        _check(lib.mflab_set_int8_engine(h, _int8_engine(config)), "lu!")
        _check(lib.mflab_getrf_ozaki(h, s, N, int(config.ozaki_moduli), m, n, A.ptr(), A.ld,
                                     A.ls, ipiv.data_ptr() if kmax > 0 else None,
                                     max(int(config.ozaki_block), block), block,
                                     info.data_ptr()), "lu!")
    else:
        _check(lib.mflab_getrf(h, s, N, m, n, A.ptr(), A.ld, A.ls,
                               ipiv.data_ptr() if kmax > 0 else None, block, info.data_ptr()),
               "lu!")
    st = _read_info(info)
    if st == -1:
        omax.zero_()
        if check:
            raise DomainError("lu!: input matrix contains non-finite entries")
    if st > 0 and check:
        raise SingularException(st)
    return MFLU(A, ipiv, st, omax[:N].clone())


def _ldlt_block_default(N: int, config: KernelConfig) -> int:
    """src/factorizations/ldlt_tuning.jl:9-15"""
    if config.ldlt_block > 0:
        return config.ldlt_block
    return 16 if N <= 2 else 12 if N == 3 else 8


def ldlt_plan(N: int, n: int, config: KernelConfig = _DEFAULT) -> dict:
    """Unblocked or lazy-blocked LDLT route (src/factorizations/ldlt.jl:329-350)."""
    if not 1 <= N <= 4:
        raise ArgumentError("only 1-4 limb MultiFloats are supported")
    strategy = config.ldlt_strategy
    if strategy not in ("auto", "unblocked", "blocked"):
        raise ArgumentError("ldlt_strategy must be :auto, :unblocked, or :blocked")
    block = max(_ldlt_block_default(N, config), 1)
    if strategy == "unblocked":
        return {"strategy": "unblocked", "reason": "forced_unblocked", "block_size": 1}
    if strategy == "blocked":
        return {"strategy": "blocked", "reason": "forced_blocked", "block_size": max(block, 2)}
    use = block > 1 and n >= max(config.ldlt_blocked_crossover, 1)
    return {"strategy": "blocked" if use else "unblocked",
            "reason": "auto_above_crossover" if use else "auto_below_crossover",
            "block_size": block if use else 1}


def ldlt_(A: MFMatrix, check: bool = True, config: KernelConfig = _DEFAULT,
          workspace=None) -> MFLDLT:
    """Bunch-Kaufman LDL^T in place; the lower triangle is authoritative
    (src/factorizations/ldlt.jl:654-717)."""
    N = _same_type(A)
    n = A.m
    if A.n != n:
        raise DimensionMismatch("ldlt! requires a square matrix")
    plan = ldlt_plan(N, n, config)
    dev = A.storage.device
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    dsub = torch.zeros((N, max(n, 1)), dtype=torch.float64, device=dev)
    pivots = torch.arange(1, n + 1, dtype=torch.int64, device=dev)
    blocks = torch.zeros(max(n, 1), dtype=torch.uint8, device=dev)
    omax = torch.zeros(N + 1, dtype=torch.float64, device=dev)
    lib, h, s = _lib_h(A)
    if n > 0:
        _check(lib.mflab_max_abs(h, s, N, n, n, A.ptr(), A.ld, A.ls, 1, omax.data_ptr()), "ldlt!")
    blocked = 1 if plan["strategy"] == "blocked" else 0
    _check(lib.mflab_sytrf(h, s, N, n, A.ptr(), A.ld, A.ls, dsub.data_ptr(), dsub.shape[1],
                           pivots.data_ptr() if n else None, blocks.data_ptr(), blocked,
                           plan["block_size"], info.data_ptr()), "ldlt!")
    st = _read_info(info)
    if st == -1:
        omax.zero_()
        if check:
            raise DomainError("ldlt!: input matrix contains non-finite entries")
    if st > 0 and check:
        raise SingularException(st)
    return MFLDLT(A, dsub[:, :n], pivots[:n], blocks[:n], st, omax[:N].clone())


def factor_blocks(F: MFLDLT) -> np.ndarray:
    """caller-owned copy of the LDLT block markers (ldlt.jl:26-32)"""
    return F.blocks.cpu().numpy().copy()


def factor_permutation(F: _Factor) -> np.ndarray:
    """final symmetric permutation p, 1-based: A[p, p] = L D L^T for LDLT
    (ldlt.jl:34-63), the retained block of A[p, p] for pivoted Cholesky
    (cholesky_pivoted.jl:30-38)"""
    if isinstance(F, (MFCholeskyPivoted, MFQR)):
        return F.permutation.cpu().numpy().copy()
    blocks = F.blocks.cpu().numpy()
    piv = F.pivots.cpu().numpy()
    n = len(blocks)
    perm = np.arange(1, n + 1)
    k = 0
    while k < n:
        b = blocks[k]
        if b == 1:
            p = piv[k] - 1
            perm[k], perm[p] = perm[p], perm[k]
            k += 1
        elif b == 2 and k < n - 1:
            p = piv[k] - 1
            perm[k + 1], perm[p] = perm[p], perm[k + 1]
            k += 2
        elif b == 0:
            break
        else:
            raise ArgumentError("invalid LDLT block structure")
    return perm


def _ldlt_diag_record(F: MFLDLT) -> np.ndarray:
    N, A = F.N, F.factors
    out = torch.zeros(6 + 4 * N, dtype=torch.float64, device=A.storage.device)
    lib, h, s = _lib_h(A)
    ds = F.dsub
    _check(lib.mflab_ldlt_diagnostics(h, s, N, A.m, A.ptr(), A.ld, A.ls, ds.data_ptr(),
                                      ds.stride(0) if ds.shape[0] > 1 else max(ds.shape[1], 1),
                                      F.blocks.data_ptr(), F.original_maximum.data_ptr(),
                                      out.data_ptr()), "factor_diagnostics")
    return out.cpu().numpy()


def factor_inertia(F: MFLDLT) -> dict:
    """(positive, negative, zero) of the accepted blocks (diagnostics.jl:162-185)"""
    r = _ldlt_diag_record(F)
    return {"positive": int(r[0]), "negative": int(r[1]), "zero": int(r[2])}


def issuccess(F: _Factor) -> bool:
    return F.info == 0


def factor_status(F: _Factor) -> int:
    return F.info


def factor_kind(F: _Factor) -> str:
    return F.kind


def factor_matrix(F: _Factor) -> MFMatrix:
    return F.factors


def factor_precision(F: _Factor) -> str:
    return limb_type_name(F.N)


def factor_provider(F: _Factor) -> str:
    return "mfla_b200"


def factor_state(F: _Factor) -> str:
    """types.jl:394-403"""
    st = factor_status(F)
    if st == 0:
        return "success"
    if st == -1:
        return "nonfinite_input"
    if st < 0:
        return "numerical_breakdown"
    if F.kind in ("cholesky", "cholesky_pivoted"):
        return "not_posdef"
    if F.kind in ("lu", "ldlt"):
        return "singular"
    return "numerical_breakdown"


def factor_pivots(F: _Factor) -> np.ndarray:
    if isinstance(F, MFLU):
        return F.ipiv.cpu().numpy().copy()
    if hasattr(F, "pivots"):
        return F.pivots.cpu().numpy().copy()
    raise ArgumentError("factor has no pivots")


def _check_solve(F: _Factor) -> None:
    if not issuccess(F):
        if F.kind == "cholesky":
            raise PosDefException(F.info)
        raise SingularException(F.info)


def ldiv_(dest: MFMatrix, F: _Factor, source: Optional[MFMatrix] = None,
          config: KernelConfig = _DEFAULT) -> MFMatrix:
    """Solve in place with a successful factor (src/solve.jl:23-545)."""
    if F.kind == "qr":
        return _ldiv_qr(dest, F, source, config)
    _check_solve(F)
    N = _same_type(dest, F.factors)
    n = F.factors.m
    if F.factors.n != n:
        raise DimensionMismatch("solve requires a square factor")
    if source is not None:
        if (source.m, source.n) != (dest.m, dest.n):
            raise DimensionMismatch("source and destination dimensions differ")
    if dest.m != n:
        raise DimensionMismatch("right-hand side dimensions differ")
    _no_alias("ldiv!", dest, F.factors)
    if source is not None and source is not dest:
        if _mightalias(dest, source):
            raise ArgumentError("ldiv! does not support partially overlapping right-hand sides")
        dest.copy_(source)
    lib, h, s = _lib_h(dest)
    L = F.factors
    with _solve_order(dest, config):
        if F.kind == "cholesky":
            rc = lib.mflab_potrs(h, s, N, n, dest.n, L.ptr(), L.ld, L.ls, dest.ptr(), dest.ld,
                                 dest.ls)
        elif F.kind == "lu":
            rc = lib.mflab_getrs(h, s, N, n, dest.n, L.ptr(), L.ld, L.ls, F.ipiv.data_ptr(),
                                 dest.ptr(), dest.ld, dest.ls)
        else:
            return _ldiv_extra(dest, F, lib, h, s)
    _check(rc, "ldiv!")
    return dest


def _ldiv_extra(dest, F, lib, h, s):
    if F.kind != "ldlt":
        raise ArgumentError(f"ldiv! is not available for {F.kind}")
    N, L = F.N, F.factors
    fail = torch.zeros(1, dtype=torch.int32, device=dest.storage.device)
    ds = F.dsub
    lsd = ds.stride(0) if ds.shape[0] > 1 else max(ds.shape[1], 1)
    _check(lib.mflab_sytrs(h, s, N, L.m, dest.n, L.ptr(), L.ld, L.ls, ds.data_ptr(), lsd,
                           F.pivots.data_ptr(), F.blocks.data_ptr(), dest.ptr(), dest.ld, dest.ls,
                           fail.data_ptr()), "ldiv!")
    f = int(fail.item())
    if 0 < f < 0x7F7F7F7F:
        raise SingularException(f)
    return dest


def solve(F: _Factor, rhs: MFMatrix, config: KernelConfig = _DEFAULT) -> MFMatrix:
    """Non-mutating solve (src/solve.jl:555-565)."""
    return ldiv_(rhs.copy(), F, config=config)


def _mf_values(t: torch.Tensor, N: int, count: int) -> list:
    a = t.cpu().numpy()
    return [a[i * N:(i + 1) * N].copy() for i in range(count)]


def factor_diagnostics(F: _Factor, atol=0.0, rtol=0.0) -> dict:
    """Numerical facts about a factor (src/diagnostics.jl:32-246).  MF-valued
    fields are numpy arrays of N limbs; absent values are None."""
    N = F.N
    A = F.factors
    dev = A.storage.device
    lib, h, s = _lib_h(A)
    base = {
        "kind": F.kind, "status": F.info, "state": factor_state(F), "success": issuccess(F),
        "precision": factor_precision(F), "provider": factor_provider(F),
        "failure_location": F.info if F.info > 0 else None,
    }
    out = torch.zeros(4 * N + 2, dtype=torch.float64, device=dev)
    if F.kind == "cholesky":
        n = A.m
        accepted = n if F.info == 0 else (F.info - 1 if F.info > 0 else 0)
        _check(lib.mflab_diag_summary(h, s, N, A.ptr(), A.ld, A.ls, accepted, None, None,
                                      out.data_ptr()), "factor_diagnostics")
        mn, mx, spread, _ = _mf_values(out, N, 4)
        has = accepted > 0
        base.update({
            "accepted_pivots": accepted,
            "minimum_diagonal": mn if has else None,
            "maximum_diagonal": mx if has else None,
            "diagonal_spread": spread if has else None,
            "finite": _finite_region(A, 1),
        })
        return base
    if F.kind == "qr":
        # diagnostics.jl:248-275; atol / rtol are forwarded to numerical_rank
        r = min(A.m, A.n)
        _check(lib.mflab_diag_summary(h, s, N, A.ptr(), A.ld, A.ls, r, None, None,
                                      out.data_ptr()), "factor_diagnostics")
        mn, mx, spread, _ = _mf_values(out, N, 4)
        has = r > 0
        base.update({
            "failure_location": None,
            "permutation": factor_permutation(F),
            "rdiag": factor_rdiag(F),
            "minimum_rdiag": mn if has else None,
            "maximum_rdiag": mx if has else None,
            "rdiag_spread": spread if has else None,
            "rank_at_threshold": numerical_rank(F, atol, rtol) if issuccess(F) else 0,
            "atol": _mf_tol(N, atol, "atol"),
            "rtol": _mf_tol(N, rtol, "rtol"),
            "finite": _finite_region(A, 0) and bool(torch.isfinite(F.tau).all().item()),
        })
        return base
    if F.kind == "cholesky_pivoted":
        # diagnostics.jl:53-70: the retained rank is the accepted pivot count
        accepted = F.rank
        _check(lib.mflab_diag_summary(h, s, N, A.ptr(), A.ld, A.ls, accepted, None, None,
                                      out.data_ptr()), "factor_diagnostics")
        mn, mx, spread, _ = _mf_values(out, N, 4)
        has = accepted > 0
        base.update({
            "rank": accepted,
            "permutation": factor_permutation(F),
            "minimum_diagonal": mn if has else None,
            "maximum_diagonal": mx if has else None,
            "diagonal_spread": spread if has else None,
            "finite": _finite_region(A, 1),
        })
        return base
    if F.kind == "lu":
        kmax = min(A.m, A.n)
        accepted = F.info - 1 if F.info > 0 else (kmax if F.info == 0 else 0)
        umax = torch.zeros(N + 1, dtype=torch.float64, device=dev)
        _check(lib.mflab_max_abs(h, s, N, A.m, A.n, A.ptr(), A.ld, A.ls, 2, umax.data_ptr()),
               "factor_diagnostics")
        _check(lib.mflab_diag_summary(h, s, N, A.ptr(), A.ld, A.ls, accepted, umax.data_ptr(),
                                      F.original_maximum.data_ptr(), out.data_ptr()),
               "factor_diagnostics")
        mn, mx, _, growth = _mf_values(out, N, 4)
        omax = F.original_maximum.cpu().numpy()
        has = accepted > 0
        base.update({
            "accepted_pivots": accepted,
            "pivots": F.ipiv.cpu().numpy().copy(),
            "minimum_pivot": mn if has else None,
            "maximum_pivot": mx if has else None,
            "original_maximum": None if F.info == -1 else omax.copy(),
            "maximum_u": umax[:N].cpu().numpy(),
            "pivot_growth": None if not np.any(omax != 0) else growth,
            "finite": _finite_region(A, 0),
        })
        return base
    return _diagnostics_extra(F, base)


def _diagnostics_extra(F, base):
    if F.kind != "ldlt":
        raise ArgumentError(f"no diagnostics for {F.kind}")
    N = F.N
    r = _ldlt_diag_record(F)
    have = r[5] == 1.0
    minb, maxe, scaled, growth = (r[6 + i * N:6 + (i + 1) * N].copy() for i in range(4))
    omax = F.original_maximum.cpu().numpy()
    omax_zero = not np.any(omax != 0)
    A = F.factors
    ds = F.dsub
    dfin = True
    if ds.shape[1] > 0:
        dfin = bool(torch.isfinite(ds).all().item())
    base.update({
        "one_by_one_pivots": int(r[3]), "two_by_two_pivots": int(r[4]),
        "pivots": F.pivots.cpu().numpy().copy(), "blocks": F.blocks.cpu().numpy().copy(),
        "inertia": {"positive": int(r[0]), "negative": int(r[1]), "zero": int(r[2])},
        "minimum_block_eigenvalue_magnitude": minb if have else None,
        "minimum_scaled_block": None if (not have or omax_zero) else scaled,
        "original_maximum": None if F.info == -1 else omax.copy(),
        "maximum_block_entry": maxe,
        "block_growth": None if omax_zero else growth,
        "finite": _finite_region(A, 0) and dfin,
    })
    return base


_UPLO_R = {"general": 0, "lower": 1, "upper": 2}


def _check_residual_dims(R: MFMatrix, A: MFMatrix, X: MFMatrix, B: MFMatrix, uplo: str):
    if uplo not in _UPLO_R:
        raise ArgumentError("uplo must be :general, :lower, or :upper")
    rows, cols = A.m, A.n
    if (R.m, R.n) != (B.m, B.n):
        raise DimensionMismatch("residual output dimensions differ")
    if R.m != rows:
        raise DimensionMismatch("residual output row count differs")
    if X.m != cols:
        raise DimensionMismatch("residual solution row count differs")
    if X.n != R.n:
        raise DimensionMismatch("residual right-hand-side count differs")
    if uplo != "general" and rows != cols:
        raise DimensionMismatch("symmetric residual requires a square matrix")


def residual_(R: MFMatrix, A: MFMatrix, X: MFMatrix, B: MFMatrix, uplo: str = "general",
              config: KernelConfig = _DEFAULT, workspace=None) -> MFMatrix:
    """R = B - A X in caller-owned storage (src/residual.jl:55-125); R may be B."""
    N = _same_type(R, A, X, B)
    _check_residual_dims(R, A, X, B, uplo)
    if _mightalias(R, X):
        raise ArgumentError("residual output must not alias x")
    if _mightalias(R, A):
        raise ArgumentError("residual output must not alias A")
    if R is not B and _mightalias(R, B) and not (R.storage.data_ptr() == B.storage.data_ptr()
                                                  and (R.r0, R.c0) == (B.r0, B.c0)):
        raise ArgumentError("residual output may equal b but must not partially alias it")
    lib, h, s = _lib_h(R)
    _check(lib.mflab_residual(h, s, N, _UPLO_R[uplo], int(R.is_vector), A.m, A.n, R.n, A.ptr(),
                              A.ld, A.ls, X.ptr(), X.ld, X.ls, B.ptr(), B.ld, B.ls, R.ptr(), R.ld,
                              R.ls), "residual!")
    return R


def residual_mixed_(R: MFMatrix, A: MFMatrix, X: MFMatrix, B: MFMatrix, uplo: str = "general",
                    config: KernelConfig = _DEFAULT) -> MFMatrix:
    """R = B - A X with every operand widened to R's limb count first
    (src/residual.jl:431-496).  Source limbs 1 (binary64) to 3."""
    src = A.N
    for M in (X, B):
        if M.N != src:
            raise ArgumentError("residual_mixed! sources must share one limb count")
    res = R.N
    if not (1 <= src < res <= 4 and res >= 2):
        raise ArgumentError("residual_mixed! supports only widening to a higher limb count")
    _check_residual_dims(R, A, X, B, uplo)
    lib, h, s = _lib_h(R)
    _check(lib.mflab_residual_mixed(h, s, src, res, _UPLO_R[uplo], A.m, A.n, R.n, A.ptr(), A.ld,
                                    A.ls, X.ptr(), X.ld, X.ls, B.ptr(), B.ld, B.ls, R.ptr(), R.ld,
                                    R.ls), "residual_mixed!")
    return R


class OpNormInf:
    """||A||_inf of one matrix on its device (the matrix term of the normwise
    backward error), for repeated backward errors against it."""

    def __init__(self, A: MFMatrix, uplo: str = "general", handle=None):
        N = _same_type(A)
        if uplo not in _UPLO_R:
            raise ArgumentError("uplo must be :general, :L or :U")
        self.N, self.m, self.k = N, A.m, A.n
        self.value = torch.zeros(N, dtype=torch.float64, device=A.storage.device)
        self.nonfinite = torch.zeros(1, dtype=torch.int32, device=A.storage.device)
        lib, h, s = _lib_h(A)
        if handle is not None:
            h = handle
        _check(lib.mflab_opnorm_inf(h, s, N, _UPLO_R[uplo], A.m, A.n, A.ptr(), A.ld, A.ls,
                                    self.value.data_ptr(), self.nonfinite.data_ptr()),
               "opnorm")


def normwise_backward_error(A: MFMatrix, X: MFMatrix, B: MFMatrix, R: MFMatrix,
                            uplo: str = "general", anorm: Optional[OpNormInf] = None):
    """||r|| / (||A|| ||x|| + ||b||) (src/residual.jl:202-269): one N-limb value
    for a vector, a list of them for a matrix right-hand side.  `anorm`
    (an OpNormInf of A) skips the pass over A."""
    N = _same_type(A, X, B, R)
    _check_residual_dims(R, A, X, B, uplo)
    out = torch.zeros(max(R.n, 1) * N, dtype=torch.float64, device=A.storage.device)
    lib, h, s = _lib_h(A)
    if anorm is not None:
        if (anorm.N, anorm.m, anorm.k) != (N, A.m, A.n):
            raise DimensionMismatch("normwise_backward_error: anorm belongs to another matrix")
        _check(lib.mflab_backward_error_norm(h, s, N, A.m, A.n, R.n, anorm.value.data_ptr(),
                                             anorm.nonfinite.data_ptr(), X.ptr(), X.ld, X.ls,
                                             B.ptr(), B.ld, B.ls, R.ptr(), R.ld, R.ls,
                                             out.data_ptr()), "normwise_backward_error")
    else:
        _check(lib.mflab_backward_error(h, s, N, _UPLO_R[uplo], A.m, A.n, R.n, A.ptr(), A.ld,
                                        A.ls, X.ptr(), X.ld, X.ls, B.ptr(), B.ld, B.ls, R.ptr(),
                                        R.ld, R.ls, out.data_ptr()), "normwise_backward_error")
    vals = out.cpu().numpy().reshape(-1, N)[:R.n]
    return vals[0].copy() if R.is_vector else [v.copy() for v in vals]


def refinement_correction_(delta: MFMatrix, F: _Factor, r: MFMatrix,
                           config: KernelConfig = _DEFAULT) -> MFMatrix:
    """Exactly one correction delta = F \\ r (src/residual.jl:302-332)."""
    _check_solve(F)
    if (delta.m, delta.n) != (r.m, r.n):
        raise DimensionMismatch("correction and residual dimensions differ")
    if r.m != F.factors.m:
        raise DimensionMismatch("correction residual rows differ from factor")
    if _mightalias(delta, F.factors):
        raise ArgumentError("correction destination must not alias factor storage")
    return ldiv_(delta, F, None if delta is r else r, config)


def _leading_limb(X: MFMatrix) -> MFMatrix:
    """the binary64 rounding of a normalised multi-double matrix (its leading
    limb) as a one-limb matrix"""
    st = X.planes()[0:1].contiguous().clone()
    if st.shape[2] == 0:
        st = torch.zeros((1, X.n, 1), dtype=torch.float64, device=X.storage.device)
    return MFMatrix(st, 0, 0, X.m, X.n, X.is_vector)


# panel width of the binary64 factor of solve_mixed_lu: the panel lives in
# the shared memory of an 8-CTA cluster, one cluster barrier per column, so
# wide panels (fewer trailing updates) win
_LU64_PANEL = 32


def solve_mixed_lu(A: MFMatrix, B: MFMatrix, tol: float = 0.0, maxiter: int = 40,
                   config: KernelConfig = _DEFAULT, residual: str = "int8",
                   timing: bool = False) -> tuple:
    """Solve A X = B for a Float64xN matrix A with a binary64 partial-pivoting
    LU of round(A) and iterative refinement with Float64xN residuals.

    Each iteration: D = LU64 \\ round(R) in binary64 (the factor's
    permutation and inverted diagonal blocks, prepared once), X += D in
    Float64xN, R = B - A X in Float64xN, then the normwise backward error of
    every column (||A||_inf computed once).  The residual goes through the
    INT8 modular GEMM (residual="int8", error at the Float64xN level of the
    plain kernel) or residual! in the reference order (residual="matched").
    Stops when all backward errors are <= tol (default 2^(-53N)) or after
    maxiter iterations.  Returns (X, report); with timing=True the report
    also holds the device times of the binary64 factor and of the
    refinement loop (CUDA events on the current stream).  The reference provides the
    pieces (lu!, residual!, refinement_correction!) but leaves the refinement
    loop to the caller.
    """
    if residual not in ("int8", "matched"):
        raise ArgumentError("residual must be :int8 or :matched")
    N = _same_type(A, B)
    n = A.m
    if A.n != n:
        raise DimensionMismatch("solve requires a square matrix")
    if B.m != n:
        raise DimensionMismatch("right-hand side dimensions differ")
    tol = tol or 2.0 ** (-53 * N)
    dev = A.storage.device
    lib, h, s = _lib_h(A)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)] if timing else None
    # ||A||_inf of the backward errors: one serial chain per row, independent
    # of the factor, so it runs on a side stream (with a handle of its own)
    # while the binary64 LU runs
    main = torch.cuda.current_stream(dev)
    side = torch.cuda.Stream(dev)
    side.wait_stream(main)
    with torch.cuda.stream(side):
        anorm = OpNormInf(A, handle=_side_handle(A.device))
    anorm.value.record_stream(main)
    anorm.nonfinite.record_stream(main)
    if timing:
        ev[0].record()
    LU = _leading_limb(A)
    ipiv = torch.arange(1, n + 1, dtype=torch.int64, device=dev)
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    _check(lib.mflab_getrf(h, s, 1, n, n, LU.ptr(), LU.ld, LU.ls, ipiv.data_ptr() if n else None,
                           _LU64_PANEL, info.data_ptr()), "lu! (binary64)")
    if timing:
        ev[1].record()
    st = _read_info(info)
    if st == -1:
        raise DomainError("lu!: input matrix contains non-finite entries")
    if st > 0:
        raise SingularException(st)
    # the permutation and the inverted 128 x 128 diagonal blocks, once for all
    # correction solves
    wb = C.c_size_t()
    _check(lib.mflab_lu64_work_bytes(n, C.byref(wb)), "lu64 workspace")
    work = torch.empty(max(wb.value, 1), dtype=torch.uint8, device=dev)
    _check(lib.mflab_lu64_prepare(h, s, n, LU.ptr(), LU.ld, ipiv.data_ptr(), work.data_ptr()),
           "lu64 prepare")
    X = MFMatrix.zeros(N, n, None if B.is_vector else B.n, device=dev)
    R = B.copy()
    D = MFMatrix.empty(1, n, None if B.is_vector else B.n, device=dev)
    main.wait_stream(side)
    rcfg = dataclasses.replace(config, gemm_strategy="ozaki", ozaki_scheme="modular",
                               ozaki_slices=0)
    history = []
    it = 0
    prepared = None
    for it in range(1, maxiter + 1):
        D.planes().copy_(R.planes()[0:1])  # round(R): the leading limbs
        _check(lib.mflab_lu64_solve(h, s, n, D.n, LU.ptr(), LU.ld, work.data_ptr(), D.ptr(),
                                    D.ld), "ldiv! (binary64)")
        _check(lib.mflab_add_widened(h, s, 1, N, n, X.n, D.ptr(), D.ld, D.ls, X.ptr(), X.ld,
                                     X.ls), "refinement update")
        if residual == "int8":
            R.copy_(B)
            if prepared is None:
                # the modulus count the tuner picks for A and the first
                # iterate; A's residues are then prepared once for every
                # residual
                moduli = rcfg.ozaki_moduli or ozaki_crt_tune_moduli(A, X)
                prepared = PreparedInt8Operand(A, moduli)
            gemm_prepared_(R, prepared, X, -1.0, 1.0, config=rcfg)
        else:
            residual_(R, A, X, B)
        be = normwise_backward_error(A, X, B, R, anorm=anorm)
        worst = float(np.max([v[0] for v in (be if isinstance(be, list) else [be])]))
        history.append(worst)
        if worst <= tol:
            break
    if timing:
        ev[2].record()
        ev[2].synchronize()
    report = {"iterations": it, "backward_error": history[-1] if history else None,
              "history": history, "converged": bool(history) and history[-1] <= tol,
              "factor": "binary64 partial-pivoting LU",
              "residual": limb_type_name(N) + (" (INT8 modular GEMM)" if residual == "int8"
                                               else " (reference order)")}
    if timing:
        report["factor_ms"] = ev[0].elapsed_time(ev[1])
        report["refine_ms"] = ev[1].elapsed_time(ev[2])
    return X, report


def capabilities(N: int) -> dict:
    """Machine-readable facts about this backend (src/capabilities.jl:14-74)."""
    supported = 2 <= N <= 4
    return {
        "provider": "mfla_b200", "scalar_type": limb_type_name(N), "base_type": "Float64",
        "supported": supported, "limb_count": N,
        "gemm": supported, "gemmt": supported, "syrk": supported, "trsv": supported,
        "trsm": supported, "cholesky": supported, "lu": supported, "ldlt": supported,
        "ldlt_lightweight_metadata": supported,
        "factor_diagnostics": supported, "vector_rhs": supported, "multi_rhs": supported,
        "factor_metadata_ownership": "factor_owned", "factor_matrix_ownership": "borrowed_input",
        "factorization_destructive": True, "factor_solve_mutates_factor": False,
        "syrk_authoritative_triangle": "lower", "syrk_inactive_triangle": "preserved",
        "device": "cuda", "gemm_routes": ["auto", "direct", "fused", "ozaki"],
        "residual": supported, "refinement_correction": supported,
        "mixed_precision_residual": supported and N in (2, 3),
        "mixed_residual_targets": {"x2": False, "x3": supported and N == 2,
                                   "x4": supported and N in (2, 3)},
    }


from . import batched  # noqa: E402  (batched SPD factor/solve and its adjoint)
from . import tuning  # noqa: E402  (persisted device tuning profiles)
