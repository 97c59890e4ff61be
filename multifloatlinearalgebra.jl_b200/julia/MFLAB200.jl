"""
    MFLAB200

Julia binding of the B200 multi-double backend: the C ABI of
`libmflab200.so` (declared in `include/mflab200.h`) bound with `ccall`, no
CUDA.jl and no kernel code generation.

It adds device arrays of `Float64x2/x3/x4` (`MFDeviceMatrix{N}`,
`MFDeviceVector{N}`: N column-major limb planes on one GPU) and methods of
MultiFloatLinearAlgebra.jl's own generic functions (`gemm!`, `syrk!`,
`gemmt!`, `trsm!`, `trsv!`, `trmm!`, `gemv!`, `symv!`, `mfdot`, `cholesky!`,
`cholesky_pivoted!`, `lu!`, `ldlt!`, `qr!`, `rrqr!`, `apply_q!`, `ldiv!`,
`solve`, `residual!`, `residual_mixed!`, `normwise_backward_error`) for them,
so a caller of the reference switches by moving the operands to the device:

    using MultiFloats, MultiFloatLinearAlgebra, MFLAB200
    A = MFDeviceArray(rand(Float64x2, 4096, 4096))       # host -> limb planes
    F = cholesky!(A)                                      # the reference's MFCholesky
    x = Array(solve(F, MFDeviceArray(b)))                 # limb planes -> host

Factorizations return the reference's factor types (`MFCholesky`, `MFLU`,
`MFLDLT`, ...) holding device matrices, so `factor_status`, `factor_state`,
`issuccess` and `factor_matrix` work unchanged.  Errors map as in the
reference: bad shapes throw `DimensionMismatch`, bad options and aliasing
`ArgumentError`, numerical failures `PosDefException` / `SingularException` /
`DomainError` with `check=true`.

Device-only choices (the INT8 tensor-core routes, the int8 engine, the
triangular-solve order) go in a `DeviceConfig` keyword; the reference's
`KernelConfig` keeps its meaning (block sizes, strategies).
"""
module MFLAB200

using LinearAlgebra
using MultiFloats
import MultiFloats: MultiFloat
import MultiFloatLinearAlgebra
import MultiFloatLinearAlgebra: KernelConfig, MFCholesky, MFCholeskyPivoted, MFLU, MFLDLT, MFQR,
    gemm!, syrk!, gemmt!, trsm!, trsv!, trmm!, gemv!, symv!, mfdot, cholesky!, cholesky_pivoted!,
    lu!, ldlt!, qr!, rrqr!, apply_q!, ldiv!, solve, residual!, residual_mixed!,
    normwise_backward_error

export MFHandle, MFDeviceArray, MFDeviceMatrix, MFDeviceVector, DeviceConfig, MFLABError,
    default_handle, device_status, solve_mixed_lu

const libmflab = get(ENV, "MFLAB200_LIB", normpath(joinpath(@__DIR__, "..", "libmflab200.so")))

const MF{N} = MultiFloat{Float64,N}

# ------------------------------------------------------------ status ----
const MFLAB_OK = Cint(0)
const MFLAB_ERR_ARG = Cint(-1)
const MFLAB_ERR_CUDA = Cint(-2)
const MFLAB_ERR_UNSUPPORTED = Cint(-3)
const MFLAB_ERR_TIMEOUT = Cint(-4)
const MFLAB_ERR_ALLOC = Cint(-5)
const MFLAB_ERR_ALIAS = Cint(-6)
const MFLAB_ERR_FLAG = Cint(-7)

"""A CUDA failure, bounded-wait timeout or device allocation failure."""
struct MFLABError <: Exception
    code::Cint
    msg::String
end
Base.showerror(io::IO, e::MFLABError) = print(io, "MFLAB200 error ", e.code, ": ", e.msg)

function check(rc::Cint)
    rc == MFLAB_OK && return nothing
    msg = unsafe_string(ccall((:mflab_status_string, libmflab), Cstring, (Cint,), rc))
    detail = unsafe_string(ccall((:mflab_last_error, libmflab), Cstring, ()))
    isempty(detail) || (msg *= " (" * detail * ")")
    rc == MFLAB_ERR_ARG && throw(DimensionMismatch(msg))
    rc in (MFLAB_ERR_FLAG, MFLAB_ERR_ALIAS, MFLAB_ERR_UNSUPPORTED) && throw(ArgumentError(msg))
    throw(MFLABError(rc, msg))
end

# ----------------------------------------------------- handles, memory ----
"""One library handle per concurrent caller, like the reference's MFWorkspace
(types.jl:71-123): it owns the device scratch of the calls issued with it."""
mutable struct MFHandle
    ptr::Ptr{Cvoid}
    device::Int
    function MFHandle(device::Integer=0)
        r = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:mflab_create, libmflab), Cint, (Ptr{Ptr{Cvoid}}, Cint), r, device))
        h = new(r[], Int(device))
        finalizer(h) do x
            x.ptr == C_NULL || ccall((:mflab_destroy, libmflab), Cint, (Ptr{Cvoid},), x.ptr)
            x.ptr = C_NULL
        end
        return h
    end
end

const _handles = Dict{Tuple{Int,Int},MFHandle}()
const _handles_lock = ReentrantLock()

"""The handle of the calling task's thread on `device` (created on first use)."""
default_handle(device::Integer=0) = lock(_handles_lock) do
    get!(() -> MFHandle(device), _handles, (Int(device), Threads.threadid()))
end

mutable struct DeviceBuffer
    ptr::Ptr{Cvoid}
    bytes::Int
    function DeviceBuffer(bytes::Integer, device::Integer=0)
        r = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:mflab_malloc, libmflab), Cint, (Cint, Csize_t, Ptr{Ptr{Cvoid}}),
                    device, bytes, r))
        b = new(r[], Int(bytes))
        finalizer(b) do x
            x.ptr == C_NULL || ccall((:mflab_free, libmflab), Cint, (Ptr{Cvoid},), x.ptr)
            x.ptr = C_NULL
        end
        return b
    end
end

synchronize(stream::Ptr{Cvoid}=C_NULL) =
    check(ccall((:mflab_stream_synchronize, libmflab), Cint, (Ptr{Cvoid},), stream))

function memcpy!(dst::Ptr, src::Ptr, bytes::Integer, kind::Integer, stream::Ptr{Cvoid}=C_NULL)
    check(ccall((:mflab_memcpy, libmflab), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Csize_t, Cint, Ptr{Cvoid}),
                dst, src, bytes, kind, stream))
end

"""A small device array of plain elements (info words, pivots, block marks)."""
struct DeviceWords{T}
    ptr::Ptr{T}
    len::Int
    owner::DeviceBuffer
end
function DeviceWords{T}(len::Integer, device::Integer=0) where {T}
    b = DeviceBuffer(max(len, 1) * sizeof(T), device)
    check(ccall((:mflab_memset, libmflab), Cint, (Ptr{Cvoid}, Cint, Csize_t, Ptr{Cvoid}),
                b.ptr, 0, max(len, 1) * sizeof(T), C_NULL))
    return DeviceWords{T}(Ptr{T}(b.ptr), Int(len), b)
end
function DeviceWords(v::Vector{T}, device::Integer=0) where {T}
    w = DeviceWords{T}(length(v), device)
    GC.@preserve v memcpy!(w.ptr, pointer(v), length(v) * sizeof(T), 0)
    return w
end
function host(w::DeviceWords{T}, stream::Ptr{Cvoid}=C_NULL) where {T}
    v = Vector{T}(undef, w.len)
    GC.@preserve v begin
        memcpy!(pointer(v), w.ptr, w.len * sizeof(T), 1, stream)
        synchronize(stream)
    end
    return v
end

# ------------------------------------------------------ device arrays ----
"""
    MFDeviceArray{N,D}

A Float64xN matrix (D = 2) or vector (D = 1) as N column-major binary64 limb
planes on one GPU: limb l of element (r, c) at `ptr + 8 (l ls + (c-1) ld + (r-1))`.
Views are pointer offsets sharing `ld`, `ls` and the owner."""
struct MFDeviceArray{N,D} <: AbstractArray{MultiFloat{Float64,N},D}
    ptr::Ptr{Float64}
    m::Int
    n::Int
    ld::Int
    ls::Int
    device::Int
    owner::Any
end
const MFDeviceMatrix{N} = MFDeviceArray{N,2}
const MFDeviceVector{N} = MFDeviceArray{N,1}

Base.size(A::MFDeviceArray{N,2}) where {N} = (A.m, A.n)
Base.size(A::MFDeviceArray{N,1}) where {N} = (A.m,)
Base.getindex(::MFDeviceArray, ::Int...) =
    throw(ArgumentError("MFDeviceArray elements live on the GPU; copy them with Array(A)"))
Base.setindex!(::MFDeviceArray, v, ::Int...) =
    throw(ArgumentError("MFDeviceArray elements live on the GPU; copy with copyto!(A, X)"))

function MFDeviceArray{N,D}(::UndefInitializer, m::Integer, n::Integer=1;
                            device::Integer=0) where {N,D}
    ld = max(Int(m), 1)
    cols = max(Int(n), 1)
    buf = DeviceBuffer(8 * N * ld * cols, device)
    return MFDeviceArray{N,D}(Ptr{Float64}(buf.ptr), Int(m), D == 1 ? 1 : Int(n), ld, ld * cols,
                              Int(device), buf)
end
MFDeviceMatrix{N}(::UndefInitializer, m::Integer, n::Integer; device::Integer=0) where {N} =
    MFDeviceArray{N,2}(undef, m, n; device=device)
MFDeviceVector{N}(::UndefInitializer, m::Integer; device::Integer=0) where {N} =
    MFDeviceArray{N,1}(undef, m, 1; device=device)

function Base.zeros(::Type{MFDeviceArray{N,D}}, m::Integer, n::Integer=1;
                    device::Integer=0) where {N,D}
    A = MFDeviceArray{N,D}(undef, m, n; device=device)
    check(ccall((:mflab_memset, libmflab), Cint, (Ptr{Cvoid}, Cint, Csize_t, Ptr{Cvoid}),
                A.ptr, 0, 8 * A.ls * N, C_NULL))
    return A
end

"""`view(A, rows, cols)` of a device matrix: unit ranges, no copy."""
function Base.view(A::MFDeviceMatrix{N}, rows::UnitRange{Int}, cols::UnitRange{Int}) where {N}
    (isempty(rows) || (1 <= first(rows) && last(rows) <= A.m)) &&
        (isempty(cols) || (1 <= first(cols) && last(cols) <= A.n)) ||
        throw(BoundsError(A, (rows, cols)))
    off = (first(cols) - 1) * A.ld + (first(rows) - 1)
    return MFDeviceArray{N,2}(A.ptr + 8 * off, length(rows), length(cols), A.ld, A.ls, A.device,
                              A.owner)
end

# A Julia Array{MultiFloat{Float64,N}} keeps the N limbs of each element side
# by side; the interleaved entry points turn that into limb planes and back
# (gemm.jl:747-755 takes such arrays).
"""Upload host data into a device array of the same size (mflab_h2d_interleaved)."""
function Base.copyto!(A::MFDeviceArray{N}, X::Array{MultiFloat{Float64,N}};
                      handle::MFHandle=default_handle(A.device),
                      stream::Ptr{Cvoid}=C_NULL) where {N}
    (size(X, 1) == A.m && size(X, 2) == A.n && ndims(X) <= 2) ||
        throw(DimensionMismatch("host array of size $(size(X)) for a $(A.m)x$(A.n) device array"))
    GC.@preserve X begin
        check(ccall((:mflab_h2d_interleaved, libmflab), Cint,
                    (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Int64, Int64, Ptr{Float64}, Int64,
                     Ptr{Float64}, Int64, Int64),
                    handle.ptr, stream, N, A.m, A.n, Ptr{Float64}(pointer(X)), max(A.m, 1),
                    A.ptr, A.ld, A.ls))
        synchronize(stream)  # X may move once GC.@preserve ends
    end
    return A
end

"""A device copy of a host Float64xN array."""
function MFDeviceArray(X::AbstractArray{MultiFloat{Float64,N},D};
                       device::Integer=0) where {N,D}
    D <= 2 || throw(ArgumentError("only vectors and matrices are supported"))
    Xc = X isa Array ? X : collect(X)
    A = MFDeviceArray{N,D}(undef, size(Xc, 1), D == 2 ? size(Xc, 2) : 1; device=device)
    return copyto!(A, Xc)
end

"""The host copy of a device array (mflab_d2h_interleaved)."""
function Base.Array(A::MFDeviceArray{N,D}; handle::MFHandle=default_handle(A.device),
                    stream::Ptr{Cvoid}=C_NULL) where {N,D}
    X = Array{MultiFloat{Float64,N}}(undef, size(A))
    GC.@preserve X begin
        check(ccall((:mflab_d2h_interleaved, libmflab), Cint,
                    (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Int64, Int64, Ptr{Float64}, Int64, Int64,
                     Ptr{Float64}, Int64),
                    handle.ptr, stream, N, A.m, A.n, A.ptr, A.ld, A.ls,
                    Ptr{Float64}(pointer(X)), max(A.m, 1)))
        synchronize(stream)
    end
    return X
end

function Base.copy(A::MFDeviceArray{N,D}) where {N,D}
    B = MFDeviceArray{N,D}(undef, A.m, A.n; device=A.device)
    for l in 0:N-1, c in 0:A.n-1
        memcpy!(B.ptr + 8 * (l * B.ls + c * B.ld), A.ptr + 8 * (l * A.ls + c * A.ld), 8 * A.m, 2)
    end
    return B
end

# -------------------------------------------------------------- config ----
"""
    DeviceConfig(; int8=:off, moduli=0, slices=0, engine=:tcgen05,
                 int8_panel=256, solve_order=:matched)

Device-only choices with no reference counterpart: `int8 = :modular` or
`:slices` runs gemm!/syrk! (and the trailing updates of cholesky!/lu!, in
panels of `int8_panel` columns) on the INT8 tensor cores (moduli / slices
0: tuned to the plain kernel's accuracy); `engine` picks the int8 product
kernel (`:tcgen05` default, `:tcgen05_1sm`, `:tcgen05_pair`, `:library`);
`solve_order = :fast` applies triangular-solve terms as unknowns finalise
(deterministic, not the reference's association)."""
Base.@kwdef struct DeviceConfig
    int8::Symbol = :off
    moduli::Int = 0
    slices::Int = 0
    engine::Symbol = :tcgen05
    int8_panel::Int = 256
    solve_order::Symbol = :matched
end

const _ENGINES = Dict(:tcgen05 => 0, :tcgen05_1sm => 0, :tcgen05_pair => 2, :library => 1)

function _prepare(h::MFHandle, dc::DeviceConfig)
    haskey(_ENGINES, dc.engine) ||
        throw(ArgumentError("engine must be :tcgen05, :tcgen05_1sm, :tcgen05_pair or :library"))
    dc.solve_order in (:matched, :fast) || throw(ArgumentError("solve_order must be :matched or :fast"))
    check(ccall((:mflab_set_int8_engine, libmflab), Cint, (Ptr{Cvoid}, Cint), h.ptr,
                _ENGINES[dc.engine]))
    check(ccall((:mflab_set_solve_order, libmflab), Cint, (Ptr{Cvoid}, Cint), h.ptr,
                dc.solve_order === :fast ? 1 : 0))
    return nothing
end

_scalar(::Val{N}, x) where {N} = _scalar(Val(N), MultiFloat{Float64,N}(x))
function _scalar(::Val{N}, x::MultiFloat{Float64,N}) where {N}
    v = zeros(Float64, 4)
    for l in 1:N
        v[l] = x._limbs[l]
    end
    return v
end

_same_device(xs::MFDeviceArray...) = all(x -> x.device == xs[1].device, xs) ||
    throw(ArgumentError("operands live on different devices"))

# ---------------------------------------------------------------- BLAS ----
# gemm!(C, A, B, alpha, beta; config, workspace) -- src/kernels/gemm.jl:747-774
function gemm!(C::MFDeviceMatrix{N}, A::MFDeviceMatrix{N}, B::MFDeviceMatrix{N},
               alpha::MF{N}=one(MF{N}), beta::MF{N}=zero(MF{N});
               config::KernelConfig=KernelConfig(), workspace=nothing,
               device_config::DeviceConfig=DeviceConfig(),
               handle::MFHandle=default_handle(C.device), stream::Ptr{Cvoid}=C_NULL) where {N}
    _same_device(C, A, B)
    size(A, 2) == size(B, 1) || throw(DimensionMismatch("gemm! inner dimensions differ"))
    size(C) == (size(A, 1), size(B, 2)) || throw(DimensionMismatch("gemm! output dimensions differ"))
    _prepare(handle, device_config)
    a, b = _scalar(Val(N), alpha), _scalar(Val(N), beta)
    m, k, n = size(A, 1), size(A, 2), size(B, 2)
    if device_config.int8 === :modular
        check(ccall((:mflab_gemm_ozaki_crt, libmflab), Cint,
                    (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Int64, Int64, Int64, Ptr{Float64}, Int64,
                     Int64, Ptr{Float64}, Int64, Int64, Ptr{Float64}, Int64, Int64, Ptr{Float64},
                     Ptr{Float64}),
                    handle.ptr, stream, N, device_config.moduli, m, n, k, A.ptr, A.ld, A.ls,
                    B.ptr, B.ld, B.ls, C.ptr, C.ld, C.ls, a, b))
    elseif device_config.int8 === :slices
        check(ccall((:mflab_gemm_ozaki, libmflab), Cint,
                    (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Int64, Int64, Int64, Ptr{Float64}, Int64,
                     Int64, Ptr{Float64}, Int64, Int64, Ptr{Float64}, Int64, Int64, Ptr{Float64},
                     Ptr{Float64}),
                    handle.ptr, stream, N, device_config.slices, m, n, k, A.ptr, A.ld, A.ls,
                    B.ptr, B.ld, B.ls, C.ptr, C.ld, C.ls, a, b))
    elseif device_config.int8 === :off
        s = config.gemm_strategy
        s in (:auto, :direct, :packed, :fused) ||
            throw(ArgumentError("gemm_strategy must be :auto, :direct, :packed or :fused"))
        s === :fused && N != 3 &&
            throw(ArgumentError("gemm_strategy=:fused is only available for Float64x3"))
        route = s in (:direct, :packed) ? 1 : 0   # :packed: the device stages tiles itself
        check(ccall((:mflab_gemm, libmflab), Cint,
                    (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Int64, Int64, Int64, Ptr{Float64}, Int64,
                     Int64, Ptr{Float64}, Int64, Int64, Ptr{Float64}, Int64, Int64, Ptr{Float64},
                     Ptr{Float64}),
                    handle.ptr, stream, N, route, m, n, k, A.ptr, A.ld, A.ls, B.ptr, B.ld, B.ls,
                    C.ptr, C.ld, C.ls, a, b))
    else
        throw(ArgumentError("int8 must be :off, :modular or :slices"))
    end
    return C
end

# syrk!(C, P, alpha, beta; uplo=:lower, config) -- src/kernels/syrk.jl:67-108
function syrk!(C::MFDeviceMatrix{N}, P::MFDeviceMatrix{N}, alpha::MF{N}=one(MF{N}),
               beta::MF{N}=zero(MF{N}); uplo::Symbol=:lower, config::KernelConfig=KernelConfig(),
               device_config::DeviceConfig=DeviceConfig(),
               handle::MFHandle=default_handle(C.device), stream::Ptr{Cvoid}=C_NULL) where {N}
    uplo in (:lower, :L) || throw(ArgumentError("syrk! currently supports only uplo=:lower or :L"))
    _same_device(C, P)
    n, k = size(P, 2), size(P, 1)
    size(C) == (n, n) || throw(DimensionMismatch("syrk! output dimensions differ"))
    _prepare(handle, device_config)
    a, b = _scalar(Val(N), alpha), _scalar(Val(N), beta)
    if device_config.int8 === :modular
        check(ccall((:mflab_syrk_lower_ozaki, libmflab), Cint,
                    (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Int64, Int64, Ptr{Float64}, Int64,
                     Int64, Ptr{Float64}, Int64, Int64, Ptr{Float64}, Ptr{Float64}),
                    handle.ptr, stream, N, device_config.moduli, 1, n, k, P.ptr, P.ld, P.ls,
                    C.ptr, C.ld, C.ls, a, b))
    else
        check(ccall((:mflab_syrk_lower, libmflab), Cint,
                    (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Int64, Int64, Ptr{Float64}, Int64, Int64,
                     Ptr{Float64}, Int64, Int64, Ptr{Float64}, Ptr{Float64}),
                    handle.ptr, stream, N, n, k, P.ptr, P.ld, P.ls, C.ptr, C.ld, C.ls, a, b))
    end
    return C
end

# gemmt!(C, A, B, alpha, beta; config) -- src/kernels/gemmt.jl:69-108
function gemmt!(C::MFDeviceMatrix{N}, A::MFDeviceMatrix{N}, B::MFDeviceMatrix{N},
                alpha::MF{N}=one(MF{N}), beta::MF{N}=zero(MF{N});
                config::KernelConfig=KernelConfig(),
                handle::MFHandle=default_handle(C.device), stream::Ptr{Cvoid}=C_NULL) where {N}
    _same_device(C, A, B)
    rows, k = size(A)
    size(B) == (rows, k) || throw(DimensionMismatch("gemmt! input dimensions differ"))
    size(C) == (rows, rows) || throw(DimensionMismatch("gemmt! output dimensions differ"))
    check(ccall((:mflab_gemmt_lower, libmflab), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Int64, Int64, Ptr{Float64}, Int64, Int64,
                 Ptr{Float64}, Int64, Int64, Ptr{Float64}, Int64, Int64, Ptr{Float64},
                 Ptr{Float64}),
                handle.ptr, stream, N, rows, k, A.ptr, A.ld, A.ls, B.ptr, B.ld, B.ls, C.ptr, C.ld,
                C.ls, _scalar(Val(N), alpha), _scalar(Val(N), beta)))
    return C
end

const _SIDE = Dict(:left => 0, :right => 1)
const _UPLO = Dict(:lower => 0, :upper => 1)
const _TRANS = Dict(:N => 0, :T => 1)
const _DIAG = Dict(:nonunit => 0, :unit => 1)

function _codes(side, uplo, trans, diag)
    haskey(_SIDE, side) || throw(ArgumentError("side must be :left or :right"))
    haskey(_UPLO, uplo) || throw(ArgumentError("uplo must be :lower or :upper"))
    haskey(_TRANS, trans) || throw(ArgumentError("trans must be :N or :T"))
    haskey(_DIAG, diag) || throw(ArgumentError("diag must be :unit or :nonunit"))
    return _SIDE[side], _UPLO[uplo], _TRANS[trans], _DIAG[diag]
end

# trsm!(B, A, alpha; side, uplo, trans, diag, config) -- src/kernels/trsm.jl:224-302
function trsm!(B::MFDeviceArray{N}, A::MFDeviceMatrix{N}, alpha::MF{N}=one(MF{N});
               side::Symbol=:left, uplo::Symbol=:lower, trans::Symbol=:N,
               diag::Symbol=:nonunit, config::KernelConfig=KernelConfig(),
               device_config::DeviceConfig=DeviceConfig(),
               handle::MFHandle=default_handle(B.device), stream::Ptr{Cvoid}=C_NULL) where {N}
    _same_device(B, A)
    sd, ul, tr, dg = _codes(side, uplo, trans, diag)
    size(A, 1) == size(A, 2) || throw(DimensionMismatch("trsm! requires a square triangular matrix"))
    (side === :left ? B.m : B.n) == size(A, 1) ||
        throw(DimensionMismatch("trsm! $(side) dimensions differ"))
    _prepare(handle, device_config)
    check(ccall((:mflab_trsm, libmflab), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Cint, Cint, Int64, Int64, Ptr{Float64},
                 Int64, Int64, Ptr{Float64}, Int64, Int64, Ptr{Float64}),
                handle.ptr, stream, N, sd, ul, tr, dg, B.m, B.n, A.ptr, A.ld, A.ls, B.ptr, B.ld,
                B.ls, _scalar(Val(N), alpha)))
    return B
end

# trsv!(x, A, alpha; uplo, trans, diag, config) -- src/kernels/trsv.jl:19-73 (the
# single-column solve keeps trsm!'s per-row ascending chains)
function trsv!(x::MFDeviceVector{N}, A::MFDeviceMatrix{N}, alpha::MF{N}=one(MF{N});
               uplo::Symbol=:lower, trans::Symbol=:N, diag::Symbol=:nonunit,
               config::KernelConfig=KernelConfig(), device_config::DeviceConfig=DeviceConfig(),
               handle::MFHandle=default_handle(x.device), stream::Ptr{Cvoid}=C_NULL) where {N}
    size(A, 1) == size(A, 2) || throw(DimensionMismatch("trsv! requires a square triangular matrix"))
    length(x) == size(A, 1) || throw(DimensionMismatch("trsv! right-hand side length differs"))
    return trsm!(x, A, alpha; side=:left, uplo=uplo, trans=trans, diag=diag, config=config,
                 device_config=device_config, handle=handle, stream=stream)
end

# trmm!(B, A, alpha; side, uplo, trans, diag) -- src/kernels/trmm.jl:82-131
function trmm!(B::MFDeviceMatrix{N}, A::MFDeviceMatrix{N}, alpha::MF{N}=one(MF{N});
               side::Symbol=:left, uplo::Symbol=:lower, trans::Symbol=:N,
               diag::Symbol=:nonunit, config::KernelConfig=KernelConfig(),
               handle::MFHandle=default_handle(B.device), stream::Ptr{Cvoid}=C_NULL) where {N}
    sd, ul, tr, dg = _codes(side, uplo, trans, diag)
    size(A, 1) == size(A, 2) || throw(DimensionMismatch("trmm! requires a square triangular matrix"))
    (side === :left ? B.m : B.n) == size(A, 1) ||
        throw(DimensionMismatch("trmm! $(side) dimensions differ"))
    check(ccall((:mflab_trmm, libmflab), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Cint, Cint, Int64, Int64, Ptr{Float64},
                 Int64, Int64, Ptr{Float64}, Int64, Int64, Ptr{Float64}),
                handle.ptr, stream, N, sd, ul, tr, dg, B.m, B.n, A.ptr, A.ld, A.ls, B.ptr, B.ld,
                B.ls, _scalar(Val(N), alpha)))
    return B
end

# gemv!(y, A, x, alpha, beta; trans) -- src/kernels/gemv.jl:99-167
function gemv!(y::MFDeviceVector{N}, A::MFDeviceMatrix{N}, x::MFDeviceVector{N},
               alpha::MF{N}=one(MF{N}), beta::MF{N}=zero(MF{N}); trans::Symbol=:N,
               config::KernelConfig=KernelConfig(),
               handle::MFHandle=default_handle(y.device), stream::Ptr{Cvoid}=C_NULL) where {N}
    trans in (:N, :T) || throw(ArgumentError("trans must be :N or :T"))
    m, n = size(A)
    length(x) == (trans === :N ? n : m) || throw(DimensionMismatch("gemv! input length differs"))
    length(y) == (trans === :N ? m : n) || throw(DimensionMismatch("gemv! output length differs"))
    check(ccall((:mflab_gemv, libmflab), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Int64, Int64, Ptr{Float64}, Int64, Int64,
                 Ptr{Float64}, Int64, Ptr{Float64}, Int64, Ptr{Float64}, Ptr{Float64}),
                handle.ptr, stream, N, trans === :T ? 1 : 0, m, n, A.ptr, A.ld, A.ls, x.ptr, x.ls,
                y.ptr, y.ls, _scalar(Val(N), alpha), _scalar(Val(N), beta)))
    return y
end

# symv!(y, A, x, alpha, beta; uplo) -- src/kernels/symv.jl:43-89
function symv!(y::MFDeviceVector{N}, A::MFDeviceMatrix{N}, x::MFDeviceVector{N},
               alpha::MF{N}=one(MF{N}), beta::MF{N}=zero(MF{N}); uplo::Symbol=:lower,
               config::KernelConfig=KernelConfig(),
               handle::MFHandle=default_handle(y.device), stream::Ptr{Cvoid}=C_NULL) where {N}
    uplo in (:lower, :upper) || throw(ArgumentError("uplo must be :lower or :upper"))
    n = size(A, 1)
    size(A, 2) == n || throw(DimensionMismatch("symv! requires a square matrix"))
    length(x) == n && length(y) == n || throw(DimensionMismatch("symv! vector lengths differ"))
    check(ccall((:mflab_symv, libmflab), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Int64, Ptr{Float64}, Int64, Int64,
                 Ptr{Float64}, Int64, Ptr{Float64}, Int64, Ptr{Float64}, Ptr{Float64}),
                handle.ptr, stream, N, uplo === :upper ? 1 : 0, n, A.ptr, A.ld, A.ls, x.ptr, x.ls,
                y.ptr, y.ls, _scalar(Val(N), alpha), _scalar(Val(N), beta)))
    return y
end

# mfdot(x, y) -- src/kernels/dot.jl:1-22: one ascending chain over the
# column-major index
function mfdot(x::MFDeviceArray{N}, y::MFDeviceArray{N};
               handle::MFHandle=default_handle(x.device), stream::Ptr{Cvoid}=C_NULL) where {N}
    (x.m, x.n) == (y.m, y.n) || throw(DimensionMismatch("dot product shapes differ"))
    out = DeviceWords{Float64}(N, x.device)
    check(ccall((:mflab_dot, libmflab), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Int64, Int64, Ptr{Float64}, Int64, Int64,
                 Ptr{Float64}, Int64, Int64, Ptr{Float64}),
                handle.ptr, stream, N, x.m, x.n, x.ptr, x.ld, x.ls, y.ptr, y.ld, y.ls, out.ptr))
    v = host(out, stream)
    return MultiFloat{Float64,N}(ntuple(l -> v[l], N))
end

# ------------------------------------------------------ factorizations ----
_info(w::DeviceWords{Cint}, stream) = Int(host(w, stream)[1])

# cholesky!(A; check, config) -- src/factorizations/cholesky.jl:68-107
function cholesky!(A::MFDeviceMatrix{N}; check::Bool=true, config::KernelConfig=KernelConfig(),
                   device_config::DeviceConfig=DeviceConfig(),
                   handle::MFHandle=default_handle(A.device), stream::Ptr{Cvoid}=C_NULL) where {N}
    size(A, 1) == size(A, 2) || throw(DimensionMismatch("cholesky! requires a square matrix"))
    info = DeviceWords{Cint}(1, A.device)
    block = max(config.cholesky_block, 1)
    _prepare(handle, device_config)
    if device_config.int8 === :modular
        MFLAB200.check(ccall((:mflab_potrf_ozaki, libmflab), Cint,
                             (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Int64, Ptr{Float64}, Int64, Int64,
                              Int64, Int64, Ptr{Cint}),
                             handle.ptr, stream, N, device_config.moduli, A.m, A.ptr, A.ld, A.ls,
                             max(device_config.int8_panel, block), block, info.ptr))
    else
        MFLAB200.check(ccall((:mflab_potrf, libmflab), Cint,
                             (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Int64, Ptr{Float64}, Int64, Int64,
                              Int64, Ptr{Cint}),
                             handle.ptr, stream, N, A.m, A.ptr, A.ld, A.ls, block, info.ptr))
    end
    st = _info(info, stream)
    st == -1 && check && throw(DomainError(A, "cholesky!: input matrix contains non-finite entries"))
    st > 0 && check && throw(LinearAlgebra.PosDefException(st))
    return MFCholesky(A, st)
end

function _max_abs(A::MFDeviceMatrix{N}, region::Integer, handle, stream) where {N}
    out = DeviceWords{Float64}(N + 1, A.device)
    A.m > 0 && A.n > 0 &&
        check(ccall((:mflab_max_abs, libmflab), Cint,
                    (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Int64, Int64, Ptr{Float64}, Int64, Int64, Cint,
                     Ptr{Float64}),
                    handle.ptr, stream, N, A.m, A.n, A.ptr, A.ld, A.ls, region, out.ptr))
    v = host(out, stream)
    return MultiFloat{Float64,N}(ntuple(l -> v[l], N))
end

# lu!(A; check, config, workspace) -- src/factorizations/lu.jl:128-195
function lu!(A::MFDeviceMatrix{N}; check::Bool=true, config::KernelConfig=KernelConfig(),
             workspace=nothing, device_config::DeviceConfig=DeviceConfig(),
             handle::MFHandle=default_handle(A.device), stream::Ptr{Cvoid}=C_NULL) where {N}
    m, n = size(A)
    kmax = min(m, n)
    omax = _max_abs(A, 0, handle, stream)
    info = DeviceWords{Cint}(1, A.device)
    ipiv = DeviceWords(collect(Int64, 1:kmax), A.device)
    block = max(config.lu_block, 1)
    _prepare(handle, device_config)
    if device_config.int8 === :modular
        MFLAB200.check(ccall((:mflab_getrf_ozaki, libmflab), Cint,
                             (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Int64, Int64, Ptr{Float64}, Int64,
                              Int64, Ptr{Int64}, Int64, Int64, Ptr{Cint}),
                             handle.ptr, stream, N, device_config.moduli, m, n, A.ptr, A.ld, A.ls,
                             kmax > 0 ? ipiv.ptr : Ptr{Int64}(C_NULL),
                             max(device_config.int8_panel, block), block, info.ptr))
    else
        MFLAB200.check(ccall((:mflab_getrf, libmflab), Cint,
                             (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Int64, Int64, Ptr{Float64}, Int64,
                              Int64, Ptr{Int64}, Int64, Ptr{Cint}),
                             handle.ptr, stream, N, m, n, A.ptr, A.ld, A.ls,
                             kmax > 0 ? ipiv.ptr : Ptr{Int64}(C_NULL), block, info.ptr))
    end
    st = _info(info, stream)
    st == -1 && check && throw(DomainError(A, "lu!: input matrix contains non-finite entries"))
    st > 0 && check && throw(LinearAlgebra.SingularException(st))
    return MFLU(A, Vector{Int}(host(ipiv, stream)), st, st == -1 ? zero(MF{N}) : omax)
end

const _LDLT_BLOCK = Dict(2 => 16, 3 => 12, 4 => 8)  # src/factorizations/ldlt_tuning.jl:9-15

# ldlt!(A; check, config, workspace) -- src/factorizations/ldlt.jl:654-717
function ldlt!(A::MFDeviceMatrix{N}; check::Bool=true, config::KernelConfig=KernelConfig(),
               workspace=nothing,
               handle::MFHandle=default_handle(A.device), stream::Ptr{Cvoid}=C_NULL) where {N}
    n = size(A, 1)
    size(A, 2) == n || throw(DimensionMismatch("ldlt! requires a square matrix"))
    strategy = config.ldlt_strategy
    strategy in (:auto, :unblocked, :blocked) ||
        throw(ArgumentError("ldlt_strategy must be :auto, :unblocked, or :blocked"))
    block = config.ldlt_block > 0 ? config.ldlt_block : _LDLT_BLOCK[N]
    blocked = strategy === :blocked ||
              (strategy === :auto && block > 1 && n >= max(config.ldlt_blocked_crossover, 1))
    blocked && (block = max(block, 2))
    omax = _max_abs(A, 1, handle, stream)
    dsub = zeros(MFDeviceArray{N,1}, n; device=A.device)
    pivots = DeviceWords(collect(Int64, 1:n), A.device)
    blocks = DeviceWords{UInt8}(n, A.device)
    info = DeviceWords{Cint}(1, A.device)
    MFLAB200.check(ccall((:mflab_sytrf, libmflab), Cint,
                         (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Int64, Ptr{Float64}, Int64, Int64,
                          Ptr{Float64}, Int64, Ptr{Int64}, Ptr{UInt8}, Cint, Int64, Ptr{Cint}),
                         handle.ptr, stream, N, n, A.ptr, A.ld, A.ls, dsub.ptr, dsub.ls,
                         n > 0 ? pivots.ptr : Ptr{Int64}(C_NULL), blocks.ptr, blocked ? 1 : 0,
                         blocked ? block : 1, info.ptr))
    st = _info(info, stream)
    st == -1 && check && throw(DomainError(A, "ldlt!: input matrix contains non-finite entries"))
    st > 0 && check && throw(LinearAlgebra.SingularException(st))
    return MFLDLT(A, dsub, Vector{Int}(host(pivots, stream)), host(blocks, stream), st,
                  st == -1 ? zero(MF{N}) : omax)
end

# ldiv!(x, F; config) -- src/solve.jl:23-365: vector and matrix right-hand
# sides take the same device solves (trsv! keeps trsm!'s order)
function ldiv!(X::MFDeviceArray{N}, F::MFCholesky{MF{N},MFDeviceMatrix{N}};
               config::KernelConfig=KernelConfig(), device_config::DeviceConfig=DeviceConfig(),
               handle::MFHandle=default_handle(X.device), stream::Ptr{Cvoid}=C_NULL) where {N}
    MultiFloatLinearAlgebra.issuccess(F) || throw(LinearAlgebra.PosDefException(F.info))
    L = F.factors
    X.m == size(L, 1) || throw(DimensionMismatch("right-hand side dimensions differ"))
    _prepare(handle, device_config)
    check(ccall((:mflab_potrs, libmflab), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Int64, Int64, Ptr{Float64}, Int64, Int64,
                 Ptr{Float64}, Int64, Int64),
                handle.ptr, stream, N, L.m, X.n, L.ptr, L.ld, L.ls, X.ptr, X.ld, X.ls))
    return X
end

function ldiv!(X::MFDeviceArray{N}, F::MFLU{MF{N},MFDeviceMatrix{N}};
               config::KernelConfig=KernelConfig(), device_config::DeviceConfig=DeviceConfig(),
               handle::MFHandle=default_handle(X.device), stream::Ptr{Cvoid}=C_NULL) where {N}
    MultiFloatLinearAlgebra.issuccess(F) || throw(LinearAlgebra.SingularException(F.info))
    LU = F.factors
    size(LU, 1) == size(LU, 2) || throw(DimensionMismatch("solve requires a square LU factor"))
    X.m == size(LU, 1) || throw(DimensionMismatch("right-hand side dimensions differ"))
    ipiv = DeviceWords(Vector{Int64}(F.ipiv), X.device)
    _prepare(handle, device_config)
    check(ccall((:mflab_getrs, libmflab), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Int64, Int64, Ptr{Float64}, Int64, Int64,
                 Ptr{Int64}, Ptr{Float64}, Int64, Int64),
                handle.ptr, stream, N, LU.m, X.n, LU.ptr, LU.ld, LU.ls, ipiv.ptr, X.ptr, X.ld,
                X.ls))
    return X
end

function ldiv!(X::MFDeviceArray{N}, F::MFLDLT{MF{N},MFDeviceMatrix{N}};
               config::KernelConfig=KernelConfig(), device_config::DeviceConfig=DeviceConfig(),
               handle::MFHandle=default_handle(X.device), stream::Ptr{Cvoid}=C_NULL) where {N}
    MultiFloatLinearAlgebra.issuccess(F) || throw(LinearAlgebra.SingularException(F.info))
    A = F.factors
    X.m == size(A, 1) || throw(DimensionMismatch("right-hand side dimensions differ"))
    pivots = DeviceWords(Vector{Int64}(F.pivots), X.device)
    blocks = DeviceWords(Vector{UInt8}(F.blocks), X.device)
    fail = DeviceWords{Cint}(1, X.device)
    _prepare(handle, device_config)
    check(ccall((:mflab_sytrs, libmflab), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Int64, Int64, Ptr{Float64}, Int64, Int64,
                 Ptr{Float64}, Int64, Ptr{Int64}, Ptr{UInt8}, Ptr{Float64}, Int64, Int64,
                 Ptr{Cint}),
                handle.ptr, stream, N, A.m, X.n, A.ptr, A.ld, A.ls, F.dsub.ptr, F.dsub.ls,
                pivots.ptr, blocks.ptr, X.ptr, X.ld, X.ls, fail.ptr))
    f = _info(fail, stream)
    0 < f < 0x7F7F7F7F && throw(LinearAlgebra.SingularException(f))
    return X
end

# solve(F, rhs; config) -- src/solve.jl:555-565: non-mutating
solve(F::Union{MFCholesky{MF{N},MFDeviceMatrix{N}},MFLU{MF{N},MFDeviceMatrix{N}},
               MFLDLT{MF{N},MFDeviceMatrix{N}}}, rhs::MFDeviceArray{N}; kwargs...) where {N} =
    ldiv!(copy(rhs), F; kwargs...)

# cholesky_pivoted!(A; tol, check) -- src/factorizations/cholesky_pivoted.jl:65-175
function cholesky_pivoted!(A::MFDeviceMatrix{N}; tol=zero(MF{N}), check::Bool=true,
                           config::KernelConfig=KernelConfig(),
                           handle::MFHandle=default_handle(A.device),
                           stream::Ptr{Cvoid}=C_NULL) where {N}
    n = size(A, 1)
    size(A, 2) == n || throw(DimensionMismatch("cholesky_pivoted! requires a square matrix"))
    perm = DeviceWords{Int64}(n, A.device)
    rank_info = DeviceWords{Int64}(2, A.device)
    MFLAB200.check(ccall((:mflab_pstrf, libmflab), Cint,
                         (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Int64, Ptr{Float64}, Int64, Int64,
                          Ptr{Float64}, Ptr{Int64}, Ptr{Int64}),
                         handle.ptr, stream, N, n, A.ptr, A.ld, A.ls, _scalar(Val(N), tol),
                         perm.ptr, rank_info.ptr))
    rank, st = host(rank_info, stream)
    st == -1 && check &&
        throw(DomainError(A, "cholesky_pivoted!: input matrix contains non-finite entries"))
    st > 0 && check && throw(LinearAlgebra.PosDefException(Int(st)))
    return MFCholeskyPivoted(A, Vector{Int}(host(perm, stream)), Int(rank), Int(st))
end

# qr!(A) / rrqr!(A) -- src/factorizations/qr.jl:692-811
function _qr(A::MFDeviceMatrix{N}, pivoted::Integer, check::Bool, what::String, handle,
             stream) where {N}
    m, n = size(A)
    r = min(m, n)
    tau = zeros(MFDeviceArray{N,1}, max(r, 1); device=A.device)
    perm = DeviceWords{Int64}(n, A.device)
    info = DeviceWords{Cint}(1, A.device)
    MFLAB200.check(ccall((:mflab_qr, libmflab), Cint,
                         (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Int64, Int64, Ptr{Float64}, Int64,
                          Int64, Ptr{Float64}, Int64, Ptr{Int64}, Ptr{Cint}),
                         handle.ptr, stream, N, pivoted, m, n, A.ptr, A.ld, A.ls, tau.ptr, tau.ls,
                         perm.ptr, info.ptr))
    st = _info(info, stream)
    st == -1 && check && throw(DomainError(A, "$(what): input matrix contains non-finite entries"))
    p = Vector{Int}(host(perm, stream))
    leaders = MultiFloatLinearAlgebra._qr_permutation_cycle_leaders!(copy(p))
    return MFQR(A, tau, p, leaders, st)
end
rrqr!(A::MFDeviceMatrix; check::Bool=true, config::KernelConfig=KernelConfig(),
      handle::MFHandle=default_handle(A.device), stream::Ptr{Cvoid}=C_NULL) =
    _qr(A, 1, check, "rrqr!", handle, stream)
qr!(A::MFDeviceMatrix; check::Bool=true, config::KernelConfig=KernelConfig(),
    handle::MFHandle=default_handle(A.device), stream::Ptr{Cvoid}=C_NULL) =
    _qr(A, 0, check, "qr!", handle, stream)

# apply_q!(B, F; trans) -- src/factorizations/qr.jl:938-956
function apply_q!(B::MFDeviceMatrix{N}, F::MFQR; trans::Symbol=:N,
                  handle::MFHandle=default_handle(B.device), stream::Ptr{Cvoid}=C_NULL) where {N}
    trans in (:N, :T) || throw(ArgumentError("trans must be :N or :T"))
    Fm = F.factors
    B.m == size(Fm, 1) || throw(DimensionMismatch("apply_q! destination row count differs"))
    check(ccall((:mflab_apply_q, libmflab), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Int64, Int64, Ptr{Float64}, Int64, Int64,
                 Ptr{Float64}, Int64, Ptr{Float64}, Int64, Int64, Int64),
                handle.ptr, stream, N, trans === :T ? 1 : 0, Fm.m, min(Fm.m, Fm.n), Fm.ptr, Fm.ld,
                Fm.ls, F.tau.ptr, F.tau.ls, B.ptr, B.ld, B.ls, B.n))
    return B
end

# ---------------------------------------------------------- residuals ----
const _RUPLO = Dict(:general => 0, :lower => 1, :upper => 2)

# residual!(R, A, X, B; uplo) -- src/residual.jl:55-125
function residual!(R::MFDeviceArray{N}, A::MFDeviceMatrix{N}, X::MFDeviceArray{N},
                   B::MFDeviceArray{N}; uplo::Symbol=:general, config::KernelConfig=KernelConfig(),
                   workspace=nothing, handle::MFHandle=default_handle(R.device),
                   stream::Ptr{Cvoid}=C_NULL) where {N}
    haskey(_RUPLO, uplo) || throw(ArgumentError("uplo must be :general, :lower, or :upper"))
    (R.m, R.n) == (B.m, B.n) && R.m == size(A, 1) && X.m == size(A, 2) && X.n == R.n ||
        throw(DimensionMismatch("residual dimensions differ"))
    check(ccall((:mflab_residual, libmflab), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Int64, Int64, Int64, Ptr{Float64},
                 Int64, Int64, Ptr{Float64}, Int64, Int64, Ptr{Float64}, Int64, Int64,
                 Ptr{Float64}, Int64, Int64),
                handle.ptr, stream, N, _RUPLO[uplo], ndims(R) == 1 ? 1 : 0, A.m, A.n, R.n,
                A.ptr, A.ld, A.ls, X.ptr, X.ld, X.ls, B.ptr, B.ld, B.ls, R.ptr, R.ld, R.ls))
    return R
end

# residual_mixed!(R, A, X, B; uplo) -- src/residual.jl:431-496 (R has more limbs)
function residual_mixed!(R::MFDeviceArray{M}, A::MFDeviceMatrix{N}, X::MFDeviceArray{N},
                         B::MFDeviceArray{N}; uplo::Symbol=:general,
                         config::KernelConfig=KernelConfig(),
                         handle::MFHandle=default_handle(R.device),
                         stream::Ptr{Cvoid}=C_NULL) where {M,N}
    haskey(_RUPLO, uplo) || throw(ArgumentError("uplo must be :general, :lower, or :upper"))
    1 <= N < M <= 4 ||
        throw(ArgumentError("residual_mixed! supports only widening to a higher limb count"))
    check(ccall((:mflab_residual_mixed, libmflab), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Int64, Int64, Int64, Ptr{Float64},
                 Int64, Int64, Ptr{Float64}, Int64, Int64, Ptr{Float64}, Int64, Int64,
                 Ptr{Float64}, Int64, Int64),
                handle.ptr, stream, N, M, _RUPLO[uplo], A.m, A.n, R.n, A.ptr, A.ld, A.ls, X.ptr,
                X.ld, X.ls, B.ptr, B.ld, B.ls, R.ptr, R.ld, R.ls))
    return R
end

# normwise_backward_error(A, X, B, R; uplo) -- src/residual.jl:202-269
function normwise_backward_error(A::MFDeviceMatrix{N}, X::MFDeviceArray{N}, B::MFDeviceArray{N},
                                 R::MFDeviceArray{N}; uplo::Symbol=:general,
                                 handle::MFHandle=default_handle(A.device),
                                 stream::Ptr{Cvoid}=C_NULL) where {N}
    haskey(_RUPLO, uplo) || throw(ArgumentError("uplo must be :general, :lower, or :upper"))
    out = DeviceWords{Float64}(max(R.n, 1) * N, A.device)
    check(ccall((:mflab_backward_error, libmflab), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Int64, Int64, Int64, Ptr{Float64}, Int64,
                 Int64, Ptr{Float64}, Int64, Int64, Ptr{Float64}, Int64, Int64, Ptr{Float64},
                 Int64, Int64, Ptr{Float64}),
                handle.ptr, stream, N, _RUPLO[uplo], A.m, A.n, R.n, A.ptr, A.ld, A.ls, X.ptr,
                X.ld, X.ls, B.ptr, B.ld, B.ls, R.ptr, R.ld, R.ls, out.ptr))
    v = host(out, stream)
    vals = [MultiFloat{Float64,N}(ntuple(l -> v[(j - 1) * N + l], N)) for j in 1:R.n]
    return ndims(R) == 1 ? vals[1] : vals
end

# ------------------------------------------------------------- status ----
"""0, or the code of a tcgen05 kernel's bounded wait that ran out on this
handle (1 producer, 2 MMA issuer, 3 epilogue, 4 drain); reading resets it."""
function device_status(handle::MFHandle=default_handle())
    v = Ref{Cint}(0)
    check(ccall((:mflab_device_status, libmflab), Cint, (Ptr{Cvoid}, Ptr{Cint}), handle.ptr, v))
    return Int(v[])
end

# ---------------------------------------------- mixed-precision solve ----
"""
    solve_mixed_lu(A, B; tol=2^(-53N), maxiter=40)

A X = B for a Float64xN device matrix A: a binary64 partial-pivoting LU of
round(A) on the device, its solve workspace prepared once (mflab_lu64_prepare:
permutation, inverted diagonal blocks, premultiplied block columns), then
iterative refinement with Float64xN residuals through the INT8 modular GEMM;
A's residues are prepared once (mflab_ozaki_crt_prepare) at the modulus count
the tuner picks for A and the first iterate (mflab_ozaki_crt_tune).  No reference counterpart: it composes lu!,
residual! and refinement_correction!.  Returns (X, iterations, worst backward
error)."""
function solve_mixed_lu(A::MFDeviceMatrix{N}, B::MFDeviceMatrix{N};
                        tol::Float64=2.0^(-53N), maxiter::Int=40,
                        handle::MFHandle=default_handle(A.device),
                        stream::Ptr{Cvoid}=C_NULL) where {N}
    n = size(A, 1)
    size(A, 2) == n || throw(DimensionMismatch("solve requires a square matrix"))
    B.m == n || throw(DimensionMismatch("right-hand side dimensions differ"))
    LU = MFDeviceArray{1,2}(undef, n, n; device=A.device)
    for c in 0:n-1   # LU = round(A): the leading limbs
        memcpy!(LU.ptr + 8 * c * LU.ld, A.ptr + 8 * c * A.ld, 8 * n, 2)
    end
    ipiv = DeviceWords(collect(Int64, 1:n), A.device)
    info = DeviceWords{Cint}(1, A.device)
    check(ccall((:mflab_getrf, libmflab), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Int64, Int64, Ptr{Float64}, Int64, Int64,
                 Ptr{Int64}, Int64, Ptr{Cint}),
                handle.ptr, stream, 1, n, n, LU.ptr, LU.ld, LU.ls, ipiv.ptr, 32, info.ptr))
    st = _info(info, stream)
    st == -1 && throw(DomainError(A, "lu!: input matrix contains non-finite entries"))
    st > 0 && throw(LinearAlgebra.SingularException(st))
    wb = Ref{Csize_t}(0)
    check(ccall((:mflab_lu64_work_bytes, libmflab), Cint, (Int64, Ptr{Csize_t}), n, wb))
    work = DeviceBuffer(max(Int(wb[]), 1), A.device)
    check(ccall((:mflab_lu64_prepare, libmflab), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Int64, Ptr{Int64}, Ptr{Cvoid}),
                handle.ptr, stream, n, LU.ptr, LU.ld, ipiv.ptr, work.ptr))
    X = zeros(MFDeviceArray{N,2}, n, B.n; device=A.device)
    R = copy(B)
    D = MFDeviceArray{1,2}(undef, n, B.n; device=A.device)
    # ||A||_inf once (mflab_opnorm_inf), for every iteration's backward error
    anorm = DeviceWords{Float64}(N, A.device)
    anf = DeviceWords{Cint}(1, A.device)
    check(ccall((:mflab_opnorm_inf, libmflab), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Int64, Int64, Ptr{Float64}, Int64, Int64,
                 Ptr{Float64}, Ptr{Cint}),
                handle.ptr, stream, N, 0, n, n, A.ptr, A.ld, A.ls, anorm.ptr, anf.ptr))
    berr = DeviceWords{Float64}(max(B.n, 1) * N, A.device)
    one_, mone = _scalar(Val(N), one(MF{N})), _scalar(Val(N), -one(MF{N}))
    prep, T = nothing, 0
    worst, it = Inf, 0
    for outer it in 1:maxiter
        for c in 0:B.n-1    # D = round(R): the leading limbs
            memcpy!(D.ptr + 8 * c * D.ld, R.ptr + 8 * c * R.ld, 8 * n, 2)
        end
        check(ccall((:mflab_lu64_solve, libmflab), Cint,
                    (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Int64, Ptr{Float64}, Int64, Ptr{Cvoid},
                     Ptr{Float64}, Int64),
                    handle.ptr, stream, n, B.n, LU.ptr, LU.ld, work.ptr, D.ptr, D.ld))
        check(ccall((:mflab_add_widened, libmflab), Cint,
                    (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Int64, Int64, Ptr{Float64}, Int64, Int64,
                     Ptr{Float64}, Int64, Int64),
                    handle.ptr, stream, 1, N, n, B.n, D.ptr, D.ld, D.ls, X.ptr, X.ld, X.ls))
        for l in 0:N-1, c in 0:B.n-1   # R = B
            memcpy!(R.ptr + 8 * (l * R.ls + c * R.ld), B.ptr + 8 * (l * B.ls + c * B.ld), 8 * n, 2)
        end
        if prep === nothing
            # the modulus count the tuner picks for A and the first iterate;
            # A's residues are then prepared once for every residual
            Tr = Ref{Cint}(0)
            check(ccall((:mflab_ozaki_crt_tune, libmflab), Cint,
                        (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Int64, Int64, Int64, Ptr{Float64}, Int64,
                         Int64, Ptr{Float64}, Int64, Int64, Ptr{Cint}),
                        handle.ptr, stream, N, n, B.n, n, A.ptr, A.ld, A.ls, X.ptr, X.ld, X.ls,
                        Tr))
            T = Int(Tr[])
            pb = Ref{Csize_t}(0)
            check(ccall((:mflab_ozaki_crt_prepare_bytes, libmflab), Cint,
                        (Cint, Cint, Int64, Int64, Ptr{Csize_t}), N, T, n, n, pb))
            prep = DeviceBuffer(max(Int(pb[]), 1), A.device)
            check(ccall((:mflab_ozaki_crt_prepare, libmflab), Cint,
                        (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Int64, Int64, Ptr{Float64}, Int64,
                         Int64, Ptr{Cvoid}),
                        handle.ptr, stream, N, T, n, n, A.ptr, A.ld, A.ls, prep.ptr))
        end
        check(ccall((:mflab_gemm_ozaki_crt_prepared, libmflab), Cint,
                    (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Int64, Int64, Int64, Ptr{Cvoid},
                     Ptr{Float64}, Int64, Int64, Ptr{Float64}, Int64, Int64, Ptr{Float64},
                     Ptr{Float64}),
                    handle.ptr, stream, N, T, n, B.n, n, prep.ptr, X.ptr, X.ld, X.ls, R.ptr,
                    R.ld, R.ls, mone, one_))
        check(ccall((:mflab_backward_error_norm, libmflab), Cint,
                    (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Int64, Int64, Int64, Ptr{Float64}, Ptr{Cint},
                     Ptr{Float64}, Int64, Int64, Ptr{Float64}, Int64, Int64, Ptr{Float64}, Int64,
                     Int64, Ptr{Float64}),
                    handle.ptr, stream, N, n, n, B.n, anorm.ptr, anf.ptr, X.ptr, X.ld, X.ls,
                    B.ptr, B.ld, B.ls, R.ptr, R.ld, R.ls, berr.ptr))
        v = host(berr, stream)
        worst = maximum(Float64(MultiFloat{Float64,N}(ntuple(l -> v[(j - 1) * N + l], N)))
                        for j in 1:B.n)
        worst <= tol && break
    end
    return X, it, worst
end

end # module
