// Interleaved Float64xN storage <-> limb planes.
//
// A Julia Matrix{MultiFloat{Float64,N}} (the reference's operand type,
// src/kernels/gemm.jl:747-755) stores the N limbs of each element next to
// each other: limb l of element (r, c) at X[(c*ldx + r)*N + l].  The device
// kernels of this library read N separate column-major planes instead.  The
// conversion is a pure permutation of doubles (no arithmetic), so it is
// bit-exact and HBM-bound: one read and one write of 8 N bytes per element.
//
// Host <-> device forms stage the host block through two 32 MiB halves of a
// handle-owned buffer (chunks of whole columns, or of rows of one column
// when a column is larger): the copy engine moves chunk j
// (cudaMemcpy2DAsync, which also takes the host leading dimension) into
// half j mod 2 and a permutation kernel turns it into planes (or planes into
// the chunk before it leaves).  The call is ordered on the caller's stream;
// the staging is why concurrent callers need their own handles.
#include <algorithm>
#include <cstdint>

#include "mflab_internal.h"

MFLAB_DEBUG_RECORD(interleave)

namespace mfl {

namespace {

constexpr int IL_THREADS = 256;
// bytes per staging half: the transfer's size, between 32 MiB and 1 GiB, so
// a matrix of up to 1 GiB moves in one copy that never waits for a kernel
constexpr size_t IL_STAGE_MIN = size_t(32) << 20, IL_STAGE_MAX = size_t(1) << 30;

// dst planes <- src interleaved (to_planes = true), or the reverse.  One
// thread per element: the N limbs of an element are contiguous in the
// interleaved form (a 16-byte load / store for N = 2 and two for N = 4 when
// aligned), and consecutive threads touch consecutive rows of each plane,
// so both sides are coalesced.
template <int N, bool TO_PLANES, bool VEC>
__global__ void __launch_bounds__(IL_THREADS)
    interleave_kernel(int64_t m, int64_t n, double *__restrict__ X, int64_t ldx,
                      double *__restrict__ P, int64_t ld, int64_t ls) {
    const int64_t r = (int64_t)blockIdx.x * IL_THREADS + threadIdx.x;
    if (r >= m) return;
    // debug builds: the strides hold the rows (ldx, ld >= m) and the planes
    if (!MFLAB_IDX_OK(ldx >= m && ld >= m && (N == 1 || ls >= ld * (n - 1) + m), 8, ld, ls))
        return;
    for (int64_t c = blockIdx.y; c < n; c += gridDim.y) {
        double *x = X + (c * ldx + r) * N;
        double *p = P + c * ld + r;
        if constexpr (TO_PLANES) {
            double v[N];
            if constexpr (VEC) {
#pragma unroll
                for (int l = 0; l < N; l += 2) {
                    const double2 t = *reinterpret_cast<const double2 *>(x + l);
                    v[l] = t.x;
                    v[l + 1] = t.y;
                }
            } else {
#pragma unroll
                for (int l = 0; l < N; ++l) v[l] = x[l];
            }
#pragma unroll
            for (int l = 0; l < N; ++l) p[l * ls] = v[l];
        } else {
            double v[N];
#pragma unroll
            for (int l = 0; l < N; ++l) v[l] = p[l * ls];
            if constexpr (VEC) {
#pragma unroll
                for (int l = 0; l < N; l += 2)
                    *reinterpret_cast<double2 *>(x + l) = make_double2(v[l], v[l + 1]);
            } else {
#pragma unroll
                for (int l = 0; l < N; ++l) x[l] = v[l];
            }
        }
    }
}

template <int N, bool TO_PLANES>
int launch_n(int64_t m, int64_t n, double *X, int64_t ldx, double *P, int64_t ld, int64_t ls,
             cudaStream_t s) {
    const dim3 grid((unsigned)((m + IL_THREADS - 1) / IL_THREADS),
                    (unsigned)std::min<int64_t>(n, 32768));
    // 16-byte vector access needs an even limb count and a 16-byte aligned base
    const bool vec = (N % 2 == 0) && ((reinterpret_cast<uintptr_t>(X) & 15) == 0);
    if (vec)
        interleave_kernel<N, TO_PLANES, (N % 2 == 0)><<<grid, IL_THREADS, 0, s>>>(m, n, X, ldx, P,
                                                                                ld, ls);
    else
        interleave_kernel<N, TO_PLANES, false><<<grid, IL_THREADS, 0, s>>>(m, n, X, ldx, P, ld, ls);
    return record_cuda_error(cudaGetLastError(), "interleave kernel");
}

template <bool TO_PLANES>
int launch(int N, int64_t m, int64_t n, double *X, int64_t ldx, double *P, int64_t ld, int64_t ls,
           cudaStream_t s) {
    switch (N) {
    case 1: return launch_n<1, TO_PLANES>(m, n, X, ldx, P, ld, ls, s);
    case 2: return launch_n<2, TO_PLANES>(m, n, X, ldx, P, ld, ls, s);
    case 3: return launch_n<3, TO_PLANES>(m, n, X, ldx, P, ld, ls, s);
    case 4: return launch_n<4, TO_PLANES>(m, n, X, ldx, P, ld, ls, s);
    }
    return MFLAB_ERR_UNSUPPORTED;
}

// common argument checks; returns MFLAB_OK when there is work to do, or a
// code (MFLAB_OK with *empty = true for an empty matrix)
int check_args(mflab_handle *h, int limbs, int64_t m, int64_t n, const void *X, int64_t ldx,
               const void *P, int64_t ld, int64_t ls, bool *empty) {
    *empty = false;
    if (!h || limbs < 1 || limbs > 4) return MFLAB_ERR_UNSUPPORTED;
    if (m < 0 || n < 0) return MFLAB_ERR_ARG;
    if (m == 0 || n == 0) {
        *empty = true;
        return MFLAB_OK;
    }
    // planes must not overlap one another
    if (!X || !P || ldx < m || ld < m || (limbs > 1 && ls < ld * (n - 1) + m))
        return MFLAB_ERR_ARG;
    return MFLAB_OK;
}

// the staging buffer (two halves of at least `bytes`, within the bounds
// above), two non-blocking streams of the highest priority and their events,
// created on the first host <-> device conversion; a larger transfer later
// regrows the halves once the streams are idle
int reserve_stage(mflab_handle *h, size_t bytes) {
    size_t want = bytes < IL_STAGE_MIN ? IL_STAGE_MIN : (bytes > IL_STAGE_MAX ? IL_STAGE_MAX : bytes);
    want = (want + IL_STAGE_MIN - 1) / IL_STAGE_MIN * IL_STAGE_MIN;
    if (h->stage && h->stage_half >= want) return MFLAB_OK;
    if (h->stage) {
        cudaError_t e = cudaSuccess;
        for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = cudaStreamSynchronize(h->il_stream[i]);
        if (e == cudaSuccess) e = cudaFree(h->stage);
        h->stage = nullptr;
        h->stage_half = 0;
        if (e != cudaSuccess) return record_cuda_error(e, "staging regrow");
    }
    int lo = 0, hi = 0;
    cudaError_t e = cudaDeviceGetStreamPriorityRange(&lo, &hi);
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) {
        if (!h->il_stream[i])
            e = cudaStreamCreateWithPriority(&h->il_stream[i], cudaStreamNonBlocking, hi);
        if (e == cudaSuccess && !h->il_done[i])
            e = cudaEventCreateWithFlags(&h->il_done[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess && !h->il_fork)
        e = cudaEventCreateWithFlags(&h->il_fork, cudaEventDisableTiming);
    if (e != cudaSuccess) return record_cuda_error(e, "staging streams");
    e = cudaMalloc(&h->stage, 2 * want);
    if (e != cudaSuccess) {
        record_cuda_error(e, "staging cudaMalloc");
        h->stage = nullptr;
        return MFLAB_ERR_ALLOC;
    }
    h->stage_half = want;
    return MFLAB_OK;
}

// Staged chunks: rb rows x cb columns fill at most one staging half (whole
// columns when a column fits, otherwise row blocks of single columns).
struct Chunks {
    int64_t rb, cb;
};
Chunks chunking(int N, int64_t m, size_t half) {
    const int64_t elem = N * (int64_t)sizeof(double);
    const int64_t rows_per_half = (int64_t)half / elem;
    if (m <= rows_per_half) return {m, std::max<int64_t>(1, rows_per_half / m)};
    return {rows_per_half, 1};
}

// Host <-> device through the staging halves.  Chunk j uses half j mod 2
// and runs on internal stream j mod 2: its copy and its permutation kernel
// are ordered on that stream (so chunk j + 2 reuses the half only after
// chunk j is done with it), while the copy engine moves chunk j + 1 on the
// other stream during chunk j's kernel.  The chunk count continues across
// calls (the handle remembers it), so two consecutive matrices of up to
// 1 GiB go to different halves: the second one's copy does not wait for the
// first one's permutation kernel, which may itself wait for SMs held by the
// caller's long kernels.  Both streams start after the caller's stream
// reaches this point (fork event) and the caller's stream continues after
// both (join events), so the call is stream-ordered like the others.  The
// high priority lets the permutation kernels start ahead of pending blocks of
// long kernels on other streams.
template <bool H2D>
int staged(mflab_handle *h, int N, int64_t m, int64_t n, double *host, int64_t ldh, double *P,
           int64_t ld, int64_t ls, cudaStream_t s) {
    int rc = reserve_stage(h, (size_t)m * n * N * sizeof(double));
    if (rc) return rc;
    const char *what = H2D ? "mflab_h2d_interleaved" : "mflab_d2h_interleaved";
    cudaError_t e = cudaEventRecord(h->il_fork, s);
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = cudaStreamWaitEvent(h->il_stream[i], h->il_fork, 0);
    if (e != cudaSuccess) return record_cuda_error(e, what);
    const Chunks ch = chunking(N, m, h->stage_half);
    const size_t hpitch = (size_t)ldh * N * sizeof(double);
    int64_t j = h->il_next;
    for (int64_t c0 = 0; c0 < n; c0 += ch.cb) {
        const int64_t w = std::min(ch.cb, n - c0);
        for (int64_t r0 = 0; r0 < m; r0 += ch.rb, ++j) {
            const int64_t hgt = std::min(ch.rb, m - r0);
            const size_t row_bytes = (size_t)hgt * N * sizeof(double);
            cudaStream_t cs = h->il_stream[j & 1];
            double *st = (double *)((char *)h->stage + (j & 1) * h->stage_half);
            double *hp = host + (c0 * ldh + r0) * N;
            double *pp = P + c0 * ld + r0;
            if (H2D) {
                e = cudaMemcpy2DAsync(st, row_bytes, hp, hpitch, row_bytes, (size_t)w,
                                      cudaMemcpyHostToDevice, cs);
                if (e != cudaSuccess) return record_cuda_error(e, what);
                if ((rc = launch<true>(N, hgt, w, st, hgt, pp, ld, ls, cs))) return rc;
            } else {
                if ((rc = launch<false>(N, hgt, w, st, hgt, pp, ld, ls, cs))) return rc;
                e = cudaMemcpy2DAsync(hp, hpitch, st, row_bytes, row_bytes, (size_t)w,
                                      cudaMemcpyDeviceToHost, cs);
                if (e != cudaSuccess) return record_cuda_error(e, what);
            }
        }
    }
    h->il_next = (int)(j & 1);
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) {
        e = cudaEventRecord(h->il_done[i], h->il_stream[i]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s, h->il_done[i], 0);
    }
    return e == cudaSuccess ? MFLAB_OK : record_cuda_error(e, what);
}

}  // namespace
}  // namespace mfl

extern "C" int mflab_interleaved_to_planes(mflab_handle *h, void *stream, int limbs, int64_t m,
                                           int64_t n, const double *X, int64_t ldx, double *P,
                                           int64_t ld, int64_t ls) {
    MFLAB_RANGE("mflab_interleaved_to_planes");
    bool empty;
    int rc = mfl::check_args(h, limbs, m, n, X, ldx, P, ld, ls, &empty);
    if (rc || empty) return rc;
    return mfl::launch<true>(limbs, m, n, (double *)X, ldx, P, ld, ls, (cudaStream_t)stream);
}

extern "C" int mflab_planes_to_interleaved(mflab_handle *h, void *stream, int limbs, int64_t m,
                                           int64_t n, const double *P, int64_t ld, int64_t ls,
                                           double *X, int64_t ldx) {
    MFLAB_RANGE("mflab_planes_to_interleaved");
    bool empty;
    int rc = mfl::check_args(h, limbs, m, n, X, ldx, P, ld, ls, &empty);
    if (rc || empty) return rc;
    return mfl::launch<false>(limbs, m, n, X, ldx, (double *)P, ld, ls, (cudaStream_t)stream);
}

extern "C" int mflab_h2d_interleaved(mflab_handle *h, void *stream, int limbs, int64_t m, int64_t n,
                                     const double *host, int64_t ldh, double *P, int64_t ld,
                                     int64_t ls) {
    MFLAB_RANGE("mflab_h2d_interleaved");
    bool empty;
    int rc = mfl::check_args(h, limbs, m, n, host, ldh, P, ld, ls, &empty);
    if (rc || empty) return rc;
    return mfl::staged<true>(h, limbs, m, n, (double *)host, ldh, P, ld, ls, (cudaStream_t)stream);
}

extern "C" int mflab_d2h_interleaved(mflab_handle *h, void *stream, int limbs, int64_t m, int64_t n,
                                     const double *P, int64_t ld, int64_t ls, double *host,
                                     int64_t ldh) {
    MFLAB_RANGE("mflab_d2h_interleaved");
    bool empty;
    int rc = mfl::check_args(h, limbs, m, n, host, ldh, P, ld, ls, &empty);
    if (rc || empty) return rc;
    return mfl::staged<false>(h, limbs, m, n, host, ldh, (double *)P, ld, ls,
                              (cudaStream_t)stream);
}
