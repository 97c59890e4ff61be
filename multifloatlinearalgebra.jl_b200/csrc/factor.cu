// Blocked multi-double Cholesky and LU with solves and factor diagnostics.
//
// Cholesky follows src/factorizations/cholesky.jl:10-107 of
// MultiFloatLinearAlgebra.jl: per block of `block` columns, a panel kernel
// factors the diagonal block (rows inside the panel only), the rows below are
// solved with trsm(side=right, lower, T) and the trailing lower triangle gets
// -1 * (A21 A21^T) + 1 * A22 from the shared mainloop.  LU follows
// src/factorizations/lu.jl:34-195: per panel column a pivot kernel (first
// strictly larger |A[r,k]|, full-row swap, reciprocal scaling) and a rank-1
// panel update, then trsm(left, lower, unit) on U12 and A22 = -A21 U12 + A22.
// Every kernel reads the device `info` word first and exits if an earlier step
// failed, so a whole factorization is enqueued without host synchronisation.
#include "mf_device.cuh"
#include <algorithm>

#include "mflab_internal.h"

MFLAB_DEBUG_RECORD(factor)

namespace mfl {

__global__ void iota1_kernel(int64_t *p, int64_t count) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) p[i] = i + 1;
}

// ------------------------------------------------------------- checks ----
template <int N>
__global__ void nonfinite_kernel(int64_t m, int64_t n, Mat A, int lower_only, int *info) {
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= m * n) return;
    int64_t r = idx % m, c = idx / m;
    if (lower_only && r < c) return;
    if (!isfinite_mf(load_mf<N>(A.p, A.ld, A.ls, r, c))) *info = -1;
}

// ------------------------------------------------------------ Cholesky ---
// one warp; w <= 32 columns of the diagonal block starting at (f, f)
template <int N>
__global__ void potrf_panel_kernel(Mat A, int64_t f, int w, int *info) {
    if (*info) return;
    __shared__ double piv[N];
    __shared__ int fail;
    const int t = threadIdx.x;
    if (t == 0) fail = 0;
    __syncthreads();
    for (int c = 0; c < w; ++c) {
        const int64_t col = f + c;
        if (t == 0) {
            mf<N> d = load_mf<N>(A.p, A.ld, A.ls, col, col);
            for (int64_t k = f; k < col; ++k) {
                mf<N> v = load_mf<N>(A.p, A.ld, A.ls, col, k);
                d = submul(d, v, v);
            }
            if (!gt(d, from_double<N>(0.0))) {
                fail = 1;
                *info = (int)(col + 1);
            } else {
                mf<N> p = sqrt_mf(d);
                store_mf<N>(A.p, A.ld, A.ls, col, col, p);
#pragma unroll
                for (int l = 0; l < N; ++l) piv[l] = p.v[l];
            }
        }
        __syncthreads();
        if (fail) return;
        mf<N> p;
#pragma unroll
        for (int l = 0; l < N; ++l) p.v[l] = piv[l];
        const int64_t row = col + 1 + t;
        if (t < w - 1 - c) {
            mf<N> v = load_mf<N>(A.p, A.ld, A.ls, row, col);
            for (int64_t k = f; k < col; ++k)
                v = submul(v, load_mf<N>(A.p, A.ld, A.ls, row, k), load_mf<N>(A.p, A.ld, A.ls, col, k));
            store_mf<N>(A.p, A.ld, A.ls, row, col, div(v, p));
        }
        __syncthreads();
    }
}

// One block step of the blocked Cholesky, fused: the diagonal block's factor
// (potrf_panel_kernel) and the solve of the rows below it (trsm_right_thread,
// A21 <- A21 inv(L11)^T), evaluated right-looking with every entry's
// operations in the reference's order.  Entry (r, j) of the block starts from
// A[r, j] and receives, for k = 0 .. j-1 in ascending order,
//     v = submul(v, x_rk, L_jk)            (submul(d, L_jk, L_jk) on the diagonal)
// then x_rj = div(v, p_j) with p_j = sqrt(d_j) — the same operands in the same
// order as the two kernels' left-looking loops, so the bits agree.  Each
// thread holds one row in registers; register j holds column k + j at step k
// (the update writes its results one register down, so no register index
// depends on k).  Warp 0 holds the block's own rows, which every CTA factors
// (a 16 x 16 block), warps 1-3 hold 96 rows below it per CTA.  Step k: thread k
// forms p_k (or records the failure), every later row forms x_rk, the block's
// rows publish L_jk, then every row updates its remaining entries.  Final
// values collect in shared memory and are written at the end: on a failure at
// column k, CTA 0 writes the block's columns before k and nothing else, as the
// two kernels would (the solve never runs after a failed panel).
constexpr int PF_W = 16, PF_NT = 128, PF_DIAG = 32;

template <int N>
__global__ void __launch_bounds__(PF_NT)
    potrf_step_kernel(Mat A, int64_t f, int w, int64_t t_rows, int *info) {
    // launched as a programmatic dependent of the previous block's update of
    // these columns: wait for that grid's results before reading anything
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (*info) return;
    extern __shared__ double pf_fin[];  // [PF_W][PF_NT][N] final values of each thread's row
    __shared__ double Ls[PF_W][PF_W][N];  // L[j][k] of the block's rows
    __shared__ double piv[N];
    __shared__ int fail;
    const int tid = threadIdx.x;
    const bool dg = tid < PF_DIAG;
    const int64_t rb = (int64_t)blockIdx.x * (PF_NT - PF_DIAG) + (tid - PF_DIAG);
    const bool has = dg ? tid < w : rb < t_rows;
    const int64_t row = dg ? f + tid : f + w + rb;
    mf<N> r[PF_W];
#pragma unroll
    for (int j = 0; j < PF_W; ++j)
        r[j] = (has && j < w) ? load_mf<N>(A.p, A.ld, A.ls, row, f + j) : from_double<N>(0.0);
    if (tid == 0) fail = 0;
    __syncthreads();
    int kf = w;  // the failed column, or w
#pragma unroll 1
    for (int k = 0; k < w; ++k) {
        if (tid == k) {  // the block's row k: register 0 is its diagonal entry
            const mf<N> d = r[0];
            if (!gt(d, from_double<N>(0.0))) {
                fail = 1;
                if (blockIdx.x == 0) *info = (int)(f + k + 1);
            } else {
                const mf<N> p = sqrt_mf(d);
#pragma unroll
                for (int l = 0; l < N; ++l) {
                    piv[l] = p.v[l];
                    pf_fin[((size_t)k * PF_NT + tid) * N + l] = p.v[l];
                }
            }
        }
        __syncthreads();
        if (fail) {
            kf = k;
            break;
        }
        mf<N> p;
#pragma unroll
        for (int l = 0; l < N; ++l) p.v[l] = piv[l];
        const bool act = has && (!dg || tid > k);
        mf<N> x = from_double<N>(0.0);
        if (act) {
            x = div(r[0], p);
#pragma unroll
            for (int l = 0; l < N; ++l) {
                pf_fin[((size_t)k * PF_NT + tid) * N + l] = x.v[l];
                if (dg) Ls[tid][k][l] = x.v[l];
            }
        }
        __syncthreads();
        if (act) {
            // register j <- column k+1+j (only the lower part of the block's rows)
#pragma unroll
            for (int j = 0; j < PF_W - 1; ++j) {
                const int c = k + 1 + j;
                if (c < w && (!dg || c <= tid)) {
                    mf<N> ljk;
#pragma unroll
                    for (int l = 0; l < N; ++l) ljk.v[l] = Ls[c][k][l];
                    r[j] = submul(r[j + 1], x, ljk);
                }
            }
        }
    }
    // final values: the block's rows from CTA 0 (lower triangle), columns
    // before the failure; the rows below only without a failure
    if (!has) return;
    if (dg) {
        if (blockIdx.x != 0) return;
        for (int j = 0; j < kf && j <= tid; ++j) {
            mf<N> v;
#pragma unroll
            for (int l = 0; l < N; ++l) v.v[l] = pf_fin[((size_t)j * PF_NT + tid) * N + l];
            store_mf<N>(A.p, A.ld, A.ls, row, f + j, v);
        }
    } else if (kf == w) {
        for (int j = 0; j < w; ++j) {
            mf<N> v;
#pragma unroll
            for (int l = 0; l < N; ++l) v.v[l] = pf_fin[((size_t)j * PF_NT + tid) * N + l];
            store_mf<N>(A.p, A.ld, A.ls, row, f + j, v);
        }
    }
}

static int lu64_lookahead_streams(mflab_handle *h);

// Blocked Cholesky in the reference's order with look-ahead.  Per block:
// the fused step kernel (panel + solve below it), then the trailing
// lower(A22) -= L21 L21^T in two parts that partition its lower triangle: the
// next block's columns (all rows) on a high-priority stream, the rest on the
// caller's stream, where it overlaps the next block's step kernel.  Every
// entry still receives the blocks' updates one after another in block order
// (the next-columns part of block b waits for the rest of block b-1, which
// updated those columns), each as the same K = block chain and epilogue, so
// the factor is the same bit for bit.  Blocks wider than PF_W take the panel
// kernel + TRSM path on the caller's stream.
template <int N>
static int potrf_n(mflab_handle *h, int64_t n, Mat A, int64_t block, int *info, cudaStream_t s) {
    const double mone[4] = {-1.0, 0.0, 0.0, 0.0}, one[4] = {1.0, 0.0, 0.0, 0.0};
    cudaError_t e = cudaMemsetAsync(info, 0, sizeof(int), s);
    if (e != cudaSuccess) return record_cuda_error(e, "potrf info");
    if (n == 0) return MFLAB_OK;
    int64_t tot = n * n;
    nonfinite_kernel<N><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(n, n, A, 1, info);
    int rc = record_cuda_error(cudaGetLastError(), "potrf check");
    if (rc) return rc;
    if (block > PF_W) {
        for (int64_t first = 0; first < n; first += block) {
            const int64_t last = first + block - 1 < n - 1 ? first + block - 1 : n - 1;
            const int w = (int)(last - first + 1);
            potrf_panel_kernel<N><<<1, 32, 0, s>>>(A, first, w, info);
            rc = record_cuda_error(cudaGetLastError(), "potrf panel");
            if (rc) return rc;
            if (last < n - 1) {
                const int64_t t = n - 1 - last;
                rc = launch_trsm_info(N, 1, 0, 1, 0, t, w, A.at(first, first), A.at(last + 1, first),
                                      one, s, info);
                if (rc) return rc;
                rc = launch_mm(N, false, true, 1, false, t, t, w, A.at(last + 1, first),
                               A.at(last + 1, first), A.at(last + 1, last + 1), mone, one, s, info);
                if (rc) return rc;
            }
        }
        return MFLAB_OK;
    }
    const size_t fin_bytes = (size_t)PF_W * PF_NT * N * sizeof(double);
    static std::atomic<unsigned long long> configured{0};
    rc = set_smem_once((const void *)potrf_step_kernel<N>, (int)fin_bytes, configured,
                       "potrf step attribute");
    if (rc) return rc;
    rc = lu64_lookahead_streams(h);
    if (rc) return rc;
    cudaStream_t sp = h->la_stream;
    cudaEvent_t ev_fork = h->la_ev[0], ev_step = h->la_ev[1], ev_rest = h->la_ev[2];
    e = cudaEventRecord(ev_fork, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(sp, ev_fork, 0);
    if (e != cudaSuccess) return record_cuda_error(e, "potrf fork");
    int b = 0;
    for (int64_t first = 0; first < n && rc == MFLAB_OK; first += block, ++b) {
        const int64_t last = first + block - 1 < n - 1 ? first + block - 1 : n - 1;
        const int w = (int)(last - first + 1);
        const int64_t t = n - 1 - last;  // rows below the block
        const unsigned grid = (unsigned)std::max<int64_t>(1, (t + PF_NT - PF_DIAG - 1) /
                                                                 (PF_NT - PF_DIAG));
        // a programmatic dependent of the previous next-columns update: the
        // step's CTAs are placed while that update drains
        rc = launch_programmatic(potrf_step_kernel<N>, dim3(grid), dim3(PF_NT), fin_bytes, sp,
                                 "potrf step", A, first, w, t, info);
        if (rc || t == 0) break;
        e = cudaEventRecord(ev_step, sp);
        // the next block's columns, after the rest of the previous block
        const int64_t wn = std::min<int64_t>(block, t);
        if (e == cudaSuccess && b > 0) e = cudaStreamWaitEvent(sp, ev_rest, 0);
        if (e != cudaSuccess) return record_cuda_error(e, "potrf look-ahead");
        rc = launch_mm(N, false, true, 1, false, t, wn, w, A.at(last + 1, first),
                       A.at(last + 1, first), A.at(last + 1, last + 1), mone, one, sp, info);
        if (rc) break;
        // the rest of the lower triangle, after the step
        if (t > wn) {
            e = cudaStreamWaitEvent(s, ev_step, 0);
            if (e != cudaSuccess) return record_cuda_error(e, "potrf look-ahead");
            rc = launch_mm(N, false, true, 1, false, t - wn, t - wn, w,
                           A.at(last + 1 + wn, first), A.at(last + 1 + wn, first),
                           A.at(last + 1 + wn, last + 1 + wn), mone, one, s, info);
            if (rc) break;
        }
        e = cudaEventRecord(ev_rest, s);
        if (e != cudaSuccess) rc = record_cuda_error(e, "potrf look-ahead");
    }
    // join: the caller's stream waits for the high-priority stream
    e = cudaEventRecord(ev_fork, sp);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ev_fork, 0);
    if (e != cudaSuccess && rc == MFLAB_OK) rc = record_cuda_error(e, "potrf join");
    return rc;
}

// Cholesky with INT8 trailing updates: panels of nb columns; inside a panel
// the blocked algorithm above (panel kernel, TRSM, lower update restricted to
// the panel's columns) in the reference order; after each panel the trailing
// matrix gets lower(A22) -= L21 L21^T through the modular INT8 route.  The
// device info word is read after every panel (one synchronisation each), so a
// failed pivot stops the factorization before the next trailing update.
template <int N>
static int potrf_ozaki_n(mflab_handle *h, int64_t n, Mat A, int64_t nb, int64_t block, int moduli,
                         int *info, cudaStream_t s) {
    const double mone[4] = {-1.0, 0.0, 0.0, 0.0}, one[4] = {1.0, 0.0, 0.0, 0.0};
    cudaError_t e = cudaMemsetAsync(info, 0, sizeof(int), s);
    if (e != cudaSuccess) return record_cuda_error(e, "potrf info");
    if (n == 0) return MFLAB_OK;
    int64_t tot = n * n;
    nonfinite_kernel<N><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(n, n, A, 1, info);
    int rc = record_cuda_error(cudaGetLastError(), "potrf check");
    if (rc) return rc;
    for (int64_t j0 = 0; j0 < n; j0 += nb) {
        const int64_t j1 = j0 + nb < n ? j0 + nb : n;  // panel columns [j0, j1)
        for (int64_t first = j0; first < j1; first += block) {
            const int64_t last = first + block - 1 < j1 - 1 ? first + block - 1 : j1 - 1;
            const int w = (int)(last - first + 1);
            potrf_panel_kernel<N><<<1, 32, 0, s>>>(A, first, w, info);
            rc = record_cuda_error(cudaGetLastError(), "potrf panel");
            if (rc) return rc;
            if (last < n - 1) {
                const int64_t t = n - 1 - last, cols = j1 - 1 - last;
                rc = launch_trsm_info(N, 1, 0, 1, 0, t, w, A.at(first, first), A.at(last + 1, first),
                                      one, s, info);
                if (rc) return rc;
                if (cols > 0) {
                    rc = launch_mm(N, false, true, 1, false, t, cols, w, A.at(last + 1, first),
                                   A.at(last + 1, first), A.at(last + 1, last + 1), mone, one, s,
                                   info);
                    if (rc) return rc;
                }
            }
        }
        int hinfo = 0;
        e = cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return record_cuda_error(e, "potrf info read");
        if (hinfo != 0) return MFLAB_OK;
        if (j1 < n) {
            rc = ozaki_crt_syrk(h, N, moduli, 0, n - j1, j1 - j0, A.at(j1, j0), A.at(j1, j1), mone,
                                one, s, nullptr);
            if (rc) return rc;
        }
    }
    return MFLAB_OK;
}

// ------------------------------------------------------------------ LU ---
// single CTA: pivot search in column k (rows k..m-1), full-row swap,
// zero-pivot test, reciprocal and scaling of the column below the pivot
// The interchange of step k is applied to the panel's columns [c_lo, c_hi)
// only; lu_swap_rest_kernel applies the panel's interchanges to every other
// column once the panel is done (no computation reads those columns in
// between, so the factor is the same as with full-row swaps at each step).
template <int N, int NT>
__global__ void __launch_bounds__(NT) lu_pivot_kernel(int64_t m, int64_t c_lo, int64_t c_hi, Mat A,
                                                      int64_t k, int64_t *ipiv, int *info) {
    // the panel's steps are programmatic dependent launches: wait for the
    // previous step's grid, let the next step's CTAs be placed meanwhile
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (*info) return;
    __shared__ double sval[NT][N];
    __shared__ int64_t sidx[NT];
    __shared__ double sinv[N];
    __shared__ int64_t spiv;
    const int t = threadIdx.x;
    // strided scan: first strictly larger |A[r,k]| in ascending r
    mf<N> best = from_double<N>(-1.0);
    int64_t bidx = -1;
    for (int64_t r = k + t; r < m; r += NT) {
        mf<N> cand = abs_mf(load_mf<N>(A.p, A.ld, A.ls, r, k));
        if (bidx < 0 || gt(cand, best)) {
            best = cand;
            bidx = r;
        }
    }
#pragma unroll
    for (int l = 0; l < N; ++l) sval[t][l] = best.v[l];
    sidx[t] = bidx;
    __syncthreads();
    for (int off = NT / 2; off > 0; off >>= 1) {
        if (t < off) {
            mf<N> a, b;
#pragma unroll
            for (int l = 0; l < N; ++l) {
                a.v[l] = sval[t][l];
                b.v[l] = sval[t + off][l];
            }
            int64_t ia = sidx[t], ib = sidx[t + off];
            bool take_b;
            if (ib < 0) take_b = false;
            else if (ia < 0) take_b = true;
            else if (gt(b, a)) take_b = true;
            else if (gt(a, b)) take_b = false;
            else take_b = ib < ia;
            if (take_b) {
#pragma unroll
                for (int l = 0; l < N; ++l) sval[t][l] = b.v[l];
                sidx[t] = ib;
            }
        }
        __syncthreads();
    }
    if (t == 0) {
        spiv = sidx[0];
        ipiv[k] = sidx[0] + 1;
    }
    __syncthreads();
    const int64_t p = spiv;
    if (p != k) {
        for (int64_t c = c_lo + t; c < c_hi; c += NT) {
#pragma unroll
            for (int l = 0; l < N; ++l) {
                double *x = A.p + l * A.ls + c * A.ld;
                double tmp = x[k];
                x[k] = x[p];
                x[p] = tmp;
            }
        }
    }
    __syncthreads();
    if (t == 0) {
        mf<N> akk = load_mf<N>(A.p, A.ld, A.ls, k, k);
        if (iszero(akk)) {
            *info = (int)(k + 1);
        } else {
            mf<N> iv = inv(akk);
#pragma unroll
            for (int l = 0; l < N; ++l) sinv[l] = iv.v[l];
        }
    }
    __syncthreads();
    if (*info) return;
    mf<N> iv;
#pragma unroll
    for (int l = 0; l < N; ++l) iv.v[l] = sinv[l];
    for (int64_t r = k + 1 + t; r < m; r += NT)
        store_mf<N>(A.p, A.ld, A.ls, r, k, mul(load_mf<N>(A.p, A.ld, A.ls, r, k), iv));
}

// The interchanges of panel steps first .. last (ipiv, ascending, as the
// sequential row swaps of lu.jl) on every column outside [first, last]: one
// thread per column.  Only the steps that ran are replayed: after a zero
// pivot at step info-1 (no interchange there) the later steps never ran.
template <int N>
__global__ void lu_swap_rest_kernel(int64_t n, Mat A, int64_t first, int64_t last,
                                    const int64_t *ipiv, const int *info) {
    const int st = *info;
    if (st < 0) return;
    const int64_t upto = st == 0 ? last : (int64_t)st - 2;  // last step with an interchange
    if (upto < first) return;
    const int64_t w = last - first + 1;
    const int64_t col = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= n - w) return;
    const int64_t c = col < first ? col : col + w;
    for (int64_t k = first; k <= upto; ++k) {
        const int64_t p = ipiv[k] - 1;
        if (p == k) continue;
#pragma unroll
        for (int l = 0; l < N; ++l) {
            double *x = A.p + l * A.ls + c * A.ld;
            const double tmp = x[k];
            x[k] = x[p];
            x[p] = tmp;
        }
    }
}

// rank-1 update of panel columns k+1..last for rows k+1..m-1 (lu.jl:47-82)
template <int N>
__global__ void lu_rank1_kernel(int64_t m, Mat A, int64_t k, int64_t last, const int *info) {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (*info) return;
    const int64_t r = k + 1 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= m) return;
    const mf<N> f = load_mf<N>(A.p, A.ld, A.ls, r, k);
    for (int64_t c = k + 1; c <= last; ++c) {
        mf<N> v = load_mf<N>(A.p, A.ld, A.ls, r, c);
        store_mf<N>(A.p, A.ld, A.ls, r, c, submul(v, f, load_mf<N>(A.p, A.ld, A.ls, k, c)));
    }
}

// ------------------------------------------------- binary64 LU (fast) ---
// The binary64 instance (the factor of the mixed-precision solver) has no
// reference order to keep; it is factored LAPACK-style: one CTA factors a
// panel of w <= 32 columns with partial pivoting, exchanging rows inside the
// panel only; one kernel then applies the panel's interchanges to the other
// columns, and the U block row and the trailing matrix are updated with the
// TRSM and FP64 GEMM kernels.
constexpr int LU64_NT = 1024;

__global__ void __launch_bounds__(LU64_NT)
    lu64_panel_kernel(int64_t m, Mat A, int64_t k0, int w, int64_t *ipiv, int *info) {
    if (*info) return;
    __shared__ double sv[LU64_NT / 32];
    __shared__ int64_t si[LU64_NT / 32];
    __shared__ int64_t spiv;
    __shared__ double sinv;
    __shared__ double su[32];
    const int t = threadIdx.x, lane = t % 32, wid = t / 32;
    double *a = A.p;
    const int64_t ld = A.ld;
    for (int c = 0; c < w; ++c) {
        const int64_t k = k0 + c;
        // pivot: the first row of largest |A[r, k]|, r >= k
        double best = -1.0;
        int64_t bi = -1;
        for (int64_t r = k + t; r < m; r += LU64_NT) {
            const double v = fabs(a[k * ld + r]);
            if (v > best) {
                best = v;
                bi = r;
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, best, off);
            const int64_t oi = __shfl_xor_sync(0xffffffffu, bi, off);
            if (oi >= 0 && (bi < 0 || ov > best || (ov == best && oi < bi))) {
                best = ov;
                bi = oi;
            }
        }
        if (lane == 0) {
            sv[wid] = best;
            si[wid] = bi;
        }
        __syncthreads();
        if (wid == 0) {
            best = lane < LU64_NT / 32 ? sv[lane] : -1.0;
            bi = lane < LU64_NT / 32 ? si[lane] : -1;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, best, off);
                const int64_t oi = __shfl_xor_sync(0xffffffffu, bi, off);
                if (oi >= 0 && (bi < 0 || ov > best || (ov == best && oi < bi))) {
                    best = ov;
                    bi = oi;
                }
            }
            if (lane == 0) {
                spiv = bi;
                ipiv[k] = bi + 1;
            }
        }
        __syncthreads();
        const int64_t p = spiv;
        if (p != k && t < w) {  // exchange rows k and p inside the panel
            const double tmp = a[(k0 + t) * ld + k];
            a[(k0 + t) * ld + k] = a[(k0 + t) * ld + p];
            a[(k0 + t) * ld + p] = tmp;
        }
        __syncthreads();
        if (t == 0) {
            const double akk = a[k * ld + k];
            if (akk == 0.0) *info = (int)(k + 1);
            sinv = 1.0 / akk;
        }
        __syncthreads();
        if (*info) return;
        const double iv = sinv;
        // U row k of the panel in shared memory, then per row: scale the
        // multiplier and update the panel columns right of k (independent
        // loads along the row, so they are in flight together)
        const int rest = w - 1 - c;
        if (t < rest) su[t] = a[(k + 1 + t) * ld + k];
        __syncthreads();
        for (int64_t r = k + 1 + t; r < m; r += LU64_NT) {
            const double l = a[k * ld + r] * iv;
            a[k * ld + r] = l;
#pragma unroll 8
            for (int j = 0; j < rest; ++j) {
                double *x = a + (k + 1 + j) * ld + r;
                *x -= l * su[j];
            }
        }
        __syncthreads();
    }
}

// Panel of the binary64 LU held in the shared memory of a cluster of CL
// CTAs (distributed shared memory) instead of streamed through one SM:
// CTA q of the cluster keeps panel rows k0 + q R .. k0 + q R + R - 1 (R =
// ceil((m - k0) / CL)) of the w <= 32 columns.  Partial pivoting with the
// first-largest rule of lu64_panel_kernel (the largest |A[r, k]|, ties to the
// smallest row), one cluster barrier and one CTA barrier per column:
//   * every CTA publishes the best active row of the next column (value,
//     current row, slot) together with that row's values in its own shared
//     memory;
//   * after the cluster barrier every warp reads the CL candidates, picks
//     the same pivot and takes the pivot row's values from the winner's
//     published copy (one round of remote loads, issued together);
//   * the interchange is logical: every CTA keeps the same map from current
//     row to (CTA, slot), each thread the current row of its own slots; the
//     data stay in place until the panel is written back;
//   * each thread updates its active slots (current row > k) and forms the
//     candidate of the next column in the same pass.
// The panel is written back with each slot's row at its final position,
// which equals physical row interchanges, and the moved rows are listed for
// the interchanges outside the panel: src[i] = the original row that ends in
// row k0 + i (i < w), and ext pairs (row >= k0 + w, original row) with a
// count in ext[0].
constexpr int LUC_CL = 8;       // CTAs of the cluster
constexpr int LUC_W = 32;       // panel width
constexpr int LUC_NT = 512;
constexpr int LUC_SMEM_MAX = 220 * 1024;

struct LucCand {
    double v;   // |A[row, c]|, -1 for none
    int row;    // current row index (absolute)
    int code;   // owner CTA * R + slot
    double vals[LUC_W];  // the row's values, columns c .. w-1
};

__device__ __forceinline__ uint32_t luc_map(const void *p, uint32_t rank) {
    uint32_t a = (uint32_t)__cvta_generic_to_shared(p), r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
    return r;
}
__device__ __forceinline__ double luc_ld_f64(uint32_t addr) {
    double v;
    asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(addr) : "memory");
    return v;
}
__device__ __forceinline__ int luc_ld_s32(uint32_t addr) {
    int v;
    asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
    return v;
}
__device__ __forceinline__ void luc_cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\t"
                 "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ bool luc_better(double v, int row, double bv, int brow) {
    return v > bv || (v == bv && v >= 0.0 && row < brow);
}
// warp-wide best of (v, row, code)
__device__ __forceinline__ void luc_warp_best(double &v, int &row, int &code) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, off);
        const int orow = __shfl_xor_sync(0xffffffffu, row, off);
        const int ocode = __shfl_xor_sync(0xffffffffu, code, off);
        if (luc_better(ov, orow, v, row)) {
            v = ov;
            row = orow;
            code = ocode;
        }
    }
}

// best of (v, row, code) over lanes 0 .. 7 (the other lanes hold no entry),
// in every lane: three exchange rounds and a broadcast
__device__ __forceinline__ void luc_best8(double &v, int &row, int &code) {
#pragma unroll
    for (int off = 4; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, off);
        const int orow = __shfl_xor_sync(0xffffffffu, row, off);
        const int ocode = __shfl_xor_sync(0xffffffffu, code, off);
        if (luc_better(ov, orow, v, row)) {
            v = ov;
            row = orow;
            code = ocode;
        }
    }
    v = __shfl_sync(0xffffffffu, v, 0);
    row = __shfl_sync(0xffffffffu, row, 0);
    code = __shfl_sync(0xffffffffu, code, 0);
}

// shared memory of the cluster panel kernel for R rows per CTA and mr panel rows
__host__ __device__ inline size_t luc_smem(int64_t R, int64_t mr) {
    return (size_t)R * LUC_W * sizeof(double) + (size_t)R * sizeof(int) +
           (size_t)mr * sizeof(int) + 2 * sizeof(LucCand) + 64;
}

__global__ void __cluster_dims__(LUC_CL, 1, 1) __launch_bounds__(LUC_NT, 1)
    lu64_cluster_panel_kernel(int64_t m, Mat A, int64_t k0, int w, int R, int64_t *ipiv,
                              int *info, int *moved) {
    extern __shared__ __align__(16) uint8_t luc_raw[];
    double *panel = (double *)luc_raw;                        // [w][R]
    int *slot_row = (int *)(panel + (size_t)R * LUC_W);       // [R] current row of a slot
    int *where = slot_row + R;                                // [mr] code of a current row
    const int64_t mr = m - k0;
    LucCand *cand = (LucCand *)(((uintptr_t)(where + mr) + 15) & ~(uintptr_t)15);  // [2]
    __shared__ double red_v[LUC_NT / 32];
    __shared__ int red_r[LUC_NT / 32], red_c[LUC_NT / 32];

    const int t = threadIdx.x, lane = t % 32, wid = t / 32;
    uint32_t rank;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
    const int64_t base = k0 + (int64_t)rank * R;  // absolute row of slot 0
    const int64_t left = mr - (int64_t)rank * R;
    const int nloc = (int)(left < 0 ? 0 : (left < R ? left : R));
    const int stop0 = *info;  // every CTA reads the same value
    if (rank == 0 && t == 0) moved[2 * LUC_W] = 0;  // count of the ext pairs

    for (int j = 0; j < w; ++j)
        for (int s = t; s < nloc; s += LUC_NT) panel[j * R + s] = A.p[(k0 + j) * A.ld + base + s];
    for (int s = t; s < R; s += LUC_NT) slot_row[s] = (int)(base + s);
    for (int64_t i = t; i < mr; i += LUC_NT) where[i] = (int)i;  // code = CTA * R + slot
    __syncthreads();

    // the best of this CTA's active rows for column c (values v, row, code per
    // thread) reduced over the CTA and published with the row's values
    auto publish = [&](int c, int buf, double v, int row, int code) {
        luc_warp_best(v, row, code);
        if (lane == 0) {
            red_v[wid] = v;
            red_r[wid] = row;
            red_c[wid] = code;
        }
        __syncthreads();
        if (wid == 0) {
            v = lane < LUC_NT / 32 ? red_v[lane] : -1.0;
            row = lane < LUC_NT / 32 ? red_r[lane] : 0x7fffffff;
            code = lane < LUC_NT / 32 ? red_c[lane] : -1;
            luc_warp_best(v, row, code);
            if (lane == 0) {
                cand[buf].v = v;
                cand[buf].row = row;
                cand[buf].code = code;
            }
            if (code >= 0 && c + lane < w) cand[buf].vals[c + lane] = panel[(c + lane) * R + code % R];
        }
    };
    {
        double v = -1.0;
        int row = 0x7fffffff, code = -1;
        for (int s = t; s < nloc; s += LUC_NT) {
            const double a = fabs(panel[s]);
            if (luc_better(a, slot_row[s], v, row)) {
                v = a;
                row = slot_row[s];
                code = (int)rank * R + s;
            }
        }
        publish(0, 0, v, row, code);
    }
    luc_cluster_sync();  // the candidates of column 0 and all shared memory initialised

    __shared__ double s_u[LUC_W];   // the pivot row, columns c .. w-1 at s_u[c ..]
    __shared__ int s_prow, s_pcode, s_ck, s_stop;
    for (int c = 0; c < w; ++c) {
        const int64_t k = k0 + c;
        const int buf = c & 1;
        if (wid == 0) {
            // warp 0: the CL candidates and their published row values (one
            // round of remote loads), the winner, the pivot row into s_u
            double v = -1.0, vals[LUC_CL];
            int prow = 0x7fffffff, q = -1;
            if (lane < LUC_CL) {
                const uint32_t a = luc_map(&cand[buf], (uint32_t)lane);
                v = luc_ld_f64(a);
                prow = luc_ld_s32(a + 8);
                q = lane;
            }
#pragma unroll
            for (int qq = 0; qq < LUC_CL; ++qq)
                vals[qq] = c + lane < w ? luc_ld_f64(luc_map(&cand[buf].vals[c + lane], (uint32_t)qq))
                                        : 0.0;
            luc_warp_best(v, prow, q);
            const int qb = q < 0 ? 0 : q;
            double u = 0.0;
#pragma unroll
            for (int qq = 0; qq < LUC_CL; ++qq) u = qq == qb ? vals[qq] : u;
            if (c + lane < w) s_u[c + lane] = u;
            if (lane == 0) {
                const uint32_t a = luc_map(&cand[buf], (uint32_t)qb);
                s_prow = prow;
                s_pcode = luc_ld_s32(a + 12);
                s_ck = where[k - k0];
                s_stop = stop0 != 0 || !(v > 0.0);
                if (rank == 0) {
                    if (stop0 == 0 && !(v > 0.0)) *info = (int)(k + 1);
                    if (stop0 == 0 && v > 0.0) ipiv[k] = (int64_t)prow + 1;
                }
            }
        }
        __syncthreads();
        if (s_stop) break;  // the same decision in every CTA
        const int prow = s_prow, pcode = s_pcode, ck = s_ck;
        const int po = pcode / R, ps = pcode % R;
        const double ivp = 1.0 / s_u[c];
        double bv = -1.0;
        int br = 0x7fffffff, bc = -1;
        for (int s = t; s < nloc; s += LUC_NT) {
            int row = slot_row[s];
            if ((int)rank == po && s == ps) row = (int)k;
            else if (prow != k && (int)rank * R + s == ck) row = prow;
            slot_row[s] = row;
            if (row <= k) continue;  // the pivot rows so far are final
            const double l = panel[c * R + s] * ivp;
            panel[c * R + s] = l;
            // independent updates of columns c+1 .. w-1, unrolled so that the
            // loads of all columns are in flight together
#pragma unroll
            for (int j = 1; j < LUC_W; ++j)
                if (c + j < w) panel[(c + j) * R + s] = fma(-l, s_u[c + j], panel[(c + j) * R + s]);
            if (c + 1 < w) {
                const double a = fabs(panel[(c + 1) * R + s]);
                if (luc_better(a, row, bv, br)) {
                    bv = a;
                    br = row;
                    bc = (int)rank * R + s;
                }
            }
        }
        if (c + 1 < w) {
            publish(c + 1, buf ^ 1, bv, br, bc);  // its barrier also orders the map update
        } else {
            __syncthreads();
        }
        if (t == 0) {  // logical interchange in the replicated row map (s_ck read above)
            where[prow - k0] = ck;
            where[k - k0] = pcode;
        }
        luc_cluster_sync();  // next candidates published; this step's remote reads done
    }
    luc_cluster_sync();  // no CTA leaves while another may still read its shared memory
    // write the panel back, every slot's row at its final position, and list
    // the moved rows
    for (int j = 0; j < w; ++j)
        for (int s = t; s < nloc; s += LUC_NT) A.p[(k0 + j) * A.ld + slot_row[s]] = panel[j * R + s];
    for (int s = t; s < nloc; s += LUC_NT) {
        const int dest = slot_row[s], orig = (int)(base + s);
        if (dest < k0 + w) {
            moved[dest - k0] = orig;
        } else if (dest != orig) {
            const int e = atomicAdd(&moved[2 * LUC_W], 1);
            if (MFLAB_IDX_OK(e < LUC_W, 5, e, dest)) {
                moved[LUC_W + e] = dest;              // ext rows
                moved[2 * LUC_W + 1 + e] = orig;      // ext sources
            }
        }
    }
}

// The same panel with its rows in registers: 256 threads hold two slots each
// (R <= 512 rows per CTA).  Register j of a row holds column c + j at step c:
// the rank-1 update writes its results one register down,
//     row[j] = fma(-l, u[j + 1], row[j + 1]),
// so the step's column is always register 0 and no register index depends
// on the column (the column loop stays rolled and its code small).  Every
// final value goes to shared memory when it is formed — the multiplier of
// an active row at its column, the whole remaining row of the pivot when it
// is chosen — and the panel is written back from there.
//
// The CTAs exchange candidates by pushing, not by a cluster barrier: after
// its CTA reduction, warp 0 of every CTA writes its best row (value, row,
// code and the row's values from the candidate column on) into its slot of
// every CTA's receive buffer with st.async, whose bytes complete on the
// receiver's mbarrier.  A step waits (bounded) for the 8 x 272 bytes of its
// buffer, and every warp then reads the 8 candidates from its own shared
// memory.  Two buffers alternate: a CTA pushes step c+2 only after it has
// all candidates of step c+1, which every CTA sends after its warps finished
// reading step c.  Pivot rule (largest magnitude, ties to the smallest
// row), logical interchanges (the slot holding row k recognises itself by
// its current row) and the moved-row list are those of
// lu64_cluster_panel_kernel.  A wait that runs out sets a shared abort flag
// and records TC-style error code 5 in *err; the CTA leaves the loop after
// its next CTA barrier, and the others, no longer receiving, time out too.
constexpr int LUR_NT = 256, LUR_RPT = 2;
constexpr uint32_t LUR_SLOT_TX = 16 + 8 + 32 * 8;  // bytes pushed per sender (header, u0, u)
constexpr long long LUR_WAIT_LIMIT = 1LL << 26;
constexpr int LUR_ERR_TIMEOUT = 5;

struct LurSlot {
    double v;       // |A[row, c]| of the candidate, -1 for none
    int row;        // its current row
    int code;       // owner CTA * R + slot
    double u0;      // A[row, c]
    double pad;
    double u[32];   // A[row, c + 1 + j], j < 31 (u[31] is zero)
};
struct LurRecv {
    LurSlot slot[LUC_CL];
};

// shared memory of the register panel kernel: the final values [w][R], two
// receive buffers, two mbarriers
__host__ __device__ inline size_t lur_smem(int64_t R) {
    return (size_t)LUC_W * R * sizeof(double) + 2 * sizeof(LurRecv) + 2 * sizeof(uint64_t) + 64;
}

// Warp-wide first-largest entry (largest v, ties to the smallest row; v < 0
// marks a lane without an entry, whose row is 0x7fffffff and code -1), in
// every lane, from three warp reductions of 32-bit keys: the high and low
// words of v's bits (ordered like v for v >= 0), then the smallest row among
// the lanes holding the maximum.
__device__ __forceinline__ void lur_warp_best(double &v, int &row, int &code) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    const unsigned hi = v >= 0.0 ? (unsigned)(b >> 32) + 1u : 0u;
    const unsigned m1 = __reduce_max_sync(0xffffffffu, hi);
    const unsigned lo = hi == m1 ? (unsigned)b : 0u;
    const unsigned m2 = __reduce_max_sync(0xffffffffu, lo);
    const bool tie = hi == m1 && (unsigned)b == m2;
    const unsigned m3 = __reduce_min_sync(0xffffffffu, tie ? (unsigned)row : 0xffffffffu);
    const unsigned win = __ballot_sync(0xffffffffu, tie && (unsigned)row == m3);
    code = __shfl_sync(0xffffffffu, code, __ffs(win) - 1);
    row = (int)m3;
    v = m1 == 0u ? -1.0
                 : __longlong_as_double((long long)(((unsigned long long)(m1 - 1u) << 32) | m2));
}

__device__ __forceinline__ void lur_push_f64(uint32_t raddr, double v, uint32_t rbar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.f64 [%0], %1, [%2];" ::"r"(
                     raddr),
                 "d"(v), "r"(rbar)
                 : "memory");
}
__device__ __forceinline__ void lur_push_v2b64(uint32_t raddr, unsigned long long a,
                                               unsigned long long b, uint32_t rbar) {
    asm volatile(
        "st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.b64 [%0], {%1, %2}, [%3];" ::"r"(
            raddr),
        "l"(a), "l"(b), "r"(rbar)
        : "memory");
}
__device__ __forceinline__ void lur_mbar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(
                     bar))
                 : "memory");
}
__device__ __forceinline__ void lur_arm(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool lur_wait(uint64_t *bar, uint32_t parity, const int *abort) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
    for (long long i = 0; i < LUR_WAIT_LIMIT; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, P1;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
        if (*(const volatile int *)abort) return false;
    }
    return false;
}

__global__ void __cluster_dims__(LUC_CL, 1, 1) __launch_bounds__(LUR_NT, 1)
    lu64_cluster_panel_reg_kernel(int64_t m, Mat A, int64_t k0, int w, int R, int64_t *ipiv,
                                  int *info, int *moved, int *err) {
    extern __shared__ __align__(16) uint8_t lur_raw[];
    double *fin = (double *)lur_raw;  // [w][R] final values
    LurRecv *recv = (LurRecv *)(fin + (size_t)LUC_W * R);  // [2]
    uint64_t *rbar = (uint64_t *)(recv + 2);               // [2]
    __shared__ double red_v[LUR_NT / 32];
    __shared__ int red_r[LUR_NT / 32], red_c[LUR_NT / 32];
    __shared__ __align__(16) double wstage[LUR_NT / 32][LUC_W];  // each warp's best row
    __shared__ int s_abort, s_stop;

    const int t = threadIdx.x, lane = t % 32, wid = t / 32;
    uint32_t rank;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
    const int64_t mr = m - k0;
    const int64_t base = k0 + (int64_t)rank * R;  // absolute row of slot 0
    const int64_t left = mr - (int64_t)rank * R;
    const int nloc = (int)(left < 0 ? 0 : (left < R ? left : R));
    const int stop0 = *info;  // every CTA reads the same value
    if (rank == 0 && t == 0) moved[2 * LUC_W] = 0;  // count of the ext pairs
    if (t == 0) {
        s_abort = 0;
        s_stop = 0;
        lur_mbar_init(&rbar[0]);
        lur_mbar_init(&rbar[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        lur_arm(&rbar[0], LUC_CL * LUR_SLOT_TX);
        lur_arm(&rbar[1], LUC_CL * LUR_SLOT_TX);
    }

    double row[LUR_RPT][LUC_W];
    bool has[LUR_RPT], act[LUR_RPT];
    int cur[LUR_RPT], code[LUR_RPT], sl[LUR_RPT];
#pragma unroll
    for (int r = 0; r < LUR_RPT; ++r) {
        sl[r] = t + LUR_NT * r;
        has[r] = sl[r] < nloc;
        act[r] = has[r];
        cur[r] = (int)(base + sl[r]);
        code[r] = (int)rank * R + sl[r];
#pragma unroll
        for (int j = 0; j < LUC_W; ++j)
            row[r][j] = has[r] && j < w ? A.p[(k0 + j) * A.ld + base + sl[r]] : 0.0;
    }
    // every CTA's mbarriers armed before anyone pushes
    luc_cluster_sync();

    // the best active row of this CTA for column c (its value in register 0),
    // pushed with its values into slot `rank` of buffer buf of every CTA:
    // the best row of each warp stages its values, warp 0 picks the CTA's
    // best and sends that warp's stage.  Every step passes this one CTA
    // barrier; the flags read after it (the same values in every thread)
    // decide whether the loop ends, and nothing is pushed when it does.
    auto publish = [&](int c, int buf) -> bool {
        double v = -1.0;
        int rw = 0x7fffffff, cd = -1;
#pragma unroll
        for (int r = 0; r < LUR_RPT; ++r) {
            const double a = fabs(row[r][0]);
            if (act[r] && luc_better(a, cur[r], v, rw)) {
                v = a;
                rw = cur[r];
                cd = code[r];
            }
        }
        lur_warp_best(v, rw, cd);
#pragma unroll
        for (int r = 0; r < LUR_RPT; ++r)
            if (cd >= 0 && cd == code[r]) {
#pragma unroll
                for (int j = 0; j < LUC_W; ++j) wstage[wid][j] = c + j < w ? row[r][j] : 0.0;
            }
        if (lane == 0) {
            red_v[wid] = v;
            red_r[wid] = rw;
            red_c[wid] = cd;
        }
        __syncthreads();
        const bool leave = *(volatile int *)&s_abort != 0 || *(volatile int *)&s_stop != 0;
        if (wid == 0 && !leave && c < w) {
            v = lane < LUR_NT / 32 ? red_v[lane] : -1.0;
            rw = lane < LUR_NT / 32 ? red_r[lane] : 0x7fffffff;
            cd = lane < LUR_NT / 32 ? red_c[lane] : -1;
            int bw = lane;  // the warp that staged it
            static_assert(LUR_NT / 32 == 8, "three rounds reduce the warps' bests");
            luc_best8(v, rw, bw);
            cd = __shfl_sync(0xffffffffu, cd, bw & 31);
            // lane j sends u[j] = column c+1+j (u[31] = 0); lane 31 also
            // the header and u0 = column c
            const double x = cd >= 0 && lane < 31 ? wstage[bw][lane + 1] : 0.0;
            const double x0 = cd >= 0 ? wstage[bw][0] : 0.0;
            const unsigned long long hdr1 =
                (unsigned long long)(unsigned)rw | ((unsigned long long)(unsigned)cd << 32);
            const uint32_t mine = (uint32_t)__cvta_generic_to_shared(&recv[buf].slot[rank]);
            const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&rbar[buf]);
            const uint32_t off = (uint32_t)offsetof(LurSlot, u) + 8u * lane;
#pragma unroll
            for (int d = 0; d < LUC_CL; ++d) {
                uint32_t ra, rb;
                asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(mine), "r"(d));
                asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(rb) : "r"(bar), "r"(d));
                lur_push_f64(ra + off, x, rb);
                if (lane == 31) {
                    lur_push_v2b64(ra, (unsigned long long)__double_as_longlong(v), hdr1, rb);
                    lur_push_f64(ra + (uint32_t)offsetof(LurSlot, u0), x0, rb);
                }
            }
        }
        return leave;
    };
    bool leave = publish(0, 0);

    int c = 0;
#pragma unroll 1
    for (; c < w && !leave; ++c) {
        const int64_t k = k0 + c;
        const int buf = c & 1;
        // this step's candidates from every CTA (bounded wait)
        // (one decision per warp, so the warp's shuffles below stay converged)
        const bool got =
            __all_sync(0xffffffffu, lur_wait(&rbar[buf], (uint32_t)((c >> 1) & 1), &s_abort));
        if (!got) {
            if (atomicExch(&s_abort, 1) == 0) atomicExch(err, LUR_ERR_TIMEOUT);
        }
        double ivp = 0.0, v = -1.0;
        int prow = 0x7fffffff, pcode = -1;
        const LurSlot *ps = nullptr;
        if (got) {
            const LurRecv &rv = recv[buf];
            int q = -1;
            if (lane < LUC_CL) {
                v = rv.slot[lane].v;
                prow = rv.slot[lane].row;
                q = lane;
            }
            static_assert(LUC_CL == 8, "three rounds reduce the CTAs' candidates");
            luc_best8(v, prow, q);
            ps = &rv.slot[q < 0 ? 0 : q];
            pcode = ps->code;
            if (t == 0) {
                if (rank == 0) {
                    if (stop0 == 0 && !(v > 0.0)) *info = (int)(k + 1);
                    if (stop0 == 0 && v > 0.0) ipiv[k] = (int64_t)prow + 1;
                }
            }
        }
        // the same decision in every CTA and every thread that has the data;
        // it takes effect after the step's CTA barrier
        const bool stop = got && (stop0 != 0 || !(v > 0.0));
        if (stop) s_stop = 1;
        if (got && !stop) {
            ivp = 1.0 / ps->u0;
#pragma unroll
            for (int r = 0; r < LUR_RPT; ++r) {
                if (!has[r]) continue;
                if (code[r] == pcode) {
                    // the pivot row: its remaining values are final (the U row)
#pragma unroll
                    for (int j = 0; j < LUC_W; ++j)
                        if (c + j < w) fin[(size_t)(c + j) * R + sl[r]] = row[r][j];
                    cur[r] = (int)k;
                } else if (cur[r] == k) {
                    cur[r] = prow;  // the row the pivot row displaces
                }
                act[r] = cur[r] > k;  // the pivot rows so far are final
            }
            double l[LUR_RPT];
#pragma unroll
            for (int r = 0; r < LUR_RPT; ++r) {
                l[r] = row[r][0] * ivp;
                if (act[r]) fin[(size_t)c * R + sl[r]] = l[r];
            }
            // register j <- column c+1+j (rows that are no longer active
            // compute values that are never used)
#pragma unroll
            for (int j = 0; j < LUC_W - 1; j += 2) {
                const double2 uj = *(const double2 *)&ps->u[j];
#pragma unroll
                for (int r = 0; r < LUR_RPT; ++r) {
                    row[r][j] = fma(-l[r], uj.x, row[r][j + 1]);
                    if (j + 2 < LUC_W) row[r][j + 1] = fma(-l[r], uj.y, row[r][j + 2]);
                }
            }
#pragma unroll
            for (int r = 0; r < LUR_RPT; ++r) row[r][LUC_W - 1] = 0.0;
        }
        // re-arm this buffer for step c+2 (its step-c phase has completed)
        if (t == 0 && got) lur_arm(&rbar[buf], LUC_CL * LUR_SLOT_TX);
        // the candidates of column c+1 (for the last column only the barrier)
        leave = publish(c + 1, buf ^ 1);
        if (leave) break;
    }
    // a singular column stops the panel: the active rows keep their current
    // values from column c on (after a stop, the step's update did not run)
    if (c < w) {
#pragma unroll
        for (int r = 0; r < LUR_RPT; ++r)
            if (act[r]) {
#pragma unroll
                for (int j = 0; j < LUC_W; ++j)
                    if (c + j < w) fin[(size_t)(c + j) * R + sl[r]] = row[r][j];
            }
    }
    luc_cluster_sync();  // no CTA leaves while another may still push into it
    // write the panel back, every slot's row at its final position, and list
    // the moved rows
#pragma unroll
    for (int r = 0; r < LUR_RPT; ++r) {
        if (!has[r]) continue;
        for (int j = 0; j < w; ++j) A.p[(k0 + j) * A.ld + cur[r]] = fin[(size_t)j * R + sl[r]];
        const int orig = (int)(base + sl[r]);
        if (cur[r] < k0 + w) {
            moved[cur[r] - k0] = orig;
        } else if (cur[r] != orig) {
            const int e = atomicAdd(&moved[2 * LUC_W], 1);
            if (MFLAB_IDX_OK(e < LUC_W, 5, e, cur[r])) {
                moved[LUC_W + e] = cur[r];            // ext rows
                moved[2 * LUC_W + 1 + e] = orig;      // ext sources
            }
        }
    }
}

// The panel's interchanges (ipiv[k0 .. k0+w), ascending, as sequential
// swaps) applied to the columns c_lo .. c_hi-1 outside the panel and, right of it, the
// block row U12 = inv(L11) A12 (L11 the panel's unit-lower w x w block): one
// warp per column.  The swaps permute the at most 2w rows involved (rows
// k0 .. k0+w-1 and the pivot rows below them): `moved` lists, for each, the
// original row whose value it receives (written by the cluster panel
// kernel); without the list (the streamed panel) thread 0 replays the swaps
// on the short list of involved rows.  A column is then one gather of its
// involved rows (coalesced across the panel rows) and a 32-step solve in
// registers.
constexpr int LUS_WARPS = 8;

__global__ void __launch_bounds__(32 * LUS_WARPS)
    lu64_swap_trsm_kernel(int64_t c_lo, int64_t c_hi, Mat A, int64_t k0, int w,
                          const int64_t *ipiv, const int *moved, const int *info) {
    if (*info) return;
    __shared__ int rows[2 * LUC_W], src[2 * LUC_W], cnt_s;
    __shared__ double L[LUC_W][LUC_W + 1];
    const int t = threadIdx.x, lane = t % 32, warp = t / 32;
    if (moved) {
        const int ext = moved[2 * LUC_W];
        if (t < w) {
            rows[t] = (int)(k0 + t);
            src[t] = moved[t];
        } else if (t >= LUC_W && t - LUC_W < ext) {
            rows[w + t - LUC_W] = moved[t];
            src[w + t - LUC_W] = moved[2 * LUC_W + 1 + t - LUC_W];
        }
        if (t == 0) cnt_s = w + ext;
    } else if (t == 0) {
        int content[2 * LUC_W];
        int cnt = w;
        for (int i = 0; i < w; ++i) rows[i] = (int)(k0 + i);
        for (int i = 0; i < w; ++i) {
            const int p = (int)(ipiv[k0 + i] - 1);
            bool seen = p < k0 + w;
            for (int j = w; j < cnt && !seen; ++j) seen = rows[j] == p;
            if (!seen) rows[cnt++] = p;
        }
        for (int j = 0; j < cnt; ++j) content[j] = j;
        for (int i = 0; i < w; ++i) {
            const int p = (int)(ipiv[k0 + i] - 1);
            int b = p - (int)k0;
            if (p >= k0 + w)
                for (int j = w; j < cnt; ++j)
                    if (rows[j] == p) b = j;
            const int x = content[i];
            content[i] = content[b];
            content[b] = x;
        }
        for (int j = 0; j < cnt; ++j) src[j] = rows[content[j]];
        cnt_s = cnt;
    }
    for (int e = t; e < w * w; e += 32 * LUS_WARPS) {
        const int i = e % w, j = e / w;
        L[i][j] = A.p[(k0 + j) * A.ld + k0 + i];
    }
    __syncthreads();
    const int cnt = cnt_s;
    const int r0 = rows[lane], s0 = src[lane];
    const bool two = lane + 32 < cnt;
    const int r1 = two ? rows[lane + 32] : 0, s1 = two ? src[lane + 32] : 0;
    // the columns c_lo .. c_hi-1 (a range on one side of the panel)
    for (int64_t c = c_lo + (int64_t)blockIdx.x * LUS_WARPS + warp; c < c_hi;
         c += (int64_t)gridDim.x * LUS_WARPS) {
        double *x = A.p + c * A.ld;
        // gather the involved rows (all reads before any write of this column)
        double v0 = lane < cnt ? x[s0] : 0.0;
        const double v1 = two ? x[s1] : 0.0;
        __syncwarp();
        if (two) x[r1] = v1;
        if (c >= k0 + w) {
            // rows k0 .. k0+w-1 are lanes 0 .. w-1 (rows[i] = k0 + i): solve L11 y = v
            for (int j = 0; j < w; ++j) {
                const double yj = __shfl_sync(0xffffffffu, v0, j);
                if (lane > j && lane < w) v0 = fma(-L[lane][j], yj, v0);
            }
        }
        if (lane < cnt) x[r0] = v0;
    }
}

// swaps (and, right of the panel, the U block row) on columns [c_lo, c_hi)
static int lu64_swap_cols(int64_t c_lo, int64_t c_hi, Mat A, int64_t k0, int w,
                          const int64_t *ipiv, const int *moved, const int *info, int sms,
                          cudaStream_t s) {
    if (c_hi <= c_lo) return MFLAB_OK;
    const int64_t grid = std::min<int64_t>((c_hi - c_lo + LUS_WARPS - 1) / LUS_WARPS, 4 * sms);
    lu64_swap_trsm_kernel<<<(unsigned)grid, 32 * LUS_WARPS, 0, s>>>(c_lo, c_hi, A, k0, w, ipiv,
                                                                    moved, info);
    return record_cuda_error(cudaGetLastError(), "getrf64 swap + trsm");
}

// A[r0:m, c_lo:c_hi] -= L21 U12 of the panel at k0 (width w; r0 = k0 + w)
static int lu64_trailing(mflab_handle *h, int64_t m, int64_t c_lo, int64_t c_hi, Mat A,
                         int64_t k0, int w, void *ws, size_t wsb, const int *info,
                         cudaStream_t s) {
    const int64_t r0 = k0 + w;
    if (c_hi <= c_lo || r0 >= m) return MFLAB_OK;
    const double mone[1] = {-1.0}, one[1] = {1.0};
    // a plain binary64 GEMM (the factor has no reference order to keep); a
    // zero pivot stops the panels, and the updates after it only touch a
    // failed factor
    int rc = dgemm_lt(m - r0, c_hi - c_lo, w, A.p + k0 * A.ld + r0, A.ld,
                      A.p + c_lo * A.ld + k0, A.ld, A.p + c_lo * A.ld + r0, A.ld, -1.0, 1.0,
                      ws, wsb, s);
    if (rc == MFLAB_ERR_UNSUPPORTED)  // no library algorithm: the device kernel
        rc = launch_mm(1, false, false, 0, false, m - r0, c_hi - c_lo, w, A.at(r0, k0),
                       A.at(k0, c_lo), A.at(r0, c_lo), mone, one, s, info);
    return rc;
}

// the high-priority stream and the events of the look-ahead factor
static int lu64_lookahead_streams(mflab_handle *h) {
    cudaError_t e = cudaSuccess;
    if (!h->la_stream) {
        int lo = 0, hi = 0;
        e = cudaDeviceGetStreamPriorityRange(&lo, &hi);
        if (e == cudaSuccess)
            e = cudaStreamCreateWithPriority(&h->la_stream, cudaStreamNonBlocking, hi);
    }
    for (int i = 0; i < 3 && e == cudaSuccess; ++i)
        if (!h->la_ev[i]) e = cudaEventCreateWithFlags(&h->la_ev[i], cudaEventDisableTiming);
    return e == cudaSuccess ? MFLAB_OK : record_cuda_error(e, "getrf64 streams");
}

// panel width nb (4..32): a panel of up to 4096 rows lives in the registers
// of an 8-CTA cluster (lu64_cluster_panel_reg_kernel), one of up to about
// 6000 rows in its shared memory (lu64_cluster_panel_kernel); a taller
// one streams through one CTA (lu64_panel_kernel, whose traffic grows with
// the width).  Look-ahead over two streams: panel p, then the interchanges,
// U block and trailing update of the next panel's columns run on a
// high-priority stream (the panel's critical path), while the interchanges,
// U block and trailing update of all other columns run on the caller's
// stream, overlapping panel p+1.  Step p's next-panel work waits for step
// p-1's other work (which updated those columns); step p's other work waits
// for panel p.  The two moved-row lists and the two GEMM workspaces alternate
// or belong to one stream each, so no buffer is shared by work in flight.
static int getrf64_fast(mflab_handle *h, int64_t m, int64_t n, Mat A, int64_t *ipiv, int *info,
                        cudaStream_t s, int nb) {
    cudaError_t e = cudaMemsetAsync(info, 0, sizeof(int), s);
    if (e != cudaSuccess) return record_cuda_error(e, "getrf info");
    const int64_t kmax = m < n ? m : n;
    if (kmax == 0) return MFLAB_OK;
    int64_t tot = m * n;
    nonfinite_kernel<1><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(m, n, A, 0, info);
    int rc = record_cuda_error(cudaGetLastError(), "getrf check");
    if (rc) return rc;
    // two workspaces of the library's binary64 GEMM (one per stream), then
    // two moved-row lists of the cluster panel (alternating panels)
    const size_t wsb = (size_t)32 << 20, mvb = 4 * LUC_W * sizeof(int);
    rc = mflab_reserve_scratch(h, 2 * wsb + 2 * mvb);
    if (rc) return rc;
    void *ws[2] = {h->scratch, (char *)h->scratch + wsb};
    int *movedb[2] = {(int *)((char *)h->scratch + 2 * wsb),
                      (int *)((char *)h->scratch + 2 * wsb + mvb)};
    const int NB = nb < 4 ? 4 : (nb > LUC_W ? LUC_W : nb);
    static std::atomic<unsigned long long> luc_configured{0};
    rc = set_smem_once((const void *)lu64_cluster_panel_kernel, LUC_SMEM_MAX, luc_configured,
                       "lu64 cluster panel attribute");
    if (rc) return rc;
    static std::atomic<unsigned long long> lur_configured{0};
    rc = set_smem_once((const void *)lu64_cluster_panel_reg_kernel, LUC_SMEM_MAX, lur_configured,
                       "lu64 register panel attribute");
    if (rc) return rc;
    rc = lu64_lookahead_streams(h);
    if (rc) return rc;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaStream_t sp = h->la_stream;  // the panels' stream
    cudaEvent_t ev_fork = h->la_ev[0], ev_panel = h->la_ev[1], ev_rest = h->la_ev[2];
    e = cudaEventRecord(ev_fork, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(sp, ev_fork, 0);
    if (e != cudaSuccess) return record_cuda_error(e, "getrf64 fork");
    int p = 0;
    for (int64_t k0 = 0; k0 < kmax && rc == MFLAB_OK; k0 += NB, ++p) {
        const int w = (int)(kmax - k0 < NB ? kmax - k0 : NB);
        int *moved = movedb[p & 1];
        // the panel in a cluster's registers or shared memory when it fits,
        // else streamed through one CTA
        const int64_t mr = m - k0, R = (mr + LUC_CL - 1) / LUC_CL;
        const size_t smem = luc_smem(R, mr);
        const bool cluster = smem <= (size_t)LUC_SMEM_MAX && R <= 0x7fffffff;
        if (cluster && R <= LUR_NT * LUR_RPT && lur_smem(R) <= (size_t)LUC_SMEM_MAX)
            lu64_cluster_panel_reg_kernel<<<LUC_CL, LUR_NT, lur_smem(R), sp>>>(
                m, A, k0, w, (int)R, ipiv, info, moved, h->dev_flags + 1);
        else if (cluster)
            lu64_cluster_panel_kernel<<<LUC_CL, LUC_NT, smem, sp>>>(m, A, k0, w, (int)R, ipiv,
                                                                    info, moved);
        else
            lu64_panel_kernel<<<1, LU64_NT, 0, sp>>>(m, A, k0, w, ipiv, info);
        rc = record_cuda_error(cudaGetLastError(), "getrf64 panel");
        if (rc) break;
        const int *mv = cluster ? moved : nullptr;
        e = cudaEventRecord(ev_panel, sp);
        // the next panel's columns, on the panels' stream, after the other
        // work of the previous step
        const int64_t nx0 = k0 + w, nx1 = std::min<int64_t>(n, nx0 + NB);
        if (e == cudaSuccess && p > 0) e = cudaStreamWaitEvent(sp, ev_rest, 0);
        if (e != cudaSuccess) return record_cuda_error(e, "getrf64 look-ahead");
        rc = lu64_swap_cols(nx0, nx1, A, k0, w, ipiv, mv, info, sms, sp);
        if (!rc) rc = lu64_trailing(h, m, nx0, nx1, A, k0, w, ws[0], wsb, info, sp);
        if (rc) break;
        // every other column, on the caller's stream, after the panel
        e = cudaStreamWaitEvent(s, ev_panel, 0);
        if (e != cudaSuccess) return record_cuda_error(e, "getrf64 look-ahead");
        rc = lu64_swap_cols(0, k0, A, k0, w, ipiv, mv, info, sms, s);
        if (!rc) rc = lu64_swap_cols(nx1, n, A, k0, w, ipiv, mv, info, sms, s);
        if (!rc) rc = lu64_trailing(h, m, nx1, n, A, k0, w, ws[1], wsb, info, s);
        if (!rc) {
            e = cudaEventRecord(ev_rest, s);
            if (e != cudaSuccess) rc = record_cuda_error(e, "getrf64 look-ahead");
        }
    }
    // join: the caller's stream waits for the panels' stream
    e = cudaEventRecord(ev_fork, sp);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ev_fork, 0);
    if (e != cudaSuccess && rc == MFLAB_OK) rc = record_cuda_error(e, "getrf64 join");
    return rc;
}

template <int N>
static int getrf_n(int64_t m, int64_t n, Mat A, int64_t *ipiv, int64_t block, int *info,
                   cudaStream_t s) {
    const double mone[4] = {-1.0, 0.0, 0.0, 0.0}, one[4] = {1.0, 0.0, 0.0, 0.0};
    cudaError_t e = cudaMemsetAsync(info, 0, sizeof(int), s);
    if (e != cudaSuccess) return record_cuda_error(e, "getrf info");
    const int64_t kmax = m < n ? m : n;
    if (kmax == 0) return MFLAB_OK;
    int64_t tot = m * n;
    nonfinite_kernel<N><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(m, n, A, 0, info);
    int rc = record_cuda_error(cudaGetLastError(), "getrf check");
    if (rc) return rc;
    for (int64_t first = 0; first < kmax; first += block) {
        const int64_t last = first + block - 1 < kmax - 1 ? first + block - 1 : kmax - 1;
        for (int64_t k = first; k <= last; ++k) {
            // the panel's steps are programmatic dependents of one another
            rc = launch_programmatic(lu_pivot_kernel<N, 512>, dim3(1), dim3(512), 0, s,
                                     "getrf pivot", m, first, last + 1, A, k, ipiv, info);
            if (rc) return rc;
            if (k < last && k + 1 < m) {
                const int64_t rows = m - k - 1;
                rc = launch_programmatic(lu_rank1_kernel<N>, dim3((unsigned)((rows + 127) / 128)),
                                         dim3(128), 0, s, "getrf rank1", m, A, k, last,
                                         (const int *)info);
                if (rc) return rc;
            }
        }
        // the panel's interchanges on the other columns (also after a zero
        // pivot, for the steps before it)
        if (n > last - first + 1) {
            const int64_t cols = n - (last - first + 1);
            lu_swap_rest_kernel<N><<<(unsigned)((cols + 127) / 128), 128, 0, s>>>(n, A, first, last,
                                                                                  ipiv, info);
            rc = record_cuda_error(cudaGetLastError(), "getrf swaps");
            if (rc) return rc;
        }
        if (last < n - 1) {
            const int64_t w = last - first + 1, rest = n - 1 - last;
            rc = launch_trsm_info(N, 0, 0, 0, 1, w, rest, A.at(first, first), A.at(first, last + 1),
                                  one, s, info);
            if (rc) return rc;
            if (last < m - 1) {
                rc = launch_mm(N, false, false, 0, N == 3, m - 1 - last, rest, w, A.at(last + 1, first),
                               A.at(first, last + 1), A.at(last + 1, last + 1), mone, one, s, info);
                if (rc) return rc;
            }
        }
    }
    return MFLAB_OK;
}

// LU with INT8 trailing updates: panels of nb columns factored by the blocked
// algorithm above (pivot search and interchanges, rank-1 updates,
// TRSM and GEMM restricted to the panel's columns), then U12 = L11^-1 A12 and
// A22 -= L21 U12 through the modular INT8 route.  The device info word is read
// after every panel (one synchronisation each) so that a zero pivot stops the
// factorization before the next trailing update.
template <int N>
static int getrf_ozaki_n(mflab_handle *h, int64_t m, int64_t n, Mat A, int64_t *ipiv, int64_t nb,
                         int64_t block, int moduli, int *info, cudaStream_t s) {
    const double mone[4] = {-1.0, 0.0, 0.0, 0.0}, one[4] = {1.0, 0.0, 0.0, 0.0};
    cudaError_t e = cudaMemsetAsync(info, 0, sizeof(int), s);
    if (e != cudaSuccess) return record_cuda_error(e, "getrf info");
    const int64_t kmax = m < n ? m : n;
    if (kmax == 0) return MFLAB_OK;
    int64_t tot = m * n;
    nonfinite_kernel<N><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(m, n, A, 0, info);
    int rc = record_cuda_error(cudaGetLastError(), "getrf check");
    if (rc) return rc;
    for (int64_t j0 = 0; j0 < kmax; j0 += nb) {
        const int64_t j1 = j0 + nb < kmax ? j0 + nb : kmax;  // panel columns [j0, j1)
        for (int64_t first = j0; first < j1; first += block) {
            const int64_t last = first + block - 1 < j1 - 1 ? first + block - 1 : j1 - 1;
            for (int64_t k = first; k <= last; ++k) {
                lu_pivot_kernel<N, 512><<<1, 512, 0, s>>>(m, first, last + 1, A, k, ipiv, info);
                rc = record_cuda_error(cudaGetLastError(), "getrf pivot");
                if (rc) return rc;
                if (k < last && k + 1 < m) {
                    const int64_t rows = m - k - 1;
                    lu_rank1_kernel<N><<<(unsigned)((rows + 127) / 128), 128, 0, s>>>(m, A, k, last,
                                                                                     info);
                    rc = record_cuda_error(cudaGetLastError(), "getrf rank1");
                    if (rc) return rc;
                }
            }
            if (n > last - first + 1) {
                const int64_t cols = n - (last - first + 1);
                lu_swap_rest_kernel<N><<<(unsigned)((cols + 127) / 128), 128, 0, s>>>(
                    n, A, first, last, ipiv, info);
                rc = record_cuda_error(cudaGetLastError(), "getrf swaps");
                if (rc) return rc;
            }
            if (last < j1 - 1) {
                const int64_t w = last - first + 1, cols = j1 - 1 - last;
                rc = launch_trsm_info(N, 0, 0, 0, 1, w, cols, A.at(first, first),
                                      A.at(first, last + 1), one, s, info);
                if (rc) return rc;
                if (last < m - 1) {
                    rc = launch_mm(N, false, false, 0, N == 3, m - 1 - last, cols, w,
                                   A.at(last + 1, first), A.at(first, last + 1),
                                   A.at(last + 1, last + 1), mone, one, s, info);
                    if (rc) return rc;
                }
            }
        }
        int hinfo = 0;
        e = cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return record_cuda_error(e, "getrf info read");
        if (hinfo != 0) return MFLAB_OK;
        if (j1 < n) {
            const int64_t w = j1 - j0;
            rc = launch_trsm_info(N, 0, 0, 0, 1, w, n - j1, A.at(j0, j0), A.at(j0, j1), one, s,
                                  info);
            if (rc) return rc;
            if (j1 < m) {
                rc = ozaki_crt_gemm(h, N, moduli, m - j1, n - j1, w, A.at(j1, j0), A.at(j0, j1),
                                    A.at(j1, j1), mone, one, s, nullptr);
                if (rc) return rc;
            }
        }
    }
    return MFLAB_OK;
}

// apply the recorded row interchanges to the right-hand sides (solve.jl:85-113);
// one thread per column, interchanges in ascending k
template <int N>
__global__ void apply_pivots_kernel(int64_t nrhs, Mat B, const int64_t *ipiv, int64_t count,
                                    int reverse) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nrhs) return;
    for (int64_t s = 0; s < count; ++s) {
        const int64_t k = reverse ? count - 1 - s : s;
        const int64_t p = ipiv[k] - 1;
        if (p != k) {
#pragma unroll
            for (int l = 0; l < N; ++l) {
                double *x = B.p + l * B.ls + c * B.ld;
                double tmp = x[k];
                x[k] = x[p];
                x[p] = tmp;
            }
        }
    }
}

// The interchanges ipiv[0..n) (1-based, applied in ascending order) as one
// gather: a single thread replays the swaps on an index array in shared
// memory (row k ends up holding original row perm[k]), then every entry
// moves once.  Same result as the sequential swaps, without a dependent
// global-memory chain per right-hand side.
__global__ void pivot_perm_kernel(int64_t n, const int64_t *ipiv, int *perm) {
    extern __shared__ int sidx[];  // [n] indices, then [n] pivots
    int *spiv = sidx + n;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        sidx[i] = (int)i;
        spiv[i] = (int)(ipiv[i] - 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int64_t k = 0; k < n; ++k) {
            const int64_t p = spiv[k];
            if (p != k) {
                const int t = sidx[k];
                sidx[k] = sidx[p];
                sidx[p] = t;
            }
        }
    }
    __syncthreads();
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) perm[i] = sidx[i];
}

template <int N>
__global__ void gather_rows_kernel(int64_t n, int64_t nrhs, Mat B, const double *src,
                                   const int *perm) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * nrhs) return;
    const int64_t i = e % n, j = e / n;
#pragma unroll
    for (int l = 0; l < N; ++l)
        B.p[l * B.ls + j * B.ld + i] = src[(l * nrhs + j) * n + perm[i]];
}

constexpr int64_t PIVOT_PERM_MAXN = 24576;  // indices and pivots in shared memory (192 KB)

template <int N>
static int apply_pivots_gather(mflab_handle *h, int64_t n, int64_t nrhs, Mat B,
                               const int64_t *ipiv, cudaStream_t s) {
    const size_t plane = (size_t)n * nrhs;
    int rc = mflab_reserve_scratch(h, plane * N * sizeof(double) + (size_t)n * sizeof(int));
    if (rc) return rc;
    double *copy = (double *)h->scratch;
    int *perm = (int *)(copy + plane * N);
    const size_t smem = 2 * (size_t)n * sizeof(int);
    static std::atomic<unsigned long long> configured{0};
    rc = set_smem_once((const void *)pivot_perm_kernel, (int)(2 * PIVOT_PERM_MAXN * sizeof(int)),
                       configured, "pivot perm attribute");
    if (rc) return rc;
    pivot_perm_kernel<<<1, 256, smem, s>>>(n, ipiv, perm);
    for (int l = 0; l < N; ++l) {
        cudaError_t e = cudaMemcpy2DAsync(copy + l * plane, n * sizeof(double), B.p + l * B.ls,
                                          B.ld * sizeof(double), n * sizeof(double), nrhs,
                                          cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return record_cuda_error(e, "getrs pivot copy");
    }
    gather_rows_kernel<N><<<(unsigned)((plane + 255) / 256), 256, 0, s>>>(n, nrhs, B, copy, perm);
    return record_cuda_error(cudaGetLastError(), "getrs pivots");
}

// --------------------------------------------------------- diagnostics ---
// Partial reductions of max |A(r,c)| and finiteness over a region
// (0 all, 1 lower r >= c, 2 upper r <= c): one record per CTA.
template <int N, int NT>
__global__ void __launch_bounds__(NT) maxabs_partial_kernel(int64_t m, int64_t n, Mat A,
                                                            int region, double *part) {
    __shared__ double sval[NT][N];
    __shared__ int sfin[NT];
    const int t = threadIdx.x;
    mf<N> best = from_double<N>(0.0);
    int fin = 1;
    const int64_t tot = m * n;
    for (int64_t idx = (int64_t)blockIdx.x * NT + t; idx < tot; idx += (int64_t)gridDim.x * NT) {
        const int64_t r = idx % m, c = idx / m;
        if (region == 1 && r < c) continue;
        if (region == 2 && r > c) continue;
        mf<N> v = load_mf<N>(A.p, A.ld, A.ls, r, c);
        if (!isfinite_mf(v)) fin = 0;
        best = max_mf(best, abs_mf(v));
    }
#pragma unroll
    for (int l = 0; l < N; ++l) sval[t][l] = best.v[l];
    sfin[t] = fin;
    __syncthreads();
    for (int off = NT / 2; off > 0; off >>= 1) {
        if (t < off) {
            mf<N> a, b;
#pragma unroll
            for (int l = 0; l < N; ++l) {
                a.v[l] = sval[t][l];
                b.v[l] = sval[t + off][l];
            }
            mf<N> r = max_mf(a, b);
#pragma unroll
            for (int l = 0; l < N; ++l) sval[t][l] = r.v[l];
            sfin[t] = sfin[t] && sfin[t + off];
        }
        __syncthreads();
    }
    if (t == 0) {
#pragma unroll
        for (int l = 0; l < N; ++l) part[blockIdx.x * (N + 1) + l] = sval[0][l];
        part[blockIdx.x * (N + 1) + N] = sfin[0] ? 1.0 : 0.0;
    }
}

template <int N>
__global__ void maxabs_final_kernel(int nparts, const double *part, double *out) {
    mf<N> best = from_double<N>(0.0);
    int fin = 1;
    for (int i = 0; i < nparts; ++i) {
        mf<N> v;
#pragma unroll
        for (int l = 0; l < N; ++l) v.v[l] = part[i * (N + 1) + l];
        best = max_mf(best, v);
        if (part[i * (N + 1) + N] == 0.0) fin = 0;
    }
#pragma unroll
    for (int l = 0; l < N; ++l) out[l] = best.v[l];
    out[N] = fin ? 1.0 : 0.0;
}

// O(n) tail of the diagnostics, one thread.  Layout of `out` (N doubles per
// value): [0] min |diag|, [1] max |diag|, [2] max/min (Inf when min == 0),
// [3] ratio num/den of the two given values (growth), [4] accepted count,
// [5] has-range flag.  diagonal_magnitude_range over the first `count`
// entries (diagnostics.jl:21-31).
template <int N>
__global__ void diag_tail_kernel(Mat A, int64_t count, const double *num, const double *den,
                                 double *out) {
    mf<N> mn = from_double<N>(0.0), mx = from_double<N>(0.0);
    if (count > 0) {
        mn = abs_mf(load_mf<N>(A.p, A.ld, A.ls, 0, 0));
        mx = mn;
        for (int64_t i = 1; i < count; ++i) {
            mf<N> v = abs_mf(load_mf<N>(A.p, A.ld, A.ls, i, i));
            mn = min_mf(mn, v);
            mx = max_mf(mx, v);
        }
    }
    mf<N> spread;
    if (iszero(mn)) spread = from_double<N>(__longlong_as_double(0x7ff0000000000000LL));
    else spread = div(mx, mn);
    mf<N> ratio = from_double<N>(0.0);
    if (num && den) {
        mf<N> a, b;
#pragma unroll
        for (int l = 0; l < N; ++l) {
            a.v[l] = num[l];
            b.v[l] = den[l];
        }
        ratio = iszero(b) ? from_double<N>(0.0) : div(a, b);
    }
#pragma unroll
    for (int l = 0; l < N; ++l) {
        out[0 * N + l] = mn.v[l];
        out[1 * N + l] = mx.v[l];
        out[2 * N + l] = spread.v[l];
        out[3 * N + l] = ratio.v[l];
    }
    out[4 * N] = (double)count;
    out[4 * N + 1] = count > 0 ? 1.0 : 0.0;
}

template <int N>
static int maxabs_n(int64_t m, int64_t n, Mat A, int region, double *part, int nparts,
                    double *out, cudaStream_t s) {
    maxabs_partial_kernel<N, 256><<<nparts, 256, 0, s>>>(m, n, A, region, part);
    int rc = record_cuda_error(cudaGetLastError(), "maxabs partial");
    if (rc) return rc;
    maxabs_final_kernel<N><<<1, 1, 0, s>>>(nparts, part, out);
    return record_cuda_error(cudaGetLastError(), "maxabs final");
}

}  // namespace mfl

using mfl::Mat;

#define MFL_DISPATCH(N, call)                                       \
    switch (N) {                                                    \
    case 2: return call<2>;                                         \
    case 3: return call<3>;                                         \
    case 4: return call<4>;                                         \
    default: return MFLAB_ERR_UNSUPPORTED;                          \
    }

extern "C" int mflab_potrf(mflab_handle *h, void *stream, int limbs, int64_t n, double *A,
                           int64_t lda, int64_t lsa, int64_t block, int *info) {
    MFLAB_RANGE("mflab_potrf");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (n < 0 || (n > 0 && lda < n) || !info) return MFLAB_ERR_ARG;
    if (block < 1) block = 1;
    if (block > 32) return MFLAB_ERR_UNSUPPORTED;
    Mat a{A, lda, lsa};
    cudaStream_t s = (cudaStream_t)stream;
    switch (limbs) {
    case 2: return mfl::potrf_n<2>(h, n, a, block, info, s);
    case 3: return mfl::potrf_n<3>(h, n, a, block, info, s);
    default: return mfl::potrf_n<4>(h, n, a, block, info, s);
    }
}

extern "C" int mflab_potrf_ozaki(mflab_handle *h, void *stream, int limbs, int moduli, int64_t n,
                                 double *A, int64_t lda, int64_t lsa, int64_t nb, int64_t block,
                                 int *info) {
    MFLAB_RANGE("mflab_potrf_ozaki");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (n < 0 || (n > 0 && lda < n) || !info || moduli < 0) return MFLAB_ERR_ARG;
    if (block < 1) block = 1;
    if (block > 32) return MFLAB_ERR_UNSUPPORTED;
    if (nb < block) nb = block;
    Mat a{A, lda, lsa};
    cudaStream_t s = (cudaStream_t)stream;
    switch (limbs) {
    case 2: return mfl::potrf_ozaki_n<2>(h, n, a, nb, block, moduli, info, s);
    case 3: return mfl::potrf_ozaki_n<3>(h, n, a, nb, block, moduli, info, s);
    default: return mfl::potrf_ozaki_n<4>(h, n, a, nb, block, moduli, info, s);
    }
}

extern "C" int mflab_potrs(mflab_handle *h, void *stream, int limbs, int64_t n, int64_t nrhs,
                           const double *L, int64_t ldl, int64_t lsl, double *B, int64_t ldb,
                           int64_t lsb) {
    MFLAB_RANGE("mflab_potrs");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (n < 0 || nrhs < 0 || (n > 0 && (ldl < n || ldb < n))) return MFLAB_ERR_ARG;
    const double one[4] = {1.0, 0.0, 0.0, 0.0};
    cudaStream_t s = (cudaStream_t)stream;
    Mat a{(double *)L, ldl, lsl}, b{B, ldb, lsb};
    int rc = mfl::launch_trsm_info(limbs, 0, 0, 0, 0, n, nrhs, a, b, one, s, nullptr, h->solve_order);
    if (rc) return rc;
    return mfl::launch_trsm_info(limbs, 0, 0, 1, 0, n, nrhs, a, b, one, s, nullptr, h->solve_order);
}

extern "C" int mflab_getrf(mflab_handle *h, void *stream, int limbs, int64_t m, int64_t n,
                           double *A, int64_t lda, int64_t lsa, int64_t *ipiv, int64_t block,
                           int *info) {
    MFLAB_RANGE("mflab_getrf");
    if (!h || !(limbs == 1 || mfl::valid_limbs(limbs))) return MFLAB_ERR_UNSUPPORTED;
    if (m < 0 || n < 0 || (m > 0 && lda < m) || !info || (m > 0 && n > 0 && !ipiv))
        return MFLAB_ERR_ARG;
    if (block < 1) block = 1;
    Mat a{A, lda, lsa};
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t kmax = m < n ? m : n;
    if (kmax > 0) {
        // ipiv = 1:kmax, as the reference initialises it (lu.jl:16-28)
        mfl::iota1_kernel<<<(unsigned)((kmax + 255) / 256), 256, 0, s>>>(ipiv, kmax);
        int rc = mfl::record_cuda_error(cudaGetLastError(), "getrf ipiv");
        if (rc) return rc;
    }
    switch (limbs) {
    case 1: return mfl::getrf64_fast(h, m, n, a, ipiv, info, s, (int)block);
    case 2: return mfl::getrf_n<2>(m, n, a, ipiv, block, info, s);
    case 3: return mfl::getrf_n<3>(m, n, a, ipiv, block, info, s);
    default: return mfl::getrf_n<4>(m, n, a, ipiv, block, info, s);
    }
}

extern "C" int mflab_getrf_ozaki(mflab_handle *h, void *stream, int limbs, int moduli, int64_t m,
                                 int64_t n, double *A, int64_t lda, int64_t lsa, int64_t *ipiv,
                                 int64_t nb, int64_t block, int *info) {
    MFLAB_RANGE("mflab_getrf_ozaki");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (m < 0 || n < 0 || (m > 0 && lda < m) || !info || (m > 0 && n > 0 && !ipiv) || moduli < 0)
        return MFLAB_ERR_ARG;
    if (block < 1) block = 1;
    if (nb < block) nb = block;
    Mat a{A, lda, lsa};
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t kmax = m < n ? m : n;
    if (kmax > 0) {
        mfl::iota1_kernel<<<(unsigned)((kmax + 255) / 256), 256, 0, s>>>(ipiv, kmax);
        int rc = mfl::record_cuda_error(cudaGetLastError(), "getrf ipiv");
        if (rc) return rc;
    }
    switch (limbs) {
    case 2: return mfl::getrf_ozaki_n<2>(h, m, n, a, ipiv, nb, block, moduli, info, s);
    case 3: return mfl::getrf_ozaki_n<3>(h, m, n, a, ipiv, nb, block, moduli, info, s);
    default: return mfl::getrf_ozaki_n<4>(h, m, n, a, ipiv, nb, block, moduli, info, s);
    }
}

extern "C" int mflab_getrs(mflab_handle *h, void *stream, int limbs, int64_t n, int64_t nrhs,
                           const double *LU, int64_t ldl, int64_t lsl, const int64_t *ipiv,
                           double *B, int64_t ldb, int64_t lsb) {
    MFLAB_RANGE("mflab_getrs");
    if (!h || !(limbs == 1 || mfl::valid_limbs(limbs))) return MFLAB_ERR_UNSUPPORTED;
    if (n < 0 || nrhs < 0 || (n > 0 && (ldl < n || ldb < n || !ipiv))) return MFLAB_ERR_ARG;
    if (n == 0 || nrhs == 0) return MFLAB_OK;
    const double one[4] = {1.0, 0.0, 0.0, 0.0};
    cudaStream_t s = (cudaStream_t)stream;
    Mat a{(double *)LU, ldl, lsl}, b{B, ldb, lsb};
    unsigned g = (unsigned)((nrhs + 127) / 128);
    int rc = MFLAB_OK;
    if (n <= mfl::PIVOT_PERM_MAXN) {
        switch (limbs) {
        case 1: rc = mfl::apply_pivots_gather<1>(h, n, nrhs, b, ipiv, s); break;
        case 2: rc = mfl::apply_pivots_gather<2>(h, n, nrhs, b, ipiv, s); break;
        case 3: rc = mfl::apply_pivots_gather<3>(h, n, nrhs, b, ipiv, s); break;
        default: rc = mfl::apply_pivots_gather<4>(h, n, nrhs, b, ipiv, s); break;
        }
    } else {
        switch (limbs) {
        case 1: mfl::apply_pivots_kernel<1><<<g, 128, 0, s>>>(nrhs, b, ipiv, n, 0); break;
        case 2: mfl::apply_pivots_kernel<2><<<g, 128, 0, s>>>(nrhs, b, ipiv, n, 0); break;
        case 3: mfl::apply_pivots_kernel<3><<<g, 128, 0, s>>>(nrhs, b, ipiv, n, 0); break;
        default: mfl::apply_pivots_kernel<4><<<g, 128, 0, s>>>(nrhs, b, ipiv, n, 0); break;
        }
        rc = mfl::record_cuda_error(cudaGetLastError(), "getrs pivots");
    }
    if (rc) return rc;
    rc = mfl::launch_trsm_info(limbs, 0, 0, 0, 1, n, nrhs, a, b, one, s, nullptr, h->solve_order);
    if (rc) return rc;
    return mfl::launch_trsm_info(limbs, 0, 1, 0, 0, n, nrhs, a, b, one, s, nullptr, h->solve_order);
}

extern "C" int mflab_max_abs(mflab_handle *h, void *stream, int limbs, int64_t m, int64_t n,
                             const double *A, int64_t lda, int64_t lsa, int region, double *out) {
    MFLAB_RANGE("mflab_max_abs");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (region < 0 || region > 2) return MFLAB_ERR_FLAG;
    if (m < 0 || n < 0 || !out) return MFLAB_ERR_ARG;
    const int nparts = 296;
    int rc = mflab_reserve_scratch(h, sizeof(double) * nparts * (limbs + 1));
    if (rc) return rc;
    double *part = (double *)h->scratch;
    Mat a{(double *)A, lda, lsa};
    cudaStream_t s = (cudaStream_t)stream;
    switch (limbs) {
    case 2: return mfl::maxabs_n<2>(m, n, a, region, part, nparts, out, s);
    case 3: return mfl::maxabs_n<3>(m, n, a, region, part, nparts, out, s);
    default: return mfl::maxabs_n<4>(m, n, a, region, part, nparts, out, s);
    }
}

extern "C" int mflab_diag_summary(mflab_handle *h, void *stream, int limbs, const double *A,
                                  int64_t lda, int64_t lsa, int64_t count, const double *num,
                                  const double *den, double *out) {
    MFLAB_RANGE("mflab_diag_summary");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (count < 0 || !out) return MFLAB_ERR_ARG;
    Mat a{(double *)A, lda, lsa};
    cudaStream_t s = (cudaStream_t)stream;
    switch (limbs) {
    case 2: mfl::diag_tail_kernel<2><<<1, 1, 0, s>>>(a, count, num, den, out); break;
    case 3: mfl::diag_tail_kernel<3><<<1, 1, 0, s>>>(a, count, num, den, out); break;
    default: mfl::diag_tail_kernel<4><<<1, 1, 0, s>>>(a, count, num, den, out); break;
    }
    return mfl::record_cuda_error(cudaGetLastError(), "diag summary");
}
