// Rank-revealing pivoted Cholesky (cholesky_pivoted.jl:65-175 of
// MultiFloatLinearAlgebra.jl): lower triangle mirrored once, then for each k
// the largest remaining diagonal (first index on ties) is swapped to k by a
// symmetric row + column swap, the column below is divided by its square
// root and the whole trailing square receives the rank-one update
// A[r,c] -= A[r,k] * A[c,k].  The upper triangle is updated too: a later
// symmetric swap moves upper entries into the lower triangle, so keeping the
// full square is what makes the result the reference's.
//
// Launch plan, no host round trip: init, finiteness check, mirror, then per
// step one single-CTA pivot kernel (search, stop decisions, swaps, column
// scaling) and one grid-wide update kernel.  A stop (rank reveal, failure,
// non-finite input) is a device word every later kernel reads first.  Each
// update reads and writes the (n-k-1)^2 trailing entries once: HBM/L2 bound.
#include "mf_device.cuh"
#include "mflab_internal.h"

namespace mfl {

struct PstrfState {
    int64_t rank;   // retained rank (n unless a stop sets it)
    int64_t info;   // 0, -1 non-finite lower triangle, k > 0 first non-positive pivot
    int64_t stop;   // set by the step that ends the factorization
    int64_t pad;
    double first[4];  // sqrt of the first pivot diagonal
};

__global__ void pstrf_init_kernel(PstrfState *st, int64_t n, int64_t *perm) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        perm[i] = i + 1;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->rank = n;
        st->info = 0;
        st->stop = 0;
    }
}

template <int N>
__global__ void pstrf_check_kernel(int64_t n, Mat A, PstrfState *st) {
    const int64_t total = n * n;
    bool bad = false;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = e / n, r = e % n;
        if (r < c) continue;
#pragma unroll
        for (int l = 0; l < N; ++l) bad = bad || !isfinite(A.p[l * A.ls + c * A.ld + r]);
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) {
        st->info = -1;  // every writer stores the same values
        st->rank = 0;
        st->stop = 1;
    }
}

// upper triangle <- lower triangle (cholesky_pivoted.jl:99-103), skipped for
// non-finite input, which is returned unchanged
template <int N>
__global__ void pstrf_mirror_kernel(int64_t n, Mat A, const PstrfState *st) {
    if (st->info == -1) return;
    const int64_t total = n * n;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = e / n, r = e % n;
        if (r >= c) continue;
#pragma unroll
        for (int l = 0; l < N; ++l) A.p[l * A.ls + c * A.ld + r] = A.p[l * A.ls + r * A.ld + c];
    }
}

constexpr int PSTRF_PIVOT_THREADS = 1024;

template <int N>
__global__ void __launch_bounds__(PSTRF_PIVOT_THREADS)
    pstrf_pivot_kernel(int64_t n, int64_t k, Mat A, int64_t *perm, PstrfState *st, scal<N> tol) {
    __shared__ double sval[N][PSTRF_PIVOT_THREADS];
    __shared__ int64_t sidx[PSTRF_PIVOT_THREADS];
    __shared__ int go;
    __shared__ double spiv[N];
    __shared__ int64_t sp;
    // the steps are programmatic dependents of one another: wait for the
    // previous grid, let the next one be placed meanwhile
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (st->stop) return;
    const int tid = threadIdx.x;
    // largest diagonal in k..n-1, the first index among equals
    int64_t bi = -1;
    mf<N> bv = from_double<N>(0.0);
    for (int64_t i = k + tid; i < n; i += PSTRF_PIVOT_THREADS) {
        const mf<N> v = load_mf<N>(A.p, A.ld, A.ls, i, i);
        if (bi < 0 || gt(v, bv)) {
            bi = i;
            bv = v;
        }
    }
#pragma unroll
    for (int l = 0; l < N; ++l) sval[l][tid] = bv.v[l];
    sidx[tid] = bi;
    __syncthreads();
    for (int s = PSTRF_PIVOT_THREADS / 2; s > 0; s >>= 1) {
        if (tid < s) {
            const int64_t ia = sidx[tid], ib = sidx[tid + s];
            if (ib >= 0) {
                mf<N> va, vb;
#pragma unroll
                for (int l = 0; l < N; ++l) {
                    va.v[l] = sval[l][tid];
                    vb.v[l] = sval[l][tid + s];
                }
                if (ia < 0 || gt(vb, va) || (!gt(va, vb) && ib < ia)) {
#pragma unroll
                    for (int l = 0; l < N; ++l) sval[l][tid] = vb.v[l];
                    sidx[tid] = ib;
                }
            }
        }
        __syncthreads();
    }
    if (tid == 0) {
        const int64_t p = sidx[0];
        mf<N> pd;
#pragma unroll
        for (int l = 0; l < N; ++l) pd.v[l] = sval[l][0];
        const mf<N> zero = from_double<N>(0.0), t = tol.get();
        const bool use_tol = !iszero(t);
        int ok = 1;
        if (k == 0) {
            if (!gt(pd, zero)) {
                st->rank = 0;
                st->info = 1;
                ok = 0;
            } else {
                const mf<N> f = sqrt_mf(pd);
#pragma unroll
                for (int l = 0; l < N; ++l) st->first[l] = f.v[l];
            }
        }
        mf<N> first;
#pragma unroll
        for (int l = 0; l < N; ++l) first.v[l] = st->first[l];
        mf<N> piv = zero;
        if (ok && ge(zero, pd)) {
            // a roundoff-sized negative pivot under a tolerance is a rank stop
            const mf<N> thr = mul(t, first);
            st->rank = k;
            if (!(use_tol && ge(mul(thr, thr), abs_mf(pd)))) st->info = k + 1;
            ok = 0;
        }
        if (ok) {
            piv = sqrt_mf(pd);
            if (use_tol && ge(mul(t, first), piv)) {
                st->rank = k;
                ok = 0;
            }
        }
        if (!ok) st->stop = 1;
        go = ok;
        sp = p;
#pragma unroll
        for (int l = 0; l < N; ++l) spiv[l] = piv.v[l];
    }
    __syncthreads();
    if (!go) return;
    const int64_t p = sp;
    if (p != k) {
        for (int64_t c = tid; c < n; c += PSTRF_PIVOT_THREADS)
#pragma unroll
            for (int l = 0; l < N; ++l) {
                double *a = A.p + l * A.ls + c * A.ld;
                const double t = a[k];
                a[k] = a[p];
                a[p] = t;
            }
        __syncthreads();
        for (int64_t r = tid; r < n; r += PSTRF_PIVOT_THREADS)
#pragma unroll
            for (int l = 0; l < N; ++l) {
                double *a = A.p + l * A.ls + r;
                const double t = a[k * A.ld];
                a[k * A.ld] = a[p * A.ld];
                a[p * A.ld] = t;
            }
        if (tid == 0) {
            const int64_t t = perm[k];
            perm[k] = perm[p];
            perm[p] = t;
        }
        __syncthreads();
    }
    mf<N> piv;
#pragma unroll
    for (int l = 0; l < N; ++l) piv.v[l] = spiv[l];
    if (tid == 0) store_mf<N>(A.p, A.ld, A.ls, k, k, piv);
    for (int64_t r = k + 1 + tid; r < n; r += PSTRF_PIVOT_THREADS)
        store_mf<N>(A.p, A.ld, A.ls, r, k, div(load_mf<N>(A.p, A.ld, A.ls, r, k), piv));
}

constexpr int PSTRF_UPD_ROWS = 128, PSTRF_UPD_COLS = 16;

template <int N>
__global__ void __launch_bounds__(PSTRF_UPD_ROWS)
    pstrf_update_kernel(int64_t n, int64_t k, Mat A, const PstrfState *st) {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (st->stop) return;
    const int64_t r = k + 1 + (int64_t)blockIdx.x * PSTRF_UPD_ROWS + threadIdx.x;
    if (r >= n) return;
    const int64_t c0 = k + 1 + (int64_t)blockIdx.y * PSTRF_UPD_COLS;
    const int64_t c1 = c0 + PSTRF_UPD_COLS < n ? c0 + PSTRF_UPD_COLS : n;
    const mf<N> lr = load_mf<N>(A.p, A.ld, A.ls, r, k);
    for (int64_t c = c0; c < c1; ++c) {
        const mf<N> lc = load_mf<N>(A.p, A.ld, A.ls, c, k);
        store_mf<N>(A.p, A.ld, A.ls, r, c, submul(load_mf<N>(A.p, A.ld, A.ls, r, c), lr, lc));
    }
}

__global__ void pstrf_finish_kernel(const PstrfState *st, int64_t *rank_info) {
    rank_info[0] = st->rank;
    rank_info[1] = st->info;
}

template <int N>
static int pstrf_n(mflab_handle *h, cudaStream_t s, int64_t n, Mat A, const double *tol,
                   int64_t *perm, int64_t *rank_info) {
    int rc = mflab_reserve_aux(h, sizeof(PstrfState));
    if (rc) return rc;
    PstrfState *st = (PstrfState *)h->aux;
    scal<N> t{};
    for (int l = 0; l < N; ++l) t.v[l] = tol[l];
    const int64_t g = (n * n + 255) / 256;
    const unsigned grid = (unsigned)(g < 4 * 148 ? (g > 0 ? g : 1) : 4 * 148);
    pstrf_init_kernel<<<(unsigned)((n + 255) / 256 > 0 ? (n + 255) / 256 : 1), 256, 0, s>>>(st, n, perm);
    pstrf_check_kernel<N><<<grid, 256, 0, s>>>(n, A, st);
    pstrf_mirror_kernel<N><<<grid, 256, 0, s>>>(n, A, st);
    for (int64_t k = 0; k < n && rc == MFLAB_OK; ++k) {
        // programmatic dependent launches: each step's CTAs are placed while
        // the previous step drains
        rc = launch_programmatic(pstrf_pivot_kernel<N>, dim3(1), dim3(PSTRF_PIVOT_THREADS), 0, s,
                                 "pstrf pivot", n, k, A, perm, st, t);
        const int64_t tr = n - k - 1;
        if (tr > 0 && rc == MFLAB_OK) {
            dim3 ug((unsigned)((tr + PSTRF_UPD_ROWS - 1) / PSTRF_UPD_ROWS),
                    (unsigned)((tr + PSTRF_UPD_COLS - 1) / PSTRF_UPD_COLS));
            rc = launch_programmatic(pstrf_update_kernel<N>, ug, dim3(PSTRF_UPD_ROWS), 0, s,
                                     "pstrf update", n, k, A, (const PstrfState *)st);
        }
    }
    if (rc) return rc;
    pstrf_finish_kernel<<<1, 1, 0, s>>>(st, rank_info);
    return record_cuda_error(cudaGetLastError(), "pstrf launch");
}

}  // namespace mfl

using mfl::Mat;

extern "C" int mflab_pstrf(mflab_handle *h, void *stream, int limbs, int64_t n, double *A,
                           int64_t lda, int64_t lsa, const double *tol, int64_t *perm,
                           int64_t *rank_info) {
    MFLAB_RANGE("mflab_pstrf");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (n < 0 || !tol || !perm || !rank_info) return MFLAB_ERR_ARG;
    for (int l = 0; l < limbs; ++l)
        if (!isfinite(tol[l])) return MFLAB_ERR_ARG;
    if (tol[0] < 0.0) return MFLAB_ERR_ARG;
    if (n > 0 && lda < n) return MFLAB_ERR_ARG;
    if ((n + mfl::PSTRF_UPD_COLS - 1) / mfl::PSTRF_UPD_COLS > 65535) return MFLAB_ERR_UNSUPPORTED;
    cudaStream_t s = (cudaStream_t)stream;
    if (n == 0)  // rank 0, info 0
        return mfl::record_cuda_error(cudaMemsetAsync(rank_info, 0, 2 * sizeof(int64_t), s),
                                      "pstrf memset");
    const Mat Am{A, lda, lsa};
    switch (limbs) {
    case 2: return mfl::pstrf_n<2>(h, s, n, Am, tol, perm, rank_info);
    case 3: return mfl::pstrf_n<3>(h, s, n, Am, tol, perm, rank_info);
    default: return mfl::pstrf_n<4>(h, s, n, Am, tol, perm, rank_info);
    }
}
