// Householder QR, rank-revealing QR, apply_q! and numerical_rank
// (src/factorizations/qr.jl of MultiFloatLinearAlgebra.jl).
//
// Every result is the reference's element by element: column norms are the
// sequential scaled sum of squares (qr.jl:96-122), each reflector
// application is one ascending projection chain per column (qr.jl:624-642),
// and the rank-revealing path follows the reference's two routes, the
// hybrid pivot search for small problems (qr.jl:192-224, 364-398) and the
// DLAQPS-style panel with delayed updates, norm downdates and panel breaks
// (qr.jl:450-604), whose end-of-panel update is the matched GEMM kernel.
//
// Parallel structure: the work that is independent across columns (trailing
// reflector applications, the F recurrence, the R row, norm downdates and
// rebuilds) runs one column per thread; the sequential pieces (a column
// norm, the pivot decision) run on one CTA.  Norm state lives in device
// planes so no step needs the host, except the panel-break test of the
// blocked route, which the host reads once per step.
#include "mf_device.cuh"
#include "mflab_internal.h"

#include <vector>

namespace mfl {

constexpr int QR_BLOCK = 16;          // _QR_BLOCK_SIZE, qr.jl:306
constexpr int QR_CTA = 256;           // single-CTA kernels
constexpr int QR_COLS_PER_CTA = 64;   // one column per thread

template <int N>
struct QRNorms {
    double *scale;  // N planes of n
    double *sum;    // N planes of n
    int *dirty;     // n
    int64_t n;
    __device__ mf<N> sc(int64_t c) const {
        mf<N> x;
#pragma unroll
        for (int l = 0; l < N; ++l) x.v[l] = scale[l * n + c];
        return x;
    }
    __device__ mf<N> su(int64_t c) const {
        mf<N> x;
#pragma unroll
        for (int l = 0; l < N; ++l) x.v[l] = sum[l * n + c];
        return x;
    }
    __device__ void set(int64_t c, const mf<N> &s, const mf<N> &u) const {
#pragma unroll
        for (int l = 0; l < N; ++l) {
            scale[l * n + c] = s.v[l];
            sum[l * n + c] = u.v[l];
        }
    }
    __device__ void set_sum(int64_t c, const mf<N> &u) const {
#pragma unroll
        for (int l = 0; l < N; ++l) sum[l * n + c] = u.v[l];
    }
    __device__ void swap(int64_t a, int64_t b) const {
        if (a == b) return;
#pragma unroll
        for (int l = 0; l < N; ++l) {
            double t = scale[l * n + a];
            scale[l * n + a] = scale[l * n + b];
            scale[l * n + b] = t;
            t = sum[l * n + a];
            sum[l * n + a] = sum[l * n + b];
            sum[l * n + b] = t;
        }
        const int d = dirty[a];
        dirty[a] = dirty[b];
        dirty[b] = d;
    }
};

// _qr_column_norm_state / _qr_delayed_column_norm_state (qr.jl:96-122,
// 226-262): rows r0..m-1 of column c, each value first corrected by
// value -= A[row, bs + p] * F[p, c] for p < prior
template <int N>
__device__ void norm_state(const Mat &A, int64_t m, int64_t r0, int64_t c, const Mat &F,
                           int64_t bs, int64_t prior, mf<N> &scale, mf<N> &sum) {
    const mf<N> one = from_double<N>(1.0);
    scale = from_double<N>(0.0);
    sum = one;
    bool seen = false;
    for (int64_t r = r0; r < m; ++r) {
        mf<N> v = load_mf<N>(A.p, A.ld, A.ls, r, c);
        for (int64_t p = 0; p < prior; ++p)
            v = submul(v, load_mf<N>(A.p, A.ld, A.ls, r, bs + p), load_mf<N>(F.p, F.ld, F.ls, p, c));
        const mf<N> mag = abs_mf(v);
        if (iszero(mag)) continue;
        if (!seen) {
            scale = mag;
            sum = one;
            seen = true;
        } else if (gt(mag, scale)) {
            const mf<N> ratio = div(scale, mag);
            sum = add(one, mul(mul(sum, ratio), ratio));
            scale = mag;
        } else {
            const mf<N> ratio = div(mag, scale);
            sum = add(sum, mul(ratio, ratio));
        }
    }
}

// _qr_norm_from_state (qr.jl:157-165)
template <int N>
__device__ __forceinline__ mf<N> norm_value(const mf<N> &scale, const mf<N> &sum) {
    return iszero(scale) ? from_double<N>(0.0) : mul(scale, sqrt_mf(sum));
}

__global__ void qr_finite_kernel_init(int *flag) { *flag = 0; }

template <int N>
__global__ void qr_finite_kernel(int64_t m, int64_t n, Mat A, int *flag) {
    bool bad = false;
    const int64_t total = m * n;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = e / m, r = e % m;
#pragma unroll
        for (int l = 0; l < N; ++l) bad = bad || !isfinite(A.p[l * A.ls + c * A.ld + r]);
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicExch(flag, 1);
}

// _qr_make_reflector! (qr.jl:606-622) for column s; tau at tau[l * lt + s].
// blocked != 0 (the DLAQPS panel, qr.jl:513-515, 530-541): afterwards save
// A[s,s] to diag, set A[s,s] = 1 and form aux[p] = -tau * sum_rows
// A[row, bs+p] v[row] for the ls earlier panel columns.
template <int N>
__global__ void __launch_bounds__(QR_CTA)
    qr_reflector_kernel(int64_t m, int64_t s, Mat A, double *tau, int64_t lt, int blocked,
                        double *diag, int64_t bs, int64_t ls, double *aux) {
    __shared__ double slead[N];
    __shared__ int go;
    const int tid = threadIdx.x;
    if (tid == 0) {
        mf<N> scale, sum;
        const Mat none{nullptr, 1, 1};
        norm_state<N>(A, m, s, s, none, 0, 0, scale, sum);
        const mf<N> nrm = norm_value(scale, sum);
        mf<N> t = from_double<N>(0.0);
        go = 0;
        if (!iszero(nrm)) {
            const mf<N> alpha = load_mf<N>(A.p, A.ld, A.ls, s, s);
            const mf<N> beta = ge(alpha, from_double<N>(0.0)) ? neg(nrm) : nrm;
            const mf<N> lead = sub(alpha, beta);
            t = div(sub(beta, alpha), beta);
#pragma unroll
            for (int l = 0; l < N; ++l) slead[l] = lead.v[l];
            store_mf<N>(A.p, A.ld, A.ls, s, s, beta);
            go = 1;
        }
#pragma unroll
        for (int l = 0; l < N; ++l) tau[l * lt + s] = t.v[l];
    }
    __syncthreads();
    if (go) {
        mf<N> lead;
#pragma unroll
        for (int l = 0; l < N; ++l) lead.v[l] = slead[l];
        for (int64_t r = s + 1 + tid; r < m; r += QR_CTA)
            store_mf<N>(A.p, A.ld, A.ls, r, s, div(load_mf<N>(A.p, A.ld, A.ls, r, s), lead));
    }
    if (!blocked) return;
    __syncthreads();
    if (tid == 0) {
        const mf<N> d = load_mf<N>(A.p, A.ld, A.ls, s, s);
#pragma unroll
        for (int l = 0; l < N; ++l) diag[l] = d.v[l];
        store_mf<N>(A.p, A.ld, A.ls, s, s, from_double<N>(1.0));
    }
    __syncthreads();
    if (tid < ls) {
        mf<N> t;
#pragma unroll
        for (int l = 0; l < N; ++l) t.v[l] = tau[l * lt + s];
        mf<N> acc = from_double<N>(0.0);
        for (int64_t r = s; r < m; ++r)
            acc = mac<N, false>(acc, load_mf<N>(A.p, A.ld, A.ls, r, bs + tid),
                                load_mf<N>(A.p, A.ld, A.ls, r, s));
        const mf<N> a = mul(neg(t), acc);
#pragma unroll
        for (int l = 0; l < N; ++l) aux[tid * N + l] = a.v[l];
    }
}

// reflector s of V (implicit one at row s) applied to columns c0.. of D,
// one column per thread (qr.jl:624-642); skipped when tau is zero
template <int N>
__device__ __forceinline__ void apply_reflector_col(int64_t m, int64_t s, const Mat &V,
                                                    const mf<N> &t, const Mat &D, int64_t c) {
    mf<N> proj = load_mf<N>(D.p, D.ld, D.ls, s, c);
    for (int64_t r = s + 1; r < m; ++r)
        proj = add(proj, mul(load_mf<N>(V.p, V.ld, V.ls, r, s), load_mf<N>(D.p, D.ld, D.ls, r, c)));
    proj = mul(proj, t);
    store_mf<N>(D.p, D.ld, D.ls, s, c, sub(load_mf<N>(D.p, D.ld, D.ls, s, c), proj));
    for (int64_t r = s + 1; r < m; ++r)
        store_mf<N>(D.p, D.ld, D.ls, r, c,
                    submul(load_mf<N>(D.p, D.ld, D.ls, r, c), load_mf<N>(V.p, V.ld, V.ls, r, s), proj));
}

template <int N>
__global__ void __launch_bounds__(QR_COLS_PER_CTA)
    qr_apply_kernel(int64_t m, int64_t s, Mat V, const double *tau, int64_t lt, Mat D, int64_t c0,
                    int64_t nd) {
    const int64_t j = (int64_t)blockIdx.x * QR_COLS_PER_CTA + threadIdx.x;
    if (j >= nd) return;
    mf<N> t;
#pragma unroll
    for (int l = 0; l < N; ++l) t.v[l] = tau[l * lt + s];
    if (iszero(t)) return;
    apply_reflector_col<N>(m, s, V, t, D, c0 + j);
}

// apply_q! (qr.jl:890-956): every reflector in order on one column of D
template <int N>
__global__ void __launch_bounds__(QR_COLS_PER_CTA)
    qr_apply_all_kernel(int64_t m, int64_t r, Mat V, const double *tau, int64_t lt, Mat D,
                        int64_t nd, int trans) {
    const int64_t c = (int64_t)blockIdx.x * QR_COLS_PER_CTA + threadIdx.x;
    if (c >= nd) return;
    for (int64_t i = 0; i < r; ++i) {
        const int64_t s = trans ? i : r - 1 - i;
        mf<N> t;
#pragma unroll
        for (int l = 0; l < N; ++l) t.v[l] = tau[l * lt + s];
        if (iszero(t)) continue;
        apply_reflector_col<N>(m, s, V, t, D, c);
    }
}

// norm state of columns c0..n-1 from rows r0 (qr.jl:143-155, 417-448)
template <int N>
__global__ void __launch_bounds__(QR_COLS_PER_CTA)
    qr_norm_init_kernel(int64_t m, int64_t r0, int64_t c0, Mat A, QRNorms<N> S) {
    const int64_t c = c0 + (int64_t)blockIdx.x * QR_COLS_PER_CTA + threadIdx.x;
    if (c >= S.n) return;
    mf<N> scale, sum;
    const Mat none{nullptr, 1, 1};
    norm_state<N>(A, m, r0, c, none, 0, 0, scale, sum);
    S.set(c, scale, sum);
    S.dirty[c] = 0;
}

// _qr_update_norm_state! for one column (qr.jl:264-304)
template <int N>
__device__ void update_norm_col(int64_t m, int64_t step, int64_t c, const Mat &A,
                                const QRNorms<N> &S, const mf<N> &floor_, const Mat &F,
                                int64_t bs, int64_t prior) {
    if (S.dirty[c]) return;
    const mf<N> scale = S.sc(c);
    const mf<N> removed = abs_mf(load_mf<N>(A.p, A.ld, A.ls, step, c));
    if (iszero(scale)) {
        S.dirty[c] = !iszero(removed);
        return;
    }
    const mf<N> ratio = div(removed, scale);
    const mf<N> ns = sub(S.su(c), mul(ratio, ratio));
    if (!isfinite_mf(ns) || ge(floor_, ns)) {
        mf<N> sc, su;
        norm_state<N>(A, m, step + 1, c, F, bs, prior, sc, su);
        S.set(c, sc, su);
        S.dirty[c] = 0;
    } else {
        S.set_sum(c, ns);
    }
}

template <int N>
__global__ void __launch_bounds__(QR_COLS_PER_CTA)
    qr_update_norms_kernel(int64_t m, int64_t step, Mat A, const double *tau, int64_t lt,
                           QRNorms<N> S, scal<N> floor_) {
    const int64_t c = step + 1 + (int64_t)blockIdx.x * QR_COLS_PER_CTA + threadIdx.x;
    if (c >= S.n) return;
    mf<N> t;
#pragma unroll
    for (int l = 0; l < N; ++l) t.v[l] = tau[l * lt + step];
    if (iszero(t)) return;
    const Mat none{nullptr, 1, 1};
    update_norm_col<N>(m, step, c, A, S, floor_.get(), none, 0, 0);
}

template <int N>
__device__ void swap_columns_cta(int64_t m, const Mat &A, int64_t a, int64_t b) {
    if (a == b) return;
    for (int64_t r = threadIdx.x; r < m; r += blockDim.x)
#pragma unroll
        for (int l = 0; l < N; ++l) {
            double *pa = A.p + l * A.ls + a * A.ld + r, *pb = A.p + l * A.ls + b * A.ld + r;
            const double t = *pa;
            *pa = *pb;
            *pb = t;
        }
}

// _qr_select_pivot_hybrid! (qr.jl:192-224) on thread 0, then the column,
// permutation and norm-state swaps (qr.jl:376-386)
template <int N>
__global__ void __launch_bounds__(QR_CTA)
    qr_hybrid_pivot_kernel(int64_t m, int64_t step, Mat A, int64_t *perm, QRNorms<N> S,
                           scal<N> one_minus_margin) {
    __shared__ int64_t sp;
    if (threadIdx.x == 0) {
        const Mat none{nullptr, 1, 1};
        const mf<N> om = one_minus_margin.get();
        int64_t piv = step;
        mf<N> sc, su;
        norm_state<N>(A, m, step, step, none, 0, 0, sc, su);
        S.set(step, sc, su);
        S.dirty[step] = 0;
        mf<N> pn = norm_value(sc, su);
        for (int64_t c = step + 1; c < S.n; ++c) {
            mf<N> cn = norm_value(S.sc(c), S.su(c));
            if (S.dirty[c] || iszero(pn) || ge(cn, mul(om, pn))) {
                norm_state<N>(A, m, step, c, none, 0, 0, sc, su);
                S.set(c, sc, su);
                S.dirty[c] = 0;
                cn = norm_value(sc, su);
            }
            bool eq = true;
#pragma unroll
            for (int l = 0; l < N; ++l) eq = eq && cn.v[l] == pn.v[l];
            if (gt(cn, pn) || (eq && perm[c] < perm[piv])) {
                piv = c;
                pn = cn;
            }
        }
        sp = piv;
    }
    __syncthreads();
    const int64_t piv = sp;
    swap_columns_cta<N>(m, A, step, piv);
    if (threadIdx.x == 0 && piv != step) {
        const int64_t t = perm[step];
        perm[step] = perm[piv];
        perm[piv] = t;
        S.swap(step, piv);
    }
}

constexpr int QR_PIVOT_CTA = 1024;

// DLAQPS step head (qr.jl:478-511): downdated pivot choice (largest norm
// from the state, smallest original column on ties), the column swap with
// its F entries, permutation and norm state, then the delayed prefix on the
// chosen column
template <int N>
__global__ void __launch_bounds__(QR_PIVOT_CTA)
    qr_dlaqps_pivot_kernel(int64_t m, int64_t step, int64_t bs, int64_t ls, Mat A, int64_t *perm,
                           QRNorms<N> S, Mat F) {
    __shared__ double sval[N][QR_PIVOT_CTA];
    __shared__ int64_t sidx[QR_PIVOT_CTA];
    const int tid = threadIdx.x;
    int64_t bi = -1;
    mf<N> bv = from_double<N>(0.0);
    for (int64_t c = step + tid; c < S.n; c += QR_PIVOT_CTA) {
        const mf<N> v = norm_value(S.sc(c), S.su(c));
        bool eq = true;
#pragma unroll
        for (int l = 0; l < N; ++l) eq = eq && v.v[l] == bv.v[l];
        if (bi < 0 || gt(v, bv) || (eq && perm[c] < perm[bi])) {
            bi = c;
            bv = v;
        }
    }
#pragma unroll
    for (int l = 0; l < N; ++l) sval[l][tid] = bv.v[l];
    sidx[tid] = bi;
    __syncthreads();
    for (int s = QR_PIVOT_CTA / 2; s > 0; s >>= 1) {
        if (tid < s && sidx[tid + s] >= 0) {
            const int64_t ia = sidx[tid], ib = sidx[tid + s];
            mf<N> va, vb;
#pragma unroll
            for (int l = 0; l < N; ++l) {
                va.v[l] = sval[l][tid];
                vb.v[l] = sval[l][tid + s];
            }
            bool eq = true;
#pragma unroll
            for (int l = 0; l < N; ++l) eq = eq && va.v[l] == vb.v[l];
            if (ia < 0 || gt(vb, va) || (eq && perm[ib] < perm[ia])) {
#pragma unroll
                for (int l = 0; l < N; ++l) sval[l][tid] = vb.v[l];
                sidx[tid] = ib;
            }
        }
        __syncthreads();
    }
    const int64_t piv = sidx[0];
    swap_columns_cta<N>(m, A, step, piv);
    if (piv != step) {
        for (int64_t e = tid; e < ls * N; e += QR_PIVOT_CTA) {
            const int64_t p = e / N;
            const int l = (int)(e % N);
            double *fa = F.p + l * F.ls + step * F.ld + p, *fb = F.p + l * F.ls + piv * F.ld + p;
            const double t = *fa;
            *fa = *fb;
            *fb = t;
        }
    }
    __syncthreads();
    if (tid == 0 && piv != step) {
        const int64_t t = perm[step];
        perm[step] = perm[piv];
        perm[piv] = t;
        S.swap(step, piv);
    }
    if (ls > 0)
        for (int64_t r = step + tid; r < m; r += QR_PIVOT_CTA) {
            mf<N> corr = from_double<N>(0.0);
            for (int64_t p = 0; p < ls; ++p)
                corr = mac<N, false>(corr, load_mf<N>(A.p, A.ld, A.ls, r, bs + p),
                                     load_mf<N>(F.p, F.ld, F.ls, p, step));
            store_mf<N>(A.p, A.ld, A.ls, r, step, sub(load_mf<N>(A.p, A.ld, A.ls, r, step), corr));
        }
}

// DLAQPS step body, one trailing column per thread (qr.jl:517-576): the new
// F row (gemv! trans = :T, then the correction through aux), the R row, and
// the norm downdate; any column left unreliable raises *unreliable
template <int N>
__global__ void __launch_bounds__(QR_COLS_PER_CTA)
    qr_dlaqps_columns_kernel(int64_t m, int64_t step, int64_t bs, int64_t ls, Mat A,
                             const double *tau, int64_t lt, const double *aux, Mat F, QRNorms<N> S,
                             scal<N> floor_, int *unreliable) {
    const int64_t c = step + 1 + (int64_t)blockIdx.x * QR_COLS_PER_CTA + threadIdx.x;
    if (c >= S.n) return;
    mf<N> t;
#pragma unroll
    for (int l = 0; l < N; ++l) t.v[l] = tau[l * lt + step];
    mf<N> acc = from_double<N>(0.0);
    for (int64_t r = step; r < m; ++r)
        acc = mac<N, false>(acc, load_mf<N>(A.p, A.ld, A.ls, r, c), load_mf<N>(A.p, A.ld, A.ls, r, step));
    mf<N> f = mul(t, acc);
    if (ls > 0) {
        mf<N> corr = from_double<N>(0.0);
        for (int64_t p = 0; p < ls; ++p) {
            mf<N> a;
#pragma unroll
            for (int l = 0; l < N; ++l) a.v[l] = aux[p * N + l];
            corr = mac<N, false>(corr, load_mf<N>(F.p, F.ld, F.ls, p, c), a);
        }
        f = add(f, corr);
    }
    store_mf<N>(F.p, F.ld, F.ls, ls, c, f);
    mf<N> corr = from_double<N>(0.0);
    for (int64_t p = 0; p <= ls; ++p)
        corr = mac<N, false>(corr, load_mf<N>(A.p, A.ld, A.ls, step, bs + p),
                             load_mf<N>(F.p, F.ld, F.ls, p, c));
    store_mf<N>(A.p, A.ld, A.ls, step, c, sub(load_mf<N>(A.p, A.ld, A.ls, step, c), corr));
    if (!iszero(t)) update_norm_col<N>(m, step, c, A, S, floor_.get(), F, bs, ls + 1);
    if (S.dirty[c]) atomicExch(unreliable, 1);
}

__global__ void qr_restore_diag_kernel(int N, Mat A, int64_t s, const double *diag) {
    for (int l = 0; l < N; ++l) A.p[l * A.ls + s * A.ld + s] = diag[l];
}

// numerical_rank (qr.jl:863-888)
template <int N>
__global__ void qr_rank_kernel(int64_t r, Mat F, scal<N> atol, scal<N> rtol, int64_t *rank) {
    mf<N> largest = from_double<N>(0.0);
    for (int64_t i = 0; i < r; ++i)
        largest = max_mf(largest, abs_mf(load_mf<N>(F.p, F.ld, F.ls, i, i)));
    const mf<N> thr = max_mf(atol.get(), mul(rtol.get(), largest));
    int64_t k = 0;
    for (; k < r; ++k)
        if (!gt(abs_mf(load_mf<N>(F.p, F.ld, F.ls, k, k)), thr)) break;
    *rank = k;
}

static inline unsigned col_grid(int64_t cols) {
    return (unsigned)((cols + QR_COLS_PER_CTA - 1) / QR_COLS_PER_CTA);
}

template <int N>
static int qr_n(mflab_handle *h, cudaStream_t s, int pivoted, int64_t m, int64_t n, Mat A,
                double *tau, int64_t lt, int64_t *perm, int *info) {
    const int64_t r = m < n ? m : n;
    // scratch: norm planes, F (QR_BLOCK x n), aux, diag, flags
    const size_t nn = (size_t)(n > 0 ? n : 1);
    const size_t doubles = 2 * N * nn + (size_t)N * QR_BLOCK * nn + QR_BLOCK * N + N;
    const size_t bytes = doubles * sizeof(double) + (nn + 4) * sizeof(int);
    int rc = mflab_reserve_scratch(h, bytes);
    if (rc) return rc;
    double *base = (double *)h->scratch;
    QRNorms<N> S{base, base + N * nn, nullptr, n};
    double *Fp = base + 2 * N * nn;
    const Mat F{Fp, QR_BLOCK, (int64_t)(QR_BLOCK * nn)};
    double *aux = Fp + (size_t)N * QR_BLOCK * nn;
    double *diag = aux + QR_BLOCK * N;
    S.dirty = (int *)(diag + N);
    int *flag = S.dirty + nn;
    int *hflag = nullptr;

    cudaError_t e = cudaSuccess;
    for (int l = 0; l < N; ++l) {
        e = cudaMemsetAsync(tau + l * lt, 0, r * sizeof(double), s);
        if (e != cudaSuccess) return record_cuda_error(e, "qr tau");
    }
    // identity permutation, finiteness
    {
        std::vector<int64_t> id(n);
        for (int64_t i = 0; i < n; ++i) id[i] = i + 1;
        if (n > 0) {
            e = cudaMemcpyAsync(perm, id.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice, s);
            if (e != cudaSuccess) return record_cuda_error(e, "qr perm");
        }
        qr_finite_kernel_init<<<1, 1, 0, s>>>(flag);
        const int64_t g = (m * n + 255) / 256;
        qr_finite_kernel<N><<<(unsigned)(g < 1184 ? (g > 0 ? g : 1) : 1184), 256, 0, s>>>(m, n, A, flag);
        int fin = 0;
        e = cudaMemcpyAsync(&fin, flag, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return record_cuda_error(e, "qr finiteness");
        if (fin) {
            const int neg1 = -1;
            e = cudaMemcpyAsync(info, &neg1, sizeof(int), cudaMemcpyHostToDevice, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            return record_cuda_error(e, "qr info");
        }
    }
    (void)hflag;
    if (!pivoted) {
        for (int64_t st = 0; st < r; ++st) {
            qr_reflector_kernel<N><<<1, QR_CTA, 0, s>>>(m, st, A, tau, lt, 0, nullptr, 0, 0, nullptr);
            if (st + 1 < n)
                qr_apply_kernel<N><<<col_grid(n - st - 1), QR_COLS_PER_CTA, 0, s>>>(
                    m, st, A, tau, lt, A, st + 1, n - st - 1);
        }
    } else {
        // constants of rrqr! (qr.jl:736-737): margin = sqrt(eps), floor = 16 eps,
        // eps = 2^(-52 N); sqrt and the products are exact powers of two
        scal<N> om{}, fl{};
        om.v[0] = 1.0;
        if (N == 2) {
            om.v[0] = 1.0 - ldexp(1.0, -52);
        } else {
            om.v[1] = -ldexp(1.0, -26 * N);
        }
        fl.v[0] = ldexp(1.0, 4 - 52 * N);
        if (n > 0)
            qr_norm_init_kernel<N><<<col_grid(n), QR_COLS_PER_CTA, 0, s>>>(m, 0, 0, A, S);
        const bool blocked = r >= QR_BLOCK && m * n >= 16384;
        if (!blocked) {
            for (int64_t st = 0; st < r; ++st) {
                qr_hybrid_pivot_kernel<N><<<1, QR_CTA, 0, s>>>(m, st, A, perm, S, om);
                qr_reflector_kernel<N><<<1, QR_CTA, 0, s>>>(m, st, A, tau, lt, 0, nullptr, 0, 0, nullptr);
                if (st + 1 < n) {
                    qr_apply_kernel<N><<<col_grid(n - st - 1), QR_COLS_PER_CTA, 0, s>>>(
                        m, st, A, tau, lt, A, st + 1, n - st - 1);
                    qr_update_norms_kernel<N><<<col_grid(n - st - 1), QR_COLS_PER_CTA, 0, s>>>(
                        m, st, A, tau, lt, S, fl);
                }
            }
        } else {
            e = cudaMallocHost(&hflag, sizeof(int));
            if (e != cudaSuccess) return record_cuda_error(e, "qr host flag");
            int64_t bs = 0;
            rc = MFLAB_OK;
            while (bs < r && rc == MFLAB_OK) {
                const int64_t req = (r - bs) < QR_BLOCK ? (r - bs) : QR_BLOCK;
                for (int l = 0; l < N && e == cudaSuccess; ++l)
                    e = cudaMemsetAsync(Fp + l * F.ls, 0, QR_BLOCK * nn * sizeof(double), s);
                if (e != cudaSuccess) {
                    rc = record_cuda_error(e, "qr F");
                    break;
                }
                int64_t actual = 0;
                for (int64_t ls = 0; ls < req; ++ls) {
                    const int64_t st = bs + ls;
                    qr_dlaqps_pivot_kernel<N><<<1, QR_PIVOT_CTA, 0, s>>>(m, st, bs, ls, A, perm, S, F);
                    qr_reflector_kernel<N><<<1, QR_CTA, 0, s>>>(m, st, A, tau, lt, 1, diag, bs, ls, aux);
                    qr_finite_kernel_init<<<1, 1, 0, s>>>(flag);
                    if (st + 1 < n)
                        qr_dlaqps_columns_kernel<N><<<col_grid(n - st - 1), QR_COLS_PER_CTA, 0, s>>>(
                            m, st, bs, ls, A, tau, lt, aux, F, S, fl, flag);
                    qr_restore_diag_kernel<<<1, 1, 0, s>>>(N, A, st, diag);
                    actual = ls + 1;
                    e = cudaMemcpyAsync(hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, s);
                    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                    if (e != cudaSuccess) {
                        rc = record_cuda_error(e, "qr panel flag");
                        break;
                    }
                    if (*hflag) break;
                }
                if (rc) break;
                const int64_t be = bs + actual;
                if (be < m && be < n) {
                    const double mone[4] = {-1.0, 0.0, 0.0, 0.0}, one[4] = {1.0, 0.0, 0.0, 0.0};
                    rc = launch_mm(N, 0, false, 0, N == 3, m - be, n - be, actual, A.at(be, bs),
                                   Mat{Fp + be * F.ld, F.ld, F.ls}, A.at(be, be), mone, one, s);
                    if (rc) break;
                }
                if (be < n)
                    qr_norm_init_kernel<N><<<col_grid(n - be), QR_COLS_PER_CTA, 0, s>>>(m, be, be, A, S);
                bs = be;
            }
            cudaFreeHost(hflag);
            if (rc) return rc;
        }
    }
    const int zero = 0;
    e = cudaMemcpyAsync(info, &zero, sizeof(int), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return record_cuda_error(e, "qr info");
    return record_cuda_error(cudaGetLastError(), "qr launch");
}

}  // namespace mfl

using mfl::Mat;

extern "C" int mflab_qr(mflab_handle *h, void *stream, int limbs, int pivoted, int64_t m,
                        int64_t n, double *A, int64_t lda, int64_t lsa, double *tau, int64_t lst,
                        int64_t *perm, int *info) {
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (m < 0 || n < 0 || !tau || !perm || !info || (pivoted & ~1)) return MFLAB_ERR_ARG;
    const int64_t r = m < n ? m : n;
    if ((m > 0 && lda < m) || lst < r) return MFLAB_ERR_ARG;
    const Mat Am{A, lda, lsa};
    cudaStream_t s = (cudaStream_t)stream;
    switch (limbs) {
    case 2: return mfl::qr_n<2>(h, s, pivoted, m, n, Am, tau, lst, perm, info);
    case 3: return mfl::qr_n<3>(h, s, pivoted, m, n, Am, tau, lst, perm, info);
    default: return mfl::qr_n<4>(h, s, pivoted, m, n, Am, tau, lst, perm, info);
    }
}

extern "C" int mflab_apply_q(mflab_handle *h, void *stream, int limbs, int trans, int64_t m,
                             int64_t r, const double *F, int64_t ldf, int64_t lsf,
                             const double *tau, int64_t lst, double *D, int64_t ldd, int64_t lsd,
                             int64_t nd) {
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (m < 0 || r < 0 || nd < 0 || (trans & ~1) || r > m) return MFLAB_ERR_ARG;
    if (m == 0 || nd == 0 || r == 0) return MFLAB_OK;
    if (ldf < m || ldd < m || lst < r) return MFLAB_ERR_ARG;
    if (mfl::views_overlap(D, ldd, lsd, m, nd, limbs, F, ldf, lsf, m, r)) return MFLAB_ERR_ALIAS;
    const Mat Fm{(double *)F, ldf, lsf}, Dm{D, ldd, lsd};
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned g = mfl::col_grid(nd);
    switch (limbs) {
    case 2: mfl::qr_apply_all_kernel<2><<<g, mfl::QR_COLS_PER_CTA, 0, s>>>(m, r, Fm, tau, lst, Dm, nd, trans); break;
    case 3: mfl::qr_apply_all_kernel<3><<<g, mfl::QR_COLS_PER_CTA, 0, s>>>(m, r, Fm, tau, lst, Dm, nd, trans); break;
    default: mfl::qr_apply_all_kernel<4><<<g, mfl::QR_COLS_PER_CTA, 0, s>>>(m, r, Fm, tau, lst, Dm, nd, trans); break;
    }
    return mfl::record_cuda_error(cudaGetLastError(), "apply_q launch");
}

extern "C" int mflab_qr_numerical_rank(mflab_handle *h, void *stream, int limbs, int64_t m,
                                       int64_t n, const double *F, int64_t ldf, int64_t lsf,
                                       const double *atol, const double *rtol, int64_t *rank) {
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (m < 0 || n < 0 || !atol || !rtol || !rank) return MFLAB_ERR_ARG;
    const int64_t r = m < n ? m : n;
    if (r > 0 && ldf < m) return MFLAB_ERR_ARG;
    const Mat Fm{(double *)F, ldf, lsf};
    cudaStream_t s = (cudaStream_t)stream;
    switch (limbs) {
    case 2: {
        mfl::scal<2> a{}, b{};
        for (int l = 0; l < 2; ++l) a.v[l] = atol[l], b.v[l] = rtol[l];
        mfl::qr_rank_kernel<2><<<1, 1, 0, s>>>(r, Fm, a, b, rank);
        break;
    }
    case 3: {
        mfl::scal<3> a{}, b{};
        for (int l = 0; l < 3; ++l) a.v[l] = atol[l], b.v[l] = rtol[l];
        mfl::qr_rank_kernel<3><<<1, 1, 0, s>>>(r, Fm, a, b, rank);
        break;
    }
    default: {
        mfl::scal<4> a{}, b{};
        for (int l = 0; l < 4; ++l) a.v[l] = atol[l], b.v[l] = rtol[l];
        mfl::qr_rank_kernel<4><<<1, 1, 0, s>>>(r, Fm, a, b, rank);
        break;
    }
    }
    return mfl::record_cuda_error(cudaGetLastError(), "numerical_rank launch");
}
