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

// The same scaled sum of squares computed by one warp, bit for bit: per chunk
// of 32 rows the lanes load their magnitudes, a warp scan gives every row the
// running maximum before it (the reference's `scale` at that row: the scale
// only ever moves to a new maximum), each lane forms its ratio and square in
// parallel, and lane 0 folds the chunk in row order with the reference's own
// operations (sum += ratio^2, or sum = 1 + sum*ratio*ratio at a new maximum,
// or sum = 1 at the first nonzero).  The divisions and products leave the
// sequential path; only the additions stay on it.  All 32 lanes must call it;
// buf is this warp's shared scratch of QR_NORM_BUF(N) doubles.
#define QR_NORM_BUF(N) (32 * (3 * (N) + 1))
template <int N>
__device__ void norm_state_warp(const Mat &A, int64_t m, int64_t r0, int64_t c, double *buf,
                                mf<N> &scale, mf<N> &sum) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const mf<N> one = from_double<N>(1.0), zero = from_double<N>(0.0);
    scale = zero;
    sum = one;
    bool seen = false;
    double *bmag = buf, *brat = buf + 32 * N, *bsq = buf + 64 * N;
    int *bflag = (int *)(buf + 96 * N);
    for (int64_t base = r0; base < m; base += 32) {
        const int64_t r = base + lane;
        const mf<N> mag = r < m ? abs_mf(load_mf<N>(A.p, A.ld, A.ls, r, c)) : zero;
        const bool nz = !iszero(mag);
        // inclusive running maximum over the lanes, then shifted by one and
        // merged with the scale carried from the previous chunks
        mf<N> pm = mag;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            mf<N> o;
#pragma unroll
            for (int l = 0; l < N; ++l) o.v[l] = __shfl_up_sync(FULL, pm.v[l], off);
            if (lane >= off && gt(o, pm)) pm = o;
        }
        mf<N> before;
#pragma unroll
        for (int l = 0; l < N; ++l) before.v[l] = __shfl_up_sync(FULL, pm.v[l], 1);
        if (lane == 0 || gt(scale, before)) before = scale;
        const bool isnew = nz && gt(mag, before);
        mf<N> ratio = zero, sq = zero;
        if (nz && !iszero(before)) {
            ratio = isnew ? div(before, mag) : div(mag, before);
            sq = mul(ratio, ratio);
        }
#pragma unroll
        for (int l = 0; l < N; ++l) {
            bmag[l * 32 + lane] = mag.v[l];
            brat[l * 32 + lane] = ratio.v[l];
            bsq[l * 32 + lane] = sq.v[l];
        }
        bflag[lane] = (nz ? 1 : 0) | (isnew ? 2 : 0);
        __syncwarp();
        if (lane == 0) {
            for (int i = 0; i < 32; ++i) {
                const int f = bflag[i];
                if (!(f & 1)) continue;
                mf<N> mi, ri, si;
#pragma unroll
                for (int l = 0; l < N; ++l) {
                    mi.v[l] = bmag[l * 32 + i];
                    ri.v[l] = brat[l * 32 + i];
                    si.v[l] = bsq[l * 32 + i];
                }
                if (!seen) {
                    scale = mi;
                    sum = one;
                    seen = true;
                } else if (f & 2) {
                    sum = add(one, mul(mul(sum, ri), ri));
                    scale = mi;
                } else {
                    sum = add(sum, si);
                }
            }
        }
        __syncwarp();
#pragma unroll
        for (int l = 0; l < N; ++l) {
            scale.v[l] = __shfl_sync(FULL, scale.v[l], 0);
            sum.v[l] = __shfl_sync(FULL, sum.v[l], 0);
        }
        seen = __shfl_sync(FULL, seen ? 1 : 0, 0) != 0;
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
    // the steps of the unblocked loops are programmatic dependents of one
    // another: wait for the previous grid, let the next one be placed
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    __shared__ double slead[N];
    __shared__ int go;
    __shared__ double nbuf[QR_NORM_BUF(N)];
    const int tid = threadIdx.x;
    mf<N> scale, sum;
    if (tid < 32) norm_state_warp<N>(A, m, s, s, nbuf, scale, sum);
    if (tid == 0) {
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

// acc folded over rows r0..m-1 in ascending order, acc = acc + X[r,cx] *
// Y[r,cy], by one warp: the lanes form 32 products at a time, lane 0 adds
// them in row order (the reference's chain; only the additions are
// sequential).  All 32 lanes call it; buf holds 32 N doubles of this warp;
// the result is returned in every lane.
template <int N>
__device__ mf<N> chain_warp(mf<N> acc, int64_t r0, int64_t m, const Mat &X, int64_t cx,
                            const Mat &Y, int64_t cy, double *buf) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    for (int64_t base = r0; base < m; base += 32) {
        const int64_t r = base + lane;
        mf<N> pr = from_double<N>(0.0);
        if (r < m) pr = mul(load_mf<N>(X.p, X.ld, X.ls, r, cx), load_mf<N>(Y.p, Y.ld, Y.ls, r, cy));
#pragma unroll
        for (int l = 0; l < N; ++l) buf[l * 32 + lane] = pr.v[l];
        __syncwarp();
        if (lane == 0) {
            const int cnt = m - base < 32 ? (int)(m - base) : 32;
            for (int i = 0; i < cnt; ++i) {
                mf<N> x;
#pragma unroll
                for (int l = 0; l < N; ++l) x.v[l] = buf[l * 32 + i];
                acc = add(acc, x);
            }
        }
        __syncwarp();
    }
#pragma unroll
    for (int l = 0; l < N; ++l) acc.v[l] = __shfl_sync(FULL, acc.v[l], 0);
    return acc;
}

// reflector s of V (implicit one at row s) applied to column c of D by one
// warp (qr.jl:624-642): the projection chain, then the rank-one update with
// the rows spread over the lanes
template <int N>
__device__ __forceinline__ void apply_reflector_col_warp(int64_t m, int64_t s, const Mat &V,
                                                         const mf<N> &t, const Mat &D, int64_t c,
                                                         double *buf) {
    const int lane = threadIdx.x & 31;
    mf<N> proj = chain_warp<N>(load_mf<N>(D.p, D.ld, D.ls, s, c), s + 1, m, V, s, D, c, buf);
    proj = mul(proj, t);
    if (lane == 0) store_mf<N>(D.p, D.ld, D.ls, s, c, sub(load_mf<N>(D.p, D.ld, D.ls, s, c), proj));
    for (int64_t r = s + 1 + lane; r < m; r += 32)
        store_mf<N>(D.p, D.ld, D.ls, r, c,
                    submul(load_mf<N>(D.p, D.ld, D.ls, r, c), load_mf<N>(V.p, V.ld, V.ls, r, s), proj));
    __syncwarp();
}

constexpr int QR_COL_WARPS = 4;  // columns (one warp each) per CTA

static inline unsigned warp_col_grid(int64_t cols) {
    return (unsigned)((cols + QR_COL_WARPS - 1) / QR_COL_WARPS);
}

template <int N>
__global__ void __launch_bounds__(32 * QR_COL_WARPS)
    qr_apply_kernel(int64_t m, int64_t s, Mat V, const double *tau, int64_t lt, Mat D, int64_t c0,
                    int64_t nd) {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    __shared__ double buf[QR_COL_WARPS][32 * N];
    const int w = threadIdx.x >> 5;
    const int64_t j = (int64_t)blockIdx.x * QR_COL_WARPS + w;
    if (j >= nd) return;  // whole warps leave together
    mf<N> t;
#pragma unroll
    for (int l = 0; l < N; ++l) t.v[l] = tau[l * lt + s];
    if (iszero(t)) return;
    apply_reflector_col_warp<N>(m, s, V, t, D, c0 + j, buf[w]);
}

// apply_q! (qr.jl:890-956): every reflector in order on one column of D
template <int N>
__global__ void __launch_bounds__(32 * QR_COL_WARPS)
    qr_apply_all_kernel(int64_t m, int64_t r, Mat V, const double *tau, int64_t lt, Mat D,
                        int64_t nd, int trans) {
    __shared__ double buf[QR_COL_WARPS][32 * N];
    const int w = threadIdx.x >> 5;
    const int64_t c = (int64_t)blockIdx.x * QR_COL_WARPS + w;
    if (c >= nd) return;
    for (int64_t i = 0; i < r; ++i) {
        const int64_t s = trans ? i : r - 1 - i;
        mf<N> t;
#pragma unroll
        for (int l = 0; l < N; ++l) t.v[l] = tau[l * lt + s];
        if (iszero(t)) continue;
        apply_reflector_col_warp<N>(m, s, V, t, D, c, buf[w]);
    }
}

// norm state of columns c0..n-1 from rows r0 (qr.jl:143-155, 417-448), one
// warp per column
constexpr int QR_NORM_WARPS = 4;

template <int N>
__global__ void __launch_bounds__(32 * QR_NORM_WARPS)
    qr_norm_init_kernel(int64_t m, int64_t r0, int64_t c0, Mat A, QRNorms<N> S) {
    __shared__ double nbuf[QR_NORM_WARPS][QR_NORM_BUF(N)];
    const int w = threadIdx.x >> 5;
    const int64_t c = c0 + (int64_t)blockIdx.x * QR_NORM_WARPS + w;
    if (c >= S.n) return;  // whole warps leave together
    mf<N> scale, sum;
    norm_state_warp<N>(A, m, r0, c, nbuf[w], scale, sum);
    if ((threadIdx.x & 31) == 0) {
        S.set(c, scale, sum);
        S.dirty[c] = 0;
    }
}

static inline unsigned norm_grid(int64_t cols) {
    return (unsigned)((cols + QR_NORM_WARPS - 1) / QR_NORM_WARPS);
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
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
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
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    __shared__ int64_t sp;
    __shared__ double nbuf[QR_NORM_BUF(N)];
    if (threadIdx.x < 32) {
        // warp 0 walks the columns in order; every lane takes the same
        // branches (the state it reads is the same), lane 0 writes
        const bool w0 = threadIdx.x == 0;
        const mf<N> om = one_minus_margin.get();
        int64_t piv = step;
        mf<N> sc, su;
        norm_state_warp<N>(A, m, step, step, nbuf, sc, su);
        if (w0) {
            S.set(step, sc, su);
            S.dirty[step] = 0;
        }
        __syncwarp();
        mf<N> pn = norm_value(sc, su);
        for (int64_t c = step + 1; c < S.n; ++c) {
            mf<N> cn = norm_value(S.sc(c), S.su(c));
            if (S.dirty[c] || iszero(pn) || ge(cn, mul(om, pn))) {
                norm_state_warp<N>(A, m, step, c, nbuf, sc, su);
                __syncwarp();
                if (w0) {
                    S.set(c, sc, su);
                    S.dirty[c] = 0;
                }
                __syncwarp();
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
        if (w0) sp = piv;
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
__global__ void __launch_bounds__(32 * QR_COL_WARPS)
    qr_dlaqps_columns_kernel(int64_t m, int64_t step, int64_t bs, int64_t ls, Mat A,
                             const double *tau, int64_t lt, const double *aux, Mat F, QRNorms<N> S,
                             scal<N> floor_, int *unreliable) {
    __shared__ double buf[QR_COL_WARPS][32 * N];
    const int w = threadIdx.x >> 5;
    const int64_t c = step + 1 + (int64_t)blockIdx.x * QR_COL_WARPS + w;
    if (c >= S.n) return;  // whole warps leave together
    mf<N> t;
#pragma unroll
    for (int l = 0; l < N; ++l) t.v[l] = tau[l * lt + step];
    // gemv! trans = :T chain of column c with the reflector (rows step..m-1)
    const mf<N> acc = chain_warp<N>(from_double<N>(0.0), step, m, A, c, A, step, buf[w]);
    if ((threadIdx.x & 31) != 0) return;
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
        // each step's kernels are programmatic dependent launches
        for (int64_t st = 0; st < r; ++st) {
            int rc = launch_programmatic(qr_reflector_kernel<N>, dim3(1), dim3(QR_CTA), 0, s,
                                         "qr reflector", m, st, A, tau, lt, 0, nullptr, 0, 0,
                                         nullptr);
            if (rc) return rc;
            if (st + 1 < n) {
                rc = launch_programmatic(qr_apply_kernel<N>, dim3(warp_col_grid(n - st - 1)),
                                         dim3(32 * QR_COL_WARPS), 0, s, "qr apply", m, st, A,
                                         (const double *)tau, lt, A, st + 1, n - st - 1);
                if (rc) return rc;
            }
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
            qr_norm_init_kernel<N><<<norm_grid(n), 32 * QR_NORM_WARPS, 0, s>>>(m, 0, 0, A, S);
        const bool blocked = r >= QR_BLOCK && m * n >= 16384;
        if (!blocked) {
            for (int64_t st = 0; st < r; ++st) {
                int rc = launch_programmatic(qr_hybrid_pivot_kernel<N>, dim3(1), dim3(QR_CTA), 0,
                                             s, "qr pivot", m, st, A, perm, S, om);
                if (rc == MFLAB_OK)
                    rc = launch_programmatic(qr_reflector_kernel<N>, dim3(1), dim3(QR_CTA), 0, s,
                                             "qr reflector", m, st, A, tau, lt, 0, nullptr, 0, 0,
                                             nullptr);
                if (rc == MFLAB_OK && st + 1 < n) {
                    rc = launch_programmatic(qr_apply_kernel<N>, dim3(warp_col_grid(n - st - 1)),
                                             dim3(32 * QR_COL_WARPS), 0, s, "qr apply", m, st, A,
                                             (const double *)tau, lt, A, st + 1, n - st - 1);
                    if (rc == MFLAB_OK)
                        rc = launch_programmatic(
                            qr_update_norms_kernel<N>, dim3(col_grid(n - st - 1)),
                            dim3(QR_COLS_PER_CTA), 0, s, "qr norms", m, st, A,
                            (const double *)tau, lt, S, fl);
                }
                if (rc) return rc;
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
                        qr_dlaqps_columns_kernel<N><<<warp_col_grid(n - st - 1), 32 * QR_COL_WARPS, 0, s>>>(
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
                    qr_norm_init_kernel<N><<<norm_grid(n - be), 32 * QR_NORM_WARPS, 0, s>>>(m, be, be, A, S);
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
    MFLAB_RANGE("mflab_qr");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (pivoted & ~1) return MFLAB_ERR_FLAG;
    if (m < 0 || n < 0 || !tau || !perm || !info) return MFLAB_ERR_ARG;
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
    MFLAB_RANGE("mflab_apply_q");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (trans & ~1) return MFLAB_ERR_FLAG;
    if (m < 0 || r < 0 || nd < 0 || r > m) return MFLAB_ERR_ARG;
    if (m == 0 || nd == 0 || r == 0) return MFLAB_OK;
    if (ldf < m || ldd < m || lst < r) return MFLAB_ERR_ARG;
    if (mfl::views_overlap(D, ldd, lsd, m, nd, limbs, F, ldf, lsf, m, r)) return MFLAB_ERR_ALIAS;
    const Mat Fm{(double *)F, ldf, lsf}, Dm{D, ldd, lsd};
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned g = mfl::warp_col_grid(nd);
    const unsigned bt = 32 * mfl::QR_COL_WARPS;
    switch (limbs) {
    case 2: mfl::qr_apply_all_kernel<2><<<g, bt, 0, s>>>(m, r, Fm, tau, lst, Dm, nd, trans); break;
    case 3: mfl::qr_apply_all_kernel<3><<<g, bt, 0, s>>>(m, r, Fm, tau, lst, Dm, nd, trans); break;
    default: mfl::qr_apply_all_kernel<4><<<g, bt, 0, s>>>(m, r, Fm, tau, lst, Dm, nd, trans); break;
    }
    return mfl::record_cuda_error(cudaGetLastError(), "apply_q launch");
}

extern "C" int mflab_qr_numerical_rank(mflab_handle *h, void *stream, int limbs, int64_t m,
                                       int64_t n, const double *F, int64_t ldf, int64_t lsf,
                                       const double *atol, const double *rtol, int64_t *rank) {
    MFLAB_RANGE("mflab_qr_numerical_rank");
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
