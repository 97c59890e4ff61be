// Bunch-Kaufman LDL^T (1x1 and 2x2 pivots) with its solve and inertia.
//
// Follows src/factorizations/ldlt.jl of MultiFloatLinearAlgebra.jl:
//   * unblocked route (ldlt.jl:352-412): one cooperative CTA runs the pivot
//     steps; each step's column scan, row scan, symmetric swap, column scaling
//     and rank-1 / rank-2 update are spread over the CTA's threads, the pivot
//     decisions are taken by thread 0 exactly as ldlt.jl:183-219 orders them;
//   * blocked route (ldlt_gemmt.jl:36-73): per panel one cooperative CTA runs
//     the lazy panel (every entry evaluated against the earlier pivots of the
//     panel, ldlt.jl:414-593), then W = L21 * D (ldlt.jl:595-632), the lower
//     trailing update A22 = -1 * L21 W^T + 1 * A22 through the shared mainloop
//     (gemmt) and the upper mirror.
// Every per-element expression and its association is the reference's, so the
// result is bitwise the oracle's; the parallel loops only distribute
// independent elements.  When a step fails (info > 0) the factor content after
// that step is left as the parallel loop wrote it.
#include "mf_device.cuh"
#include "mflab_internal.h"

namespace mfl {

template <int N>
struct Ldlt {
    Mat A;
    int64_t n;
    double *dsub;  // dsub[l * lsd + k]
    int64_t lsd;
    int64_t *pivots;  // 1-based
    uint8_t *blocks;
    __device__ mf<N> at(int64_t r, int64_t c) const { return load_mf<N>(A.p, A.ld, A.ls, r, c); }
    __device__ void put(int64_t r, int64_t c, const mf<N> &v) const {
        store_mf<N>(A.p, A.ld, A.ls, r, c, v);
    }
    __device__ mf<N> ds(int64_t k) const {
        mf<N> v;
#pragma unroll
        for (int l = 0; l < N; ++l) v.v[l] = dsub[l * lsd + k];
        return v;
    }
    __device__ void set_ds(int64_t k, const mf<N> &v) const {
#pragma unroll
        for (int l = 0; l < N; ++l) dsub[l * lsd + k] = v.v[l];
    }
    // lazily updated Schur-complement entry (ldlt.jl:414-449)
    __device__ mf<N> panel_entry(int64_t i1, int64_t i2, int64_t pf, int64_t pivot_first) const {
        const int64_t row = i1 > i2 ? i1 : i2, col = i1 > i2 ? i2 : i1;
        mf<N> v = at(row, col);
        int64_t q = pf;
        while (q < pivot_first) {
            if (blocks[q] == 1) {
                v = sub(v, mul(at(row, q), mul(at(q, q), at(col, q))));
                q += 1;
            } else {
                const mf<N> rf = at(row, q), rs = at(row, q + 1);
                const mf<N> cf = at(col, q), cs = at(col, q + 1);
                const mf<N> c1 = add(mul(at(q, q), cf), mul(ds(q), cs));
                const mf<N> c2 = add(mul(ds(q), cf), mul(at(q + 1, q + 1), cs));
                v = sub(v, add(mul(rf, c1), mul(rs, c2)));
                q += 2;
            }
        }
        return v;
    }
    __device__ mf<N> entry(int64_t i, int64_t j, bool lazy, int64_t pf, int64_t k) const {
        return lazy ? panel_entry(i, j, pf, k) : at(i, j);
    }
};

// ldlt.jl:65-101; returns nonsingular
template <int N>
__device__ bool solve_2x2(const mf<N> &d11, const mf<N> &d21, const mf<N> &d22, const mf<N> &first,
                          const mf<N> &second, mf<N> &x1, mf<N> &x2) {
    const mf<N> scale = max_mf(max_mf(abs_mf(d11), abs_mf(d21)), abs_mf(d22));
    x1 = from_double<N>(0.0);
    x2 = from_double<N>(0.0);
    if (iszero(scale) || !isfinite_mf(scale)) return false;
    const mf<N> a = div(d11, scale), b = div(d21, scale), c = div(d22, scale);
    const mf<N> r1 = div(first, scale), r2 = div(second, scale);
    if (ge(abs_mf(a), abs_mf(b))) {
        if (iszero(a)) return false;
        const mf<N> t = div(b, a);
        const mf<N> u = submul(c, t, b);
        if (iszero(u) || !isfinite_mf(u)) return false;
        const mf<N> y2 = div(submul(r2, t, r1), u);
        x1 = div(submul(r1, b, y2), a);
        x2 = y2;
        return true;
    }
    if (iszero(b)) return false;
    const mf<N> t = div(a, b);
    const mf<N> u = submul(b, t, c);
    if (iszero(u) || !isfinite_mf(u)) return false;
    const mf<N> y2 = div(submul(r1, t, r2), u);
    x1 = div(submul(r2, c, y2), b);
    x2 = y2;
    return true;
}

// shared scratch of the cooperative kernels
template <int N, int NT>
struct CoopShared {
    double val[NT][N];
    int64_t idx[NT];
    double bcast[8][N];
    int64_t ibcast[4];
    int flag;
};

// first strictly larger |entry(r, k)| over r in [r0, n) (smallest index among the maxima)
template <int N, int NT>
__device__ void coop_colmax(const Ldlt<N> &F, CoopShared<N, NT> &sh, int64_t r0, int64_t k,
                            bool lazy, int64_t pf, mf<N> &best, int64_t &bidx) {
    const int t = threadIdx.x;
    mf<N> b = from_double<N>(0.0);
    int64_t bi = -1;
    for (int64_t r = r0 + t; r < F.n; r += NT) {
        const mf<N> c = abs_mf(F.entry(r, k, lazy, pf, k));
        if (bi < 0 || gt(c, b)) {
            b = c;
            bi = r;
        }
    }
#pragma unroll
    for (int l = 0; l < N; ++l) sh.val[t][l] = b.v[l];
    sh.idx[t] = bi;
    __syncthreads();
    for (int off = NT / 2; off > 0; off >>= 1) {
        if (t < off) {
            mf<N> a, c;
#pragma unroll
            for (int l = 0; l < N; ++l) {
                a.v[l] = sh.val[t][l];
                c.v[l] = sh.val[t + off][l];
            }
            const int64_t ia = sh.idx[t], ic = sh.idx[t + off];
            bool take;
            if (ic < 0) take = false;
            else if (ia < 0) take = true;
            else if (gt(c, a)) take = true;
            else if (gt(a, c)) take = false;
            else take = ic < ia;
            if (take) {
#pragma unroll
                for (int l = 0; l < N; ++l) sh.val[t][l] = c.v[l];
                sh.idx[t] = ic;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int l = 0; l < N; ++l) best.v[l] = sh.val[0][l];
    bidx = sh.idx[0];
    __syncthreads();
}

// max |entry| along row imax of the active matrix (ldlt.jl:203-209)
template <int N, int NT>
__device__ mf<N> coop_rowmax(const Ldlt<N> &F, CoopShared<N, NT> &sh, int64_t k, int64_t imax,
                             bool lazy, int64_t pf) {
    const int t = threadIdx.x;
    mf<N> b = from_double<N>(0.0);
    for (int64_t c = k + t; c < imax; c += NT) b = max_mf(b, abs_mf(F.entry(imax, c, lazy, pf, k)));
    for (int64_t r = imax + 1 + t; r < F.n; r += NT) b = max_mf(b, abs_mf(F.entry(r, imax, lazy, pf, k)));
#pragma unroll
    for (int l = 0; l < N; ++l) sh.val[t][l] = b.v[l];
    __syncthreads();
    for (int off = NT / 2; off > 0; off >>= 1) {
        if (t < off) {
            mf<N> a, c;
#pragma unroll
            for (int l = 0; l < N; ++l) {
                a.v[l] = sh.val[t][l];
                c.v[l] = sh.val[t + off][l];
            }
            const mf<N> r = max_mf(a, c);
#pragma unroll
            for (int l = 0; l < N; ++l) sh.val[t][l] = r.v[l];
        }
        __syncthreads();
    }
    mf<N> out;
#pragma unroll
    for (int l = 0; l < N; ++l) out.v[l] = sh.val[0][l];
    __syncthreads();
    return out;
}

template <int N, int NT>
__device__ void put_bcast(CoopShared<N, NT> &sh, int slot, const mf<N> &v) {
#pragma unroll
    for (int l = 0; l < N; ++l) sh.bcast[slot][l] = v.v[l];
}
template <int N, int NT>
__device__ mf<N> get_bcast(CoopShared<N, NT> &sh, int slot) {
    mf<N> v;
#pragma unroll
    for (int l = 0; l < N; ++l) v.v[l] = sh.bcast[slot][l];
    return v;
}

// Bunch-Kaufman pivot choice (ldlt.jl:183-219 / 451-508); returns block size,
// pivot row in *piv.  All threads call it and get the same answer.
template <int N, int NT>
__device__ int select_bk(const Ldlt<N> &F, CoopShared<N, NT> &sh, int64_t k, const mf<N> &alpha,
                         bool lazy, int64_t pf, int64_t *piv) {
    const int t = threadIdx.x;
    const int64_t n = F.n;
    if (t == 0) put_bcast(sh, 0, abs_mf(F.entry(k, k, lazy, pf, k)));
    __syncthreads();
    const mf<N> absakk = get_bcast(sh, 0);
    __syncthreads();
    if (k == n - 1) {
        *piv = k;
        return iszero(absakk) ? 0 : 1;
    }
    mf<N> colmax;
    int64_t imax;
    coop_colmax(F, sh, k + 1, k, lazy, pf, colmax, imax);
    if (iszero(max_mf(absakk, colmax))) {
        *piv = k;
        return 0;
    }
    if (ge(absakk, mul(alpha, colmax))) {
        *piv = k;
        return 1;
    }
    const mf<N> rowmax = coop_rowmax(F, sh, k, imax, lazy, pf);
    if (ge(absakk, mul(mul(alpha, colmax), div(colmax, rowmax)))) {
        *piv = k;
        return 1;
    }
    if (t == 0) put_bcast(sh, 1, abs_mf(F.entry(imax, imax, lazy, pf, k)));
    __syncthreads();
    const mf<N> cand = get_bcast(sh, 1);
    __syncthreads();
    *piv = imax;
    return ge(cand, mul(alpha, rowmax)) ? 1 : 2;
}

// P A P^T on the active part plus the row swap of the earlier L columns
// (ldlt.jl:155-181): all rows first, then the active columns.
template <int N, int NT>
__device__ void coop_sym_swap(const Ldlt<N> &F, int64_t a, int64_t b, int64_t active_first) {
    if (a == b) return;
    const int t = threadIdx.x;
    for (int64_t c = t; c < F.n; c += NT) {
#pragma unroll
        for (int l = 0; l < N; ++l) {
            double *col = F.A.p + l * F.A.ls + c * F.A.ld;
            const double x = col[a];
            col[a] = col[b];
            col[b] = x;
        }
    }
    __syncthreads();
    for (int64_t r = active_first + t; r < F.n; r += NT) {
#pragma unroll
        for (int l = 0; l < N; ++l) {
            double *pa = F.A.p + l * F.A.ls + a * F.A.ld + r;
            double *pb = F.A.p + l * F.A.ls + b * F.A.ld + r;
            const double x = *pa;
            *pa = *pb;
            *pb = x;
        }
    }
    __syncthreads();
}

// unblocked route, one CTA (ldlt.jl:352-412)
template <int N, int NT>
__global__ void __launch_bounds__(NT) ldlt_unblocked_kernel(Ldlt<N> F, scal<N> alpha_s, int *info) {
    __shared__ CoopShared<N, NT> sh;
    if (*info) return;
    const int t = threadIdx.x;
    const int64_t n = F.n;
    const mf<N> alpha = alpha_s.get();
    int64_t k = 0;
    while (k < n) {
        int64_t piv;
        const int bs = select_bk<N, NT>(F, sh, k, alpha, false, 0, &piv);
        if (bs == 0) {
            if (t == 0) *info = (int)(k + 1);
            return;
        }
        if (bs == 1) {
            if (t == 0) {
                F.pivots[k] = piv + 1;
                F.blocks[k] = 1;
            }
            coop_sym_swap<N, NT>(F, k, piv, k);
            const mf<N> d = F.at(k, k);
            if (iszero(d)) {
                if (t == 0) *info = (int)(k + 1);
                return;
            }
            for (int64_t r = k + 1 + t; r < n; r += NT) F.put(r, k, div(F.at(r, k), d));
            __syncthreads();
            if (k < n - 1) {
                // rank-1 update of the lower active part with its mirror
                const int64_t m = n - k - 1;
                const int64_t tot = m * (m + 1) / 2;
                for (int64_t e = t; e < tot; e += NT) {
                    // column-major enumeration of the lower triangle of the active part
                    int64_t c = (int64_t)((2.0 * m + 1.0 - sqrt((2.0 * m + 1.0) * (2.0 * m + 1.0) - 8.0 * e)) / 2.0);
                    while (c > 0 && c * m - c * (c - 1) / 2 > e) --c;
                    while ((c + 1) * m - (c + 1) * c / 2 <= e) ++c;
                    const int64_t r = c + (e - (c * m - c * (c - 1) / 2));
                    const int64_t col = k + 1 + c, row = k + 1 + r;
                    const mf<N> coef = mul(d, F.at(col, k));
                    const mf<N> v = submul(F.at(row, col), F.at(row, k), coef);
                    F.put(row, col, v);
                    F.put(col, row, v);
                }
                __syncthreads();
            }
            k += 1;
        } else {
            if (!(k < n - 1)) {
                if (t == 0) *info = (int)(k + 1);
                return;
            }
            if (t == 0) {
                F.pivots[k] = piv + 1;
                F.blocks[k] = 2;
                F.blocks[k + 1] = 0;
            }
            coop_sym_swap<N, NT>(F, k + 1, piv, k);
            const mf<N> d11 = F.at(k, k), d21 = F.at(k + 1, k), d22 = F.at(k + 1, k + 1);
            if (t == 0) F.set_ds(k, d21);
            mf<N> x1, x2;
            if (!solve_2x2(d11, d21, d22, from_double<N>(0.0), from_double<N>(0.0), x1, x2)) {
                if (t == 0) *info = (int)(k + 1);
                return;
            }
            if (t == 0) sh.flag = 0;
            __syncthreads();
            for (int64_t r = k + 2 + t; r < n; r += NT) {
                const bool ok = solve_2x2(d11, d21, d22, F.at(r, k), F.at(r, k + 1), x1, x2);
                if (!(ok && isfinite_mf(x1) && isfinite_mf(x2))) {
                    sh.flag = 1;
                } else {
                    F.put(r, k, x1);
                    F.put(r, k + 1, x2);
                }
            }
            __syncthreads();
            if (sh.flag) {
                if (t == 0) *info = (int)(k + 1);
                return;
            }
            if (k + 1 < n - 1) {
                // rank-2 update (ldlt.jl:261-326): rows in full groups of four
                // from the column use v - (f1 c1 + f2 c2), the remainder rows
                // (v - f1 c1) - f2 c2
                const int64_t m = n - k - 2;
                const int64_t tot = m * (m + 1) / 2;
                for (int64_t e = t; e < tot; e += NT) {
                    int64_t c = (int64_t)((2.0 * m + 1.0 - sqrt((2.0 * m + 1.0) * (2.0 * m + 1.0) - 8.0 * e)) / 2.0);
                    while (c > 0 && c * m - c * (c - 1) / 2 > e) --c;
                    while ((c + 1) * m - (c + 1) * c / 2 <= e) ++c;
                    const int64_t r = c + (e - (c * m - c * (c - 1) / 2));
                    const int64_t col = k + 2 + c, row = k + 2 + r;
                    const mf<N> l1 = F.at(col, k), l2 = F.at(col, k + 1);
                    const mf<N> c1 = add(mul(d11, l1), mul(d21, l2));
                    const mf<N> c2 = add(mul(d21, l1), mul(d22, l2));
                    const mf<N> v0 = F.at(row, col), f1 = F.at(row, k), f2 = F.at(row, k + 1);
                    const int64_t span = n - col;  // rows col..n-1
                    const bool grouped = (row - col) < 4 * (span / 4);
                    mf<N> v;
                    if (grouped)
                        v = sub(v0, add(mul(f1, c1), mul(f2, c2)));
                    else
                        v = submul(submul(v0, f1, c1), f2, c2);
                    F.put(row, col, v);
                    F.put(col, row, v);
                }
                __syncthreads();
            }
            if (t == 0) {
                F.put(k + 1, k, from_double<N>(0.0));
                F.put(k, k + 1, from_double<N>(0.0));
            }
            __syncthreads();
            k += 2;
        }
    }
}

// one lazy panel (ldlt.jl:510-593); status[0] = info, status[1] = panel_last
template <int N, int NT>
__global__ void __launch_bounds__(NT) ldlt_panel_kernel(Ldlt<N> F, scal<N> alpha_s, int64_t pf,
                                                        int64_t requested_last, int *info,
                                                        int64_t *panel_last_out) {
    __shared__ CoopShared<N, NT> sh;
    if (*info) return;
    const int t = threadIdx.x;
    const int64_t n = F.n;
    const mf<N> alpha = alpha_s.get();
    int64_t pl = requested_last;
    int64_t k = pf;
    auto fail = [&](int64_t kk) {
        if (t == 0) {
            *info = (int)(kk + 1);
            *panel_last_out = pl;
        }
    };
    while (k <= pl) {
        int64_t piv;
        const int bs = select_bk<N, NT>(F, sh, k, alpha, true, pf, &piv);
        if (bs == 0) return fail(k);
        if (bs == 2 && k == pl) {
            if (!(k < n - 1)) return fail(k);
            pl += 1;
        }
        if (bs == 1) {
            if (t == 0) {
                F.pivots[k] = piv + 1;
                F.blocks[k] = 1;
            }
            coop_sym_swap<N, NT>(F, k, piv, k);
            const mf<N> d = F.panel_entry(k, k, pf, k);
            if (iszero(d)) return fail(k);
            // entries first (they read column k's unswapped-then-swapped values
            // and the earlier pivots), then the writes
            __syncthreads();
            if (t == 0) F.put(k, k, d);
            for (int64_t r = k + 1 + t; r < n; r += NT) F.put(r, k, div(F.panel_entry(r, k, pf, k), d));
            __syncthreads();
            k += 1;
        } else {
            if (t == 0) {
                F.pivots[k] = piv + 1;
                F.blocks[k] = 2;
                F.blocks[k + 1] = 0;
            }
            coop_sym_swap<N, NT>(F, k + 1, piv, k);
            const mf<N> d11 = F.panel_entry(k, k, pf, k);
            const mf<N> d21 = F.panel_entry(k + 1, k, pf, k);
            const mf<N> d22 = F.panel_entry(k + 1, k + 1, pf, k);
            __syncthreads();
            if (t == 0) {
                F.put(k, k, d11);
                F.put(k + 1, k + 1, d22);
                F.set_ds(k, d21);
                sh.flag = 0;
            }
            mf<N> x1, x2;
            if (!solve_2x2(d11, d21, d22, from_double<N>(0.0), from_double<N>(0.0), x1, x2))
                return fail(k);
            __syncthreads();
            for (int64_t r = k + 2 + t; r < n; r += NT) {
                const mf<N> e1 = F.panel_entry(r, k, pf, k), e2 = F.panel_entry(r, k + 1, pf, k);
                const bool ok = solve_2x2(d11, d21, d22, e1, e2, x1, x2);
                if (!(ok && isfinite_mf(x1) && isfinite_mf(x2))) {
                    sh.flag = 1;
                } else {
                    F.put(r, k, x1);
                    F.put(r, k + 1, x2);
                }
            }
            __syncthreads();
            if (sh.flag) return fail(k);
            if (t == 0) {
                F.put(k + 1, k, from_double<N>(0.0));
                F.put(k, k + 1, from_double<N>(0.0));
            }
            __syncthreads();
            k += 2;
        }
    }
    if (t == 0) *panel_last_out = pl;
}

// W = L21 * D for the panel (ldlt.jl:595-632): one thread per trailing row
template <int N>
__global__ void ldlt_weighted_kernel(Ldlt<N> F, int64_t pf, int64_t pl, Mat W) {
    const int64_t lr = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t row = pl + 1 + lr;
    if (row >= F.n) return;
    int64_t q = pf;
    while (q <= pl) {
        const int64_t lc = q - pf;
        if (F.blocks[q] == 1) {
            store_mf<N>(W.p, W.ld, W.ls, lr, lc, mul(F.at(row, q), F.at(q, q)));
            q += 1;
        } else {
            const mf<N> d11 = F.at(q, q), d21 = F.ds(q), d22 = F.at(q + 1, q + 1);
            const mf<N> f = F.at(row, q), s = F.at(row, q + 1);
            store_mf<N>(W.p, W.ld, W.ls, lr, lc, add(mul(f, d11), mul(s, d21)));
            store_mf<N>(W.p, W.ld, W.ls, lr, lc + 1, add(mul(f, d21), mul(s, d22)));
            q += 2;
        }
    }
}

// upper mirror of a square block: A(c, r) = A(r, c) for r > c
template <int N>
__global__ void mirror_kernel(int64_t n, Mat A, const int *info) {
    if (info && *info) return;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * n) return;
    const int64_t r = e % n, c = e / n;
    if (r <= c) return;
#pragma unroll
    for (int l = 0; l < N; ++l) A.p[l * A.ls + r * A.ld + c] = A.p[l * A.ls + c * A.ld + r];
}

template <int N>
__global__ void ldlt_init_kernel(int64_t n, Mat A, double *dsub, int64_t lsd, int64_t *pivots,
                                 uint8_t *blocks, int *info) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    pivots[i] = i + 1;
    blocks[i] = 0;
#pragma unroll
    for (int l = 0; l < N; ++l) dsub[l * lsd + i] = 0.0;
}

template <int N>
__global__ void ldlt_lower_nonfinite_kernel(int64_t n, Mat A, int *info) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * n) return;
    const int64_t r = e % n, c = e / n;
    if (r < c) return;
    if (!isfinite_mf(load_mf<N>(A.p, A.ld, A.ls, r, c))) *info = -1;
}

template <int N>
__global__ void ldlt_alpha_kernel(double *out) {
    // (1 + sqrt(17)) / 8 in working precision (ldlt.jl:691)
    const mf<N> a = div(add(from_double<N>(1.0), sqrt_mf(from_double<N>(17.0))), from_double<N>(8.0));
#pragma unroll
    for (int l = 0; l < N; ++l) out[l] = a.v[l];
}

constexpr int LDLT_NT = 512;

template <int N>
static int sytrf_n(mflab_handle *h, int64_t n, Mat A, double *dsub, int64_t lsd, int64_t *pivots,
                   uint8_t *blocks, int blocked, int64_t block, int *info, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(info, 0, sizeof(int), s);
    if (e != cudaSuccess) return record_cuda_error(e, "sytrf info");
    if (n == 0) return MFLAB_OK;
    ldlt_init_kernel<N><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, A, dsub, lsd, pivots, blocks, info);
    ldlt_lower_nonfinite_kernel<N><<<(unsigned)((n * n + 255) / 256), 256, 0, s>>>(n, A, info);
    mirror_kernel<N><<<(unsigned)((n * n + 255) / 256), 256, 0, s>>>(n, A, info);
    int rc = record_cuda_error(cudaGetLastError(), "sytrf prepare");
    if (rc) return rc;
    // alpha in working precision, read back once
    const size_t wbytes = sizeof(double) * (size_t)N * (size_t)n * (size_t)(block + 1);
    rc = mflab_reserve_scratch(h, wbytes + 256 + 64);
    if (rc) return rc;
    double *W = (double *)h->scratch;
    double *alpha_dev = (double *)((char *)h->scratch + (wbytes + 255) / 256 * 256);
    int64_t *pl_dev = (int64_t *)(alpha_dev + 4);
    ldlt_alpha_kernel<N><<<1, 1, 0, s>>>(alpha_dev);
    scal<N> al{};
    double alpha_host[4] = {0, 0, 0, 0};
    e = cudaMemcpyAsync(alpha_host, alpha_dev, sizeof(double) * N, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return record_cuda_error(e, "sytrf alpha");
    for (int l = 0; l < N; ++l) al.v[l] = alpha_host[l];
    Ldlt<N> F{A, n, dsub, lsd, pivots, blocks};
    if (!blocked) {
        ldlt_unblocked_kernel<N, LDLT_NT><<<1, LDLT_NT, 0, s>>>(F, al, info);
        return record_cuda_error(cudaGetLastError(), "sytrf unblocked");
    }
    const double mone[4] = {-1.0, 0.0, 0.0, 0.0}, one[4] = {1.0, 0.0, 0.0, 0.0};
    int64_t pf = 0;
    while (pf < n) {
        const int64_t req = pf + block - 1 < n - 1 ? pf + block - 1 : n - 1;
        ldlt_panel_kernel<N, LDLT_NT><<<1, LDLT_NT, 0, s>>>(F, al, pf, req, info, pl_dev);
        rc = record_cuda_error(cudaGetLastError(), "sytrf panel");
        if (rc) return rc;
        int info_h = 0;
        int64_t pl = 0;
        e = cudaMemcpyAsync(&info_h, info, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&pl, pl_dev, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return record_cuda_error(e, "sytrf panel status");
        if (info_h) return MFLAB_OK;
        if (pl < n - 1) {
            const int64_t tc = n - 1 - pl, pw = pl - pf + 1;
            Mat Wm{W, n, n * (block + 1)};
            ldlt_weighted_kernel<N><<<(unsigned)((tc + 127) / 128), 128, 0, s>>>(F, pf, pl, Wm);
            rc = record_cuda_error(cudaGetLastError(), "sytrf weighted");
            if (rc) return rc;
            rc = launch_mm(N, false, true, 1, false, tc, tc, pw, A.at(pl + 1, pf), Wm,
                           A.at(pl + 1, pl + 1), mone, one, s, info);
            if (rc) return rc;
            mirror_kernel<N><<<(unsigned)((tc * tc + 255) / 256), 256, 0, s>>>(tc, A.at(pl + 1, pl + 1), info);
            rc = record_cuda_error(cudaGetLastError(), "sytrf mirror");
            if (rc) return rc;
        }
        pf = pl + 1;
    }
    return MFLAB_OK;
}

// ------------------------------------------------------------ solve -------
// forward (reverse == 0) / reverse row interchanges (solve.jl:213-249);
// one thread per right-hand-side column
template <int N>
__global__ void ldlt_pivots_kernel(int64_t n, int64_t nrhs, Mat B, const int64_t *pivots,
                                   const uint8_t *blocks, int reverse) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nrhs) return;
    auto swap = [&](int64_t a, int64_t b) {
        if (a == b) return;
#pragma unroll
        for (int l = 0; l < N; ++l) {
            double *x = B.p + l * B.ls + c * B.ld;
            const double t = x[a];
            x[a] = x[b];
            x[b] = t;
        }
    };
    if (!reverse) {
        int64_t k = 0;
        while (k < n) {
            if (blocks[k] == 1) {
                swap(k, pivots[k] - 1);
                k += 1;
            } else {
                swap(k + 1, pivots[k] - 1);
                k += 2;
            }
        }
    } else {
        int64_t k = n - 1;
        while (k >= 0) {
            if (blocks[k] == 1) {
                swap(k, pivots[k] - 1);
                k -= 1;
            } else {
                swap(k, pivots[k - 1] - 1);
                k -= 2;
            }
        }
    }
}

// D solve (solve.jl:251-296): independent per (block, column)
template <int N>
__global__ void ldlt_dsolve_kernel(int64_t n, int64_t nrhs, Mat F, const double *dsub,
                                   int64_t lsd, const uint8_t *blocks, Mat B, int *fail) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t c = blockIdx.y;
    if (k >= n || c >= nrhs) return;
    if (blocks[k] == 1) {
        store_mf<N>(B.p, B.ld, B.ls, k, c,
                    div(load_mf<N>(B.p, B.ld, B.ls, k, c), load_mf<N>(F.p, F.ld, F.ls, k, k)));
    } else if (blocks[k] == 2) {
        mf<N> d21;
#pragma unroll
        for (int l = 0; l < N; ++l) d21.v[l] = dsub[l * lsd + k];
        mf<N> x1, x2;
        const bool ok = solve_2x2(load_mf<N>(F.p, F.ld, F.ls, k, k), d21,
                                  load_mf<N>(F.p, F.ld, F.ls, k + 1, k + 1),
                                  load_mf<N>(B.p, B.ld, B.ls, k, c),
                                  load_mf<N>(B.p, B.ld, B.ls, k + 1, c), x1, x2);
        if (!ok) {
            atomicMin(fail, (int)(k + 1));
        } else {
            store_mf<N>(B.p, B.ld, B.ls, k, c, x1);
            store_mf<N>(B.p, B.ld, B.ls, k + 1, c, x2);
        }
    }
}

// ----------------------------------------------------- diagnostics --------
// One thread: inertia, block counts and block quality of an LDLT factor
// (diagnostics.jl:109-246).  out: [0] positive [1] negative [2] zero
// [3] 1x1 count [4] 2x2 count [5] has-min-block, then N-limb values
// min block eigenvalue magnitude, max block entry.
template <int N>
__global__ void ldlt_diag_kernel(int64_t n, Mat F, const double *dsub, int64_t lsd,
                                 const uint8_t *blocks, const double *omax, double *out) {
    int64_t pos = 0, neg = 0, zer = 0, one = 0, two = 0;
    bool have_min = false;
    mf<N> minb = from_double<N>(0.0), maxe = from_double<N>(0.0);
    const mf<N> z = from_double<N>(0.0);
    int64_t k = 0;
    while (k < n) {
        const uint8_t b = blocks[k];
        if (b == 1) {
            const mf<N> v = load_mf<N>(F.p, F.ld, F.ls, k, k);
            if (gt(v, z)) pos++;
            else if (lt(v, z)) neg++;
            else zer++;
            one++;
            const mf<N> bv = abs_mf(v);
            minb = have_min ? min_mf(minb, bv) : bv;
            have_min = true;
            maxe = max_mf(maxe, bv);
            k += 1;
        } else if (b == 2 && k < n - 1) {
            two++;
            const mf<N> d11 = load_mf<N>(F.p, F.ld, F.ls, k, k);
            const mf<N> d22 = load_mf<N>(F.p, F.ld, F.ls, k + 1, k + 1);
            mf<N> d21;
#pragma unroll
            for (int l = 0; l < N; ++l) d21.v[l] = dsub[l * lsd + k];
            const mf<N> scale = max_mf(max_mf(abs_mf(d11), abs_mf(d21)), abs_mf(d22));
            // inertia of the 2x2 block (diagnostics.jl:118-134)
            if (iszero(scale)) {
                zer += 2;
            } else {
                const mf<N> a = div(d11, scale), bb = div(d21, scale), c = div(d22, scale);
                const mf<N> det = sub(mul(a, c), mul(bb, bb));
                const mf<N> tr = add(a, c);
                if (lt(det, z)) {
                    pos++;
                    neg++;
                } else if (gt(det, z)) {
                    if (gt(tr, z)) pos += 2;
                    else neg += 2;
                } else {
                    if (gt(tr, z)) {
                        pos++;
                        zer++;
                    } else if (lt(tr, z)) {
                        neg++;
                        zer++;
                    } else {
                        zer += 2;
                    }
                }
            }
            // smallest |eigenvalue| of the block (diagnostics.jl:136-154)
            mf<N> bv = z;
            if (!iszero(scale)) {
                const mf<N> a = div(d11, scale), bb = div(d21, scale), c = div(d22, scale);
                const mf<N> amc = sub(a, c);
                const mf<N> disc = sqrt_mf(add(mul(amc, amc), mul(mul(from_double<N>(4.0), bb), bb)));
                const mf<N> first = div(add(add(a, c), disc), from_double<N>(2.0));
                const mf<N> second = div(sub(add(a, c), disc), from_double<N>(2.0));
                const mf<N> largest = max_mf(abs_mf(first), abs_mf(second));
                if (!iszero(largest)) {
                    const mf<N> det = abs_mf(sub(mul(a, c), mul(bb, bb)));
                    bv = mul(scale, div(det, largest));
                }
            }
            minb = have_min ? min_mf(minb, bv) : bv;
            have_min = true;
            maxe = max_mf(max_mf(max_mf(maxe, abs_mf(d11)), abs_mf(d21)), abs_mf(d22));
            k += 2;
        } else {
            break;
        }
    }
    out[0] = (double)pos;
    out[1] = (double)neg;
    out[2] = (double)zer;
    out[3] = (double)one;
    out[4] = (double)two;
    out[5] = have_min ? 1.0 : 0.0;
    mf<N> om;
#pragma unroll
    for (int l = 0; l < N; ++l) om.v[l] = omax ? omax[l] : 0.0;
    const bool omz = iszero(om);
    const mf<N> scaled = (omz || !have_min) ? z : div(minb, om);
    const mf<N> growth = omz ? z : div(maxe, om);
#pragma unroll
    for (int l = 0; l < N; ++l) {
        out[6 + l] = minb.v[l];
        out[6 + N + l] = maxe.v[l];
        out[6 + 2 * N + l] = scaled.v[l];
        out[6 + 3 * N + l] = growth.v[l];
    }
}

}  // namespace mfl

using mfl::Mat;

extern "C" int mflab_sytrf(mflab_handle *h, void *stream, int limbs, int64_t n, double *A,
                           int64_t lda, int64_t lsa, double *dsub, int64_t lsd, int64_t *pivots,
                           uint8_t *blocks, int blocked, int64_t block, int *info) {
    MFLAB_RANGE("mflab_sytrf");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (n < 0 || (n > 0 && (lda < n || !dsub || !pivots || !blocks || lsd < n)) || !info)
        return MFLAB_ERR_ARG;
    if (blocked && block < 2) block = 2;
    if (block > 64) return MFLAB_ERR_UNSUPPORTED;
    Mat a{A, lda, lsa};
    cudaStream_t s = (cudaStream_t)stream;
    switch (limbs) {
    case 2: return mfl::sytrf_n<2>(h, n, a, dsub, lsd, pivots, blocks, blocked, block, info, s);
    case 3: return mfl::sytrf_n<3>(h, n, a, dsub, lsd, pivots, blocks, blocked, block, info, s);
    default: return mfl::sytrf_n<4>(h, n, a, dsub, lsd, pivots, blocks, blocked, block, info, s);
    }
}

extern "C" int mflab_sytrs(mflab_handle *h, void *stream, int limbs, int64_t n, int64_t nrhs,
                           const double *F, int64_t ldf, int64_t lsf, const double *dsub,
                           int64_t lsd, const int64_t *pivots, const uint8_t *blocks, double *B,
                           int64_t ldb, int64_t lsb, int *fail) {
    MFLAB_RANGE("mflab_sytrs");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (n < 0 || nrhs < 0 || (n > 0 && (ldf < n || ldb < n)) || !fail) return MFLAB_ERR_ARG;
    if (n == 0 || nrhs == 0) return MFLAB_OK;
    if (nrhs > 65535) return MFLAB_ERR_UNSUPPORTED;
    const double one[4] = {1.0, 0.0, 0.0, 0.0};
    cudaStream_t s = (cudaStream_t)stream;
    Mat f{(double *)F, ldf, lsf}, b{B, ldb, lsb};
    cudaError_t e = cudaMemsetAsync(fail, 0x7f, sizeof(int), s);  // 0x7f7f7f7f = no failure
    if (e != cudaSuccess) return mfl::record_cuda_error(e, "sytrs flag");
    const unsigned g = (unsigned)((nrhs + 127) / 128);
    const dim3 gd((unsigned)((n + 127) / 128), (unsigned)nrhs);
    int rc;
    switch (limbs) {
    case 2: mfl::ldlt_pivots_kernel<2><<<g, 128, 0, s>>>(n, nrhs, b, pivots, blocks, 0); break;
    case 3: mfl::ldlt_pivots_kernel<3><<<g, 128, 0, s>>>(n, nrhs, b, pivots, blocks, 0); break;
    default: mfl::ldlt_pivots_kernel<4><<<g, 128, 0, s>>>(n, nrhs, b, pivots, blocks, 0); break;
    }
    rc = mfl::launch_trsm_info(limbs, 0, 0, 0, 1, n, nrhs, f, b, one, s, nullptr, h->solve_order);
    if (rc) return rc;
    switch (limbs) {
    case 2: mfl::ldlt_dsolve_kernel<2><<<gd, 128, 0, s>>>(n, nrhs, f, dsub, lsd, blocks, b, fail); break;
    case 3: mfl::ldlt_dsolve_kernel<3><<<gd, 128, 0, s>>>(n, nrhs, f, dsub, lsd, blocks, b, fail); break;
    default: mfl::ldlt_dsolve_kernel<4><<<gd, 128, 0, s>>>(n, nrhs, f, dsub, lsd, blocks, b, fail); break;
    }
    rc = mfl::launch_trsm_info(limbs, 0, 0, 1, 1, n, nrhs, f, b, one, s, nullptr, h->solve_order);
    if (rc) return rc;
    switch (limbs) {
    case 2: mfl::ldlt_pivots_kernel<2><<<g, 128, 0, s>>>(n, nrhs, b, pivots, blocks, 1); break;
    case 3: mfl::ldlt_pivots_kernel<3><<<g, 128, 0, s>>>(n, nrhs, b, pivots, blocks, 1); break;
    default: mfl::ldlt_pivots_kernel<4><<<g, 128, 0, s>>>(n, nrhs, b, pivots, blocks, 1); break;
    }
    return mfl::record_cuda_error(cudaGetLastError(), "sytrs");
}

extern "C" int mflab_ldlt_diagnostics(mflab_handle *h, void *stream, int limbs, int64_t n,
                                      const double *F, int64_t ldf, int64_t lsf,
                                      const double *dsub, int64_t lsd, const uint8_t *blocks,
                                      const double *omax, double *out) {
    MFLAB_RANGE("mflab_ldlt_diagnostics");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (n < 0 || !out) return MFLAB_ERR_ARG;
    Mat f{(double *)F, ldf, lsf};
    cudaStream_t s = (cudaStream_t)stream;
    switch (limbs) {
    case 2: mfl::ldlt_diag_kernel<2><<<1, 1, 0, s>>>(n, f, dsub, lsd, blocks, omax, out); break;
    case 3: mfl::ldlt_diag_kernel<3><<<1, 1, 0, s>>>(n, f, dsub, lsd, blocks, omax, out); break;
    default: mfl::ldlt_diag_kernel<4><<<1, 1, 0, s>>>(n, f, dsub, lsd, blocks, omax, out); break;
    }
    return mfl::record_cuda_error(cudaGetLastError(), "ldlt diagnostics");
}
