// Batched SPD factor + solve of many independent uneven blocks, and its
// adjoint: a persistent launch factors each block and runs its forward
// substitution (one CTA per block), a second launch runs the backward
// substitutions (one group of lanes per block, several blocks per warp).
//
// No reference counterpart (MultiFloatLinearAlgebra.jl factors one matrix per
// call); every block follows the reference's own single-matrix order, so each
// block's factor and solution are bitwise those of cholesky!(S_i; block) and
// ldiv!(x_i, F_i) (src/factorizations/cholesky.jl:10-107, src/solve.jl:54-83,
// src/kernels/trsm.jl:18-112).
//
// Packed layout: block i is an n_i x n_i column-major matrix at S[off_i]
// (ld = n_i) and its right-hand side a vector at X[boff_i]; limb planes are
// ls_s / ls_x apart.  A CTA takes the next block index from a device counter
// (atomicAdd: blocks are handed out in the caller's order, normally
// descending size) until all blocks are done; there is no inter-CTA waiting.
// Per block, all data stays in global memory (L2-resident at these sizes).
#include <atomic>

#include "mf_device.cuh"
#include "mflab_internal.h"

namespace mfl {

constexpr int BATCH_NT = 256;   // default threads per CTA
constexpr int BATCH_MAXN = 512;  // largest block size
// The per-CTA shared row buffer (forward values, then backward products)
// holds the batch's largest block (dynamic shared memory, 32 bytes per row),
// so batches of small blocks leave room for many CTAs per SM: each block's
// factor and solve are chains of dependent steps, and throughput comes from
// blocks in flight.

template <int N>
struct BlockView {
    Mat A;
    int64_t n;
    __device__ mf<N> at(int64_t r, int64_t c) const { return load_mf<N>(A.p, A.ld, A.ls, r, c); }
    __device__ void put(int64_t r, int64_t c, const mf<N> &v) const {
        store_mf<N>(A.p, A.ld, A.ls, r, c, v);
    }
};

// blocked Cholesky of one block by the whole CTA of NT threads; returns info
// (0 / column)
template <int N, int NT>
__device__ int cta_potrf(const BlockView<N> &F, int64_t block, double (*bc)[4], int *flag) {
    const int t = threadIdx.x;
    const int64_t n = F.n;
    const mf<N> mone = from_double<N>(-1.0), one = from_double<N>(1.0);
    for (int64_t first = 0; first < n; first += block) {
        const int64_t last = first + block - 1 < n - 1 ? first + block - 1 : n - 1;
        // panel (cholesky.jl:10-34)
        for (int64_t col = first; col <= last; ++col) {
            if (t == 0) {
                mf<N> d = F.at(col, col);
                for (int64_t k = first; k < col; ++k) {
                    const mf<N> v = F.at(col, k);
                    d = submul(d, v, v);
                }
                if (!gt(d, from_double<N>(0.0))) {
                    *flag = (int)(col + 1);
                } else {
                    const mf<N> p = sqrt_mf(d);
                    F.put(col, col, p);
#pragma unroll
                    for (int l = 0; l < N; ++l) bc[0][l] = p.v[l];
                }
            }
            __syncthreads();
            if (*flag) return *flag;
            mf<N> p;
#pragma unroll
            for (int l = 0; l < N; ++l) p.v[l] = bc[0][l];
            for (int64_t row = col + 1 + t; row <= last; row += NT) {
                mf<N> v = F.at(row, col);
                for (int64_t k = first; k < col; ++k) v = submul(v, F.at(row, k), F.at(col, k));
                F.put(row, col, div(v, p));
            }
            __syncthreads();
        }
        if (last < n - 1) {
            // A21 <- A21 / L11^T: trsm(side=right, lower, T), one row per thread
            for (int64_t row = last + 1 + t; row < n; row += NT) {
                for (int64_t col = first; col <= last; ++col) {
                    mf<N> v = F.at(row, col);
                    for (int64_t k = first; k < col; ++k) v = submul(v, F.at(row, k), F.at(col, k));
                    F.put(row, col, div(v, F.at(col, col)));
                }
            }
            __syncthreads();
            // lower trailing update: -1 * (A21 A21^T) + 1 * A22 (syrk.jl:1-50)
            const int64_t m = n - 1 - last;
            const int64_t tot = m * (m + 1) / 2;
            // packed lower-triangle index e -> (r, c): column c starts at
            // c*m - c(c-1)/2; e grows with the loop, so c only moves forward
            int64_t c = 0;
            for (int64_t e = t; e < tot; e += NT) {
                while ((c + 1) * m - (c + 1) * c / 2 <= e) ++c;
                const int64_t r = c + (e - (c * m - c * (c - 1) / 2));
                const int64_t row = last + 1 + r, col = last + 1 + c;
                mf<N> acc = from_double<N>(0.0);
                for (int64_t k = first; k <= last; ++k) acc = add(acc, mul(F.at(row, k), F.at(col, k)));
                F.put(row, col, add(mul(mone, acc), mul(one, F.at(row, col))));
            }
            __syncthreads();
        }
    }
    return 0;
}

// x <- L^{-1} x, the forward half of solve.jl:54-83, one vector, in place, by
// a CTA of NT threads (thread t owns rows t, t + NT, ... of the wavefront; the
// running values sit in the shared row buffer)
template <int N, int NT>
__device__ void cta_forward(const BlockView<N> &F, double *x, int64_t ls_x, double (*bc)[4],
                            double (*prod)[4]) {
    const int t = threadIdx.x;
    const int64_t n = F.n;
    auto xget = [&](int64_t i) {
        mf<N> v;
#pragma unroll
        for (int l = 0; l < N; ++l) v.v[l] = x[l * ls_x + i];
        return v;
    };
    auto xput = [&](int64_t i, const mf<N> &v) {
#pragma unroll
        for (int l = 0; l < N; ++l) x[l * ls_x + i] = v.v[l];
    };
    auto vget = [&](int64_t i) {
        mf<N> v;
#pragma unroll
        for (int l = 0; l < N; ++l) v.v[l] = prod[i][l];
        return v;
    };
    auto vput = [&](int64_t i, const mf<N> &v) {
#pragma unroll
        for (int l = 0; l < N; ++l) prod[i][l] = v.v[l];
    };
    // forward substitution, wavefront: row r receives its terms k = 0..r-1 in
    // ascending order as the unknowns are finalised
    for (int64_t r = t; r < n; r += NT) vput(r, xget(r));
    // The critical path of a step runs through the owner of row k + 1 (its
    // update by x_k, then its division): that thread reads L[k+1, k] and
    // L[k+1, k+1] before the step's barrier, so neither load waits on it.
    mf<N> dk = F.at(0, 0), ak = dk;
    for (int64_t k = 0; k < n; ++k) {
        const bool next = k + 1 < n && ((k + 1) % NT) == t;
        mf<N> an = ak, dn = dk;
        if (next) {
            an = F.at(k + 1, k);
            dn = F.at(k + 1, k + 1);
        }
        if ((k % NT) == t) {
            const mf<N> vk = div(vget(k), dk);
            xput(k, vk);
#pragma unroll
            for (int l = 0; l < N; ++l) bc[k & 1][l] = vk.v[l];
        }
        __syncthreads();
        mf<N> xk;
#pragma unroll
        for (int l = 0; l < N; ++l) xk.v[l] = bc[k & 1][l];
        for (int64_t r = k + 1 + ((t - (k + 1)) % NT + NT) % NT; r < n; r += NT)
            vput(r, submul(vget(r), r == k + 1 ? an : F.at(r, k), xk));
        if (next) dk = dn;
    }
    __syncthreads();
}

template <int N, int NT>
__global__ void __launch_bounds__(NT)
    spd_batched_kernel(int64_t nblocks, const int64_t *sizes, const int64_t *offsets,
                       const int64_t *boffsets, const int64_t *order, double *S, int64_t ls_s,
                       double *X, int64_t ls_x, int64_t block, int *info, int *counter,
                       int solve, int64_t maxn) {
    __shared__ double bc[2][4];
    extern __shared__ double prod_raw[];  // [max block size][4]
    double(*prod)[4] = reinterpret_cast<double(*)[4]>(prod_raw);
    __shared__ int64_t job;
    __shared__ int flag;
    const int t = threadIdx.x;
    for (;;) {
        if (t == 0) {
            job = atomicAdd(counter, 1);
            flag = 0;
        }
        __syncthreads();
        const int64_t idx = job;
        if (idx >= nblocks) return;
        const int64_t b = order[idx];
        const int64_t n = sizes[b];
        if (n > maxn) {  // the row buffer holds maxn rows: refuse the block
            if (t == 0) info[b] = -1;
            __syncthreads();
            continue;
        }
        BlockView<N> F{Mat{S + offsets[b], n > 0 ? n : 1, ls_s}, n};
        const int st = cta_potrf<N, NT>(F, block, bc, &flag);
        if (t == 0) info[b] = st;
        if (st == 0 && solve) cta_forward<N, NT>(F, X + boffsets[b], ls_x, bc, prod);
        __syncthreads();
    }
}

// Backward substitution x <- L^{-T} y of every factored block, after the
// factor kernel's forward pass.  The reference's chain for row r is
// v = y[r]; v -= L[k, r] * x[k] for k = r+1..n-1 ascending; v /= L[r, r]
// (solve.jl:54-83 through trsm.jl's upper-transposed loop): one dependent
// subtraction per term, n(n-1)/2 per block, that no reordering may shorten.
// A group of BW_G lanes serves one block: the group forms the products of a
// row in parallel (coalesced reads of column r of L) into its shared slice,
// then its first lane runs the chain.  A warp carries 32 / BW_G blocks, so
// every instruction of the chains advances that many blocks at once, where a
// whole CTA per block would leave all but one thread waiting on the chain.
constexpr int BW_G = 4;                 // lanes per block
constexpr int BW_PER_WARP = 32 / BW_G;  // blocks per warp (one warp per CTA)

template <int N>
__global__ void __launch_bounds__(32)
    spd_batched_backward_kernel(int64_t nblocks, const int64_t *sizes, const int64_t *offsets,
                                const int64_t *boffsets, const int64_t *order, const double *L,
                                int64_t ls_s, double *X, int64_t ls_x, const int *info,
                                int64_t maxn) {
    extern __shared__ double bw_prod[];  // BW_PER_WARP slices of maxn * N (+1 pad)
    const int lane = threadIdx.x;
    const int g = lane / BW_G, m = lane % BW_G;
    const int64_t idx = (int64_t)blockIdx.x * BW_PER_WARP + g;
    int64_t b = 0, n = 0;
    if (idx < nblocks) {
        b = order[idx];
        n = sizes[b];
        if (n > maxn || info[b] != 0) n = 0;  // nothing to solve for this group
    }
    // The groups step together: step i solves row n - 1 - i of every block
    // (a chain of i terms in each), so the warp's loops have the same trip
    // counts in all groups and its lanes stay converged; a group whose block
    // is smaller (blocks come in descending size, so rarely) sits out its
    // last steps.
    const int nmax = __reduce_max_sync(0xffffffffu, (unsigned)n);
    double *P = bw_prod + (size_t)g * (size_t)(maxn * N + 1);
    const double *Lb = L + (n ? offsets[b] : 0);
    double *x = X + (n ? boffsets[b] : 0);
    for (int i = 0; i < nmax; ++i) {
        const bool act = i < n;
        const int64_t r = n - 1 - i;
        const double *col = Lb + r * n;
        if (act) {
            for (int j = m; j < i; j += BW_G) {
                const int64_t k = r + 1 + j;
                mf<N> a, xv;
#pragma unroll
                for (int l = 0; l < N; ++l) {
                    a.v[l] = __ldg(col + l * ls_s + k);
                    xv.v[l] = x[l * ls_x + k];
                }
                const mf<N> p = mul(a, xv);
#pragma unroll
                for (int l = 0; l < N; ++l) P[k * N + l] = p.v[l];
            }
        }
        __syncwarp();
        if (act && m == 0) {
            mf<N> v, d;
#pragma unroll
            for (int l = 0; l < N; ++l) {
                v.v[l] = x[l * ls_x + r];
                d.v[l] = __ldg(col + l * ls_s + r);
            }
            // the next term is read from shared memory while the current
            // subtraction runs, keeping the load off the chain
            mf<N> p = v;
            if (r + 1 < n) {
#pragma unroll
                for (int l = 0; l < N; ++l) p.v[l] = P[(r + 1) * N + l];
            }
            for (int64_t k = r + 1; k < n; ++k) {
                mf<N> pn = p;
                if (k + 1 < n) {
#pragma unroll
                    for (int l = 0; l < N; ++l) pn.v[l] = P[(k + 1) * N + l];
                }
                v = sub(v, p);
                p = pn;
            }
            v = div(v, d);
#pragma unroll
            for (int l = 0; l < N; ++l) x[l * ls_x + r] = v.v[l];
        }
        __syncwarp();
    }
}

// Adjoint of x = S^{-1} b for loss gradients: given the factor L (in place),
// x and xbar, writes bbar = S^{-1} xbar (over xbar) and
// Sbar = -(bbar x^T + x bbar^T) / 2 into the packed Sbar buffer.  Phase 0
// runs the forward substitution of xbar, the backward kernel follows, and
// phase 1 forms Sbar.
template <int N, int NT>
__global__ void __launch_bounds__(NT)
    spd_batched_adjoint_kernel(int64_t nblocks, const int64_t *sizes, const int64_t *offsets,
                               const int64_t *boffsets, const int64_t *order, const double *L,
                               int64_t ls_s, const double *X, double *XB, int64_t ls_x,
                               double *SB, const int *info, int *counter, int64_t maxn,
                               int phase) {
    __shared__ double bc[2][4];
    extern __shared__ double prod_raw[];  // [max block size][4]
    double(*prod)[4] = reinterpret_cast<double(*)[4]>(prod_raw);
    __shared__ int64_t job;
    const int t = threadIdx.x;
    for (;;) {
        if (t == 0) job = atomicAdd(counter, 1);
        __syncthreads();
        const int64_t idx = job;
        if (idx >= nblocks) return;
        const int64_t b = order[idx];
        const int64_t n = sizes[b];
        if (info[b] == 0 && n <= maxn && phase == 0) {
            BlockView<N> F{Mat{(double *)L + offsets[b], n > 0 ? n : 1, ls_s}, n};
            cta_forward<N, NT>(F, XB + boffsets[b], ls_x, bc, prod);
        } else if (info[b] == 0 && n <= maxn) {
            const double *x = X + boffsets[b];
            const double *xb = XB + boffsets[b];
            double *sb = SB + offsets[b];
            for (int64_t e = t; e < n * n; e += NT) {
                const int64_t r = e % n, c = e / n;
                mf<N> xr, xc, br, bcv;
#pragma unroll
                for (int l = 0; l < N; ++l) {
                    xr.v[l] = x[l * ls_x + r];
                    xc.v[l] = x[l * ls_x + c];
                    br.v[l] = xb[l * ls_x + r];
                    bcv.v[l] = xb[l * ls_x + c];
                }
                mf<N> g = add(mul(br, xc), mul(xr, bcv));
#pragma unroll
                for (int l = 0; l < N; ++l) sb[l * ls_s + c * n + r] = -0.5 * g.v[l];
            }
        }
        __syncthreads();
    }
}

}  // namespace mfl

static int batched_check(int limbs, int64_t nblocks, int64_t maxn) {
    if (!mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (nblocks < 0 || maxn < 0) return MFLAB_ERR_ARG;
    if (maxn > mfl::BATCH_MAXN) return MFLAB_ERR_UNSUPPORTED;
    return MFLAB_OK;
}

template <int NT>
static void launch_batched(int limbs, int grid, int64_t maxn, cudaStream_t s, int64_t nblocks,
                           const int64_t *sizes, const int64_t *offsets, const int64_t *boffsets,
                           const int64_t *order, double *S, int64_t ls_s, double *X, int64_t ls_x,
                           int64_t block, int *info, int *counter, int solve) {
    const size_t smem = (size_t)(maxn > 0 ? maxn : 1) * 4 * sizeof(double);
    switch (limbs) {
    case 2: mfl::spd_batched_kernel<2, NT><<<grid, NT, smem, s>>>(nblocks, sizes, offsets, boffsets, order, S, ls_s, X, ls_x, block, info, counter, solve, maxn); break;
    case 3: mfl::spd_batched_kernel<3, NT><<<grid, NT, smem, s>>>(nblocks, sizes, offsets, boffsets, order, S, ls_s, X, ls_x, block, info, counter, solve, maxn); break;
    default: mfl::spd_batched_kernel<4, NT><<<grid, NT, smem, s>>>(nblocks, sizes, offsets, boffsets, order, S, ls_s, X, ls_x, block, info, counter, solve, maxn); break;
    }
}

template <int N>
static int launch_backward_n(cudaStream_t s, int64_t nblocks, int64_t maxn, const int64_t *sizes,
                             const int64_t *offsets, const int64_t *boffsets,
                             const int64_t *order, const double *L, int64_t ls_s, double *X,
                             int64_t ls_x, const int *info) {
    const size_t smem = (size_t)mfl::BW_PER_WARP * (size_t)((maxn > 0 ? maxn : 1) * N + 1) *
                        sizeof(double);
    if (smem > 48 * 1024) {  // large blocks only: the opt-in above the default limit
        static std::atomic<unsigned long long> done{0};
        constexpr int max_smem =
            mfl::BW_PER_WARP * (mfl::BATCH_MAXN * N + 1) * (int)sizeof(double);
        int rc = mfl::set_smem_once((const void *)mfl::spd_batched_backward_kernel<N>, max_smem,
                                    done, "spd batched backward smem");
        if (rc) return rc;
    }
    const int64_t grid = (nblocks + mfl::BW_PER_WARP - 1) / mfl::BW_PER_WARP;
    mfl::spd_batched_backward_kernel<N><<<(unsigned)grid, 32, smem, s>>>(
        nblocks, sizes, offsets, boffsets, order, L, ls_s, X, ls_x, info, maxn);
    return 0;
}

static int launch_backward(int limbs, cudaStream_t s, int64_t nblocks, int64_t maxn,
                           const int64_t *sizes, const int64_t *offsets, const int64_t *boffsets,
                           const int64_t *order, const double *L, int64_t ls_s, double *X,
                           int64_t ls_x, const int *info) {
    switch (limbs) {
    case 2: return launch_backward_n<2>(s, nblocks, maxn, sizes, offsets, boffsets, order, L, ls_s, X, ls_x, info);
    case 3: return launch_backward_n<3>(s, nblocks, maxn, sizes, offsets, boffsets, order, L, ls_s, X, ls_x, info);
    default: return launch_backward_n<4>(s, nblocks, maxn, sizes, offsets, boffsets, order, L, ls_s, X, ls_x, info);
    }
}

template <int NT>
static void launch_adjoint(int limbs, int grid, int64_t maxn, cudaStream_t s, int64_t nblocks,
                           const int64_t *sizes, const int64_t *offsets, const int64_t *boffsets,
                           const int64_t *order, const double *L, int64_t ls_s, const double *X,
                           double *XB, int64_t ls_x, double *SB, const int *info, int *counter,
                           int phase) {
    const size_t smem = (size_t)(maxn > 0 ? maxn : 1) * 4 * sizeof(double);
    switch (limbs) {
    case 2: mfl::spd_batched_adjoint_kernel<2, NT><<<grid, NT, smem, s>>>(nblocks, sizes, offsets, boffsets, order, L, ls_s, X, XB, ls_x, SB, info, counter, maxn, phase); break;
    case 3: mfl::spd_batched_adjoint_kernel<3, NT><<<grid, NT, smem, s>>>(nblocks, sizes, offsets, boffsets, order, L, ls_s, X, XB, ls_x, SB, info, counter, maxn, phase); break;
    default: mfl::spd_batched_adjoint_kernel<4, NT><<<grid, NT, smem, s>>>(nblocks, sizes, offsets, boffsets, order, L, ls_s, X, XB, ls_x, SB, info, counter, maxn, phase); break;
    }
}

extern "C" int mflab_spd_batched_ex(mflab_handle *h, void *stream, int limbs, int64_t nblocks,
                                    int64_t max_size, const int64_t *sizes,
                                    const int64_t *offsets, const int64_t *boffsets,
                                    const int64_t *order, double *S, int64_t ls_s, double *X,
                                    int64_t ls_x, int64_t block, int solve, int *info,
                                    int *counter, int grid, int threads) {
    MFLAB_RANGE("mflab_spd_batched_ex");
    if (!h) return MFLAB_ERR_UNSUPPORTED;
    int rc = batched_check(limbs, nblocks, max_size);
    if (rc) return rc;
    if (threads != 64 && threads != 128 && threads != 256 && threads != 512) return MFLAB_ERR_ARG;
    if (block < 1) block = 1;
    if (nblocks == 0) return MFLAB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), s);
    if (e != cudaSuccess) return mfl::record_cuda_error(e, "spd batched counter");
    if (grid <= 0) grid = 148 * 4;
    if (threads == 64)
        launch_batched<64>(limbs, grid, max_size, s, nblocks, sizes, offsets, boffsets, order, S, ls_s, X, ls_x, block, info, counter, solve);
    else if (threads == 128)
        launch_batched<128>(limbs, grid, max_size, s, nblocks, sizes, offsets, boffsets, order, S, ls_s, X, ls_x, block, info, counter, solve);
    else if (threads == 256)
        launch_batched<256>(limbs, grid, max_size, s, nblocks, sizes, offsets, boffsets, order, S, ls_s, X, ls_x, block, info, counter, solve);
    else
        launch_batched<512>(limbs, grid, max_size, s, nblocks, sizes, offsets, boffsets, order, S, ls_s, X, ls_x, block, info, counter, solve);
    e = cudaGetLastError();
    if (e != cudaSuccess) return mfl::record_cuda_error(e, "spd batched");
    if (solve) {
        // the factor kernel ran the forward half; the backward chains follow
        int rc2 = launch_backward(limbs, s, nblocks, max_size, sizes, offsets, boffsets, order,
                                  S, ls_s, X, ls_x, info);
        if (rc2) return rc2;
        return mfl::record_cuda_error(cudaGetLastError(), "spd batched backward");
    }
    return MFLAB_OK;
}

extern "C" int mflab_spd_batched(mflab_handle *h, void *stream, int limbs, int64_t nblocks,
                                 int64_t max_size, const int64_t *sizes, const int64_t *offsets,
                                 const int64_t *boffsets, const int64_t *order, double *S,
                                 int64_t ls_s, double *X, int64_t ls_x, int64_t block, int solve,
                                 int *info, int *counter, int grid) {
    MFLAB_RANGE("mflab_spd_batched");
    return mflab_spd_batched_ex(h, stream, limbs, nblocks, max_size, sizes, offsets, boffsets,
                                order, S, ls_s, X, ls_x, block, solve, info, counter, grid,
                                mfl::BATCH_NT);
}

extern "C" int mflab_spd_batched_adjoint_ex(mflab_handle *h, void *stream, int limbs,
                                            int64_t nblocks, int64_t max_size,
                                            const int64_t *sizes, const int64_t *offsets,
                                            const int64_t *boffsets, const int64_t *order,
                                            const double *L, int64_t ls_s, const double *X,
                                            double *XB, int64_t ls_x, double *SB, const int *info,
                                            int *counter, int grid, int threads) {
    MFLAB_RANGE("mflab_spd_batched_adjoint_ex");
    if (!h) return MFLAB_ERR_UNSUPPORTED;
    int rc = batched_check(limbs, nblocks, max_size);
    if (rc) return rc;
    if (threads != 64 && threads != 128 && threads != 256 && threads != 512) return MFLAB_ERR_ARG;
    if (nblocks == 0) return MFLAB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), s);
    if (e != cudaSuccess) return mfl::record_cuda_error(e, "spd adjoint counter");
    if (grid <= 0) grid = 148 * 4;
    for (int phase = 0; phase < 2; ++phase) {
        if (phase == 1) {
            // bbar's backward chains, then the counter again for phase 1
            rc = launch_backward(limbs, s, nblocks, max_size, sizes, offsets, boffsets, order, L,
                                 ls_s, XB, ls_x, info);
            if (rc) return rc;
            e = cudaMemsetAsync(counter, 0, sizeof(int), s);
            if (e != cudaSuccess) return mfl::record_cuda_error(e, "spd adjoint counter");
        }
        if (threads == 64)
            launch_adjoint<64>(limbs, grid, max_size, s, nblocks, sizes, offsets, boffsets, order, L, ls_s, X, XB, ls_x, SB, info, counter, phase);
        else if (threads == 128)
            launch_adjoint<128>(limbs, grid, max_size, s, nblocks, sizes, offsets, boffsets, order, L, ls_s, X, XB, ls_x, SB, info, counter, phase);
        else if (threads == 256)
            launch_adjoint<256>(limbs, grid, max_size, s, nblocks, sizes, offsets, boffsets, order, L, ls_s, X, XB, ls_x, SB, info, counter, phase);
        else
            launch_adjoint<512>(limbs, grid, max_size, s, nblocks, sizes, offsets, boffsets, order, L, ls_s, X, XB, ls_x, SB, info, counter, phase);
        e = cudaGetLastError();
        if (e != cudaSuccess) return mfl::record_cuda_error(e, "spd adjoint");
    }
    return MFLAB_OK;
}

extern "C" int mflab_spd_batched_adjoint(mflab_handle *h, void *stream, int limbs,
                                         int64_t nblocks, int64_t max_size, const int64_t *sizes,
                                         const int64_t *offsets, const int64_t *boffsets,
                                         const int64_t *order, const double *L, int64_t ls_s,
                                         const double *X, double *XB, int64_t ls_x, double *SB,
                                         const int *info, int *counter, int grid) {
    MFLAB_RANGE("mflab_spd_batched_adjoint");
    return mflab_spd_batched_adjoint_ex(h, stream, limbs, nblocks, max_size, sizes, offsets,
                                        boffsets, order, L, ls_s, X, XB, ls_x, SB, info, counter,
                                        grid, mfl::BATCH_NT);
}
