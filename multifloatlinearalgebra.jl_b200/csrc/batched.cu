// Batched SPD factor + solve of many independent uneven blocks in one
// persistent launch, and its adjoint.
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
#include "mf_device.cuh"
#include "mflab_internal.h"

namespace mfl {

constexpr int BATCH_NT = 256;   // default threads per CTA
constexpr int BATCH_MAXN = 512;  // largest block size the shared buffers hold

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
            for (int64_t e = t; e < tot; e += NT) {
                int64_t c = (int64_t)((2.0 * m + 1.0 - sqrt((2.0 * m + 1.0) * (2.0 * m + 1.0) - 8.0 * e)) / 2.0);
                while (c > 0 && c * m - c * (c - 1) / 2 > e) --c;
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

// x <- L^{-T} L^{-1} x (solve.jl:54-83), one vector, in place, by a CTA of NT
// threads (thread t holds rows t, t + NT, ... of the forward wavefront)
template <int N, int NT>
__device__ void cta_potrs(const BlockView<N> &F, double *x, int64_t ls_x, double (*bc)[4],
                          double (*prod)[4]) {
    constexpr int MAXR = BATCH_MAXN / NT;
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
    // forward substitution, wavefront: row r receives its terms k = 0..r-1 in
    // ascending order as the unknowns are finalised
    mf<N> v[MAXR];
#pragma unroll
    for (int q = 0; q < MAXR; ++q)
        v[q] = t + q * NT < n ? xget(t + q * NT) : from_double<N>(0.0);
    for (int64_t k = 0; k < n; ++k) {
        if ((k % NT) == t) {
            const int qk = (int)(k / NT);
            mf<N> vk;
#pragma unroll
            for (int q = 0; q < MAXR; ++q)
                if (q == qk) vk = v[q];
            vk = div(vk, F.at(k, k));
            xput(k, vk);
#pragma unroll
            for (int l = 0; l < N; ++l) bc[k & 1][l] = vk.v[l];
        }
        __syncthreads();
        mf<N> xk;
#pragma unroll
        for (int l = 0; l < N; ++l) xk.v[l] = bc[k & 1][l];
#pragma unroll
        for (int q = 0; q < MAXR; ++q) {
            const int64_t r = t + q * NT;
            if (r > k && r < n) v[q] = submul(v[q], F.at(r, k), xk);
        }
    }
    __syncthreads();
    // backward substitution with L^T: the reference's chain for row r is
    // v = x[r]; v -= L[k, r] * x[k] for k = r+1..n-1 ascending; v /= L[r, r].
    // The products are formed in parallel, the subtraction chain stays serial.
    for (int64_t r = n - 1; r >= 0; --r) {
        for (int64_t k = r + 1 + t; k < n; k += NT) {
            const mf<N> p = mul(F.at(k, r), xget(k));
#pragma unroll
            for (int l = 0; l < N; ++l) prod[k][l] = p.v[l];
        }
        __syncthreads();
        if (t == 0) {
            mf<N> vr = xget(r);
            for (int64_t k = r + 1; k < n; ++k) {
                mf<N> p;
#pragma unroll
                for (int l = 0; l < N; ++l) p.v[l] = prod[k][l];
                vr = sub(vr, p);
            }
            xput(r, div(vr, F.at(r, r)));
        }
        __syncthreads();
    }
}

template <int N, int NT>
__global__ void __launch_bounds__(NT)
    spd_batched_kernel(int64_t nblocks, const int64_t *sizes, const int64_t *offsets,
                       const int64_t *boffsets, const int64_t *order, double *S, int64_t ls_s,
                       double *X, int64_t ls_x, int64_t block, int *info, int *counter,
                       int solve) {
    __shared__ double bc[2][4];
    __shared__ double prod[BATCH_MAXN][4];
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
        BlockView<N> F{Mat{S + offsets[b], n > 0 ? n : 1, ls_s}, n};
        const int st = cta_potrf<N, NT>(F, block, bc, &flag);
        if (t == 0) info[b] = st;
        if (st == 0 && solve) cta_potrs<N, NT>(F, X + boffsets[b], ls_x, bc, prod);
        __syncthreads();
    }
}

// Adjoint of x = S^{-1} b for loss gradients: given the factor L (in place),
// x and xbar, writes bbar = S^{-1} xbar (over xbar) and
// Sbar = -(bbar x^T + x bbar^T) / 2 into the packed Sbar buffer.
template <int N, int NT>
__global__ void __launch_bounds__(NT)
    spd_batched_adjoint_kernel(int64_t nblocks, const int64_t *sizes, const int64_t *offsets,
                               const int64_t *boffsets, const int64_t *order, const double *L,
                               int64_t ls_s, const double *X, double *XB, int64_t ls_x,
                               double *SB, const int *info, int *counter) {
    __shared__ double bc[2][4];
    __shared__ double prod[BATCH_MAXN][4];
    __shared__ int64_t job;
    const int t = threadIdx.x;
    for (;;) {
        if (t == 0) job = atomicAdd(counter, 1);
        __syncthreads();
        const int64_t idx = job;
        if (idx >= nblocks) return;
        const int64_t b = order[idx];
        const int64_t n = sizes[b];
        if (info[b] == 0) {
            BlockView<N> F{Mat{(double *)L + offsets[b], n > 0 ? n : 1, ls_s}, n};
            cta_potrs<N, NT>(F, XB + boffsets[b], ls_x, bc, prod);
            __syncthreads();
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
static void launch_batched(int limbs, int grid, cudaStream_t s, int64_t nblocks,
                           const int64_t *sizes, const int64_t *offsets, const int64_t *boffsets,
                           const int64_t *order, double *S, int64_t ls_s, double *X, int64_t ls_x,
                           int64_t block, int *info, int *counter, int solve) {
    switch (limbs) {
    case 2: mfl::spd_batched_kernel<2, NT><<<grid, NT, 0, s>>>(nblocks, sizes, offsets, boffsets, order, S, ls_s, X, ls_x, block, info, counter, solve); break;
    case 3: mfl::spd_batched_kernel<3, NT><<<grid, NT, 0, s>>>(nblocks, sizes, offsets, boffsets, order, S, ls_s, X, ls_x, block, info, counter, solve); break;
    default: mfl::spd_batched_kernel<4, NT><<<grid, NT, 0, s>>>(nblocks, sizes, offsets, boffsets, order, S, ls_s, X, ls_x, block, info, counter, solve); break;
    }
}

template <int NT>
static void launch_adjoint(int limbs, int grid, cudaStream_t s, int64_t nblocks,
                           const int64_t *sizes, const int64_t *offsets, const int64_t *boffsets,
                           const int64_t *order, const double *L, int64_t ls_s, const double *X,
                           double *XB, int64_t ls_x, double *SB, const int *info, int *counter) {
    switch (limbs) {
    case 2: mfl::spd_batched_adjoint_kernel<2, NT><<<grid, NT, 0, s>>>(nblocks, sizes, offsets, boffsets, order, L, ls_s, X, XB, ls_x, SB, info, counter); break;
    case 3: mfl::spd_batched_adjoint_kernel<3, NT><<<grid, NT, 0, s>>>(nblocks, sizes, offsets, boffsets, order, L, ls_s, X, XB, ls_x, SB, info, counter); break;
    default: mfl::spd_batched_adjoint_kernel<4, NT><<<grid, NT, 0, s>>>(nblocks, sizes, offsets, boffsets, order, L, ls_s, X, XB, ls_x, SB, info, counter); break;
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
    if (threads != 128 && threads != 256 && threads != 512) return MFLAB_ERR_ARG;
    if (block < 1) block = 1;
    if (nblocks == 0) return MFLAB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), s);
    if (e != cudaSuccess) return mfl::record_cuda_error(e, "spd batched counter");
    if (grid <= 0) grid = 148 * 4;
    if (threads == 128)
        launch_batched<128>(limbs, grid, s, nblocks, sizes, offsets, boffsets, order, S, ls_s, X, ls_x, block, info, counter, solve);
    else if (threads == 256)
        launch_batched<256>(limbs, grid, s, nblocks, sizes, offsets, boffsets, order, S, ls_s, X, ls_x, block, info, counter, solve);
    else
        launch_batched<512>(limbs, grid, s, nblocks, sizes, offsets, boffsets, order, S, ls_s, X, ls_x, block, info, counter, solve);
    return mfl::record_cuda_error(cudaGetLastError(), "spd batched");
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
    if (threads != 128 && threads != 256 && threads != 512) return MFLAB_ERR_ARG;
    if (nblocks == 0) return MFLAB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), s);
    if (e != cudaSuccess) return mfl::record_cuda_error(e, "spd adjoint counter");
    if (grid <= 0) grid = 148 * 4;
    if (threads == 128)
        launch_adjoint<128>(limbs, grid, s, nblocks, sizes, offsets, boffsets, order, L, ls_s, X, XB, ls_x, SB, info, counter);
    else if (threads == 256)
        launch_adjoint<256>(limbs, grid, s, nblocks, sizes, offsets, boffsets, order, L, ls_s, X, XB, ls_x, SB, info, counter);
    else
        launch_adjoint<512>(limbs, grid, s, nblocks, sizes, offsets, boffsets, order, L, ls_s, X, XB, ls_x, SB, info, counter);
    return mfl::record_cuda_error(cudaGetLastError(), "spd adjoint");
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
