// Multi-double triangular solves, src/kernels/trsm.jl:1-302 and trsv.jl:19-73
// of MultiFloatLinearAlgebra.jl.
//
// Order contract: the reference computes, for every unknown,
//     v = B[i]; for k in the substitution order: v -= coef(i,k) * X[k]; v /= A[i,i]
// (left side; right side uses B[i,k] * coef(k,j)).  Each kernel below keeps that
// exact per-element chain:
//   * trsm_left_cta: forward substitution, one CTA per right-hand-side column.
//     The column's running values live in registers (rows distributed
//     cyclically over the threads).  Step k finalises X[k] (owner divides by
//     the diagonal), broadcasts it through shared memory, and every later row
//     applies its term k.  Each row thus receives its terms in the reference's
//     ascending order while the rows progress in parallel.
//   * trsm_left_thread: one thread per right-hand-side column, the plain
//     serial loop (used when the triangle is short, e.g. LU's U12 block).
//   * trsm_right_thread: one thread per row of B, the plain serial loop (the
//     Cholesky panel solve A21 <- A21 / L11^T).
#include "mf_device.cuh"
#include "mflab_internal.h"

namespace mfl {

template <int N>
__device__ __forceinline__ mf<N> tri_coef(const Mat &A, int64_t r, int64_t c, bool transposed) {
    return transposed ? load_mf<N>(A.p, A.ld, A.ls, c, r) : load_mf<N>(A.p, A.ld, A.ls, r, c);
}

template <int N>
__global__ void scale_kernel(int64_t m, int64_t n, Mat B, scal<N> alpha) {
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= m * n) return;
    int64_t r = idx % m, c = idx / m;
    mf<N> v = load_mf<N>(B.p, B.ld, B.ls, r, c);
    store_mf<N>(B.p, B.ld, B.ls, r, c, mul(v, alpha.get()));
}

// one CTA per column; NT threads; each thread owns up to MAXR rows
template <int N, int NT, int MAXR>
__global__ void __launch_bounds__(NT) trsm_left_cta(int64_t m, int64_t n, Mat A, Mat B,
                                                    bool eff_lower, bool transposed, bool unit,
                                                    const int *info) {
    if (info && *info) return;
    __shared__ double xs[2][N];
    const int64_t col = blockIdx.x;
    if (col >= n) return;
    const int t = threadIdx.x;
    mf<N> v[MAXR];
#pragma unroll
    for (int q = 0; q < MAXR; ++q) {
        int64_t r = t + (int64_t)q * NT;
        v[q] = r < m ? load_mf<N>(B.p, B.ld, B.ls, r, col) : from_double<N>(0.0);
    }
    for (int64_t s = 0; s < m; ++s) {
        const int64_t k = eff_lower ? s : m - 1 - s;  // row finalised at this step
        const int slot = (int)(s & 1);
        if ((k % NT) == t) {
            const int qk = (int)(k / NT);
            mf<N> x;
#pragma unroll
            for (int q = 0; q < MAXR; ++q)
                if (q == qk) x = v[q];
            if (!unit) x = div(x, load_mf<N>(A.p, A.ld, A.ls, k, k));
#pragma unroll
            for (int q = 0; q < MAXR; ++q)
                if (q == qk) v[q] = x;
            store_mf<N>(B.p, B.ld, B.ls, k, col, x);
#pragma unroll
            for (int l = 0; l < N; ++l) xs[slot][l] = x.v[l];
        }
        __syncthreads();
        mf<N> xk;
#pragma unroll
        for (int l = 0; l < N; ++l) xk.v[l] = xs[slot][l];
#pragma unroll
        for (int q = 0; q < MAXR; ++q) {
            const int64_t r = t + (int64_t)q * NT;
            const bool later = eff_lower ? (r > k) : (r < k);
            if (r < m && later) v[q] = submul(v[q], tri_coef<N>(A, r, k, transposed), xk);
        }
    }
}

// Backward substitution (effective upper, left side) in the reference order:
// row r's chain v = B[r]; v -= coef(r,k) * X[k] for k = r+1..m-1 ascending.
// One CTA per right-hand-side column: the products of row r are formed by all
// threads into shared memory, thread 0 runs the subtraction chain and the
// division.  The column is read from and written to global memory.
template <int N, int NT>
__global__ void __launch_bounds__(NT) trsm_left_backward_cta(int64_t m, int64_t n, Mat A, Mat B,
                                                             bool transposed, bool unit,
                                                             const int *info) {
    if (info && *info) return;
    extern __shared__ double prod[];  // [m][N]
    const int64_t col = blockIdx.x;
    if (col >= n) return;
    const int t = threadIdx.x;
    for (int64_t r = m - 1; r >= 0; --r) {
        for (int64_t k = r + 1 + t; k < m; k += NT) {
            const mf<N> p = mul(tri_coef<N>(A, r, k, transposed), load_mf<N>(B.p, B.ld, B.ls, k, col));
#pragma unroll
            for (int l = 0; l < N; ++l) prod[k * N + l] = p.v[l];
        }
        __syncthreads();
        if (t == 0) {
            // the chain of subtractions is the row's latency; the product of
            // the next term is read from shared memory while the current one
            // is subtracted
            mf<N> v = load_mf<N>(B.p, B.ld, B.ls, r, col);
            mf<N> pn;
#pragma unroll
            for (int l = 0; l < N; ++l) pn.v[l] = r + 1 < m ? prod[(r + 1) * N + l] : 0.0;
            for (int64_t k = r + 1; k < m; ++k) {
                const mf<N> p = pn;
                if (k + 1 < m) {
#pragma unroll
                    for (int l = 0; l < N; ++l) pn.v[l] = prod[(k + 1) * N + l];
                }
                v = sub(v, p);
            }
            if (!unit) v = div(v, load_mf<N>(A.p, A.ld, A.ls, r, r));
            store_mf<N>(B.p, B.ld, B.ls, r, col, v);
        }
        __syncthreads();
    }
}

template <int N>
__global__ void trsm_left_thread(int64_t m, int64_t n, Mat A, Mat B, bool eff_lower,
                                 bool transposed, bool unit, const int *info) {
    if (info && *info) return;
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    if (eff_lower) {
        for (int64_t row = 0; row < m; ++row) {
            mf<N> v = load_mf<N>(B.p, B.ld, B.ls, row, c);
            for (int64_t k = 0; k < row; ++k)
                v = submul(v, tri_coef<N>(A, row, k, transposed), load_mf<N>(B.p, B.ld, B.ls, k, c));
            if (!unit) v = div(v, load_mf<N>(A.p, A.ld, A.ls, row, row));
            store_mf<N>(B.p, B.ld, B.ls, row, c, v);
        }
    } else {
        for (int64_t row = m - 1; row >= 0; --row) {
            mf<N> v = load_mf<N>(B.p, B.ld, B.ls, row, c);
            for (int64_t k = row + 1; k < m; ++k)
                v = submul(v, tri_coef<N>(A, row, k, transposed), load_mf<N>(B.p, B.ld, B.ls, k, c));
            if (!unit) v = div(v, load_mf<N>(A.p, A.ld, A.ls, row, row));
            store_mf<N>(B.p, B.ld, B.ls, row, c, v);
        }
    }
}

template <int N>
__global__ void trsm_right_thread(int64_t m, int64_t n, Mat A, Mat B, bool eff_lower,
                                  bool transposed, bool unit, const int *info) {
    if (info && *info) return;
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= m) return;
    if (eff_lower) {
        for (int64_t col = n - 1; col >= 0; --col) {
            mf<N> v = load_mf<N>(B.p, B.ld, B.ls, r, col);
            for (int64_t k = col + 1; k < n; ++k)
                v = submul(v, load_mf<N>(B.p, B.ld, B.ls, r, k), tri_coef<N>(A, k, col, transposed));
            if (!unit) v = div(v, load_mf<N>(A.p, A.ld, A.ls, col, col));
            store_mf<N>(B.p, B.ld, B.ls, r, col, v);
        }
    } else {
        for (int64_t col = 0; col < n; ++col) {
            mf<N> v = load_mf<N>(B.p, B.ld, B.ls, r, col);
            for (int64_t k = 0; k < col; ++k)
                v = submul(v, load_mf<N>(B.p, B.ld, B.ls, r, k), tri_coef<N>(A, k, col, transposed));
            if (!unit) v = div(v, load_mf<N>(A.p, A.ld, A.ls, col, col));
            store_mf<N>(B.p, B.ld, B.ls, r, col, v);
        }
    }
}

// Binary64 diagonal-block solve of the blocked left solve below: one CTA
// per right-hand-side column, the jb x jb block (jb <= 64) in shared memory,
// row t of the column in thread t.
constexpr int TRSM64_NB = 64;

__global__ void __launch_bounds__(TRSM64_NB)
    trsm64_diag_kernel(int64_t jb, Mat A, Mat B, bool lower, bool unit) {
    __shared__ double a[TRSM64_NB][TRSM64_NB + 1];
    __shared__ double xk;
    const int t = threadIdx.x;
    const int64_t col = blockIdx.x;
    for (int c = 0; c < jb; ++c)
        if (t < jb) a[t][c] = A.p[(int64_t)c * A.ld + t];
    double v = t < jb ? B.p[col * B.ld + t] : 0.0;
    __syncthreads();
    for (int s = 0; s < jb; ++s) {
        const int k = lower ? s : (int)jb - 1 - s;
        if (t == k) {
            if (!unit) v = __ddiv_rn(v, a[k][k]);
            xk = v;
        }
        __syncthreads();
        if (t < jb && (lower ? t > k : t < k)) v = __dsub_rn(v, __dmul_rn(a[t][k], xk));
        __syncthreads();
    }
    if (t < jb) B.p[col * B.ld + t] = v;
}

// Blocked left solve op(A) X = B for binary64 (no reference order to keep):
// 64 x 64 diagonal blocks solved from shared memory, the rows below (forward)
// or above (backward) updated with the FP64 GEMM kernel.  A not transposed.
static int trsm64_blocked(int64_t m, int64_t n, Mat A, Mat B, bool lower, bool unit,
                          cudaStream_t s, const int *info) {
    const double mone[1] = {-1.0}, one[1] = {1.0};
    const int64_t nblk = (m + TRSM64_NB - 1) / TRSM64_NB;
    for (int64_t bi = 0; bi < nblk; ++bi) {
        const int64_t blk = lower ? bi : nblk - 1 - bi;
        const int64_t j0 = blk * TRSM64_NB;
        const int64_t jb = m - j0 < TRSM64_NB ? m - j0 : TRSM64_NB;
        trsm64_diag_kernel<<<(unsigned)n, TRSM64_NB, 0, s>>>(jb, A.at(j0, j0), B.at(j0, 0), lower,
                                                             unit);
        int rc = record_cuda_error(cudaGetLastError(), "trsm64 diagonal");
        if (rc) return rc;
        if (lower && j0 + jb < m) {
            rc = launch_mm(1, false, false, 0, false, m - j0 - jb, n, jb, A.at(j0 + jb, j0),
                           B.at(j0, 0), B.at(j0 + jb, 0), mone, one, s, info);
        } else if (!lower && j0 > 0) {
            rc = launch_mm(1, false, false, 0, false, j0, n, jb, A.at(0, j0), B.at(j0, 0),
                           B.at(0, 0), mone, one, s, info);
        }
        if (rc) return rc;
    }
    return MFLAB_OK;
}

template <int N>
static int run_trsm(int side, int uplo, int trans, int diag, int64_t m, int64_t n, Mat A, Mat B,
                    const double *alpha, cudaStream_t s, const int *info, int order) {
    if (m <= 0 || n <= 0) return MFLAB_OK;
    bool one = alpha[0] == 1.0;
    for (int l = 1; l < N; ++l) one = one && alpha[l] == 0.0;
    if (!one) {
        scal<N> al{};
        for (int l = 0; l < N; ++l) al.v[l] = alpha[l];
        int64_t tot = m * n;
        scale_kernel<N><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(m, n, B, al);
        int rc = record_cuda_error(cudaGetLastError(), "trsm scale");
        if (rc) return rc;
    }
    const bool transposed = trans == 1;
    const bool eff_lower = (uplo == 0) == !transposed;
    const bool unit = diag == 1;
    if (side == 1) {
        trsm_right_thread<N><<<(unsigned)((m + 127) / 128), 128, 0, s>>>(m, n, A, B, eff_lower,
                                                                         transposed, unit, info);
        return record_cuda_error(cudaGetLastError(), "trsm right");
    }
    // The wavefront kernel applies row r's terms as the unknowns are finalised.
    // That is the reference's ascending-k chain only for forward substitution
    // (effective lower): in backward substitution the reference's chain for
    // row r starts with X[r+1], the last unknown finalised before X[r], so each
    // row's chain is serial after its predecessor; those solves use the
    // product-parallel CTA kernel (or the per-column loop for short triangles).
    // The binary64 instance (N == 1) has no reference order to keep and uses
    // the wavefront in both directions.
    // the fast order applies every term as soon as its unknown is final, in both
    // directions (deterministic, not the reference's association)
    const bool wavefront_ok = eff_lower || N == 1 || order == MFLAB_ORDER_FAST;
    if (N == 1 && !transposed && m > 2 * TRSM64_NB && n <= 65535 && !info)
        return trsm64_blocked(m, n, A, B, eff_lower, unit, s, info);
    if (!eff_lower && !wavefront_ok && m > 64 && n < 4096 && (size_t)m * N * 8 <= 200 * 1024) {
        const size_t smem = (size_t)m * N * sizeof(double);
        static std::atomic<unsigned long long> configured{0};
        if (int rc = set_smem_once((const void *)trsm_left_backward_cta<N, 256>, 200 * 1024,
                                   configured, "trsm backward attribute"))
            return rc;
        trsm_left_backward_cta<N, 256><<<(unsigned)n, 256, smem, s>>>(m, n, A, B, transposed,
                                                                       unit, info);
        return record_cuda_error(cudaGetLastError(), "trsm left backward");
    }
    if (m <= 64 || n >= 4096 || !wavefront_ok) {
        trsm_left_thread<N><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(m, n, A, B, eff_lower,
                                                                        transposed, unit, info);
        return record_cuda_error(cudaGetLastError(), "trsm left thread");
    }
    if (n > 2147483647LL) return MFLAB_ERR_UNSUPPORTED;
    if (m <= 256 * 8) {
        trsm_left_cta<N, 256, 8><<<(unsigned)n, 256, 0, s>>>(m, n, A, B, eff_lower, transposed,
                                                             unit, info);
    } else if (m <= 256 * 16) {
        trsm_left_cta<N, 256, 16><<<(unsigned)n, 256, 0, s>>>(m, n, A, B, eff_lower, transposed,
                                                              unit, info);
    } else {
        trsm_left_thread<N><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(m, n, A, B, eff_lower,
                                                                        transposed, unit, info);
    }
    return record_cuda_error(cudaGetLastError(), "trsm left cta");
}

int launch_trsm_info(int N, int side, int uplo, int trans, int diag, int64_t m, int64_t n, Mat A,
                     Mat B, const double *alpha, cudaStream_t s, const int *info, int order) {
    switch (N) {
    case 1: return run_trsm<1>(side, uplo, trans, diag, m, n, A, B, alpha, s, info, order);
    case 2: return run_trsm<2>(side, uplo, trans, diag, m, n, A, B, alpha, s, info, order);
    case 3: return run_trsm<3>(side, uplo, trans, diag, m, n, A, B, alpha, s, info, order);
    case 4: return run_trsm<4>(side, uplo, trans, diag, m, n, A, B, alpha, s, info, order);
    default: return MFLAB_ERR_UNSUPPORTED;
    }
}

int launch_trsm(int N, int side, int uplo, int trans, int diag, int64_t m, int64_t n, Mat A, Mat B,
                const double *alpha, cudaStream_t s) {
    return launch_trsm_info(N, side, uplo, trans, diag, m, n, A, B, alpha, s, nullptr);
}

}  // namespace mfl

extern "C" int mflab_trsm(mflab_handle *h, void *stream, int limbs, int side, int uplo, int trans,
                          int diag, int64_t m, int64_t n, const double *A, int64_t lda,
                          int64_t lsa, double *B, int64_t ldb, int64_t lsb, const double *alpha) {
    MFLAB_RANGE("mflab_trsm");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (side < 0 || side > 1 || uplo < 0 || uplo > 1 || trans < 0 || trans > 1 || diag < 0 ||
        diag > 1)
        return MFLAB_ERR_FLAG;
    if (m < 0 || n < 0 || !alpha) return MFLAB_ERR_ARG;
    const int64_t na = side == 0 ? m : n;
    if ((na > 0 && lda < na) || (m > 0 && ldb < m)) return MFLAB_ERR_ARG;
    return mfl::launch_trsm_info(limbs, side, uplo, trans, diag, m, n,
                                 mfl::Mat{(double *)A, lda, lsa}, mfl::Mat{B, ldb, lsb}, alpha,
                                 (cudaStream_t)stream, nullptr, h->solve_order);
}
