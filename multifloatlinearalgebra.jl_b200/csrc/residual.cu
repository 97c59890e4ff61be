// Residuals, mixed-precision residuals and the normwise backward error
// (src/residual.jl of MultiFloatLinearAlgebra.jl).
//
//   residual!        r = b - A x through the shared mainloop: R <- B, then
//                    gemm!/gemv!(R, A, X, -1, 1) (residual.jl:55-125); with
//                    uplo = lower/upper the symmetric operand mode reproduces
//                    symv!'s ascending-column chain over the authoritative
//                    triangle (symv.jl:1-36).
//   residual_mixed!  r = b - A x computed in a higher limb count: every
//                    operand is converted first and each output is the chain
//                    acc = B; acc -= A[i,k] * X[k,j] for k ascending
//                    (residual.jl:343-428).  Source limb counts 1 (binary64)
//                    to 3, residual limb counts 2 to 4.
//   backward error   ||r|| / (||A|| ||x|| + ||b||) in the reference's
//                    overflow-safe scaled form (residual.jl:178-200), per
//                    right-hand-side column.
#include "mf_device.cuh"
#include "mflab_internal.h"

namespace mfl {

template <int N>
__global__ void copy_planes_kernel(int64_t m, int64_t n, Mat S, Mat D) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m * n) return;
    const int64_t r = e % m, c = e / m;
    store_mf<N>(D.p, D.ld, D.ls, r, c, load_mf<N>(S.p, S.ld, S.ls, r, c));
}

__device__ __forceinline__ bool sym_transposed(int uplo, int64_t r, int64_t c) {
    return (uplo == 1 && c > r) || (uplo == 2 && c < r);
}

template <int NS, int NR>
__device__ __forceinline__ mf<NR> widen(const double *P, int64_t ld, int64_t ls, int64_t r,
                                        int64_t c) {
    mf<NR> x;
#pragma unroll
    for (int l = 0; l < NR; ++l) x.v[l] = l < NS ? P[l * ls + c * ld + r] : 0.0;
    return x;
}

// one thread per output (i, j); uplo 0 general, 1 lower, 2 upper
template <int NS, int NR>
__global__ void residual_mixed_kernel(int64_t m, int64_t k, int64_t nrhs, Mat A, Mat X, Mat B,
                                      Mat R, int uplo) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t j = blockIdx.y;
    if (i >= m || j >= nrhs) return;
    mf<NR> acc = widen<NS, NR>(B.p, B.ld, B.ls, i, j);
    for (int64_t kk = 0; kk < k; ++kk) {
        const bool tr = sym_transposed(uplo, i, kk);
        const mf<NR> a = tr ? widen<NS, NR>(A.p, A.ld, A.ls, kk, i) : widen<NS, NR>(A.p, A.ld, A.ls, i, kk);
        acc = sub(acc, mul(a, widen<NS, NR>(X.p, X.ld, X.ls, kk, j)));
    }
    store_mf<NR>(R.p, R.ld, R.ls, i, j, acc);
}

// row sums of |A| (authoritative triangle for uplo 1/2), ascending columns
template <int N>
__global__ void abs_row_sum_kernel(int64_t m, int64_t k, Mat A, int uplo, double *rowsum,
                                   int *nonfinite) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    mf<N> s = from_double<N>(0.0);
    bool fin = true;
    // The sum is one chain of k dependent additions; the entries are read
    // four columns ahead of it so that no load waits on the chain.
    auto ld = [&](int64_t c) {
        if (c >= k) return from_double<N>(0.0);
        const bool tr = sym_transposed(uplo, i, c);
        const mf<N> v = tr ? load_mf<N>(A.p, A.ld, A.ls, c, i) : load_mf<N>(A.p, A.ld, A.ls, i, c);
        // authoritative entries only: the transposed reads cover the other half
        if (!tr && !isfinite_mf(v)) fin = false;
        return v;
    };
    mf<N> v0 = ld(0), v1 = ld(1), v2 = ld(2), v3 = ld(3);
    for (int64_t c = 0; c < k; c += 4) {
        const mf<N> n0 = ld(c + 4), n1 = ld(c + 5), n2 = ld(c + 6), n3 = ld(c + 7);
        s = add(s, abs_mf(v0));
        if (c + 1 < k) s = add(s, abs_mf(v1));
        if (c + 2 < k) s = add(s, abs_mf(v2));
        if (c + 3 < k) s = add(s, abs_mf(v3));
        v0 = n0;
        v1 = n1;
        v2 = n2;
        v3 = n3;
    }
#pragma unroll
    for (int l = 0; l < N; ++l) rowsum[l * m + i] = s.v[l];
    if (!fin) atomicExch(nonfinite, 1);
}

// ||A||_inf = max over rows of the row sums (Base.max order is irrelevant to the value)
template <int N, int NT>
__global__ void __launch_bounds__(NT) max_rowsum_kernel(int64_t m, const double *rowsum,
                                                        double *out) {
    __shared__ double sv[NT][N];
    const int t = threadIdx.x;
    mf<N> b = from_double<N>(0.0);
    for (int64_t i = t; i < m; i += NT) {
        mf<N> v;
#pragma unroll
        for (int l = 0; l < N; ++l) v.v[l] = rowsum[l * m + i];
        b = max_mf(b, v);
    }
#pragma unroll
    for (int l = 0; l < N; ++l) sv[t][l] = b.v[l];
    __syncthreads();
    for (int off = NT / 2; off > 0; off >>= 1) {
        if (t < off) {
            mf<N> a, c;
#pragma unroll
            for (int l = 0; l < N; ++l) {
                a.v[l] = sv[t][l];
                c.v[l] = sv[t + off][l];
            }
            const mf<N> r = max_mf(a, c);
#pragma unroll
            for (int l = 0; l < N; ++l) sv[t][l] = r.v[l];
        }
        __syncthreads();
    }
    if (t == 0) {
#pragma unroll
        for (int l = 0; l < N; ++l) out[l] = sv[0][l];
    }
}

// residual.jl:178-200
template <int N>
__device__ mf<N> backward_error_value(const mf<N> &an, const mf<N> &xn, const mf<N> &bn,
                                      const mf<N> &rn, bool finite) {
    if (!finite) return from_double<N>(__longlong_as_double(0x7ff8000000000000LL));
    const mf<N> inf = from_double<N>(__longlong_as_double(0x7ff0000000000000LL));
    const mf<N> zero = from_double<N>(0.0);
    const mf<N> primary = max_mf(an, bn);
    if (iszero(primary)) return iszero(rn) ? zero : inf;
    const mf<N> solution_scale = max_mf(xn, from_double<N>(1.0));
    const mf<N> den = add(mul(div(an, primary), div(xn, solution_scale)),
                          div(div(bn, primary), solution_scale));
    if (iszero(den)) return iszero(rn) ? zero : inf;
    const mf<N> num = div(div(rn, primary), solution_scale);
    return div(num, den);
}

// one block per right-hand-side column: column norms, finiteness, the value
template <int N, int NT>
__global__ void __launch_bounds__(NT) backward_error_kernel(int64_t m, int64_t k, Mat X, Mat B,
                                                            Mat R, const double *anorm,
                                                            const int *a_nonfinite, double *out) {
    __shared__ double sv[3][NT][N];
    __shared__ int sf[NT];
    const int t = threadIdx.x;
    const int64_t j = blockIdx.x;
    mf<N> xb = from_double<N>(0.0), bb = xb, rb = xb;
    int fin = 1;
    for (int64_t r = t; r < k; r += NT) {
        const mf<N> v = load_mf<N>(X.p, X.ld, X.ls, r, j);
        if (!isfinite_mf(v)) fin = 0;
        xb = max_mf(xb, abs_mf(v));
    }
    for (int64_t r = t; r < m; r += NT) {
        const mf<N> vb = load_mf<N>(B.p, B.ld, B.ls, r, j), vr = load_mf<N>(R.p, R.ld, R.ls, r, j);
        if (!isfinite_mf(vb) || !isfinite_mf(vr)) fin = 0;
        bb = max_mf(bb, abs_mf(vb));
        rb = max_mf(rb, abs_mf(vr));
    }
#pragma unroll
    for (int l = 0; l < N; ++l) {
        sv[0][t][l] = xb.v[l];
        sv[1][t][l] = bb.v[l];
        sv[2][t][l] = rb.v[l];
    }
    sf[t] = fin;
    __syncthreads();
    for (int off = NT / 2; off > 0; off >>= 1) {
        if (t < off) {
            for (int q = 0; q < 3; ++q) {
                mf<N> a, c;
#pragma unroll
                for (int l = 0; l < N; ++l) {
                    a.v[l] = sv[q][t][l];
                    c.v[l] = sv[q][t + off][l];
                }
                const mf<N> r = max_mf(a, c);
#pragma unroll
                for (int l = 0; l < N; ++l) sv[q][t][l] = r.v[l];
            }
            sf[t] = sf[t] && sf[t + off];
        }
        __syncthreads();
    }
    if (t == 0) {
        mf<N> an, xn, bn, rn;
#pragma unroll
        for (int l = 0; l < N; ++l) {
            an.v[l] = anorm[l];
            xn.v[l] = sv[0][0][l];
            bn.v[l] = sv[1][0][l];
            rn.v[l] = sv[2][0][l];
        }
        const bool finite = sf[0] && !*a_nonfinite;
        const mf<N> v = backward_error_value(an, xn, bn, rn, finite);
#pragma unroll
        for (int l = 0; l < N; ++l) out[j * N + l] = v.v[l];
    }
}

template <int N>
static int residual_n(int uplo, int vector_rhs, int64_t m, int64_t k, int64_t nrhs, Mat A, Mat X,
                      Mat B, Mat R, cudaStream_t s) {
    if (R.p != B.p) {
        const int64_t tot = m * nrhs;
        copy_planes_kernel<N><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(m, nrhs, B, R);
        int rc = record_cuda_error(cudaGetLastError(), "residual copy");
        if (rc) return rc;
    }
    const double mone[4] = {-1.0, 0.0, 0.0, 0.0}, one[4] = {1.0, 0.0, 0.0, 0.0};
    // gemv!/symv! (vector) and symv! per column use acc + a*b; gemm! (matrix,
    // general) takes the :auto route, fused for Float64x3
    const bool fused = uplo == 0 && !vector_rhs && N == 3;
    return launch_mm(N, uplo == 0 ? 0 : uplo == 1 ? 2 : 3, false, 0, fused, m, nrhs, k, A, X, R,
                     mone, one, s, nullptr);
}

}  // namespace mfl

using mfl::Mat;

extern "C" int mflab_residual(mflab_handle *h, void *stream, int limbs, int uplo, int vector_rhs,
                              int64_t m, int64_t k, int64_t nrhs, const double *A, int64_t lda,
                              int64_t lsa, const double *X, int64_t ldx, int64_t lsx,
                              const double *B, int64_t ldb, int64_t lsb, double *R, int64_t ldr,
                              int64_t lsr) {
    MFLAB_RANGE("mflab_residual");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (uplo < 0 || uplo > 2) return MFLAB_ERR_FLAG;
    if (m < 0 || k < 0 || nrhs < 0) return MFLAB_ERR_ARG;
    if (uplo != 0 && m != k) return MFLAB_ERR_ARG;
    if (m == 0 || nrhs == 0) return MFLAB_OK;
    if (lda < m || ldx < (k > 0 ? k : 1) || ldb < m || ldr < m) return MFLAB_ERR_ARG;
    if (mfl::views_overlap(R, ldr, lsr, m, nrhs, limbs, X, ldx, lsx, k, nrhs) ||
        mfl::views_overlap(R, ldr, lsr, m, nrhs, limbs, A, lda, lsa, m, k))
        return MFLAB_ERR_ALIAS;
    if (R != B && mfl::views_overlap(R, ldr, lsr, m, nrhs, limbs, B, ldb, lsb, m, nrhs))
        return MFLAB_ERR_ALIAS;
    Mat a{(double *)A, lda, lsa}, x{(double *)X, ldx, lsx}, b{(double *)B, ldb, lsb}, r{R, ldr, lsr};
    cudaStream_t s = (cudaStream_t)stream;
    switch (limbs) {
    case 2: return mfl::residual_n<2>(uplo, vector_rhs, m, k, nrhs, a, x, b, r, s);
    case 3: return mfl::residual_n<3>(uplo, vector_rhs, m, k, nrhs, a, x, b, r, s);
    default: return mfl::residual_n<4>(uplo, vector_rhs, m, k, nrhs, a, x, b, r, s);
    }
}

extern "C" int mflab_residual_mixed(mflab_handle *h, void *stream, int src_limbs, int res_limbs,
                                    int uplo, int64_t m, int64_t k, int64_t nrhs, const double *A,
                                    int64_t lda, int64_t lsa, const double *X, int64_t ldx,
                                    int64_t lsx, const double *B, int64_t ldb, int64_t lsb,
                                    double *R, int64_t ldr, int64_t lsr) {
    MFLAB_RANGE("mflab_residual_mixed");
    if (!h) return MFLAB_ERR_UNSUPPORTED;
    if (!(src_limbs >= 1 && src_limbs < res_limbs && res_limbs <= 4 && res_limbs >= 2))
        return MFLAB_ERR_UNSUPPORTED;
    if (uplo < 0 || uplo > 2) return MFLAB_ERR_FLAG;
    if (m < 0 || k < 0 || nrhs < 0) return MFLAB_ERR_ARG;
    if (uplo != 0 && m != k) return MFLAB_ERR_ARG;
    if (m == 0 || nrhs == 0) return MFLAB_OK;
    if (nrhs > 65535) return MFLAB_ERR_UNSUPPORTED;
    if (lda < m || ldx < (k > 0 ? k : 1) || ldb < m || ldr < m) return MFLAB_ERR_ARG;
    Mat a{(double *)A, lda, lsa}, x{(double *)X, ldx, lsx}, b{(double *)B, ldb, lsb}, r{R, ldr, lsr};
    cudaStream_t s = (cudaStream_t)stream;
    dim3 g((unsigned)((m + 127) / 128), (unsigned)nrhs);
    const int key = src_limbs * 10 + res_limbs;
    switch (key) {
    case 12: mfl::residual_mixed_kernel<1, 2><<<g, 128, 0, s>>>(m, k, nrhs, a, x, b, r, uplo); break;
    case 13: mfl::residual_mixed_kernel<1, 3><<<g, 128, 0, s>>>(m, k, nrhs, a, x, b, r, uplo); break;
    case 14: mfl::residual_mixed_kernel<1, 4><<<g, 128, 0, s>>>(m, k, nrhs, a, x, b, r, uplo); break;
    case 23: mfl::residual_mixed_kernel<2, 3><<<g, 128, 0, s>>>(m, k, nrhs, a, x, b, r, uplo); break;
    case 24: mfl::residual_mixed_kernel<2, 4><<<g, 128, 0, s>>>(m, k, nrhs, a, x, b, r, uplo); break;
    case 34: mfl::residual_mixed_kernel<3, 4><<<g, 128, 0, s>>>(m, k, nrhs, a, x, b, r, uplo); break;
    default: return MFLAB_ERR_UNSUPPORTED;
    }
    return mfl::record_cuda_error(cudaGetLastError(), "residual_mixed");
}

extern "C" int mflab_backward_error(mflab_handle *h, void *stream, int limbs, int uplo, int64_t m,
                                    int64_t k, int64_t nrhs, const double *A, int64_t lda,
                                    int64_t lsa, const double *X, int64_t ldx, int64_t lsx,
                                    const double *B, int64_t ldb, int64_t lsb, const double *R,
                                    int64_t ldr, int64_t lsr, double *out) {
    MFLAB_RANGE("mflab_backward_error");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (uplo < 0 || uplo > 2) return MFLAB_ERR_FLAG;
    if (m < 0 || k < 0 || nrhs < 0 || !out) return MFLAB_ERR_ARG;
    if (uplo != 0 && m != k) return MFLAB_ERR_ARG;
    if (nrhs == 0) return MFLAB_OK;
    const size_t need = sizeof(double) * (size_t)limbs * (size_t)(m + 8) + 64;
    int rc = mflab_reserve_scratch(h, need);
    if (rc) return rc;
    double *rowsum = (double *)h->scratch;
    double *anorm = rowsum + (size_t)limbs * (m > 0 ? m : 1);
    int *anf = (int *)(anorm + 4);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(anf, 0, sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(anorm, 0, sizeof(double) * 4, s);
    if (e != cudaSuccess) return mfl::record_cuda_error(e, "backward error init");
    Mat a{(double *)A, lda, lsa}, x{(double *)X, ldx, lsx}, b{(double *)B, ldb, lsb},
        r{(double *)R, ldr, lsr};
    const unsigned gm = (unsigned)((m + 127) / 128);
    switch (limbs) {
    case 2:
        if (m > 0) {
            mfl::abs_row_sum_kernel<2><<<gm, 128, 0, s>>>(m, k, a, uplo, rowsum, anf);
            mfl::max_rowsum_kernel<2, 256><<<1, 256, 0, s>>>(m, rowsum, anorm);
        }
        mfl::backward_error_kernel<2, 256><<<(unsigned)nrhs, 256, 0, s>>>(m, k, x, b, r, anorm, anf, out);
        break;
    case 3:
        if (m > 0) {
            mfl::abs_row_sum_kernel<3><<<gm, 128, 0, s>>>(m, k, a, uplo, rowsum, anf);
            mfl::max_rowsum_kernel<3, 256><<<1, 256, 0, s>>>(m, rowsum, anorm);
        }
        mfl::backward_error_kernel<3, 256><<<(unsigned)nrhs, 256, 0, s>>>(m, k, x, b, r, anorm, anf, out);
        break;
    default:
        if (m > 0) {
            mfl::abs_row_sum_kernel<4><<<gm, 128, 0, s>>>(m, k, a, uplo, rowsum, anf);
            mfl::max_rowsum_kernel<4, 256><<<1, 256, 0, s>>>(m, rowsum, anorm);
        }
        mfl::backward_error_kernel<4, 256><<<(unsigned)nrhs, 256, 0, s>>>(m, k, x, b, r, anorm, anf, out);
        break;
    }
    return mfl::record_cuda_error(cudaGetLastError(), "backward error");
}

// ||A||_inf alone (the matrix term of the backward error, residual.jl:178-200)
// into the caller's device buffers: anorm[limbs] and *nonfinite (0 / 1), for
// repeated backward errors against one matrix (iterative refinement).
extern "C" int mflab_opnorm_inf(mflab_handle *h, void *stream, int limbs, int uplo, int64_t m,
                                int64_t k, const double *A, int64_t lda, int64_t lsa,
                                double *anorm, int *nonfinite) {
    MFLAB_RANGE("mflab_opnorm_inf");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (uplo < 0 || uplo > 2) return MFLAB_ERR_FLAG;
    if (m < 0 || k < 0 || !anorm || !nonfinite) return MFLAB_ERR_ARG;
    if (uplo != 0 && m != k) return MFLAB_ERR_ARG;
    const size_t need = sizeof(double) * (size_t)limbs * (size_t)(m + 8) + 64;
    int rc = mflab_reserve_scratch(h, need);
    if (rc) return rc;
    double *rowsum = (double *)h->scratch;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(nonfinite, 0, sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(anorm, 0, sizeof(double) * limbs, s);
    if (e != cudaSuccess) return mfl::record_cuda_error(e, "opnorm init");
    if (m == 0) return MFLAB_OK;
    mfl::Mat a{(double *)A, lda, lsa};
    const unsigned gm = (unsigned)((m + 127) / 128);
    switch (limbs) {
    case 2:
        mfl::abs_row_sum_kernel<2><<<gm, 128, 0, s>>>(m, k, a, uplo, rowsum, nonfinite);
        mfl::max_rowsum_kernel<2, 256><<<1, 256, 0, s>>>(m, rowsum, anorm);
        break;
    case 3:
        mfl::abs_row_sum_kernel<3><<<gm, 128, 0, s>>>(m, k, a, uplo, rowsum, nonfinite);
        mfl::max_rowsum_kernel<3, 256><<<1, 256, 0, s>>>(m, rowsum, anorm);
        break;
    default:
        mfl::abs_row_sum_kernel<4><<<gm, 128, 0, s>>>(m, k, a, uplo, rowsum, nonfinite);
        mfl::max_rowsum_kernel<4, 256><<<1, 256, 0, s>>>(m, rowsum, anorm);
        break;
    }
    return mfl::record_cuda_error(cudaGetLastError(), "opnorm");
}

// the backward errors of mflab_backward_error with ||A||_inf and its
// finiteness flag from mflab_opnorm_inf (the matrix is not read)
extern "C" int mflab_backward_error_norm(mflab_handle *h, void *stream, int limbs, int64_t m,
                                         int64_t k, int64_t nrhs, const double *anorm,
                                         const int *nonfinite, const double *X, int64_t ldx,
                                         int64_t lsx, const double *B, int64_t ldb, int64_t lsb,
                                         const double *R, int64_t ldr, int64_t lsr, double *out) {
    MFLAB_RANGE("mflab_backward_error_norm");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (m < 0 || k < 0 || nrhs < 0 || !out || !anorm || !nonfinite) return MFLAB_ERR_ARG;
    if (nrhs == 0) return MFLAB_OK;
    mfl::Mat x{(double *)X, ldx, lsx}, b{(double *)B, ldb, lsb}, r{(double *)R, ldr, lsr};
    cudaStream_t s = (cudaStream_t)stream;
    switch (limbs) {
    case 2:
        mfl::backward_error_kernel<2, 256><<<(unsigned)nrhs, 256, 0, s>>>(m, k, x, b, r, anorm,
                                                                         nonfinite, out);
        break;
    case 3:
        mfl::backward_error_kernel<3, 256><<<(unsigned)nrhs, 256, 0, s>>>(m, k, x, b, r, anorm,
                                                                         nonfinite, out);
        break;
    default:
        mfl::backward_error_kernel<4, 256><<<(unsigned)nrhs, 256, 0, s>>>(m, k, x, b, r, anorm,
                                                                         nonfinite, out);
        break;
    }
    return mfl::record_cuda_error(cudaGetLastError(), "backward error (given norm)");
}

namespace mfl {
// X <- X + widen(D): the correction step of iterative refinement
template <int NS, int NR>
__global__ void add_widened_kernel(int64_t m, int64_t n, Mat D, Mat X) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m * n) return;
    const int64_t r = e % m, c = e / m;
    store_mf<NR>(X.p, X.ld, X.ls, r, c,
                 add(load_mf<NR>(X.p, X.ld, X.ls, r, c), widen<NS, NR>(D.p, D.ld, D.ls, r, c)));
}
}  // namespace mfl

extern "C" int mflab_add_widened(mflab_handle *h, void *stream, int src_limbs, int dst_limbs,
                                 int64_t m, int64_t n, const double *D, int64_t ldd, int64_t lsd,
                                 double *X, int64_t ldx, int64_t lsx) {
    MFLAB_RANGE("mflab_add_widened");
    if (!h) return MFLAB_ERR_UNSUPPORTED;
    if (m < 0 || n < 0) return MFLAB_ERR_ARG;
    if (m == 0 || n == 0) return MFLAB_OK;
    Mat d{(double *)D, ldd, lsd}, x{X, ldx, lsx};
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned g = (unsigned)((m * n + 255) / 256);
    switch (src_limbs * 10 + dst_limbs) {
    case 12: mfl::add_widened_kernel<1, 2><<<g, 256, 0, s>>>(m, n, d, x); break;
    case 13: mfl::add_widened_kernel<1, 3><<<g, 256, 0, s>>>(m, n, d, x); break;
    case 14: mfl::add_widened_kernel<1, 4><<<g, 256, 0, s>>>(m, n, d, x); break;
    case 23: mfl::add_widened_kernel<2, 3><<<g, 256, 0, s>>>(m, n, d, x); break;
    case 24: mfl::add_widened_kernel<2, 4><<<g, 256, 0, s>>>(m, n, d, x); break;
    case 34: mfl::add_widened_kernel<3, 4><<<g, 256, 0, s>>>(m, n, d, x); break;
    default: return MFLAB_ERR_UNSUPPORTED;
    }
    return mfl::record_cuda_error(cudaGetLastError(), "add_widened");
}
