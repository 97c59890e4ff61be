// INT8-slice (Ozaki scheme I) multi-double GEMM on the tensor cores.
//
// No reference counterpart: MultiFloatLinearAlgebra.jl has only the FP64
// networks.  Published method: Ozaki, Ogita, Oishi, Rump (2012), error-free
// transformation of matrix products; Ootomo, Ozaki, Yokota (2024), DGEMM on
// integer matrix multiplication units.
//
// 1. Scaling.  Row i of A gets the power of two 2^Ea_i with |A(i,:)| < 2^(Ea_i-1),
//    column j of B gets 2^Eb_j likewise (leading-limb maxima, frexp).
// 2. Exact digit split.  Each scaled multi-double x in (-1/2, 1/2) is written
//    as sum_{s=1..S} d_s 2^(-7 s) + r with signed digits d_s = rint(128 * r_{s-1})
//    in [-64, 64]; the running remainder is kept exact by limb-wise
//    subtraction and a TwoSum re-distillation of the limbs after each digit.
// 3. Level products.  Digits are stored A8[i][s][k] and B8[j][S-1-s][k]
//    (B's slice order reversed), so for a significance level L = s + t
//    (s, t >= 1, L <= S+1) every pair (s, L-s) is adjacent along K:
//        I_L = A8[:, 0:(L-1)k] * B8[:, (S-L+1)k : S k]^T      (int8 x int8 -> int32)
//    is ONE integer GEMM with K = (L-1) k, exact as long as
//    (L-1) k 65^2 < 2^31.
// 4. Accumulation.  C(i,j) = 2^(Ea_i + Eb_j) sum_L 2^(-7L) I_L(i,j): the S int32
//    levels are added, least significant first, into a Float64xN accumulator
//    with the add network, scaled by the power of two, and the alpha/beta
//    epilogue of the plain kernel is applied.
// The truncation (digit remainders and levels above S+1) bounds the error by
// about k 2^(Ea+Eb) 2^(-7S); the slice count S is the accuracy knob.
#include <cublasLt.h>

#include <climits>
#include <cmath>

#include "mf_device.cuh"
#include "mflab_internal.h"
#include "ozaki_common.cuh"

namespace mfl {

__device__ __forceinline__ int exp_of(double a) {
    int e;
    frexp(a, &e);
    return e;
}

// row maxima of A (m x k, column-major planes): grid (ceil(m/256), kchunks)
template <int N>
__global__ void oz_row_exp_kernel(int64_t m, int64_t k, Mat A, int64_t kchunk, int *rowexp) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int64_t k0 = (int64_t)blockIdx.y * kchunk;
    const int64_t k1 = k0 + kchunk < k ? k0 + kchunk : k;
    double mx = 0.0;
    bool bad = false;
    for (int64_t kk = k0; kk < k1; ++kk) {
        const double *p = A.p + kk * A.ld + i;
#pragma unroll
        for (int l = 0; l < N; ++l) bad |= !isfinite(p[l * A.ls]);
        mx = fmax(mx, fabs(p[0]));
    }
    int e = bad ? OZ_EXP_BAD : (mx > 0.0 ? exp_of(mx) : OZ_EXP_EMPTY);
    atomicMax(&rowexp[i], e);
}

// column maxima of B (k x n): one warp per column
template <int N>
__global__ void oz_col_exp_kernel(int64_t k, int64_t n, Mat B, int *colexp) {
    const int64_t j = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    if (j >= n) return;
    double mx = 0.0;
    int bad = 0;
    for (int64_t kk = lane; kk < k; kk += 32) {
        const double *p = B.p + j * B.ld + kk;
#pragma unroll
        for (int l = 0; l < N; ++l) bad |= !isfinite(p[l * B.ls]);
        mx = fmax(mx, fabs(p[0]));
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
        bad |= __shfl_xor_sync(0xffffffffu, bad, off);
    }
    if (lane == 0) colexp[j] = bad ? OZ_EXP_BAD : (mx > 0.0 ? exp_of(mx) : OZ_EXP_EMPTY);
}

// digits of one scaled value; emit(s, d) is called for s = 0..S-1
template <int N, typename Emit>
__device__ __forceinline__ void oz_digits(mf<N> x, int S, Emit emit) {
    for (int s = 0; s < S; ++s) {
#pragma unroll
        for (int l = 0; l < N; ++l) x.v[l] = __dmul_rn(x.v[l], 128.0);
        const double d = rint(x.v[0]);
        x.v[0] = __dsub_rn(x.v[0], d);  // exact: |x0| < 2^52
        // re-distill so that x.v[0] carries the value of the remainder
#pragma unroll
        for (int l = N - 1; l > 0; --l) two_sum(x.v[l - 1], x.v[l], x.v[l - 1], x.v[l]);
        emit(s, (int)d);
    }
}

// A digits: 32 x 32 tile (rows x k) per block of 32 x 8 threads, transposed
// through shared memory so that both the plane reads (along rows) and the
// int8 writes (along k) are coalesced.
template <int N>
__global__ void __launch_bounds__(256) oz_split_a_kernel(int64_t m, int64_t mp, int64_t k,
                                                         int64_t kp, int S, Mat A,
                                                         const int *rowexp, int8_t *A8) {
    __shared__ double t[N][32][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int64_t i0 = (int64_t)blockIdx.x * 32, k0 = (int64_t)blockIdx.y * 32;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int kk = ty + 8 * j;
        const int64_t i = i0 + tx, kg = k0 + kk;
        const bool ok = i < m && kg < k;
#pragma unroll
        for (int l = 0; l < N; ++l) t[l][kk][tx] = ok ? A.p[l * A.ls + kg * A.ld + i] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int ii = ty + 8 * j;
        const int64_t i = i0 + ii, kg = k0 + tx;
        if (i >= mp || kg >= kp) continue;
        const int e = i < m ? rowexp[i] : OZ_EXP_EMPTY;  // padding rows: zero digits
        const int sh = oz_scale_exp(e);
        mf<N> x;
#pragma unroll
        for (int l = 0; l < N; ++l) x.v[l] = (e == OZ_EXP_BAD) ? 0.0 : ldexp(t[l][tx][ii], -sh);
        int8_t *dst = A8 + (size_t)i * S * kp + kg;
        oz_digits<N>(x, S, [&](int s, int d) { dst[(size_t)s * kp] = (int8_t)d; });
    }
}

// B digits: column j of B is contiguous along k; slice order reversed
template <int N>
__global__ void oz_split_b_kernel(int64_t k, int64_t n, int64_t np, int64_t kp, int S, Mat B,
                                  const int *colexp, int8_t *B8) {
    const int64_t kg = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t j = blockIdx.y;
    if (kg >= kp || j >= np) return;
    const int e = j < n ? colexp[j] : OZ_EXP_EMPTY;  // padding columns: zero digits
    const int sh = oz_scale_exp(e);
    mf<N> x;
#pragma unroll
    for (int l = 0; l < N; ++l)
        x.v[l] = (kg < k && j < n && e != OZ_EXP_BAD) ? ldexp(B.p[l * B.ls + j * B.ld + kg], -sh)
                                                        : 0.0;
    int8_t *dst = B8 + (size_t)j * S * kp + kg;
    oz_digits<N>(x, S, [&](int s, int d) { dst[(size_t)(S - 1 - s) * kp] = (int8_t)d; });
}

// C = alpha * 2^(Ea+Eb) sum_L 2^(-7L) I_L (+ beta * C)
template <int N>
__global__ void oz_accum_kernel(int64_t m, int64_t n, int S, const int32_t *I, int64_t ldi,
                                size_t plane, const int *rowexp, const int *colexp, Mat C,
                                scal<N> alpha, scal<N> beta, int overwrite) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t j = blockIdx.y;
    if (i >= m || j >= n) return;
    const int ea = rowexp[i], eb = colexp[j];
    mf<N> acc = from_double<N>(0.0);
    if (ea == OZ_EXP_BAD || eb == OZ_EXP_BAD) {
        acc = from_double<N>(__longlong_as_double(0x7ff8000000000000LL));
    } else {
        for (int L = S + 1; L >= 2; --L) {
            const double v = (double)I[(size_t)(L - 2) * plane + (size_t)j * ldi + i];
            acc = add(acc, from_double<N>(ldexp(v, 7 * (S + 1 - L))));
        }
        const int sh = oz_scale_exp(ea) + oz_scale_exp(eb) - 7 * (S + 1);
#pragma unroll
        for (int l = 0; l < N; ++l) acc.v[l] = ldexp(acc.v[l], sh);
    }
    mf<N> r = mul(alpha.get(), acc);
    if (!overwrite) r = add(r, mul(beta.get(), load_mf<N>(C.p, C.ld, C.ls, i, j)));
    store_mf<N>(C.p, C.ld, C.ls, i, j, r);
}

// Sampled scale gap for the slice-count tuner: for sampled entries (i, j),
// g = log2(k 2^(Ea'_i + Eb'_j) / sum_k |a_ik| |b_kj|) (leading limbs, binary64),
// the number of bits between the truncation scale of the digit products and
// the entry's own magnitude scale.  One warp per sample; the maximum over
// samples is kept in eighths of a bit (atomicMax).
// TA / TB: the operand is given transposed (A as a k x m, B as an n x k
// column-major matrix), for the Gram products of the SYRK forms.
template <bool TA, bool TB>
__global__ void oz_gap_kernel(int64_t m, int64_t n, int64_t k, Mat A, Mat B, const int *rowexp,
                              const int *colexp, int samples, int *gap8) {
    const int s = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    if (s >= samples) return;
    // deterministic spread of the samples over the matrix (64-bit LCG)
    unsigned long long h = 6364136223846793005ULL * (unsigned long long)(s + 1) + 1442695040888963407ULL;
    const int64_t i = (int64_t)((h >> 17) % (unsigned long long)m);
    h = 6364136223846793005ULL * h + 1442695040888963407ULL;
    const int64_t j = (int64_t)((h >> 17) % (unsigned long long)n);
    const int ea = rowexp[i], eb = colexp[j];
    if (ea == OZ_EXP_BAD || eb == OZ_EXP_BAD || ea == OZ_EXP_EMPTY || eb == OZ_EXP_EMPTY) return;
    double d = 0.0;
    for (int64_t kk = lane; kk < k; kk += 32)
        d = fma(fabs(TA ? A.p[i * A.ld + kk] : A.p[kk * A.ld + i]),
                fabs(TB ? B.p[kk * B.ld + j] : B.p[j * B.ld + kk]), d);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) d += __shfl_xor_sync(0xffffffffu, d, off);
    if (lane == 0 && d > 0.0) {
        const double g = log2((double)k) + (double)(oz_scale_exp(ea) + oz_scale_exp(eb)) - log2(d);
        atomicMax(gap8, (int)ceil(8.0 * g));
    }
}

// ----------------------------------------------------------- host side ---
struct OzPlan {
    int S;
    int64_t kp;     // k rounded up to 16 (int8 rows 16-byte aligned; zero digits pad)
    int64_t mp, np; // m, n rounded up to 16: the padding rows/columns hold zero digits
    int64_t ldi;    // leading dimension of an int32 level plane (= mp)
    size_t plane;   // elements between level planes (multiple of 64)
    size_t a8, b8, lev, exps, ws, total;
};

static OzPlan oz_plan(int64_t m, int64_t n, int64_t k, int S) {
    // (kp, mp, np padding below)
    OzPlan p;
    p.S = S;
    // padded to the tcgen05 tile (128 x 256 outputs, 128-byte K steps); the
    // padding rows, columns and K positions hold zero digits
    p.kp = (k + 127) / 128 * 128;
    p.mp = (m + 127) / 128 * 128;
    p.np = (n + 255) / 256 * 256;
    p.ldi = p.mp;
    p.plane = ((size_t)p.ldi * p.np + 63) / 64 * 64;
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    p.a8 = al((size_t)p.mp * S * p.kp);
    p.b8 = al((size_t)p.np * S * p.kp);
    p.lev = al((size_t)S * p.plane * sizeof(int32_t));
    p.exps = al((size_t)(m + n) * sizeof(int));
    p.ws = (size_t)64 << 20;
    p.total = p.a8 + p.b8 + p.lev + p.exps + p.ws;
    return p;
}

static cublasLtHandle_t lt_handle() {
    static cublasLtHandle_t h = nullptr;
    if (!h) cublasLtCreate(&h);
    return h;
}

// I = Aop^T * Bop with int8 operands stored K-major (ld = lda / ldb bytes)
int int8_gemm_tn(int64_t m, int64_t n, int64_t K, const int8_t *A, int64_t lda,
                        const int8_t *B, int64_t ldb, int32_t *I, int64_t ldi, void *ws, size_t wsb,
                        cudaStream_t s) {
    cublasLtHandle_t h = lt_handle();
    if (!h) return MFLAB_ERR_CUDA;
    cublasLtMatmulDesc_t op = nullptr;
    cublasLtMatrixLayout_t Ad = nullptr, Bd = nullptr, Cd = nullptr;
    cublasLtMatmulPreference_t pref = nullptr;
    int rc = MFLAB_OK;
    cublasOperation_t ta = CUBLAS_OP_T, tb = CUBLAS_OP_N;
    cublasLtMatmulHeuristicResult_t res{};
    int nres = 0;
    int32_t one = 1, zero = 0;
    if (cublasLtMatmulDescCreate(&op, CUBLAS_COMPUTE_32I, CUDA_R_32I) != CUBLAS_STATUS_SUCCESS ||
        cublasLtMatmulDescSetAttribute(op, CUBLASLT_MATMUL_DESC_TRANSA, &ta, sizeof(ta)) ||
        cublasLtMatmulDescSetAttribute(op, CUBLASLT_MATMUL_DESC_TRANSB, &tb, sizeof(tb)) ||
        cublasLtMatrixLayoutCreate(&Ad, CUDA_R_8I, K, m, lda) ||
        cublasLtMatrixLayoutCreate(&Bd, CUDA_R_8I, K, n, ldb) ||
        cublasLtMatrixLayoutCreate(&Cd, CUDA_R_32I, m, n, ldi) ||
        cublasLtMatmulPreferenceCreate(&pref) ||
        cublasLtMatmulPreferenceSetAttribute(pref, CUBLASLT_MATMUL_PREF_MAX_WORKSPACE_BYTES, &wsb,
                                             sizeof(wsb)) ||
        cublasLtMatmulAlgoGetHeuristic(h, op, Ad, Bd, Cd, Cd, pref, 1, &res, &nres) ||
        nres == 0) {
        rc = MFLAB_ERR_UNSUPPORTED;
    } else if (cublasLtMatmul(h, op, &one, A, Ad, B, Bd, &zero, I, Cd, I, Cd, &res.algo, ws, wsb,
                              s) != CUBLAS_STATUS_SUCCESS) {
        rc = MFLAB_ERR_CUDA;
    }
    if (pref) cublasLtMatmulPreferenceDestroy(pref);
    if (Cd) cublasLtMatrixLayoutDestroy(Cd);
    if (Bd) cublasLtMatrixLayoutDestroy(Bd);
    if (Ad) cublasLtMatrixLayoutDestroy(Ad);
    if (op) cublasLtMatmulDescDestroy(op);
    return rc;
}

// C = alpha A B + beta C in binary64 through the library (column-major, no
// transposes): the plain trailing update of the binary64 LU
int dgemm_lt(int64_t m, int64_t n, int64_t k, const double *A, int64_t lda, const double *B,
             int64_t ldb, double *C, int64_t ldc, double alpha, double beta, void *ws, size_t wsb,
             cudaStream_t s) {
    if (m <= 0 || n <= 0) return MFLAB_OK;
    cublasLtHandle_t h = lt_handle();
    if (!h) return MFLAB_ERR_CUDA;
    cublasLtMatmulDesc_t op = nullptr;
    cublasLtMatrixLayout_t Ad = nullptr, Bd = nullptr, Cd = nullptr;
    cublasLtMatmulPreference_t pref = nullptr;
    int rc = MFLAB_OK;
    cublasLtMatmulHeuristicResult_t res{};
    int nres = 0;
    if (cublasLtMatmulDescCreate(&op, CUBLAS_COMPUTE_64F, CUDA_R_64F) != CUBLAS_STATUS_SUCCESS ||
        cublasLtMatrixLayoutCreate(&Ad, CUDA_R_64F, m, k, lda) ||
        cublasLtMatrixLayoutCreate(&Bd, CUDA_R_64F, k, n, ldb) ||
        cublasLtMatrixLayoutCreate(&Cd, CUDA_R_64F, m, n, ldc) ||
        cublasLtMatmulPreferenceCreate(&pref) ||
        cublasLtMatmulPreferenceSetAttribute(pref, CUBLASLT_MATMUL_PREF_MAX_WORKSPACE_BYTES, &wsb,
                                             sizeof(wsb)) ||
        cublasLtMatmulAlgoGetHeuristic(h, op, Ad, Bd, Cd, Cd, pref, 1, &res, &nres) ||
        nres == 0) {
        rc = MFLAB_ERR_UNSUPPORTED;
    } else if (cublasLtMatmul(h, op, &alpha, A, Ad, B, Bd, &beta, C, Cd, C, Cd, &res.algo, ws, wsb,
                              s) != CUBLAS_STATUS_SUCCESS) {
        rc = MFLAB_ERR_CUDA;
    }
    if (pref) cublasLtMatmulPreferenceDestroy(pref);
    if (Cd) cublasLtMatrixLayoutDestroy(Cd);
    if (Bd) cublasLtMatrixLayoutDestroy(Bd);
    if (Ad) cublasLtMatrixLayoutDestroy(Ad);
    if (op) cublasLtMatmulDescDestroy(op);
    return rc;
}

template <int N>
static int oz_exponents(int64_t m, int64_t n, int64_t k, Mat A, Mat B, int *rowexp, int *colexp,
                        cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(rowexp, 0x80, sizeof(int) * m, s);  // 0x80808080 < any exponent
    if (e != cudaSuccess) return record_cuda_error(e, "ozaki exps");
    // short k chunks: enough blocks to cover every SM even for few rows
    int64_t kchunk = 32;
    if ((k + kchunk - 1) / kchunk > 65535) kchunk = (k + 65534) / 65535;
    dim3 gr((unsigned)((m + 255) / 256), (unsigned)((k + kchunk - 1) / kchunk));
    oz_row_exp_kernel<N><<<gr, 256, 0, s>>>(m, k, A, kchunk, rowexp);
    if (n > 0) oz_col_exp_kernel<N><<<(unsigned)((n + 7) / 8), 256, 0, s>>>(k, n, B, colexp);
    return record_cuda_error(cudaGetLastError(), "ozaki exponents");
}

// row exponents of A alone / column exponents of B alone (the prepared
// operand of the modular route and its per-call right operand)
int ozaki_row_exps(int N, int64_t m, int64_t k, Mat A, int *rowexp, cudaStream_t s) {
    if (m <= 0) return MFLAB_OK;
    switch (N) {
    case 2: return oz_exponents<2>(m, 0, k, A, A, rowexp, nullptr, s);
    case 3: return oz_exponents<3>(m, 0, k, A, A, rowexp, nullptr, s);
    case 4: return oz_exponents<4>(m, 0, k, A, A, rowexp, nullptr, s);
    default: return MFLAB_ERR_UNSUPPORTED;
    }
}

int ozaki_col_exps(int N, int64_t k, int64_t n, Mat B, int *colexp, cudaStream_t s) {
    if (n <= 0) return MFLAB_OK;
    switch (N) {
    case 2: oz_col_exp_kernel<2><<<(unsigned)((n + 7) / 8), 256, 0, s>>>(k, n, B, colexp); break;
    case 3: oz_col_exp_kernel<3><<<(unsigned)((n + 7) / 8), 256, 0, s>>>(k, n, B, colexp); break;
    case 4: oz_col_exp_kernel<4><<<(unsigned)((n + 7) / 8), 256, 0, s>>>(k, n, B, colexp); break;
    default: return MFLAB_ERR_UNSUPPORTED;
    }
    return record_cuda_error(cudaGetLastError(), "ozaki column exponents");
}

// optional phase events (profiling entry point only): [0] after exponents and
// tuning, [1] after the digit split, [2] after the level GEMMs, [3] at the end
static cudaEvent_t *g_phase_ev = nullptr;
void ozaki_phase(int i, cudaStream_t s) {
    if (g_phase_ev) cudaEventRecord(g_phase_ev[i], s);
}
void ozaki_set_phase_events(cudaEvent_t *ev) { g_phase_ev = ev; }
static inline void phase(int i, cudaStream_t s) { ozaki_phase(i, s); }

template <int N>
static int ozaki_n(int64_t m, int64_t n, int64_t k, Mat A, Mat B, Mat C, const double *alpha,
                   const double *beta, int S, char *base, const OzPlan &p, const int *rowexp,
                   const int *colexp, cudaStream_t s, int engine, int *tc_err,
                   const TcOpts &opts) {
    phase(0, s);
    int8_t *A8 = (int8_t *)base;
    int8_t *B8 = (int8_t *)(base + p.a8);
    int32_t *I = (int32_t *)(base + p.a8 + p.b8);
    void *ws = base + p.a8 + p.b8 + p.lev + p.exps;
    dim3 ga((unsigned)((p.mp + 31) / 32), (unsigned)((p.kp + 31) / 32));
    oz_split_a_kernel<N><<<ga, dim3(32, 8), 0, s>>>(m, p.mp, k, p.kp, S, A, rowexp, A8);
    dim3 gb((unsigned)((p.kp + 255) / 256), (unsigned)p.np);
    oz_split_b_kernel<N><<<gb, 256, 0, s>>>(k, n, p.np, p.kp, S, B, colexp, B8);
    int rc = record_cuda_error(cudaGetLastError(), "ozaki split");
    if (rc) return rc;
    phase(1, s);
    const int64_t ld8 = (int64_t)S * p.kp;
    for (int L = 2; L <= S + 1; ++L) {
        if (engine != MFLAB_INT8_LIBRARY)
            rc = int8_gemm_tc(p.mp, p.np, (int64_t)(L - 1) * p.kp, A8, ld8, ld8, B8, ld8, ld8,
                              (int64_t)(S - L + 1) * p.kp, I + (size_t)(L - 2) * p.plane, p.ldi,
                              tc_err, s, opts);
        else
            rc = int8_gemm_tn(p.mp, p.np, (int64_t)(L - 1) * p.kp, A8, ld8,
                              B8 + (int64_t)(S - L + 1) * p.kp, ld8,
                              I + (size_t)(L - 2) * p.plane, p.ldi, ws, p.ws, s);
        if (rc) return rc;
    }
    phase(2, s);
    scal<N> al{}, be{};
    int overwrite = 1;
    for (int l = 0; l < N; ++l) {
        al.v[l] = alpha[l];
        be.v[l] = beta[l];
        if (beta[l] != 0.0) overwrite = 0;
    }
    dim3 gc((unsigned)((m + 127) / 128), (unsigned)n);
    oz_accum_kernel<N><<<gc, 128, 0, s>>>(m, n, S, I, p.ldi, p.plane, rowexp, colexp, C, al, be,
                                          overwrite);
    phase(3, s);
    return record_cuda_error(cudaGetLastError(), "ozaki accumulate");
}

// data-independent slice count: N limbs, the reduction length and a 2^24
// margin for the ratio between the row/column scales and sum |a||b|
int ozaki_default_slices(int N, int64_t k) {
    int lk = 0;
    while ((1LL << lk) < k) ++lk;
    return (53 * N + 1 + lk + 24 + 6) / 7;
}

// largest slice count whose level sums stay exact in int32
int ozaki_max_slices(int64_t k) {
    const double kp = (double)((k + 127) / 128 * 128);
    int smax = (int)(2147483647.0 / (kp * 65.0 * 65.0));
    if (smax * kp * 65.0 * 65.0 >= 2147483647.0) --smax;
    return smax < 64 ? smax : 64;
}

// Slice-count tuner: enough 7-bit digits to reach the working precision of
// N limbs (53 N + 1 bits) beyond the largest sampled scale gap, plus a 6-bit
// margin for entries the sample missed.
static int tuned_slices(int N, int gap8) {
    const double gap = gap8 > 0 ? gap8 / 8.0 : 0.0;
    return (int)ceil((53.0 * N + 1.0 + gap + 6.0) / 7.0);
}

static const int OZ_SAMPLES = 2048;

// Row / column scale exponents of A and B into the handle's aux scratch
// (rowexp[m], colexp[n]); with tune != 0 also the sampled scale gap in
// eighths of a bit (*gap8_host, one synchronisation).
int ozaki_scales(mflab_handle *h, int N, int64_t m, int64_t n, int64_t k, Mat A, Mat B,
                 cudaStream_t s, int tune, int *gap8_host, int **rowexp_out, int **colexp_out) {
    int rc = mflab_reserve_aux(h, sizeof(int) * (size_t)(m + n + 64));
    if (rc) return rc;
    int *rowexp = (int *)h->aux;
    int *colexp = rowexp + m;
    int *gap8 = colexp + n;
    switch (N) {
    case 2: rc = oz_exponents<2>(m, n, k, A, B, rowexp, colexp, s); break;
    case 3: rc = oz_exponents<3>(m, n, k, A, B, rowexp, colexp, s); break;
    case 4: rc = oz_exponents<4>(m, n, k, A, B, rowexp, colexp, s); break;
    default: return MFLAB_ERR_UNSUPPORTED;
    }
    if (rc) return rc;
    *rowexp_out = rowexp;
    *colexp_out = colexp;
    if (tune) {
        cudaError_t e = cudaMemsetAsync(gap8, 0, sizeof(int), s);
        if (e != cudaSuccess) return record_cuda_error(e, "ozaki tune");
        oz_gap_kernel<false, false><<<(OZ_SAMPLES + 7) / 8, 256, 0, s>>>(
            m, n, k, A, B, rowexp, colexp, OZ_SAMPLES, gap8);
        int g = 0;
        e = cudaMemcpyAsync(&g, gap8, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return record_cuda_error(e, "ozaki tune read");
        *gap8_host = g;
    }
    return MFLAB_OK;
}

// Scales of a Gram product lower(A A^T) (trans = 0, A n x k) or lower(A^T A)
// (trans = 1, A k x n): one exponent per row of the left factor, which is
// also the column exponent of the right one (*exps[n] in the aux scratch);
// tune != 0 returns the sampled scale gap (one stream synchronisation).
int ozaki_gram_scales(mflab_handle *h, int N, int trans, int64_t n, int64_t k, Mat A,
                      cudaStream_t s, int tune, int *gap8_host, int **exps_out) {
    int rc = mflab_reserve_aux(h, sizeof(int) * (size_t)(n + 64));
    if (rc) return rc;
    int *exps = (int *)h->aux;
    int *gap8 = exps + n;
    if (trans == 0) {
        switch (N) {
        case 2: rc = oz_exponents<2>(n, 0, k, A, A, exps, exps + n, s); break;
        case 3: rc = oz_exponents<3>(n, 0, k, A, A, exps, exps + n, s); break;
        case 4: rc = oz_exponents<4>(n, 0, k, A, A, exps, exps + n, s); break;
        default: return MFLAB_ERR_UNSUPPORTED;
        }
    } else {
        switch (N) {
        case 2: oz_col_exp_kernel<2><<<(unsigned)((n + 7) / 8), 256, 0, s>>>(k, n, A, exps); break;
        case 3: oz_col_exp_kernel<3><<<(unsigned)((n + 7) / 8), 256, 0, s>>>(k, n, A, exps); break;
        case 4: oz_col_exp_kernel<4><<<(unsigned)((n + 7) / 8), 256, 0, s>>>(k, n, A, exps); break;
        default: return MFLAB_ERR_UNSUPPORTED;
        }
        rc = record_cuda_error(cudaGetLastError(), "ozaki gram exponents");
    }
    if (rc) return rc;
    *exps_out = exps;
    if (tune) {
        cudaError_t e = cudaMemsetAsync(gap8, 0, sizeof(int), s);
        if (e != cudaSuccess) return record_cuda_error(e, "ozaki gram tune");
        const unsigned g = (OZ_SAMPLES + 7) / 8;
        if (trans == 0)  // left A (n x k), right A^T given as A
            oz_gap_kernel<false, true><<<g, 256, 0, s>>>(n, n, k, A, A, exps, exps, OZ_SAMPLES, gap8);
        else             // left A^T given as A (k x n), right A
            oz_gap_kernel<true, false><<<g, 256, 0, s>>>(n, n, k, A, A, exps, exps, OZ_SAMPLES, gap8);
        int gv = 0;
        e = cudaMemcpyAsync(&gv, gap8, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return record_cuda_error(e, "ozaki gram tune read");
        *gap8_host = gv;
    }
    return MFLAB_OK;
}

int ozaki_gemm(mflab_handle *h, int N, int S, int64_t m, int64_t n, int64_t k, Mat A, Mat B,
               Mat C, const double *alpha, const double *beta, cudaStream_t s, int *S_used) {
    if (S < 0 || S > 64) return MFLAB_ERR_ARG;
    if ((n + 255) / 256 * 256 > 65535LL || m > INT_MAX) return MFLAB_ERR_UNSUPPORTED;
    int *rowexp = nullptr, *colexp = nullptr;
    int g = 0;
    int rc = ozaki_scales(h, N, m, n, k, A, B, s, S == 0, &g, &rowexp, &colexp);
    if (rc) return rc;
    if (S == 0) S = tuned_slices(N, g);
    const int smax = ozaki_max_slices(k);
    if (S > smax) S = smax;
    if (S < 1) return MFLAB_ERR_UNSUPPORTED;
    if (S_used) *S_used = S;
    const OzPlan p = oz_plan(m, n, k, S);
    rc = mflab_reserve_scratch(h, p.total);
    if (rc) return rc;
    char *base = (char *)h->scratch;
    int *tc_err = h->dev_flags + 1;
    switch (N) {
    case 2: return ozaki_n<2>(m, n, k, A, B, C, alpha, beta, S, base, p, rowexp, colexp, s, h->int8_engine, tc_err, tc_opts(h));
    case 3: return ozaki_n<3>(m, n, k, A, B, C, alpha, beta, S, base, p, rowexp, colexp, s, h->int8_engine, tc_err, tc_opts(h));
    default: return ozaki_n<4>(m, n, k, A, B, C, alpha, beta, S, base, p, rowexp, colexp, s, h->int8_engine, tc_err, tc_opts(h));
    }
}

}  // namespace mfl

extern "C" int mflab_gemm_ozaki_route(mflab_handle *h, void *stream, int limbs, int64_t m,
                                      int64_t n, int64_t k, const double *A, int64_t lda,
                                      int64_t lsa, const double *B, int64_t ldb, int64_t lsb,
                                      double *C, int64_t ldc, int64_t lsc, const double *alpha,
                                      const double *beta) {
    MFLAB_RANGE("mflab_gemm_ozaki_route");
    // the modular route first; the slice route when the modulus table cannot
    // reach the tuned requirement
    const mfl::Mat Am{(double *)A, lda, lsa}, Bm{(double *)B, ldb, lsb}, Cm{C, ldc, lsc};
    cudaStream_t s = (cudaStream_t)stream;
    if (k == 0) return mfl::launch_mm(limbs, false, false, 0, false, m, n, k, Am, Bm, Cm, alpha, beta, s);
    int rc = mfl::ozaki_crt_gemm(h, limbs, 0, m, n, k, Am, Bm, Cm, alpha, beta, s, &h->last_moduli);
    if (rc != MFLAB_ERR_UNSUPPORTED) return rc;
    return mfl::ozaki_gemm(h, limbs, 0, m, n, k, Am, Bm, Cm, alpha, beta, s, &h->last_slices);
}

extern "C" int mflab_gemm_ozaki(mflab_handle *h, void *stream, int limbs, int slices, int64_t m,
                                int64_t n, int64_t k, const double *A, int64_t lda, int64_t lsa,
                                const double *B, int64_t ldb, int64_t lsb, double *C, int64_t ldc,
                                int64_t lsc, const double *alpha, const double *beta) {
    MFLAB_RANGE("mflab_gemm_ozaki");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (m < 0 || n < 0 || k < 0 || !alpha || !beta) return MFLAB_ERR_ARG;
    if (m == 0 || n == 0) return MFLAB_OK;
    if (lda < (m > 0 ? m : 1) || ldb < (k > 0 ? k : 1) || ldc < m) return MFLAB_ERR_ARG;
    if (mfl::views_overlap(C, ldc, lsc, m, n, limbs, A, lda, lsa, m, k) ||
        mfl::views_overlap(C, ldc, lsc, m, n, limbs, B, ldb, lsb, k, n))
        return MFLAB_ERR_ALIAS;
    if (slices < 0) return MFLAB_ERR_ARG;
    if (k == 0)
        return mfl::launch_mm(limbs, false, false, 0, false, m, n, k,
                              mfl::Mat{(double *)A, lda, lsa}, mfl::Mat{(double *)B, ldb, lsb},
                              mfl::Mat{C, ldc, lsc}, alpha, beta, (cudaStream_t)stream);
    return mfl::ozaki_gemm(h, limbs, slices, m, n, k, mfl::Mat{(double *)A, lda, lsa},
                           mfl::Mat{(double *)B, ldb, lsb}, mfl::Mat{C, ldc, lsc}, alpha, beta,
                           (cudaStream_t)stream, &h->last_slices);
}

extern "C" int mflab_ozaki_last_slices(mflab_handle *h) { return h ? h->last_slices : 0; }

extern "C" int mflab_ozaki_default_slices(int limbs, int64_t k) {
    return mfl::ozaki_default_slices(limbs, k);
}

// ------------------------------------------------------ measurement -------
// mflab_gemm_ozaki with per-phase device times: ms[0] exponents + tuning,
// ms[1] digit split, ms[2] int8 level GEMMs, ms[3] accumulation; *int8_ops
// receives the integer multiply-add operations (2 m n K summed over levels).
// Synchronises the stream.
extern "C" int mflab_gemm_ozaki_phases(mflab_handle *h, void *stream, int limbs, int slices,
                                       int64_t m, int64_t n, int64_t k, const double *A,
                                       int64_t lda, int64_t lsa, const double *B, int64_t ldb,
                                       int64_t lsb, double *C, int64_t ldc, int64_t lsc,
                                       const double *alpha, const double *beta, float *ms,
                                       double *int8_ops) {
    MFLAB_RANGE("mflab_gemm_ozaki_phases");
    if (!h || !ms || !int8_ops) return MFLAB_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t ev[5];
    for (auto &e : ev) cudaEventCreate(&e);
    cudaEventRecord(ev[4], s);
    mfl::g_phase_ev = ev;
    int rc = mflab_gemm_ozaki(h, stream, limbs, slices, m, n, k, A, lda, lsa, B, ldb, lsb, C, ldc,
                              lsc, alpha, beta);
    mfl::g_phase_ev = nullptr;
    if (rc == MFLAB_OK) {
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = mfl::record_cuda_error(e, "ozaki phases");
    }
    if (rc == MFLAB_OK) {
        cudaEventElapsedTime(&ms[0], ev[4], ev[0]);
        cudaEventElapsedTime(&ms[1], ev[0], ev[1]);
        cudaEventElapsedTime(&ms[2], ev[1], ev[2]);
        cudaEventElapsedTime(&ms[3], ev[2], ev[3]);
        const int S = h->last_slices;
        const double kp = (double)((k + 127) / 128 * 128);
        const double mp = (double)((m + 127) / 128 * 128), np = (double)((n + 255) / 256 * 256);
        *int8_ops = 2.0 * mp * np * kp * (double)S * (S + 1) / 2.0;
    }
    for (auto &e : ev) cudaEventDestroy(e);
    return rc;
}

// Device time of one int8 x int8 -> int32 TN GEMM (m x n x k) through the same
// library path as the level products, after one warm-up call; *ms receives
// the best of `reps` timed calls.  Uses the handle scratch.  Synchronises.
namespace mfl {
// uniformly distributed bytes from a counter hash (splitmix64 finaliser)
__global__ void fill_random_bytes_kernel(uint64_t *p, size_t words, uint64_t seed) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < words;
         i += (size_t)gridDim.x * blockDim.x) {
        uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ULL;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        p[i] = z ^ (z >> 31);
    }
}
}  // namespace mfl

extern "C" int mflab_probe_int8_gemm(mflab_handle *h, void *stream, int64_t m, int64_t n,
                                     int64_t k, int reps, int fill, float *ms) {
    MFLAB_RANGE("mflab_probe_int8_gemm");
    if (!h || !ms || m <= 0 || n <= 0 || k <= 0 || reps <= 0) return MFLAB_ERR_ARG;
    if (fill != 0 && fill != 1) return MFLAB_ERR_FLAG;
    const int64_t kp = (k + 15) / 16 * 16, ldi = (m + 15) / 16 * 16;
    const size_t a = (size_t)m * kp, b = (size_t)n * kp, c = (size_t)ldi * n * 4, ws = 64 << 20;
    int rc = mflab_reserve_scratch(h, a + b + c + ws + 1024);
    if (rc) return rc;
    char *base = (char *)h->scratch;
    int8_t *A8 = (int8_t *)base, *B8 = (int8_t *)(base + (a + 255) / 256 * 256);
    int32_t *I = (int32_t *)(base + (a + 255) / 256 * 256 + (b + 255) / 256 * 256);
    char *wsp = (char *)I + (c + 255) / 256 * 256;
    cudaStream_t s = (cudaStream_t)stream;
    if (fill == 0) {
        cudaMemsetAsync(A8, 0x11, a, s);
        cudaMemsetAsync(B8, 0x23, b, s);
    } else {  // the operand bytes of the INT8 routes are close to uniform
        mfl::fill_random_bytes_kernel<<<1184, 256, 0, s>>>((uint64_t *)A8, a / 8, 1);
        mfl::fill_random_bytes_kernel<<<1184, 256, 0, s>>>((uint64_t *)B8, b / 8, 2);
    }
    rc = mfl::int8_gemm_tn(m, n, kp, A8, kp, B8, kp, I, ldi, wsp, ws, s);
    if (rc) return rc;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int r = 0; r < reps && rc == MFLAB_OK; ++r) {
        cudaEventRecord(e0, s);
        rc = mfl::int8_gemm_tn(m, n, kp, A8, kp, B8, kp, I, ldi, wsp, ws, s);
        cudaEventRecord(e1, s);
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) rc = mfl::record_cuda_error(e, "int8 probe");
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        if (t < best) best = t;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = best;
    return rc;
}

extern "C" int mflab_set_int8_engine(mflab_handle *h, int engine) {
    if (!h) return MFLAB_ERR_ARG;
    if (engine != MFLAB_INT8_TCGEN05 && engine != MFLAB_INT8_LIBRARY &&
        engine != MFLAB_INT8_TCGEN05_PAIR)
        return MFLAB_ERR_FLAG;
    h->int8_engine = engine;
    return MFLAB_OK;
}

extern "C" int mflab_device_status(mflab_handle *h, int *status) {
    if (!h || !status) return MFLAB_ERR_ARG;
    int v = 0;
    cudaError_t e = cudaMemcpy(&v, h->dev_flags + 1, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && v != 0) e = cudaMemset(h->dev_flags + 1, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return mfl::record_cuda_error(e, "device status");
    *status = v;
    return MFLAB_OK;
}
