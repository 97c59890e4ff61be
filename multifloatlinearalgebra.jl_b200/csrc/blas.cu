// Matched-order multi-double GEMM / SYRK / GEMMT on the FP64 pipe.
//
// Reduction-order contract (src/kernels/gemm.jl:138-265, syrk.jl:1-50,
// gemmt.jl:1-52 of MultiFloatLinearAlgebra.jl): every output element is ONE
// serial chain acc = 0; for k ascending: acc = acc + a(i,k)*b(k,j), followed
// by alpha*acc (beta == 0: C is never read) or alpha*acc + beta*C.  No split-k
// and no tree reduction, so with the same scalar networks the result is
// bitwise the reference's.
//
// Mapping: a CTA owns a BM x BN output tile; each thread owns TM x TN outputs
// strided by the thread grid so shared-memory reads are conflict-free
// broadcasts.  k-slabs of BK columns of every limb plane are staged in shared
// memory with cp.async into a double buffer while the previous slab is
// consumed.  The kernel is FP64-issue bound: per k step a thread reads
// (TM + TN)*N doubles and executes TM*TN*ops(N) FP64 instructions.
#include "mf_device.cuh"
#include "mflab_internal.h"

MFLAB_DEBUG_RECORD(blas)

namespace mfl {

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool pred) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    int src_size = pred ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem),
                 "r"(src_size)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int n>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(n) : "memory");
}

template <int N, int BM, int BN, int BK, int TM, int TN>
struct MMShape {
    static constexpr int TX = BM / TM;
    static constexpr int TY = BN / TN;
    static constexpr int NT = TX * TY;
    static constexpr size_t smem_bytes = sizeof(double) * 2 * N * BK * (BM + BN);
};

// TA: 0 a(i,k) = A[i,k]; 1 a(i,k) = A[k,i]; 2 symmetric from the lower
// triangle (k <= i ? A[i,k] : A[k,i]); 3 symmetric from the upper triangle.
// mode bits: MM_PACKED C is a packed lower triangle (column-major
// (0,0),(1,0)..(n-1,0),(1,1)..), limb stride C.ls; with TRMM the chain of
// C(i,j) runs over k <= idx (or k >= idx with MM_KGE), idx = i (or j with
// MM_RIGHT), and with MM_UNIT its diagonal term k == idx adds the other
// operand's entry instead of a product (trmm.jl:1-80).
template <int N, int BM, int BN, int BK, int TM, int TN, int TA, bool TB, bool TRI, bool FUSED,
          bool TRMM>
__global__ void __launch_bounds__(MMShape<N, BM, BN, BK, TM, TN>::NT)
    mm_kernel(int64_t m, int64_t n, int64_t K, Mat A, Mat B, Mat C, scal<N> alpha, scal<N> beta,
              int overwrite, const int *info, int mode) {
    using S = MMShape<N, BM, BN, BK, TM, TN>;
    constexpr int NT = S::NT, TX = S::TX, TY = S::TY;
    // a kernel launched after this one as a programmatic dependent (the
    // blocked Cholesky's next step) may be placed now; it waits for this
    // grid's completion before reading (no effect otherwise)
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    extern __shared__ double smem[];
    double *As = smem;                   // [2][N][BK][BM]
    double *Bs = smem + 2 * N * BK * BM;  // [2][N][BK][BN]
    const int tid = threadIdx.x;
    const int tx = tid % TX, ty = tid / TX;
    const int64_t row0 = (int64_t)blockIdx.x * BM, col0 = (int64_t)blockIdx.y * BN;
    if (TRI && row0 + BM - 1 < col0) return;  // tile strictly above the diagonal
    // debug builds: C's column stride holds its rows
    if (!(mode & MM_PACKED) && !MFLAB_IDX_OK(C.ld >= m, 6, C.ld, m)) return;
    if (info && *info) return;                 // an earlier factorization step failed
    // reduction range of this tile: all of K, or the triangular part TRMM needs
    int64_t kbeg = 0, kend = K;
    if (TRMM) {
        const bool right = mode & MM_RIGHT;
        const int64_t lo = right ? col0 : row0, hi = right ? col0 + BN : row0 + BM;
        if (mode & MM_KGE) kbeg = lo < K ? lo : K;
        else kend = hi < K ? hi : K;
    }

    mf<N> acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = from_double<N>(0.0);

    auto load_tile = [&](int buf, int64_t k0) {
        for (int e = tid; e < BM * BK; e += NT) {
            int i, kk;
            if (TA != 1) {
                i = e % BM;
                kk = e / BM;
            } else {
                kk = e % BK;
                i = e / BK;
            }
            int64_t gi = row0 + i, gk = k0 + kk;
            bool ok = gi < m && gk < kend;
            bool tr = TA == 1 || (TA == 2 && gk > gi) || (TA == 3 && gk < gi);
            const double *src = ok ? (tr ? A.p + gi * A.ld + gk : A.p + gk * A.ld + gi) : A.p;
#pragma unroll
            for (int l = 0; l < N; ++l)
                cp_async8(&As[((buf * N + l) * BK + kk) * BM + i], src + (ok ? l * A.ls : 0), ok);
        }
        for (int e = tid; e < BN * BK; e += NT) {
            int j, kk;
            if (!TB) {
                kk = e % BK;
                j = e / BK;
            } else {
                j = e % BN;
                kk = e / BN;
            }
            int64_t gj = col0 + j, gk = k0 + kk;
            bool ok = gj < n && gk < kend;
            const double *src = ok ? (TB ? B.p + gk * B.ld + gj : B.p + gj * B.ld + gk) : B.p;
#pragma unroll
            for (int l = 0; l < N; ++l)
                cp_async8(&Bs[((buf * N + l) * BK + kk) * BN + j], src + (ok ? l * B.ls : 0), ok);
        }
    };

    auto step = [&](int buf, int kk, int64_t gk) {
        mf<N> a[TM], b[TN];
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int l = 0; l < N; ++l) a[i].v[l] = As[((buf * N + l) * BK + kk) * BM + tx + i * TX];
#pragma unroll
        for (int j = 0; j < TN; ++j)
#pragma unroll
            for (int l = 0; l < N; ++l) b[j].v[l] = Bs[((buf * N + l) * BK + kk) * BN + ty + j * TY];
        if constexpr (!TRMM) {
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) acc[i][j] = mac<N, FUSED>(acc[i][j], a[i], b[j]);
        } else {
            const bool right = mode & MM_RIGHT, kge = mode & MM_KGE, unit = mode & MM_UNIT;
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) {
                    const int64_t idx = right ? col0 + ty + j * TY : row0 + tx + i * TX;
                    if (gk == idx) {
                        if (unit) acc[i][j] = add(acc[i][j], right ? a[i] : b[j]);
                        else acc[i][j] = mac<N, false>(acc[i][j], a[i], b[j]);
                    } else if (kge ? gk > idx : gk < idx) {
                        acc[i][j] = mac<N, false>(acc[i][j], a[i], b[j]);
                    }
                }
        }
    };

    const int64_t nk = kend > kbeg ? (kend - kbeg + BK - 1) / BK : 0;
    if (nk > 0) {
        load_tile(0, kbeg);
        cp_async_commit();
    }
    for (int64_t kt = 0; kt < nk; ++kt) {
        const int buf = (int)(kt & 1);
        const int64_t k0 = kbeg + kt * BK;
        if (kt + 1 < nk) load_tile(buf ^ 1, k0 + BK);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const int64_t rem = kend - k0;
        if (rem >= BK) {
#pragma unroll 2
            for (int kk = 0; kk < BK; ++kk) step(buf, kk, k0 + kk);
        } else {
            for (int kk = 0; kk < (int)rem; ++kk) step(buf, kk, k0 + kk);
        }
        __syncthreads();
    }

    const mf<N> al = alpha.get(), be = beta.get();
#pragma unroll
    for (int i = 0; i < TM; ++i) {
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int64_t gi = row0 + tx + i * TX, gj = col0 + ty + j * TY;
            if (gi < m && gj < n && (!TRI || gi >= gj)) {
                mf<N> r = mul(al, acc[i][j]);
                if (mode & MM_PACKED) {
                    double *c = C.p + gj * (2 * n - gj + 1) / 2 + (gi - gj);
                    if (!overwrite) {
                        mf<N> old;
#pragma unroll
                        for (int l = 0; l < N; ++l) old.v[l] = c[l * C.ls];
                        r = add(r, mul(be, old));
                    }
#pragma unroll
                    for (int l = 0; l < N; ++l) c[l * C.ls] = r.v[l];
                } else {
                    if (!overwrite) r = add(r, mul(be, load_mf<N>(C.p, C.ld, C.ls, gi, gj)));
                    store_mf<N>(C.p, C.ld, C.ls, gi, gj, r);
                }
            }
        }
    }
}

template <int N, int BM, int BN, int BK, int TM, int TN, int TA, bool TB, bool TRI, bool FUSED,
          bool TRMM>
static int run_mm(int64_t m, int64_t n, int64_t k, Mat A, Mat B, Mat C, const double *alpha,
                  const double *beta, cudaStream_t s, const int *info, int mode) {
    using S = MMShape<N, BM, BN, BK, TM, TN>;
    auto kern = mm_kernel<N, BM, BN, BK, TM, TN, TA, TB, TRI, FUSED, TRMM>;
    static std::atomic<unsigned long long> configured{0};
    if (int rc = set_smem_once((const void *)kern, (int)S::smem_bytes, configured,
                               "mm_kernel attribute"))
        return rc;
    scal<N> al{}, be{};
    int overwrite = 1;
    for (int l = 0; l < N; ++l) {
        al.v[l] = alpha[l];
        be.v[l] = beta[l];
        if (beta[l] != 0.0) overwrite = 0;
    }
    if (m <= 0 || n <= 0) return MFLAB_OK;
    dim3 grid((unsigned)((m + BM - 1) / BM), (unsigned)((n + BN - 1) / BN));
    if (grid.y > 65535) return MFLAB_ERR_UNSUPPORTED;
    kern<<<grid, S::NT, S::smem_bytes, s>>>(m, n, k, A, B, C, al, be, overwrite, info, mode);
    return record_cuda_error(cudaGetLastError(), "mm_kernel launch");
}

// tile shapes per limb count (FP64-issue bound; registers: TM*TN*N accumulators).
// Products at most 16 columns wide (a blocked factorization's next block
// columns, a few right-hand sides) take 32 x 16 tiles of two outputs per
// thread: a 64 x 64 tile would leave three quarters of its threads idle and
// put the whole product on a few CTAs.  Every output is the same chain in
// either shape.
template <int N, int TA, bool TB, bool TRI, bool FUSED, bool TRMM = false>
static int run_mm_n(int64_t m, int64_t n, int64_t k, Mat A, Mat B, Mat C, const double *alpha,
                    const double *beta, cudaStream_t s, const int *info, int mode) {
    if constexpr (N >= 2 && !FUSED && !TRMM) {
        if (n <= 16)
            return run_mm<N, 32, 16, (N == 2 ? 16 : 8), 2, 1, TA, TB, TRI, FUSED, TRMM>(
                m, n, k, A, B, C, alpha, beta, s, info, mode);
    }
    if constexpr (N == 1)
        return run_mm<1, 64, 64, 16, 4, 4, TA, TB, TRI, FUSED, TRMM>(m, n, k, A, B, C, alpha, beta, s, info, mode);
    else if constexpr (N == 2)
        return run_mm<2, 64, 64, 16, 4, 4, TA, TB, TRI, FUSED, TRMM>(m, n, k, A, B, C, alpha, beta, s, info, mode);
    else if constexpr (N == 3)
        return run_mm<3, 64, 64, 8, 4, 4, TA, TB, TRI, FUSED, TRMM>(m, n, k, A, B, C, alpha, beta, s, info, mode);
    else
        return run_mm<4, 64, 32, 8, 4, 2, TA, TB, TRI, FUSED, TRMM>(m, n, k, A, B, C, alpha, beta, s, info, mode);
}

template <int N>
static int dispatch_mm(int ta, bool tb, int tri, bool fused3, int64_t m, int64_t n, int64_t k,
                       Mat A, Mat B, Mat C, const double *alpha, const double *beta,
                       cudaStream_t s, const int *info, int mode) {
    if (ta == 0 && !tb && !tri) {
        if (N == 3 && fused3)
            return run_mm_n<N, 0, false, false, true>(m, n, k, A, B, C, alpha, beta, s, info, mode);
        return run_mm_n<N, 0, false, false, false>(m, n, k, A, B, C, alpha, beta, s, info, mode);
    }
    if (ta == 1 && !tb && tri) return run_mm_n<N, 1, false, true, false>(m, n, k, A, B, C, alpha, beta, s, info, mode);
    if (ta == 1 && !tb && !tri) return run_mm_n<N, 1, false, false, false>(m, n, k, A, B, C, alpha, beta, s, info, mode);
    if (ta == 0 && tb && tri) return run_mm_n<N, 0, true, true, false>(m, n, k, A, B, C, alpha, beta, s, info, mode);
    if (ta == 2 && !tb && !tri) return run_mm_n<N, 2, false, false, false>(m, n, k, A, B, C, alpha, beta, s, info, mode);
    if (ta == 3 && !tb && !tri) return run_mm_n<N, 3, false, false, false>(m, n, k, A, B, C, alpha, beta, s, info, mode);
    return MFLAB_ERR_UNSUPPORTED;
}

int launch_mm(int N, int ta, bool tb, int tri, bool fused3, int64_t m, int64_t n, int64_t k,
              Mat A, Mat B, Mat C, const double *alpha, const double *beta, cudaStream_t s,
              const int *info, int mode) {
    switch (N) {
    case 1:
        if (ta == 0 && !tb && !tri)
            return run_mm_n<1, 0, false, false, false>(m, n, k, A, B, C, alpha, beta, s, info, mode);
        return MFLAB_ERR_UNSUPPORTED;
    case 2: return dispatch_mm<2>(ta, tb, tri, fused3, m, n, k, A, B, C, alpha, beta, s, info, mode);
    case 3: return dispatch_mm<3>(ta, tb, tri, fused3, m, n, k, A, B, C, alpha, beta, s, info, mode);
    case 4: return dispatch_mm<4>(ta, tb, tri, fused3, m, n, k, A, B, C, alpha, beta, s, info, mode);
    default: return MFLAB_ERR_UNSUPPORTED;
    }
}

// C = alpha * a * b with the triangular chain of the mode bits (beta = 0):
// left products a = op(A) (ta 0/1), b = the saved B; right products a = the
// saved B, b = op(A) (tb 0/1).
template <int N>
static int dispatch_trmm(int ta, bool tb, int64_t m, int64_t n, int64_t k, Mat A, Mat B, Mat C,
                         const double *alpha, const double *zero, cudaStream_t s, int mode) {
    if (ta == 0 && !tb) return run_mm_n<N, 0, false, false, false, true>(m, n, k, A, B, C, alpha, zero, s, nullptr, mode);
    if (ta == 1 && !tb) return run_mm_n<N, 1, false, false, false, true>(m, n, k, A, B, C, alpha, zero, s, nullptr, mode);
    if (ta == 0 && tb) return run_mm_n<N, 0, true, false, false, true>(m, n, k, A, B, C, alpha, zero, s, nullptr, mode);
    return MFLAB_ERR_UNSUPPORTED;
}

int launch_trmm_mm(int N, int ta, bool tb, int mode, int64_t m, int64_t n, int64_t k, Mat A, Mat B,
                   Mat C, const double *alpha, cudaStream_t s) {
    const double zero[4] = {0.0, 0.0, 0.0, 0.0};
    switch (N) {
    case 2: return dispatch_trmm<2>(ta, tb, m, n, k, A, B, C, alpha, zero, s, mode);
    case 3: return dispatch_trmm<3>(ta, tb, m, n, k, A, B, C, alpha, zero, s, mode);
    case 4: return dispatch_trmm<4>(ta, tb, m, n, k, A, B, C, alpha, zero, s, mode);
    default: return MFLAB_ERR_UNSUPPORTED;
    }
}

}  // namespace mfl

using mfl::Mat;

extern "C" int mflab_gemm(mflab_handle *h, void *stream, int limbs, int route, int64_t m,
                          int64_t n, int64_t k, const double *A, int64_t lda, int64_t lsa,
                          const double *B, int64_t ldb, int64_t lsb, double *C, int64_t ldc,
                          int64_t lsc, const double *alpha, const double *beta);

extern "C" int mflab_gemm_ozaki_route(mflab_handle *h, void *stream, int limbs, int64_t m,
                                      int64_t n, int64_t k, const double *A, int64_t lda,
                                      int64_t lsa, const double *B, int64_t ldb, int64_t lsb,
                                      double *C, int64_t ldc, int64_t lsc, const double *alpha,
                                      const double *beta);

extern "C" int mflab_gemm(mflab_handle *h, void *stream, int limbs, int route, int64_t m,
                          int64_t n, int64_t k, const double *A, int64_t lda, int64_t lsa,
                          const double *B, int64_t ldb, int64_t lsb, double *C, int64_t ldc,
                          int64_t lsc, const double *alpha, const double *beta) {
    MFLAB_RANGE("mflab_gemm");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (m < 0 || n < 0 || k < 0 || !alpha || !beta) return MFLAB_ERR_ARG;
    if (m == 0 || n == 0) return MFLAB_OK;
    if (lda < (m > 0 ? m : 1) || ldb < (k > 0 ? k : 1) || ldc < m) return MFLAB_ERR_ARG;
    if (mfl::views_overlap(C, ldc, lsc, m, n, limbs, A, lda, lsa, m, k) ||
        mfl::views_overlap(C, ldc, lsc, m, n, limbs, B, ldb, lsb, k, n))
        return MFLAB_ERR_ALIAS;
    cudaStream_t s = (cudaStream_t)stream;
    if (route == MFLAB_GEMM_OZAKI)
        return mflab_gemm_ozaki_route(h, stream, limbs, m, n, k, A, lda, lsa, B, ldb, lsb, C, ldc,
                                      lsc, alpha, beta);
    if (route != MFLAB_GEMM_AUTO && route != MFLAB_GEMM_DIRECT) return MFLAB_ERR_FLAG;
    bool fused = (limbs == 3 && route == MFLAB_GEMM_AUTO);
    return mfl::launch_mm(limbs, false, false, 0, fused, m, n, k, Mat{(double *)A, lda, lsa},
                          Mat{(double *)B, ldb, lsb}, Mat{C, ldc, lsc}, alpha, beta, s);
}

// y = alpha * op(A) x + beta * y (gemv.jl:1-167): one ascending chain per
// output (columns for trans = 0, rows for trans = 1), the plain network (no
// fused Float64x3 step), y unread when beta == 0; the GEMM kernel with one
// right-hand column.  x and y are contiguous vectors with limb strides lsx, lsy.
extern "C" int mflab_gemv(mflab_handle *h, void *stream, int limbs, int trans, int64_t m,
                          int64_t n, const double *A, int64_t lda, int64_t lsa, const double *x,
                          int64_t lsx, double *y, int64_t lsy, const double *alpha,
                          const double *beta) {
    MFLAB_RANGE("mflab_gemv");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (trans != 0 && trans != 1) return MFLAB_ERR_FLAG;
    if (m < 0 || n < 0 || !alpha || !beta) return MFLAB_ERR_ARG;
    if (m > 0 && lda < m) return MFLAB_ERR_ARG;
    const int64_t rows = trans ? n : m, len = trans ? m : n;
    if (rows == 0) return MFLAB_OK;
    if (mfl::views_overlap(y, rows, lsy, rows, 1, limbs, A, lda, lsa, m, n) ||
        mfl::views_overlap(y, rows, lsy, rows, 1, limbs, x, len > 0 ? len : 1, lsx, len, 1))
        return MFLAB_ERR_ALIAS;
    return mfl::launch_mm(limbs, trans, false, 0, false, rows, 1, len, Mat{(double *)A, lda, lsa},
                          Mat{(double *)x, len > 0 ? len : 1, lsx}, Mat{y, rows, lsy}, alpha, beta,
                          (cudaStream_t)stream);
}

// y = alpha * A x + beta * y with A symmetric, read only from its uplo
// triangle (symv.jl:1-89): row r's chain runs over ascending columns, taking
// A[r, c] from the authoritative triangle and A[c, r] across it.
extern "C" int mflab_symv(mflab_handle *h, void *stream, int limbs, int uplo, int64_t n,
                          const double *A, int64_t lda, int64_t lsa, const double *x, int64_t lsx,
                          double *y, int64_t lsy, const double *alpha, const double *beta) {
    MFLAB_RANGE("mflab_symv");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (uplo != 0 && uplo != 1) return MFLAB_ERR_FLAG;
    if (n < 0 || !alpha || !beta) return MFLAB_ERR_ARG;
    if (n == 0) return MFLAB_OK;
    if (lda < n) return MFLAB_ERR_ARG;
    if (mfl::views_overlap(y, n, lsy, n, 1, limbs, A, lda, lsa, n, n) ||
        mfl::views_overlap(y, n, lsy, n, 1, limbs, x, n, lsx, n, 1))
        return MFLAB_ERR_ALIAS;
    return mfl::launch_mm(limbs, 2 + uplo, false, 0, false, n, 1, n, Mat{(double *)A, lda, lsa},
                          Mat{(double *)x, n, lsx}, Mat{y, n, lsy}, alpha, beta,
                          (cudaStream_t)stream);
}

namespace mfl {
// sum over the column-major linear index of x .* y, one ascending chain
// (dot.jl:1-22) by one thread
template <int N>
__global__ void dot_kernel(int64_t m, int64_t n, Mat X, Mat Y, double *out) {
    mf<N> acc = from_double<N>(0.0);
    for (int64_t c = 0; c < n; ++c)
        for (int64_t r = 0; r < m; ++r)
            acc = add(acc, mul(load_mf<N>(X.p, X.ld, X.ls, r, c), load_mf<N>(Y.p, Y.ld, Y.ls, r, c)));
#pragma unroll
    for (int l = 0; l < N; ++l) out[l] = acc.v[l];
}
}  // namespace mfl

// out (device, limbs doubles) = mfdot(x, y) for two m x n arrays (vectors:
// n = 1), in ascending column-major order (dot.jl:1-22).  One serial chain,
// as the reference's.
extern "C" int mflab_dot(mflab_handle *h, void *stream, int limbs, int64_t m, int64_t n,
                         const double *x, int64_t ldx, int64_t lsx, const double *y, int64_t ldy,
                         int64_t lsy, double *out) {
    MFLAB_RANGE("mflab_dot");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (m < 0 || n < 0 || !out || (m > 0 && (ldx < m || ldy < m))) return MFLAB_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    Mat X{(double *)x, ldx, lsx}, Y{(double *)y, ldy, lsy};
    switch (limbs) {
    case 2: mfl::dot_kernel<2><<<1, 1, 0, s>>>(m, n, X, Y, out); break;
    case 3: mfl::dot_kernel<3><<<1, 1, 0, s>>>(m, n, X, Y, out); break;
    default: mfl::dot_kernel<4><<<1, 1, 0, s>>>(m, n, X, Y, out); break;
    }
    return mfl::record_cuda_error(cudaGetLastError(), "dot");
}

// packed lower(C) = alpha * P[k0:k1, :]^T P[k0:k1, :] + beta * packed lower(C)
// (syrk.jl:110-254): the SYRK chains over the reduction rows k0 .. k1-1, stored
// column-major packed, (0,0),(1,0)..(n-1,0),(1,1)..; limb stride lsc.
extern "C" int mflab_syrk_packed(mflab_handle *h, void *stream, int limbs, int64_t n, int64_t kp,
                                 int64_t k0, int64_t k1, const double *P, int64_t ldp, int64_t lsp,
                                 double *C, int64_t lsc, const double *alpha, const double *beta) {
    MFLAB_RANGE("mflab_syrk_packed");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (n < 0 || kp < 0 || !alpha || !beta) return MFLAB_ERR_ARG;
    if (!(0 <= k0 && k0 < k1 && k1 <= kp)) return MFLAB_ERR_ARG;
    if (n == 0) return MFLAB_OK;
    const int64_t len = n * (n + 1) / 2;
    if (ldp < kp || lsc < len) return MFLAB_ERR_ARG;
    if (mfl::views_overlap(C, len, lsc, len, 1, limbs, P, ldp, lsp, kp, n)) return MFLAB_ERR_ALIAS;
    return mfl::launch_mm(limbs, true, false, 1, false, n, n, k1 - k0,
                          Mat{(double *)P + k0, ldp, lsp}, Mat{(double *)P + k0, ldp, lsp},
                          Mat{C, len, lsc}, alpha, beta, (cudaStream_t)stream, nullptr,
                          mfl::MM_PACKED);
}

// B = alpha * op(A) * B (side 0) or alpha * B * op(A) (side 1), in place
// (trmm.jl:82-131).  Each B(i,j) is one ascending chain over the triangle of
// op(A) (trmm.jl:1-80): left lower k = 0..i, left upper k = i..m-1, right
// lower k = j..n-1, right upper k = 0..j, the diagonal term B(i,j) itself for
// diag = unit.  B is saved to the handle's scratch and the product written
// back, so every chain reads the original B.
extern "C" int mflab_trmm(mflab_handle *h, void *stream, int limbs, int side, int uplo, int trans,
                          int diag, int64_t m, int64_t n, const double *A, int64_t lda,
                          int64_t lsa, double *B, int64_t ldb, int64_t lsb, const double *alpha) {
    MFLAB_RANGE("mflab_trmm");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if ((side | uplo | trans | diag) & ~1) return MFLAB_ERR_FLAG;
    if (m < 0 || n < 0 || !alpha) return MFLAB_ERR_ARG;
    const int64_t na = side ? n : m;
    if (m == 0 || n == 0) return MFLAB_OK;
    if (lda < na || ldb < m) return MFLAB_ERR_ARG;
    if (mfl::views_overlap(B, ldb, lsb, m, n, limbs, A, lda, lsa, na, na)) return MFLAB_ERR_ALIAS;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t plane = (size_t)m * n;
    int rc = mflab_reserve_scratch(h, plane * limbs * sizeof(double));
    if (rc) return rc;
    double *saved = (double *)h->scratch;
    for (int l = 0; l < limbs; ++l) {
        cudaError_t e = cudaMemcpy2DAsync(saved + l * plane, m * sizeof(double), B + l * lsb,
                                          ldb * sizeof(double), m * sizeof(double), n,
                                          cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return mfl::record_cuda_error(e, "trmm save");
    }
    const Mat Bs{saved, m, (int64_t)plane}, Am{(double *)A, lda, lsa}, Bm{B, ldb, lsb};
    const bool eff_lower = (uplo == 0) == (trans == 0);
    const int unit = diag ? mfl::MM_UNIT : 0;
    if (side == 0)
        return mfl::launch_trmm_mm(limbs, trans, false, (eff_lower ? 0 : mfl::MM_KGE) | unit, m,
                                   n, m, Am, Bs, Bm, alpha, s);
    return mfl::launch_trmm_mm(limbs, 0, trans != 0,
                               mfl::MM_RIGHT | (eff_lower ? mfl::MM_KGE : 0) | unit, m, n, n, Bs,
                               Am, Bm, alpha, s);
}

extern "C" int mflab_syrk_lower(mflab_handle *h, void *stream, int limbs, int64_t n, int64_t k,
                                const double *P, int64_t ldp, int64_t lsp, double *C, int64_t ldc,
                                int64_t lsc, const double *alpha, const double *beta) {
    MFLAB_RANGE("mflab_syrk_lower");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (n < 0 || k < 0 || !alpha || !beta) return MFLAB_ERR_ARG;
    if (n == 0) return MFLAB_OK;
    if (ldp < (k > 0 ? k : 1) || ldc < n) return MFLAB_ERR_ARG;
    if (mfl::views_overlap(C, ldc, lsc, n, n, limbs, P, ldp, lsp, k, n)) return MFLAB_ERR_ALIAS;
    return mfl::launch_mm(limbs, true, false, 1, false, n, n, k, Mat{(double *)P, ldp, lsp},
                          Mat{(double *)P, ldp, lsp}, Mat{C, ldc, lsc}, alpha, beta,
                          (cudaStream_t)stream);
}

extern "C" int mflab_gemmt_lower(mflab_handle *h, void *stream, int limbs, int64_t n, int64_t k,
                                 const double *A, int64_t lda, int64_t lsa, const double *B,
                                 int64_t ldb, int64_t lsb, double *C, int64_t ldc, int64_t lsc,
                                 const double *alpha, const double *beta) {
    MFLAB_RANGE("mflab_gemmt_lower");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (n < 0 || k < 0 || !alpha || !beta) return MFLAB_ERR_ARG;
    if (n == 0) return MFLAB_OK;
    if (lda < n || ldb < n || ldc < n) return MFLAB_ERR_ARG;
    if (mfl::views_overlap(C, ldc, lsc, n, n, limbs, A, lda, lsa, n, k) ||
        mfl::views_overlap(C, ldc, lsc, n, n, limbs, B, ldb, lsb, n, k))
        return MFLAB_ERR_ALIAS;
    return mfl::launch_mm(limbs, false, true, 1, false, n, n, k, Mat{(double *)A, lda, lsa},
                          Mat{(double *)B, ldb, lsb}, Mat{C, ldc, lsc}, alpha, beta,
                          (cudaStream_t)stream);
}
