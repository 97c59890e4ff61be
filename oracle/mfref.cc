/*
 * mfref: CPU restatement of MultiFloatLinearAlgebra.jl's dense multi-double
 * hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the oracle: the test-suite, the
 * smoke check and the CPU-baseline leg of the benchmark call it to check and
 * time the CUDA product.  The product library never links or calls it.
 *
 * Storage: a Float64xN matrix is N column-major binary64 planes.  Limb l of
 * element (r, c) of a matrix P with leading dimension ld and limb stride ls is
 * P[l*ls + c*ld + r] (0-based r, c).
 *
 * Every routine restates the reference's loop order and scalar expressions so
 * that, with the same networks, results are bitwise those of the reference
 * (citations are paths inside the reference project):
 *   gemm        src/kernels/gemm.jl:138-303 (+ the x3 fused route :309-489)
 *   syrk_lower  src/kernels/syrk.jl:1-108
 *   gemmt_lower src/kernels/gemmt.jl:1-108
 *   trsm        src/kernels/trsm.jl:1-302;  trsv src/kernels/trsv.jl:19-73
 *   potrf       src/factorizations/cholesky.jl:10-107
 *   getrf       src/factorizations/lu.jl:34-195
 *   sytrf       src/factorizations/ldlt.jl:65-717, ldlt_gemmt.jl:1-73
 *   solves      src/solve.jl:23-365
 * Division, square root and reciprocal are MultiFloats.jl routines that the
 * reference does not contain; the ones here are a long division (N+1 quotient
 * digits) and two Heron iterations.  Parity for those is within tolerance.
 *
 * Compile with -ffp-contract=off and without -ffast-math.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

/* dynamic parallel-for over [0, n) on `threads` host threads */
template <class F>
static void par_for(int64_t n, int threads, F &&fn) {
    if (threads < 1) threads = 1;
    if (threads == 1 || n <= 1) {
        for (int64_t i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<int64_t> next(0);
    auto worker = [&]() {
        for (;;) {
            int64_t i = next.fetch_add(1);
            if (i >= n) break;
            fn(i);
        }
    };
    std::vector<std::thread> pool;
    int nt = (int64_t)threads < n ? threads : (int)n;
    for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto &th : pool) th.join();
}

extern "C" {

/* ------------------------------------------------------------ lanes ----- */
typedef double v4d __attribute__((vector_size(32), aligned(8)));

static inline v4d bcast(double x) { v4d r = {x, x, x, x}; return r; }
static inline v4d load4(const double *p) {
    v4d r;
    memcpy(&r, p, sizeof r);
    return r;
}
static inline void store4(double *p, v4d v) { memcpy(p, &v, sizeof v); }
static inline v4d fma4(v4d a, v4d b, v4d c) {
    v4d r;
    for (int i = 0; i < 4; ++i) r[i] = __builtin_fma(a[i], b[i], c[i]);
    return r;
}

#define R double
#define FMA(a, b, c) __builtin_fma((a), (b), (c))
#define NM(x) x##_s
#include "mfnet_body.inc"
#undef R
#undef FMA
#undef NM

#define R v4d
#define FMA(a, b, c) fma4((a), (b), (c))
#define NM(x) x##_v
#include "mfnet_body.inc"
#undef R
#undef FMA
#undef NM

/* ------------------------------------------------ scalar multi-double --- */
#define MAXN 4

static void mf_add(int N, const double *x, const double *y, double *z) {
    double t[MAXN];
    switch (N) {
    case 1: z[0] = x[0] + y[0]; return;
    case 2: add2_s(x, y, t); break;
    case 3: add3_s(x, y, t); break;
    default: add4_s(x, y, t); break;
    }
    memcpy(z, t, sizeof(double) * N);
}

static void mf_mul(int N, const double *x, const double *y, double *z) {
    double t[MAXN];
    switch (N) {
    case 1: z[0] = x[0] * y[0]; return;
    case 2: mul2_s(x, y, t); break;
    case 3: mul3_s(x, y, t); break;
    default: mul4_s(x, y, t); break;
    }
    memcpy(z, t, sizeof(double) * N);
}

static void mf_neg(int N, const double *x, double *z) {
    for (int l = 0; l < N; ++l) z[l] = -x[l];
}

static void mf_sub(int N, const double *x, const double *y, double *z) {
    double ny[MAXN];
    mf_neg(N, y, ny);
    mf_add(N, x, ny, z);
}

/* z = x - a*b, the reference's `x -= a * b` */
static void mf_submul(int N, const double *x, const double *a, const double *b, double *z) {
    double p[MAXN];
    mf_mul(N, a, b, p);
    mf_sub(N, x, p, z);
}

static void mf_set(int N, double v, double *z) {
    z[0] = v;
    for (int l = 1; l < N; ++l) z[l] = 0.0;
}

static int mf_iszero(int N, const double *x) {
    for (int l = 0; l < N; ++l)
        if (x[l] != 0.0) return 0;
    return 1;
}

static int mf_isfinite(int N, const double *x) {
    for (int l = 0; l < N; ++l)
        if (!isfinite(x[l])) return 0;
    return 1;
}

/* lexicographic limb order (exact value order for normalised values) */
static int mf_lt(int N, const double *x, const double *y) {
    for (int l = 0; l < N; ++l) {
        if (x[l] < y[l]) return 1;
        if (x[l] > y[l]) return 0;
    }
    return 0;
}
static int mf_gt(int N, const double *x, const double *y) { return mf_lt(N, y, x); }
static int mf_ge(int N, const double *x, const double *y) {
    for (int l = 0; l < N; ++l) {
        if (x[l] > y[l]) return 1;
        if (x[l] < y[l]) return 0;
        if (!(x[l] == y[l])) return 0; /* NaN */
    }
    return 1;
}

static void mf_abs(int N, const double *x, double *z) {
    if (signbit(x[0]))
        mf_neg(N, x, z);
    else
        memcpy(z, x, sizeof(double) * N);
}

/* Base.max(x, y) = isless(y, x) ? x : y */
static void mf_max(int N, const double *x, const double *y, double *z) {
    double t[MAXN];
    memcpy(t, mf_lt(N, y, x) ? x : y, sizeof(double) * N);
    memcpy(z, t, sizeof(double) * N);
}
static void mf_min(int N, const double *x, const double *y, double *z) {
    double t[MAXN];
    memcpy(t, mf_lt(N, y, x) ? y : x, sizeof(double) * N);
    memcpy(z, t, sizeof(double) * N);
}

/* long division: N+1 quotient digits q_i = r_0 / y_0, r <- r - y*q_i,
   summed from the top with the add network */
static void mf_div(int N, const double *x, const double *y, double *z) {
    if (N == 1) {
        z[0] = x[0] / y[0];
        return;
    }
    double r[MAXN], q[MAXN + 1], qi[MAXN], t[MAXN];
    memcpy(r, x, sizeof(double) * N);
    for (int i = 0; i <= N; ++i) {
        q[i] = r[0] / y[0];
        if (i < N) {
            mf_set(N, q[i], qi);
            mf_mul(N, y, qi, t);
            mf_sub(N, r, t, r);
        }
    }
    double acc[MAXN];
    mf_set(N, q[0], acc);
    for (int i = 1; i <= N; ++i) {
        mf_set(N, q[i], qi);
        mf_add(N, acc, qi, acc);
    }
    memcpy(z, acc, sizeof(double) * N);
}

static void mf_inv(int N, const double *x, double *z) {
    double one[MAXN];
    mf_set(N, 1.0, one);
    mf_div(N, one, x, z);
}

/* two Heron iterations s <- (s + x/s)/2 from the binary64 square root */
static void mf_sqrt(int N, const double *x, double *z) {
    if (x[0] == 0.0) {
        mf_set(N, 0.0, z);
        return;
    }
    double s[MAXN], t[MAXN];
    mf_set(N, sqrt(x[0]), s);
    if (N > 1) {
        for (int it = 0; it < 2; ++it) {
            mf_div(N, x, s, t);
            mf_add(N, s, t, s);
            for (int l = 0; l < N; ++l) s[l] *= 0.5;
        }
    }
    memcpy(z, s, sizeof(double) * N);
}

/* ------------------------------------------------- exported scalar ops -- */
void mfr_add(int N, const double *x, const double *y, double *z) { mf_add(N, x, y, z); }
void mfr_sub(int N, const double *x, const double *y, double *z) { mf_sub(N, x, y, z); }
void mfr_mul(int N, const double *x, const double *y, double *z) { mf_mul(N, x, y, z); }
void mfr_div(int N, const double *x, const double *y, double *z) { mf_div(N, x, y, z); }
void mfr_sqrt(int N, const double *x, double *z) { mf_sqrt(N, x, z); }
void mfr_inv(int N, const double *x, double *z) { mf_inv(N, x, z); }
void mfr_mulacc_x3(const double *acc, const double *x, const double *y, double *z) {
    double t[3];
    mulacc3_s(acc, x, y, t);
    memcpy(z, t, sizeof t);
}
/* elementwise over count values stored limb-major (limb stride ls) */
void mfr_add_n(int N, int64_t count, const double *x, const double *y, double *z, int64_t ls) {
    for (int64_t i = 0; i < count; ++i) {
        double a[MAXN], b[MAXN], c[MAXN];
        for (int l = 0; l < N; ++l) {
            a[l] = x[l * ls + i];
            b[l] = y[l * ls + i];
        }
        mf_add(N, a, b, c);
        for (int l = 0; l < N; ++l) z[l * ls + i] = c[l];
    }
}
void mfr_mul_n(int N, int64_t count, const double *x, const double *y, double *z, int64_t ls) {
    for (int64_t i = 0; i < count; ++i) {
        double a[MAXN], b[MAXN], c[MAXN];
        for (int l = 0; l < N; ++l) {
            a[l] = x[l * ls + i];
            b[l] = y[l * ls + i];
        }
        mf_mul(N, a, b, c);
        for (int l = 0; l < N; ++l) z[l * ls + i] = c[l];
    }
}

/* ------------------------------------------------------ element access -- */
#define EL(P, ld, ls, r, c, l) (P)[(int64_t)(l) * (ls) + (int64_t)(c) * (ld) + (r)]

static inline void getm(int N, const double *P, int64_t ld, int64_t ls, int64_t r, int64_t c,
                        double *out) {
    for (int l = 0; l < N; ++l) out[l] = EL(P, ld, ls, r, c, l);
}
static inline void putm(int N, double *P, int64_t ld, int64_t ls, int64_t r, int64_t c,
                        const double *v) {
    for (int l = 0; l < N; ++l) EL(P, ld, ls, r, c, l) = v[l];
}

/* ---------------------------------------------------------------- GEMM -- */
#define GEMM_FN_(s) gemm_cols_##s
#define GEMM_FN(s) GEMM_FN_(s)

/* N = 2 */
#define GN 2
#define GSUF 2
#define MAC_V(acc, a, b) do { v4d p_[2]; mul2_v(a, b, p_); add2_v(acc, p_, acc); } while (0)
#define MAC_S(acc, a, b) do { double p_[2]; mul2_s(a, b, p_); add2_s(acc, p_, acc); } while (0)
#define MULV mul2_v
#define ADDV add2_v
#define MULS mul2_s
#define ADDS add2_s
#include "gemm_body.inc"
#undef GN
#undef GSUF
#undef MAC_V
#undef MAC_S
#undef MULV
#undef ADDV
#undef MULS
#undef ADDS

/* N = 3, standard acc + x*y */
#define GN 3
#define GSUF 3
#define MAC_V(acc, a, b) do { v4d p_[3]; mul3_v(a, b, p_); add3_v(acc, p_, acc); } while (0)
#define MAC_S(acc, a, b) do { double p_[3]; mul3_s(a, b, p_); add3_s(acc, p_, acc); } while (0)
#define MULV mul3_v
#define ADDV add3_v
#define MULS mul3_s
#define ADDS add3_s
#include "gemm_body.inc"
#undef GSUF
#undef MAC_V
#undef MAC_S

/* N = 3, fused mulacc_x3 (the reference's default x3 GEMM route) */
#define GSUF 3f
#define MAC_V(acc, a, b) do { v4d r_[3]; mulacc3_v(acc, a, b, r_); acc[0] = r_[0]; acc[1] = r_[1]; acc[2] = r_[2]; } while (0)
#define MAC_S(acc, a, b) do { double r_[3]; mulacc3_s(acc, a, b, r_); acc[0] = r_[0]; acc[1] = r_[1]; acc[2] = r_[2]; } while (0)
#include "gemm_body.inc"
#undef GN
#undef GSUF
#undef MAC_V
#undef MAC_S
#undef MULV
#undef ADDV
#undef MULS
#undef ADDS

/* N = 4 */
#define GN 4
#define GSUF 4
#define MAC_V(acc, a, b) do { v4d p_[4]; mul4_v(a, b, p_); add4_v(acc, p_, acc); } while (0)
#define MAC_S(acc, a, b) do { double p_[4]; mul4_s(a, b, p_); add4_s(acc, p_, acc); } while (0)
#define MULV mul4_v
#define ADDV add4_v
#define MULS mul4_s
#define ADDS add4_s
#include "gemm_body.inc"
#undef GN
#undef GSUF
#undef MAC_V
#undef MAC_S
#undef MULV
#undef ADDV
#undef MULS
#undef ADDS

/* C = alpha*A*B + beta*C.  A m x k, B k x n, C m x n.  x3_fused selects the
   mulacc_x3 route for N == 3.  Column panels of 32/24/16 (x2/x3/x4; 3/4 of
   that with >= 8 threads) are distributed over threads (gemm.jl:1-7, 267-303). */
int mfr_gemm(int N, int64_t m, int64_t n, int64_t k, const double *A, int64_t lda, int64_t lsa,
             const double *B, int64_t ldb, int64_t lsb, double *C, int64_t ldc, int64_t lsc,
             const double *alpha, const double *beta, int x3_fused, int threads) {
    if (N < 2 || N > 4) return -1;
    int overwrite = mf_iszero(N, beta);
    int base = N == 2 ? 32 : N == 3 ? 24 : 16;
    int64_t panel = threads >= 8 ? (base * 3 / 4 > 12 ? base * 3 / 4 : 12) : base;
    int64_t jobs = (n + panel - 1) / panel;
par_for(jobs, threads, [&](int64_t job) {
        int64_t c0 = job * panel, c1 = c0 + panel < n ? c0 + panel : n;
        switch (N) {
        case 2: gemm_cols_2(m, k, A, lda, lsa, B, ldb, lsb, C, ldc, lsc, alpha, beta, overwrite, c0, c1); break;
        case 3:
            if (x3_fused)
                gemm_cols_3f(m, k, A, lda, lsa, B, ldb, lsb, C, ldc, lsc, alpha, beta, overwrite, c0, c1);
            else
                gemm_cols_3(m, k, A, lda, lsa, B, ldb, lsb, C, ldc, lsc, alpha, beta, overwrite, c0, c1);
            break;
        default: gemm_cols_4(m, k, A, lda, lsa, B, ldb, lsb, C, ldc, lsc, alpha, beta, overwrite, c0, c1); break;
        }
    });
    return 0;
}

/* ------------------------------------------------------- SYRK / GEMMT --- */
/* lower triangle of C = alpha * P^T P + beta * C, P is k x n (syrk.jl:1-50).
   Each C(row, col), row >= col, is one ascending-k chain of P[k,row]*P[k,col]. */
int mfr_syrk_lower(int N, int64_t n, int64_t k, const double *P, int64_t ldp, int64_t lsp,
                   double *C, int64_t ldc, int64_t lsc, const double *alpha, const double *beta,
                   int threads) {
    int overwrite = mf_iszero(N, beta);
par_for(n, threads, [&](int64_t col) {
        for (int64_t row = col; row < n; ++row) {
            double acc[MAXN], a[MAXN], b[MAXN], res[MAXN], cv[MAXN];
            mf_set(N, 0.0, acc);
            for (int64_t kk = 0; kk < k; ++kk) {
                getm(N, P, ldp, lsp, kk, row, a);
                getm(N, P, ldp, lsp, kk, col, b);
                double p[MAXN];
                mf_mul(N, a, b, p);
                mf_add(N, acc, p, acc);
            }
            mf_mul(N, alpha, acc, res);
            if (!overwrite) {
                getm(N, C, ldc, lsc, row, col, cv);
                mf_mul(N, beta, cv, cv);
                mf_add(N, res, cv, res);
            }
            putm(N, C, ldc, lsc, row, col, res);
        }
    });
    return 0;
}

/* packed lower triangle of C (column-major packed, (0,0),(1,0)..(n-1,0),(1,1)..,
   limb stride lsc) = alpha * P[k0:k1,:]^T P[k0:k1,:] + beta * C
   (syrk.jl:110-254, _packed_lower_index syrk.jl:110-117): the SYRK chain over
   the reduction rows k0..k1-1 in ascending order. */
int mfr_syrk_packed(int N, int64_t n, int64_t k0, int64_t k1, const double *P, int64_t ldp,
                    int64_t lsp, double *C, int64_t lsc, const double *alpha, const double *beta,
                    int threads) {
    int overwrite = mf_iszero(N, beta);
    par_for(n, threads, [&](int64_t col) {
        int64_t idx = col * (2 * n - col + 1) / 2;
        for (int64_t row = col; row < n; ++row, ++idx) {
            double acc[MAXN], a[MAXN], b[MAXN], res[MAXN], cv[MAXN];
            mf_set(N, 0.0, acc);
            for (int64_t kk = k0; kk < k1; ++kk) {
                getm(N, P, ldp, lsp, kk, row, a);
                getm(N, P, ldp, lsp, kk, col, b);
                double p[MAXN];
                mf_mul(N, a, b, p);
                mf_add(N, acc, p, acc);
            }
            mf_mul(N, alpha, acc, res);
            if (!overwrite) {
                getm(N, C, 1, lsc, idx, 0, cv);
                mf_mul(N, beta, cv, cv);
                mf_add(N, res, cv, res);
            }
            putm(N, C, 1, lsc, idx, 0, res);
        }
    });
    return 0;
}

/* lower triangle of C = alpha * A * B^T + beta * C, A and B are n x k
   (gemmt.jl:1-52): chain of A[row,k]*B[col,k]. */
int mfr_gemmt_lower(int N, int64_t n, int64_t k, const double *A, int64_t lda, int64_t lsa,
                    const double *B, int64_t ldb, int64_t lsb, double *C, int64_t ldc,
                    int64_t lsc, const double *alpha, const double *beta, int threads) {
    int overwrite = mf_iszero(N, beta);
par_for(n, threads, [&](int64_t col) {
        for (int64_t row = col; row < n; ++row) {
            double acc[MAXN], a[MAXN], b[MAXN], res[MAXN], cv[MAXN];
            mf_set(N, 0.0, acc);
            for (int64_t kk = 0; kk < k; ++kk) {
                getm(N, A, lda, lsa, row, kk, a);
                getm(N, B, ldb, lsb, col, kk, b);
                double p[MAXN];
                mf_mul(N, a, b, p);
                mf_add(N, acc, p, acc);
            }
            mf_mul(N, alpha, acc, res);
            if (!overwrite) {
                getm(N, C, ldc, lsc, row, col, cv);
                mf_mul(N, beta, cv, cv);
                mf_add(N, res, cv, res);
            }
            putm(N, C, ldc, lsc, row, col, res);
        }
    });
    return 0;
}

/* ---------------------------------------------------------------- TRSM -- */
static inline void trsm_coef(int N, const double *A, int64_t lda, int64_t lsa, int64_t r,
                             int64_t c, int transposed, double *out) {
    if (transposed)
        getm(N, A, lda, lsa, c, r, out);
    else
        getm(N, A, lda, lsa, r, c, out);
}

/* B = alpha * op(A) * B (side 0) or alpha * B * op(A) (side 1) in place
   (trmm.jl:1-131), in the reference's element order so every chain reads
   B entries that are not yet overwritten: left, effective lower: rows
   bottom-up, chain coef(i,k) B[k,j] for k = 0..i-1, then the diagonal term;
   left, effective upper: diagonal term, then k = i+1..m-1; right, effective
   lower: columns left to right, diagonal term B[i,j] A[j,j] then B[i,k]
   coef(k,j) for k = j+1..n-1; right, effective upper: columns right to left,
   k = 0..j-1, then the diagonal term.  diag = unit adds B[i,j] itself. */
int mfr_trmm(int N, int side, int uplo, int trans, int diag, int64_t m, int64_t n,
             const double *A, int64_t lda, int64_t lsa, double *B, int64_t ldb, int64_t lsb,
             const double *alpha, int threads) {
    const int eff_lower = (uplo == 0) == (trans == 0);
    auto diag_term = [&](int64_t i, int64_t j, int64_t d, double *acc) {
        double bv[MAXN], av[MAXN], p[MAXN];
        getm(N, B, ldb, lsb, i, j, bv);
        if (diag) {
            mf_add(N, acc, bv, acc);
            return;
        }
        getm(N, A, lda, lsa, d, d, av);
        if (side == 0) mf_mul(N, av, bv, p);
        else mf_mul(N, bv, av, p);
        mf_add(N, acc, p, acc);
    };
    if (side == 0) {
        par_for(n, threads, [&](int64_t j) {
            for (int64_t t = 0; t < m; ++t) {
                const int64_t i = eff_lower ? m - 1 - t : t;
                double acc[MAXN], c[MAXN], bv[MAXN], p[MAXN], res[MAXN];
                mf_set(N, 0.0, acc);
                if (!eff_lower) diag_term(i, j, i, acc);
                const int64_t lo = eff_lower ? 0 : i + 1, hi = eff_lower ? i : m;
                for (int64_t k = lo; k < hi; ++k) {
                    trsm_coef(N, A, lda, lsa, i, k, trans, c);
                    getm(N, B, ldb, lsb, k, j, bv);
                    mf_mul(N, c, bv, p);
                    mf_add(N, acc, p, acc);
                }
                if (eff_lower) diag_term(i, j, i, acc);
                mf_mul(N, alpha, acc, res);
                putm(N, B, ldb, lsb, i, j, res);
            }
        });
    } else {
        par_for(m, threads, [&](int64_t i) {
            for (int64_t t = 0; t < n; ++t) {
                const int64_t j = eff_lower ? t : n - 1 - t;
                double acc[MAXN], c[MAXN], bv[MAXN], p[MAXN], res[MAXN];
                mf_set(N, 0.0, acc);
                if (eff_lower) diag_term(i, j, j, acc);
                const int64_t lo = eff_lower ? j + 1 : 0, hi = eff_lower ? n : j;
                for (int64_t k = lo; k < hi; ++k) {
                    getm(N, B, ldb, lsb, i, k, bv);
                    trsm_coef(N, A, lda, lsa, k, j, trans, c);
                    mf_mul(N, bv, c, p);
                    mf_add(N, acc, p, acc);
                }
                if (!eff_lower) diag_term(i, j, j, acc);
                mf_mul(N, alpha, acc, res);
                putm(N, B, ldb, lsb, i, j, res);
            }
        });
    }
    return 0;
}

/* side: 0 left, 1 right; uplo: 0 lower, 1 upper; trans: 0 N, 1 T; diag: 0
   nonunit, 1 unit.  B is m x n; A is m x m (left) or n x n (right).
   trsm.jl:224-302: B *= alpha unless alpha == 1, then substitution with one
   ascending-k chain per element `values -= coef * B[k]` and `/= A[i,i]`. */
int mfr_trsm(int N, int side, int uplo, int trans, int diag, int64_t m, int64_t n,
             const double *A, int64_t lda, int64_t lsa, double *B, int64_t ldb, int64_t lsb,
             const double *alpha, int threads) {
    double one[MAXN];
    mf_set(N, 1.0, one);
    int scale = 0;
    for (int l = 0; l < N; ++l)
        if (alpha[l] != one[l]) scale = 1;
    if (scale) {
        for (int64_t c = 0; c < n; ++c)
            for (int64_t r = 0; r < m; ++r) {
                double v[MAXN];
                getm(N, B, ldb, lsb, r, c, v);
                mf_mul(N, v, alpha, v);
                putm(N, B, ldb, lsb, r, c, v);
            }
    }
    int transposed = trans == 1;
    int eff_lower = (uplo == 0) == !transposed;
    int unit = diag == 1;
    if (side == 0) {
par_for(n, threads, [&](int64_t c) {
            double v[MAXN], coef[MAXN], bk[MAXN], d[MAXN];
            if (eff_lower) {
                for (int64_t row = 0; row < m; ++row) {
                    getm(N, B, ldb, lsb, row, c, v);
                    for (int64_t kk = 0; kk < row; ++kk) {
                        trsm_coef(N, A, lda, lsa, row, kk, transposed, coef);
                        getm(N, B, ldb, lsb, kk, c, bk);
                        mf_submul(N, v, coef, bk, v);
                    }
                    if (!unit) {
                        getm(N, A, lda, lsa, row, row, d);
                        mf_div(N, v, d, v);
                    }
                    putm(N, B, ldb, lsb, row, c, v);
                }
            } else {
                for (int64_t row = m - 1; row >= 0; --row) {
                    getm(N, B, ldb, lsb, row, c, v);
                    for (int64_t kk = row + 1; kk < m; ++kk) {
                        trsm_coef(N, A, lda, lsa, row, kk, transposed, coef);
                        getm(N, B, ldb, lsb, kk, c, bk);
                        mf_submul(N, v, coef, bk, v);
                    }
                    if (!unit) {
                        getm(N, A, lda, lsa, row, row, d);
                        mf_div(N, v, d, v);
                    }
                    putm(N, B, ldb, lsb, row, c, v);
                }
            }
        });
    } else {
par_for(m, threads, [&](int64_t r) {
            double v[MAXN], coef[MAXN], bk[MAXN], d[MAXN];
            if (eff_lower) {
                for (int64_t col = n - 1; col >= 0; --col) {
                    getm(N, B, ldb, lsb, r, col, v);
                    for (int64_t kk = col + 1; kk < n; ++kk) {
                        getm(N, B, ldb, lsb, r, kk, bk);
                        trsm_coef(N, A, lda, lsa, kk, col, transposed, coef);
                        mf_submul(N, v, bk, coef, v);
                    }
                    if (!unit) {
                        getm(N, A, lda, lsa, col, col, d);
                        mf_div(N, v, d, v);
                    }
                    putm(N, B, ldb, lsb, r, col, v);
                }
            } else {
                for (int64_t col = 0; col < n; ++col) {
                    getm(N, B, ldb, lsb, r, col, v);
                    for (int64_t kk = 0; kk < col; ++kk) {
                        getm(N, B, ldb, lsb, r, kk, bk);
                        trsm_coef(N, A, lda, lsa, kk, col, transposed, coef);
                        mf_submul(N, v, bk, coef, v);
                    }
                    if (!unit) {
                        getm(N, A, lda, lsa, col, col, d);
                        mf_div(N, v, d, v);
                    }
                    putm(N, B, ldb, lsb, r, col, v);
                }
            }
        });
    }
    return 0;
}

/* ------------------------------------------------------------ Cholesky -- */
static int potrf_panel(int N, double *A, int64_t lda, int64_t lsa, int64_t first, int64_t last) {
    for (int64_t col = first; col <= last; ++col) {
        double d[MAXN], v[MAXN], w[MAXN], zero[MAXN], pivot[MAXN];
        getm(N, A, lda, lsa, col, col, d);
        for (int64_t kk = first; kk < col; ++kk) {
            getm(N, A, lda, lsa, col, kk, v);
            mf_submul(N, d, v, v, d);
        }
        mf_set(N, 0.0, zero);
        if (!mf_gt(N, d, zero)) return (int)(col + 1);
        mf_sqrt(N, d, pivot);
        putm(N, A, lda, lsa, col, col, pivot);
        for (int64_t row = col + 1; row <= last; ++row) {
            getm(N, A, lda, lsa, row, col, v);
            for (int64_t kk = first; kk < col; ++kk) {
                double a[MAXN], b[MAXN];
                getm(N, A, lda, lsa, row, kk, a);
                getm(N, A, lda, lsa, col, kk, b);
                mf_submul(N, v, a, b, v);
            }
            mf_div(N, v, pivot, w);
            putm(N, A, lda, lsa, row, col, w);
        }
    }
    return 0;
}

static int lower_finite(int N, const double *A, int64_t lda, int64_t lsa, int64_t n) {
    for (int64_t c = 0; c < n; ++c)
        for (int64_t r = c; r < n; ++r) {
            double v[MAXN];
            getm(N, A, lda, lsa, r, c, v);
            if (!mf_isfinite(N, v)) return 0;
        }
    return 1;
}

/* returns info: 0, -1 (non-finite lower triangle) or the failing column (1-based) */
int mfr_potrf(int N, int64_t n, double *A, int64_t lda, int64_t lsa, int64_t block, int threads) {
    if (!lower_finite(N, A, lda, lsa, n)) return -1;
    if (block < 1) block = 1;
    double mone[MAXN], one[MAXN];
    mf_set(N, -1.0, mone);
    mf_set(N, 1.0, one);
    for (int64_t first = 0; first < n; first += block) {
        int64_t last = first + block - 1 < n - 1 ? first + block - 1 : n - 1;
        int info = potrf_panel(N, A, lda, lsa, first, last);
        if (info) return info;
        if (last < n - 1) {
            int64_t w = last - first + 1, t = n - 1 - last;
            /* A21 <- A21 / L11^T */
            mfr_trsm(N, 1, 0, 1, 0, t, w, A + first * lda + first, lda, lsa,
                     A + first * lda + last + 1, lda, lsa, one, threads);
            /* A22 <- -1 * A21 A21^T + 1 * A22 (lower), panel = A21^T (w x t) */
            /* syrk with P = A21^T: P[k, row] = A21[row, k] -> chain A21[row,k]*A21[col,k] */
            double *A21 = A + first * lda + last + 1;
            double *A22 = A + (last + 1) * lda + last + 1;
par_for(t, threads, [&](int64_t col) {
                for (int64_t row = col; row < t; ++row) {
                    double acc[MAXN], a[MAXN], b[MAXN], res[MAXN], cv[MAXN], p[MAXN];
                    mf_set(N, 0.0, acc);
                    for (int64_t kk = 0; kk < w; ++kk) {
                        getm(N, A21, lda, lsa, row, kk, a);
                        getm(N, A21, lda, lsa, col, kk, b);
                        mf_mul(N, a, b, p);
                        mf_add(N, acc, p, acc);
                    }
                    mf_mul(N, mone, acc, res);
                    getm(N, A22, lda, lsa, row, col, cv);
                    mf_mul(N, one, cv, cv);
                    mf_add(N, res, cv, res);
                    putm(N, A22, lda, lsa, row, col, res);
                }
            });
        }
    }
    return 0;
}

/* B <- A^{-1} B with a Cholesky factor (solve.jl:54-83) */
/* Rank-revealing pivoted Cholesky (cholesky_pivoted.jl:65-175), in place.
   perm (1-based) and out[0] = rank, out[1] = info (0, -1 non-finite lower
   triangle with A unchanged, k > 0 first non-positive pivot).  The lower
   triangle is mirrored once; each step picks the first largest remaining
   diagonal, swaps rows then columns, stores sqrt at (k,k), divides the column
   below and applies the full-square rank-one update A[r,c] -= A[r,k]*A[c,k]. */
int mfr_pstrf(int N, int64_t n, double *A, int64_t lda, int64_t lsa, const double *tol,
              int64_t *perm, int64_t *out, int threads) {
    for (int64_t c = 0; c < n; ++c)
        for (int64_t r = c; r < n; ++r) {
            double v[MAXN];
            getm(N, A, lda, lsa, r, c, v);
            if (!mf_isfinite(N, v)) {
                for (int64_t i = 0; i < n; ++i) perm[i] = i + 1;
                out[0] = 0;
                out[1] = -1;
                return 0;
            }
        }
    for (int64_t c = 0; c < n; ++c)
        for (int64_t r = 0; r < c; ++r) {
            double v[MAXN];
            getm(N, A, lda, lsa, c, r, v);
            putm(N, A, lda, lsa, r, c, v);
        }
    for (int64_t i = 0; i < n; ++i) perm[i] = i + 1;
    int64_t rank = n, info = 0;
    double zero[MAXN], first[MAXN];
    mf_set(N, 0.0, zero);
    mf_set(N, 0.0, first);
    const int use_tol = !mf_iszero(N, tol);
    for (int64_t k = 0; k < n; ++k) {
        int64_t p = k;
        double pd[MAXN], cand[MAXN], piv[MAXN];
        getm(N, A, lda, lsa, k, k, pd);
        for (int64_t i = k + 1; i < n; ++i) {
            getm(N, A, lda, lsa, i, i, cand);
            if (mf_gt(N, cand, pd)) {
                p = i;
                memcpy(pd, cand, sizeof(double) * N);
            }
        }
        if (k == 0) {
            if (!mf_gt(N, pd, zero)) {
                rank = 0;
                info = 1;
                break;
            }
            mf_sqrt(N, pd, first);
        }
        if (mf_ge(N, zero, pd)) {
            double thr[MAXN], thr2[MAXN], apd[MAXN];
            mf_mul(N, tol, first, thr);
            mf_mul(N, thr, thr, thr2);
            mf_abs(N, pd, apd);
            rank = k;
            if (!(use_tol && mf_ge(N, thr2, apd))) info = k + 1;
            break;
        }
        mf_sqrt(N, pd, piv);
        if (use_tol) {
            double lim[MAXN];
            mf_mul(N, tol, first, lim);
            if (mf_ge(N, lim, piv)) {
                rank = k;
                break;
            }
        }
        if (p != k) {
            for (int64_t c = 0; c < n; ++c) {
                double a[MAXN], b[MAXN];
                getm(N, A, lda, lsa, k, c, a);
                getm(N, A, lda, lsa, p, c, b);
                putm(N, A, lda, lsa, k, c, b);
                putm(N, A, lda, lsa, p, c, a);
            }
            for (int64_t r = 0; r < n; ++r) {
                double a[MAXN], b[MAXN];
                getm(N, A, lda, lsa, r, k, a);
                getm(N, A, lda, lsa, r, p, b);
                putm(N, A, lda, lsa, r, k, b);
                putm(N, A, lda, lsa, r, p, a);
            }
            const int64_t t = perm[k];
            perm[k] = perm[p];
            perm[p] = t;
        }
        putm(N, A, lda, lsa, k, k, piv);
        for (int64_t r = k + 1; r < n; ++r) {
            double v[MAXN];
            getm(N, A, lda, lsa, r, k, v);
            mf_div(N, v, piv, v);
            putm(N, A, lda, lsa, r, k, v);
        }
        par_for(n - k - 1, threads, [&](int64_t cc) {
            const int64_t c = k + 1 + cc;
            double f[MAXN], lr[MAXN], v[MAXN];
            getm(N, A, lda, lsa, c, k, f);
            for (int64_t r = k + 1; r < n; ++r) {
                getm(N, A, lda, lsa, r, k, lr);
                getm(N, A, lda, lsa, r, c, v);
                mf_submul(N, v, lr, f, v);
                putm(N, A, lda, lsa, r, c, v);
            }
        });
    }
    out[0] = rank;
    out[1] = info;
    return 0;
}

int mfr_potrs(int N, int64_t n, int64_t nrhs, const double *A, int64_t lda, int64_t lsa, double *B,
              int64_t ldb, int64_t lsb, int threads) {
    double one[MAXN];
    mf_set(N, 1.0, one);
    mfr_trsm(N, 0, 0, 0, 0, n, nrhs, A, lda, lsa, B, ldb, lsb, one, threads);
    mfr_trsm(N, 0, 0, 1, 0, n, nrhs, A, lda, lsa, B, ldb, lsb, one, threads);
    return 0;
}

/* ------------------------------------------------------------------ LU -- */
static void swap_rows(int N, double *A, int64_t lda, int64_t lsa, int64_t ncols, int64_t r1,
                      int64_t r2) {
    if (r1 == r2) return;
    for (int64_t c = 0; c < ncols; ++c)
        for (int l = 0; l < N; ++l) {
            double t = EL(A, lda, lsa, r1, c, l);
            EL(A, lda, lsa, r1, c, l) = EL(A, lda, lsa, r2, c, l);
            EL(A, lda, lsa, r2, c, l) = t;
        }
}

static int all_finite(int N, const double *A, int64_t lda, int64_t lsa, int64_t m, int64_t n) {
    for (int64_t c = 0; c < n; ++c)
        for (int64_t r = 0; r < m; ++r) {
            double v[MAXN];
            getm(N, A, lda, lsa, r, c, v);
            if (!mf_isfinite(N, v)) return 0;
        }
    return 1;
}

/* ipiv is 1-based like the reference.  Returns 0, -1 or the zero pivot index. */
int mfr_getrf(int N, int64_t m, int64_t n, double *A, int64_t lda, int64_t lsa, int64_t *ipiv,
              int64_t block, int threads) {
    int64_t kmax = m < n ? m : n;
    for (int64_t i = 0; i < kmax; ++i) ipiv[i] = i + 1;
    if (!all_finite(N, A, lda, lsa, m, n)) return -1;
    if (block < 1) block = 1;
    double mone[MAXN], one[MAXN];
    mf_set(N, -1.0, mone);
    mf_set(N, 1.0, one);
    for (int64_t first = 0; first < kmax; first += block) {
        int64_t last = first + block - 1 < kmax - 1 ? first + block - 1 : kmax - 1;
        for (int64_t k = first; k <= last; ++k) {
            int64_t piv = k;
            double pv[MAXN], cand[MAXN], v[MAXN];
            getm(N, A, lda, lsa, k, k, v);
            mf_abs(N, v, pv);
            for (int64_t row = k + 1; row < m; ++row) {
                getm(N, A, lda, lsa, row, k, v);
                mf_abs(N, v, cand);
                if (mf_gt(N, cand, pv)) {
                    piv = row;
                    memcpy(pv, cand, sizeof(double) * N);
                }
            }
            ipiv[k] = piv + 1;
            swap_rows(N, A, lda, lsa, n, k, piv);
            double akk[MAXN], inv[MAXN];
            getm(N, A, lda, lsa, k, k, akk);
            if (mf_iszero(N, akk)) return (int)(k + 1);
            mf_inv(N, akk, inv);
            for (int64_t row = k + 1; row < m; ++row) {
                getm(N, A, lda, lsa, row, k, v);
                mf_mul(N, v, inv, v);
                putm(N, A, lda, lsa, row, k, v);
            }
            if (k < last) {
                for (int64_t col = k + 1; col <= last; ++col) {
                    double mult[MAXN], f[MAXN];
                    getm(N, A, lda, lsa, k, col, mult);
                    for (int64_t row = k + 1; row < m; ++row) {
                        getm(N, A, lda, lsa, row, col, v);
                        getm(N, A, lda, lsa, row, k, f);
                        mf_submul(N, v, f, mult, v);
                        putm(N, A, lda, lsa, row, col, v);
                    }
                }
            }
        }
        if (last < n - 1) {
            int64_t w = last - first + 1, rest = n - 1 - last;
            double *U12 = A + (last + 1) * lda + first;
            mfr_trsm(N, 0, 0, 0, 1, w, rest, A + first * lda + first, lda, lsa, U12, lda, lsa, one,
                     threads);
            if (last < m - 1) {
                double *A21 = A + first * lda + last + 1;
                double *A22 = A + (last + 1) * lda + last + 1;
                int x3f = 1;
                mfr_gemm(N, m - 1 - last, rest, w, A21, lda, lsa, U12, lda, lsa, A22, lda, lsa, mone,
                         one, x3f, threads);
            }
        }
    }
    return 0;
}

static void apply_pivots(int N, double *B, int64_t ldb, int64_t lsb, int64_t nrhs,
                         const int64_t *ipiv, int64_t count) {
    for (int64_t k = 0; k < count; ++k) {
        int64_t p = ipiv[k] - 1;
        if (p != k) swap_rows(N, B, ldb, lsb, nrhs, k, p);
    }
}

/* solve.jl:147-181 */
int mfr_getrs(int N, int64_t n, int64_t nrhs, const double *A, int64_t lda, int64_t lsa,
              const int64_t *ipiv, double *B, int64_t ldb, int64_t lsb, int threads) {
    double one[MAXN];
    mf_set(N, 1.0, one);
    apply_pivots(N, B, ldb, lsb, nrhs, ipiv, n);
    mfr_trsm(N, 0, 0, 0, 1, n, nrhs, A, lda, lsa, B, ldb, lsb, one, threads);
    mfr_trsm(N, 0, 1, 0, 0, n, nrhs, A, lda, lsa, B, ldb, lsb, one, threads);
    return 0;
}

/* ---------------------------------------------------------------- LDLT -- */
/* ldlt.jl:65-101.  returns nonsingular flag */
static int ldlt_solve_2x2(int N, const double *d11, const double *d21, const double *d22,
                          const double *first, const double *second, double *x1, double *x2) {
    double scale[MAXN], t1[MAXN], t2[MAXN], t3[MAXN];
    mf_abs(N, d11, t1);
    mf_abs(N, d21, t2);
    mf_abs(N, d22, t3);
    mf_max(N, t1, t2, scale);
    mf_max(N, scale, t3, scale);
    if (mf_iszero(N, scale) || !mf_isfinite(N, scale)) {
        mf_set(N, 0.0, x1);
        mf_set(N, 0.0, x2);
        return 0;
    }
    double a[MAXN], b[MAXN], c[MAXN], r1[MAXN], r2[MAXN];
    mf_div(N, d11, scale, a);
    mf_div(N, d21, scale, b);
    mf_div(N, d22, scale, c);
    mf_div(N, first, scale, r1);
    mf_div(N, second, scale, r2);
    double aa[MAXN], ab[MAXN], t[MAXN], u[MAXN], w[MAXN], y1[MAXN], y2[MAXN];
    mf_abs(N, a, aa);
    mf_abs(N, b, ab);
    if (mf_ge(N, aa, ab)) {
        if (mf_iszero(N, a)) goto fail;
        mf_div(N, b, a, t);
        mf_submul(N, c, t, b, u);
        if (mf_iszero(N, u) || !mf_isfinite(N, u)) goto fail;
        mf_submul(N, r2, t, r1, w);
        mf_div(N, w, u, y2);
        mf_submul(N, r1, b, y2, w);
        mf_div(N, w, a, y1);
    } else {
        if (mf_iszero(N, b)) goto fail;
        mf_div(N, a, b, t);
        mf_submul(N, b, t, c, u);
        if (mf_iszero(N, u) || !mf_isfinite(N, u)) goto fail;
        mf_submul(N, r1, t, r2, w);
        mf_div(N, w, u, y2);
        mf_submul(N, r2, c, y2, w);
        mf_div(N, w, b, y1);
    }
    memcpy(x1, y1, sizeof(double) * N);
    memcpy(x2, y2, sizeof(double) * N);
    return 1;
fail:
    mf_set(N, 0.0, x1);
    mf_set(N, 0.0, x2);
    return 0;
}

static void ldlt_symmetric_swap(int N, double *A, int64_t lda, int64_t lsa, int64_t n,
                                int64_t first, int64_t second, int64_t active_first) {
    if (first == second) return;
    for (int l = 0; l < N; ++l) {
        for (int64_t c = 0; c < active_first; ++c) {
            double t = EL(A, lda, lsa, first, c, l);
            EL(A, lda, lsa, first, c, l) = EL(A, lda, lsa, second, c, l);
            EL(A, lda, lsa, second, c, l) = t;
        }
        for (int64_t c = active_first; c < n; ++c) {
            double t = EL(A, lda, lsa, first, c, l);
            EL(A, lda, lsa, first, c, l) = EL(A, lda, lsa, second, c, l);
            EL(A, lda, lsa, second, c, l) = t;
        }
        for (int64_t r = active_first; r < n; ++r) {
            double t = EL(A, lda, lsa, r, first, l);
            EL(A, lda, lsa, r, first, l) = EL(A, lda, lsa, r, second, l);
            EL(A, lda, lsa, r, second, l) = t;
        }
    }
}

/* the lazily updated Schur-complement entry (ldlt.jl:414-449) */
static void ldlt_panel_entry(int N, const double *A, int64_t lda, int64_t lsa, int64_t i1,
                             int64_t i2, int64_t panel_first, int64_t pivot_first,
                             const double *dsub, int64_t lsd, const uint8_t *blocks, double *out) {
    int64_t row = i1 > i2 ? i1 : i2, col = i1 > i2 ? i2 : i1;
    double v[MAXN];
    getm(N, A, lda, lsa, row, col, v);
    int64_t q = panel_first;
    while (q < pivot_first) {
        double a[MAXN], b[MAXN], c[MAXN], t[MAXN];
        if (blocks[q] == 1) {
            getm(N, A, lda, lsa, q, q, a);
            getm(N, A, lda, lsa, col, q, b);
            mf_mul(N, a, b, t);
            getm(N, A, lda, lsa, row, q, c);
            mf_submul(N, v, c, t, v);
            q += 1;
        } else {
            double rf[MAXN], rs[MAXN], cf[MAXN], cs[MAXN], dq[MAXN], dq1[MAXN], ds[MAXN];
            double c1[MAXN], c2[MAXN], t1[MAXN], t2[MAXN];
            getm(N, A, lda, lsa, row, q, rf);
            getm(N, A, lda, lsa, row, q + 1, rs);
            getm(N, A, lda, lsa, col, q, cf);
            getm(N, A, lda, lsa, col, q + 1, cs);
            getm(N, A, lda, lsa, q, q, dq);
            getm(N, A, lda, lsa, q + 1, q + 1, dq1);
            for (int l = 0; l < N; ++l) ds[l] = dsub[l * lsd + q];
            mf_mul(N, dq, cf, t1);
            mf_mul(N, ds, cs, t2);
            mf_add(N, t1, t2, c1);
            mf_mul(N, ds, cf, t1);
            mf_mul(N, dq1, cs, t2);
            mf_add(N, t1, t2, c2);
            mf_mul(N, rf, c1, t1);
            mf_mul(N, rs, c2, t2);
            mf_add(N, t1, t2, t);
            mf_sub(N, v, t, v);
            q += 2;
        }
    }
    memcpy(out, v, sizeof(double) * N);
}

/* Bunch-Kaufman pivot choice; returns block size (0, 1, 2), pivot in *piv.
   unblocked form reads A directly (lazy == 0), panel form evaluates entries
   lazily (ldlt.jl:183-219, 451-508). */
static int select_bk(int N, const double *A, int64_t lda, int64_t lsa, int64_t n, int64_t k,
                     const double *alpha, int lazy, int64_t panel_first, const double *dsub,
                     int64_t lsd, const uint8_t *blocks, int64_t *piv) {
#define ENTRY(i, j, out)                                                                     \
    do {                                                                                     \
        if (lazy)                                                                            \
            ldlt_panel_entry(N, A, lda, lsa, (i), (j), panel_first, k, dsub, lsd, blocks, out); \
        else                                                                                 \
            getm(N, A, lda, lsa, (i), (j), out);                                             \
    } while (0)
    double v[MAXN], absakk[MAXN], colmax[MAXN], cand[MAXN], zero[MAXN];
    mf_set(N, 0.0, zero);
    ENTRY(k, k, v);
    mf_abs(N, v, absakk);
    if (k == n - 1) {
        *piv = k;
        return mf_iszero(N, absakk) ? 0 : 1;
    }
    int64_t imax = k + 1;
    ENTRY(imax, k, v);
    mf_abs(N, v, colmax);
    for (int64_t row = k + 2; row < n; ++row) {
        ENTRY(row, k, v);
        mf_abs(N, v, cand);
        if (mf_gt(N, cand, colmax)) {
            memcpy(colmax, cand, sizeof(double) * N);
            imax = row;
        }
    }
    double mx[MAXN], t[MAXN];
    mf_max(N, absakk, colmax, mx);
    if (mf_iszero(N, mx)) {
        *piv = k;
        return 0;
    }
    mf_mul(N, alpha, colmax, t);
    if (mf_ge(N, absakk, t)) {
        *piv = k;
        return 1;
    }
    double rowmax[MAXN];
    mf_set(N, 0.0, rowmax);
    for (int64_t c = k; c < imax; ++c) {
        ENTRY(imax, c, v);
        mf_abs(N, v, cand);
        mf_max(N, rowmax, cand, rowmax);
    }
    for (int64_t r = imax + 1; r < n; ++r) {
        ENTRY(r, imax, v);
        mf_abs(N, v, cand);
        mf_max(N, rowmax, cand, rowmax);
    }
    double q[MAXN];
    mf_mul(N, alpha, colmax, t);
    mf_div(N, colmax, rowmax, q);
    mf_mul(N, t, q, t);
    if (mf_ge(N, absakk, t)) {
        *piv = k;
        return 1;
    }
    ENTRY(imax, imax, v);
    mf_abs(N, v, cand);
    mf_mul(N, alpha, rowmax, t);
    *piv = imax;
    return mf_ge(N, cand, t) ? 1 : 2;
#undef ENTRY
}

static void mirror_lower_to_upper(int N, double *A, int64_t lda, int64_t lsa, int64_t n) {
    for (int l = 0; l < N; ++l)
        for (int64_t c = 0; c < n; ++c)
            for (int64_t r = c + 1; r < n; ++r) EL(A, lda, lsa, c, r, l) = EL(A, lda, lsa, r, c, l);
}

static int sytrf_unblocked(int N, double *A, int64_t lda, int64_t lsa, int64_t n, double *dsub,
                           int64_t lsd, int64_t *pivots, uint8_t *blocks, const double *alpha) {
    int64_t k = 0;
    while (k < n) {
        int64_t piv;
        int bs = select_bk(N, A, lda, lsa, n, k, alpha, 0, 0, dsub, lsd, blocks, &piv);
        if (bs == 0) return (int)(k + 1);
        if (bs == 1) {
            pivots[k] = piv + 1;
            blocks[k] = 1;
            ldlt_symmetric_swap(N, A, lda, lsa, n, k, piv, k);
            double d[MAXN], v[MAXN];
            getm(N, A, lda, lsa, k, k, d);
            if (mf_iszero(N, d)) return (int)(k + 1);
            for (int64_t row = k + 1; row < n; ++row) {
                getm(N, A, lda, lsa, row, k, v);
                mf_div(N, v, d, v);
                putm(N, A, lda, lsa, row, k, v);
            }
            if (k < n - 1) {
                /* rank-1 update, ldlt.jl:221-259 */
                for (int64_t col = k + 1; col < n; ++col) {
                    double coef[MAXN], lc[MAXN], f[MAXN];
                    getm(N, A, lda, lsa, col, k, lc);
                    mf_mul(N, d, lc, coef);
                    for (int64_t row = col; row < n; ++row) {
                        getm(N, A, lda, lsa, row, col, v);
                        getm(N, A, lda, lsa, row, k, f);
                        mf_submul(N, v, f, coef, v);
                        putm(N, A, lda, lsa, row, col, v);
                        putm(N, A, lda, lsa, col, row, v);
                    }
                }
            }
            k += 1;
        } else {
            if (!(k < n - 1)) return (int)(k + 1);
            pivots[k] = piv + 1;
            blocks[k] = 2;
            blocks[k + 1] = 0;
            ldlt_symmetric_swap(N, A, lda, lsa, n, k + 1, piv, k);
            double d11[MAXN], d21[MAXN], d22[MAXN], z[MAXN], x1[MAXN], x2[MAXN];
            getm(N, A, lda, lsa, k, k, d11);
            getm(N, A, lda, lsa, k + 1, k, d21);
            getm(N, A, lda, lsa, k + 1, k + 1, d22);
            for (int l = 0; l < N; ++l) dsub[l * lsd + k] = d21[l];
            mf_set(N, 0.0, z);
            if (!ldlt_solve_2x2(N, d11, d21, d22, z, z, x1, x2)) return (int)(k + 1);
            for (int64_t row = k + 2; row < n; ++row) {
                double f[MAXN], s[MAXN];
                getm(N, A, lda, lsa, row, k, f);
                getm(N, A, lda, lsa, row, k + 1, s);
                int ok = ldlt_solve_2x2(N, d11, d21, d22, f, s, x1, x2);
                if (!(ok && mf_isfinite(N, x1) && mf_isfinite(N, x2))) return (int)(k + 1);
                putm(N, A, lda, lsa, row, k, x1);
                putm(N, A, lda, lsa, row, k + 1, x2);
            }
            if (k + 1 < n - 1) {
                /* rank-2 update, ldlt.jl:261-326: the 4-row SIMD groups use
                   v - (f1*c1 + f2*c2); remainder rows use (v - f1*c1) - f2*c2 */
                for (int64_t col = k + 2; col < n; ++col) {
                    double l1[MAXN], l2[MAXN], c1[MAXN], c2[MAXN], t1[MAXN], t2[MAXN];
                    getm(N, A, lda, lsa, col, k, l1);
                    getm(N, A, lda, lsa, col, k + 1, l2);
                    mf_mul(N, d11, l1, t1);
                    mf_mul(N, d21, l2, t2);
                    mf_add(N, t1, t2, c1);
                    mf_mul(N, d21, l1, t1);
                    mf_mul(N, d22, l2, t2);
                    mf_add(N, t1, t2, c2);
                    int64_t row = col;
                    while (row + 3 < n) {
                        for (int64_t i = row; i < row + 4; ++i) {
                            double v[MAXN], f1[MAXN], f2[MAXN], s[MAXN];
                            getm(N, A, lda, lsa, i, col, v);
                            getm(N, A, lda, lsa, i, k, f1);
                            getm(N, A, lda, lsa, i, k + 1, f2);
                            mf_mul(N, f1, c1, t1);
                            mf_mul(N, f2, c2, t2);
                            mf_add(N, t1, t2, s);
                            mf_sub(N, v, s, v);
                            putm(N, A, lda, lsa, i, col, v);
                            putm(N, A, lda, lsa, col, i, v);
                        }
                        row += 4;
                    }
                    for (; row < n; ++row) {
                        double v[MAXN], f1[MAXN], f2[MAXN];
                        getm(N, A, lda, lsa, row, col, v);
                        getm(N, A, lda, lsa, row, k, f1);
                        getm(N, A, lda, lsa, row, k + 1, f2);
                        mf_submul(N, v, f1, c1, v);
                        mf_submul(N, v, f2, c2, v);
                        putm(N, A, lda, lsa, row, col, v);
                        putm(N, A, lda, lsa, col, row, v);
                    }
                }
            }
            double z0[MAXN];
            mf_set(N, 0.0, z0);
            putm(N, A, lda, lsa, k + 1, k, z0);
            putm(N, A, lda, lsa, k, k + 1, z0);
            k += 2;
        }
    }
    return 0;
}

/* lazy blocked panel (ldlt.jl:510-593); returns info, sets *panel_last */
static int sytrf_panel(int N, double *A, int64_t lda, int64_t lsa, int64_t n, int64_t pf,
                       int64_t requested_last, double *dsub, int64_t lsd, int64_t *pivots,
                       uint8_t *blocks, const double *alpha, int64_t *panel_last_out) {
    int64_t pl = requested_last;
    int64_t k = pf;
    while (k <= pl) {
        int64_t piv;
        int bs = select_bk(N, A, lda, lsa, n, k, alpha, 1, pf, dsub, lsd, blocks, &piv);
        if (bs == 0) {
            *panel_last_out = pl;
            return (int)(k + 1);
        }
        if (bs == 2 && k == pl) {
            if (!(k < n - 1)) {
                *panel_last_out = pl;
                return (int)(k + 1);
            }
            pl += 1;
        }
        if (bs == 1) {
            pivots[k] = piv + 1;
            blocks[k] = 1;
            ldlt_symmetric_swap(N, A, lda, lsa, n, k, piv, k);
            double d[MAXN], e[MAXN];
            ldlt_panel_entry(N, A, lda, lsa, k, k, pf, k, dsub, lsd, blocks, d);
            if (mf_iszero(N, d)) {
                *panel_last_out = pl;
                return (int)(k + 1);
            }
            putm(N, A, lda, lsa, k, k, d);
            for (int64_t row = k + 1; row < n; ++row) {
                ldlt_panel_entry(N, A, lda, lsa, row, k, pf, k, dsub, lsd, blocks, e);
                mf_div(N, e, d, e);
                putm(N, A, lda, lsa, row, k, e);
            }
            k += 1;
        } else {
            pivots[k] = piv + 1;
            blocks[k] = 2;
            blocks[k + 1] = 0;
            ldlt_symmetric_swap(N, A, lda, lsa, n, k + 1, piv, k);
            double d11[MAXN], d21[MAXN], d22[MAXN], z[MAXN], x1[MAXN], x2[MAXN];
            ldlt_panel_entry(N, A, lda, lsa, k, k, pf, k, dsub, lsd, blocks, d11);
            ldlt_panel_entry(N, A, lda, lsa, k + 1, k, pf, k, dsub, lsd, blocks, d21);
            ldlt_panel_entry(N, A, lda, lsa, k + 1, k + 1, pf, k, dsub, lsd, blocks, d22);
            putm(N, A, lda, lsa, k, k, d11);
            putm(N, A, lda, lsa, k + 1, k + 1, d22);
            for (int l = 0; l < N; ++l) dsub[l * lsd + k] = d21[l];
            mf_set(N, 0.0, z);
            if (!ldlt_solve_2x2(N, d11, d21, d22, z, z, x1, x2)) {
                *panel_last_out = pl;
                return (int)(k + 1);
            }
            for (int64_t row = k + 2; row < n; ++row) {
                double f[MAXN], s[MAXN];
                ldlt_panel_entry(N, A, lda, lsa, row, k, pf, k, dsub, lsd, blocks, f);
                ldlt_panel_entry(N, A, lda, lsa, row, k + 1, pf, k, dsub, lsd, blocks, s);
                int ok = ldlt_solve_2x2(N, d11, d21, d22, f, s, x1, x2);
                if (!(ok && mf_isfinite(N, x1) && mf_isfinite(N, x2))) {
                    *panel_last_out = pl;
                    return (int)(k + 1);
                }
                putm(N, A, lda, lsa, row, k, x1);
                putm(N, A, lda, lsa, row, k + 1, x2);
            }
            double z0[MAXN];
            mf_set(N, 0.0, z0);
            putm(N, A, lda, lsa, k + 1, k, z0);
            putm(N, A, lda, lsa, k, k + 1, z0);
            k += 2;
        }
    }
    *panel_last_out = pl;
    return 0;
}

/* blocked == 1 selects the lazy-panel + gemmt route (ldlt_gemmt.jl:36-73) with
   the given panel width.  pivots are 1-based.  Returns info. */
int mfr_sytrf(int N, int64_t n, double *A, int64_t lda, int64_t lsa, double *dsub, int64_t lsd,
              int64_t *pivots, uint8_t *blocks, int blocked, int64_t block, int threads) {
    for (int64_t i = 0; i < n; ++i) {
        pivots[i] = i + 1;
        blocks[i] = 0;
        for (int l = 0; l < N; ++l) dsub[l * lsd + i] = 0.0;
    }
    if (!lower_finite(N, A, lda, lsa, n)) return -1;
    mirror_lower_to_upper(N, A, lda, lsa, n);
    double alpha[MAXN], one[MAXN], s17[MAXN], eight[MAXN], mone[MAXN];
    mf_set(N, 1.0, one);
    mf_set(N, 17.0, s17);
    mf_set(N, 8.0, eight);
    mf_set(N, -1.0, mone);
    mf_sqrt(N, s17, s17);
    mf_add(N, one, s17, alpha);
    mf_div(N, alpha, eight, alpha);
    if (!blocked) return sytrf_unblocked(N, A, lda, lsa, n, dsub, lsd, pivots, blocks, alpha);
    if (block < 2) block = 2;
    double *W = (double *)malloc(sizeof(double) * (size_t)N * (size_t)(n > 0 ? n : 1) * (size_t)(block + 1));
    int64_t ldw = n > 0 ? n : 1, lsw = ldw * (block + 1);
    int64_t pf = 0;
    int info = 0;
    while (pf < n) {
        int64_t req = pf + block - 1 < n - 1 ? pf + block - 1 : n - 1;
        int64_t pl;
        info = sytrf_panel(N, A, lda, lsa, n, pf, req, dsub, lsd, pivots, blocks, alpha, &pl);
        if (info) break;
        if (pl < n - 1) {
            int64_t tc = n - 1 - pl, pw = pl - pf + 1;
            /* weighted panel W = L21 * D (ldlt.jl:595-632) */
            int64_t q = pf;
            while (q <= pl) {
                int64_t lc = q - pf;
                if (blocks[q] == 1) {
                    double d[MAXN], v[MAXN];
                    getm(N, A, lda, lsa, q, q, d);
                    for (int64_t lr = 0; lr < tc; ++lr) {
                        getm(N, A, lda, lsa, pl + 1 + lr, q, v);
                        mf_mul(N, v, d, v);
                        putm(N, W, ldw, lsw, lr, lc, v);
                    }
                    q += 1;
                } else {
                    double d11[MAXN], d21[MAXN], d22[MAXN];
                    getm(N, A, lda, lsa, q, q, d11);
                    for (int l = 0; l < N; ++l) d21[l] = dsub[l * lsd + q];
                    getm(N, A, lda, lsa, q + 1, q + 1, d22);
                    for (int64_t lr = 0; lr < tc; ++lr) {
                        double f[MAXN], s[MAXN], t1[MAXN], t2[MAXN], w1[MAXN], w2[MAXN];
                        getm(N, A, lda, lsa, pl + 1 + lr, q, f);
                        getm(N, A, lda, lsa, pl + 1 + lr, q + 1, s);
                        mf_mul(N, f, d11, t1);
                        mf_mul(N, s, d21, t2);
                        mf_add(N, t1, t2, w1);
                        mf_mul(N, f, d21, t1);
                        mf_mul(N, s, d22, t2);
                        mf_add(N, t1, t2, w2);
                        putm(N, W, ldw, lsw, lr, lc, w1);
                        putm(N, W, ldw, lsw, lr, lc + 1, w2);
                    }
                    q += 2;
                }
            }
            double *L21 = A + pf * lda + pl + 1;
            double *A22 = A + (pl + 1) * lda + pl + 1;
            mfr_gemmt_lower(N, tc, pw, L21, lda, lsa, W, ldw, lsw, A22, lda, lsa, mone, one, threads);
            mirror_lower_to_upper(N, A22, lda, lsa, tc);
        }
        pf = pl + 1;
    }
    free(W);
    return info;
}

static void ldlt_pivots_forward(int N, double *B, int64_t ldb, int64_t lsb, int64_t nrhs,
                                int64_t n, const int64_t *pivots, const uint8_t *blocks) {
    int64_t k = 0;
    while (k < n) {
        if (blocks[k] == 1) {
            swap_rows(N, B, ldb, lsb, nrhs, k, pivots[k] - 1);
            k += 1;
        } else {
            swap_rows(N, B, ldb, lsb, nrhs, k + 1, pivots[k] - 1);
            k += 2;
        }
    }
}

static void ldlt_pivots_reverse(int N, double *B, int64_t ldb, int64_t lsb, int64_t nrhs,
                                int64_t n, const int64_t *pivots, const uint8_t *blocks) {
    int64_t k = n - 1;
    while (k >= 0) {
        if (blocks[k] == 1) {
            swap_rows(N, B, ldb, lsb, nrhs, k, pivots[k] - 1);
            k -= 1;
        } else {
            swap_rows(N, B, ldb, lsb, nrhs, k, pivots[k - 1] - 1);
            k -= 2;
        }
    }
}

/* solve.jl:298-365.  returns 0 or the singular 2x2 block index */
int mfr_sytrs(int N, int64_t n, int64_t nrhs, const double *A, int64_t lda, int64_t lsa,
              const double *dsub, int64_t lsd, const int64_t *pivots, const uint8_t *blocks,
              double *B, int64_t ldb, int64_t lsb, int threads) {
    double one[MAXN];
    mf_set(N, 1.0, one);
    ldlt_pivots_forward(N, B, ldb, lsb, nrhs, n, pivots, blocks);
    mfr_trsm(N, 0, 0, 0, 1, n, nrhs, A, lda, lsa, B, ldb, lsb, one, threads);
    int64_t k = 0;
    while (k < n) {
        if (blocks[k] == 1) {
            double d[MAXN], v[MAXN];
            getm(N, A, lda, lsa, k, k, d);
            for (int64_t c = 0; c < nrhs; ++c) {
                getm(N, B, ldb, lsb, k, c, v);
                mf_div(N, v, d, v);
                putm(N, B, ldb, lsb, k, c, v);
            }
            k += 1;
        } else {
            double d11[MAXN], d21[MAXN], d22[MAXN];
            getm(N, A, lda, lsa, k, k, d11);
            for (int l = 0; l < N; ++l) d21[l] = dsub[l * lsd + k];
            getm(N, A, lda, lsa, k + 1, k + 1, d22);
            for (int64_t c = 0; c < nrhs; ++c) {
                double f[MAXN], s[MAXN], x1[MAXN], x2[MAXN];
                getm(N, B, ldb, lsb, k, c, f);
                getm(N, B, ldb, lsb, k + 1, c, s);
                if (!ldlt_solve_2x2(N, d11, d21, d22, f, s, x1, x2)) return (int)(k + 1);
                putm(N, B, ldb, lsb, k, c, x1);
                putm(N, B, ldb, lsb, k + 1, c, x2);
            }
            k += 2;
        }
    }
    mfr_trsm(N, 0, 0, 1, 1, n, nrhs, A, lda, lsa, B, ldb, lsb, one, threads);
    ldlt_pivots_reverse(N, B, ldb, lsb, nrhs, n, pivots, blocks);
    return 0;
}

/* ------------------------------------------------ mixed residual -------- */
/* residual.jl:343-428: every operand widened from ns to nr limbs (zero limbs
   appended), acc = B[i,j]; acc -= A[i,k] * X[k,j] for k ascending.  uplo 0
   general, 1 lower, 2 upper (symmetric access to the authoritative triangle). */
int mfr_residual_mixed(int ns, int nr, int uplo, int64_t m, int64_t k, int64_t nrhs,
                       const double *A, int64_t lda, int64_t lsa, const double *X, int64_t ldx,
                       int64_t lsx, const double *B, int64_t ldb, int64_t lsb, double *R,
                       int64_t ldr, int64_t lsr) {
    for (int64_t j = 0; j < nrhs; ++j)
        for (int64_t i = 0; i < m; ++i) {
            double acc[MAXN] = {0, 0, 0, 0};
            for (int l = 0; l < ns; ++l) acc[l] = EL(B, ldb, lsb, i, j, l);
            for (int64_t kk = 0; kk < k; ++kk) {
                double a[MAXN] = {0, 0, 0, 0}, x[MAXN] = {0, 0, 0, 0};
                int tr = (uplo == 1 && kk > i) || (uplo == 2 && kk < i);
                for (int l = 0; l < ns; ++l) {
                    a[l] = tr ? EL(A, lda, lsa, kk, i, l) : EL(A, lda, lsa, i, kk, l);
                    x[l] = EL(X, ldx, lsx, kk, j, l);
                }
                mf_submul(nr, acc, a, x, acc);
            }
            for (int l = 0; l < nr; ++l) EL(R, ldr, lsr, i, j, l) = acc[l];
        }
    return 0;
}

/* ------------------------------------------- exact superaccumulator ----- */
/* Kulisch-style fixed-point accumulator over the whole binary64 range: base
   2^32 digits held in int64 so that ~2^31 signed additions need no carry.
   Bit position 0 is 2^EXP_LO. */
#define EXP_LO (-1200)
#define NDIG 72 /* 72*32 = 2304 bits: 2^-1200 .. 2^1104 */
typedef struct {
    int64_t d[NDIG];
    int64_t adds;
} kacc_t;

static void kacc_norm(kacc_t *a) {
    int64_t carry = 0;
    for (int i = 0; i < NDIG; ++i) {
        int64_t v = a->d[i] + carry;
        int64_t lo = v & 0xffffffffLL;
        carry = (v - lo) >> 32;
        a->d[i] = lo;
    }
    a->d[NDIG - 1] += carry << 32; /* sign lives in the top digit */
    a->adds = 0;
}

static void kacc_add(kacc_t *a, double x) {
    if (x == 0.0) return;
    int e;
    double f = frexp(x, &e); /* x = f * 2^e, 0.5 <= |f| < 1 */
    int64_t mant = (int64_t)ldexp(f, 53); /* exact, |mant| < 2^53 */
    int64_t bit = (int64_t)(e - 53) - EXP_LO;
    if (bit < 0) { /* below 2^EXP_LO: cannot happen for binary64 (min 2^-1074) */
        return;
    }
    int64_t idx = bit >> 5, sh = bit & 31;
    int neg = mant < 0;
    uint64_t um = (uint64_t)(neg ? -mant : mant);
    /* um << sh spans up to 85 bits: split into three 32-bit digits */
    unsigned __int128 wide = (unsigned __int128)um << sh;
    uint64_t lo = (uint64_t)(wide & 0xffffffffULL);
    uint64_t mid = (uint64_t)((wide >> 32) & 0xffffffffULL);
    uint64_t hi = (uint64_t)(wide >> 64);
    int64_t s = neg ? -1 : 1;
    a->d[idx] += s * (int64_t)lo;
    if (idx + 1 < NDIG) a->d[idx + 1] += s * (int64_t)mid;
    if (idx + 2 < NDIG) a->d[idx + 2] += s * (int64_t)hi;
    if (++a->adds > (1LL << 29)) kacc_norm(a);
}

/* add the exact product x*y */
static void kacc_add_prod(kacc_t *a, double x, double y) {
    double p = x * y;
    double e = __builtin_fma(x, y, -p);
    kacc_add(a, p);
    kacc_add(a, e);
}

/* round the accumulated value to a double (faithful) */
static double kacc_value(kacc_t *a) {
    kacc_norm(a);
    /* two's complement over the digit vector: top digit holds the sign */
    int neg = a->d[NDIG - 1] < 0;
    int64_t dig[NDIG];
    if (neg) {
        /* negate: value = -(sum) */
        int64_t carry = 0;
        for (int i = 0; i < NDIG; ++i) {
            int64_t v = -a->d[i] + carry;
            int64_t lo = v & 0xffffffffLL;
            carry = (v - lo) >> 32;
            dig[i] = lo;
        }
    } else {
        memcpy(dig, a->d, sizeof dig);
    }
    int top = -1;
    for (int i = NDIG - 1; i >= 0; --i)
        if (dig[i] != 0) {
            top = i;
            break;
        }
    if (top < 0) return 0.0;
    double v = 0.0;
    for (int i = top; i >= 0 && i >= top - 3; --i) v += ldexp((double)dig[i], 32 * i + EXP_LO);
    return neg ? -v : v;
}

/* For sampled entries (rows[s], cols[s]) of C = A*B: err[s] = |C_hat - C_exact|
   rounded, scale[s] = sum_k |A[i,k]| |B[k,j]| (leading limbs, binary64), and
   exact[s] = the exact value rounded to binary64. */
int mfr_exact_gemm_check(int N, int64_t k, const double *A, int64_t lda, int64_t lsa,
                         const double *B, int64_t ldb, int64_t lsb, const double *C, int64_t ldc,
                         int64_t lsc, int64_t nsamp, const int64_t *rows, const int64_t *cols,
                         double *err, double *scale, double *exact, int threads) {
par_for(nsamp, threads, [&](int64_t s) {
        kacc_t acc;
        memset(&acc, 0, sizeof acc);
        int64_t i = rows[s], j = cols[s];
        double sc = 0.0;
        for (int64_t kk = 0; kk < k; ++kk) {
            double a[MAXN], b[MAXN];
            getm(N, A, lda, lsa, i, kk, a);
            getm(N, B, ldb, lsb, kk, j, b);
            for (int la = 0; la < N; ++la)
                for (int lb = 0; lb < N; ++lb) kacc_add_prod(&acc, a[la], b[lb]);
            sc += fabs(a[0]) * fabs(b[0]);
        }
        kacc_t cp = acc;
        exact[s] = kacc_value(&cp);
        for (int l = 0; l < N; ++l) kacc_add(&acc, -EL(C, ldc, lsc, i, j, l));
        err[s] = fabs(kacc_value(&acc));
        scale[s] = sc;
    });
    return 0;
}

/* R = B - A*X exactly, rounded to binary64 per entry.  A n x n (general),
   X n x nrhs, B n x nrhs.  Used for backward errors. */
int mfr_exact_residual(int N, int64_t n, int64_t nrhs, const double *A, int64_t lda, int64_t lsa,
                       const double *X, int64_t ldx, int64_t lsx, const double *B, int64_t ldb,
                       int64_t lsb, double *R, int64_t ldr, int threads) {
par_for((nrhs) * (n), threads, [&](int64_t idx_) {
        int64_t c = idx_ / (n), i = idx_ % (n);
            kacc_t acc;
            memset(&acc, 0, sizeof acc);
            for (int l = 0; l < N; ++l) kacc_add(&acc, EL(B, ldb, lsb, i, c, l));
            for (int64_t kk = 0; kk < n; ++kk) {
                double a[MAXN], x[MAXN];
                getm(N, A, lda, lsa, i, kk, a);
                getm(N, X, ldx, lsx, kk, c, x);
                for (int la = 0; la < N; ++la)
                    for (int lb = 0; lb < N; ++lb) kacc_add_prod(&acc, -a[la], x[lb]);
            }
            R[c * ldr + i] = kacc_value(&acc);
        });
    return 0;
}

/* exact sum of the limbs of each value rounded to binary64 (limb-major) */
void mfr_to_double(int N, int64_t count, const double *x, int64_t ls, double *out) {
    for (int64_t i = 0; i < count; ++i) {
        kacc_t acc;
        memset(&acc, 0, sizeof acc);
        for (int l = 0; l < N; ++l) kacc_add(&acc, x[l * ls + i]);
        out[i] = kacc_value(&acc);
    }
}

int mfr_max_threads(void) {
    unsigned n = std::thread::hardware_concurrency();
    return n ? (int)n : 1;
}


#include "qr_body.inc"

} /* extern "C" */
