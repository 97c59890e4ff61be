// Modular INT8 route for the multi-double GEMM: exact products of scaled
// integer operands through residue arithmetic (Chinese remainder theorem).
//
// No reference counterpart: MultiFloatLinearAlgebra.jl has only the FP64
// networks.  Published method: Ozaki, Uchino, Imamura (2025), "Ozaki scheme
// II: a GEMM-oriented emulation of floating-point matrix multiplication using
// an integer modular technique"; the CRT reconstruction below is plain
// multi-word integer arithmetic of this file's own design.
//
// 1. Scaling (shared with the digit-slice route): row i of A is scaled by
//    2^-sa_i, column j of B by 2^-sb_j, so that every scaled entry lies in
//    (-1/2, 1/2).
// 2. Integer digits.  The scaled value z is written as Q signed integer digits
//    of h bits, z 2^(Q h) = sum_q D_q 2^(h (Q-1-q)) + remainder, |D_q| <= 2^(h+1),
//    by the digit step of the slice route with 2^h in place of 2^7 (scale by
//    2^h, round every limb to an integer, keep the exact remainder).  Float64x2
//    uses one digit (Q = 1: the whole operand as one integer of h = beta bits);
//    Float64x3/x4 use Q = 2.
// 3. Residues.  For T pairwise coprime moduli p_t <= 256 (product P) every
//    digit is reduced mod p_t to a signed byte; for each digit level L (pairs
//    q + r = L, adjacent along K as in the slice route) and each modulus, ONE
//    int8 GEMM gives G_L mod p_t exactly in int32 (|residues| <= 128, so
//    Q k 2^14 < 2^31).  All T moduli of a level run in one launch.
// 4. Reconstruction.  G_L = sum_t r_t U_t mod P with U_t = (P/p_t) ((P/p_t)^-1
//    mod p_t), taken in the symmetric range (-P/2, P/2); P > 2 Q k max|D|^2
//    makes this the exact integer sum_{q+r=L} D_q E_r.  G_L is converted to
//    Float64xN with the add network, the levels are added least significant
//    first, scaled by 2^(sa_i + sb_j - 2 Q h) and the alpha/beta epilogue of
//    the plain kernel is applied.
// The digits drop nothing but the final remainders and the levels L >= Q, so
// the error is about k 2^(sa+sb) 2^(-Q h) (the same form as the slice route
// with 7 S replaced by Q h) at T int8 GEMMs per level instead of S (S+1)/2.
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "int8_tc_common.cuh"
#include "mf_device.cuh"
#include "mflab_internal.h"
#include "ozaki_common.cuh"

MFLAB_DEBUG_RECORD(ozaki_crt)

namespace mfl {

constexpr int CRT_MAXT = CRT_TABLE_SIZE;
constexpr int CRT_WD = 5;     // max 32-bit words of one digit (h <= 157)
constexpr int CRT_WP = 12;    // max 32-bit words of a CRT sum (< 2^384)
constexpr int CRT_MAXH = 32 * CRT_WD - 3;

// weights of the digit bytes: wt[t][j] packs 2^(8 b) mod p_t for bytes
// b = 4j .. 4j+3 of a digit's two's-complement words (one byte each);
// negoff[WD-3][t] = (128 - 2^(32 WD) mod p_t) mod p_t, the offset that turns
// the residue of the words of a negative digit into (digit + 128) mod p_t
struct CrtSplitConst {
    uint32_t wt[CRT_MAXT][CRT_WD];
    uint32_t negoff[CRT_WD - 2][CRT_MAXT];
};

// reconstruction constants for one modulus count T
struct CrtAccConst {
    uint32_t U[CRT_MAXT][CRT_WP];  // U_t words, little endian
    uint32_t P[CRT_WP];            // P words
    double pinv;                   // 1 / P (rounded)
};

// The reconstruction sum X = sum_t r_t U_t on the FP64 pipe: U_t is cut into
// CRT_CW-bit chunks held as doubles, so every product r_t * chunk (r_t < 2^8)
// is below 2^47 and a chunk's sum over at most 49 moduli stays below 2^53:
// exact in binary64.  The chunk sums are then moved into 64-bit partial word
// sums at bit 39 c.
constexpr int CRT_CW = 39;
constexpr int CRT_NC = 9;  // chunks of a U_t (P < 2^342)
static_assert(CRT_MAXT * 255.0 * 549755813888.0 < 9007199254740992.0,
              "chunk sums must stay exact in binary64");

// kernel copy of the constants (a kernel parameter, under 4 KB)
struct CrtAccDev {
    double Ud[CRT_MAXT][CRT_NC];  // chunk c of U_t: bits [39 c, 39 c + 39)
    uint32_t P[CRT_WP];
    double pinv;
};

// chunks a WP-word sum can need: P < 2^(32 WP), at most CRT_NC
template <int WP>
struct CrtChunks {
    static constexpr int value =
        (32 * WP + CRT_CW - 1) / CRT_CW < CRT_NC ? (32 * WP + CRT_CW - 1) / CRT_CW : CRT_NC;
};

// chunk sums (exact integers below 2^53) -> 64-bit partial word sums
template <int WP>
__host__ __device__ __forceinline__ void crt_chunks_to_words(const double (&A)[CrtChunks<WP>::value],
                                                             uint64_t (&X)[WP]) {
#pragma unroll
    for (int w = 0; w < WP; ++w) X[w] = 0;
#pragma unroll
    for (int cc = 0; cc < CrtChunks<WP>::value; ++cc) {
        const uint64_t a = (uint64_t)A[cc];
        const int bit = CRT_CW * cc, w0 = bit >> 5, sh = bit & 31;
        if (w0 < WP) X[w0] += (uint32_t)(a << sh);
        if (w0 + 1 < WP) X[w0 + 1] += a >> (32 - sh);
    }
}

// 2^k for k in [-1022, 1023]
__device__ __forceinline__ double pow2i(int k) {
    return __longlong_as_double((long long)(k + 1023) << 52);
}

// d * 2^e with a single rounding (exact unless the result is subnormal);
// exponents beyond the double range saturate to 0 / inf as ldexp would
__device__ __forceinline__ double scale2(double d, int e) {
    e = e < -2044 ? -2044 : (e > 2046 ? 2046 : e);
    const int e1 = e >> 1;
    return (d * pow2i(e1)) * pow2i(e - e1);
}

// ------------------------------------------------------------- digits ----
// One h-bit digit D of the scaled value z (z is updated to the remainder):
// WD little-endian 32-bit words holding D in two's complement
// (|D| < 2^(32 WD - 1)) and the sign of D.
template <int N, int WD>
__device__ __forceinline__ void crt_digit(mf<N> &z, int h, uint32_t (&w)[WD], bool &neg) {
    double d[N];
#pragma unroll
    for (int l = 0; l < N; ++l) {
        z.v[l] = z.v[l] * pow2i(h);                // exact (h <= 157, |z| < 2)
        d[l] = rint(z.v[l]);
        z.v[l] = __dsub_rn(z.v[l], d[l]);          // exact: |z_l - rint(z_l)| <= 1/2
    }
#pragma unroll
    for (int l = N - 1; l > 0; --l) two_sum(z.v[l - 1], z.v[l], z.v[l - 1], z.v[l]);
    // D = sum_l d_l: every d_l is an integer, |d_l| = mm 2^e with a 53-bit
    // mantissa; signed 32-bit slices of each are added word by word
    int64_t c[WD];
#pragma unroll
    for (int j = 0; j < WD; ++j) c[j] = 0;
#pragma unroll
    for (int l = 0; l < N; ++l) {
        if (d[l] != 0.0) {
            const uint64_t bits = (uint64_t)__double_as_longlong(d[l]);
            const bool sneg = (bits >> 63) != 0;
            uint64_t mm = (bits & ((1ULL << 52) - 1)) | (1ULL << 52);
            int e = (int)((bits >> 52) & 0x7ff) - 1075;
            if (e < 0) {  // the bits shifted out are zero: d_l is an integer
                mm >>= -e;
                e = 0;
            }
#pragma unroll
            for (int j = 0; j < WD; ++j) {
                const int dd = 32 * j - e;  // bit of mm that lands on bit 0 of word j
                uint32_t part = 0;
                if (dd >= 0 && dd < 64) part = (uint32_t)(mm >> dd);
                else if (dd < 0 && dd > -32) part = (uint32_t)(mm << (-dd));
                c[j] += sneg ? -(int64_t)part : (int64_t)part;
            }
        }
    }
    int64_t carry = 0;
#pragma unroll
    for (int j = 0; j < WD; ++j) {
        const int64_t t = c[j] + carry;
        w[j] = (uint32_t)t;
        carry = t >> 32;  // arithmetic: ends at -1 exactly when D < 0
    }
    neg = carry < 0;
}

// The same digit for h <= CRT_FAST_H and WD <= 4, with the sum formed as one
// 128-bit two's-complement integer: the leading limb's 53-bit mantissa
// shifted by its exponent (below 64 bits of shift for these h), each lower
// limb converted exactly to an int64 (|d_l| <= 2^(h-54) + 1 < 2^63) and
// added with carries.  D is the same exact integer, so the words and the
// sign are those of crt_digit.
constexpr int CRT_FAST_H = 116;

template <int N, int WD>
__device__ __forceinline__ void crt_digit_fast(mf<N> &z, int h, uint32_t (&w)[WD], bool &neg) {
    static_assert(WD <= 4, "128-bit sum");
    double d[N];
#pragma unroll
    for (int l = 0; l < N; ++l) {
        z.v[l] = z.v[l] * pow2i(h);                // exact (h <= 157, |z| < 2)
        d[l] = rint(z.v[l]);
        z.v[l] = __dsub_rn(z.v[l], d[l]);          // exact: |z_l - rint(z_l)| <= 1/2
    }
#pragma unroll
    for (int l = N - 1; l > 0; --l) two_sum(z.v[l - 1], z.v[l], z.v[l - 1], z.v[l]);
    uint64_t lo = 0, hi = 0;
    {
        const uint64_t bits = (uint64_t)__double_as_longlong(d[0]);
        const int e = (int)((bits >> 52) & 0x7ff) - 1075;
        if (d[0] != 0.0 && e >= 0) {  // |d_0| >= 2^53: mantissa << e, e < 64
            const uint64_t mm = (bits & ((1ULL << 52) - 1)) | (1ULL << 52);
            lo = mm << e;
            hi = e ? mm >> (64 - e) : 0ULL;
            if (bits >> 63) {  // negate the 128-bit value
                lo = ~lo + 1ULL;
                hi = ~hi + (lo == 0ULL ? 1ULL : 0ULL);
            }
        } else {  // |d_0| < 2^53: an exact int64
            const int64_t v = __double2ll_rn(d[0]);
            lo = (uint64_t)v;
            hi = v < 0 ? ~0ULL : 0ULL;
        }
    }
#pragma unroll
    for (int l = 1; l < N; ++l) {
        const int64_t v = __double2ll_rn(d[l]);
        const uint64_t a = (uint64_t)v, ah = v < 0 ? ~0ULL : 0ULL;
        const uint64_t s0 = lo + a;
        hi = hi + ah + (s0 < lo ? 1ULL : 0ULL);
        lo = s0;
    }
    const uint32_t ws[4] = {(uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32)};
#pragma unroll
    for (int j = 0; j < WD; ++j) w[j] = ws[j];
    neg = (int64_t)hi < 0;
}

// the digit step of the split kernels: the 128-bit path where it applies
template <int N, int WD>
__device__ __forceinline__ void crt_digit_any(mf<N> &z, int h, uint32_t (&w)[WD], bool &neg) {
    if constexpr (WD <= 4) {
        if (h <= CRT_FAST_H) {
            crt_digit_fast<N, WD>(z, h, w, neg);
            return;
        }
    }
    crt_digit<N, WD>(z, h, w, neg);
}

// (D + 128) mod p from the two's-complement words of D (off = 128 for D >= 0,
// the modulus' negoff for D < 0); the stored byte is this value - 128, an
// int8 congruent to D mod p
template <int WD>
__device__ __forceinline__ uint32_t crt_residue(const uint32_t (&w)[WD], const uint32_t *wt,
                                                uint32_t off, int p) {
    uint32_t acc = off;
#pragma unroll
    for (int j = 0; j < WD; ++j) acc = __dp4a(w[j], wt[j], acc);  // < 20 * 255^2 + 512
    return acc % (uint32_t)p;
}

// elements per thread of the split kernels: 8 for Float64x2, 4 for more limbs
// (their staging tile and registers would not fit twice the elements)
template <int N>
struct CrtSplitU {
    static constexpr int value = N == 2 ? 8 : 4;
};

// residue bytes of U consecutive elements (digit words w[u], signs ng[u]) for
// the moduli t < T: one U-byte store per modulus plane
template <int WD, int U>
__device__ __forceinline__ void crt_emit(const uint32_t (&w)[U][WD], const bool (&ng)[U], int T,
                                         int8_t *dst, size_t plane8, const CrtSplitConst &c) {
#pragma unroll
    for (int t = 0; t < CRT_MAXT; ++t) {
        if (t >= T) break;
        const int p = crt_modulus(t);
        const uint32_t noff = c.negoff[WD - 3][t];
        uint32_t wt[WD];
#pragma unroll
        for (int j = 0; j < WD; ++j) wt[j] = c.wt[t][j];
        uint32_t packed[U / 4];
#pragma unroll
        for (int g = 0; g < U / 4; ++g) {
            packed[g] = 0;  // bytes of elements 4g+3 .. 4g, by multiply-add
#pragma unroll
            for (int u = 3; u >= 0; --u)
                packed[g] = packed[g] * 256u +
                            crt_residue<WD>(w[4 * g + u], wt, ng[4 * g + u] ? noff : 128u, p);
        }
        if constexpr (U == 8)
            *(uint2 *)(dst + (size_t)t * plane8) =
                make_uint2(packed[0] ^ 0x80808080u, packed[1] ^ 0x80808080u);
        else
            *(uint32_t *)(dst + (size_t)t * plane8) = packed[0] ^ 0x80808080u;
    }
}

// A (m x k, column-major planes) -> residue planes A8[t][i][q'][k] (int8,
// rows of Q kp bytes, plane stride plane8; q' = q, or Q-1-q with rev).  A
// block stages a 32-row x 64-k tile of every limb plane in shared memory; each
// of its 32 x 8 threads then owns 8 consecutive k of one row and writes 8
// bytes per (t, q) (4 of each for more than two limbs).
template <int N, int WD>
__global__ void __launch_bounds__(256)
    crt_split_a_kernel(int64_t m, int64_t mp, int64_t k, int64_t kp, int Q, int h, int T, Mat A,
                       const int *rowexp, int8_t *A8, size_t plane8, int rev,
                       const __grid_constant__ CrtSplitConst c) {
    constexpr int U = CrtSplitU<N>::value, AK = 8 * U;  // k extent of the tile
    __shared__ double tile[N][AK][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int64_t i0 = (int64_t)blockIdx.x * 32, k0 = (int64_t)blockIdx.y * AK;
#pragma unroll
    for (int j = 0; j < AK / 8; ++j) {
        const int kk = ty + 8 * j;
        const int64_t i = i0 + tx, kg = k0 + kk;
        const bool ok = i < m && kg < k;
#pragma unroll
        for (int l = 0; l < N; ++l) tile[l][kk][tx] = ok ? A.p[l * A.ls + kg * A.ld + i] : 0.0;
    }
    __syncthreads();
    const int ii = ty * 4 + (tx >> 3), kq = (tx & 7) * U;
    const int64_t i = i0 + ii, kg = k0 + kq;
    if (i >= mp || kg >= kp) return;  // kp is a multiple of 128: kg + U - 1 < kp
    const int e = i < m ? rowexp[i] : OZ_EXP_EMPTY;
    const int sh = oz_scale_exp(e);
    mf<N> z[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
#pragma unroll
        for (int l = 0; l < N; ++l)
            z[u].v[l] = (e == OZ_EXP_BAD) ? 0.0 : scale2(tile[l][kq + u][ii], -sh);
#pragma unroll
        for (int l = N - 1; l > 0; --l) two_sum(z[u].v[l - 1], z[u].v[l], z[u].v[l - 1], z[u].v[l]);
    }
    int8_t *dst = A8 + (size_t)i * Q * kp + kg;
    if (!MFLAB_IDX_OK(kg + U <= kp && i < mp, 3, i, kg)) return;
    for (int q = 0; q < Q; ++q) {
        uint32_t w[U][WD];
        bool ng[U];
#pragma unroll
        for (int u = 0; u < U; ++u) crt_digit_any<N, WD>(z[u], h, w[u], ng[u]);
        crt_emit<WD, U>(w, ng, T, dst + (size_t)(rev ? Q - 1 - q : q) * kp, plane8, c);
    }
}

// B (k x n) -> residue planes B8[t][j][q'][k] with q' = Q-1-q when rev (the
// right operand: pairs of one level adjacent along K), q' = q otherwise (the
// left operand of a Gram product A^T A, whose rows are B's columns).  Each
// thread owns U consecutive k of one column.
template <int N, int WD>
__global__ void __launch_bounds__(128)
    crt_split_b_kernel(int64_t k, int64_t n, int64_t np, int64_t kp, int Q, int h, int T, Mat B,
                       const int *colexp, int8_t *B8, size_t plane8, int rev,
                       const __grid_constant__ CrtSplitConst c) {
    constexpr int U = CrtSplitU<N>::value;
    const int64_t kg = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * U;
    const int64_t j = blockIdx.y;
    if (kg >= kp || j >= np) return;
    const int e = j < n ? colexp[j] : OZ_EXP_EMPTY;
    const int sh = oz_scale_exp(e);
    mf<N> z[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int64_t kk = kg + u;
        const bool ok = kk < k && j < n && e != OZ_EXP_BAD;
#pragma unroll
        for (int l = 0; l < N; ++l)
            z[u].v[l] = ok ? scale2(B.p[l * B.ls + j * B.ld + kk], -sh) : 0.0;
#pragma unroll
        for (int l = N - 1; l > 0; --l) two_sum(z[u].v[l - 1], z[u].v[l], z[u].v[l - 1], z[u].v[l]);
    }
    int8_t *dst = B8 + (size_t)j * Q * kp + kg;
    if (!MFLAB_IDX_OK(kg + U <= kp && j < np, 3, j, kg)) return;
    for (int q = 0; q < Q; ++q) {
        uint32_t w[U][WD];
        bool ng[U];
#pragma unroll
        for (int u = 0; u < U; ++u) crt_digit_any<N, WD>(z[u], h, w[u], ng[u]);
        crt_emit<WD, U>(w, ng, T, dst + (size_t)(rev ? Q - 1 - q : q) * kp, plane8, c);
    }
}

// launch shapes of the two split kernels
template <int N>
static inline dim3 crt_split_a_grid(int64_t mp, int64_t kp) {
    return dim3((unsigned)((mp + 31) / 32), (unsigned)(kp / (8 * CrtSplitU<N>::value)));
}
template <int N>
static inline dim3 crt_split_b_grid(int64_t np, int64_t kp) {
    return dim3((unsigned)((kp / CrtSplitU<N>::value + 127) / 128), (unsigned)np);
}

// ------------------------------------------------------ reconstruction ----
// q = round(X / P) from the chunk sums: X ~ sum_c A_c 2^(39 c) by Horner
// (relative error below 2^-49), and X / P lies within 3/8 of an integer
template <int WP>
__host__ __device__ __forceinline__ uint32_t crt_quotient(const double (&A)[CrtChunks<WP>::value],
                                                         double pinv) {
    constexpr int NC = CrtChunks<WP>::value;
    double xd = A[NC - 1];
#pragma unroll
    for (int cc = NC - 2; cc >= 0; --cc) xd = fma(xd, 549755813888.0, A[cc]);  // 2^39
    return (uint32_t)floor(xd * pinv + 0.5);
}

// X (WP words of 64-bit partial sums) -> G = X - round(X / P) P as magnitude
// words + sign (host and device: the host copy backs
// mflab_ozaki_crt_reduce_host).  Precondition, kept by the planner: the
// represented value satisfies |G| <= 3P / 8 (it is G mod P in the symmetric
// range), so X / P lies within 3/8 of the integer q = round(X / P) and the
// double estimate of X / P (crt_quotient, relative error < 2^-48) rounds to
// exactly the q passed in.  All products are 32 x 32 -> 64 bit.
template <int WP>
__host__ __device__ __forceinline__ bool crt_reduce(const uint64_t (&X)[WP], const uint32_t *Pw,
                                                    uint32_t q, uint32_t (&mag)[WP]) {
    uint32_t x[WP];
    uint64_t cy = 0;
#pragma unroll
    for (int w = 0; w < WP; ++w) {
        const uint64_t s = X[w] + cy;
        x[w] = (uint32_t)s;
        cy = s >> 32;
    }
    // Y = X - q P (two's complement over WP words; the final borrow is the sign)
    uint32_t y[WP];
    uint64_t hi = 0;   // carry of q P
    uint32_t br = 0;   // borrow
#pragma unroll
    for (int w = 0; w < WP; ++w) {
        const uint64_t qp = (uint64_t)q * Pw[w] + hi;
        hi = qp >> 32;
        const uint64_t d = (uint64_t)x[w] - (uint32_t)qp - br;
        y[w] = (uint32_t)d;
        br = (uint32_t)(d >> 63);
    }
    // |Y|: negate the words when Y < 0
    const uint32_t flip = br ? 0xffffffffu : 0u;
    uint32_t ca = br;
#pragma unroll
    for (int w = 0; w < WP; ++w) {
        const uint64_t t = (uint64_t)(y[w] ^ flip) + ca;
        mag[w] = (uint32_t)t;
        ca = (uint32_t)(t >> 32);
    }
    return br != 0;
}

// Float64xN value of a WP-word magnitude times 2^e2: the top 53 (N+1) bits as
// N+1 truncated 53-bit chunks (the guard chunk rounds into the N limbs),
// renormalised with fast two-sums (exact for values of at most 53 N
// significant bits)
template <int N, int WP>
__device__ __forceinline__ mf<N> crt_words_to_mf(const uint32_t (&mag)[WP], int e2) {
    int pos = -1;
#pragma unroll
    for (int w = 0; w < WP; ++w) pos = mag[w] ? w : pos;
    if (pos < 0) return from_double<N>(0.0);
    // barrel shift by whole words so that word pos lands on WP - 1
    uint32_t a[WP];
#pragma unroll
    for (int w = 0; w < WP; ++w) a[w] = mag[w];
    const int sw = WP - 1 - pos;
#pragma unroll
    for (int b = 8; b >= 1; b >>= 1) {
        if (b < WP && (sw & b)) {
#pragma unroll
            for (int w = WP - 1; w >= 0; --w) a[w] = w >= b ? a[w - b] : 0u;
        }
    }
    const int lz = __clz(a[WP - 1]);
#pragma unroll
    for (int w = WP - 1; w > 0; --w) a[w] = __funnelshift_l(a[w - 1], a[w], lz);
    a[0] <<= lz;
    // the window's bit 32 WP - 1 has weight 2^(32 pos + 31 - lz + e2)
    const int top = 32 * pos + 32 - lz + e2;
    double c[N + 1];
#pragma unroll
    for (int l = N; l >= 0; --l) {
        const int b0 = 32 * WP - 53 * (l + 1);  // lowest bit of chunk l in the window
        uint64_t ch;
        if (b0 >= 0) {
            const int wi = b0 >> 5, off = b0 & 31;
            ch = (uint64_t)a[wi] >> off;
            if (wi + 1 < WP) ch |= (uint64_t)a[wi + 1] << (32 - off);
            if (wi + 2 < WP && off > 11) ch |= (uint64_t)a[wi + 2] << (64 - off);
        } else {  // the window ends inside the chunk: its low bits are zero
            ch = b0 > -53 ? ((uint64_t)a[0] | ((uint64_t)a[1] << 32)) << (-b0) : 0;
        }
        ch &= (1ULL << 53) - 1;
        c[l] = scale2((double)ch, top - 53 * (l + 1));
    }
    // The chunks are exact, of one sign, and each nonzero one lies above the sum
    // of those below it (they fill lower units of its 53-bit grid), so a
    // bottom-up sweep of error-free fast two-sums carries the rounding of the
    // lower chunks into the upper ones; a top-down sweep of two-sums (no order
    // condition) leaves every term below half an ulp of the one above; the last
    // term is folded into limb N-1.
#pragma unroll
    for (int l = N - 1; l >= 0; --l) fast_two_sum(c[l], c[l + 1], c[l], c[l + 1]);
#pragma unroll
    for (int l = 0; l < N; ++l) two_sum(c[l], c[l + 1], c[l], c[l + 1]);
    mf<N> g;
#pragma unroll
    for (int l = 0; l < N; ++l) g.v[l] = c[l];
    g.v[N - 1] = __dadd_rn(g.v[N - 1], c[N]);
    return g;
}

// C = alpha * 2^(sa+sb-2Qh) sum_L 2^(h (2Q-2-L)) G_L (+ beta * C); R holds
// the residues G_L mod p_t as bytes, plane (L T + t) at R + (L T + t) plane.
// A block covers 128 rows of one column: the Q T residue segments of its rows
// (128 bytes each, 128-byte aligned) are copied to shared memory with
// cp.async in one round trip, then each thread reconstructs its entry.
constexpr int CRT_ACC_ROWS = 128;

template <int N, int WP>
__global__ void __launch_bounds__(CRT_ACC_ROWS, 3)
    crt_accum_kernel(int64_t m, int64_t n, int Q, int h, int T, const uint8_t *R, int64_t ldi,
                     size_t plane, const int *rowexp, const int *colexp, Mat C, scal<N> alpha,
                     scal<N> beta, int flags, const __grid_constant__ CrtAccDev c) {
    __shared__ __align__(16) uint8_t sres[2 * CRT_MAXT][CRT_ACC_ROWS];
    const int tid = threadIdx.x;
    const int64_t i0 = (int64_t)blockIdx.x * CRT_ACC_ROWS, i = i0 + tid;
    const int64_t j = blockIdx.y;
    // flags bit 2: lower triangle only (the GEMM skipped the tiles above it)
    if ((flags & 4) && i0 + CRT_ACC_ROWS - 1 < j) return;
    // rows i0 .. i0+127 lie inside the padded planes (ldi = mp, a multiple of 128)
    const int segs = Q * T * (CRT_ACC_ROWS / 16);
    for (int s = tid; s < segs; s += CRT_ACC_ROWS) {
        const int pl = s / (CRT_ACC_ROWS / 16), part = s % (CRT_ACC_ROWS / 16);
        const uint8_t *g = R + (size_t)pl * plane + (size_t)j * ldi + i0 + part * 16;
        const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&sres[pl][part * 16]);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(g) : "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    if (i >= m || ((flags & 4) && i < j)) return;
    const int ea = rowexp[i], eb = colexp[j];
    mf<N> acc = from_double<N>(0.0);
    if (ea == OZ_EXP_BAD || eb == OZ_EXP_BAD) {
        acc = from_double<N>(__longlong_as_double(0x7ff8000000000000LL));
    } else {
        for (int L = Q - 1; L >= 0; --L) {
            const uint8_t *src = &sres[L * T][tid];
            constexpr int NC = CrtChunks<WP>::value;
            double A[NC];
#pragma unroll
            for (int cc = 0; cc < NC; ++cc) A[cc] = 0.0;
#pragma unroll
            for (int t = 0; t < CRT_MAXT; ++t) {
                if (t >= T) break;
                // the residue byte as an exact double: 2^52 + r minus 2^52
                const double rd = __hiloint2double(0x43300000, (int)src[t * CRT_ACC_ROWS]) -
                                  4503599627370496.0;
#pragma unroll
                for (int cc = 0; cc < NC; ++cc) A[cc] = fma(rd, c.Ud[t][cc], A[cc]);
            }
            uint64_t X[WP];
            crt_chunks_to_words<WP>(A, X);
            uint32_t mag[WP];
            const bool ng = crt_reduce<WP>(X, c.P, crt_quotient<WP>(A, c.pinv), mag);
            const int sh = oz_scale_exp(ea) + oz_scale_exp(eb) - 2 * Q * h + h * (2 * Q - 2 - L);
            mf<N> g = crt_words_to_mf<N, WP>(mag, sh);
            if (ng) g = neg(g);
            acc = L == Q - 1 ? g : add(acc, g);
        }
    }
    // flags bit 0: beta == 0 (C is not read); bit 1: alpha == 1
    mf<N> r = (flags & 2) ? acc : mul(alpha.get(), acc);
    if (!(flags & 1)) r = add(r, mul(beta.get(), load_mf<N>(C.p, C.ld, C.ls, i, j)));
    store_mf<N>(C.p, C.ld, C.ls, i, j, r);
}

// ---------------------------------- reconstruction on the tensor cores ----
// The sum X = sum_t r_t U_t of the reconstruction as an int8 product: the
// residues r_t (unsigned bytes, r_t < p_t <= 256) of 128 entries of one
// column of C are the rows of A (K runs over the moduli, zero beyond T) and
// the little-endian bytes u_{t,b} of the U_t are the rows of B, so one
// tcgen05.mma.kind::i8 (u8 x u8 -> s32, M = 128, N = CrtTcN bytes, K = 32)
// per 32 moduli yields the byte sums S_b = sum_t r_t u_{t,b} exactly (below
// 49 * 255^2 < 2^22), and X = sum_b S_b 2^(8 b).  From X on (q = round(X / P),
// X - q P, conversion, levels, epilogue) the arithmetic is crt_accum_kernel's
// on the same integer, so the two kernels give the same bits.
//
// Persistent CTAs of 4 warps walk tasks of 128 rows x J columns (J = 2 for
// one digit level, 1 for two: J Q slots of one column and level):
//   1. the warps turn residue segments into K-major operand rows: lane l loads
//      the 32-bit words (entries 4l .. 4l+3) of 16 moduli (coalesced), then
//      transposes the 4 x 16 bytes with byte permutes and stores one 16-byte
//      chunk per entry into the 128-byte swizzled row layout (the entries are
//      visited in a lane-rotated order, so a warp's stores hit every bank).
//      A slot takes 32 bytes of a row per 32 moduli, so 128 / (32 ksteps)
//      slots share one 128-row operand tile;
//   2. thread 0 issues the task's MMAs (one per slot and 32 moduli; a slot's
//      operand starts at its byte offset inside the swizzled rows) and commits
//      them to an mbarrier;
//   3. after the bounded wait, warp w reads TMEM lanes 32w .. 32w+31, one
//      entry per thread, and finishes the entries.
// Occupancy hides the latency of the load -> MMA -> epilogue chain of a task:
// the TMEM allocation is J Q NB columns (rounded up to a power of two), and
// as many CTAs as fit into 512 columns share an SM.
constexpr int CRT_TC_THREADS = 128;
constexpr uint32_t CRT_TC_ATILE = 128 * 128;  // one operand tile: 128 rows x 128 B

// bytes of U_t (< P < 2^(32 WP - 14)) rounded up to the MMA's N step
template <int WP>
struct CrtTcN {
    static constexpr int value = WP == 8 ? 32 : 48;
};

// kernel copy of the tensor-core reconstruction constants
struct __align__(16) CrtTcDev {
    uint32_t ub[48][16];  // byte (t % 4) of ub[b][t / 4] = byte b of U_t; zero for t >= T
    uint32_t P[CRT_WP];
    double pinv;
};

// 32-bit add / subtract with the carry flag (a chain keeps its order: the
// statements are volatile and no other instruction touches the flag)
__device__ __forceinline__ uint32_t add_cc(uint32_t a, uint32_t b) {
    uint32_t r;
    asm volatile("add.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t addc_cc(uint32_t a, uint32_t b) {
    uint32_t r;
    asm volatile("addc.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t sub_cc(uint32_t a, uint32_t b) {
    uint32_t r;
    asm volatile("sub.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t subc_cc(uint32_t a, uint32_t b) {
    uint32_t r;
    asm volatile("subc.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t subc(uint32_t a, uint32_t b) {
    uint32_t r;
    asm volatile("subc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}

// X from the byte sums S_b < 2^22: WP normalized 32-bit words.  With
// lo_w = S_4w + 2^8 S_4w+1 and hi_w = S_4w+2 + 2^8 S_4w+3 (both < 2^31),
// X = sum_w (lo_w + 2^16 hi_w) 2^(32 w): word w adds lo_w + (hi_(w-1) >> 16)
// (no overflow) and hi_w << 16 in one carry chain; X < 2^(32 WP) leaves no
// carry out of the top word.
template <int WP, int NB>
__device__ __forceinline__ void crt_bytesums_to_words(const uint32_t (&S)[NB], uint32_t (&x)[WP]) {
    uint32_t lo[WP], hi[WP];
#pragma unroll
    for (int w = 0; w < WP; ++w) {
        const uint32_t s0 = 4 * w < NB ? S[4 * w] : 0u, s1 = 4 * w + 1 < NB ? S[4 * w + 1] : 0u;
        const uint32_t s2 = 4 * w + 2 < NB ? S[4 * w + 2] : 0u,
                       s3 = 4 * w + 3 < NB ? S[4 * w + 3] : 0u;
        lo[w] = s0 + (s1 << 8);
        hi[w] = s2 + (s3 << 8);
    }
    x[0] = add_cc(lo[0], hi[0] << 16);
#pragma unroll
    for (int w = 1; w < WP; ++w) x[w] = addc_cc(lo[w] + (hi[w - 1] >> 16), hi[w] << 16);
}

// crt_reduce for normalized words x (0 <= x < 2^(32 WP)) with carry chains:
// G = X - q P as magnitude words + sign, the same words crt_reduce gives
template <int WP>
__device__ __forceinline__ bool crt_reduce_norm(const uint32_t (&x)[WP], const uint32_t *Pw,
                                                uint32_t q, uint32_t (&mag)[WP]) {
    uint32_t qp[WP], hi = 0;
#pragma unroll
    for (int w = 0; w < WP; ++w) {
        const uint64_t t = (uint64_t)q * Pw[w] + hi;
        qp[w] = (uint32_t)t;
        hi = (uint32_t)(t >> 32);
    }
    uint32_t y[WP];
    y[0] = sub_cc(x[0], qp[0]);
#pragma unroll
    for (int w = 1; w < WP; ++w) y[w] = subc_cc(x[w], qp[w]);
    const uint32_t flip = subc(0u, 0u);  // all ones when X < q P
    // |Y| = (Y ^ flip) - flip over all words (flip in every word is -1 or 0)
    mag[0] = sub_cc(y[0] ^ flip, flip);
#pragma unroll
    for (int w = 1; w < WP; ++w) mag[w] = subc_cc(y[w] ^ flip, flip);
    return flip != 0u;
}

// levels and columns of one task: Q = 1 digit level and 2 columns for
// Float64x2, 2 levels and 1 column for more limbs (2 slots either way)
template <int N>
struct CrtTcShape {
    static constexpr int Q = N == 2 ? 1 : 2, J = N == 2 ? 2 : 1, SLOTS = Q * J;
};

template <int N, int WP>
__global__ void __launch_bounds__(CRT_TC_THREADS)
    crt_accum_tc_kernel(int64_t m, int64_t n, int h, int T, const uint8_t *R, int64_t ldi,
                        size_t plane, const int *rowexp, const int *colexp, Mat C, scal<N> alpha,
                        scal<N> beta, int flags, uint32_t tmem_cols, int *err,
                        const __grid_constant__ CrtTcDev c) {
    constexpr int NB = CrtTcN<WP>::value, Q = CrtTcShape<N>::Q, J = CrtTcShape<N>::J,
                  SLOTS = CrtTcShape<N>::SLOTS;
    const int ksteps = (T + 31) >> 5, kchunks = 2 * ksteps;
    const int spt = 8 / kchunks;  // slots per operand tile
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t *sB = smem;            // NB rows x 128 B (a multiple of 1024 B)
    uint8_t *sA = smem + NB * 128;  // ceil(SLOTS / spt) tiles of 128 rows x 128 B
    uint64_t *done = (uint64_t *)(sA + (size_t)((SLOTS + spt - 1) / spt) * CRT_TC_ATILE);
    uint32_t *tmem_slot = (uint32_t *)(done + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    // B: row b = bytes b of U_0 .. U_63; 16-byte chunk ch of a row sits at
    // chunk position ch ^ (b & 7) of the 128-byte swizzle
    for (int e = threadIdx.x; e < NB * 4; e += CRT_TC_THREADS) {
        const int b = e >> 2, ch = e & 3;
        const uint4 v = make_uint4(c.ub[b][4 * ch], c.ub[b][4 * ch + 1], c.ub[b][4 * ch + 2],
                                   c.ub[b][4 * ch + 3]);
        *(uint4 *)(sB + (b >> 3) * 1024 + (b & 7) * 128 + ((ch ^ (b & 7)) << 4)) = v;
    }
    if (threadIdx.x == 0) {
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    constexpr uint32_t idesc = idesc_u8(128, NB);

    const int64_t mblk = (m + 127) >> 7, tasks = mblk * ((n + J - 1) / J);
    uint32_t phase = 0;
    for (int64_t task = blockIdx.x; task < tasks; task += gridDim.x) {
        const int64_t i0 = (task % mblk) * 128, j0 = (task / mblk) * J;
        // flags bit 2: lower triangle only (the GEMM skipped the tiles above it)
        if ((flags & 4) && i0 + 127 < j0) continue;
        // debug builds: the task's 128 rows lie inside the padded planes
        if (!MFLAB_IDX_OK(i0 + 128 <= ldi, 4, i0, j0)) continue;
        // 1. residue segments -> K-major rows (rows i0 .. i0+127 lie inside the
        //    padded planes; columns j >= n read nothing)
        for (int pr = warp; pr < SLOTS * kchunks; pr += CRT_TC_THREADS / 32) {
            const int ch = pr % kchunks, sl = pr / kchunks, jj = sl / Q, L = sl % Q;
            const int64_t j = j0 + jj;
            const uint8_t *src = R + (size_t)L * T * plane + (size_t)j * ldi + i0 + 4 * lane;
            uint32_t w[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                const int t = 16 * ch + u;
                w[u] = (t < T && j < n) ? __ldg((const uint32_t *)(src + (size_t)t * plane)) : 0u;
            }
            uint8_t *dst = sA + (size_t)(sl / spt) * CRT_TC_ATILE;
            const int cl = (sl % spt) * kchunks + ch;  // logical chunk of the row
#pragma unroll
            for (int st = 0; st < 4; ++st) {
                const int rr = (st + (lane >> 1)) & 3, row = 4 * lane + rr;
                const uint32_t sel = (uint32_t)rr | ((uint32_t)(rr + 4) << 4);
                uint32_t o[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const uint32_t lo = __byte_perm(w[4 * q], w[4 * q + 1], sel);
                    const uint32_t hi = __byte_perm(w[4 * q + 2], w[4 * q + 3], sel);
                    o[q] = __byte_perm(lo, hi, 0x5410);
                }
                *(uint4 *)(dst + row * 128 + ((cl ^ (row & 7)) << 4)) =
                    make_uint4(o[0], o[1], o[2], o[3]);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // 2. the task's MMAs
        if (threadIdx.x == 0) {
            for (int sl = 0; sl < SLOTS; ++sl) {
                const uint32_t a0 = smem_u32(sA + (size_t)(sl / spt) * CRT_TC_ATILE) +
                                    (uint32_t)(sl % spt) * 32u * (uint32_t)ksteps;
                for (int ks = 0; ks < ksteps; ++ks)
                    mma_i8(tmem + (uint32_t)(sl * NB), smem_desc_sw128(a0 + 32 * ks),
                           smem_desc_sw128(smem_u32(sB) + 32 * ks), idesc, (uint32_t)ks);
            }
            mma_commit(done);
        }
        // the CTA's own MMAs: the drain bound, one decision for the whole CTA
        const bool ok = mbar_wait(done, phase, TC_DRAIN_LIMIT);
        phase ^= 1;
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) atomicExch(err, TC_ERR_DRAIN);
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // 3. one row per thread: the SLOTS sums of its entries side by side
        const int64_t i = i0 + 32 * warp + lane;
        const int ea = i < m ? rowexp[i] : 0;
        uint32_t S[SLOTS][NB];
        __syncwarp();
#pragma unroll
        for (int sl = 0; sl < SLOTS; ++sl) {
            uint32_t v0[16], v1[16], v2[16];
            const uint32_t ta = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(sl * NB);
            tmem_ld16_async(ta, v0);
            tmem_ld16_async(ta + 16, v1);
            if constexpr (NB > 32) tmem_ld16_async(ta + 32, v2);
            tmem_wait_ld();
            tmem_pin(v0);
            tmem_pin(v1);
            if constexpr (NB > 32) tmem_pin(v2);
#pragma unroll
            for (int b = 0; b < 16; ++b) {
                S[sl][b] = v0[b];
                S[sl][16 + b] = v1[b];
                if constexpr (NB > 32) S[sl][32 + b] = v2[b];
            }
        }
        mf<N> g[SLOTS];
#pragma unroll
        for (int sl = 0; sl < SLOTS; ++sl) {
            const int jj = sl / Q, L = sl % Q;
            const int64_t j = j0 + jj;
            const int eb = j < n ? colexp[j] : 0;
            uint32_t x[WP];
            crt_bytesums_to_words<WP, NB>(S[sl], x);
            double xd = (double)x[WP - 1];
#pragma unroll
            for (int w = WP - 2; w >= 0; --w) xd = fma(xd, 4294967296.0, (double)x[w]);
            const uint32_t q = (uint32_t)floor(xd * c.pinv + 0.5);
            uint32_t mag[WP];
            const bool ng = crt_reduce_norm<WP>(x, c.P, q, mag);
            const int sh = oz_scale_exp(ea) + oz_scale_exp(eb) - 2 * Q * h + h * (2 * Q - 2 - L);
            g[sl] = crt_words_to_mf<N, WP>(mag, sh);
            if (ng) g[sl] = neg(g[sl]);
        }
#pragma unroll
        for (int jj = 0; jj < J; ++jj) {
            const int64_t j = j0 + jj;
            mf<N> acc = g[jj * Q + Q - 1];
#pragma unroll
            for (int L = Q - 2; L >= 0; --L) acc = add(acc, g[jj * Q + L]);
            if (j < n && i < m && !((flags & 4) && i < j)) {
                const int eb = colexp[j];
                if (ea == OZ_EXP_BAD || eb == OZ_EXP_BAD)
                    acc = from_double<N>(__longlong_as_double(0x7ff8000000000000LL));
                // flags bit 0: beta == 0 (C is not read); bit 1: alpha == 1
                mf<N> r = (flags & 2) ? acc : mul(alpha.get(), acc);
                if (!(flags & 1)) r = add(r, mul(beta.get(), load_mf<N>(C.p, C.ld, C.ls, i, j)));
                store_mf<N>(C.p, C.ld, C.ls, i, j, r);
            }
        }
        __syncwarp();
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(tmem_cols)
                     : "memory");
    }
}

// residues of int32 sums modulo p as bytes (library-engine path)
__global__ void crt_mod_kernel(const int32_t *G, uint8_t *R, size_t count, int p) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    int r = G[e] % p;
    R[e] = (uint8_t)(r < 0 ? r + p : r);
}

// ----------------------------------------------------------- host side ---
// little-endian base-2^32 integers for the constants
using Big = std::vector<uint32_t>;

static Big big_mul_small(const Big &a, uint32_t s) {
    Big r(a.size() + 1, 0);
    uint64_t cy = 0;
    for (size_t i = 0; i < a.size(); ++i) {
        const uint64_t v = (uint64_t)a[i] * s + cy;
        r[i] = (uint32_t)v;
        cy = v >> 32;
    }
    r[a.size()] = (uint32_t)cy;
    while (r.size() > 1 && r.back() == 0) r.pop_back();
    return r;
}

static Big big_div_small(const Big &a, uint32_t s, uint32_t *rem) {
    Big r(a.size(), 0);
    uint64_t cur = 0;
    for (size_t i = a.size(); i-- > 0;) {
        cur = (cur << 32) | a[i];
        r[i] = (uint32_t)(cur / s);
        cur %= s;
    }
    if (rem) *rem = (uint32_t)cur;
    while (r.size() > 1 && r.back() == 0) r.pop_back();
    return r;
}

static int big_bitlen(const Big &a) {
    for (size_t i = a.size(); i-- > 0;)
        if (a[i]) {
            int b = 0;
            while (b < 32 && (a[i] >> b)) ++b;
            return (int)i * 32 + b;
        }
    return 0;
}

static uint32_t inv_mod(uint32_t a, uint32_t p) {
    int64_t t = 0, nt = 1, r = p, nr = a % p;
    while (nr) {
        const int64_t qq = r / nr;
        int64_t tmp = t - qq * nt;
        t = nt;
        nt = tmp;
        tmp = r - qq * nr;
        r = nr;
        nr = tmp;
    }
    if (t < 0) t += p;
    return (uint32_t)t;
}

struct CrtTables {
    CrtAccConst acc;
    CrtAccDev dev;
    CrtTcDev tc;
    int bitlen;  // bit length of P
};

static const CrtSplitConst &crt_split_const() {
    static CrtSplitConst c;
    static std::once_flag once;
    std::call_once(once, [] {
        for (int t = 0; t < CRT_MAXT; ++t) {
            const uint32_t p = (uint32_t)crt_modulus(t);
            for (int j = 0; j < CRT_WD; ++j) {
                uint32_t word = 0;
                for (int u = 0; u < 4; ++u) {
                    uint32_t v = 1 % p;  // 2^(8 b) mod p, b = 4j + u
                    for (int b = 0; b < 4 * j + u; ++b) v = (v * 256u) % p;
                    word |= v << (8 * u);
                }
                c.wt[t][j] = word;
            }
            for (int wd = 3; wd <= CRT_WD; ++wd) {
                uint32_t v = 1 % p;  // 2^(32 wd) mod p
                for (int b = 0; b < 32 * wd; ++b) v = (v * 2u) % p;
                c.negoff[wd - 3][t] = (128u % p + p - v) % p;
            }
        }
    });
    return c;
}

static const CrtTables &crt_tables(int T) {
    static CrtTables tab[CRT_MAXT + 1];
    static std::once_flag once[CRT_MAXT + 1];
    std::call_once(once[T], [T] {
        CrtTables &c = tab[T];
        memset(&c, 0, sizeof(c));
        Big P{1};
        for (int t = 0; t < T; ++t) P = big_mul_small(P, (uint32_t)crt_modulus(t));
        c.bitlen = big_bitlen(P);
        for (int t = 0; t < T; ++t) {
            const uint32_t p = (uint32_t)crt_modulus(t);
            uint32_t r = 0;
            const Big M = big_div_small(P, p, nullptr);
            big_div_small(M, p, &r);
            const Big U = big_mul_small(M, inv_mod(r, p));
            for (size_t w = 0; w < U.size() && w < (size_t)CRT_WP; ++w) c.acc.U[t][w] = U[w];
            for (int b = 0; b < 48; ++b) {
                const uint32_t byte = (size_t)(b >> 2) < U.size() ? (U[b >> 2] >> (8 * (b & 3))) & 0xffu : 0u;
                c.tc.ub[b][t >> 2] |= byte << (8 * (t & 3));
            }
            for (int cc = 0; cc < CRT_NC; ++cc) {
                uint64_t v = 0;  // bits [39 cc, 39 cc + 39) of U_t
                for (int b = 0; b < CRT_CW; ++b) {
                    const int bit = CRT_CW * cc + b, w = bit >> 5;
                    if ((size_t)w < U.size() && ((U[w] >> (bit & 31)) & 1u)) v |= 1ULL << b;
                }
                c.dev.Ud[t][cc] = (double)v;
            }
        }
        long double pd = 0.0L;
        for (size_t w = P.size(); w-- > 0;) pd = pd * 4294967296.0L + (long double)P[w];
        for (size_t w = 0; w < P.size() && w < (size_t)CRT_WP; ++w) c.acc.P[w] = P[w];
        c.acc.pinv = (double)(1.0L / pd);
        memcpy(c.dev.P, c.acc.P, sizeof(c.dev.P));
        c.dev.pinv = c.acc.pinv;
        memcpy(c.tc.P, c.acc.P, sizeof(c.tc.P));
        c.tc.pinv = c.acc.pinv;
    });
    return tab[T];
}

static int ceil_log2(int64_t v) {
    int l = 0;
    while ((1LL << l) < v) ++l;
    return l;
}

struct CrtPlan {
    int Q, h, T, WD, WP;
    int64_t kp, mp, np, ldi;
    size_t plane, plane8a, plane8b, a8, b8, lev, ws, total;
};

// largest digit width h that T moduli support for Q digits and padded depth
// kp, with P > 2 max|G_L| for every level sum G_L:
//   Q = 1: the scaled entry is below 2^(h-1) (1 + 2^-52) in magnitude and
//          every limb rounds by at most 1/2, so |D| <= 2^(h-1) (1 + 2^(3-h))
//          and |G| <= kp 2^(2h-2) 1.002; 2h <= fl - log2(kp) gives
//          2 |G| < 2^fl <= P;
//   Q = 2: digits are bounded by 2^(h+1) (the second one carries the
//          remainder of the first), level sums have up to 2 kp terms, and
//          P > 2 Q kp 2^(2h+2) is kept.
static int crt_h_for(int T, int Q, int64_t kp) {
    const int fl = crt_tables(T).bitlen - 1;  // P >= 2^fl
    const int h = Q == 1 ? (fl - ceil_log2(kp)) / 2 : (fl - ceil_log2((int64_t)Q * kp) - 4) / 2;
    return h < CRT_MAXH ? h : CRT_MAXH;
}

static void crt_layout(CrtPlan &p);

// Plan of one call.  T_req > 0: that many moduli, digits as wide as they
// allow; T_req == 0: the tuner's requirement from the sampled scale gap.
// Returns MFLAB_ERR_UNSUPPORTED when no table entry reaches the requirement.
static int crt_plan(int N, int64_t m, int64_t n, int64_t k, int T_req, int gap8, CrtPlan &p) {
    p.kp = (k + 127) / 128 * 128;
    if (p.kp == 0) p.kp = 128;
    if (T_req > 0) {
        if (T_req > CRT_MAXT) return MFLAB_ERR_ARG;
        p.Q = N == 2 ? 1 : 2;
        p.T = T_req;
        p.h = crt_h_for(p.T, p.Q, p.kp);
    } else {
        // bits below the row/column scale needed: working precision
        // 53 N + 1, the sampled gap, a 6-bit margin and 1 bit for the
        // (-1/2, 1/2) scaling; Q = 2 adds 1 bit for the dropped levels
        const double gap = gap8 > 0 ? gap8 / 8.0 : 0.0;
        const int beta = (int)ceil(53.0 * N + 1.0 + gap + 6.0 + 1.0);
        p.Q = N == 2 ? 1 : 2;
        p.h = p.Q == 1 ? beta : (beta + 2) / 2;
        p.T = 0;
        for (int T = 1; T <= CRT_MAXT; ++T)
            if (crt_h_for(T, p.Q, p.kp) >= p.h) {
                p.T = T;
                break;
            }
        if (p.T == 0 || p.h > CRT_MAXH) return MFLAB_ERR_UNSUPPORTED;
    }
    if (p.h < 8) return MFLAB_ERR_UNSUPPORTED;
    if ((int64_t)p.Q * p.kp * 16384 >= 2147483648LL) return MFLAB_ERR_UNSUPPORTED;
    p.WD = (p.h + 3 + 31) / 32;  // |digit| <= 2^(h+1) plus a sign bit
    if (p.WD < 3) p.WD = 3;
    const int need = crt_tables(p.T).bitlen + 14;  // X < T 256 P
    p.WP = need <= 256 ? 8 : need <= 320 ? 10 : 12;
    p.mp = (m + 127) / 128 * 128;
    p.np = (n + 255) / 256 * 256;
    crt_layout(p);
    return MFLAB_OK;
}

// buffer layout of a plan whose padded shapes mp, np are set
static void crt_layout(CrtPlan &p) {
    p.ldi = p.mp;
    p.plane = ((size_t)p.ldi * p.np + 255) / 256 * 256;
    p.plane8a = (size_t)p.mp * p.Q * p.kp;
    p.plane8b = (size_t)p.np * p.Q * p.kp;
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    p.a8 = al((size_t)p.T * p.plane8a);
    p.b8 = al((size_t)p.T * p.plane8b);
    p.lev = al((size_t)p.Q * p.T * p.plane);                 // byte residues
    p.ws = ((size_t)64 << 20) + al(p.plane * sizeof(int32_t));  // library path only
    p.total = p.a8 + p.b8 + p.lev + p.ws;
}

template <int N, int WD>
static void crt_split(const CrtPlan &p, int64_t m, int64_t n, int64_t k, Mat A, Mat B,
                      const int *rowexp, const int *colexp, int8_t *A8, int8_t *B8,
                      cudaStream_t s) {
    const CrtSplitConst &c = crt_split_const();
    const dim3 ga = crt_split_a_grid<N>(p.mp, p.kp);
    crt_split_a_kernel<N, WD><<<ga, dim3(32, 8), 0, s>>>(m, p.mp, k, p.kp, p.Q, p.h, p.T, A,
                                                         rowexp, A8, p.plane8a, 0, c);
    const dim3 gb = crt_split_b_grid<N>(p.np, p.kp);
    crt_split_b_kernel<N, WD><<<gb, 128, 0, s>>>(k, n, p.np, p.kp, p.Q, p.h, p.T, B, colexp, B8,
                                                 p.plane8b, 1, c);
}

// the left operand alone (rows of A -> A8) or the right one alone (B -> B8)
template <int N, int WD>
static void crt_split_one(const CrtPlan &p, bool left, int64_t rows, int64_t k, Mat X,
                          const int *exps, int8_t *X8, cudaStream_t s) {
    const CrtSplitConst &c = crt_split_const();
    if (left) {
        const dim3 ga = crt_split_a_grid<N>(p.mp, p.kp);
        crt_split_a_kernel<N, WD><<<ga, dim3(32, 8), 0, s>>>(rows, p.mp, k, p.kp, p.Q, p.h, p.T, X,
                                                             exps, X8, p.plane8a, 0, c);
    } else {
        const dim3 gb = crt_split_b_grid<N>(p.np, p.kp);
        crt_split_b_kernel<N, WD><<<gb, 128, 0, s>>>(k, rows, p.np, p.kp, p.Q, p.h, p.T, X, exps,
                                                     X8, p.plane8b, 1, c);
    }
}

template <int N>
static void crt_split_one_n(const CrtPlan &p, bool left, int64_t rows, int64_t k, Mat X,
                            const int *exps, int8_t *X8, cudaStream_t s) {
    if (p.WD <= 3) crt_split_one<N, 3>(p, left, rows, k, X, exps, X8, s);
    else if (p.WD == 4) crt_split_one<N, 4>(p, left, rows, k, X, exps, X8, s);
    else crt_split_one<N, 5>(p, left, rows, k, X, exps, X8, s);
}

template <int N>
static void crt_split_n(const CrtPlan &p, int64_t m, int64_t n, int64_t k, Mat A, Mat B,
                        const int *rowexp, const int *colexp, int8_t *A8, int8_t *B8,
                        cudaStream_t s) {
    if (p.WD <= 3) crt_split<N, 3>(p, m, n, k, A, B, rowexp, colexp, A8, B8, s);
    else if (p.WD == 4) crt_split<N, 4>(p, m, n, k, A, B, rowexp, colexp, A8, B8, s);
    else crt_split<N, 5>(p, m, n, k, A, B, rowexp, colexp, A8, B8, s);
}

template <int N, int WP>
static void crt_accum(const CrtPlan &p, int64_t m, int64_t n, const uint8_t *I, const int *rowexp,
                      const int *colexp, Mat C, const scal<N> &al, const scal<N> &be,
                      int flags, cudaStream_t s) {
    dim3 g((unsigned)((m + CRT_ACC_ROWS - 1) / CRT_ACC_ROWS), (unsigned)n);
    crt_accum_kernel<N, WP><<<g, CRT_ACC_ROWS, 0, s>>>(m, n, p.Q, p.h, p.T, I, p.ldi, p.plane, rowexp,
                                              colexp, C, al, be, flags, crt_tables(p.T).dev);
}

// The tensor-core reconstruction: persistent CTAs, as many per SM as their
// TMEM allocations fit into the SM's 512 columns (the dynamic shared memory
// is raised until the occupancy says so, so no allocation ever waits).
// Returns false when the launch shape cannot be had (the caller then runs
// crt_accum).
template <int N, int WP>
static bool crt_accum_tc(const CrtPlan &p, int64_t m, int64_t n, const uint8_t *I,
                         const int *rowexp, const int *colexp, Mat C, const scal<N> &al,
                         const scal<N> &be, int flags, int *err, cudaStream_t s) {
    constexpr int NB = CrtTcN<WP>::value;
    if (p.T > 64 || m <= 0 || n <= 0 || p.Q != CrtTcShape<N>::Q) return false;
    constexpr int J = CrtTcShape<N>::J, slots = CrtTcShape<N>::SLOTS;
    const int spt = 8 / (2 * ((p.T + 31) / 32));
    uint32_t cols = 32;
    while ((int)cols < slots * NB) cols <<= 1;
    const int max_ctas = 512 / (int)cols;
    int dev = 0, sms = 0, smem_sm = 0, smem_blk = 0, reserved = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&smem_blk, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) !=
            cudaSuccess)
        return false;
    size_t smem = 1024 + (size_t)NB * 128 + (size_t)((slots + spt - 1) / spt) * CRT_TC_ATILE + 16;
    // at most max_ctas blocks of (smem + reserved) bytes on one SM
    const size_t floor_smem = (size_t)smem_sm / (size_t)(max_ctas + 1) + 1;
    if (smem + (size_t)reserved < floor_smem) smem = floor_smem - (size_t)reserved;
    smem = (smem + 127) / 128 * 128;
    if (smem > (size_t)smem_blk) return false;
    auto kern = crt_accum_tc_kernel<N, WP>;
    // the largest shared-memory carveout, so that as many CTAs as the
    // shared memory allows share an SM (the default lets the driver pick a
    // carveout that holds one)
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess ||
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared) != cudaSuccess)
        return false;
    // max_ctas per SM by the shared memory; the grid does not depend on how
    // many of them are resident at once (tasks carry no dependencies)
    const int64_t tasks = (m + 127) / 128 * ((n + J - 1) / J);
    const int64_t slots_all = (int64_t)sms * max_ctas;
    const int grid = (int)(tasks < slots_all ? tasks : slots_all);
    kern<<<grid, CRT_TC_THREADS, smem, s>>>(m, n, p.h, p.T, I, p.ldi, p.plane, rowexp,
                                            colexp, C, al, be, flags, cols, err,
                                            crt_tables(p.T).tc);
    return true;
}

// the reconstruction: on the tensor cores with a tcgen05 engine, else (or
// when that launch shape is unavailable) crt_accum
template <int N>
static void crt_reconstruct(mflab_handle *hd, const CrtPlan &p, int64_t m, int64_t n,
                            const uint8_t *Rs, const int *rowexp, const int *colexp, Mat C,
                            const scal<N> &al, const scal<N> &be, int flags, cudaStream_t s) {
    if (tc_engine(hd)) {
        int *err = hd->dev_flags + 1;
        bool done = false;
        if (p.WP == 8) done = crt_accum_tc<N, 8>(p, m, n, Rs, rowexp, colexp, C, al, be, flags, err, s);
        else if (p.WP == 10) done = crt_accum_tc<N, 10>(p, m, n, Rs, rowexp, colexp, C, al, be, flags, err, s);
        else done = crt_accum_tc<N, 12>(p, m, n, Rs, rowexp, colexp, C, al, be, flags, err, s);
        if (done) return;
        (void)cudaGetLastError();
    }
    if (p.WP == 8) crt_accum<N, 8>(p, m, n, Rs, rowexp, colexp, C, al, be, flags, s);
    else if (p.WP == 10) crt_accum<N, 10>(p, m, n, Rs, rowexp, colexp, C, al, be, flags, s);
    else crt_accum<N, 12>(p, m, n, Rs, rowexp, colexp, C, al, be, flags, s);
}

// A8_ready: the residue planes of A from mflab_ozaki_crt_prepare (then the
// scratch holds no A planes and A is not read), or nullptr
template <int N>
static int crt_gemm_n(mflab_handle *hd, const CrtPlan &p, int64_t m, int64_t n, int64_t k, Mat A,
                      Mat B, Mat C, const double *alpha, const double *beta, const int *rowexp,
                      const int *colexp, cudaStream_t s, const int8_t *A8_ready = nullptr) {
    char *base = (char *)hd->scratch;
    const size_t a8 = A8_ready ? 0 : p.a8;
    int8_t *A8 = A8_ready ? (int8_t *)A8_ready : (int8_t *)base;
    int8_t *B8 = (int8_t *)(base + a8);
    uint8_t *Rs = (uint8_t *)(base + a8 + p.b8);
    char *ws = base + a8 + p.b8 + p.lev;
    ozaki_phase(0, s);
    if (A8_ready) crt_split_one_n<N>(p, false, n, k, B, colexp, B8, s);
    else crt_split_n<N>(p, m, n, k, A, B, rowexp, colexp, A8, B8, s);
    int rc = record_cuda_error(cudaGetLastError(), "modular split");
    if (rc) return rc;
    ozaki_phase(1, s);
    const int64_t ld8 = (int64_t)p.Q * p.kp;
    for (int L = 0; L < p.Q && rc == MFLAB_OK; ++L) {
        const int64_t K = (int64_t)(L + 1) * p.kp, bx = (int64_t)(p.Q - 1 - L) * p.kp;
        uint8_t *RL = Rs + (size_t)L * p.T * p.plane;
        if (tc_engine(hd)) {
            rc = int8_gemm_tc_mod(p.mp, p.np, K, A8, ld8, ld8, B8, ld8, ld8, bx, RL, p.ldi,
                                  hd->dev_flags + 1, s, tc_opts(hd), p.T, (int64_t)p.plane);
        } else {
            int32_t *G = (int32_t *)(ws + ((size_t)64 << 20));
            const size_t cnt = (size_t)p.ldi * p.np;
            for (int t = 0; t < p.T && rc == MFLAB_OK; ++t) {
                rc = int8_gemm_tn(p.mp, p.np, K, A8 + (size_t)t * p.plane8a, ld8,
                                  B8 + (size_t)t * p.plane8b + bx, ld8, G, p.ldi, ws,
                                  (size_t)64 << 20, s);
                if (rc) break;
                crt_mod_kernel<<<(unsigned)((cnt + 255) / 256), 256, 0, s>>>(
                    G, RL + (size_t)t * p.plane, cnt, crt_modulus(t));
                rc = record_cuda_error(cudaGetLastError(), "modular residues");
            }
        }
    }
    if (rc) return rc;
    ozaki_phase(2, s);
    scal<N> al{}, be{};
    int flags = 3;  // bit 0: beta == 0, bit 1: alpha == 1
    for (int l = 0; l < N; ++l) {
        al.v[l] = alpha[l];
        be.v[l] = beta[l];
        if (beta[l] != 0.0) flags &= ~1;
        if (alpha[l] != (l == 0 ? 1.0 : 0.0)) flags &= ~2;
    }
    crt_reconstruct<N>(hd, p, m, n, Rs, rowexp, colexp, C, al, be, flags, s);
    ozaki_phase(3, s);
    return record_cuda_error(cudaGetLastError(), "modular accumulate");
}

int ozaki_crt_gemm(mflab_handle *hd, int N, int T, int64_t m, int64_t n, int64_t k, Mat A, Mat B,
                   Mat C, const double *alpha, const double *beta, cudaStream_t s,
                   int *T_used) {
    if (T < 0 || T > CRT_MAXT) return MFLAB_ERR_ARG;
    if ((n + 255) / 256 * 256 > 65535LL || m > 0x3fffffffLL) return MFLAB_ERR_UNSUPPORTED;
    CrtPlan p;
    // the requirement check needs no device work when T is given
    int rc = T > 0 ? crt_plan(N, m, n, k, T, 0, p) : MFLAB_OK;
    if (rc) return rc;
    if ((int64_t)(T > 0 ? p.T : CRT_MAXT) * ((m + 127) / 128 * 128) > 0x7fffffffLL)
        return MFLAB_ERR_UNSUPPORTED;
    int *rowexp = nullptr, *colexp = nullptr;
    int g = 0;
    rc = ozaki_scales(hd, N, m, n, k, A, B, s, T == 0, &g, &rowexp, &colexp);
    if (rc) return rc;
    if (T == 0) {
        rc = crt_plan(N, m, n, k, 0, g, p);
        if (rc) return rc;
    }
    if ((int64_t)p.T * p.mp > 0x7fffffffLL || (int64_t)p.T * p.np > 0x7fffffffLL)
        return MFLAB_ERR_UNSUPPORTED;
    rc = mflab_reserve_scratch(hd, p.total);
    if (rc) return rc;
    if (T_used) *T_used = p.T;
    switch (N) {
    case 2: return crt_gemm_n<2>(hd, p, m, n, k, A, B, C, alpha, beta, rowexp, colexp, s);
    case 3: return crt_gemm_n<3>(hd, p, m, n, k, A, B, C, alpha, beta, rowexp, colexp, s);
    default: return crt_gemm_n<4>(hd, p, m, n, k, A, B, C, alpha, beta, rowexp, colexp, s);
    }
}

// ------------------------------------------------------ Gram products ---
// Residue digits of the one factor of lower(A A^T) (trans = 0, A n x k: the
// left operand's rows are A's rows) or lower(A^T A) (trans = 1, A k x n: its
// rows are A's columns).  The right operand is the same factor with the digit
// order reversed, identical for one digit.
template <int N, int WD>
static void crt_split_gram(const CrtPlan &p, int trans, int64_t n, int64_t k, Mat A,
                           const int *exps, int8_t *A8, int8_t *B8, cudaStream_t s) {
    const CrtSplitConst &c = crt_split_const();
    for (int role = 0; role < (p.Q == 1 ? 1 : 2); ++role) {
        int8_t *dst = role == 0 ? A8 : B8;
        if (trans == 0) {
            const dim3 ga = crt_split_a_grid<N>(p.mp, p.kp);
            crt_split_a_kernel<N, WD><<<ga, dim3(32, 8), 0, s>>>(n, p.mp, k, p.kp, p.Q, p.h, p.T, A,
                                                                 exps, dst, p.plane8a, role, c);
        } else {
            const dim3 gb = crt_split_b_grid<N>(p.np, p.kp);
            crt_split_b_kernel<N, WD><<<gb, 128, 0, s>>>(k, n, p.np, p.kp, p.Q, p.h, p.T, A, exps,
                                                         dst, p.plane8b, role, c);
        }
    }
}

template <int N>
static int crt_syrk_n(mflab_handle *hd, const CrtPlan &p, int trans, int64_t n, int64_t k, Mat A,
                      Mat C, const double *alpha, const double *beta, const int *exps,
                      cudaStream_t s) {
    char *base = (char *)hd->scratch;
    int8_t *A8 = (int8_t *)base;
    int8_t *B8 = p.Q == 1 ? A8 : (int8_t *)(base + p.a8);
    uint8_t *Rs = (uint8_t *)(base + p.a8 + p.b8);
    char *ws = base + p.a8 + p.b8 + p.lev;
    ozaki_phase(0, s);
    if (p.WD <= 3) crt_split_gram<N, 3>(p, trans, n, k, A, exps, A8, B8, s);
    else if (p.WD == 4) crt_split_gram<N, 4>(p, trans, n, k, A, exps, A8, B8, s);
    else crt_split_gram<N, 5>(p, trans, n, k, A, exps, A8, B8, s);
    int rc = record_cuda_error(cudaGetLastError(), "modular gram split");
    if (rc) return rc;
    ozaki_phase(1, s);
    const int64_t ld8 = (int64_t)p.Q * p.kp;
    for (int L = 0; L < p.Q && rc == MFLAB_OK; ++L) {
        const int64_t K = (int64_t)(L + 1) * p.kp, bx = (int64_t)(p.Q - 1 - L) * p.kp;
        uint8_t *RL = Rs + (size_t)L * p.T * p.plane;
        if (tc_engine(hd)) {
            rc = int8_gemm_tc_mod(p.mp, p.np, K, A8, ld8, ld8, B8, ld8, ld8, bx, RL, p.ldi,
                                  hd->dev_flags + 1, s, tc_opts(hd), p.T, (int64_t)p.plane, 1);
        } else {  // the library computes whole products; only the lower part is used
            int32_t *G = (int32_t *)(ws + ((size_t)64 << 20));
            const size_t cnt = (size_t)p.ldi * p.np;
            for (int t = 0; t < p.T && rc == MFLAB_OK; ++t) {
                rc = int8_gemm_tn(p.mp, p.np, K, A8 + (size_t)t * p.plane8a, ld8,
                                  B8 + (size_t)t * p.plane8b + bx, ld8, G, p.ldi, ws,
                                  (size_t)64 << 20, s);
                if (rc) break;
                crt_mod_kernel<<<(unsigned)((cnt + 255) / 256), 256, 0, s>>>(
                    G, RL + (size_t)t * p.plane, cnt, crt_modulus(t));
                rc = record_cuda_error(cudaGetLastError(), "modular residues");
            }
        }
    }
    if (rc) return rc;
    ozaki_phase(2, s);
    scal<N> al{}, be{};
    int flags = 3 | 4;  // bit 0: beta == 0, bit 1: alpha == 1, bit 2: lower triangle
    for (int l = 0; l < N; ++l) {
        al.v[l] = alpha[l];
        be.v[l] = beta[l];
        if (beta[l] != 0.0) flags &= ~1;
        if (alpha[l] != (l == 0 ? 1.0 : 0.0)) flags &= ~2;
    }
    crt_reconstruct<N>(hd, p, n, n, Rs, exps, exps, C, al, be, flags, s);
    ozaki_phase(3, s);
    return record_cuda_error(cudaGetLastError(), "modular gram accumulate");
}

// lower(C) = alpha op(A) op(A)^T + beta lower(C) through the modular route,
// op(A) = A (trans = 0, A n x k) or A^T (trans = 1, A k x n); the strict
// upper triangle of C is neither read nor written.
int ozaki_crt_syrk(mflab_handle *hd, int N, int T, int trans, int64_t n, int64_t k, Mat A, Mat C,
                   const double *alpha, const double *beta, cudaStream_t s, int *T_used) {
    if (T < 0 || T > CRT_MAXT) return MFLAB_ERR_ARG;
    const int64_t np = (n + 255) / 256 * 256;
    if (np > 65535LL) return MFLAB_ERR_UNSUPPORTED;
    CrtPlan p;
    int rc = T > 0 ? crt_plan(N, n, n, k, T, 0, p) : MFLAB_OK;
    if (rc) return rc;
    int *exps = nullptr;
    int g = 0;
    rc = ozaki_gram_scales(hd, N, trans, n, k, A, s, T == 0, &g, &exps);
    if (rc) return rc;
    if (T == 0) {
        rc = crt_plan(N, n, n, k, 0, g, p);
        if (rc) return rc;
    }
    p.mp = p.np = np;  // square tile grid: the GEMM walks the lower-triangle tiles
    crt_layout(p);
    if ((int64_t)p.T * p.mp > 0x7fffffffLL) return MFLAB_ERR_UNSUPPORTED;
    rc = mflab_reserve_scratch(hd, p.total);
    if (rc) return rc;
    if (T_used) *T_used = p.T;
    switch (N) {
    case 2: return crt_syrk_n<2>(hd, p, trans, n, k, A, C, alpha, beta, exps, s);
    case 3: return crt_syrk_n<3>(hd, p, trans, n, k, A, C, alpha, beta, exps, s);
    default: return crt_syrk_n<4>(hd, p, trans, n, k, A, C, alpha, beta, exps, s);
    }
}

}  // namespace mfl

// C = alpha*A*B + beta*C through the modular INT8 route; moduli = 0 lets the
// sampled-gap tuner choose (one stream synchronisation).  Same argument
// conventions and checks as mflab_gemm_ozaki.
extern "C" int mflab_gemm_ozaki_crt(mflab_handle *h, void *stream, int limbs, int moduli,
                                    int64_t m, int64_t n, int64_t k, const double *A, int64_t lda,
                                    int64_t lsa, const double *B, int64_t ldb, int64_t lsb,
                                    double *C, int64_t ldc, int64_t lsc, const double *alpha,
                                    const double *beta) {
    MFLAB_RANGE("mflab_gemm_ozaki_crt");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (m < 0 || n < 0 || k < 0 || !alpha || !beta) return MFLAB_ERR_ARG;
    if (m == 0 || n == 0) return MFLAB_OK;
    if (lda < (m > 0 ? m : 1) || ldb < (k > 0 ? k : 1) || ldc < m) return MFLAB_ERR_ARG;
    if (mfl::views_overlap(C, ldc, lsc, m, n, limbs, A, lda, lsa, m, k) ||
        mfl::views_overlap(C, ldc, lsc, m, n, limbs, B, ldb, lsb, k, n))
        return MFLAB_ERR_ALIAS;
    if (moduli < 0) return MFLAB_ERR_ARG;
    if (k == 0)
        return mfl::launch_mm(limbs, false, false, 0, false, m, n, k,
                              mfl::Mat{(double *)A, lda, lsa}, mfl::Mat{(double *)B, ldb, lsb},
                              mfl::Mat{C, ldc, lsc}, alpha, beta, (cudaStream_t)stream);
    return mfl::ozaki_crt_gemm(h, limbs, moduli, m, n, k, mfl::Mat{(double *)A, lda, lsa},
                               mfl::Mat{(double *)B, ldb, lsb}, mfl::Mat{C, ldc, lsc}, alpha,
                               beta, (cudaStream_t)stream, &h->last_moduli);
}

extern "C" int mflab_ozaki_last_moduli(mflab_handle *h) { return h ? h->last_moduli : 0; }

// The modulus count mflab_gemm_ozaki_crt(moduli = 0) would choose for these
// operands (the same scale pass and sampled gap, one stream
// synchronisation), without the product: a caller that prepares A once for
// many products with it takes the count from here.  Products at that count
// use digits as wide as the count allows (crt_h_for), at least as wide as
// the tuned call's.
extern "C" int mflab_ozaki_crt_tune(mflab_handle *h, void *stream, int limbs, int64_t m,
                                    int64_t n, int64_t k, const double *A, int64_t lda,
                                    int64_t lsa, const double *B, int64_t ldb, int64_t lsb,
                                    int *moduli) {
    MFLAB_RANGE("mflab_ozaki_crt_tune");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (m < 1 || n < 1 || k < 1 || !moduli) return MFLAB_ERR_ARG;
    if (lda < m || ldb < k) return MFLAB_ERR_ARG;
    if ((n + 255) / 256 * 256 > 65535LL || m > 0x3fffffffLL) return MFLAB_ERR_UNSUPPORTED;
    int *rowexp = nullptr, *colexp = nullptr;
    int g = 0;
    int rc = mfl::ozaki_scales(h, limbs, m, n, k, mfl::Mat{(double *)A, lda, lsa},
                               mfl::Mat{(double *)B, ldb, lsb}, (cudaStream_t)stream, 1, &g,
                               &rowexp, &colexp);
    if (rc) return rc;
    mfl::CrtPlan p;
    rc = mfl::crt_plan(limbs, m, n, k, 0, g, p);
    if (rc) return rc;
    *moduli = p.T;
    return MFLAB_OK;
}

// lower(C) = alpha * op(A) op(A)^T + beta * lower(C) through the modular
// route: trans = 0, A n x k (the trailing-update form A A^T); trans = 1, A
// k x n (the reference syrk! form P^T P).  moduli = 0: tuner.
extern "C" int mflab_syrk_lower_ozaki(mflab_handle *h, void *stream, int limbs, int moduli,
                                      int trans, int64_t n, int64_t k, const double *A,
                                      int64_t lda, int64_t lsa, double *C, int64_t ldc,
                                      int64_t lsc, const double *alpha, const double *beta) {
    MFLAB_RANGE("mflab_syrk_lower_ozaki");
    if (!h || !mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (trans != 0 && trans != 1) return MFLAB_ERR_FLAG;
    if (n < 0 || k < 0 || !alpha || !beta || moduli < 0) return MFLAB_ERR_ARG;
    if (n == 0) return MFLAB_OK;
    const int64_t ar = trans ? k : n, ac = trans ? n : k;
    if (lda < (ar > 0 ? ar : 1) || ldc < n) return MFLAB_ERR_ARG;
    if (mfl::views_overlap(C, ldc, lsc, n, n, limbs, A, lda, lsa, ar, ac)) return MFLAB_ERR_ALIAS;
    const mfl::Mat Am{(double *)A, lda, lsa}, Cm{C, ldc, lsc};
    cudaStream_t s = (cudaStream_t)stream;
    if (k == 0)  // C = beta C on the lower triangle
        return mfl::launch_mm(limbs, trans ? 1 : 0, !trans, 1, false, n, n, 0, Am, Am, Cm, alpha,
                              beta, s);
    return mfl::ozaki_crt_syrk(h, limbs, moduli, trans, n, k, Am, Cm, alpha, beta, s,
                               &h->last_moduli);
}



// Host-only planner of the modular route (no device work): for `limbs`, depth
// k and either a modulus count (moduli > 0) or the tuner's sampled gap in
// eighths of a bit (moduli == 0), the digit count Q, digit width h and
// modulus count T a call would use.
extern "C" int mflab_ozaki_crt_plan(int limbs, int64_t k, int moduli, int gap8, int *Q, int *h,
                                    int *T) {
    if (!mfl::valid_limbs(limbs) || k < 0 || moduli < 0 || !Q || !h || !T) return MFLAB_ERR_ARG;
    mfl::CrtPlan p;
    const int rc = mfl::crt_plan(limbs, 1, 1, k, moduli, gap8, p);
    if (rc) return rc;
    *Q = p.Q;
    *h = p.h;
    *T = p.T;
    return MFLAB_OK;
}

// Host copy of the reconstruction step for tests: for `count` problems, G
// holds T int32 values per problem (any representatives of the residues
// mod p_t, as the int8 GEMMs produce them); mag receives 12 little-endian
// words of |x| and neg the sign of the x with |x| <= 3P/8 and x = G_t mod
// p_t for all t (the range the planner guarantees for every level sum).
extern "C" int mflab_ozaki_crt_reduce_host(int T, int count, const int32_t *G, uint32_t *mag,
                                           int *neg) {
    using namespace mfl;
    if (T < 1 || T > CRT_MAXT || count < 0 || !G || !mag || !neg) return MFLAB_ERR_ARG;
    // the device's arithmetic: residues as exact doubles, FMA chunk sums
    const CrtAccDev &c = crt_tables(T).dev;
    for (int e = 0; e < count; ++e) {
        double A[CrtChunks<CRT_WP>::value] = {0.0};
        for (int t = 0; t < T; ++t) {
            const int p = crt_modulus(t);
            int r = G[(size_t)e * T + t] % p;
            r += r < 0 ? p : 0;
            for (int cc = 0; cc < CrtChunks<CRT_WP>::value; ++cc)
                A[cc] = fma((double)r, c.Ud[t][cc], A[cc]);
        }
        uint64_t X[CRT_WP];
        crt_chunks_to_words<CRT_WP>(A, X);
        uint32_t mg[CRT_WP];
        neg[e] = crt_reduce<CRT_WP>(X, c.P, crt_quotient<CRT_WP>(A, c.pinv), mg) ? 1 : 0;
        for (int w = 0; w < CRT_WP; ++w) mag[(size_t)e * CRT_WP + w] = mg[w];
    }
    return MFLAB_OK;
}

// modulus t of the table (0 <= t < count), or the table size for t < 0
extern "C" int mflab_ozaki_crt_modulus(int t) {
    if (t < 0) return mfl::CRT_MAXT;
    return t < mfl::CRT_MAXT ? mfl::crt_modulus(t) : 0;
}

// mflab_gemm_ozaki_crt with per-phase device times (ms[0] scales + tuning,
// ms[1] residue split, ms[2] int8 GEMMs, ms[3] reconstruction) and the
// integer multiply-add operations of the GEMMs (2 m n K summed).  Synchronises.
extern "C" int mflab_gemm_ozaki_crt_phases(mflab_handle *h, void *stream, int limbs, int moduli,
                                           int64_t m, int64_t n, int64_t k, const double *A,
                                           int64_t lda, int64_t lsa, const double *B,
                                           int64_t ldb, int64_t lsb, double *C, int64_t ldc,
                                           int64_t lsc, const double *alpha, const double *beta,
                                           float *ms, double *int8_ops) {
    MFLAB_RANGE("mflab_gemm_ozaki_crt_phases");
    if (!h || !ms || !int8_ops) return MFLAB_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t ev[5];
    for (auto &e : ev) cudaEventCreate(&e);
    cudaEventRecord(ev[4], s);
    mfl::ozaki_set_phase_events(ev);
    int rc = mflab_gemm_ozaki_crt(h, stream, limbs, moduli, m, n, k, A, lda, lsa, B, ldb, lsb, C,
                                  ldc, lsc, alpha, beta);
    mfl::ozaki_set_phase_events(nullptr);
    if (rc == MFLAB_OK) {
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = mfl::record_cuda_error(e, "modular phases");
    }
    if (rc == MFLAB_OK) {
        cudaEventElapsedTime(&ms[0], ev[4], ev[0]);
        cudaEventElapsedTime(&ms[1], ev[0], ev[1]);
        cudaEventElapsedTime(&ms[2], ev[1], ev[2]);
        cudaEventElapsedTime(&ms[3], ev[2], ev[3]);
        mfl::CrtPlan p;
        mfl::crt_plan(limbs, m, n, k, h->last_moduli, 0, p);
        const double kp = (double)p.kp, mp = (double)p.mp, np = (double)p.np;
        *int8_ops = 2.0 * mp * np * kp * (double)p.T * p.Q * (p.Q + 1) / 2.0;
    }
    for (auto &e : ev) cudaEventDestroy(e);
    return rc;
}

// ------------------------------------------------ prepared left operand ---
// A Float64xN matrix used as the left operand of many modular GEMMs (the
// residual B - A X of every refinement step): its row exponents and residue
// planes for a fixed modulus count, computed once into caller memory.
// Layout: rowexp[m] int32 (rounded up to 256 bytes), then the residue planes
// A8[T][mp][Q kp] of the plan.
namespace {
size_t prep_rowexp_bytes(int64_t m) { return ((size_t)m * sizeof(int) + 255) / 256 * 256; }
int prep_plan(int N, int T, int64_t m, int64_t n, int64_t k, mfl::CrtPlan &p) {
    if (!mfl::valid_limbs(N)) return MFLAB_ERR_UNSUPPORTED;
    if (T <= 0 || T > mfl::CRT_MAXT) return MFLAB_ERR_FLAG;
    if (m < 0 || n < 0 || k < 1) return MFLAB_ERR_ARG;
    if ((n + 255) / 256 * 256 > 65535LL || m > 0x3fffffffLL) return MFLAB_ERR_UNSUPPORTED;
    int rc = mfl::crt_plan(N, m, n, k, T, 0, p);
    if (rc) return rc;
    if ((int64_t)p.T * p.mp > 0x7fffffffLL || (int64_t)p.T * p.np > 0x7fffffffLL)
        return MFLAB_ERR_UNSUPPORTED;
    return MFLAB_OK;
}
}  // namespace

extern "C" int mflab_ozaki_crt_prepare_bytes(int limbs, int moduli, int64_t m, int64_t k,
                                             size_t *bytes) {
    if (!bytes) return MFLAB_ERR_ARG;
    mfl::CrtPlan p;
    int rc = prep_plan(limbs, moduli, m, 1, k, p);
    if (rc) return rc;
    *bytes = prep_rowexp_bytes(m) + p.a8;
    return MFLAB_OK;
}

extern "C" int mflab_ozaki_crt_prepare(mflab_handle *h, void *stream, int limbs, int moduli,
                                       int64_t m, int64_t k, const double *A, int64_t lda,
                                       int64_t lsa, void *prep) {
    MFLAB_RANGE("mflab_ozaki_crt_prepare");
    if (!h) return MFLAB_ERR_UNSUPPORTED;
    mfl::CrtPlan p;
    int rc = prep_plan(limbs, moduli, m, 1, k, p);
    if (rc) return rc;
    if (!prep || (m > 0 && k > 0 && (!A || lda < m))) return MFLAB_ERR_ARG;
    if (m == 0) return MFLAB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const mfl::Mat Am{(double *)A, lda, lsa};
    int *rowexp = (int *)prep;
    int8_t *A8 = (int8_t *)prep + prep_rowexp_bytes(m);
    rc = mfl::ozaki_row_exps(limbs, m, k, Am, rowexp, s);
    if (rc) return rc;
    switch (limbs) {
    case 2: mfl::crt_split_one_n<2>(p, true, m, k, Am, rowexp, A8, s); break;
    case 3: mfl::crt_split_one_n<3>(p, true, m, k, Am, rowexp, A8, s); break;
    default: mfl::crt_split_one_n<4>(p, true, m, k, Am, rowexp, A8, s); break;
    }
    return mfl::record_cuda_error(cudaGetLastError(), "modular prepare");
}

extern "C" int mflab_gemm_ozaki_crt_prepared(mflab_handle *h, void *stream, int limbs, int moduli,
                                             int64_t m, int64_t n, int64_t k, const void *prep,
                                             const double *B, int64_t ldb, int64_t lsb, double *C,
                                             int64_t ldc, int64_t lsc, const double *alpha,
                                             const double *beta) {
    MFLAB_RANGE("mflab_gemm_ozaki_crt_prepared");
    if (!h) return MFLAB_ERR_UNSUPPORTED;
    mfl::CrtPlan p;
    int rc = prep_plan(limbs, moduli, m, n, k, p);
    if (rc) return rc;
    if (!prep || !alpha || !beta || (n > 0 && k > 0 && (!B || ldb < k)) ||
        (m > 0 && n > 0 && ldc < m))
        return MFLAB_ERR_ARG;
    if (m == 0 || n == 0) return MFLAB_OK;
    if (mfl::views_overlap(C, ldc, lsc, m, n, limbs, B, ldb, lsb, k, n)) return MFLAB_ERR_ALIAS;
    cudaStream_t s = (cudaStream_t)stream;
    rc = mflab_reserve_scratch(h, p.total - p.a8);
    if (rc) return rc;
    rc = mflab_reserve_aux(h, sizeof(int) * (size_t)(n + 64));
    if (rc) return rc;
    int *colexp = (int *)h->aux;
    const mfl::Mat Bm{(double *)B, ldb, lsb}, Cm{C, ldc, lsc};
    rc = mfl::ozaki_col_exps(limbs, k, n, Bm, colexp, s);
    if (rc) return rc;
    const int *rowexp = (const int *)prep;
    const int8_t *A8 = (const int8_t *)prep + prep_rowexp_bytes(m);
    h->last_moduli = p.T;
    const mfl::Mat none{nullptr, 0, 0};
    switch (limbs) {
    case 2: return mfl::crt_gemm_n<2>(h, p, m, n, k, none, Bm, Cm, alpha, beta, rowexp, colexp, s, A8);
    case 3: return mfl::crt_gemm_n<3>(h, p, m, n, k, none, Bm, Cm, alpha, beta, rowexp, colexp, s, A8);
    default: return mfl::crt_gemm_n<4>(h, p, m, n, k, none, Bm, Cm, alpha, beta, rowexp, colexp, s, A8);
    }
}
