// Multi-double (Float64x2/x3/x4) arithmetic on the FP64 pipe.
//
// Every operation is written with the explicit round-to-nearest intrinsics
// (__dadd_rn, __dsub_rn, __dmul_rn, __fma_rn) so that the compiler can never
// contract or reassociate an error-free transformation.  Networks (reference
// paths are inside MultiFloatLinearAlgebra.jl):
//   two_sum       Knuth TwoSum; MultiFloats.two_sum as called at
//                 src/kernels/mulacc_x3.jl:29-33
//   fast_two_sum  Dekker; benchmark/ordered_twosum.jl:10-15
//   two_prod      product + FMA error (docs/MULACC_X3_PROOF_CONTRACT.md:37)
//   add3          src/kernels/mulacc_x3.jl:41-59
//   mul3          src/kernels/mulacc_x3.jl:20-39 + benchmark/fused_mulacc_x3.jl:59-71
//   mulacc3       src/kernels/mulacc_x3.jl:61-66
//   add4          benchmark/ordered_twosum.jl:46-82 with plain TwoSum
//   add2, mul2    Joldes-Muller-Popescu 2017 AccurateDWPlusDW / DWTimesDW3
//   mul4          Hida-Li-Bailey 2001 quad-double product structure, TwoSum
//                 accumulation by order, branch-free renormalisation
//   div           long division with N+1 quotient digits
//   sqrt          binary64 root followed by two Heron steps
// The x2 add/mul, x4 mul, div and sqrt of MultiFloats.jl 3.2.6 are not part of
// the reference, so those networks are this library's own choice.
#pragma once
#include <cstdint>

namespace mfl {

template <int N>
struct mf {
    double v[N];
};

__device__ __forceinline__ void two_sum(double a, double b, double &s, double &e) {
    double t = __dadd_rn(a, b);
    double ap = __dsub_rn(t, b);
    double bp = __dsub_rn(t, ap);
    double da = __dsub_rn(a, ap);
    double db = __dsub_rn(b, bp);
    s = t;
    e = __dadd_rn(da, db);
}

__device__ __forceinline__ void fast_two_sum(double a, double b, double &s, double &e) {
    double t = __dadd_rn(a, b);
    double bp = __dsub_rn(t, a);
    s = t;
    e = __dsub_rn(b, bp);
}

__device__ __forceinline__ void two_prod(double a, double b, double &p, double &e) {
    double t = __dmul_rn(a, b);
    p = t;
    e = __fma_rn(a, b, -t);
}

#define MFL_TS(a, b) two_sum((a), (b), (a), (b))
#define MFL_FTS(a, b) fast_two_sum((a), (b), (a), (b))

// --------------------------------------------------- x1 (plain binary64) ---
// The binary64 instance of the kernels serves the FP64 factor of the
// mixed-precision LU solver; it has no reference counterpart.
__device__ __forceinline__ mf<1> add(const mf<1> &x, const mf<1> &y) {
    return mf<1>{{__dadd_rn(x.v[0], y.v[0])}};
}
__device__ __forceinline__ mf<1> mul(const mf<1> &x, const mf<1> &y) {
    return mf<1>{{__dmul_rn(x.v[0], y.v[0])}};
}

// ------------------------------------------------------------------ x2 ---
__device__ __forceinline__ mf<2> add(const mf<2> &x, const mf<2> &y) {
    double sh = x.v[0], sl = y.v[0], th = x.v[1], tl = y.v[1];
    MFL_TS(sh, sl);
    MFL_TS(th, tl);
    double c = __dadd_rn(sl, th);
    MFL_FTS(sh, c);
    double w = __dadd_rn(tl, c);
    MFL_FTS(sh, w);
    return mf<2>{{sh, w}};
}

__device__ __forceinline__ mf<2> mul(const mf<2> &x, const mf<2> &y) {
    double ch, cl1;
    two_prod(x.v[0], y.v[0], ch, cl1);
    double tl = __dmul_rn(x.v[0], y.v[1]);
    double cl2 = __fma_rn(x.v[1], y.v[0], tl);
    double cl3 = __dadd_rn(cl1, cl2);
    MFL_FTS(ch, cl3);
    return mf<2>{{ch, cl3}};
}

// ------------------------------------------------------------------ x3 ---
__device__ __forceinline__ mf<3> raw_add3(double x0, double x1, double x2, double y0, double y1,
                                          double y2) {
    double a = x0, b = y0, c = x1, d = y1, e = x2, f = y2;
    MFL_TS(a, b);
    MFL_TS(c, d);
    MFL_TS(e, f);
    MFL_FTS(a, c);
    b = __dadd_rn(b, f);
    MFL_TS(d, e);
    MFL_FTS(a, d);
    MFL_TS(b, c);
    c = __dadd_rn(c, e);
    MFL_TS(c, d);
    MFL_TS(b, c);
    MFL_FTS(a, b);
    c = __dadd_rn(c, d);
    MFL_FTS(b, c);
    MFL_FTS(a, b);
    MFL_FTS(b, c);
    return mf<3>{{a, b, c}};
}

__device__ __forceinline__ mf<3> add(const mf<3> &x, const mf<3> &y) {
    return raw_add3(x.v[0], x.v[1], x.v[2], y.v[0], y.v[1], y.v[2]);
}

__device__ __forceinline__ void prefix3(const mf<3> &x, const mf<3> &y, double &q0, double &q1,
                                        double &q2) {
    double p00, e00, p01, e01, p10, e10;
    two_prod(x.v[0], y.v[0], p00, e00);
    two_prod(x.v[0], y.v[1], p01, e01);
    two_prod(x.v[1], y.v[0], p10, e10);
    double p02 = __dmul_rn(x.v[0], y.v[2]);
    double p11 = __dmul_rn(x.v[1], y.v[1]);
    double p20 = __dmul_rn(x.v[2], y.v[0]);
    MFL_TS(p01, p10);
    e01 = __dadd_rn(e01, e10);
    p02 = __dadd_rn(p02, p20);
    MFL_TS(e00, p01);
    p02 = __dadd_rn(p02, p11);
    MFL_FTS(p00, e00);
    p01 = __dadd_rn(p01, p10);
    e01 = __dadd_rn(e01, p02);
    p01 = __dadd_rn(p01, e01);
    q0 = p00;
    q1 = e00;
    q2 = p01;
}

__device__ __forceinline__ mf<3> mul(const mf<3> &x, const mf<3> &y) {
    double p0, p1, p2;
    prefix3(x, y, p0, p1, p2);
    MFL_TS(p1, p2);
    MFL_FTS(p0, p1);
    MFL_FTS(p1, p2);
    MFL_FTS(p0, p1);
    return mf<3>{{p0, p1, p2}};
}

__device__ __forceinline__ mf<3> mulacc3(const mf<3> &acc, const mf<3> &x, const mf<3> &y) {
    double p0, p1, p2;
    prefix3(x, y, p0, p1, p2);
    MFL_TS(p1, p2);
    return raw_add3(acc.v[0], acc.v[1], acc.v[2], p0, p1, p2);
}

// ------------------------------------------------------------------ x4 ---
__device__ __forceinline__ mf<4> add(const mf<4> &x, const mf<4> &y) {
    double a = x.v[0], b = y.v[0], c = x.v[1], d = y.v[1];
    double e = x.v[2], f = y.v[2], g = x.v[3], h = y.v[3];
    MFL_TS(a, b);
    MFL_TS(c, d);
    MFL_TS(e, f);
    MFL_TS(g, h);
    MFL_FTS(a, c);
    b = __dadd_rn(b, h);
    MFL_TS(d, e);
    MFL_TS(f, g);
    MFL_TS(b, g);
    MFL_FTS(c, d);
    MFL_TS(e, f);
    MFL_FTS(a, c);
    MFL_FTS(d, e);
    MFL_TS(b, d);
    MFL_FTS(c, g);
    e = __dadd_rn(e, f);
    MFL_TS(b, c);
    MFL_TS(d, e);
    MFL_FTS(a, b);
    MFL_TS(c, d);
    e = __dadd_rn(e, g);
    MFL_FTS(b, c);
    MFL_TS(d, e);
    MFL_FTS(a, b);
    MFL_FTS(c, d);
    MFL_FTS(b, c);
    d = __dadd_rn(d, e);
    MFL_FTS(a, b);
    MFL_FTS(c, d);
    MFL_FTS(b, c);
    MFL_FTS(c, d);
    return mf<4>{{a, b, c, d}};
}

__device__ __forceinline__ mf<4> mul(const mf<4> &x, const mf<4> &y) {
    double p00, e00, p01, e01, p10, e10, p02, e02, p11, e11, p20, e20;
    two_prod(x.v[0], y.v[0], p00, e00);
    two_prod(x.v[0], y.v[1], p01, e01);
    two_prod(x.v[1], y.v[0], p10, e10);
    two_prod(x.v[0], y.v[2], p02, e02);
    two_prod(x.v[1], y.v[1], p11, e11);
    two_prod(x.v[2], y.v[0], p20, e20);
    double q3 = __dmul_rn(x.v[0], y.v[3]);
    q3 = __dadd_rn(q3, __dmul_rn(x.v[1], y.v[2]));
    q3 = __dadd_rn(q3, __dmul_rn(x.v[2], y.v[1]));
    q3 = __dadd_rn(q3, __dmul_rn(x.v[3], y.v[0]));
    double s1 = p01, u = p10;
    MFL_TS(s1, u);
    double v = s1;
    s1 = e00;
    MFL_TS(s1, v);
    double s2 = p02, w1 = p20;
    MFL_TS(s2, w1);
    double w2 = p11;
    MFL_TS(s2, w2);
    double w3 = e01;
    MFL_TS(s2, w3);
    double w4 = e10;
    MFL_TS(s2, w4);
    double w5 = u;
    MFL_TS(s2, w5);
    double w6 = v;
    MFL_TS(s2, w6);
    double s3 = __dadd_rn(q3, e02);
    s3 = __dadd_rn(s3, e11);
    s3 = __dadd_rn(s3, e20);
    s3 = __dadd_rn(s3, w1);
    s3 = __dadd_rn(s3, w2);
    s3 = __dadd_rn(s3, w3);
    s3 = __dadd_rn(s3, w4);
    s3 = __dadd_rn(s3, w5);
    s3 = __dadd_rn(s3, w6);
    double s0 = p00;
    MFL_TS(s2, s3);
    MFL_TS(s1, s2);
    MFL_TS(s0, s1);
    MFL_FTS(s0, s1);
    MFL_FTS(s1, s2);
    MFL_FTS(s2, s3);
    return mf<4>{{s0, s1, s2, s3}};
}

#undef MFL_TS
#undef MFL_FTS

// ------------------------------------------------------------- generic ---
// acc + a*b with the network the reference uses for that limb count and route
template <int N, bool FUSED3>
__device__ __forceinline__ mf<N> mac(const mf<N> &acc, const mf<N> &a, const mf<N> &b) {
    if constexpr (N == 3 && FUSED3) {
        return mulacc3(acc, a, b);
    } else {
        return add(acc, mul(a, b));
    }
}

template <int N>
__device__ __forceinline__ mf<N> neg(const mf<N> &x) {
    mf<N> r;
#pragma unroll
    for (int l = 0; l < N; ++l) r.v[l] = -x.v[l];
    return r;
}

template <int N>
__device__ __forceinline__ mf<N> sub(const mf<N> &x, const mf<N> &y) {
    return add(x, neg(y));
}

// x - a*b, the reference's `x -= a * b`
template <int N>
__device__ __forceinline__ mf<N> submul(const mf<N> &x, const mf<N> &a, const mf<N> &b) {
    return sub(x, mul(a, b));
}

template <int N>
__device__ __forceinline__ mf<N> from_double(double d) {
    mf<N> r;
    r.v[0] = d;
#pragma unroll
    for (int l = 1; l < N; ++l) r.v[l] = 0.0;
    return r;
}

template <int N>
__device__ __forceinline__ bool iszero(const mf<N> &x) {
    bool z = true;
#pragma unroll
    for (int l = 0; l < N; ++l) z = z && (x.v[l] == 0.0);
    return z;
}

template <int N>
__device__ __forceinline__ bool isfinite_mf(const mf<N> &x) {
    bool f = true;
#pragma unroll
    for (int l = 0; l < N; ++l) f = f && isfinite(x.v[l]);
    return f;
}

// lexicographic limb order: the value order for normalised values
template <int N>
__device__ __forceinline__ bool lt(const mf<N> &x, const mf<N> &y) {
#pragma unroll
    for (int l = 0; l < N; ++l) {
        if (x.v[l] < y.v[l]) return true;
        if (x.v[l] > y.v[l]) return false;
    }
    return false;
}

template <int N>
__device__ __forceinline__ bool gt(const mf<N> &x, const mf<N> &y) {
    return lt(y, x);
}

template <int N>
__device__ __forceinline__ bool ge(const mf<N> &x, const mf<N> &y) {
#pragma unroll
    for (int l = 0; l < N; ++l) {
        if (x.v[l] > y.v[l]) return true;
        if (x.v[l] < y.v[l]) return false;
        if (!(x.v[l] == y.v[l])) return false;
    }
    return true;
}

template <int N>
__device__ __forceinline__ mf<N> abs_mf(const mf<N> &x) {
    return signbit(x.v[0]) ? neg(x) : x;
}

// Base.max(x, y) = isless(y, x) ? x : y
template <int N>
__device__ __forceinline__ mf<N> max_mf(const mf<N> &x, const mf<N> &y) {
    return lt(y, x) ? x : y;
}
template <int N>
__device__ __forceinline__ mf<N> min_mf(const mf<N> &x, const mf<N> &y) {
    return lt(y, x) ? y : x;
}

template <int N>
__device__ __forceinline__ mf<N> div(const mf<N> &x, const mf<N> &y) {
    mf<N> r = x;
    double q[N + 1];
#pragma unroll
    for (int i = 0; i <= N; ++i) {
        q[i] = __ddiv_rn(r.v[0], y.v[0]);
        if (i < N) r = sub(r, mul(y, from_double<N>(q[i])));
    }
    mf<N> acc = from_double<N>(q[0]);
#pragma unroll
    for (int i = 1; i <= N; ++i) acc = add(acc, from_double<N>(q[i]));
    return acc;
}

__device__ __forceinline__ mf<1> div(const mf<1> &x, const mf<1> &y) {
    return mf<1>{{__ddiv_rn(x.v[0], y.v[0])}};
}

template <int N>
__device__ __forceinline__ mf<N> inv(const mf<N> &x) {
    return div(from_double<N>(1.0), x);
}

template <int N>
__device__ __forceinline__ mf<N> sqrt_mf(const mf<N> &x) {
    if (x.v[0] == 0.0) return from_double<N>(0.0);
    mf<N> s = from_double<N>(__dsqrt_rn(x.v[0]));
#pragma unroll
    for (int it = 0; it < 2; ++it) {
        s = add(s, div(x, s));
#pragma unroll
        for (int l = 0; l < N; ++l) s.v[l] = __dmul_rn(s.v[l], 0.5);
    }
    return s;
}

__device__ __forceinline__ mf<1> sqrt_mf(const mf<1> &x) { return mf<1>{{__dsqrt_rn(x.v[0])}}; }

// ----------------------------------------------------- plane access -------
// A Float64xN matrix is N column-major planes: limb l of (r, c) is
// P[l*ls + c*ld + r].
template <int N>
__device__ __forceinline__ mf<N> load_mf(const double *__restrict__ P, int64_t ld, int64_t ls,
                                         int64_t r, int64_t c) {
    mf<N> x;
#pragma unroll
    for (int l = 0; l < N; ++l) x.v[l] = P[l * ls + c * ld + r];
    return x;
}

template <int N>
__device__ __forceinline__ void store_mf(double *__restrict__ P, int64_t ld, int64_t ls, int64_t r,
                                         int64_t c, const mf<N> &x) {
#pragma unroll
    for (int l = 0; l < N; ++l) P[l * ls + c * ld + r] = x.v[l];
}

template <int N>
struct scal {
    double v[4];
    __device__ __forceinline__ mf<N> get() const {
        mf<N> r;
#pragma unroll
        for (int l = 0; l < N; ++l) r.v[l] = v[l];
        return r;
    }
};

}  // namespace mfl
