/*
 * Measurement helper of the mflab200 library (no counterpart in the
 * reference: it measures the FP64 pipe rate used as the roofline denominator
 * of the multi-double kernels).
 */
#ifndef MFLAB200_PROBE_H
#define MFLAB200_PROBE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
/* kind 0: dependent DFMA chains, kind 1: DADD/DSUB chains.  Launches
   blocks x threads threads, each with 8 chains of `iters` x 2 instructions, on
   `stream`; *instructions receives the FP64 instruction count.  `out` is a
   device buffer of blocks*threads doubles. */
int mflab_probe_fp64(void *stream, int kind, int blocks, int threads, int64_t iters, double *out,
                     double *instructions);

/* The INT8-slice GEMM (mflab_gemm_ozaki, same arguments) with per-phase device
   times in ms[4]: exponents + slice tuning, digit split, int8 level GEMMs,
   accumulation; *int8_ops = 2 m n roundup(k,16) S(S+1)/2.  Synchronises. */
int mflab_gemm_ozaki_phases(struct mflab_handle *h, void *stream, int limbs, int slices, int64_t m,
                            int64_t n, int64_t k, const double *A, int64_t lda, int64_t lsa,
                            const double *B, int64_t ldb, int64_t lsb, double *C, int64_t ldc,
                            int64_t lsc, const double *alpha, const double *beta, float *ms,
                            double *int8_ops);

/* mflab_gemm_ozaki_crt (same arguments) with per-phase device times in
   ms[4]: exponents + tuning, residue split, int8 GEMMs, reconstruction;
   *int8_ops = 2 m n roundup(k,128) T Q(Q+1)/2 of the padded shapes.
   Synchronises. */
int mflab_gemm_ozaki_crt_phases(struct mflab_handle *h, void *stream, int limbs, int moduli,
                                int64_t m, int64_t n, int64_t k, const double *A, int64_t lda,
                                int64_t lsa, const double *B, int64_t ldb, int64_t lsb, double *C,
                                int64_t ldc, int64_t lsc, const double *alpha, const double *beta,
                                float *ms, double *int8_ops);

/* Host copy of the modular route's reconstruction (tests): for `count`
   problems of T int32 residue representatives each (G[e*T + t] ~ x mod p_t),
   the 12 little-endian 32-bit words of |x| (mag[e*12 ...]) and its sign
   (neg[e]) for the x with |x| <= 3P/8 (the range the route's planner keeps
   every level sum in).  No device work. */
int mflab_ozaki_crt_reduce_host(int T, int count, const int32_t *G, uint32_t *mag, int *neg);

/* Best device time (ms) of `reps` int8 x int8 -> int32 TN GEMMs of m x n x k
   through the library path the INT8 routes can use, on operands of constant
   bytes (fill 0) or of uniformly distributed bytes (fill 1, the operand
   statistics of the routes: the tensor pipe's power, and so its clock under
   the power cap, depends on the data).  Synchronises. */
int mflab_probe_int8_gemm(struct mflab_handle *h, void *stream, int64_t m, int64_t n, int64_t k,
                          int reps, int fill, float *ms);

/* One int8 x int8 -> int32 GEMM C = A[:, 0:K] * B[:, b_xoff:b_xoff+K]^T with
   K-major operands (A mp x a_cols, B np x b_cols, leading dims in bytes) and
   column-major C (ldc >= mp), through engine MFLAB_INT8_TCGEN05 (one-SM
   tcgen05 kernel), MFLAB_INT8_TCGEN05_PAIR (SM-pair kernel) — both need
   mp % 128 == 0, np % 256 == 0, K % 128 == 0 — or MFLAB_INT8_LIBRARY.  *err
   (device int) receives the kernel's bounded-wait status.  Used by the tests
   and the roofline probe. */
int mflab_int8_gemm_tn(struct mflab_handle *h, void *stream, int engine, int64_t mp, int64_t np,
                       int64_t K, const int8_t *A, int64_t lda, int64_t a_cols, const int8_t *B,
                       int64_t ldb, int64_t b_cols, int64_t b_xoff, int32_t *C, int64_t ldc,
                       int *err);

/* Test hooks of the tcgen05 kernels issued through this handle: wait_limit
   bounds their waits of one role on another (mbarrier polls; 0 restores the
   default), inject = 1 makes the MMA issuer of each launch first wait a
   short fixed bound on a barrier nothing arrives on, so that wait runs out
   with copies in flight and the kernel takes its timeout path (error code in the device status word,
   every issued copy and MMA drained, TMEM freed).  Nothing faults or hangs;
   the next launch with inject = 0 runs normally.  No reference counterpart. */
int mflab_set_tc_debug(struct mflab_handle *h, int64_t wait_limit, int inject);

/* Index checks of a debug build (libmflab200_debug.so, compiled with
   -DMFLAB_DEBUG): out[0] = the number of failed device index checks since
   the last reset, out[1..3] = the first one's check code and two index
   values (codes: 1 TMA coordinate off the 16-byte rule or past K, 2 int8 GEMM
   epilogue store outside the padded output, 3 residue split past its row,
   4 reconstruction task outside the residue planes, 5 moved-row list of the
   binary64 LU panel full, 6 GEMM column stride below the row count, 7 solve
   step load outside its matrix, 8 interleaved copy strides).  A failed check
   skips the access instead of trapping.  reset != 0 clears the records.
   A release build always reports zeros.  mflab_debug_build() is 1 in a debug
   build. */
int mflab_debug_violations(long long *out, int reset);
int mflab_debug_build(void);
#ifdef __cplusplus
}
#endif
#endif
