/*
 * mflab200: C ABI of the B200 (sm_100a) multi-double dense linear-algebra
 * backend for Float64x2 / Float64x3 / Float64x4.
 *
 * Every entry point replaces a Julia generic function of
 * MultiFloatLinearAlgebra.jl on the dense hot path; the citation on each
 * declaration is the reference function (path:line inside that project) whose
 * arguments, results and failure behaviour it keeps.
 *
 * Conventions
 *   - A Float64xN matrix lives in device memory as N column-major binary64
 *     planes ("limb planes"): limb l of element (r, c) (0-based) of matrix X
 *     is X[l*lsx + c*ldx + r].  ldx is the column stride, lsx the plane
 *     stride, both in doubles.  Sub-matrix views are plain pointer offsets.
 *   - `limbs` is N in {2, 3, 4}.  Scalars (alpha, beta) are HOST arrays of
 *     `limbs` doubles.
 *   - `stream` is a cudaStream_t (NULL = the legacy default stream).  All
 *     work is stream-ordered; nothing synchronises unless stated.
 *   - Return value: MFLAB_OK (0) or a negative MFLAB_ERR_* code for bad
 *     shapes (the reference's DimensionMismatch), bad option codes
 *     (ArgumentError), CUDA failures or bounded-wait timeouts.  Numerical status of a
 *     factorization (0, -1 non-finite input, k > 0 failing pivot) is written
 *     to a DEVICE int, exactly the reference's `info` field.
 *   - Pivot vectors are 1-based int64 on the device, as in the reference.
 *   - No entry point falls back to the CPU: without a usable device it
 *     returns an error.
 */
#ifndef MFLAB200_H
#define MFLAB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MFLAB_OK 0
#define MFLAB_ERR_ARG (-1)         /* shape / size / pointer error (DimensionMismatch) */
#define MFLAB_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define MFLAB_ERR_UNSUPPORTED (-3) /* limb count or option not supported */
#define MFLAB_ERR_TIMEOUT (-4)     /* a bounded device wait ran out */
#define MFLAB_ERR_ALLOC (-5)       /* device memory could not be reserved */
#define MFLAB_ERR_ALIAS (-6)       /* output aliases an input (types.jl:261-267) */
#define MFLAB_ERR_FLAG (-7)        /* an option code (side, uplo, trans, diag, route, order,
                                      region, engine) outside its range (ArgumentError,
                                      as trsv.jl:32-34 raises for a bad uplo / trans) */

/* GEMM routes (gemm.jl:44-136 gemm_plan strategies) */
#define MFLAB_GEMM_AUTO 0   /* reference :auto: fused mulacc for x3, direct otherwise */
#define MFLAB_GEMM_DIRECT 1 /* reference :direct: acc + a*b for every limb count */
#define MFLAB_GEMM_OZAKI 2  /* INT8-slice tensor-core route (no reference counterpart) */

/* triangular-solve orders (mflab_set_solve_order) */
#define MFLAB_ORDER_MATCHED 0 /* the reference's per-element chains: bitwise equal to it */
#define MFLAB_ORDER_FAST 1    /* terms applied as unknowns finalise, both directions:
                                 deterministic, not the reference's association */

/* engines of the int8 products of the INT8 routes (mflab_set_int8_engine) */
#define MFLAB_INT8_TCGEN05 0      /* the library's own tcgen05 / TMA / TMEM kernel, one CTA per SM */
#define MFLAB_INT8_LIBRARY 1      /* cuBLASLt int8 GEMM */
#define MFLAB_INT8_TCGEN05_PAIR 2 /* the library's own tcgen05 kernel on SM pairs (cta_group::2) */

typedef struct mflab_handle mflab_handle;

/* ------------------------------------------------------------ library --- */
/* library version as 10000*major + 100*minor + patch */
int mflab_version(void);
/* short description of an MFLAB_* code */
const char *mflab_status_string(int code);
/* message of the last error raised on the calling host thread ("" if none) */
const char *mflab_last_error(void);

/* A handle owns per-caller device scratch, like the reference's MFWorkspace
   (types.jl:71-123): one handle per concurrent caller. */
int mflab_create(mflab_handle **out, int device);
int mflab_destroy(mflab_handle *h);

/* Order of the backward substitutions issued through this handle (trsm,
   potrs, getrs, sytrs): MFLAB_ORDER_MATCHED (default) keeps the reference's
   per-row ascending chains (src/kernels/trsm.jl:18-112), which make each
   backward row wait for the previous one; MFLAB_ORDER_FAST applies every term
   as soon as its unknown is final.  No reference counterpart. */
int mflab_set_solve_order(mflab_handle *h, int order);

/* ----------------------------------------------------- device memory --- */
/* Device memory and stream-ordered copies for bindings without a CUDA
   runtime of their own (the Julia layer's MFDeviceMatrix planes and the
   4-byte info words of the factorizations live here).  kind: 0 host to
   device, 1 device to host, 2 device to device.  The reference works on host
   arrays and has no counterpart; these replace the Matrix{Float64xN}
   allocations a caller of gemm!/cholesky! (gemm.jl:747-755,
   cholesky.jl:68-107) would make. */
int mflab_malloc(int device, size_t bytes, void **ptr);
int mflab_free(void *ptr);
int mflab_memcpy(void *dst, const void *src, size_t bytes, int kind, void *stream);
int mflab_memset(void *dst, int value, size_t bytes, void *stream);
int mflab_stream_synchronize(void *stream);

/* ------------------------------------------- interleaved <-> limb planes --- */
/* A Julia Matrix{MultiFloat{Float64,N}} — the reference's operand type
   (AbstractMatrix{MultiFloat{Float64,N}}, src/kernels/gemm.jl:747-755,
   src/MultiFloatLinearAlgebra.jl:34-49) — stores the N limbs of each element
   together: limb l of element (r, c) at X[(c*ldx + r)*limbs + l], ldx in
   elements.  These four calls move such a matrix onto / off the limb planes
   P[l*ls + c*ld + r] the other entry points take, bit for bit (a permutation
   of doubles; limbs 1..4).  Stream-ordered.

   Host forms: `host` is host memory (pinned for an asynchronous copy;
   pageable memory is accepted, the copy then completes before the call
   returns).  They stage chunks through a buffer of two halves the handle
   allocates on first use, each half sized to the transfer (32 MiB to
   1 GiB, grown by a later larger transfer once the handle's copies are
   done), so two streams converting at once need two handles.
   Device forms: X is device memory; no staging, no allocation. */
int mflab_h2d_interleaved(mflab_handle *h, void *stream, int limbs, int64_t m, int64_t n,
                          const double *host, int64_t ldh, double *P, int64_t ld, int64_t ls);
int mflab_d2h_interleaved(mflab_handle *h, void *stream, int limbs, int64_t m, int64_t n,
                          const double *P, int64_t ld, int64_t ls, double *host, int64_t ldh);
int mflab_interleaved_to_planes(mflab_handle *h, void *stream, int limbs, int64_t m, int64_t n,
                                const double *X, int64_t ldx, double *P, int64_t ld, int64_t ls);
int mflab_planes_to_interleaved(mflab_handle *h, void *stream, int limbs, int64_t m, int64_t n,
                                const double *P, int64_t ld, int64_t ls, double *X, int64_t ldx);

/* ---------------------------------------------------------- BLAS-like --- */
/* C = alpha*A*B + beta*C; A m x k, B k x n, C m x n.  With beta == 0 C is not
   read.  route: MFLAB_GEMM_*.
   Replaces gemm!(C, A, B, alpha, beta; config) — src/kernels/gemm.jl:747-774. */
int mflab_gemm(mflab_handle *h, void *stream, int limbs, int route, int64_t m, int64_t n,
               int64_t k, const double *A, int64_t lda, int64_t lsa, const double *B, int64_t ldb,
               int64_t lsb, double *C, int64_t ldc, int64_t lsc, const double *alpha,
               const double *beta);

/* C = alpha*A*B + beta*C on the INT8 tensor cores (Ozaki scheme: exact
   signed 7-bit digit slices, int8 x int8 -> int32 level products, Float64xN
   accumulation).  slices = digit count S per operand; 0 lets the slice tuner
   choose S from the scale gap of 2048 sampled entries (one stream
   synchronisation).  The error is about k * 2^(row scale + column scale) *
   2^(-7S).  S is capped so that S * roundup(k, 16) * 65^2 < 2^31.  Uses handle scratch of about
   S*(m+n)*k bytes + 4*S*m*n bytes.  Non-finite input rows/columns give NaN.
   No reference counterpart: the gemm_strategy=:ozaki route of gemm!
   (src/kernels/gemm.jl:747-774 keeps the reference's signature). */
int mflab_gemm_ozaki(mflab_handle *h, void *stream, int limbs, int slices, int64_t m, int64_t n,
                     int64_t k, const double *A, int64_t lda, int64_t lsa, const double *B,
                     int64_t ldb, int64_t lsb, double *C, int64_t ldc, int64_t lsc,
                     const double *alpha, const double *beta);

/* data-independent digit count for `limbs` and reduction length k (a 24-bit
   scale-gap allowance; no reference counterpart). */
int mflab_ozaki_default_slices(int limbs, int64_t k);

/* slice count used by the last INT8-slice GEMM on this handle (no reference
   counterpart). */
int mflab_ozaki_last_slices(mflab_handle *h);

/* C = alpha*A*B + beta*C on the INT8 tensor cores through residues (Ozaki
   scheme II form): the scaled operands become Q integer digits of h bits
   (Float64x2: Q = 1; Float64x3/x4: Q = 2), each digit is reduced modulo
   `moduli` pairwise coprime numbers <= 256, one int8 GEMM per modulus and
   digit level gives the exact residues of the integer products, and the
   Chinese remainder theorem rebuilds them before the Float64xN accumulation.
   moduli = 0 lets the tuner choose from the sampled scale gap (one stream
   synchronisation); MFLAB_ERR_UNSUPPORTED when the requirement exceeds the
   modulus table (then use mflab_gemm_ozaki).  The error is about
   k * 2^(row scale + column scale) * 2^(-Q h).  Needs Q * roundup(k, 128) < 2^17.
   Handle scratch: about moduli * Q * (m + n) * k bytes + 4 * moduli * Q * m * n bytes.
   Non-finite input rows/columns give NaN.  No reference counterpart: a route
   of gemm! (src/kernels/gemm.jl:747-774 keeps the reference's signature). */
int mflab_gemm_ozaki_crt(mflab_handle *h, void *stream, int limbs, int moduli, int64_t m,
                         int64_t n, int64_t k, const double *A, int64_t lda, int64_t lsa,
                         const double *B, int64_t ldb, int64_t lsb, double *C, int64_t ldc,
                         int64_t lsc, const double *alpha, const double *beta);

/* A prepared left operand of the modular INT8 route, for many products
   C = alpha A B + beta C with one A (the residuals B - A X of iterative
   refinement): mflab_ozaki_crt_prepare stores A's row exponents and residue
   planes for `moduli` (1..49, fixed; else MFLAB_ERR_FLAG) in `prep`, caller-owned device memory of
   mflab_ozaki_crt_prepare_bytes(limbs, moduli, m, k) bytes; A is not read
   again.  mflab_gemm_ozaki_crt_prepared then splits only B and runs the same
   int8 GEMMs and reconstruction as mflab_gemm_ozaki_crt(moduli), with the
   same result bit for bit; limbs, moduli, m and k must be those of the
   preparation.  k >= 1.  No reference counterpart. */
int mflab_ozaki_crt_prepare_bytes(int limbs, int moduli, int64_t m, int64_t k, size_t *bytes);
int mflab_ozaki_crt_prepare(mflab_handle *h, void *stream, int limbs, int moduli, int64_t m,
                            int64_t k, const double *A, int64_t lda, int64_t lsa, void *prep);
int mflab_gemm_ozaki_crt_prepared(mflab_handle *h, void *stream, int limbs, int moduli, int64_t m,
                                  int64_t n, int64_t k, const void *prep, const double *B,
                                  int64_t ldb, int64_t lsb, double *C, int64_t ldc, int64_t lsc,
                                  const double *alpha, const double *beta);

/* lower(C) = alpha * op(A) * op(A)^T + beta * lower(C) through the modular
   INT8 route (the SYRK / trailing-update form of mflab_gemm_ozaki_crt):
   trans = 1 takes A as k x n and forms A^T A (the syrk!(C, P, alpha, beta)
   form, src/kernels/syrk.jl:67-108); trans = 0 takes A as n x k and forms
   A A^T (the Cholesky trailing update).  Only the 256 x 256 tiles that meet
   the lower triangle are multiplied; the strict upper triangle of C is
   neither read nor written.  moduli = 0: tuner (one stream synchronisation).
   No reference counterpart for the route itself. */
int mflab_syrk_lower_ozaki(mflab_handle *h, void *stream, int limbs, int moduli, int trans,
                           int64_t n, int64_t k, const double *A, int64_t lda, int64_t lsa,
                           double *C, int64_t ldc, int64_t lsc, const double *alpha,
                           const double *beta);

/* Blocked lower Cholesky with INT8 trailing updates: panels of nb columns are
   factored as in mflab_potrf (inner block `block` <= 32, reference order
   inside the panel, cholesky.jl:68-107), then the trailing matrix gets
   lower(A22) -= L21 L21^T through mflab_syrk_lower_ozaki (moduli = 0: tuned
   per update).  *info as mflab_potrf; the device info word is read after
   every panel (one synchronisation per panel). */
int mflab_potrf_ozaki(mflab_handle *h, void *stream, int limbs, int moduli, int64_t n, double *A,
                      int64_t lda, int64_t lsa, int64_t nb, int64_t block, int *info);

/* Blocked partial-pivoting LU with INT8 trailing updates: panels of nb
   columns are factored as in mflab_getrf (inner block `block`, reference
   order and full-row interchanges inside the panel, lu.jl:34-195), then U12
   by TRSM and A22 -= L21 U12 through mflab_gemm_ozaki_crt (moduli = 0: tuned
   per update).  ipiv and *info as mflab_getrf; the device info word is read
   after every panel (one synchronisation per panel). */
int mflab_getrf_ozaki(mflab_handle *h, void *stream, int limbs, int moduli, int64_t m, int64_t n,
                      double *A, int64_t lda, int64_t lsa, int64_t *ipiv, int64_t nb,
                      int64_t block, int *info);

/* modulus count used by the last mflab_gemm_ozaki_crt on this handle (no
   reference counterpart). */
int mflab_ozaki_last_moduli(mflab_handle *h);

/* The modulus count that mflab_gemm_ozaki_crt with moduli = 0 would choose
   for A (m x k) and B (k x n): the same scale pass and sampled scale gap, one
   stream synchronisation, no product.  A caller that prepares A once
   (mflab_ozaki_crt_prepare) takes the count from here.  A product at a given
   count uses digits as wide as that count allows, at least as wide as the
   tuned call's (which are only as wide as the sampled gap requires), so its
   error is at most the tuned call's; the low bits can differ from it.
   MFLAB_ERR_UNSUPPORTED when the requirement exceeds the modulus table.  No
   reference counterpart. */
int mflab_ozaki_crt_tune(mflab_handle *h, void *stream, int limbs, int64_t m, int64_t n,
                         int64_t k, const double *A, int64_t lda, int64_t lsa, const double *B,
                         int64_t ldb, int64_t lsb, int *moduli);

/* Host-only plan of mflab_gemm_ozaki_crt: digit count *Q, digit width *h
   (bits) and modulus count *T for `limbs`, depth k and either moduli > 0 or,
   with moduli == 0, a scale gap of gap8/8 bits (the tuner's input).  No
   device work; no reference counterpart. */
int mflab_ozaki_crt_plan(int limbs, int64_t k, int moduli, int gap8, int *Q, int *h, int *T);

/* modulus number t of the route's table (0 <= t < table size), or the table
   size when t < 0.  No reference counterpart. */
int mflab_ozaki_crt_modulus(int t);

/* Engine of the int8 level products of mflab_gemm_ozaki on this handle:
   MFLAB_INT8_TCGEN05 (default) or MFLAB_INT8_LIBRARY.  No reference
   counterpart. */
int mflab_set_int8_engine(mflab_handle *h, int engine);

/* Device-side status word of the tcgen05 kernels issued through this handle:
   0, or the code of a bounded wait that ran out (MFLAB_ERR_TIMEOUT is then
   the caller's conclusion: 1 producer, 2 MMA issuer, 3 epilogue, 4 drain).
   Reading it resets it to 0.  Synchronises.  No reference counterpart. */
int mflab_device_status(mflab_handle *h, int *status);

/* y = alpha * op(A) * x + beta * y: op(A) = A (trans 0, A m x n) or A^T
   (trans 1); one ascending chain per output with the plain network, y unread
   when beta == 0.  x, y contiguous with limb strides lsx, lsy.
   Replaces gemv!(y, A, x, alpha, beta; trans) — src/kernels/gemv.jl:99-167. */
int mflab_gemv(mflab_handle *h, void *stream, int limbs, int trans, int64_t m, int64_t n,
               const double *A, int64_t lda, int64_t lsa, const double *x, int64_t lsx, double *y,
               int64_t lsy, const double *alpha, const double *beta);

/* y = alpha * A * x + beta * y, A symmetric read from its lower (uplo 0) or
   upper (uplo 1) triangle only.
   Replaces symv!(y, A, x, alpha, beta; uplo) — src/kernels/symv.jl:43-89. */
int mflab_symv(mflab_handle *h, void *stream, int limbs, int uplo, int64_t n, const double *A,
               int64_t lda, int64_t lsa, const double *x, int64_t lsx, double *y, int64_t lsy,
               const double *alpha, const double *beta);

/* out (device, limbs doubles) = sum over the column-major index of x .* y for
   two m x n arrays, one ascending chain.
   Replaces mfdot(x, y) — src/kernels/dot.jl:1-22. */
int mflab_dot(mflab_handle *h, void *stream, int limbs, int64_t m, int64_t n, const double *x,
              int64_t ldx, int64_t lsx, const double *y, int64_t ldy, int64_t lsy, double *out);

/* lower(C) = alpha * P^T * P + beta * lower(C); P is k x n, C n x n.  The
   strict upper triangle of C is neither read nor written.
   Replaces syrk!(C, P, alpha, beta; uplo=:lower) — src/kernels/syrk.jl:67-108. */
int mflab_syrk_lower(mflab_handle *h, void *stream, int limbs, int64_t n, int64_t k,
                     const double *P, int64_t ldp, int64_t lsp, double *C, int64_t ldc,
                     int64_t lsc, const double *alpha, const double *beta);

/* Packed lower triangle C (column-major packed: (0,0),(1,0)..(n-1,0),(1,1)..,
   n(n+1)/2 entries per limb plane, limb stride lsc) = alpha * P[k0:k1,:]^T *
   P[k0:k1,:] + beta * C, P kp x n, 0 <= k0 < k1 <= kp (the reference's
   reduction_first - 1 and reduction_last); beta == 0 never reads C.
   Replaces syrk_packed!(packed, panel, alpha, beta; reduction_first,
   reduction_last) — src/kernels/syrk.jl:110-254. */
int mflab_syrk_packed(mflab_handle *h, void *stream, int limbs, int64_t n, int64_t kp,
                      int64_t k0, int64_t k1, const double *P, int64_t ldp, int64_t lsp,
                      double *C, int64_t lsc, const double *alpha, const double *beta);

/* lower(C) = alpha * A * B^T + beta * lower(C); A, B are n x k.
   Replaces gemmt!(C, A, B, alpha, beta) — src/kernels/gemmt.jl:69-108. */
int mflab_gemmt_lower(mflab_handle *h, void *stream, int limbs, int64_t n, int64_t k,
                      const double *A, int64_t lda, int64_t lsa, const double *B, int64_t ldb,
                      int64_t lsb, double *C, int64_t ldc, int64_t lsc, const double *alpha,
                      const double *beta);

/* side: 0 = left (op(A) X = alpha B, A m x m), 1 = right (X op(A) = alpha B,
   A n x n); uplo: 0 lower, 1 upper; trans: 0 N, 1 T; diag: 0 nonunit, 1 unit.
   B (m x n) is overwritten with X.
   Replaces trsm!(B, A, alpha; side, uplo, trans, diag) — src/kernels/trsm.jl:224-302,
   and for n == 1, side == 0 also trsv! — src/kernels/trsv.jl:19-73. */
int mflab_trsm(mflab_handle *h, void *stream, int limbs, int side, int uplo, int trans, int diag,
               int64_t m, int64_t n, const double *A, int64_t lda, int64_t lsa, double *B,
               int64_t ldb, int64_t lsb, const double *alpha);

/* B = alpha * op(A) * B (side 0, A m x m) or alpha * B * op(A) (side 1,
   A n x n), in place; uplo selects the triangle of A that is read, trans 0/1,
   diag 1 takes op(A)'s diagonal as one (never read).  Uses the handle's
   scratch for a copy of B (m n limbs doubles).
   Replaces trmm!(B, A, alpha; side, uplo, trans, diag) — src/kernels/trmm.jl:82-131. */
int mflab_trmm(mflab_handle *h, void *stream, int limbs, int side, int uplo, int trans, int diag,
               int64_t m, int64_t n, const double *A, int64_t lda, int64_t lsa, double *B,
               int64_t ldb, int64_t lsb, const double *alpha);

/* ---------------------------------------------------------- residuals --- */
/* R = B - A X (A m x k, X k x nrhs, B and R m x nrhs; R may equal B).
   uplo: 0 general, 1 symmetric from the lower triangle, 2 from the upper
   (m == k; the other triangle is never read).  vector_rhs selects the gemv!
   accumulation network for Float64x3 (gemm! takes the fused route).
   Replaces residual!(r, A, x, b; uplo) — src/residual.jl:55-125. */
int mflab_residual(mflab_handle *h, void *stream, int limbs, int uplo, int vector_rhs, int64_t m,
                   int64_t k, int64_t nrhs, const double *A, int64_t lda, int64_t lsa,
                   const double *X, int64_t ldx, int64_t lsx, const double *B, int64_t ldb,
                   int64_t lsb, double *R, int64_t ldr, int64_t lsr);

/* R = B - A X with every operand widened from src_limbs (1 = binary64) to
   res_limbs before the arithmetic; R has res_limbs planes.  Supported pairs:
   1 -> 2/3/4, 2 -> 3/4, 3 -> 4.
   Replaces residual_mixed!(r, A, x, b; uplo) — src/residual.jl:431-496 (which
   has 2 -> 3/4 and 3 -> 4; binary64 sources serve the mixed-precision LU). */
int mflab_residual_mixed(mflab_handle *h, void *stream, int src_limbs, int res_limbs, int uplo,
                         int64_t m, int64_t k, int64_t nrhs, const double *A, int64_t lda,
                         int64_t lsa, const double *X, int64_t ldx, int64_t lsx, const double *B,
                         int64_t ldb, int64_t lsb, double *R, int64_t ldr, int64_t lsr);

/* X <- X + widen(D): adds a src_limbs-limb correction (1 = binary64) to a
   dst_limbs-limb solution with the add network (the update step of iterative
   refinement; the reference leaves that loop to the caller,
   docs/SOLVER_BACKEND_CONTRACT.md:1-6).  m x n, 1 <= src < dst <= 4. */
int mflab_add_widened(mflab_handle *h, void *stream, int src_limbs, int dst_limbs, int64_t m,
                      int64_t n, const double *D, int64_t ldd, int64_t lsd, double *X, int64_t ldx,
                      int64_t lsx);

/* Normwise backward error ||r||inf / (||A||inf ||x||inf + ||b||inf) per
   right-hand-side column in the scaled form of the reference (0 for a zero
   denominator and zero residual, Inf otherwise, NaN for non-finite
   authoritative inputs).  out (device): nrhs values of `limbs` doubles.
   Replaces normwise_backward_error(A, x, b, r; uplo) — src/residual.jl:202-269. */
int mflab_backward_error(mflab_handle *h, void *stream, int limbs, int uplo, int64_t m, int64_t k,
                         int64_t nrhs, const double *A, int64_t lda, int64_t lsa, const double *X,
                         int64_t ldx, int64_t lsx, const double *B, int64_t ldb, int64_t lsb,
                         const double *R, int64_t ldr, int64_t lsr, double *out);

/* ||A||_inf (the matrix term of normwise_backward_error, residual.jl:178-200,
   same row-sum order) into device buffers anorm[limbs] and *nonfinite (1 when
   A holds a non-finite authoritative entry), for repeated backward errors
   against one matrix. */
int mflab_opnorm_inf(mflab_handle *h, void *stream, int limbs, int uplo, int64_t m, int64_t k,
                     const double *A, int64_t lda, int64_t lsa, double *anorm, int *nonfinite);

/* mflab_backward_error with ||A||_inf and its flag from mflab_opnorm_inf (A is
   not read): the iterative-refinement form. */
int mflab_backward_error_norm(mflab_handle *h, void *stream, int limbs, int64_t m, int64_t k,
                              int64_t nrhs, const double *anorm, const int *nonfinite,
                              const double *X, int64_t ldx, int64_t lsx, const double *B,
                              int64_t ldb, int64_t lsb, const double *R, int64_t ldr, int64_t lsr,
                              double *out);

/* ----------------------------------------------------- factorizations --- */
/* Blocked lower Cholesky in place (block <= 32 columns; the reference default
   is 16).  Only the lower triangle is read or written.  *info (device int):
   0 success, -1 non-finite lower triangle, k > 0 the first column whose
   Schur-complement diagonal is not positive.
   Replaces cholesky!(A; check=false, config) — src/factorizations/cholesky.jl:68-107. */
int mflab_potrf(mflab_handle *h, void *stream, int limbs, int64_t n, double *A, int64_t lda,
                int64_t lsa, int64_t block, int *info);

/* Rank-revealing pivoted Cholesky in place: the lower triangle is read,
   mirrored, and factored with symmetric diagonal pivoting; tol (host, limbs
   doubles, finite, >= 0) is the relative pivot threshold.  perm (device
   int64[n], 1-based) receives the symmetric permutation and rank_info
   (device int64[2]) the retained rank and the status: 0, -1 non-finite lower
   triangle (A unchanged), k > 0 the first non-positive pivot.
   Replaces cholesky_pivoted!(A; tol, check=false) —
   src/factorizations/cholesky_pivoted.jl:65-175. */
int mflab_pstrf(mflab_handle *h, void *stream, int limbs, int64_t n, double *A, int64_t lda,
                int64_t lsa, const double *tol, int64_t *perm, int64_t *rank_info);

/* Householder QR in place (pivoted = 0: qr!, the columns in their given
   order; pivoted = 1: rrqr!, deterministic column pivoting).  Reflectors
   below the diagonal, R on and above it; tau (device, r = min(m, n) values
   per limb plane, plane stride lst >= r); perm (device int64[n], 1-based):
   A_original[:, perm] = Q R; *info (device int): 0, or -1 for non-finite
   input (A unchanged, tau zero, identity permutation).
   Replaces qr!(A) — src/factorizations/qr.jl:763-811, and rrqr!(A) —
   src/factorizations/qr.jl:692-761. */
int mflab_qr(mflab_handle *h, void *stream, int limbs, int pivoted, int64_t m, int64_t n,
             double *A, int64_t lda, int64_t lsa, double *tau, int64_t lst, int64_t *perm,
             int *info);

/* D (m x nd) <- Q D (trans 0) or Q^T D (trans 1) with the first r reflectors
   of a QR factor F (m x >= r) and its tau.
   Replaces apply_q!(B, F; trans) — src/factorizations/qr.jl:890-956. */
int mflab_apply_q(mflab_handle *h, void *stream, int limbs, int trans, int64_t m, int64_t r,
                  const double *F, int64_t ldf, int64_t lsf, const double *tau, int64_t lst,
                  double *D, int64_t ldd, int64_t lsd, int64_t nd);

/* *rank (device int64) = leading count of |R[i,i]| > max(atol, rtol *
   max_i |R[i,i]|); atol, rtol host limbs.
   Replaces numerical_rank(F; atol, rtol) — src/factorizations/qr.jl:863-888. */
int mflab_qr_numerical_rank(mflab_handle *h, void *stream, int limbs, int64_t m, int64_t n,
                            const double *F, int64_t ldf, int64_t lsf, const double *atol,
                            const double *rtol, int64_t *rank);

/* B <- S^{-1} B with a successful Cholesky factor L (n x n), B n x nrhs.
   Replaces ldiv!(B, F::MFCholesky) — src/solve.jl:54-83 (vector form :23-50). */
int mflab_potrs(mflab_handle *h, void *stream, int limbs, int64_t n, int64_t nrhs,
                const double *L, int64_t ldl, int64_t lsl, double *B, int64_t ldb, int64_t lsb);

/* Blocked partial-pivoting LU in place; ipiv (device, min(m,n) int64,
   1-based) records the row swapped with row k at step k.  *info: 0, -1
   non-finite input, k > 0 exactly zero pivot at column k.  limbs may also be 1
   (plain binary64, the factor of the mixed-precision solver).
   Replaces lu!(A; check=false, config) — src/factorizations/lu.jl:128-195. */
int mflab_getrf(mflab_handle *h, void *stream, int limbs, int64_t m, int64_t n, double *A,
                int64_t lda, int64_t lsa, int64_t *ipiv, int64_t block, int *info);

/* B <- A^{-1} B with a successful LU factor: row interchanges, unit-lower
   then upper triangular solves.
   Replaces ldiv!(B, F::MFLU) — src/solve.jl:147-181 (vector form :115-145). */
int mflab_getrs(mflab_handle *h, void *stream, int limbs, int64_t n, int64_t nrhs,
                const double *LU, int64_t ldl, int64_t lsl, const int64_t *ipiv, double *B,
                int64_t ldb, int64_t lsb);

/* Repeated solves with one binary64 LU factor (the correction solves of the
   mixed-precision LU solver; no reference counterpart).  After mflab_getrf
   (limbs = 1), mflab_lu64_prepare stores in `work` (mflab_lu64_work_bytes(n)
   bytes of device memory, owned by the caller: 2 n^2 doubles and a little
   more) the row permutation of ipiv, the inverses of the 128 x 128 diagonal
   blocks of L and U, and each off-diagonal block column of L and U times its
   inverted diagonal block; mflab_lu64_solve then overwrites B (n x nrhs
   binary64, column-major) with inv(A) B: one gather and one kernel per block
   row and direction, reading only `work` (LU and ldl are checked, not read).
   Results differ from mflab_getrs in rounding only.  n <= 24576. */
int mflab_lu64_work_bytes(int64_t n, size_t *bytes);
int mflab_lu64_prepare(mflab_handle *h, void *stream, int64_t n, const double *LU, int64_t ldl,
                       const int64_t *ipiv, void *work);
int mflab_lu64_solve(mflab_handle *h, void *stream, int64_t n, int64_t nrhs, const double *LU,
                     int64_t ldl, const void *work, double *B, int64_t ldb);

/* Bunch-Kaufman LDL^T in place (lower triangle authoritative on input; the
   upper triangle is overwritten by the working mirror).  dsub (device,
   limbs planes of n doubles, plane stride lsd >= n) receives the off-diagonal
   of each 2x2 block, pivots (device int64, 1-based) the step pivots, blocks
   (device uint8) 1 / 2 at a block start and 0 on a 2x2 continuation.
   blocked = 0: the unblocked route; 1: the lazy-panel route with `block`
   columns per panel (<= 64; the reference uses 16/12/8 for x2/x3/x4 and
   blocks from n >= 512).  *info: 0, -1 non-finite lower triangle, k > 0 first
   singular step.  The blocked route synchronises the stream once per panel.
   Replaces ldlt!(A; check=false, config) — src/factorizations/ldlt.jl:654-717,
   ldlt_gemmt.jl:36-73. */
int mflab_sytrf(mflab_handle *h, void *stream, int limbs, int64_t n, double *A, int64_t lda,
                int64_t lsa, double *dsub, int64_t lsd, int64_t *pivots, uint8_t *blocks,
                int blocked, int64_t block, int *info);

/* B <- A^{-1} B with a successful LDLT factor: forward interchanges,
   unit-lower solve, block-diagonal solve, transposed unit-lower solve, reverse
   interchanges.  *fail (device int) is set to the 1-based start of a singular
   2x2 block, else to 0x7f7f7f7f.
   Replaces ldiv!(B, F::MFLDLT) — src/solve.jl:298-365. */
int mflab_sytrs(mflab_handle *h, void *stream, int limbs, int64_t n, int64_t nrhs, const double *F,
                int64_t ldf, int64_t lsf, const double *dsub, int64_t lsd, const int64_t *pivots,
                const uint8_t *blocks, double *B, int64_t ldb, int64_t lsb, int *fail);

/* Inertia and block quality of an LDLT factor (one device thread).  out
   (device, 6 + 4*limbs doubles): positive, negative, zero counts, 1x1 and 2x2
   block counts, has-blocks flag, then min block |eigenvalue|, max block entry,
   their ratios to omax (limbs doubles each; 0 when omax is zero).
   Replaces factor_inertia / factor_diagnostics(::MFLDLT) —
   src/diagnostics.jl:109-246. */
int mflab_ldlt_diagnostics(mflab_handle *h, void *stream, int limbs, int64_t n, const double *F,
                           int64_t ldf, int64_t lsf, const double *dsub, int64_t lsd,
                           const uint8_t *blocks, const double *omax, double *out);

/* ------------------------------------------------------- batched SPD --- */
/* Factor (and with solve != 0 also solve) nblocks independent SPD blocks:
   one persistent launch factors every block and runs its forward
   substitution, a second launch runs the backward substitutions (their
   one-term-at-a-time chains, several blocks per warp).  Block b is sizes[b] x sizes[b], column-major at
   S + offsets[b] (ld = sizes[b]), its right-hand side a vector at X +
   boffsets[b]; limb planes are ls_s / ls_x apart.  CTAs take blocks in the
   order order[0..nblocks) from the device counter (reset here with one
   stream-ordered memset).  Each block follows cholesky!(S_b; block) and
   ldiv!(x_b, F_b) exactly; info[b] receives 0 or the failing column.
   max_size <= 512 bounds every sizes[b] (it sizes the per-CTA shared
   buffer); a block larger than max_size is left untouched with info[b] = -1.  grid <= 0 picks 4 CTAs per SM.  No allocation, no
   synchronisation.  No reference counterpart (the reference factors one
   matrix per call: src/factorizations/cholesky.jl:68-107). */
int mflab_spd_batched(mflab_handle *h, void *stream, int limbs, int64_t nblocks, int64_t max_size,
                      const int64_t *sizes, const int64_t *offsets, const int64_t *boffsets,
                      const int64_t *order, double *S, int64_t ls_s, double *X, int64_t ls_x,
                      int64_t block, int solve, int *info, int *counter, int grid);

/* Adjoint of x_b = S_b^{-1} b_b reusing the factors of mflab_spd_batched: XB
   holds xbar on entry and bbar = S^{-1} xbar on exit; SB (packed like S)
   receives Sbar = -(bbar x^T + x bbar^T) / 2.  Blocks with info != 0 are
   skipped.  No reference counterpart. */
int mflab_spd_batched_adjoint(mflab_handle *h, void *stream, int limbs, int64_t nblocks,
                              int64_t max_size, const int64_t *sizes, const int64_t *offsets,
                              const int64_t *boffsets, const int64_t *order, const double *L,
                              int64_t ls_s, const double *X, double *XB, int64_t ls_x, double *SB,
                              const int *info, int *counter, int grid);

/* mflab_spd_batched / mflab_spd_batched_adjoint with the CTA size chosen:
   threads = 64, 128, 256 or 512 (the plain entries use 256).  Neither the CTA
   size nor the number of persistent CTAs (grid) changes any result: every
   block's arithmetic is per element in the reference order; they are the
   knobs of the batched autotuner.  No reference counterpart. */
int mflab_spd_batched_ex(mflab_handle *h, void *stream, int limbs, int64_t nblocks,
                         int64_t max_size, const int64_t *sizes, const int64_t *offsets,
                         const int64_t *boffsets, const int64_t *order, double *S, int64_t ls_s,
                         double *X, int64_t ls_x, int64_t block, int solve, int *info,
                         int *counter, int grid, int threads);
int mflab_spd_batched_adjoint_ex(mflab_handle *h, void *stream, int limbs, int64_t nblocks,
                                 int64_t max_size, const int64_t *sizes, const int64_t *offsets,
                                 const int64_t *boffsets, const int64_t *order, const double *L,
                                 int64_t ls_s, const double *X, double *XB, int64_t ls_x,
                                 double *SB, const int *info, int *counter, int grid,
                                 int threads);

/* ------------------------------------------------------- diagnostics --- */
/* out (device, limbs+1 doubles) = [max |A(r,c)| over the region, finite flag]
   with region 0 all entries, 1 lower (r >= c), 2 upper (r <= c).
   Serves _maximum_abs / _lower_maximum_abs / _all_finite /
   _lower_triangle_finite (src/types.jl:306-331) and _lu_maximum_u
   (src/diagnostics.jl:74-81). */
int mflab_max_abs(mflab_handle *h, void *stream, int limbs, int64_t m, int64_t n, const double *A,
                  int64_t lda, int64_t lsa, int region, double *out);

/* mflab_max_abs without a handle and without any device allocation, for
   callers that cannot let a library allocate: code whose device memory all
   belongs to its own pool allocator, and code that must not take the implicit
   device-wide synchronisation of cudaMalloc/cudaFree in an asynchronous
   pipeline.  Partial results live in a fixed 640 KiB device array (one record
   per column) that every device loading the library holds until exit, so n is
   limited to 16384 columns (MFLAB_ERR_UNSUPPORTED beyond, with a message in
   mflab_last_error).  The first call on a device looks up that array's device
   address with the device current; make that first call before any stream
   capture.  All calls share the array: calls that overlap on the GPU race.
   No counterpart in the reference. */
int mflab_max_abs_noalloc(void *stream, int limbs, int64_t m, int64_t n, const double *A,
                          int64_t lda, int64_t lsa, int region, double *out);

/* O(n) tail of factor_diagnostics (src/diagnostics.jl:21-107): out (device,
   4*limbs+2 doubles) = [min |A(i,i)|, max |A(i,i)|, max/min (Inf if min is
   zero), num/den (0 if den is zero), count, count > 0] over i < count.
   num/den (device, limbs doubles each) may be NULL. */
int mflab_diag_summary(mflab_handle *h, void *stream, int limbs, const double *A, int64_t lda,
                       int64_t lsa, int64_t count, const double *num, const double *den,
                       double *out);

#ifdef __cplusplus
}
#endif
#endif /* MFLAB200_H */
