// Repeated binary64 LU solves with inverted diagonal blocks (the correction
// solves of the mixed-precision LU solver: one binary64 factor, many solves
// with a few right-hand sides each).
//
// No reference counterpart and no reference order to keep: the binary64
// factor only drives iterative refinement, whose Float64xN residuals decide
// the accuracy.  A forward or backward substitution with a few right-hand
// sides is a chain of dependent steps; done row by row or in 64-row blocks
// with a triangular solve and a GEMM per block it is launch- and
// latency-bound (hundreds of small kernels per solve).  Here the 128 x 128
// diagonal blocks of L (unit lower) and U are inverted once after the
// factorization, the row interchanges are turned into one permutation, and
// every off-diagonal block column is premultiplied by its inverted diagonal
// block, M_{r,i} = L_{r,i} inv(DL_i) (rows below block i) and
// U_{r,i} inv(DU_i) (rows above it), all stored in a caller-owned workspace.
// A solve is then one gather and one kernel per block row and direction,
// whose CTAs share the work without redundancy and without waiting for one
// another: with b_i the block's current right-hand side rows,
//   the block's rows:      y_i = inv(D_i) b_i          (a few CTAs)
//   every remaining row r: W_r -= M_{r,i} b_i          (= L_{r,i} y_i)
//
// Workspace: perm[n] int32 (rounded up to 256 bytes), then the inverted L
// blocks and the inverted U blocks, nblk = ceil(n / 128) of 128 x 128
// doubles each (column-major, ld 128; a last partial block is padded), then
// ML and MU, n x n column-major (ld n) each, of which the blocks below /
// above the diagonal are used.
#include <algorithm>

#include "mflab_internal.h"

MFLAB_DEBUG_RECORD(lu64)

namespace mfl {

namespace {

constexpr int IB = 128;        // diagonal block size
constexpr int64_t PIVOT_PERM_MAXN_LU64 = 24576;  // indices in shared memory (96 KB)

size_t perm_bytes(int64_t n) { return ((size_t)n * 4 + 255) / 256 * 256; }
int64_t nblocks(int64_t n) { return (n + IB - 1) / IB; }

// In-place inversion of one diagonal block (jb x jb, jb <= 128) in shared
// memory: unit lower L (which = 0) or upper U (which = 1); block b of the
// factor goes to inv + b * IB * IB (ld IB).  One CTA per (block, which).
//   L: for j = jb-1 .. 0, column j of inv(L) below the diagonal is
//      -inv(L)[j+1:, j+1:] L[j+1:, j];
//   U: for j = 0 .. jb-1, inv(U)[j][j] = 1 / U[j][j] and the column above it
//      is -inv(U)[:j, :j] U[:j, j] inv(U)[j][j].
__global__ void __launch_bounds__(IB)
    lu64_inv_diag_kernel(int64_t n, const double *__restrict__ LU, int64_t ldl, double *invL,
                         double *invU) {
    extern __shared__ double sm[];  // [IB][IB + 1] block, then [IB] column copy
    double *blk = sm;
    double *v = sm + IB * (IB + 1);
    const int b = blockIdx.x, which = blockIdx.y, t = threadIdx.x;
    const int64_t j0 = (int64_t)b * IB;
    const int jb = (int)(n - j0 < IB ? n - j0 : IB);
    // column c of the block at blk[c * (IB + 1) + r]
    for (int c = 0; c < jb; ++c)
        if (t < jb) blk[c * (IB + 1) + t] = LU[(j0 + c) * ldl + j0 + t];
    __syncthreads();
    if (which == 0) {
        for (int j = jb - 1; j >= 0; --j) {
            if (t < jb) v[t] = t > j ? blk[j * (IB + 1) + t] : 0.0;  // L[:, j] below j
            __syncthreads();
            if (t > j && t < jb) {
                // row t of inv(L)[j+1:, j+1:] (final) times L[j+1:, j]
                double acc = v[t];  // inv(L)[t][t] = 1
                for (int i = j + 1; i < t; ++i) acc = fma(blk[i * (IB + 1) + t], v[i], acc);
                blk[j * (IB + 1) + t] = -acc;
            }
            __syncthreads();
        }
    } else {
        for (int j = 0; j < jb; ++j) {
            if (t <= j) v[t] = blk[j * (IB + 1) + t];  // U[:j+1, j]
            __syncthreads();
            const double djj = 1.0 / v[j];
            if (t < j) {
                // row t of inv(U)[:j, :j] (final) times U[:j, j]
                double acc = 0.0;
                for (int i = t; i < j; ++i) acc = fma(blk[i * (IB + 1) + t], v[i], acc);
                blk[j * (IB + 1) + t] = -acc * djj;
            } else if (t == j) {
                blk[j * (IB + 1) + t] = djj;
            }
            __syncthreads();
        }
    }
    // store with zeros outside the triangle and the unit diagonal of inv(L)
    double *dst = (which == 0 ? invL : invU) + (int64_t)b * IB * IB;
    for (int c = 0; c < IB; ++c) {
        double x = 0.0;
        if (t < jb && c < jb) {
            if (which == 0) x = t > c ? blk[c * (IB + 1) + t] : (t == c ? 1.0 : 0.0);
            else x = t <= c ? blk[c * (IB + 1) + t] : 0.0;
        }
        dst[c * IB + t] = x;
    }
}

// perm[i] = the original row that ends up in row i after the interchanges
// ipiv[0..n) (1-based, applied in ascending order): replayed by one thread on
// an index array in shared memory
__global__ void lu64_perm_kernel(int64_t n, const int64_t *ipiv, int *perm) {
    extern __shared__ int sidx[];
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) sidx[i] = (int)i;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int64_t k = 0; k < n; ++k) {
            const int64_t p = ipiv[k] - 1;
            if (p != k) {
                const int x = sidx[k];
                sidx[k] = sidx[p];
                sidx[p] = x;
            }
        }
    }
    __syncthreads();
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) perm[i] = sidx[i];
}

// W[i, c] = B[perm[i], c]
__global__ void lu64_gather_kernel(int64_t n, int64_t nrhs, const double *B, int64_t ldb,
                                   const int *perm, double *W, int64_t ldw) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * nrhs) return;
    const int64_t i = e % n, c = e / n;
    W[c * ldw + i] = B[c * ldb + perm[i]];
}

// One block step of a triangular solve.  Block i spans rows [j0, j0 + jb)
// and b = W[j0 : j0 + jb, :] holds its final right-hand side rows.
//   CTA k < ceil(jb / 32):  Out[j0 + 32k + r, c] = (inv(D_i) b)[32k + r, c]
//   the other CTAs, 32 rows r of [r_begin, r_end) each:
//                           W[r, c] -= (M[r, block i] b)[r, c]
// The rows written to W are outside the block, so no CTA reads what another
// writes.  A CTA stages its 32 x jb slice of inv(D_i) or M (k-major) and b
// (16 right-hand sides at a time) in shared memory; thread (row, warp)
// accumulates two right-hand sides over the jb columns.
constexpr int MS_ROWS = 32, MS_NT = 256, MS_RHS = 16;

__global__ void __launch_bounds__(MS_NT)
    lu64_mstep_kernel(int64_t nrhs, int64_t j0, int jb, const double *__restrict__ M, int64_t ldm,
                      const double *__restrict__ inv, double *W, int64_t ldw, double *Out,
                      int64_t ldo, int64_t r_begin, int64_t r_end) {
    static_assert(MS_NT / 32 * 2 == MS_RHS, "two right-hand sides per warp");
    __shared__ double tile[IB][MS_ROWS];             // [k][row]
    __shared__ __align__(16) double bT[IB][MS_RHS];  // [k][rhs]
    const int t = threadIdx.x, lane = t % 32, warp = t / 32;
    const int ndiag = (jb + MS_ROWS - 1) / MS_ROWS;
    const bool diag = (int)blockIdx.x < ndiag;
    // diag: the first row inside the block; else the first absolute row of R
    const int64_t rb = diag ? (int64_t)blockIdx.x * MS_ROWS
                            : r_begin + ((int64_t)blockIdx.x - ndiag) * MS_ROWS;
    const int64_t left = diag ? (int64_t)jb - rb : r_end - rb;
    const int nrows = (int)(left < MS_ROWS ? left : MS_ROWS);
    // launched as a programmatic dependent of the previous step: the next
    // step may start its prologue now, and this one stages its slice of M
    // or inv(D_i) (written before the solve) before waiting for the
    // previous step's results
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    // all loads of a thread in flight together (unrolled, then stored)
    {
        const double *src = diag ? inv + rb : M + j0 * ldm + rb;
        const int64_t ld = diag ? IB : ldm;
        double x[IB * MS_ROWS / MS_NT];
#pragma unroll
        for (int u = 0; u < IB * MS_ROWS / MS_NT; ++u) {
            const int e = t + u * MS_NT, r = e % MS_ROWS, k = e / MS_ROWS;
            x[u] = (r < nrows && k < jb &&
                    MFLAB_IDX_OK(rb + r < (diag ? (int64_t)IB : ldm), 7, rb + r, k))
                       ? src[(int64_t)k * ld + r]
                       : 0.0;
        }
#pragma unroll
        for (int u = 0; u < IB * MS_ROWS / MS_NT; ++u) {
            const int e = t + u * MS_NT;
            tile[e / MS_ROWS][e % MS_ROWS] = x[u];
        }
    }
    // the previous steps have completed and their writes are visible
    asm volatile("griddepcontrol.wait;" ::: "memory");
    for (int64_t c0 = 0; c0 < nrhs; c0 += MS_RHS) {
        const int cw = (int)(nrhs - c0 < MS_RHS ? nrhs - c0 : MS_RHS);
        double y[IB * MS_RHS / MS_NT];
#pragma unroll
        for (int u = 0; u < IB * MS_RHS / MS_NT; ++u) {
            const int e = t + u * MS_NT, k = e % IB, c = e / IB;
            y[u] = (k < jb && c < cw) ? W[(c0 + c) * ldw + j0 + k] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < IB * MS_RHS / MS_NT; ++u) {
            const int e = t + u * MS_NT;
            bT[e % IB][e / IB] = y[u];
        }
        __syncthreads();
        double a0 = 0.0, a1 = 0.0;
#pragma unroll 8
        for (int k = 0; k < IB; ++k) {
            const double m = tile[k][lane];
            const double2 bb = *(const double2 *)&bT[k][2 * warp];
            a0 = fma(m, bb.x, a0);
            a1 = fma(m, bb.y, a1);
        }
        const int c = 2 * warp;
        if (lane < nrows) {
            if (diag) {
                if (c < cw) Out[(c0 + c) * ldo + j0 + rb + lane] = a0;
                if (c + 1 < cw) Out[(c0 + c + 1) * ldo + j0 + rb + lane] = a1;
            } else {
                if (c < cw) W[(c0 + c) * ldw + rb + lane] -= a0;
                if (c + 1 < cw) W[(c0 + c + 1) * ldw + rb + lane] -= a1;
            }
        }
        __syncthreads();
    }
}

// one step, launched with programmatic stream serialization (its prologue
// overlaps the previous step); grid: the block's row groups, then R's
int mstep_launch(cudaStream_t s, int64_t nrhs, int64_t j0, int jb, const double *M, int64_t ldm,
                 const double *inv, double *W, int64_t ldw, double *Out, int64_t ldo,
                 int64_t r_begin, int64_t r_end) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((jb + MS_ROWS - 1) / MS_ROWS +
                                  (r_end - r_begin + MS_ROWS - 1) / MS_ROWS));
    cfg.blockDim = dim3(MS_NT);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return record_cuda_error(cudaLaunchKernelEx(&cfg, lu64_mstep_kernel, nrhs, j0, jb, M, ldm,
                                                inv, W, ldw, Out, ldo, r_begin, r_end),
                             "lu64 solve step");
}

std::atomic<unsigned long long> g_inv_configured{0};

}  // namespace
}  // namespace mfl

extern "C" int mflab_lu64_work_bytes(int64_t n, size_t *bytes) {
    if (n < 0 || !bytes) return MFLAB_ERR_ARG;
    *bytes = mfl::perm_bytes(n) + 2 * (size_t)mfl::nblocks(n) * mfl::IB * mfl::IB * sizeof(double) +
             2 * (size_t)n * n * sizeof(double);
    return MFLAB_OK;
}

extern "C" int mflab_lu64_prepare(mflab_handle *h, void *stream, int64_t n, const double *LU,
                                  int64_t ldl, const int64_t *ipiv, void *work) {
    MFLAB_RANGE("mflab_lu64_prepare");
    if (!h) return MFLAB_ERR_UNSUPPORTED;
    if (n < 0 || (n > 0 && (!LU || !ipiv || !work || ldl < n))) return MFLAB_ERR_ARG;
    if (n == 0) return MFLAB_OK;
    if (n > mfl::PIVOT_PERM_MAXN_LU64) return MFLAB_ERR_UNSUPPORTED;
    cudaStream_t s = (cudaStream_t)stream;
    int *perm = (int *)work;
    double *invL = (double *)((char *)work + mfl::perm_bytes(n));
    double *invU = invL + (size_t)mfl::nblocks(n) * mfl::IB * mfl::IB;
    const int smem = (mfl::IB * (mfl::IB + 1) + mfl::IB) * (int)sizeof(double);
    int rc = mfl::set_smem_once((const void *)mfl::lu64_inv_diag_kernel, smem,
                                mfl::g_inv_configured, "lu64 inverse attribute");
    if (rc) return rc;
    static std::atomic<unsigned long long> perm_configured{0};
    rc = mfl::set_smem_once((const void *)mfl::lu64_perm_kernel,
                            (int)(mfl::PIVOT_PERM_MAXN_LU64 * sizeof(int)), perm_configured,
                            "lu64 perm attribute");
    if (rc) return rc;
    mfl::lu64_perm_kernel<<<1, 256, (size_t)n * sizeof(int), s>>>(n, ipiv, perm);
    mfl::lu64_inv_diag_kernel<<<dim3((unsigned)mfl::nblocks(n), 2), mfl::IB, smem, s>>>(
        n, LU, ldl, invL, invU);
    rc = mfl::record_cuda_error(cudaGetLastError(), "lu64 prepare");
    if (rc) return rc;
    // ML = L_{r,i} inv(DL_i) below block i, MU = U_{r,i} inv(DU_i) above it
    // (binary64 GEMMs of the library)
    double *ML = invU + (size_t)mfl::nblocks(n) * mfl::IB * mfl::IB, *MU = ML + (size_t)n * n;
    const size_t wsb = (size_t)32 << 20;
    rc = mflab_reserve_scratch(h, wsb);
    if (rc) return rc;
    for (int64_t i = 0; i < mfl::nblocks(n) && rc == MFLAB_OK; ++i) {
        const int64_t j0 = i * mfl::IB, jb = std::min<int64_t>(mfl::IB, n - j0);
        const double *iL = invL + i * mfl::IB * mfl::IB, *iU = invU + i * mfl::IB * mfl::IB;
        if (j0 + jb < n)
            rc = mfl::dgemm_lt(n - j0 - jb, jb, jb, LU + j0 * ldl + j0 + jb, ldl, iL, mfl::IB,
                               ML + j0 * n + j0 + jb, n, 1.0, 0.0, h->scratch, wsb, s);
        if (rc == MFLAB_OK && j0 > 0)
            rc = mfl::dgemm_lt(j0, jb, jb, LU + j0 * ldl, ldl, iU, mfl::IB, MU + j0 * n, n, 1.0,
                               0.0, h->scratch, wsb, s);
    }
    return rc;
}

extern "C" int mflab_lu64_solve(mflab_handle *h, void *stream, int64_t n, int64_t nrhs,
                                const double *LU, int64_t ldl, const void *work, double *B,
                                int64_t ldb) {
    MFLAB_RANGE("mflab_lu64_solve");
    if (!h) return MFLAB_ERR_UNSUPPORTED;
    if (n < 0 || nrhs < 0 || (n > 0 && (!LU || !work || !B || ldl < n || ldb < n)))
        return MFLAB_ERR_ARG;
    if (n == 0 || nrhs == 0) return MFLAB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const int *perm = (const int *)work;
    const double *invL = (const double *)((const char *)work + mfl::perm_bytes(n));
    const double *invU = invL + (size_t)mfl::nblocks(n) * mfl::IB * mfl::IB;
    // W: the permuted right-hand sides, then the forward solution
    int rc = mflab_reserve_scratch(h, (size_t)n * nrhs * sizeof(double));
    if (rc) return rc;
    double *W = (double *)h->scratch;
    const int64_t tot = n * nrhs;
    mfl::lu64_gather_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(n, nrhs, B, ldb, perm, W,
                                                                         n);
    rc = mfl::record_cuda_error(cudaGetLastError(), "lu64 gather");
    if (rc) return rc;
    const double *ML = invU + (size_t)mfl::nblocks(n) * mfl::IB * mfl::IB, *MU = ML + (size_t)n * n;
    const int64_t nb = mfl::nblocks(n);
    // forward: L y = P b, y written into B, W updated below each block
    for (int64_t i = 0; i < nb && rc == MFLAB_OK; ++i) {
        const int64_t j0 = i * mfl::IB;
        const int jb = (int)std::min<int64_t>(mfl::IB, n - j0);
        rc = mfl::mstep_launch(s, nrhs, j0, jb, ML, n, invL + i * mfl::IB * mfl::IB, W, n, B, ldb,
                               j0 + jb, n);
    }
    // backward: U x = y, x written into W, B (holding y) updated above each block
    for (int64_t i = nb - 1; i >= 0 && rc == MFLAB_OK; --i) {
        const int64_t j0 = i * mfl::IB;
        const int jb = (int)std::min<int64_t>(mfl::IB, n - j0);
        rc = mfl::mstep_launch(s, nrhs, j0, jb, MU, n, invU + i * mfl::IB * mfl::IB, B, ldb, W, n,
                               0, j0);
    }
    if (rc) return rc;
    rc = mfl::record_cuda_error(cudaGetLastError(), "lu64 solve");
    if (rc) return rc;
    // the solution (in W) back into B
    cudaError_t e = cudaMemcpy2DAsync(B, ldb * sizeof(double), W, n * sizeof(double),
                                      n * sizeof(double), nrhs, cudaMemcpyDeviceToDevice, s);
    return mfl::record_cuda_error(e, "lu64 solve copy");
}
