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
// factorization, and the row interchanges are turned into one permutation,
// both stored in a caller-owned workspace.  A solve is then one gather and
// one kernel per block row and direction: every CTA forms
// y_i = inv(D_i) b_i (the 128 x 128 block product, recomputed per CTA, so no
// CTA waits for another) and subtracts L_{r,i} y_i (U_{r,i} x_i) from its
// own tile of the remaining rows; CTA 0 also stores y_i.
//
// Workspace: perm[n] int32 (rounded up to 256 bytes), then the inverted L
// blocks and the inverted U blocks, nblk = ceil(n / 128) of 128 x 128
// doubles each (column-major, ld 128; a last partial block is padded).
#include <algorithm>

#include "mflab_internal.h"

namespace mfl {

namespace {

constexpr int IB = 128;        // diagonal block size
constexpr int IB_RHS = 16;     // right-hand sides per pass of the solve kernel
constexpr int SOLVE_NT = 1024;  // threads of the solve kernel
constexpr int SOLVE_ROWS = 128;  // rows of the remaining matrix per CTA
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

// One block step of a triangular solve.  Block i spans rows [j0, j0 + jb).
//   y = inv(D_i) * W[j0 : j0 + jb, c0 : c0 + cw]   (computed by every CTA)
//   CTA 0 stores y into Out[j0 : j0 + jb, c0 : c0 + cw];
//   every CTA updates its tile of the remaining rows R (below the block for
//   the forward solve, above it for the backward one):
//   W[r, c] -= T[r, j0 : j0 + jb] * y[:, c]   (T = L or U, column-major)
// The remaining rows of W and the block's rows are disjoint, so CTAs that
// still read W's block rows never see another CTA's update.
// The 128 x 128 inverse, then the CTA's 128 x jb tile of T, are staged in
// shared memory by all 1024 threads at once (16 independent loads each).
// Each product is done by 512 threads: thread (row, quarter) accumulates all
// 16 right-hand sides over a quarter of the 128 columns (one matrix load and
// eight broadcast double2 loads per column), and the four partial sums are
// added in shared memory.
constexpr int SOLVE_PARTS = 4;

__device__ __forceinline__ void lu64_block_product(const double *mat, const double2 *xT,
                                                   double *part, int t, int jmax) {
    // part[p][c][r] = sum_{j in quarter p, j < jmax} mat[j][r] x[j][c]
    if (t >= SOLVE_PARTS * IB) return;
    const int r = t % IB, p = t / IB;
    double acc[IB_RHS];
#pragma unroll
    for (int c = 0; c < IB_RHS; ++c) acc[c] = 0.0;
    const int jb0 = p * (IB / SOLVE_PARTS);
    const int jb1 = jb0 + IB / SOLVE_PARTS < jmax ? jb0 + IB / SOLVE_PARTS : jmax;
#pragma unroll 4
    for (int j = jb0; j < jb1; ++j) {
        const double a = mat[j * IB + r];
#pragma unroll
        for (int c2 = 0; c2 < IB_RHS / 2; ++c2) {
            const double2 x = xT[j * (IB_RHS / 2) + c2];
            acc[2 * c2] = fma(a, x.x, acc[2 * c2]);
            acc[2 * c2 + 1] = fma(a, x.y, acc[2 * c2 + 1]);
        }
    }
#pragma unroll
    for (int c = 0; c < IB_RHS; ++c) part[(p * IB_RHS + c) * IB + r] = acc[c];
}

__global__ void __launch_bounds__(SOLVE_NT)
    lu64_block_step_kernel(int64_t n, int64_t nrhs, int64_t j0, int jb, const double *__restrict__ T,
                           int64_t ldt, const double *__restrict__ inv, double *W, int64_t ldw,
                           double *Out, int64_t ldo, int64_t r_begin, int64_t r_end) {
    static_assert(SOLVE_NT == 8 * IB && SOLVE_ROWS == IB && IB_RHS == 16, "thread layout");
    extern __shared__ double sm[];
    double *mat = sm;                              // [IB columns][IB rows]: inv(D), then T
    double2 *sbT = (double2 *)(mat + IB * IB);     // [IB][IB_RHS / 2]: W's block rows
    double2 *syT = sbT + IB * IB_RHS / 2;          // [IB][IB_RHS / 2]: y
    double *part = (double *)(syT + IB * IB_RHS / 2);  // [PARTS][IB_RHS][IB]
    const int t = threadIdx.x;
    const int64_t r0 = r_begin + (int64_t)blockIdx.x * SOLVE_ROWS;
    for (int64_t c0 = 0; c0 < nrhs; c0 += IB_RHS) {
        const int cw = (int)(nrhs - c0 < IB_RHS ? nrhs - c0 : IB_RHS);
#pragma unroll
        for (int u = 0; u < IB * IB / SOLVE_NT; ++u) {
            const int e = t + u * SOLVE_NT;
            mat[e] = inv[e];
        }
        for (int e = t; e < IB * IB_RHS; e += SOLVE_NT) {
            const int r = e % IB, c = e / IB;
            ((double *)sbT)[r * IB_RHS + c] =
                (r < jb && c < cw) ? W[(c0 + c) * ldw + j0 + r] : 0.0;
        }
        __syncthreads();
        lu64_block_product(mat, sbT, part, t, IB);
        __syncthreads();
        for (int e = t; e < IB * IB_RHS; e += SOLVE_NT) {
            const int r = e % IB, c = e / IB;
            double y = 0.0;
#pragma unroll
            for (int p = 0; p < SOLVE_PARTS; ++p) y += part[(p * IB_RHS + c) * IB + r];
            ((double *)syT)[r * IB_RHS + c] = y;
            if (blockIdx.x == 0 && r < jb && c < cw) Out[(c0 + c) * ldo + j0 + r] = y;
        }
        // this CTA's tile of T: rows r0 .. r0 + 127, columns j0 .. j0 + jb - 1
        const int r = t % IB, cq = t / IB;
        const bool live = r0 + r < r_end;
#pragma unroll
        for (int u = 0; u < IB * IB / SOLVE_NT; ++u) {
            const int j = cq + 8 * u;
            mat[j * IB + r] = (live && j < jb) ? T[(j0 + j) * ldt + r0 + r] : 0.0;
        }
        __syncthreads();
        lu64_block_product(mat, syT, part, t, jb);
        __syncthreads();
        for (int e = t; e < IB * IB_RHS; e += SOLVE_NT) {
            const int rr = e % IB, c = e / IB;
            if (r0 + rr >= r_end || c >= cw) continue;
            double acc = 0.0;
#pragma unroll
            for (int p = 0; p < SOLVE_PARTS; ++p) acc += part[(p * IB_RHS + c) * IB + rr];
            W[(c0 + c) * ldw + r0 + rr] -= acc;
        }
        __syncthreads();
    }
}

constexpr int SOLVE_SMEM =
    (IB * IB + 2 * IB * IB_RHS + SOLVE_PARTS * IB_RHS * IB) * (int)sizeof(double);

std::atomic<unsigned long long> g_inv_configured{0};

}  // namespace
}  // namespace mfl

extern "C" int mflab_lu64_work_bytes(int64_t n, size_t *bytes) {
    if (n < 0 || !bytes) return MFLAB_ERR_ARG;
    *bytes = mfl::perm_bytes(n) + 2 * (size_t)mfl::nblocks(n) * mfl::IB * mfl::IB * sizeof(double);
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
    return mfl::record_cuda_error(cudaGetLastError(), "lu64 prepare");
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
    static std::atomic<unsigned long long> step_configured{0};
    rc = mfl::set_smem_once((const void *)mfl::lu64_block_step_kernel, mfl::SOLVE_SMEM,
                            step_configured, "lu64 solve attribute");
    if (rc) return rc;
    const int64_t nb = mfl::nblocks(n);
    // forward: L y = P b, y written into B, W updated below each block
    for (int64_t i = 0; i < nb; ++i) {
        const int64_t j0 = i * mfl::IB;
        const int jb = (int)std::min<int64_t>(mfl::IB, n - j0);
        const int64_t rb = j0 + jb, re = n;
        const unsigned grid = (unsigned)std::max<int64_t>(1, (re - rb + mfl::SOLVE_ROWS - 1) /
                                                                 mfl::SOLVE_ROWS);
        mfl::lu64_block_step_kernel<<<grid, mfl::SOLVE_NT, mfl::SOLVE_SMEM, s>>>(
            n, nrhs, j0, jb, LU, ldl, invL + i * mfl::IB * mfl::IB, W, n, B, ldb, rb, re);
    }
    // backward: U x = y, x written into W, B (holding y) updated above each block
    for (int64_t i = nb - 1; i >= 0; --i) {
        const int64_t j0 = i * mfl::IB;
        const int jb = (int)std::min<int64_t>(mfl::IB, n - j0);
        const unsigned grid =
            (unsigned)std::max<int64_t>(1, (j0 + mfl::SOLVE_ROWS - 1) / mfl::SOLVE_ROWS);
        mfl::lu64_block_step_kernel<<<grid, mfl::SOLVE_NT, mfl::SOLVE_SMEM, s>>>(
            n, nrhs, j0, jb, LU, ldl, invU + i * mfl::IB * mfl::IB, B, ldb, W, n, 0, j0);
    }
    rc = mfl::record_cuda_error(cudaGetLastError(), "lu64 solve");
    if (rc) return rc;
    // the solution (in W) back into B
    cudaError_t e = cudaMemcpy2DAsync(B, ldb * sizeof(double), W, n * sizeof(double),
                                      n * sizeof(double), nrhs, cudaMemcpyDeviceToDevice, s);
    return mfl::record_cuda_error(e, "lu64 solve copy");
}
