// Internal declarations shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include <atomic>

#include <nvtx3/nvToolsExt.h>

#include "../../include/mflab200.h"

namespace mfl {

struct Mat {
    double *p;
    int64_t ld;  // column stride (elements)
    int64_t ls;  // limb-plane stride (elements)
    __host__ __device__ Mat at(int64_t r, int64_t c) const { return Mat{p + c * ld + r, ld, ls}; }
};

// Operand access of the shared multi-double mainloop.
//   a(i,k): ta 0 A[i,k], 1 A[k,i], 2 symmetric from the lower triangle,
//           3 symmetric from the upper triangle;   b(k,j) = tb ? B[j,k] : B[k,j]
// tri == 1 writes only C(i,j) with i >= j (SYRK / GEMMT lower triangle).
enum { MM_PACKED = 1, MM_RIGHT = 2, MM_KGE = 4, MM_UNIT = 8 };
int launch_mm(int N, int ta, bool tb, int tri, bool fused3, int64_t m, int64_t n, int64_t k,
              Mat A, Mat B, Mat C, const double *alpha, const double *beta, cudaStream_t s,
              const int *info = nullptr, int mode = 0);
// triangular products (trmm.jl): C(i,j) = alpha * chain over the k range the
// MM_RIGHT / MM_KGE / MM_UNIT bits select; C must not overlap A or B.
int launch_trmm_mm(int N, int ta, bool tb, int mode, int64_t m, int64_t n, int64_t k, Mat A, Mat B,
                   Mat C, const double *alpha, cudaStream_t s);

// Triangular solve (trsm.jl semantics); returns an MFLAB_* code.
int launch_trsm(int N, int side, int uplo, int trans, int diag, int64_t m, int64_t n, Mat A, Mat B,
                const double *alpha, cudaStream_t s);
int launch_trsm_info(int N, int side, int uplo, int trans, int diag, int64_t m, int64_t n, Mat A,
                     Mat B, const double *alpha, cudaStream_t s, const int *info,
                     int order = 0);

int record_cuda_error(cudaError_t e, const char *where);

// An NVTX range named after the C entry point for the duration of the call,
// so profiles (Nsight Systems timelines, ncu --nvtx filters) attribute the
// kernels to the API call that issued them; a no-op without a tool attached.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};
#define MFLAB_RANGE(name) ::mfl::NvtxRange mflab_nvtx_range_(name)

// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) of a kernel once per
// device of the process (the attribute is per device); `done` is the
// kernel's own bit mask of configured devices.  Thread-safe.
inline int set_smem_once(const void *func, int bytes, std::atomic<unsigned long long> &done,
                         const char *what) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return record_cuda_error(e, what);
    const unsigned long long bit = 1ULL << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return 0;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return record_cuda_error(e, what);
    done.fetch_or(bit, std::memory_order_release);
    return 0;
}

// A kernel launch with programmatic stream serialization: the kernel's CTAs
// may be placed while the previous kernel on the stream drains (once its CTAs
// have run griddepcontrol.launch_dependents); the kernel must run
// griddepcontrol.wait before it reads anything the previous one writes.
template <typename... KArgs, typename... Args>
inline int launch_programmatic(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                               cudaStream_t s, const char *what, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return record_cuda_error(cudaLaunchKernelEx(&cfg, kern, args...), what);
}

inline int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return MFLAB_OK;
    return MFLAB_ERR_CUDA;
}


// Launch options of the tcgen05 int8 GEMM kernels: the CTA-pair kernel
// (int8_tc2.cu) or the one-SM kernel (int8_tc.cu), the bound of their
// role-to-role waits in mbarrier polls (0: the default) and, for tests of
// the timeout path, an injected wait that runs out.
struct TcOpts {
    int pair = 0;
    long long limit = 0;
    int inject = 0;
};

// int8 x int8 -> int32 TN GEMM through the library (ozaki.cu) and through the
// tcgen05 kernels (int8_tc.cu, int8_tc2.cu)
int int8_gemm_tn(int64_t m, int64_t n, int64_t K, const int8_t *A, int64_t lda, const int8_t *B,
                 int64_t ldb, int32_t *I, int64_t ldi, void *ws, size_t wsb, cudaStream_t s);
// binary64 C = alpha A B + beta C through the library (ozaki.cu)
int dgemm_lt(int64_t m, int64_t n, int64_t k, const double *A, int64_t lda, const double *B,
             int64_t ldb, double *C, int64_t ldc, double alpha, double beta, void *ws, size_t wsb,
             cudaStream_t s);
int int8_gemm_tc(int64_t mp, int64_t np, int64_t K, const int8_t *A, int64_t lda, int64_t a_cols,
                 const int8_t *B, int64_t ldb, int64_t b_cols, int64_t b_xoff, int32_t *C,
                 int64_t ldc, int *err, cudaStream_t s, const TcOpts &o, int nz = 1,
                 int64_t c_zstride = 0);
int int8_gemm_tc_mod(int64_t mp, int64_t np, int64_t K, const int8_t *A, int64_t lda,
                     int64_t a_cols, const int8_t *B, int64_t ldb, int64_t b_cols, int64_t b_xoff,
                     uint8_t *R, int64_t ldr, int *err, cudaStream_t s, const TcOpts &o, int nz,
                     int64_t r_zstride, int tri = 0);
void record_error_message(const char *msg);
// modular INT8 route (ozaki_crt.cu); T = 0 lets the tuner choose.  The SYRK
// form writes lower(C) = alpha op(A) op(A)^T + beta lower(C), op(A) = A
// (trans 0, n x k) or A^T (trans 1, A k x n)
int ozaki_crt_syrk(mflab_handle *hd, int N, int T, int trans, int64_t n, int64_t k, Mat A, Mat C,
                   const double *alpha, const double *beta, cudaStream_t s, int *T_used);
int ozaki_crt_gemm(mflab_handle *hd, int N, int T, int64_t m, int64_t n, int64_t k, Mat A, Mat B,
                   Mat C, const double *alpha, const double *beta, cudaStream_t s, int *T_used);

inline bool valid_limbs(int N) { return N >= 2 && N <= 4; }

// Whether two limb-plane views may share an element (Base.mightalias
// semantics, types.jl:252-267).  Views with the same column and plane strides
// are compared by their 2-D index ranges, so disjoint blocks of one matrix
// (e.g. A21 and A22) do not alias; otherwise the address ranges decide.
inline int64_t floor_div(int64_t a, int64_t b) {
    int64_t q = a / b;
    return (a % b != 0 && ((a < 0) != (b < 0))) ? q - 1 : q;
}
inline bool views_overlap(const double *a, int64_t ld_a, int64_t ls_a, int64_t rows_a,
                          int64_t cols_a, int limbs, const double *b, int64_t ld_b, int64_t ls_b,
                          int64_t rows_b, int64_t cols_b) {
    if (rows_a <= 0 || cols_a <= 0 || rows_b <= 0 || cols_b <= 0) return false;
    const double *a_end = a + (int64_t)(limbs - 1) * ls_a + (cols_a - 1) * ld_a + rows_a;
    const double *b_end = b + (int64_t)(limbs - 1) * ls_b + (cols_b - 1) * ld_b + rows_b;
    if (!(a < b_end && b < a_end)) return false;
    if (ld_a != ld_b || ls_a != ls_b || ld_a <= 0) return true;
    if (rows_a > ld_a || rows_b > ld_a) return true;
    const int64_t off = b - a;
    for (int l = -(limbs - 1); l <= limbs - 1; ++l) {
        const int64_t o = off - (int64_t)l * ls_a;
        const int64_t q = floor_div(o, ld_a), r = o - q * ld_a;
        const int64_t reps[2][2] = {{r, q}, {r - ld_a, q + 1}};
        for (auto &rep : reps) {
            const bool rows = rep[0] < rows_a && 0 < rep[0] + rows_b;
            const bool cols = rep[1] < cols_a && 0 < rep[1] + cols_b;
            if (rows && cols) return true;
        }
    }
    return false;
}

}  // namespace mfl

struct mflab_handle {
    int device;
    // device scratch owned by the handle (grown on demand, freed by destroy)
    void *scratch;
    size_t scratch_bytes;
    int *dev_flags;  // small device words: info, timeout flags
    // second, independent scratch for small per-call metadata that must
    // survive a growth of `scratch` (e.g. Ozaki row/column exponents)
    void *aux;
    size_t aux_bytes;
    int last_slices;  // slice count the last Ozaki call used
    int last_moduli;  // modulus count the last modular (CRT) INT8 call used
    int solve_order;  // MFLAB_ORDER_MATCHED or MFLAB_ORDER_FAST for triangular solves
    int int8_engine;  // MFLAB_INT8_TCGEN05 or MFLAB_INT8_LIBRARY for the level products
    // role-wait bound (0: default) and timeout injection of the tcgen05 kernels
    long long tc_limit;
    int tc_inject;
    // staging of the interleaved host <-> limb-plane copies (64 MiB, on first
    // use) and the two high-priority streams that alternate over its halves
    void *stage;
    size_t stage_half;  // bytes per staging half (0 until the first conversion)
    int il_next;        // staging half / internal stream of the next chunk
    cudaStream_t il_stream[2];
    cudaEvent_t il_fork, il_done[2];
    // the high-priority panel stream of the look-ahead binary64 LU and its
    // events (fork/join, panel done, other columns done), on first use
    cudaStream_t la_stream;
    cudaEvent_t la_ev[3];
};

int mflab_reserve_aux(mflab_handle *h, size_t bytes);

// grow the handle's scratch to at least `bytes`; returns MFLAB_OK or an error
int mflab_reserve_scratch(mflab_handle *h, size_t bytes);

namespace mfl {
// launch options of the tcgen05 kernels issued through handle h
inline TcOpts tc_opts(const mflab_handle *h) {
    TcOpts o;
    o.pair = h->int8_engine == MFLAB_INT8_TCGEN05_PAIR;
    o.limit = h->tc_limit;
    o.inject = h->tc_inject;
    return o;
}
inline bool tc_engine(const mflab_handle *h) { return h->int8_engine != MFLAB_INT8_LIBRARY; }
}  // namespace mfl

// Debug builds (-DMFLAB_DEBUG, libmflab200_debug.so): device index checks.
// MFLAB_IDX_OK(cond, code, a, b) is true when cond holds; otherwise it
// records the violation (the first one's code and two index values, and a
// count) in the translation unit's debug record and is false, so the guarded
// access is skipped — a check never traps.  MFLAB_DEBUG_RECORD(tu) defines
// that record and its host reader mfl_dbg_read_<tu>; mflab_debug_violations
// sums the readers.  Release builds compile the checks to `true`.
namespace mfl {
__device__ __forceinline__ bool dbg_note(unsigned long long *rec, int code, long long a,
                                         long long b) {
    if (atomicAdd(&rec[0], 1ULL) == 0ULL) {
        rec[1] = (unsigned long long)code;
        rec[2] = (unsigned long long)a;
        rec[3] = (unsigned long long)b;
    }
    return false;
}
}  // namespace mfl
#ifdef MFLAB_DEBUG
#define MFLAB_DEBUG_RECORD(tu)                                                            \
    static __device__ unsigned long long mfl_dbg_rec[4];                                  \
    int mfl_dbg_read_##tu(long long *out, int reset) {                                    \
        unsigned long long v[4] = {0, 0, 0, 0};                                           \
        cudaError_t e = cudaMemcpyFromSymbol(v, mfl_dbg_rec, sizeof(v));                  \
        for (int i = 0; i < 4; ++i) out[i] = (long long)v[i];                             \
        if (e == cudaSuccess && reset) {                                                  \
            const unsigned long long z[4] = {0, 0, 0, 0};                                 \
            e = cudaMemcpyToSymbol(mfl_dbg_rec, z, sizeof(z));                            \
        }                                                                                 \
        return e == cudaSuccess ? 0 : -1;                                                 \
    }
#define MFLAB_IDX_OK(cond, code, a, b) \
    ((cond) || ::mfl::dbg_note(mfl_dbg_rec, (code), (long long)(a), (long long)(b)))
#else
#define MFLAB_DEBUG_RECORD(tu)                                \
    int mfl_dbg_read_##tu(long long *out, int) {              \
        for (int i = 0; i < 4; ++i) out[i] = 0;               \
        return 0;                                             \
    }
#define MFLAB_IDX_OK(cond, code, a, b) (true)
#endif
// the translation units with a debug record
#define MFLAB_DEBUG_UNITS(X) X(int8_tc) X(ozaki_crt) X(lu64) X(factor) X(interleave) X(blas)
#define MFLAB_DEBUG_DECL(tu) int mfl_dbg_read_##tu(long long *out, int reset);
MFLAB_DEBUG_UNITS(MFLAB_DEBUG_DECL)
