// int8 x int8 -> int32 GEMM on the 5th-generation tensor cores (tcgen05),
// the level / residue products of the two INT8 multi-double routes.
//
// C[m0:m0+256, n0:n0+256] = A[rows, K] * B[cols, K]^T with both operands
// K-major int8 (rows of the digit matrices), exact int32 accumulation;
// independent problems z (moduli) are stacked in one launch.
//
// Persistent kernel, one CTA (10 warps) per SM walking a static list of
// 256 x 256 output tiles:
//   * warp 0 lane 0: TMA producer.  Per 128-byte K step it loads the A tile
//     (256 rows x 128 B) and the B tile (256 rows x 128 B) into one of 3 shared
//     memory stages with cp.async.bulk.tensor (128-byte swizzle, no multicast),
//     completion tracked by the stage's "full" mbarrier (expect_tx); it runs
//     ahead into the next tile while the epilogue drains the current one.
//   * warp 1: owns 512 TMEM columns (the 128 x 256 accumulators of the tile's
//     two row halves); lane 0 waits for a full stage, issues per 32-byte K
//     slice two tcgen05.mma.cta_group::1.kind::i8 (M=128, N=256, K=32) that
//     read the same B tile, so a 64 KiB stage feeds twice the MMA work of a
//     128-row tile, and tcgen05.commit's the stage's "empty" mbarrier.
//   * warps 2-9: epilogue.  Each reads its 32 TMEM lanes (rows) of one half
//     with tcgen05.ld.32x32b.x16 and stores the column-major result (a warp
//     writes 32 consecutive rows of one column).
// Every mbarrier wait is bounded.  A wait of one role on another that runs out
// (the launch's role bound) records an error code in *err and raises a shared
// abort flag that ends every role's loop; the CTA then drains what it has
// itself issued — the producer waits for its copies in flight, the MMA
// issuer for its MMAs (both with the larger drain bound, which only runs out
// if the hardware stops completing them) — frees its TMEM and returns.
// Operands: the padded digit matrices (rows multiple of 128 / 256, K multiple
// of 128), so no tile needs bounds checks beyond the last half row tile.
#include <mutex>

#include "int8_tc_common.cuh"

MFLAB_DEBUG_RECORD(int8_tc)

namespace mfl {

constexpr int TC_BM = 256, TC_MMA_M = 128, TC_BN = 256, TC_STAGES = 3;
constexpr uint32_t TC_A_BYTES = TC_BM * TC_BK;               // 32 KiB
constexpr uint32_t TC_B_BYTES = TC_BN * TC_BK;               // 32 KiB
constexpr uint32_t TC_STAGE_BYTES = TC_A_BYTES + TC_B_BYTES;  // 64 KiB
constexpr uint32_t TC_SMEM = TC_STAGES * TC_STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;
constexpr uint32_t TC_TMEM_COLS = 256;  // one 128 x 256 accumulator

// Persistent, warp-specialised kernel: one CTA per SM walks the 256 x 256
// output tiles tile = blockIdx.x + i * gridDim.x (problem z outermost, then
// column tiles, then row tiles, so that neighbouring CTAs share B tiles in L2).
//   warp 0 lane 0   TMA producer over all k-steps of all its tiles
//   warp 1          TMEM owner (512 columns: the 128 x 256 accumulators of the
//                   tile's upper and lower row halves); lane 0 issues per
//                   32-byte K slice two M=128 MMAs that share the B operand
//   warps 2..9      epilogue: warps 2-5 drain the upper half, 6-9 the lower
//                   half (warp w reads TMEM lanes 32 (w % 4) .. 32 (w % 4) + 31)
// A row tile that starts 128 rows before the end of the matrix (m % 256 ==
// 128) computes and stores its upper half only.
// MODE 0 stores the int32 sums; MODE 1 stores their residues modulo
// crt_modulus(z) as bytes (C is then a byte matrix: ldc and c_zstride in
// bytes), the only part of the sums the modular route needs.
constexpr int TC_THREADS = 320;
constexpr uint32_t TC_TMEM_ALLOC = 2 * TC_TMEM_COLS;

template <int MODE>
__global__ void __launch_bounds__(TC_THREADS, 1)
    int8_tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA,
                        const __grid_constant__ CUtensorMap tmB, int K, int b_xoff, void *Cv,
                        int64_t ldc, int a_zrows, int b_zrows, int64_t c_zstride, int tiles_m,
                        int tiles_n, int nz, int tri, int *err, TcDebug dbg) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *full = (uint64_t *)(smem + TC_STAGES * TC_STAGE_BYTES);
    uint64_t *empty = full + TC_STAGES;
    uint64_t *tfull = empty + TC_STAGES;   // accumulators ready (MMA -> epilogue)
    uint64_t *tempty = tfull + 1;          // accumulators drained (epilogue -> MMA)
    uint64_t *drain = tempty + 1;          // all MMAs of this CTA complete
    uint64_t *never = drain + 1;           // injected timeouts wait here (no arrivals)
    uint32_t *tmem_slot = (uint32_t *)(never + 1);
    int *abort_flag = (int *)(tmem_slot + 1);

    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int ksteps = K / TC_BK;
    const int per_z = tri ? tiles_m * (tiles_m + 1) / 2 : tiles_m * tiles_n;
    const int total = per_z * nz;
    const long long lim = dbg.limit;

    if (threadIdx.x == 0) {
        for (int s = 0; s < TC_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(tfull, 1);
        mbar_init(tempty, 8);  // one arrival per epilogue warp
        mbar_init(drain, 1);
        mbar_init(never, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(TC_TMEM_ALLOC)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer
            int ks = 0;
            for (int tile = blockIdx.x; tile < total && !*(volatile int *)abort_flag;
                 tile += gridDim.x) {
                int z, mt, nt;
                tc_tile(tile, per_z, tiles_m, tri, z, mt, nt);
                const int am0 = z * a_zrows + mt * TC_BM;
                const int bn0 = z * b_zrows + nt * TC_BN;
                bool ok = true;
                for (int kb = 0; kb < ksteps; ++kb, ++ks) {
                    const int s = ks % TC_STAGES;
                    if (ks >= TC_STAGES &&
                        !mbar_wait(&empty[s], ((ks / TC_STAGES) - 1) & 1, lim, abort_flag)) {
                        if (!*(volatile int *)abort_flag) atomicExch(err, TC_ERR_PRODUCER);
                        atomicExch(abort_flag, 1);
                        ok = false;
                        break;
                    }
                    uint8_t *sa = smem + s * TC_STAGE_BYTES;
                    uint8_t *sb = sa + TC_A_BYTES;
                    mbar_expect_tx(&full[s], TC_STAGE_BYTES);
                    // rows past the last plane read the map's zero fill; rows
                    // of the next plane (m % 256 == 128) feed no stored result
                    // debug builds: a copy whose inner coordinate breaks the
                    // 16-byte rule is skipped (the stage then never fills and
                    // the bounded waits report it)
                    const int xa = kb * TC_BK, xb = b_xoff + kb * TC_BK;
                    if (MFLAB_IDX_OK((xa & 15) == 0 && (xb & 15) == 0 && xa < K, 1, xa, xb)) {
                        tma_load_2d(sa, &tmA, xa, am0, &full[s]);
                        tma_load_2d(sb, &tmB, xb, bn0, &full[s]);
                    }
                }
                if (!ok) break;
            }
            // Drain: the copies of the last (up to TC_STAGES) issued steps must
            // have landed before the CTA exits.  Each of those steps is the
            // latest phase of its stage (a stage is refilled only after the
            // MMAs consumed it), and its phase completes when its bytes land,
            // whether or not the MMA issuer got to it.
            for (int i = ks - TC_STAGES > 0 ? ks - TC_STAGES : 0; i < ks; ++i)
                if (!mbar_wait(&full[i % TC_STAGES], (i / TC_STAGES) & 1, TC_DRAIN_LIMIT))
                    atomicExch(err, TC_ERR_DRAIN);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---------------- MMA issuer
            const uint32_t idesc = idesc_i8(TC_MMA_M, TC_BN);
            if (dbg.inject && !mbar_wait(never, 0, TC_INJECT_POLLS)) {
                atomicExch(err, TC_ERR_MMA);
                atomicExch(abort_flag, 1);
            }
            int ks = 0, it = 0;
            for (int tile = blockIdx.x; tile < total && !*(volatile int *)abort_flag;
                 tile += gridDim.x, ++it) {
                int z, mt, nt;
                tc_tile(tile, per_z, tiles_m, tri, z, mt, nt);
                const bool two_halves = mt * TC_BM + TC_MMA_M < a_zrows;
                if (it > 0 && !mbar_wait(tempty, (it - 1) & 1, lim, abort_flag)) {
                    if (!*(volatile int *)abort_flag) atomicExch(err, TC_ERR_MMA);
                    atomicExch(abort_flag, 1);
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                bool ok = true;
                for (int kb = 0; kb < ksteps; ++kb, ++ks) {
                    const int s = ks % TC_STAGES;
                    if (!mbar_wait(&full[s], (ks / TC_STAGES) & 1, lim, abort_flag)) {
                        if (!*(volatile int *)abort_flag) atomicExch(err, TC_ERR_MMA);
                        atomicExch(abort_flag, 1);
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t sa = smem_u32(smem + s * TC_STAGE_BYTES);
                    const uint32_t sb = sa + TC_A_BYTES;
#pragma unroll
                    for (int kk = 0; kk < TC_BK / 32; ++kk) {
                        const uint32_t accf = (kb > 0 || kk > 0) ? 1u : 0u;
                        const uint64_t bd = smem_desc_sw128(sb + kk * 32);
                        mma_i8(tmem, smem_desc_sw128(sa + kk * 32), bd, idesc, accf);
                        if (two_halves)
                            mma_i8(tmem + TC_TMEM_COLS,
                                   smem_desc_sw128(sa + TC_MMA_M * TC_BK + kk * 32), bd, idesc,
                                   accf);
                    }
                    mma_commit(&empty[s]);
                }
                mma_commit(tfull);  // also on abort: the epilogue then sees the flag
                if (!ok) break;
            }
            // every MMA issued by this thread has completed once `drain` flips
            mma_commit(drain);
            if (!mbar_wait(drain, 0, TC_DRAIN_LIMIT)) atomicExch(err, TC_ERR_DRAIN);
        }
    } else {
        // ---------------- epilogue: TMEM -> registers -> C
        const int q = warp & 3;            // TMEM lane quarter of this warp
        const int half = (warp - 2) >> 2;  // 0: upper 128 rows, 1: lower 128 rows
        int it = 0;
        for (int tile = blockIdx.x; tile < total; tile += gridDim.x, ++it) {
            if (!mbar_wait(tfull, it & 1, lim, abort_flag)) {
                if (!*(volatile int *)abort_flag) atomicExch(err, TC_ERR_EPILOGUE);
                atomicExch(abort_flag, 1);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (*(volatile int *)abort_flag) break;
            int z, mt, nt;
            tc_tile(tile, per_z, tiles_m, tri, z, mt, nt);
            const int row = mt * TC_BM + half * TC_MMA_M + q * 32 + lane;
            const bool live = mt * TC_BM + half * TC_MMA_M < a_zrows;
            const int n0 = nt * TC_BN;
            void *Cz = MODE == 0 ? (void *)((int32_t *)Cv + (int64_t)z * c_zstride)
                                 : (void *)((uint8_t *)Cv + (int64_t)z * c_zstride);
            const int pz = crt_modulus(z);
            const double pzinv = 1.0 / (double)pz;
#pragma unroll 1
            for (int c0 = 0; c0 < TC_BN && live; c0 += 16) {
                uint32_t v[16];
                tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(half * TC_TMEM_COLS + c0),
                          v);
                if (MFLAB_IDX_OK(row < a_zrows && n0 + c0 + 16 <= tiles_n * TC_BN, 2, row, n0 + c0))
                    tc_store16<MODE>(Cz, ldc, row, n0 + c0, v, pz, pzinv);
            }
            // accumulators drained: the MMA warp may overwrite them
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(tempty);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(TC_TMEM_ALLOC)
                     : "memory");
    }
}

// ---------------------------------------------------------------- host ----
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    return fn;
}

// rows x cols int8 row-major matrix (ld bytes), box of box_rows x 128 bytes
int tc_make_map(CUtensorMap *map, const int8_t *base, int64_t rows, int64_t cols, int64_t ld,
                int box_rows) {
    auto fn = encode_fn();
    if (!fn) return MFLAB_ERR_UNSUPPORTED;
    if (((uintptr_t)base & 15) || (ld & 15)) return MFLAB_ERR_ARG;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld};
    cuuint32_t box[2] = {(cuuint32_t)TC_BK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void *)base, dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? MFLAB_OK : MFLAB_ERR_UNSUPPORTED;
}

template <int MODE>
int launch_tc_pair(const CUtensorMap &ta, const CUtensorMap &tb, int64_t mp, int64_t np,
                   int64_t K, int64_t b_xoff, void *C, int64_t ldc, int *err, cudaStream_t s,
                   int nz, int64_t c_zstride, int tri, const TcDebug &dbg);

template <int MODE>
static int launch_tc(int64_t mp, int64_t np, int64_t K, const int8_t *A, int64_t lda,
                     int64_t a_cols, const int8_t *B, int64_t ldb, int64_t b_cols, int64_t b_xoff,
                     void *C, int64_t ldc, int *err, cudaStream_t s, int nz, int64_t c_zstride,
                     int tri, const TcOpts &o) {
    if (mp % TC_MMA_M || np % TC_BN || K % TC_BK || b_xoff % 16 || K <= 0 || nz < 1)
        return MFLAB_ERR_ARG;
    if (K > a_cols || b_xoff + K > b_cols || K > 0x7fffffff || b_xoff > 0x7fffffff)
        return MFLAB_ERR_ARG;
    if (mp * nz > 0x7fffffff || np * nz > 0x7fffffff || np / TC_BN > 65535 || nz > 65535)
        return MFLAB_ERR_UNSUPPORTED;
    if (MODE == 1 && nz > CRT_TABLE_SIZE) return MFLAB_ERR_ARG;
    TcDebug dbg;
    dbg.limit = o.limit > 0 ? o.limit : TC_ROLE_LIMIT;
    dbg.inject = o.inject;
    // a CTA stages 256-row boxes of both operands, a CTA of a pair 128-row ones
    const int box = o.pair ? TC_MMA_M : TC_BM;
    CUtensorMap ta, tb;
    int rc = tc_make_map(&ta, A, mp * nz, a_cols, lda, box);
    if (rc) return rc;
    rc = tc_make_map(&tb, B, np * nz, b_cols, ldb, box);
    if (rc) return rc;
    if (o.pair)
        return launch_tc_pair<MODE>(ta, tb, mp, np, K, b_xoff, C, ldc, err, s, nz, c_zstride, tri,
                                    dbg);
    static std::atomic<unsigned long long> configured{0};
    rc = set_smem_once((const void *)int8_tc_gemm_kernel<MODE>, (int)TC_SMEM, configured,
                       "int8 tc attribute");
    if (rc) return rc;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
        sms = 148;
    const int64_t tiles_m = (mp + TC_BM - 1) / TC_BM;
    if (tri && tiles_m != np / TC_BN) return MFLAB_ERR_ARG;
    const int64_t tiles =
        (tri ? tiles_m * (tiles_m + 1) / 2 : tiles_m * (np / TC_BN)) * nz;
    if (tiles > 0x7fffffff) return MFLAB_ERR_UNSUPPORTED;
    const unsigned grid = (unsigned)(tiles < sms ? tiles : sms);
    int8_tc_gemm_kernel<MODE><<<grid, TC_THREADS, TC_SMEM, s>>>(
        ta, tb, (int)K, (int)b_xoff, C, ldc, (int)mp, (int)np, c_zstride, (int)tiles_m,
        (int)(np / TC_BN), nz, tri, err, dbg);
    return record_cuda_error(cudaGetLastError(), "int8 tc gemm");
}

// C (mp x np int32, ldc) = A[0:mp, a-range] * B[0:np, b_xoff : b_xoff + K]^T.
// A is mp x a_cols, B np x b_cols, row-major int8 with leading dims lda, ldb.
// Requires mp % 128 == 0, np % 256 == 0, K % 128 == 0, b_xoff % 16 == 0.
// nz > 1 stacks problems: problem z reads rows [z mp, (z+1) mp) of A (which
// then holds nz mp rows), rows [z np, (z+1) np) of B and writes C + z c_zstride.
int int8_gemm_tc(int64_t mp, int64_t np, int64_t K, const int8_t *A, int64_t lda, int64_t a_cols,
                 const int8_t *B, int64_t ldb, int64_t b_cols, int64_t b_xoff, int32_t *C,
                 int64_t ldc, int *err, cudaStream_t s, const TcOpts &o, int nz,
                 int64_t c_zstride) {
    return launch_tc<0>(mp, np, K, A, lda, a_cols, B, ldb, b_cols, b_xoff, C, ldc, err, s, nz,
                        c_zstride, 0, o);
}

// As int8_gemm_tc with nz stacked problems, but problem z stores the residues
// of its sums modulo crt_modulus(z) as bytes: R + z r_zstride, column-major
// with leading dimension ldr (bytes).  tri != 0 computes only the 256 x 256
// tiles that meet the lower triangle (needs ceil(mp / 256) == np / 256).
int int8_gemm_tc_mod(int64_t mp, int64_t np, int64_t K, const int8_t *A, int64_t lda,
                     int64_t a_cols, const int8_t *B, int64_t ldb, int64_t b_cols, int64_t b_xoff,
                     uint8_t *R, int64_t ldr, int *err, cudaStream_t s, const TcOpts &o, int nz,
                     int64_t r_zstride, int tri) {
    return launch_tc<1>(mp, np, K, A, lda, a_cols, B, ldb, b_cols, b_xoff, R, ldr, err, s, nz,
                        r_zstride, tri, o);
}

}  // namespace mfl

// Test / measurement entry: one int8 x int8 -> int32 TN GEMM through either
// engine (0 = tcgen05 kernel, 1 = library).  Shapes as int8_gemm_tc.  The
// tcgen05 kernel's timeout status is written to *err (device int, 0 = ok).
extern "C" int mflab_int8_gemm_tn(mflab_handle *h, void *stream, int engine, int64_t mp,
                                  int64_t np, int64_t K, const int8_t *A, int64_t lda,
                                  int64_t a_cols, const int8_t *B, int64_t ldb, int64_t b_cols,
                                  int64_t b_xoff, int32_t *C, int64_t ldc, int *err) {
    MFLAB_RANGE("mflab_int8_gemm_tn");
    if (!h || !A || !B || !C || !err) return MFLAB_ERR_ARG;
    if (engine != MFLAB_INT8_TCGEN05 && engine != MFLAB_INT8_LIBRARY &&
        engine != MFLAB_INT8_TCGEN05_PAIR)
        return MFLAB_ERR_FLAG;
    cudaStream_t s = (cudaStream_t)stream;
    if (engine != MFLAB_INT8_LIBRARY) {
        mfl::TcOpts o = mfl::tc_opts(h);
        o.pair = engine == MFLAB_INT8_TCGEN05_PAIR;
        return mfl::int8_gemm_tc(mp, np, K, A, lda, a_cols, B, ldb, b_cols, b_xoff, C, ldc, err, s,
                                 o);
    }
    const size_t ws = (size_t)64 << 20;
    int rc = mflab_reserve_scratch(h, ws);
    if (rc) return rc;
    return mfl::int8_gemm_tn(mp, np, K, A, lda, B + b_xoff, ldb, C, ldc, h->scratch, ws, s);
}
