// int8 x int8 -> int32 GEMM on CTA pairs (tcgen05 cta_group::2): the level /
// residue products of the two INT8 multi-double routes, as in int8_tc.cu,
// with a 256 x 256 output tile per pair of SMs instead of per SM.
//
// A cluster of two CTAs on two SMs computes C[m0:m0+256, n0:n0+256]:
//   * each CTA stages its own half of the operands per 128-byte K step:
//     rows m0 + 128 r .. +127 of A and rows n0 + 128 r .. +127 of B
//     (r = the CTA's rank in the pair), 16 KiB each, with plain TMA loads
//     into its own shared memory (no multicast); both CTAs' loads count on
//     the leader CTA's "full" mbarrier, on which the leader alone expects
//     the 64 KiB of the step;
//   * the leader's MMA thread issues per 32-byte K slice one
//     tcgen05.mma.cta_group::2.kind::i8 of M = 256, N = 256: each SM's tensor
//     core multiplies its 128 A rows by all 256 B rows (its own half and the
//     peer's) into its own TMEM (128 lanes x 256 columns);
//   * stage release, accumulator-ready and drain signals reach both CTAs
//     through tcgen05.commit with a two-CTA mask; the epilogue warps of both
//     CTAs report a drained accumulator on the leader's barrier.
// Per SM a step stages 32 KiB for a 128 x 256 x 128 product — the same bytes
// per product as the one-SM kernel's 64 KiB for 256 x 256 x 128 — but the
// SM's accumulator takes only 256 of the 512 TMEM columns, so two of them
// alternate: the epilogue of tile i overlaps the MMAs of tile i + 1, and the
// 32 KiB stages allow 6 steps in flight.
//
// Every wait is bounded as in int8_tc.cu.  On a role timeout a CTA records
// the error, raises its own and the peer's abort flag and stops issuing;
// then both CTAs drain (see the end of the kernel): the leader's MMAs
// complete (drain commit to both CTAs), and every copy either CTA has in
// flight is accounted on the leader's full barriers and waited for before
// either CTA frees its TMEM or exits.
#include <mutex>

#include "int8_tc_common.cuh"

namespace mfl {

namespace {

constexpr int P_BM = 256, P_HALF = 128, P_BN = 256, P_STAGES = 6;
constexpr uint32_t P_A_BYTES = P_HALF * TC_BK;               // 16 KiB: this CTA's A rows
constexpr uint32_t P_B_BYTES = P_HALF * TC_BK;               // 16 KiB: this CTA's B rows
constexpr uint32_t P_STAGE_BYTES = P_A_BYTES + P_B_BYTES;    // 32 KiB per CTA
constexpr uint32_t P_ACC_COLS = 256;                         // one 128 x 256 accumulator
constexpr uint32_t P_TMEM_ALLOC = 2 * P_ACC_COLS;            // two alternating accumulators
constexpr int P_EPI_WARPS = 8;
constexpr int P_THREADS = 64 + 32 * P_EPI_WARPS;             // producer, MMA, epilogue warps
constexpr uint32_t P_SMEM = P_STAGES * P_STAGE_BYTES + 1024 /*align*/ + 512 /*barriers*/;
constexpr uint16_t P_BOTH = 0x3;                             // both CTAs of the pair

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// shared::cluster address of the variable at shared::cta address `a` in the
// CTA of rank `rank`
__device__ __forceinline__ uint32_t map_rank(uint32_t a, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
    return r;
}

__device__ __forceinline__ void cluster_sync() {
    asm volatile(
        "barrier.cluster.arrive.release.aligned;\n\t"
        "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ void st_cluster(uint32_t addr, int v) {
    asm volatile("st.relaxed.cluster.shared::cluster.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}

// tiled TMA load into this CTA's shared memory whose completion counts on
// the mbarrier at shared::cluster address `bar` (the leader's)
__device__ __forceinline__ void tma_load_2d_pair(void *dst, const CUtensorMap *map, int x, int y,
                                                 uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void mma_i8_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                            uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8, %9, %10, %11, %12}, "
        "p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0),
        "r"(0), "r"(0), "r"(0), "r"(0)
        : "memory");
}

// arrive on the mbarrier at the same offset in both CTAs once every MMA this
// thread issued so far has completed
__device__ __forceinline__ void mma_commit_both(uint64_t *bar) {
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64"
        " [%0], %1;" ::"r"(smem_u32(bar)),
        "h"(P_BOTH)
        : "memory");
}

__device__ __forceinline__ void mbar_arrive_remote(uint32_t bar) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar)
                 : "memory");
}

// raise the abort flag of this CTA and of its peer
__device__ __forceinline__ void pair_abort(int *abort_flag, uint32_t peer) {
    atomicExch(abort_flag, 1);
    st_cluster(map_rank(smem_u32(abort_flag), peer), 1);
}

// Shared-memory layout (per CTA, same offsets in both): P_STAGES stages of
// [A half | B half], then the barriers and small words.
struct PairSync {
    uint64_t full[P_STAGES];   // leader: both CTAs' copies of a step landed
    uint64_t empty[P_STAGES];  // both: the step's MMAs are done with the stage
    uint64_t tfull[2];         // both: accumulator b holds a finished tile
    uint64_t tempty[2];        // leader: both CTAs' epilogues drained accumulator b
    uint64_t drain;            // both: every MMA of the pair has completed
    uint64_t never;            // injected timeouts wait here (no arrivals)
    uint32_t tmem_slot;
    int abort_flag;
    int issued[2];             // leader: K steps each CTA's producer issued
    int consumed;              // leader: K steps whose MMAs were issued
};

template <int MODE>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(P_THREADS, 1)
    int8_tc_pair_kernel(const __grid_constant__ CUtensorMap tmA,
                        const __grid_constant__ CUtensorMap tmB, int K, int b_xoff, void *Cv,
                        int64_t ldc, int a_zrows, int b_zrows, int64_t c_zstride, int tiles_m,
                        int tiles_n, int nz, int tri, int *err, TcDebug dbg) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    PairSync *sy = (PairSync *)(smem + P_STAGES * P_STAGE_BYTES);

    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const uint32_t rank = cluster_rank(), peer = rank ^ 1u;
    const bool leader = rank == 0;
    const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
    const int ksteps = K / TC_BK;
    const int per_z = tri ? tiles_m * (tiles_m + 1) / 2 : tiles_m * tiles_n;
    const int total = per_z * nz;
    const long long lim = dbg.limit;
    int *abort_flag = &sy->abort_flag;

    if (threadIdx.x == 0) {
        for (int s = 0; s < P_STAGES; ++s) {
            mbar_init(&sy->full[s], 1);
            mbar_init(&sy->empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&sy->tfull[b], 1);
            mbar_init(&sy->tempty[b], 2 * P_EPI_WARPS);
        }
        mbar_init(&sy->drain, 1);
        mbar_init(&sy->never, 1);
        sy->abort_flag = 0;
        sy->issued[0] = sy->issued[1] = 0;
        sy->consumed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&sy->tmem_slot)),
                     "r"(P_TMEM_ALLOC)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    }
    // barriers initialised and TMEM allocated in both CTAs before any use
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    cluster_sync();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = sy->tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer (both CTAs)
            int ks = 0;
            for (int tile = pair; tile < total && !*(volatile int *)abort_flag; tile += npairs) {
                int z, mt, nt;
                tc_tile(tile, per_z, tiles_m, tri, z, mt, nt);
                const int am0 = z * a_zrows + mt * P_BM + (int)rank * P_HALF;
                const int bn0 = z * b_zrows + nt * P_BN + (int)rank * P_HALF;
                bool ok = true;
                for (int kb = 0; kb < ksteps; ++kb, ++ks) {
                    const int s = ks % P_STAGES;
                    if (ks >= P_STAGES &&
                        !mbar_wait(&sy->empty[s], ((ks / P_STAGES) - 1) & 1, lim, abort_flag)) {
                        if (!*(volatile int *)abort_flag) atomicExch(err, TC_ERR_PRODUCER);
                        pair_abort(abort_flag, peer);
                        ok = false;
                        break;
                    }
                    uint8_t *sa = smem + s * P_STAGE_BYTES;
                    uint8_t *sb = sa + P_A_BYTES;
                    const uint32_t fb = map_rank(smem_u32(&sy->full[s]), 0);
                    if (leader) mbar_expect_tx(&sy->full[s], 2 * P_STAGE_BYTES);
                    // rows past the last plane read the map's zero fill; rows of
                    // the next plane (m % 256 == 128) feed no stored result
                    tma_load_2d_pair(sa, &tmA, kb * TC_BK, am0, fb);
                    tma_load_2d_pair(sb, &tmB, b_xoff + kb * TC_BK, bn0, fb);
                }
                if (!ok) break;
            }
            // publish this CTA's issued step count on the leader (drain)
            if (leader) sy->issued[0] = ks;
            else st_cluster(map_rank(smem_u32(&sy->issued[1]), 0), ks);
        }
    } else if (warp == 1) {
        if (lane == 0 && leader) {
            // ---------------- MMA issuer (leader only)
            const uint32_t idesc = idesc_i8(P_BM, P_BN);
            if (dbg.inject && !mbar_wait(&sy->never, 0, TC_INJECT_POLLS)) {
                atomicExch(err, TC_ERR_MMA);
                pair_abort(abort_flag, peer);
            }
            int ks = 0, it = 0;
            for (int tile = pair; tile < total && !*(volatile int *)abort_flag;
                 tile += npairs, ++it) {
                const int b = it & 1;
                if (it >= 2 &&
                    !mbar_wait<true>(&sy->tempty[b], ((it >> 1) - 1) & 1, lim, abort_flag)) {
                    if (!*(volatile int *)abort_flag) atomicExch(err, TC_ERR_MMA);
                    pair_abort(abort_flag, peer);
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc = tmem + (uint32_t)b * P_ACC_COLS;
                bool ok = true;
                for (int kb = 0; kb < ksteps; ++kb) {
                    const int s = ks % P_STAGES;
                    if (!mbar_wait(&sy->full[s], (ks / P_STAGES) & 1, lim, abort_flag)) {
                        if (!*(volatile int *)abort_flag) atomicExch(err, TC_ERR_MMA);
                        pair_abort(abort_flag, peer);
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t sa = smem_u32(smem + s * P_STAGE_BYTES);
                    const uint32_t sb = sa + P_A_BYTES;
#pragma unroll
                    for (int kk = 0; kk < TC_BK / 32; ++kk)
                        mma_i8_pair(acc, smem_desc_sw128(sa + kk * 32),
                                    smem_desc_sw128(sb + kk * 32), idesc,
                                    (kb > 0 || kk > 0) ? 1u : 0u);
                    mma_commit_both(&sy->empty[s]);
                    ++ks;
                }
                // also on abort: the epilogues then see the flag
                mma_commit_both(&sy->tfull[b]);
                if (!ok) break;
            }
            sy->consumed = ks;
            // both CTAs' drain barriers flip once every MMA issued here is done
            mma_commit_both(&sy->drain);
        }
    } else {
        // ---------------- epilogue (both CTAs): TMEM -> registers -> C
        const int q = warp & 3;                 // TMEM lane quarter of this warp
        const int ch = (warp - 2) >> 2;         // column half of the tile
        const uint32_t tempty_lead[2] = {map_rank(smem_u32(&sy->tempty[0]), 0),
                                         map_rank(smem_u32(&sy->tempty[1]), 0)};
        int it = 0;
        for (int tile = pair; tile < total; tile += npairs, ++it) {
            const int b = it & 1;
            if (!mbar_wait(&sy->tfull[b], (it >> 1) & 1, lim, abort_flag)) {
                if (!*(volatile int *)abort_flag) atomicExch(err, TC_ERR_EPILOGUE);
                pair_abort(abort_flag, peer);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (*(volatile int *)abort_flag) break;
            int z, mt, nt;
            tc_tile(tile, per_z, tiles_m, tri, z, mt, nt);
            const int row0 = mt * P_BM + (int)rank * P_HALF;
            const int row = row0 + q * 32 + lane;
            const bool live = row0 < a_zrows;
            const int n0 = nt * P_BN + ch * (P_BN / 2);
            void *Cz = MODE == 0 ? (void *)((int32_t *)Cv + (int64_t)z * c_zstride)
                                 : (void *)((uint8_t *)Cv + (int64_t)z * c_zstride);
            const int pz = crt_modulus(z);
            const double pzinv = 1.0 / (double)pz;
            const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)b * P_ACC_COLS +
                                  (uint32_t)ch * (P_BN / 2);
#pragma unroll 1
            for (int c0 = 0; c0 < P_BN / 2 && live; c0 += 16) {
                uint32_t v[16];
                tmem_ld16(base + (uint32_t)c0, v);
                tc_store16<MODE>(Cz, ldc, row, n0 + c0, v, pz, pzinv);
            }
            // accumulator b drained by this warp: report it to the leader's MMA
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive_remote(tempty_lead[b]);
        }
    }

    // ---------------- drain and exit (both CTAs, all threads)
    // 1. every MMA of the pair has completed (they read both CTAs' shared
    //    memory and write both CTAs' TMEM)
    __syncwarp();
    if (warp == 1 && lane == 0 && !mbar_wait(&sy->drain, 0, TC_DRAIN_LIMIT))
        atomicExch(err, TC_ERR_DRAIN);
    // 2. the step counts are published and no role issues anything new
    __syncwarp();
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    cluster_sync();
    // 3. the leader accounts for every copy still in flight and waits for it:
    //    steps [consumed, max(issued)) are each the latest phase of their
    //    stage (a stage is refilled only after the MMAs consumed it); the
    //    leader expected 64 KiB for the steps it issued itself, so it cancels
    //    the peer's 32 KiB where the peer did not issue the step, and expects
    //    the peer's 32 KiB where only the peer did
    if (leader && threadIdx.x == 0) {
        const int i0 = sy->issued[0], i1 = sy->issued[1];
        const int hi = i0 > i1 ? i0 : i1;
        for (int j = sy->consumed; j < hi; ++j) {
            uint64_t *f = &sy->full[j % P_STAGES];
            if (j < i0 && j >= i1) mbar_complete_tx(f, P_STAGE_BYTES);
            if (j >= i0 && j < i1) mbar_expect_tx(f, P_STAGE_BYTES);
            if (!mbar_wait(f, (j / P_STAGES) & 1, TC_DRAIN_LIMIT)) atomicExch(err, TC_ERR_DRAIN);
        }
    }
    // 4. nothing of either CTA is in flight: free the TMEM of the pair
    __syncwarp();
    cluster_sync();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(P_TMEM_ALLOC)
                     : "memory");
    }
}

}  // namespace

// Launch of the pair kernel for the shapes of int8_gemm_tc (same checks done
// by the caller); the grid is a multiple of two CTAs, at most one pair per
// two SMs.
template <int MODE>
int launch_tc_pair(const CUtensorMap &ta, const CUtensorMap &tb, int64_t mp, int64_t np,
                   int64_t K, int64_t b_xoff, void *C, int64_t ldc, int *err, cudaStream_t s,
                   int nz, int64_t c_zstride, int tri, const TcDebug &dbg) {
    static std::atomic<unsigned long long> configured{0};
    int rc = set_smem_once((const void *)int8_tc_pair_kernel<MODE>, (int)P_SMEM, configured,
                           "int8 tc pair attribute");
    if (rc) return rc;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 2)
        sms = 148;
    const int64_t tiles_m = (mp + P_BM - 1) / P_BM;
    if (tri && tiles_m != np / P_BN) return MFLAB_ERR_ARG;
    const int64_t tiles = (tri ? tiles_m * (tiles_m + 1) / 2 : tiles_m * (np / P_BN)) * nz;
    if (tiles > 0x7fffffff) return MFLAB_ERR_UNSUPPORTED;
    const int64_t pairs = tiles < sms / 2 ? tiles : sms / 2;
    int8_tc_pair_kernel<MODE><<<(unsigned)(2 * pairs), P_THREADS, P_SMEM, s>>>(
        ta, tb, (int)K, (int)b_xoff, C, ldc, (int)mp, (int)np, c_zstride, (int)tiles_m,
        (int)(np / P_BN), nz, tri, err, dbg);
    return record_cuda_error(cudaGetLastError(), "int8 tc pair gemm");
}

template int launch_tc_pair<0>(const CUtensorMap &, const CUtensorMap &, int64_t, int64_t, int64_t,
                               int64_t, void *, int64_t, int *, cudaStream_t, int, int64_t, int,
                               const TcDebug &);
template int launch_tc_pair<1>(const CUtensorMap &, const CUtensorMap &, int64_t, int64_t, int64_t,
                               int64_t, void *, int64_t, int *, cudaStream_t, int, int64_t, int,
                               const TcDebug &);

}  // namespace mfl
