// PTX helpers shared by the tcgen05 kernels (int8_tc.cu: the int8 GEMM with
// one CTA per SM; int8_tc2.cu: CTA pairs with cta_group::2; ozaki_crt.cu: the
// CRT reconstruction): mbarriers, TMA tile loads, shared-memory and
// instruction descriptors, MMA issue, TMEM loads, the bounded waits and the
// int8 -> int32 / residue-byte epilogue store.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdint>

#include "mflab_internal.h"
#include "ozaki_common.cuh"

namespace mfl {

constexpr int TC_BK = 128;  // K bytes per pipeline step (one 128-byte swizzle row)

// Bounds of the kernels' spin waits, in mbarrier polls (each poll may
// suspend the thread for a while inside mbarrier.try_wait).  A wait of one
// role on another (producer <-> MMA <-> epilogue) uses the launch's role
// bound (TC_ROLE_LIMIT unless a test lowers it); the drain of copies and
// MMAs a CTA has itself issued uses TC_DRAIN_LIMIT, which only runs out if
// the hardware stops completing them.
constexpr long long TC_ROLE_LIMIT = 1LL << 24;
constexpr long long TC_DRAIN_LIMIT = 1LL << 26;

// error codes written to *err
constexpr int TC_ERR_PRODUCER = 1, TC_ERR_MMA = 2, TC_ERR_EPILOGUE = 3, TC_ERR_DRAIN = 4;

// Debug settings of a launch: `limit` bounds the role waits; inject = 1
// makes the MMA issuer wait (TC_INJECT_POLLS polls) on a barrier nothing
// arrives on before its first tile, so the timeout path runs with copies in
// flight and the MMA issuer is the role that times out.
constexpr long long TC_INJECT_POLLS = 256;
struct TcDebug {
    long long limit = TC_ROLE_LIMIT;
    int inject = 0;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// cancel `bytes` of expected transactions of the current phase
__device__ __forceinline__ void mbar_complete_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.complete_tx.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, P1;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// the same with cluster-scope acquire (arrivals from the peer CTA)
__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, P1;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait for the completion of phase `parity`; false when the bound
// runs out or (abort != nullptr) the shared abort flag is raised
template <bool CLUSTER = false>
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit,
                                          const int *abort = nullptr) {
    for (long long i = 0; i < limit; ++i) {
        if (CLUSTER ? mbar_try_wait_cluster(bar, parity) : mbar_try_wait(bar, parity)) return true;
        if (abort && *(const volatile int *)abort) return false;
    }
    return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// 2-D tiled TMA load into this CTA's shared memory, completion counted on
// the mbarrier at shared::cta address `bar` (no multicast)
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row atoms of
// 1024 bytes (stride byte offset 1024, leading byte offset 16 unused)
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;                 // leading byte offset (16 B units)
    d |= (uint64_t)(1024 >> 4) << 32;       // stride byte offset (16 B units)
    d |= (uint64_t)1 << 46;                 // descriptor version for tcgen05
    d |= (uint64_t)2 << 61;                 // SWIZZLE_128B
    return d;
}

// instruction descriptor: s8 x s8 -> s32, both operands K-major, M x N
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N) {
    return (2u << 4)      // D format s32
           | (1u << 7)    // A signed 8-bit
           | (1u << 10)   // B signed 8-bit
           | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// instruction descriptor: u8 x u8 -> s32, both operands K-major, M x N
__host__ __device__ constexpr uint32_t idesc_u8(int M, int N) {
    return (2u << 4)  // D format s32; A and B formats 0: unsigned 8-bit
           | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D (+)= A * B^T on this CTA's tensor core (accumulate = 0: D = A * B^T)
__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred PRED_enable_input_d;\n\t"
        "setp.ne.b32 PRED_enable_input_d, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, PRED_enable_input_d;\n\t}"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// arrive once on `bar` when every MMA this thread issued so far has completed
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 32 lanes x 16 columns of 32-bit accumulators, without waiting (the caller
// issues tmem_wait_ld before reading v)
__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
          "=r"(v[14]), "=r"(v[15])
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ void tmem_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// after tmem_wait_ld: ties the loaded registers to a point after the wait,
// so that no use of them is scheduled before it
template <int K>
__device__ __forceinline__ void tmem_pin(uint32_t (&v)[K]) {
#pragma unroll
    for (int i = 0; i < K; ++i) asm volatile("" : "+r"(v[i])::"memory");
}

// 32 lanes x 16 columns of 32-bit accumulators from TMEM address taddr
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
          "=r"(v[14]), "=r"(v[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Store 16 accumulators of one row (columns n0 .. n0+15): MODE 0 the int32
// sums, MODE 1 their residues modulo pz as bytes.  A warp stores 32
// consecutive rows of each column.
template <int MODE>
__device__ __forceinline__ void tc_store16(void *Cz, int64_t ldc, int row, int n0,
                                           const uint32_t (&v)[16], int pz, double pzinv) {
    if (MODE == 0) {
        int32_t *C = (int32_t *)Cz;
#pragma unroll
        for (int j = 0; j < 16; ++j) C[(int64_t)(n0 + j) * ldc + row] = (int32_t)v[j];
    } else {
        uint8_t *R = (uint8_t *)Cz;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int g = (int)v[j];
            // floor(g / p) or one off; the remainder is then fixed up exactly
            const int qq = (int)floor((double)g * pzinv);
            int rr = g - qq * pz;
            rr += rr < 0 ? pz : 0;
            rr -= rr >= pz ? pz : 0;
            R[(int64_t)(n0 + j) * ldc + row] = (uint8_t)rr;
        }
    }
}

// coordinates of output tile number `tile` of a 256 x 256 tiling: all
// tiles_m x tiles_n tiles of each problem z (row tiles fastest), or with
// `tri` only the tiles that meet the lower triangle of a square grid
// (column by column)
__device__ __forceinline__ void tc_tile(int tile, int per_z, int tiles_m, int tri, int &z, int &mt,
                                        int &nt) {
    z = tile / per_z;
    int r = tile % per_z;
    if (!tri) {
        mt = r % tiles_m;
        nt = r / tiles_m;
        return;
    }
    nt = 0;
    while (r >= tiles_m - nt) {
        r -= tiles_m - nt;
        ++nt;
    }
    mt = nt + r;
}

// host: rows x cols int8 row-major matrix (ld bytes) as a TMA map with boxes
// of box_rows x 128 bytes, 128-byte swizzle
int tc_make_map(CUtensorMap *map, const int8_t *base, int64_t rows, int64_t cols, int64_t ld,
                int box_rows);

}  // namespace mfl
