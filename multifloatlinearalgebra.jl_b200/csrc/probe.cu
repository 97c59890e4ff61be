// Throughput probes for the roofline denominators that the driver-measured
// peaks do not cover: the FP64 pipe instruction rate (DFMA and DADD).
// Each thread runs CHAINS independent dependency chains for `iters` steps; the
// result is written out so nothing is eliminated.
#include "mflab_internal.h"

namespace mfl {

template <int CHAINS, bool ADD>
__global__ void fp64_probe_kernel(int64_t iters, double seed, double *out) {
    double x[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) x[c] = seed + threadIdx.x * 1e-9 + c * 1e-7;
    const double a = 0.9999999999, b = 1e-12;
    for (int64_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < CHAINS; ++c) {
            if (ADD) {
                x[c] = __dadd_rn(x[c], b);
                x[c] = __dsub_rn(x[c], b);
            } else {
                x[c] = __fma_rn(x[c], a, b);
                x[c] = __fma_rn(x[c], a, b);
            }
        }
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) s += x[c];
    out[(int64_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace mfl

// Runs the probe on `blocks` x `threads` for `iters` steps and returns the
// number of FP64 instructions executed in *instructions (host).  `out` must
// hold blocks*threads doubles on the device.  Timing is the caller's.
extern "C" int mflab_probe_fp64(void *stream, int kind, int blocks, int threads, int64_t iters,
                                double *out, double *instructions) {
    MFLAB_RANGE("mflab_probe_fp64");
    if (blocks <= 0 || threads <= 0 || threads > 1024 || iters <= 0 || !out || !instructions)
        return MFLAB_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    constexpr int CH = 8;
    if (kind == 0)
        mfl::fp64_probe_kernel<CH, false><<<blocks, threads, 0, s>>>(iters, 1.0, out);
    else
        mfl::fp64_probe_kernel<CH, true><<<blocks, threads, 0, s>>>(iters, 1.0, out);
    *instructions = (double)blocks * threads * (double)iters * CH * 2.0;
    return mfl::record_cuda_error(cudaGetLastError(), "fp64 probe");
}
