// Allocation-free variant of the max-|entry| / finiteness reduction.
//
// mflab_max_abs (factor.cu) keeps its partial results in the handle's device
// scratch, which the handle grows with cudaMalloc on first use.  Some callers
// cannot let a library allocate: code that hands every byte of device memory
// to its own pool allocator (PyTorch's caching allocator, CUDA.jl's memory
// pool) and code that must not pay the implicit device-wide synchronisation
// of cudaMalloc / cudaFree inside an asynchronous pipeline.
// mflab_max_abs_noalloc serves them: it takes no handle, allocates nothing,
// and keeps its partial results in a fixed file-scope device array.
//
// Partition: one partial record per column of the matrix (max |A(r,c)| over
// the requested region of that column, and a finite flag), then one thread
// reduces the column records.  The maximum of absolute values does not depend
// on the reduction order, so the result is the one mflab_max_abs returns.
#include <mutex>
#include <string>

#include "mf_device.cuh"
#include "mflab_internal.h"

namespace mfl {

// Stated maximum: 16384 columns; a record is (limbs + 1) doubles with
// limbs <= 4, so the array is 16384 * 5 * 8 bytes = 640 KiB on every device
// that loads the library, for the life of the process.
constexpr int64_t NOALLOC_MAX_COLUMNS = 16384;
static __device__ __align__(256) double g_noalloc_records[NOALLOC_MAX_COLUMNS * 5];

// Host code cannot use g_noalloc_records directly: its host-side name is only
// a stand-in, not a device address.  The device address is looked up once per
// device, with that device current, and cached here.
constexpr int NOALLOC_MAX_DEVICES = 64;
static double *g_records_addr[NOALLOC_MAX_DEVICES];
static std::mutex g_records_mutex;

static int records_address(int device, double **addr) {
    if (device < 0 || device >= NOALLOC_MAX_DEVICES) return MFLAB_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_records_mutex);
    if (!g_records_addr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_records);
        if (e != cudaSuccess) return record_cuda_error(e, "max_abs_noalloc symbol address");
        g_records_addr[device] = (double *)p;
    }
    *addr = g_records_addr[device];
    return MFLAB_OK;
}

template <int N, int NT>
__global__ void __launch_bounds__(NT) column_record_kernel(int64_t m, Mat A, int region,
                                                           double *records) {
    __shared__ double sval[NT][N];
    __shared__ int sfin[NT];
    const int64_t c = blockIdx.x;
    const int t = threadIdx.x;
    mf<N> best = from_double<N>(0.0);
    int fin = 1;
    for (int64_t r = t; r < m; r += NT) {
        if (region == 1 && r < c) continue;
        if (region == 2 && r > c) continue;
        mf<N> v = load_mf<N>(A.p, A.ld, A.ls, r, c);
        if (!isfinite_mf(v)) fin = 0;
        best = max_mf(best, abs_mf(v));
    }
#pragma unroll
    for (int l = 0; l < N; ++l) sval[t][l] = best.v[l];
    sfin[t] = fin;
    __syncthreads();
    for (int off = NT / 2; off > 0; off >>= 1) {
        if (t < off) {
            mf<N> a, b;
#pragma unroll
            for (int l = 0; l < N; ++l) {
                a.v[l] = sval[t][l];
                b.v[l] = sval[t + off][l];
            }
            mf<N> r = max_mf(a, b);
#pragma unroll
            for (int l = 0; l < N; ++l) sval[t][l] = r.v[l];
            sfin[t] = sfin[t] && sfin[t + off];
        }
        __syncthreads();
    }
    if (t == 0) {
        // every record the reduction reads is written here first, so stale
        // contents from an earlier call are never used
#pragma unroll
        for (int l = 0; l < N; ++l) records[c * (N + 1) + l] = sval[0][l];
        records[c * (N + 1) + N] = sfin[0] ? 1.0 : 0.0;
    }
}

template <int N>
__global__ void column_record_reduce_kernel(int64_t n, const double *records, double *out) {
    mf<N> best = from_double<N>(0.0);
    int fin = 1;
    for (int64_t c = 0; c < n; ++c) {
        mf<N> v;
#pragma unroll
        for (int l = 0; l < N; ++l) v.v[l] = records[c * (N + 1) + l];
        best = max_mf(best, v);
        if (records[c * (N + 1) + N] == 0.0) fin = 0;
    }
#pragma unroll
    for (int l = 0; l < N; ++l) out[l] = best.v[l];
    out[N] = fin ? 1.0 : 0.0;
}

template <int N>
static int max_abs_noalloc_n(int64_t m, int64_t n, Mat A, int region, double *records,
                             double *out, cudaStream_t s) {
    if (n > 0) {
        column_record_kernel<N, 256><<<(unsigned)n, 256, 0, s>>>(m, A, region, records);
        int rc = record_cuda_error(cudaGetLastError(), "max_abs_noalloc columns");
        if (rc) return rc;
    }
    column_record_reduce_kernel<N><<<1, 1, 0, s>>>(n, records, out);
    return record_cuda_error(cudaGetLastError(), "max_abs_noalloc reduce");
}

}  // namespace mfl

extern "C" int mflab_max_abs_noalloc(void *stream, int limbs, int64_t m, int64_t n,
                                     const double *A, int64_t lda, int64_t lsa, int region,
                                     double *out) {
    if (!mfl::valid_limbs(limbs)) return MFLAB_ERR_UNSUPPORTED;
    if (region < 0 || region > 2) return MFLAB_ERR_FLAG;
    if (m < 0 || n < 0 || !out || (m > 0 && n > 0 && lda < m)) return MFLAB_ERR_ARG;
    if (n > mfl::NOALLOC_MAX_COLUMNS) {
        mfl::record_error_message(("mflab_max_abs_noalloc: " + std::to_string(n) +
                                   " columns exceed the fixed scratch of " +
                                   std::to_string(mfl::NOALLOC_MAX_COLUMNS) + " column records")
                                      .c_str());
        return MFLAB_ERR_UNSUPPORTED;
    }
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return mfl::record_cuda_error(e, "max_abs_noalloc device");
    double *records = nullptr;
    int rc = mfl::records_address(device, &records);
    if (rc) return rc;
    mfl::Mat a{(double *)A, lda, lsa};
    cudaStream_t s = (cudaStream_t)stream;
    switch (limbs) {
    case 2: return mfl::max_abs_noalloc_n<2>(m, n, a, region, records, out, s);
    case 3: return mfl::max_abs_noalloc_n<3>(m, n, a, region, records, out, s);
    default: return mfl::max_abs_noalloc_n<4>(m, n, a, region, records, out, s);
    }
}
