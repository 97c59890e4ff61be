// Library-level C-ABI entry points: version, status strings, handles.
#include <cstring>
#include <string>

#include "mflab_internal.h"

namespace {
thread_local std::string g_last_error;
}

namespace mfl {
int record_cuda_error(cudaError_t e, const char *where) {
    if (e == cudaSuccess) return MFLAB_OK;
    g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
    return MFLAB_ERR_CUDA;
}
void record_error_message(const char *msg) { g_last_error = msg; }
}  // namespace mfl

extern "C" int mflab_version(void) { return 10000 * 0 + 100 * 1 + 0; }

extern "C" const char *mflab_status_string(int code) {
    switch (code) {
    case MFLAB_OK: return "ok";
    case MFLAB_ERR_ARG: return "dimension mismatch or invalid size";
    case MFLAB_ERR_CUDA: return "CUDA runtime error";
    case MFLAB_ERR_UNSUPPORTED: return "unsupported limb count or option";
    case MFLAB_ERR_TIMEOUT: return "bounded device wait timed out";
    case MFLAB_ERR_ALLOC: return "device memory reservation failed";
    case MFLAB_ERR_ALIAS: return "output aliases an input";
    case MFLAB_ERR_FLAG: return "invalid option code";
    default: return "unknown status";
    }
}

extern "C" const char *mflab_last_error(void) { return g_last_error.c_str(); }

extern "C" int mflab_create(mflab_handle **out, int device) {
    if (!out) return MFLAB_ERR_ARG;
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return mfl::record_cuda_error(e == cudaSuccess ? cudaErrorNoDevice : e, "mflab_create");
    if (device < 0 || device >= count) return MFLAB_ERR_ARG;
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return mfl::record_cuda_error(e, "mflab_create cudaSetDevice");
    mflab_handle *h = new mflab_handle();
    h->device = device;
    h->scratch = nullptr;
    h->scratch_bytes = 0;
    h->dev_flags = nullptr;
    h->aux = nullptr;
    h->aux_bytes = 0;
    h->last_slices = 0;
    h->last_moduli = 0;
    h->solve_order = MFLAB_ORDER_MATCHED;
    h->int8_engine = MFLAB_INT8_TCGEN05;
    h->tc_limit = 0;
    h->tc_inject = 0;
    h->stage = nullptr;
    h->il_stream[0] = h->il_stream[1] = nullptr;
    h->stage_half = 0;
    h->il_next = 0;
    h->il_fork = h->il_done[0] = h->il_done[1] = nullptr;
    h->la_stream = nullptr;
    h->la_ev[0] = h->la_ev[1] = h->la_ev[2] = nullptr;
    e = cudaMalloc((void **)&h->dev_flags, 64 * sizeof(int));
    if (e != cudaSuccess) {
        delete h;
        mfl::record_cuda_error(e, "mflab_create flags");
        return MFLAB_ERR_ALLOC;
    }
    cudaMemset(h->dev_flags, 0, 64 * sizeof(int));
    *out = h;
    return MFLAB_OK;
}

extern "C" int mflab_destroy(mflab_handle *h) {
    if (!h) return MFLAB_OK;
    cudaSetDevice(h->device);
    cudaDeviceSynchronize();
    if (h->scratch) cudaFree(h->scratch);
    if (h->aux) cudaFree(h->aux);
    if (h->stage) cudaFree(h->stage);
    for (int i = 0; i < 2; ++i) {
        if (h->il_stream[i]) cudaStreamDestroy(h->il_stream[i]);
        if (h->il_done[i]) cudaEventDestroy(h->il_done[i]);
    }
    if (h->il_fork) cudaEventDestroy(h->il_fork);
    if (h->la_stream) cudaStreamDestroy(h->la_stream);
    for (int i = 0; i < 3; ++i)
        if (h->la_ev[i]) cudaEventDestroy(h->la_ev[i]);
    if (h->dev_flags) cudaFree(h->dev_flags);
    delete h;
    return MFLAB_OK;
}

int mflab_reserve_scratch(mflab_handle *h, size_t bytes) {
    if (bytes <= h->scratch_bytes) return MFLAB_OK;
    if (h->scratch) {
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return mfl::record_cuda_error(e, "scratch sync");
        cudaFree(h->scratch);
        h->scratch = nullptr;
        h->scratch_bytes = 0;
    }
    size_t want = bytes + bytes / 8;
    cudaError_t e = cudaMalloc(&h->scratch, want);
    if (e != cudaSuccess) {
        mfl::record_cuda_error(e, "scratch cudaMalloc");
        h->scratch = nullptr;
        return MFLAB_ERR_ALLOC;
    }
    h->scratch_bytes = want;
    return MFLAB_OK;
}

int mflab_reserve_aux(mflab_handle *h, size_t bytes) {
    if (bytes <= h->aux_bytes) return MFLAB_OK;
    if (h->aux) {
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return mfl::record_cuda_error(e, "aux sync");
        cudaFree(h->aux);
        h->aux = nullptr;
        h->aux_bytes = 0;
    }
    size_t want = bytes + bytes / 4 + 4096;
    cudaError_t e = cudaMalloc(&h->aux, want);
    if (e != cudaSuccess) {
        mfl::record_cuda_error(e, "aux cudaMalloc");
        h->aux = nullptr;
        return MFLAB_ERR_ALLOC;
    }
    h->aux_bytes = want;
    return MFLAB_OK;
}

extern "C" int mflab_set_solve_order(mflab_handle *h, int order) {
    if (!h) return MFLAB_ERR_ARG;
    if (order != MFLAB_ORDER_MATCHED && order != MFLAB_ORDER_FAST) return MFLAB_ERR_FLAG;
    h->solve_order = order;
    return MFLAB_OK;
}

extern "C" int mflab_set_tc_debug(mflab_handle *h, int64_t wait_limit, int inject) {
    if (!h) return MFLAB_ERR_ARG;
    if (wait_limit < 0) return MFLAB_ERR_ARG;
    if (inject != 0 && inject != 1) return MFLAB_ERR_FLAG;
    h->tc_limit = wait_limit;
    h->tc_inject = inject;
    return MFLAB_OK;
}

// ------------------------------------------------ memory for bindings ---
// Device memory and copies for a binding that has no CUDA runtime of its own
// (the Julia layer holds MFDeviceMatrix planes allocated here).

extern "C" int mflab_malloc(int device, size_t bytes, void **ptr) {
    if (!ptr) return MFLAB_ERR_ARG;
    *ptr = nullptr;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess && bytes > 0) e = cudaMalloc(ptr, bytes);
    if (e != cudaSuccess) {
        mfl::record_cuda_error(e, "mflab_malloc");
        *ptr = nullptr;
        return MFLAB_ERR_ALLOC;
    }
    return MFLAB_OK;
}

extern "C" int mflab_free(void *ptr) {
    if (!ptr) return MFLAB_OK;
    return mfl::record_cuda_error(cudaFree(ptr), "mflab_free");
}

extern "C" int mflab_memcpy(void *dst, const void *src, size_t bytes, int kind, void *stream) {
    if (bytes == 0) return MFLAB_OK;
    if (!dst || !src) return MFLAB_ERR_ARG;
    cudaMemcpyKind k;
    switch (kind) {
    case 0: k = cudaMemcpyHostToDevice; break;
    case 1: k = cudaMemcpyDeviceToHost; break;
    case 2: k = cudaMemcpyDeviceToDevice; break;
    default: return MFLAB_ERR_FLAG;
    }
    return mfl::record_cuda_error(cudaMemcpyAsync(dst, src, bytes, k, (cudaStream_t)stream),
                                  "mflab_memcpy");
}

extern "C" int mflab_memset(void *dst, int value, size_t bytes, void *stream) {
    if (bytes == 0) return MFLAB_OK;
    if (!dst) return MFLAB_ERR_ARG;
    return mfl::record_cuda_error(cudaMemsetAsync(dst, value, bytes, (cudaStream_t)stream),
                                  "mflab_memset");
}

extern "C" int mflab_stream_synchronize(void *stream) {
    return mfl::record_cuda_error(cudaStreamSynchronize((cudaStream_t)stream),
                                  "mflab_stream_synchronize");
}

// index-check violations recorded by a debug build since the last reset:
// out[0] the count, out[1..3] the first one's check code and index values
// (all zero in a release build)
extern "C" int mflab_debug_violations(long long *out, int reset) {
    if (!out) return MFLAB_ERR_ARG;
    long long tot[4] = {0, 0, 0, 0};
#define MFLAB_DEBUG_SUM(tu)                                                  \
    {                                                                        \
        long long v[4];                                                      \
        if (mfl_dbg_read_##tu(v, reset) != 0) return MFLAB_ERR_CUDA;         \
        if (v[0] && !tot[0]) {                                               \
            tot[1] = v[1];                                                   \
            tot[2] = v[2];                                                   \
            tot[3] = v[3];                                                   \
        }                                                                    \
        tot[0] += v[0];                                                      \
    }
    MFLAB_DEBUG_UNITS(MFLAB_DEBUG_SUM)
#undef MFLAB_DEBUG_SUM
    for (int i = 0; i < 4; ++i) out[i] = tot[i];
    return MFLAB_OK;
}

// 1 in a debug build (-DMFLAB_DEBUG), else 0
extern "C" int mflab_debug_build(void) {
#ifdef MFLAB_DEBUG
    return 1;
#else
    return 0;
#endif
}
