// placeholder replaced by the INT8-slice route
#include "mflab_internal.h"
extern "C" int mflab_gemm_ozaki_route(mflab_handle *h, void *stream, int limbs, int64_t m,
                                      int64_t n, int64_t k, const double *A, int64_t lda,
                                      int64_t lsa, const double *B, int64_t ldb, int64_t lsb,
                                      double *C, int64_t ldc, int64_t lsc, const double *alpha,
                                      const double *beta) {
    return MFLAB_ERR_UNSUPPORTED;
}
