// Pieces shared by the two INT8 routes (ozaki.cu: digit slices; ozaki_crt.cu:
// modular residues): the per-row / per-column power-of-two scales.
#pragma once

#include <climits>

#include "mflab_internal.h"

namespace mfl {

constexpr int OZ_EXP_EMPTY = INT_MIN / 2;   // a row/column with no nonzero entry
constexpr int OZ_EXP_BAD = INT_MAX;         // a row/column holding a non-finite entry

__host__ __device__ __forceinline__ int oz_scale_exp(int e) {
    // |x| < 2^e  ->  scaled by 2^-(e+1) lies in (-1/2, 1/2)
    return (e == OZ_EXP_EMPTY || e == OZ_EXP_BAD) ? 0 : e + 1;
}

// Row exponents of A (rowexp[m]) and column exponents of B (colexp[n]) in the
// handle's aux scratch; tune != 0 also returns the sampled scale gap in
// eighths of a bit in *gap8_host (one stream synchronisation).
int ozaki_scales(mflab_handle *h, int N, int64_t m, int64_t n, int64_t k, Mat A, Mat B,
                 cudaStream_t s, int tune, int *gap8_host, int **rowexp, int **colexp);

// records phase event i on s when the phases entry point is timing a call
void ozaki_phase(int i, cudaStream_t s);
// ev[0..3] receive the phase events of the next route call (nullptr: off)
void ozaki_set_phase_events(cudaEvent_t *ev);

}  // namespace mfl
