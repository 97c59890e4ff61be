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

constexpr int CRT_TABLE_SIZE = 49;  // entries of crt_modulus

// Pairwise coprime moduli, greedy from 256 downwards (each is the largest
// number <= 256 coprime to all before it).  Residues fit a signed byte.
__host__ __device__ constexpr int crt_modulus(int t) {
    switch (t) {
    case 0: return 256;  case 1: return 255;  case 2: return 253;  case 3: return 251;
    case 4: return 247;  case 5: return 241;  case 6: return 239;  case 7: return 233;
    case 8: return 229;  case 9: return 227;  case 10: return 223; case 11: return 217;
    case 12: return 211; case 13: return 199; case 14: return 197; case 15: return 193;
    case 16: return 191; case 17: return 181; case 18: return 179; case 19: return 173;
    case 20: return 167; case 21: return 163; case 22: return 157; case 23: return 151;
    case 24: return 149; case 25: return 139; case 26: return 137; case 27: return 131;
    case 28: return 127; case 29: return 113; case 30: return 109; case 31: return 107;
    case 32: return 103; case 33: return 101; case 34: return 97;  case 35: return 89;
    case 36: return 83;  case 37: return 79;  case 38: return 73;  case 39: return 71;
    case 40: return 67;  case 41: return 61;  case 42: return 59;  case 43: return 53;
    case 44: return 47;  case 45: return 43;  case 46: return 41;  case 47: return 37;
    case 48: return 29;
    default: return 1;
    }
}

// Row exponents of A (rowexp[m]) and column exponents of B (colexp[n]) in the
// handle's aux scratch; tune != 0 also returns the sampled scale gap in
// eighths of a bit in *gap8_host (one stream synchronisation).
int ozaki_scales(mflab_handle *h, int N, int64_t m, int64_t n, int64_t k, Mat A, Mat B,
                 cudaStream_t s, int tune, int *gap8_host, int **rowexp, int **colexp);

// Exponents of a Gram product: one per row of the left factor of
// lower(A A^T) (trans = 0, A n x k) or lower(A^T A) (trans = 1, A k x n),
// *exps[n] in the aux scratch; tune != 0 also returns the sampled gap.
int ozaki_gram_scales(mflab_handle *h, int N, int trans, int64_t n, int64_t k, Mat A,
                      cudaStream_t s, int tune, int *gap8_host, int **exps);

// row exponents of A alone, column exponents of B alone (device arrays)
int ozaki_row_exps(int N, int64_t m, int64_t k, Mat A, int *rowexp, cudaStream_t s);
int ozaki_col_exps(int N, int64_t k, int64_t n, Mat B, int *colexp, cudaStream_t s);

// records phase event i on s when the phases entry point is timing a call
void ozaki_phase(int i, cudaStream_t s);
// ev[0..3] receive the phase events of the next route call (nullptr: off)
void ozaki_set_phase_events(cudaEvent_t *ev);

}  // namespace mfl
