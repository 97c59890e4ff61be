/*
 * Measurement helper of the mflab200 library (no counterpart in the
 * reference: it measures the FP64 pipe rate used as the roofline denominator
 * of the multi-double kernels).
 */
#ifndef MFLAB200_PROBE_H
#define MFLAB200_PROBE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
/* kind 0: dependent DFMA chains, kind 1: DADD/DSUB chains.  Launches
   blocks x threads threads, each with 8 chains of `iters` x 2 instructions, on
   `stream`; *instructions receives the FP64 instruction count.  `out` is a
   device buffer of blocks*threads doubles. */
int mflab_probe_fp64(void *stream, int kind, int blocks, int threads, int64_t iters, double *out,
                     double *instructions);
#ifdef __cplusplus
}
#endif
#endif
