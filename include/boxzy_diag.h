/*
 * boxzy_diag.h -- measurement helper of libboxzy_gpu.so (no reference counterpart).
 *
 * The hydro step is bound by the FP64 pipe, and the FP64 peak of the device is
 * not among the measured peaks the roofline uses, so the library measures it:
 * independent chains of double-precision fused multiply-adds on every SM, timed
 * with CUDA events.  One DFMA counts as two floating-point operations.
 */
#ifndef BOXZY_DIAG_H
#define BOXZY_DIAG_H
#ifdef __cplusplus
extern "C" {
#endif

/* Measured FP64 FMA throughput of the current device in TFLOP/s; *sm_mhz (may be
 * NULL) receives nothing (clocks are sampled by the caller).  Returns 0 on success. */
int bx_fp64_peak(double *tflops, double *ms);

#ifdef __cplusplus
}
#endif
#endif
