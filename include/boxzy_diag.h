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

/* Self-check of the divisions by a shared denominator (HLL flux) and by a grid
 * constant with a precomputed reciprocal (cell sizes, cell volume): n random
 * (numerator, denominator) pairs with exponents in [-exp_range, exp_range] (plus
 * exact multiples, near-ties and signed zeros) are divided each way on the device;
 * returns the number of results that differ from IEEE division in any bit (zeros of
 * either sign compare equal, except for the five-numerator form of the HLL flux,
 * whose zeros keep the IEEE sign) and one example. */
int bx_check_shared_division(unsigned long long n, unsigned long long seed, int exp_range,
                             unsigned long long *mismatches, double *example_a,
                             double *example_d);

#ifdef __cplusplus
}
#endif
#endif
