/*
 * lmie_b200.h -- entry points of liblmie_b200.so beyond the reference's
 * interface (include/lmie_interface.h).  None of these has a counterpart in
 * the reference; they expose device timing and device-resident re-runs for
 * benchmarking, and device information.
 */
#ifndef LMIE_B200_H
#define LMIE_B200_H

#include <stddef.h>

#include "lmie_interface.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Stages of one solve, timed with CUDA events when timing is on:
 * 0 upload, 1 Mie recurrences and coefficients (K1), 2 radius reduction of
 * the cross sections (K2), 3 angular accumulation (K3), 4 normalisation,
 * 5 GSF expansion, 6 Legendre expansion, 7 phase matrix at user angles,
 * 8 download. */
#define LMIEB_N_STAGES 9

/* Selects the GPU the library uses (default: the CUDA runtime's current
 * device).  Must precede the first solve; one process drives one GPU. */
int lmieb_set_device(int device);

/* Turn per-stage CUDA-event timing of lmie_solution on (1) or off (0). */
int lmieb_set_timing(int on);

/* Copies the stage times (ms) of the last timed solve into ms[0..n-1];
 * returns LMIEB_N_STAGES. */
int lmieb_last_timing(double *ms, int n);

/* Re-runs the device stages 1..7 of the last solve `reps` times on the
 * inputs still resident in device memory (no host work, no copies), each
 * repetition bracketed by CUDA events on the library's stream; with
 * flush_l2 a 256 MiB buffer is written before each repetition (outside the
 * timed interval).  Returns the summed device time in *ms_total and the
 * summed per-stage times in ms_stage[0..LMIEB_N_STAGES-1] (either may be
 * NULL).  Returns 0 or -1. */
int lmieb_rerun_device(int reps, int flush_l2, double *ms_total, double *ms_stage);

/* Algorithmic work of the last solve: flops[0] angular S1/S2 contraction,
 * flops[1] Mie recurrences, flops[2] Gauss-angle expansions, flops[3] phase
 * matrix at the user angles; the number of kernel launches one device run
 * issues; and the bytes the last solve copied host-to-device and back.  Any
 * pointer may be NULL. */
int lmieb_last_work(double *flops, long long *launches, size_t *h2d, size_t *d2h);

/* Measures the FP64 FMA throughput of the device (TFLOP/s) with a short
 * register-resident microbenchmark on the library's stream. */
int lmieb_fp64_peak(double *tflops);

/* Name, SM count and compute capability of the device the library uses. */
int lmieb_device_info(char *name, int len, int *sms, int *cc_major, int *cc_minor);

/* The CUDA stream all of the library's work is issued on (cudaStream_t). */
int lmieb_stream(void **stream);

#ifdef __cplusplus
}
#endif

#endif /* LMIE_B200_H */
