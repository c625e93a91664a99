/*
 * lmie_b200.h -- entry points of liblmie_b200.so beyond the reference's
 * interface (include/lmie_interface.h): batched and split-precision solves,
 * the adjoint, tuning, radius sharing over a group of GPUs (the reference's
 * use_mpi), device timing and device-resident re-runs for benchmarking, and
 * device information.
 */
#ifndef LMIE_B200_H
#define LMIE_B200_H

#include <stddef.h>

#include "lmie_interface.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Solves n_cases independent polydisperse problems, in[i] -> out[i], with
 * the same meaning, outputs and errors as calling
 * lmie_solution(&in[i], &out[i], alloc_out, verbose, n_threads, 0) for each
 * i.  The host preparation of the cases runs on n_threads threads; cases
 * that share their derivative layout and requested outputs are solved
 * together in batched device launches (size-parameter-balanced work lists),
 * so thousands of small and large cases keep the whole GPU busy.  This entry
 * point has no counterpart in the reference, whose callers loop over
 * lmie_solution.  Returns 0, or -1 if any case fails. */
int lmie_solution_batch(int n_cases, lmie_in_data *in, lmie_out_data *out, int alloc_out,
                        int verbose, int n_threads);

/* Arithmetic of the batched solve.
 * LMIEB_PRECISION_FP64: every stage in FP64, the reference's arithmetic
 *   (within 1e-10 of it); lmie_solution and lmie_solution_batch use it.
 * LMIEB_PRECISION_TF32X3: the angular S1/S2 contraction runs on the tensor
 *   cores with each operand split into two TF32 terms (lo*hi + hi*lo + hi*hi):
 *   the hi*hi products accumulate in FP32 over segments of 32 orders
 *   (lmieb_set_split_segment) added into an FP32 running sum, the cross terms
 *   over a radius group; the Mie recurrences, a_n/b_n, the phase-matrix quadratic
 *   forms, the radius sums, the normalisation and the expansions stay FP64.
 *   The phase matrix then carries a relative error of a few 1e-7 of its
 *   largest element.  Problems this mode does not cover (save_control != 0,
 *   more than 4 index1 or 3 index2 derivative slots) run in FP64. */
#define LMIEB_PRECISION_FP64 0
#define LMIEB_PRECISION_TF32X3 1
/* LMIEB_PRECISION_INT8: the angular S1/S2 contraction runs on the int8 tensor
 *   cores as an exact fixed-point sum: each operand value is scaled by powers
 *   of two (per order, per angle row, per operand column) to 47 fractional
 *   bits and split into six signed 8-bit digits; the 21 digit products that
 *   carry the result are summed exactly in int32 and combined in FP64.  Each
 *   product carries about 2^-46 of the largest term of its row and column
 *   (FP64: 2^-53); everything else is the FP64 form's arithmetic.  A case
 *   whose truncation n_coef could depend on that difference -- some
 *   |beta_l| (l < n_coef) within the contraction's error bound of `accuracy`
 *   -- is solved again in FP64 within the same call, so n_coef is always the
 *   FP64 form's.  Problems this mode does not cover (save_control != 0, more
 *   than 4 index1 or 3 index2 derivative slots) and cases of fewer than 16 or
 *   more than 5120 orders run in FP64. */
#define LMIEB_PRECISION_INT8 2

/* Batch calls cut their cases into `chunks` parts (0: automatic -- one part
 * per 640 cases, at most 6; 1: one part) and prepare, pack, unpack and
 * scatter one part on the host while the device works on another; with three
 * or more parts the first is a quarter and the last half the size of the
 * others.  With one
 * part a whole batch that fits the device stays resident for
 * lmieb_rerun_device.  Returns 0, or -1 for chunks < 0. */
int lmieb_set_pipeline(int chunks);

/* Work items per SM the angular stage of `precision` is cut into (default 64
 * for FP64, 2 for the tensor-core stage); results differ only in the order of
 * partial sums.  Returns 0 or -1. */
int lmieb_set_work_granularity(int precision, double items_per_sm);
double lmieb_get_work_granularity(int precision);

/* Segment length of the tensor-core angular stage, in chunks of 16 orders:
 * its hi*hi products accumulate in FP32 (which the tensor cores truncate)
 * over one segment, then go into a running sum; shorter segments are more
 * accurate and cost more sum traffic.  Default 2.  Returns 0, or -1 outside
 * 1..64. */
int lmieb_set_split_segment(int chunks);
int lmieb_get_split_segment(void);

/* Orders per block of the phase matrix at the user angles (its tiles: 64 user
 * angles by this many orders; a case with more orders is spread over several
 * blocks whose sums are added in order): a multiple of 64 from 64 to 4096,
 * default 256; results differ only in the order of partial sums.  Returns 0
 * or -1. */
int lmieb_set_user_angle_part(int orders);
int lmieb_get_user_angle_part(void);

/* Autotuner: solves the batch in[0..n_cases) (outputs in out, allocated by
 * the caller or a previous call) repeatedly.  It first picks the angular work
 * granularity (32, 64, 128, 256 items per SM for FP64; 1, 2, 4 for the
 * tensor-core stage) by the device time of the kernels (per-stage CUDA events,
 * one sub-batch) plus the host time of packing the work items, then the
 * orders per block of the user-angle phase matrix (128, 256, 512) by that
 * stage's device time, then the pipeline depth (1, 2, 3, 4, 6 parts) by the
 * wall time of the public batch call, and keeps all three for later calls
 * (lmieb_set_work_granularity, lmieb_set_user_angle_part,
 * lmieb_set_pipeline).  Reports the granularity, the pipeline depth and the
 * best wall time (ms) through the non-NULL pointers.  Returns 0 or -1. */
int lmie_solution_autotune(int n_cases, lmie_in_data *in, lmie_out_data *out, int n_threads, int precision,
                           int *best_chunks, double *best_items, double *best_ms);

/* One 128 x 64 product of the LMIEB_PRECISION_INT8 contraction (K orders, a
 * positive multiple of 32 up to 5120; seeded operands growing like the
 * angular products) against long-double sums on the host: the largest error
 * of an element relative to max|a_i.| max|b_n.| of its row and column.
 * Returns 0 or -1. */
int lmieb_oz_selftest(int K, double *max_rel_err);

/* The same with the product waits bounded by wait_cycles (1 .. 2^31 SM clock
 * cycles; lmieb_oz_selftest uses 2^31, about a second) and, when withhold is
 * nonzero, the first chunk's products never issued: the wait for them runs
 * out, the kernel releases its tensor memory, sets its error word and returns,
 * and the call returns -1 with the device still usable -- the failure path of
 * the product kernel's bounded waits, taken without a fault. */
int lmieb_oz_selftest_wait(int K, long long wait_cycles, int withhold, double *max_rel_err);

/* Graph replay of the product path: a sub-batch whose kernel sequence is one
 * its slot ran recently (each slot keeps four) -- the same structure of
 * cases, radii, orders and angles in the same device arena, as in retrieval
 * loops that change the refractive index or the size-distribution weights
 * between calls, or the parts of a repeated pipelined call -- runs as one
 * CUDA graph, captured the second time the sequence comes.  Counts of the sequences captured and replayed since the library was
 * loaded (timing mode, radius groups and save_control launch kernel by
 * kernel).  Returns 0. */
int lmieb_graph_stats(long long *captures, long long *replays);

/* Device memory: out[0] free and out[1] total bytes of the current device
 * (cudaMemGetInfo), out[2] device bytes and out[3] pinned host bytes the
 * library holds (arenas, staging buffers, pools).  Returns 0 or -1. */
int lmieb_memory(long long out[4]);

/* lmie_solution_batch with the arithmetic chosen by `precision`. */
int lmie_solution_batch2(int n_cases, lmie_in_data *in, lmie_out_data *out, int alloc_out,
                         int verbose, int n_threads, int precision);

/* ---- adjoint (reverse-mode) gradient of an output-weighted scalar ----
 *
 * A binned size distribution shared by all wavelengths: bin b spans
 * [edges[b], edges[b+1]] (same length unit as the wavelengths), carries the
 * number weight weight[b] (uniform number density inside the bin) and is
 * integrated with n_quad Gauss-Legendre radii.  The quadrature radius r of
 * bin b has the weight W_r = weight[b] q_r (q_r its Gauss weight); the
 * distribution is normalised by N = sum_r W_r, as lmie_solution normalises
 * n(r).  The reference cannot express such a distribution in one call; it is
 * the per-radius SIZE_DIST_MONO solves combined with these weights. */
typedef struct {
     int n_bins;
     int n_quad;
     const double *edges;       /* [n_bins + 1], ascending, > 0 */
     const double *weight;      /* [n_bins], > 0 */
} lmie_bins;

/* Loss weights of one wavelength: the loss is
 *   L = c_cext Cext + c_csca Csca + c_g g
 *       + sum_i (d_p11[i] P11(theta_i) + d_p12[i] P12(theta_i)),
 * theta_i = i 180 / (n_angles - 1) degrees, with Cext, Csca, g and the phase
 * matrix normalised as lmie_solution returns them (P11 = a1, P12 = b1, the
 * elements pf[0] and pf[4] of its 6-element phase matrix).  The phase matrix
 * is evaluated from the Mie sums at theta_i directly, which is what
 * lmie_solution returns with accuracy = 0 (no truncation of the expansion).
 * d_p11 / d_p12 may be NULL (zero weights). */
typedef struct {
     double c_cext, c_csca, c_g;
     const double *d_p11;       /* [n_angles] */
     const double *d_p12;       /* [n_angles] */
} lmie_loss_weights;

/* Reverse-mode gradient of L = sum over the n_lambda wavelengths of their
 * losses, for the binned distribution `bins`, wavelength lambda[k] and
 * m = mr[k] - i mi[k].  Returns the loss in *loss, dL/dmr[k] in grad_mr[k],
 * dL/dmi[k] in grad_mi[k] and dL/dweight[b] in grad_weight[b] (any of the
 * gradient pointers may be NULL).  If values is not NULL it receives per
 * wavelength [Cext, Csca, g, P11(theta_0..), P12(theta_0..)]
 * (3 + 2 n_angles doubles each).
 *
 * One forward sweep (Mie recurrences, coefficients, the phase matrix at the
 * n_angles angles) and one reverse sweep in FP64: the derivative of the
 * logarithmic derivative D_n(z) is taken in closed form (dD_n/dz =
 * n(n+1)/z^2 - 1 - D_n^2, from the Riccati-Bessel equation), and the reverse
 * sweep re-runs the recurrences from checkpoints stored every 64 orders
 * instead of per-order arrays.  This entry point has no counterpart in the
 * reference.  Returns 0 or -1. */
int lmie_solution_adjoint(int n_lambda, const double *lambda, const double *mr, const double *mi,
                          const lmie_bins *bins, int n_angles, const lmie_loss_weights *weights,
                          double *loss, double *grad_mr, double *grad_mi, double *grad_weight,
                          double *values);

/* Checks the tensor-core contraction machinery on the device: a 128 x 64
 * product over K orders (K a positive multiple of 16, at most 4096) of seeded
 * random operands through the operand split, shared-memory layout,
 * descriptors, tcgen05.mma issue and tensor-memory reads of the
 * split-precision angular stage, with one FP32 accumulation over all of K
 * (the stage itself accumulates segments of 32 orders into a running sum),
 * against an
 * FP64 product on the host.  Writes the largest error relative to the
 * largest element of the product.  Returns 0 or -1. */
int lmieb_tc_selftest(int K, double *max_rel_err);

/* Stages of one solve, timed with CUDA events when timing is on:
 * 0 upload, 1 Mie recurrences and coefficients (K1), 2 radius reduction of
 * the cross sections (K2), 3 angular accumulation (K3), 4 normalisation,
 * 5 GSF expansion, 6 Legendre expansion, 7 phase matrix at user angles,
 * 8 download. */
#define LMIEB_N_STAGES 9

/* Host-side phases of the last lmie_solution_batch / lmie_solution_batch2
 * call, wall-clock ms: 0 preparation of the cases (size distributions,
 * derivative split, per-radius truncations; n_threads threads), 1 packing of
 * the device inputs, 2 device work with its host<->device copies, 3 unpacking
 * of the device outputs, 4 scatter into the callers' lmie_out_data; and on the
 * device's clock (CUDA events): 5 the span from the first sub-batch's upload
 * to the last one's download, 6 the sum of the sub-batches' own spans (more
 * than 5 where consecutive sub-batches overlap).  Returns LMIEB_N_HOST. */
#define LMIEB_N_HOST 7
int lmieb_last_host_timing(double *ms, int n);

/* save_control: the per-radius kernels (save1, save2) of the last
 * save_control 1 solve, or of the last save_control 2 call whose kernels were
 * not on the device, stay on the device.  A save_control 2 call hashes the
 * kernels it is given (all of their values, through the caller's row
 * pointers) and uploads them only when they differ from the kept set, so the
 * re-weighting calls of a retrieval loop send the kernels once.  Reports how
 * many save_control 2 calls found their kernels on the device (hits) and how
 * many uploaded them (misses) since the library was loaded.  Returns 0. */
int lmieb_save_cache_stats(long long *hits, long long *misses);

/* Selects the GPU the library uses (default: the CUDA runtime's current
 * device).  Must precede the first solve; one process drives one GPU. */
int lmieb_set_device(int device);

/* Turn per-stage CUDA-event timing of lmie_solution on (1) or off (0). */
int lmieb_set_timing(int on);

/* Copies the stage times (ms) of the last timed solve into ms[0..n-1];
 * returns LMIEB_N_STAGES. */
int lmieb_last_timing(double *ms, int n);

/* Re-runs the device stages 1..7 of the last solve `reps` times on the
 * inputs still resident in device memory (no host work, no copies); only
 * defined when that solve ran as one sub-batch (see lmieb_set_pipeline) --
 * with LMIEB_PRECISION_INT8, one sub-batch and the FP64 re-solve of its
 * uncertain cases, re-run one after the other -- else returns -1.  The kernel sequence is captured once per resident solve
 * into a CUDA graph; each replay is bracketed by CUDA events on the
 * library's stream, and with flush_l2 a 256 MiB buffer is written before each
 * repetition (outside the timed interval).  Returns the summed device time of
 * the replays in *ms_total, and in ms_stage[0..LMIEB_N_STAGES-1] the summed
 * per-stage times of as many further runs launched kernel by kernel between
 * events (either pointer may be NULL).  Returns 0 or -1. */
int lmieb_rerun_device(int reps, int flush_l2, double *ms_total, double *ms_stage);

/* Algorithmic work of the last solve: flops[0] angular S1/S2 contraction,
 * flops[1] Mie recurrences, flops[2] Gauss-angle expansions, flops[3] phase
 * matrix at the user angles; the number of kernel launches one device run
 * issues; and the bytes the last solve copied host-to-device and back.  Any
 * pointer may be NULL. */
int lmieb_last_work(double *flops, long long *launches, size_t *h2d, size_t *d2h);

/* Cases of the last batch call that LMIEB_PRECISION_INT8 solved again in
 * FP64 because their truncation n_coef was not certain at the fixed-point
 * contraction's error.  Returns 0. */
int lmieb_last_redo(long long *cases);

/* The LMIEB_PRECISION_INT8 product kernel of the last solve: the
 * tensor-core operations it runs (2 per 8-bit multiply-add) and, after
 * lmieb_rerun_device, its device time summed over the re-runs' stage-timed
 * passes (ms; CUDA events around its launch).  Either pointer may be NULL.
 * Returns 0. */
int lmieb_last_int8_kernel(double *tensor_ops, double *ms);

/* Measures the FP64 FMA throughput of the device (TFLOP/s) with a short
 * register-resident microbenchmark on the library's stream. */
int lmieb_fp64_peak(double *tflops);

/* Cross sections of single spheres with no device allocation.  This entry
 * point has no counterpart in the reference.  It is for callers that cannot
 * call cudaMalloc -- for example a model embedded in a host application whose
 * memory pool already owns the whole GPU, or a retrieval loop that cannot
 * afford cudaMalloc's implicit device-wide synchronisation -- and that bring
 * their own device buffers.
 *
 * For each radius[i] (device memory, n_radii of them, same length unit as
 * lambda) and m = mr - i*mi it writes to `out` (device memory, [4][n_radii])
 * the values lmie_solution returns for a SIZE_DIST_MONO distribution of that
 * radius: out[0][i] cext, out[1][i] csca, out[2][i] cbak, out[3][i] g.
 *
 * Limits: 1 <= n_radii <= 1024 and size parameters 0 < 2 pi r / lambda <= 900;
 * larger requests return -1 with an ERROR line (out-of-range radii get NaN).
 * The truncation orders n1, n2 of every radius are computed on the host with
 * the same formulas and libm as in lmie_solution (the radii are copied to the
 * host, the orders back into the static array below).
 * The work uses a fixed 24 MiB scratch array compiled into the library, which
 * every GPU that loads the library keeps until the process exits; no call
 * allocates or frees device memory.  All calls on a device share that array:
 * calls that overlap on the GPU (other threads, other streams) race on it.
 * The first call on a device looks up the array's device address; every call
 * copies the radii to the host and waits for `stream`.  Runs on the calling thread's current device on
 * `stream` (a cudaStream_t; NULL for the default stream) and returns after
 * the results are in `out`.  Returns 0 or -1. */
int lmie_cross_sections_noalloc(int n_radii, const double *radius, double lambda,
                                double mr, double mi, double *out, void *stream);

/* ---- radius sharing over processes, one per GPU ----------------------------
 * Replaces the reference's MPI build of lmie_solution(..., use_mpi = 1), which
 * deals the radii of one solve out to worker ranks round-robin and adds up
 * their cross sections and phase-matrix integrals on the master
 * (src/lmie_schedule.c:459-921, lmie_core_master / lmie_core_slave).  Here
 * every process of a group drives its own GPU: process `rank` of `world`
 * solves the radii i with i % world == rank (i in quadrature order), the
 * group sums the integrals -- 4 (1 + n_derivs) (1 + n_qang) doubles, with
 * n_qang = 0 without calc_gc and calc_lc, else lmie_calc_max_coef() -- and
 * every process then finishes the solve (normalisation, expansions, phase
 * matrix) and returns the whole result.  Every process of the group must make
 * the same calls with the same inputs.  save_control must be 0.
 * The summed block carries one double more: the number of processes whose
 * solve failed before the sum.  A process that fails there (host preparation,
 * device memory, upload, a kernel) still takes part in the sum with zero
 * integrals and a count of 1, and returns -1; every process whose sum holds
 * a nonzero count returns -1 as well -- none is left waiting in the group's
 * collective. */

/* In-place sum over the group of the `count` doubles at DEVICE address buf
 * (the integrals, then the failure count), which this process's solve has
 * just written on `stream` (a cudaStream_t, already synchronised when the
 * function is called).  The sum must be complete when the function returns;
 * 0 means success. */
typedef int (*lmieb_reduce_fn)(double *buf, long long count, void *stream, void *ctx);

/* From this call on, lmie_solution() and lmie_solution2*() called with
 * use_mpi != 0 share their radii with the group (rank, world), summing with
 * reduce(buf, count, stream, ctx); use_mpi = 0 keeps the whole solve on this
 * GPU.  world 1 with reduce NULL ends the sharing.  Returns 0 or -1. */
int lmieb_set_radius_group(int rank, int world, lmieb_reduce_fn reduce, void *ctx);

/* The same with the library's own NCCL all-reduce (FP64 sum over NVLink /
 * NVSwitch), queued on the solve's stream between the integrals and the
 * normalisation with no host synchronisation.  `id` is the 128-byte
 * ncclUniqueId that one process of the group got from lmieb_nccl_unique_id()
 * and sent to the others (over MPI, a file, a TCP store).  NCCL is loaded at
 * run time (libnccl.so.2: the one already in the process, else the system's).
 * Collective over the group.  Returns 0 or -1. */
int lmieb_nccl_unique_id(void *id);
int lmieb_set_radius_group_nccl(const void *id, int rank, int world);

/* The group in use: *rank and *world (0 and 1 when none); returns 1 when
 * use_mpi calls share their radii, else 0. */
int lmieb_get_radius_group(int *rank, int *world);

/* Two-call form for callers that sum on the host themselves (an
 * MPI_Allreduce of doubles, say).  lmieb_partial_size() is the number of
 * doubles of the integrals of `in`; lmieb_solution_partial() solves the radii
 * i % world == rank of `in` and writes their integrals to acc; after the
 * caller has summed acc over ranks 0..world-1, lmieb_solution_finish() fills
 * `out` as lmie_solution(in, out, alloc_out, verbose, 0, 0) would.  Return
 * -1 (size) or 0 / -1. */
long long lmieb_partial_size(const lmie_in_data *in);
int lmieb_solution_partial(lmie_in_data *in, int rank, int world, double *acc, int verbose);
int lmieb_solution_finish(lmie_in_data *in, lmie_out_data *out, int alloc_out, const double *acc,
                          int verbose);

/* Name, SM count and compute capability of the device the library uses. */
int lmieb_device_info(char *name, int len, int *sms, int *cc_major, int *cc_minor);

/* The CUDA stream all of the library's work is issued on (cudaStream_t). */
int lmieb_stream(void **stream);

#ifdef __cplusplus
}
#endif

#endif /* LMIE_B200_H */
