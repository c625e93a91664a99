/*
 * lmieb.h -- internal interface between the C host layer (host_*.c) and the
 * CUDA driver (driver.cu) of liblmie_b200.so.  Not installed; the public
 * interface is include/lmie_interface.h and include/lmie_b200.h.
 *
 * The host layer does what the reference does on the host before its Mie
 * core: size-distribution quadrature, moments, derivative split, and the
 * per-radius size parameters and truncation integers (computed with the host
 * libm so that n1(r), n2(r) and the global n1 are the reference's integers).
 * Everything from the Mie recurrences to the phase matrix at user angles runs
 * on the GPU.
 */
#ifndef LMIEB_H
#define LMIEB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One polydisperse problem, ready for the device.  Derivative slots are in
 * the caller's order kk = 0..nd-1; idx1/idx2 split them like the reference's
 * create_derivs_indexes (src/lmie_interface.c:304-353). */
typedef struct {
     int n;                     /* radii */
     int nd, nd1, nd2;
     const int *idx1;           /* [nd1] */
     const int *idx2;           /* [nd2] */

     double lambda;
     double mr, mi;             /* m = mr - i mi */
     const double *lambda_l;    /* [nd] */
     const double *mr_l;        /* [nd] */
     const double *mi_l;        /* [nd] */

     /* per radius (host-computed, reference src/lmie_core.c:263-292) */
     const double *x;           /* [n]        size parameter 2 pi r / lambda */
     const double *xl;          /* [nd1 * n]  d x / d p for index1 slot k (row k) */
     const double *w;           /* [(1+nd)*n] row 0: f = nr qw; row 1+kk: f_l (index1) or f_l2 (index2) */
     const int *n1r;            /* [n] */
     const int *n2r;            /* [n] */

     int n1;                    /* global truncation at r2 */
     int n_qang;                /* 2 n1 when gc or lc is wanted, else 0 */
     int n_coef;                /* 2 n1 */

     int want_gc, want_lc;      /* expansions requested (reference: gc/lc pointers non-NULL) */
     int pf_from;               /* 0: no phase matrix, 1: from gc, 2: from lc */
     int n_angles;
     const double *mu_user;     /* [n_angles] cos(theta_i), theta_i = i 180/(n_angles-1) degrees:
                                   a function of n_angles alone, so the device layer keeps
                                   one copy per distinct count */
     double accuracy;

     int save_control;          /* 0, 1 or 2 */
     const double *const *save1_rows;            /* save_control 2: rows [4][n] */
     const double *const *const *save2_rows;     /* save_control 2: rows [4][n][n_qang] (NULL if n_qang 0) */
     const double *w2;          /* [nd*n] save_control 2: nr_l qw + nr qw_l per slot */

     int precision;             /* LMIEB_PRECISION_* of include/lmie_b200.h */

     /* radius sharing over a group of processes (include/lmie_b200.h): the
        radii above are this process's share (n may be 0), and acc_mode says
        how far the device goes.  The integrals ("acc") of a case are
        4 (1+nd) (1 + n_qang) doubles: Cext, Csca, |S_back|^2, g sums per column,
        then the phase-matrix sums, rows col*4+e of n_qang, all before
        normalisation.  save_control must be 0 and the batch one case. */
     int acc_mode;              /* LMIEB_ACC_* */
     const double *acc_in;      /* LMIEB_ACC_FINISH: the group's summed integrals */
} lmieb_problem;

enum {
     LMIEB_ACC_WHOLE = 0,       /* the whole solve */
     LMIEB_ACC_PARTIAL = 1,     /* the share's integrals only, to lmieb_result.acc */
     LMIEB_ACC_FINISH = 2,      /* no radii: finish from acc_in */
     LMIEB_ACC_GROUP = 3        /* the share's integrals, summed over the registered group, finished */
};

/* Results, in device column order: column 0 = value, column 1+kk = slot kk. */
typedef struct {
     double *scal;              /* [(1+nd)*4] cext, csca, cbak, g (normalised) */
     double *gc;                /* [(1+nd)*6*n_coef] or NULL */
     double *lc;                /* [(1+nd)*6*n_coef] or NULL */
     double *pf;                /* [(1+nd)*6*n_angles] or NULL */
    /* When set, gc / lc / pf go straight to these rows instead ((1+nd)*6
     * pointers each, row col*6+e of n_coef or n_angles doubles): the
     * callers' own output rows. */
    double **gc_rows, **lc_rows, **pf_rows;
     int n_coef_out;            /* truncated count (the reference's return value) */
     double *save1;             /* [4*n] (save_control 1) or NULL */
     double *save2;             /* [4*n*n_qang] (save_control 1) or NULL */
     double *acc;               /* LMIEB_ACC_PARTIAL: the integrals (lmieb_problem) */
} lmieb_result;

/* Runs the device solve of one problem.  Returns 0 or -1 (after printing
 * "ERROR: ..."). */
int lmieb_device_solve(const lmieb_problem *p, lmieb_result *r);

/* A process of the registered radius group whose lmie_solution(use_mpi) fails
 * on the host before its device solve: takes part in the group's reduction
 * with a failure mark (4 (1 + n_derivs) (1 + n_qang) zero integrals and a
 * count of 1), so that the other processes return -1 too instead of waiting.
 * Returns -1. */
int lmieb_group_abort(int n_derivs, int n_qang);

/* 1 while the environment variable LMIEB_FAULT names `site` (host-side fault
 * injection for the tests of the failure paths), else 0. */
int lmieb_fault_injected(const char *site);

/* Runs n problems as batches on the device.  All problems must share the
 * derivative layout (nd, idx1, idx2), the requested outputs (want_gc,
 * want_lc, pf_from) and use save_control 0 when n > 1.  The cases are cut
 * into sub-batches that fit the device memory budget. */
int lmieb_device_solve_batch(int n, const lmieb_problem *p, lmieb_result *r);

/* Pipelined form of lmieb_device_solve_batch for callers that overlap their
 * own host work with the device: lmieb_device_fit gives how many of p[0..n)
 * fit one sub-batch; lmieb_device_submit packs them and queues their device
 * work (first != 0 resets the timing and work counters), returning a ticket
 * (>= 0) or -1; lmieb_device_collect waits for a ticket and unpacks its
 * results into the lmieb_result arrays given at submission (0 or -1).  Two
 * sub-batches can be in flight; submitting a third collects the oldest. */
int lmieb_device_fit(int n, const lmieb_problem *p);
long long lmieb_device_submit(int n, const lmieb_problem *p, lmieb_result *r, int first);
int lmieb_device_collect(long long ticket);

/* Records the time (ms) of host phase `phase` (0 prepare, 4 finish) of the
 * current batch call; phases 1-3 are timed inside the device layer. */
void lmieb_host_phase(int phase, double ms);

/* Device timing of the last lmieb_device_solve (ms per stage), for bench.py. */
int lmieb_last_timing(double *ms, int n);

/* fn(arg, i) for i in [0, n) on up to n_threads host threads of the library's
 * pool (internal: not exported) */
void lmieb_host_parallel(int n, int n_threads, void (*fn)(void *, int), void *arg);
/* whether per-stage timing is on (internal: not exported) */
int lmieb_timing_state(void);

#ifdef __cplusplus
}
#endif

#endif
