/*
 * host_api.c -- the drop-in C interface of liblmie_b200 (include/lmie_interface.h).
 *
 * Same entry points, argument meaning, output layout and error behaviour as
 * the reference's src/lmie_interface.c; the Mie work itself is done on the
 * GPU by lmieb_device_solve (driver.cu).  There is no CPU fallback: without a
 * usable GPU every solve returns -1 with an ERROR line.
 */
#include <complex.h>
#include <pthread.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "host.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ---- row-pointer arrays (layout of reference misc/gutil_alloc.c:18-70) ---- */
double *lmieb_arr1(size_t n) {
     return (double *) calloc(n ? n : 1, sizeof(double));
}

double **lmieb_arr2(size_t m, size_t n) {
     size_t i;
     double **p = (double **) calloc(1, m * sizeof(double *) + m * n * sizeof(double) + 8);
     double *d;
     if (!p)
          return NULL;
     d = (double *) (p + m);
     for (i = 0; i < m; ++i)
          p[i] = d + i * n;
     return p;
}

double ***lmieb_arr3(size_t a, size_t b, size_t c) {
     size_t i;
     double ***p = (double ***) calloc(1, a * sizeof(double **) + a * b * sizeof(double *) +
                                          a * b * c * sizeof(double) + 8);
     double **q, *d;
     if (!p)
          return NULL;
     q = (double **) (p + a);
     d = (double *) (q + a * b);
     for (i = 0; i < a; ++i)
          p[i] = q + i * b;
     for (i = 0; i < a * b; ++i)
          q[i] = d + i * c;
     return p;
}

/* ---- truncation (reference src/lmie_core.c:18-38) ------------------------- */
int lmieb_calc_n1(double x) {
     return (int) (x + 4.05 * pow(x, 1. / 3.) + 8);
}

int lmieb_calc_n2(int n1, double zr, double zi) {
     double az = cabs(zr + I * zi);
     double t = n1 > az ? (double) n1 : az;
     return (int) (t + 6.40 * pow(t, 1. / 3.) + 8);
}

/* ---- size distribution names (reference misc/rtutil_support.c:508-535) ---- */
static const char *const dist_names[N_SIZE_DIST_TYPES] = {
     "none", "modified_gamma", "log_normal", "power_law", "gamma",
     "modified_power_law", "modified_bimodal_log_normal", "exponential", "mono"
};

enum size_dist_type size_dist_code(const char *name) {
     int i;
     for (i = 0; i < N_SIZE_DIST_TYPES; ++i)
          if (name && strcmp(dist_names[i], name) == 0)
               return (enum size_dist_type) i;
     fprintf(stderr, "ERROR: invalid size distribution type name: %s\n", name ? name : "(null)");
     return (enum size_dist_type) -1;
}

const char *size_dist_name(enum size_dist_type code) {
     if ((int) code < 0 || (int) code >= N_SIZE_DIST_TYPES) {
          fprintf(stderr, "ERROR: invalid size distribution type index: %d\n", (int) code);
          return NULL;
     }
     return dist_names[code];
}

size_t size_dist_name_max_length(void) {
     return sizeof("modified_bimodal_log_normal");
}

/* ---- allocation helpers (reference src/lmie_interface.c:24-192) ----------- */
int lmie_calc_max_coef(double lambda, enum size_dist_type dist_type,
                       double a1, double a2, double a3, double r1, double r2) {
     (void) a3;
     if (dist_type == SIZE_DIST_POWER_LAW)
          lmieb_power_law_range(a1, a2, &r1, &r2);
     return 2 * lmieb_calc_n1(2. * M_PI * r2 / lambda);
}

int lmie_in_alloc(lmie_in_data *in, int n_derivs) {
     if (n_derivs > 0) {
          in->lambda_l = lmieb_arr1(n_derivs);
          in->mr_l = lmieb_arr1(n_derivs);
          in->mi_l = lmieb_arr1(n_derivs);
          in->a1_l = lmieb_arr1(n_derivs);
          in->a2_l = lmieb_arr1(n_derivs);
          in->a3_l = lmieb_arr1(n_derivs);
          in->a4_l = lmieb_arr1(n_derivs);
          in->a5_l = lmieb_arr1(n_derivs);
          in->r1_l = lmieb_arr1(n_derivs);
          in->r2_l = lmieb_arr1(n_derivs);
     }
     return 0;
}

void lmie_in_free(lmie_in_data *in, int flag) {
     if (flag) {
          free(in->lambda_l);
          free(in->mr_l);
          free(in->mi_l);
          free(in->a1_l);
          free(in->a2_l);
          free(in->a3_l);
          free(in->a4_l);
          free(in->a5_l);
          free(in->r1_l);
          free(in->r2_l);
     }
}

int lmie_out_alloc(lmie_in_data *in, lmie_out_data *out, int max_coef) {
     int nd = in->n_derivs;
     if (nd > 0) {
          out->r1_l = lmieb_arr1(nd);
          out->r2_l = lmieb_arr1(nd);
          out->norm_l = lmieb_arr1(nd);
          out->reff_l = lmieb_arr1(nd);
          out->veff_l = lmieb_arr1(nd);
          out->gavg_l = lmieb_arr1(nd);
          out->vavg_l = lmieb_arr1(nd);
          out->ravg_l = lmieb_arr1(nd);
          out->rvw_l = lmieb_arr1(nd);
          out->cext_l = lmieb_arr1(nd);
          out->csca_l = lmieb_arr1(nd);
          out->cbak_l = lmieb_arr1(nd);
          out->g_l = lmieb_arr1(nd);
     }
     out->gc = NULL;
     if (in->calc_gc) {
          out->gc = lmieb_arr2(6, max_coef);
          if (nd > 0)
               out->gc_l = lmieb_arr3(nd, 6, max_coef);
     }
     out->lc = NULL;
     if (in->calc_lc) {
          out->lc = lmieb_arr2(6, max_coef);
          if (nd > 0)
               out->lc_l = lmieb_arr3(nd, 6, max_coef);
     }
     out->pf = NULL;
     if (in->calc_pf) {
          out->theta = lmieb_arr1(in->n_angles);
          out->pf = lmieb_arr2(6, in->n_angles);
          if (nd > 0)
               out->pf_l = lmieb_arr3(nd, 6, in->n_angles);
     }
     if (in->save_control != 2) {
          out->save1 = NULL;
          out->save2 = NULL;
     }
     return 0;
}

void lmie_out_free(lmie_out_data *out, int flag) {
     if (flag) {
          free(out->r1_l);
          free(out->r2_l);
          free(out->norm_l);
          free(out->reff_l);
          free(out->veff_l);
          free(out->gavg_l);
          free(out->vavg_l);
          free(out->ravg_l);
          free(out->rvw_l);
          free(out->cext_l);
          free(out->csca_l);
          free(out->cbak_l);
          free(out->g_l);
     }
     if (out->gc) {
          free(out->gc);
          if (flag)
               free(out->gc_l);
     }
     if (out->lc) {
          free(out->lc);
          if (flag)
               free(out->lc_l);
     }
     if (out->pf) {
          free(out->theta);
          free(out->pf);
          if (flag)
               free(out->pf_l);
     }
     /* save1/save2 belong to the caller (reference src/lmie_interface.c:163-168) */
}

void lmie_in_zero_derivs(lmie_in_data *in, int n_derivs) {
     int i;
     for (i = 0; i < n_derivs; ++i) {
          in->lambda_l[i] = 0.;
          in->mr_l[i] = 0.;
          in->mi_l[i] = 0.;
          in->a1_l[i] = 0.;
          in->a2_l[i] = 0.;
          in->a3_l[i] = 0.;
          in->a4_l[i] = 0.;
          in->a5_l[i] = 0.;
          in->r1_l[i] = 0.;
          in->r2_l[i] = 0.;
     }
}

/* ---- solve entry points ---------------------------------------------------- */
int lmie_solution(lmie_in_data *in, lmie_out_data *out, int alloc_out, int verbose,
                  int n_threads, int use_mpi) {
     if (alloc_out) {
          int max_coef = lmie_calc_max_coef(in->lambda, in->dist_type, in->a1, in->a2,
                                            in->a3, in->r1, in->r2);
          if (lmie_out_alloc(in, out, max_coef)) {
               fprintf(stderr, "ERROR: lmie_out_alloc()\n");
               return -1;
          }
     }
     if (lmie_solution2_l(in->calc_gc, in->calc_lc, in->calc_pf,
                          in->dist_type, in->n_int1, in->n_int2, in->n_quad,
                          in->n_angles, in->n_derivs, in->save_control,
                          in->lambda, in->mr, in->mi,
                          in->a1, in->a2, in->a3, in->a4, in->a5,
                          in->r1, in->r2,
                          in->lambda_l, in->mr_l, in->mi_l,
                          in->a1_l, in->a2_l, in->a3_l, in->a4_l, in->a5_l,
                          in->r1_l, in->r2_l,
                          in->accuracy, &out->n_coef,
                          &out->r1, &out->r2,
                          &out->norm, &out->reff, &out->veff,
                          &out->gavg, &out->vavg, &out->ravg, &out->rvw,
                          &out->cext, &out->csca, &out->cbak, &out->g,
                          out->gc, out->lc, out->theta, out->pf,
                          out->r1_l, out->r2_l,
                          out->norm_l, out->reff_l, out->veff_l,
                          out->gavg_l, out->vavg_l, out->ravg_l, out->rvw_l,
                          out->cext_l, out->csca_l, out->cbak_l, out->g_l,
                          out->gc_l, out->lc_l, out->pf_l,
                          &out->save1, &out->save2,
                          verbose, n_threads, use_mpi)) {
          fprintf(stderr, "ERROR: lmie_solution2_l()\n");
          return -1;
     }
     return 0;
}

int lmie_solution2(int calc_gc, int calc_lc, int calc_pf,
                   enum size_dist_type dist_type,
                   int n_int1, int n_int2,
                   int n_quad, int n_angles, int save_control,
                   double lambda, double mr, double mi,
                   double a1, double a2, double a3, double a4, double a5,
                   double r1, double r2,
                   double accuracy, int *n_coef,
                   double *r21, double *r22,
                   double *norm, double *reff, double *veff,
                   double *gavg, double *vavg, double *ravg, double *rvw,
                   double *cext, double *csca, double *cbak, double *g,
                   double **gc, double **lc, double *theta, double **pf,
                   double ***save1, double ****save2,
                   int verbose, int n_threads, int use_mpi) {
     return lmie_solution2_l(calc_gc, calc_lc, calc_pf, dist_type, n_int1, n_int2, n_quad,
                             n_angles, 0, save_control, lambda, mr, mi, a1, a2, a3, a4, a5,
                             r1, r2, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL,
                             accuracy, n_coef, r21, r22, norm, reff, veff, gavg, vavg, ravg, rvw,
                             cext, csca, cbak, g, gc, lc, theta, pf,
                             NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL,
                             NULL, NULL, NULL, NULL, NULL, NULL, NULL,
                             save1, save2, verbose, n_threads, use_mpi);
}

/* The reference's MPI workers wait here for radii from the master
 * (src/lmie_interface.c:514-526).  Radius groups here are symmetric: every
 * process calls lmie_solution(..., use_mpi = 1) with the same inputs after
 * joining the group (lmieb_set_radius_group*), so there is no worker loop. */
int lmie_solution_slave(void) {
     fprintf(stderr, "ERROR: lmie_solution_slave(): no master/worker protocol in this library; "
             "call lmie_solution(..., use_mpi = 1) on every process of a radius group "
             "(lmieb_set_radius_group_nccl) instead\n");
     return -1;
}

/* Scratch owned by one lmie_solution2_l call. */
/* ---- one case: host preparation, device solve, scatter ------------------- */

/* Everything one lmie_solution2_l call needs: its arguments (inputs and the
 * caller's output pointers) and the scratch of its host preparation. */
typedef struct {
     /* inputs */
     int calc_gc, calc_lc, calc_pf, dist_type, n_int1, n_int2, n_quad, n_angles, n_derivs, save_control;
     double lambda, mr, mi, a1, a2, a3, a4, a5, r1, r2, accuracy;
     double *lambda_l, *mr_l, *mi_l, *a1_l, *a2_l, *a3_l, *a4_l, *a5_l, *r1_l, *r2_l;
     int verbose;
     /* outputs */
     int *n_coef;
     double *r21, *r22, *norm, *reff, *veff, *gavg, *vavg, *ravg, *rvw, *cext, *csca, *cbak, *g;
     double **gc, **lc, *theta, **pf;
     double *r21_l, *r22_l, *norm_l, *reff_l, *veff_l, *gavg_l, *vavg_l, *ravg_l, *rvw_l;
     double *cext_l, *csca_l, *cbak_l, *g_l;
     double ***gc_l, ***lc_l, ***pf_l;
     double ***save1;
     double ****save2;
     /* state */
     int rc;
     int n, nd, n_coef_all;
     double *qx, *qw, *nr, *qx_l, *qw_l, *nr_l;
     double *x, *xl, *w, *w2, *mu_user, *dev_out;
     double **rows;             /* the caller's output rows, in device column order */
     int *n1r, *n2r, *idx1, *idx2;
     /* the arrays above (qx .. idx2) come out of one zeroed block (a second
        one holds this process's share of the radii): a case's scratch is
        released with one or two calls, not one per array */
     char *blk, *blk2, *blk_at;
     size_t blk_size, blk_left;
     /* radius sharing (lmieb.h): the mode and this process's share */
     int acc_mode, share_rank, share_world;
     const double *acc_in;
     double *acc_out;
     lmieb_problem P;
     lmieb_result R;
} case_job;

/* Released case blocks, kept by size class (powers of two from 4 KB) for the
 * cases of later calls: returning them to the C heap gave the pages back to
 * the system, and the next call's allocations faulted them in again (about
 * a microsecond per case on each side).  At most BLK_POOL_MAX bytes stay.
 * Each class is a stack of pointers, so that a release does not touch the
 * block itself; a batch releases its cases under one lock. */
#define BLK_CLASSES 20
#define BLK_POOL_MAX ((size_t) 1 << 30)
typedef struct {
     char **p;
     int n, cap;
} blk_stack;
static pthread_mutex_t blk_mu = PTHREAD_MUTEX_INITIALIZER;
static blk_stack blk_pool[BLK_CLASSES];
static size_t blk_pooled;

static int blk_class(size_t bytes) {
     int c = 0;
     while (c < BLK_CLASSES && ((size_t) 4096 << c) < bytes)
          ++c;
     return c;
}

/* A zeroed block of at least `bytes` (a pooled one when there is one). */
static char *blk_get(size_t bytes) {
     const int c = blk_class(bytes);
     char *p = NULL;
     if (c == BLK_CLASSES)
          return (char *) calloc(1, bytes);
     pthread_mutex_lock(&blk_mu);
     if (blk_pool[c].n > 0) {
          p = blk_pool[c].p[--blk_pool[c].n];
          blk_pooled -= (size_t) 4096 << c;
     }
     pthread_mutex_unlock(&blk_mu);
     if (!p)
          return (char *) calloc(1, (size_t) 4096 << c);
     memset(p, 0, bytes);
     return p;
}

/* Keeps the block in the pool; 0 when it must go back to the heap instead
   (its class too large, the pool full).  Called with blk_mu held. */
static int blk_keep(char *p, size_t bytes) {
     const int c = blk_class(bytes);
     blk_stack *st;
     if (c == BLK_CLASSES || blk_pooled + ((size_t) 4096 << c) > BLK_POOL_MAX)
          return 0;
     st = &blk_pool[c];
     if (st->n == st->cap) {
          const int cap = st->cap ? 2 * st->cap : 256;
          char **q = (char **) realloc(st->p, (size_t) cap * sizeof(char *));
          if (!q)
               return 0;
          st->p = q;
          st->cap = cap;
     }
     st->p[st->n++] = p;
     blk_pooled += (size_t) 4096 << c;
     return 1;
}

/* Releases the scratch of one case (idempotent). */
static void job_free(case_job *j) {
     if (j->blk) {
          int kept;
          pthread_mutex_lock(&blk_mu);
          kept = blk_keep(j->blk, j->blk_size);
          pthread_mutex_unlock(&blk_mu);
          if (!kept)
               free(j->blk);
     }
     free(j->blk2);
     j->blk = j->blk2 = j->blk_at = NULL;
     j->blk_size = j->blk_left = 0;
     j->rows = NULL;
     j->qx = j->qw = j->nr = j->qx_l = j->qw_l = j->nr_l = NULL;
     j->x = j->xl = j->w = j->w2 = j->mu_user = j->dev_out = NULL;
     j->n1r = j->n2r = j->idx1 = j->idx2 = NULL;
}

/* bytes one array of the block takes (16-byte aligned; at least 16, as an
   empty array is still a valid pointer) */
static size_t blk_round(size_t bytes) {
     return bytes ? (bytes + 15) & ~(size_t) 15 : 16;
}

/* The next `bytes` of the case's block (zeroed), or NULL when the block the
   case was sized for is used up. */
static void *job_take(case_job *j, size_t bytes) {
     void *p;
     bytes = blk_round(bytes);
     if (!j->blk_at || bytes > j->blk_left)
          return NULL;
     p = j->blk_at;
     j->blk_at += bytes;
     j->blk_left -= bytes;
     return p;
}

/* Keeps radius i of a prepared case when i % share_world == share_rank (the
 * reference's MPI master deals its radii out to the workers the same way,
 * src/lmie_schedule.c:574-597), none when finishing from summed integrals.
 * Returns the number kept, or -1 when the host is out of memory. */
static int share_radii(case_job *j, int n, int nd, int nd1) {
     const int w = j->share_world, r0 = j->share_rank;
     const int m = j->acc_mode == LMIEB_ACC_FINISH ? 0 : (n > r0 ? (n - r0 + w - 1) / w : 0);
     const size_t mm = m > 0 ? (size_t) m : 1;
     const size_t bx = blk_round(mm * 8), bxl = blk_round(mm * (nd1 > 0 ? nd1 : 1) * 8);
     const size_t bw = blk_round(mm * (1 + nd) * 8), bn = blk_round(mm * 4);
     char *b = (char *) calloc(1, bx + bxl + bw + 2 * bn);
     double *x = (double *) b, *xl = (double *) (b + bx), *wt = (double *) (b + bx + bxl);
     int *n1r = (int *) (b + bx + bxl + bw), *n2r = (int *) (b + bx + bxl + bw + bn);
     int t, k;
     if (!b)
          return -1;
     for (t = 0; t < m; ++t) {
          const int i = r0 + t * w;
          x[t] = j->x[i];
          n1r[t] = j->n1r[i];
          n2r[t] = j->n2r[i];
          for (k = 0; k < nd1; ++k)
               xl[(size_t) k * m + t] = j->xl[(size_t) k * n + i];
          for (k = 0; k <= nd; ++k)
               wt[(size_t) k * m + t] = j->w[(size_t) k * n + i];
     }
     free(j->blk2);
     j->blk2 = b;
     j->x = x; j->xl = xl; j->w = wt; j->n1r = n1r; j->n2r = n2r;
     return m;
}

/* Host steps before the Mie core (reference src/lmie_interface.c:404-451,
 * src/lmie_schedule.c:1004-1072, src/lmie_core.c:263-292): size distribution,
 * moments, derivative split, per-radius size parameters and truncation,
 * user angles; fills j->P and points j->R at the output staging. */
/* cos(theta_i) of n equally spaced user angles theta_i = i 180/(n-1) degrees
 * (the reference's arithmetic, misc/rtutil_scat_int.c:487-503) */
static void user_cosines_fill(int n, double *mu) {
     const double d = 180. / (n - 1);
     int i;
     for (i = 0; i < n; ++i)
          mu[i] = cos((i * d) * (M_PI / 180.0));
}

/* The cosines of one count, computed once per count up to MU_CACHE_MAX and
 * kept: the cases of a batch share their user angles.  NULL above the limit
 * (the caller fills its own array). */
#define MU_CACHE_MAX 4096
static pthread_mutex_t mu_cache_mu = PTHREAD_MUTEX_INITIALIZER;
static double *mu_cache[MU_CACHE_MAX + 1];

static const double *user_cosines(int n) {
     double *p;
     if (n < 1 || n > MU_CACHE_MAX)
          return NULL;
     pthread_mutex_lock(&mu_cache_mu);
     p = mu_cache[n];
     if (!p && (p = (double *) malloc(sizeof(double) * (size_t) n)) != NULL) {
          user_cosines_fill(n, p);
          mu_cache[n] = p;
     }
     pthread_mutex_unlock(&mu_cache_mu);
     return p;
}

static int job_prepare(case_job *j) {
     int n, nd = j->n_derivs > 0 ? j->n_derivs : 0, nd1 = 0, nd2 = 0, i, k;
     const double *mu_user = NULL;
     int n1, n_qang, ncol;
     double x2;
     double complex m;
     lmieb_dist_in din;
     lmieb_dist_out dout;
     lmieb_moments_out mom;

     j->nd = nd;
     /* input check (reference src/lmie_interface.c:404-408) */
     if (j->calc_pf && (!j->calc_gc && !j->calc_lc)) {
          fprintf(stderr, "ERROR: either calc_gc or calc_lc must be set to true when "
                  "calc_pf is true\n");
          return -1;
     }
     if (j->save_control < 0 || j->save_control > 2) {
          fprintf(stderr, "ERROR: invalid save_control: %d\n", j->save_control);
          return -1;
     }
     if (j->calc_pf && j->n_angles < 1) {
          fprintf(stderr, "ERROR: n_angles must be >= 1 when calc_pf is true\n");
          return -1;
     }
     n = lmieb_dist_count(j->dist_type, j->n_int1, j->n_int2, j->n_quad);
     if (n <= 0) {
          if (n == 0)
               fprintf(stderr, "ERROR: size distribution has no quadrature points\n");
          return -1;
     }
     j->n = n;
     {
          /* the block: every array below at its largest (the Mie split nd1 <= nd) */
          const size_t un = (size_t) n, und = (size_t) (nd > 0 ? nd : 1), ncol1 = (size_t) (1 + nd);
          const size_t bytes = 3 * blk_round(un * 8) + 3 * blk_round(un * nd * 8) + 2 * blk_round(und * 4) +
                               blk_round(un * 8) + blk_round(un * und * 8) + blk_round(un * ncol1 * 8) +
                               2 * blk_round(un * 4) +
                               (j->save_control == 2 ? blk_round(un * und * 8) : 0) +
                               (j->calc_pf && j->n_angles > 0 ? blk_round((size_t) j->n_angles * 8) : 0) +
                               blk_round(ncol1 * 4 * 8) + blk_round(3 * ncol1 * 6 * sizeof(double *));
          j->blk = blk_get(bytes);
          if (!j->blk) {
               fprintf(stderr, "ERROR: lmie_b200: out of host memory for a case's scratch\n");
               return -1;
          }
          j->blk_at = j->blk;
          j->blk_size = j->blk_left = bytes;
     }

     /* size distribution quadrature and moments */
     j->qx = (double *) job_take(j, (size_t) n * 8);
     j->qw = (double *) job_take(j, (size_t) n * 8);
     j->nr = (double *) job_take(j, (size_t) n * 8);
     j->qx_l = (double *) job_take(j, (size_t) n * nd * 8);
     j->qw_l = (double *) job_take(j, (size_t) n * nd * 8);
     j->nr_l = (double *) job_take(j, (size_t) n * nd * 8);
     memset(&din, 0, sizeof(din));
     din.dist_type = j->dist_type; din.n_int1 = j->n_int1; din.n_int2 = j->n_int2;
     din.n_quad = j->n_quad; din.nd = nd;
     din.a1 = j->a1; din.a2 = j->a2; din.a3 = j->a3; din.a4 = j->a4; din.a5 = j->a5;
     din.r1 = j->r1; din.r2 = j->r2;
     din.a1_l = j->a1_l; din.a2_l = j->a2_l; din.a3_l = j->a3_l; din.a4_l = j->a4_l;
     din.a5_l = j->a5_l; din.r1_l = j->r1_l; din.r2_l = j->r2_l;
     dout.qx = j->qx; dout.qw = j->qw; dout.nr = j->nr;
     dout.qx_l = j->qx_l; dout.qw_l = j->qw_l; dout.nr_l = j->nr_l;
     dout.r1_l = j->r21_l; dout.r2_l = j->r22_l; dout.norm_l = j->norm_l;
     if (lmieb_particle_dist(&din, &dout) < 0) {
          fprintf(stderr, "ERROR: get_particle_dist()\n");
          return -1;
     }
     *j->r21 = dout.r1;
     *j->r22 = dout.r2;
     *j->norm = dout.norm;
     mom.reff_l = j->reff_l; mom.veff_l = j->veff_l; mom.gavg_l = j->gavg_l;
     mom.vavg_l = j->vavg_l; mom.ravg_l = j->ravg_l; mom.rvw_l = j->rvw_l;
     lmieb_moments(n, nd, j->qx, j->qw, j->nr, j->qx_l, j->qw_l, j->nr_l, &mom);
     *j->reff = mom.reff; *j->veff = mom.veff; *j->gavg = mom.gavg;
     *j->vavg = mom.vavg; *j->ravg = mom.ravg; *j->rvw = mom.rvw;

     /* derivative split (reference src/lmie_interface.c:304-353) */
     j->idx1 = (int *) job_take(j, (size_t) (nd > 0 ? nd : 1) * 4);
     j->idx2 = (int *) job_take(j, (size_t) (nd > 0 ? nd : 1) * 4);
     for (i = 0; i < nd; ++i) {
          if (j->lambda_l[i] != 0. || j->mr_l[i] != 0. || j->mi_l[i] != 0. ||
              j->r21_l[i] != 0. || j->r22_l[i] != 0.)
               j->idx1[nd1++] = i;
          else
               j->idx2[nd2++] = i;
     }

     /* global truncation (reference src/lmie_schedule.c:1004-1017) */
     m = j->mr - I * j->mi;
     x2 = 2. * M_PI * *j->r22 / j->lambda;
     n1 = lmieb_calc_n1(x2);
     n_qang = (!j->gc && !j->lc) ? 0 : 2 * n1;
     j->n_coef_all = 2 * n1;

     /* per-radius size parameters, truncation and weights
      * (reference src/lmie_core.c:263-292) */
     j->x = (double *) job_take(j, (size_t) n * 8);
     j->xl = (double *) job_take(j, (size_t) n * (nd > 0 ? nd : 1) * 8);
     j->w = (double *) job_take(j, (size_t) n * (1 + nd) * 8);
     j->n1r = (int *) job_take(j, (size_t) n * 4);
     j->n2r = (int *) job_take(j, (size_t) n * 4);
     for (i = 0; i < n; ++i) {
          double x = 2. * M_PI * j->qx[i] / j->lambda;
          double complex z = m * x;
          j->x[i] = x;
          j->n1r[i] = lmieb_calc_n1(x);
          j->n2r[i] = lmieb_calc_n2(j->n1r[i], creal(z), cimag(z));
          j->w[i] = j->nr[i] * j->qw[i];
          for (k = 0; k < nd1; ++k) {
               int kk = j->idx1[k];
               j->xl[(size_t) k * n + i] = 2. * M_PI * (j->qx_l[(size_t) i * nd + kk] -
                                           j->qx[i] * j->lambda_l[kk] / j->lambda) / j->lambda;
               j->w[(size_t) (1 + kk) * n + i] = j->nr_l[(size_t) i * nd + kk] * j->qw[i] +
                                                 j->nr[i] * j->qw_l[(size_t) i * nd + kk];
          }
          for (k = 0; k < nd2; ++k) {
               int kk = j->idx2[k];
               j->w[(size_t) (1 + kk) * n + i] = j->nr_l[(size_t) i * nd + kk] * j->qw[i];
          }
     }
     if (n1 < 1 || j->n1r[n - 1] < 1) {
          fprintf(stderr, "ERROR: invalid size parameter (lambda = %g, r2 = %g)\n", j->lambda, *j->r22);
          return -1;
     }
     for (i = 0; i < n; ++i) {
          if (j->n1r[i] > n1) {
               fprintf(stderr, "ERROR: radius %d (r = %g) lies above r2 = %g\n", i, j->qx[i], *j->r22);
               return -1;
          }
     }

     if (j->acc_mode != LMIEB_ACC_WHOLE) {
          if (j->save_control != 0) {
               fprintf(stderr, "ERROR: radius sharing (use_mpi) needs save_control = 0\n");
               return -1;
          }
          n = share_radii(j, n, nd, nd1);
          if (n < 0) {
               fprintf(stderr, "ERROR: lmie_b200: out of host memory for a case's scratch\n");
               return -1;
          }
     }

     /* save_control: allocate / gather the per-radius kernels */
     if (j->save_control == 1) {
          *j->save1 = lmieb_arr2(4, n);
          *j->save2 = lmieb_arr3(4, n, n_qang > 0 ? n_qang : 1);
     }
     if (j->save_control == 2) {
          if (!j->save1 || !*j->save1 || (n_qang > 0 && (!j->save2 || !*j->save2))) {
               fprintf(stderr, "ERROR: save_control = 2 needs save1 and save2 from a "
                       "save_control = 1 call\n");
               return -1;
          }
          j->w2 = (double *) job_take(j, (size_t) n * (nd > 0 ? nd : 1) * 8);
          for (i = 0; i < n; ++i)
               for (k = 0; k < nd2; ++k) {
                    int kk = j->idx2[k];
                    j->w2[(size_t) kk * n + i] = j->nr_l[(size_t) i * nd + kk] * j->qw[i] +
                                                 j->nr[i] * j->qw_l[(size_t) i * nd + kk];
               }
          /* the caller's kernels are read through their row pointers by the
             device layer, which keeps the last set it saw on the device */
     }

     /* user angles (reference misc/rtutil_scat_int.c:487-503,580): the
        caller's theta, and their cosines shared by every case of that count */
     if (j->calc_pf) {
          double d = 180. / (j->n_angles - 1);
          for (i = 0; i < j->n_angles; ++i)
               j->theta[i] = i * d;
          mu_user = user_cosines(j->n_angles);
          if (!mu_user) {
               j->mu_user = (double *) job_take(j, (size_t) j->n_angles * 8);
               user_cosines_fill(j->n_angles, j->mu_user);
               mu_user = j->mu_user;
          }
     }

     /* device problem and result staging */
     memset(&j->P, 0, sizeof(j->P));
     j->P.n = n; j->P.nd = nd; j->P.nd1 = nd1; j->P.nd2 = nd2;
     j->P.idx1 = j->idx1; j->P.idx2 = j->idx2;
     j->P.lambda = j->lambda; j->P.mr = j->mr; j->P.mi = j->mi;
     j->P.lambda_l = j->lambda_l; j->P.mr_l = j->mr_l; j->P.mi_l = j->mi_l;
     j->P.x = j->x; j->P.xl = j->xl; j->P.w = j->w; j->P.n1r = j->n1r; j->P.n2r = j->n2r;
     j->P.n1 = n1; j->P.n_qang = n_qang; j->P.n_coef = j->n_coef_all;
     j->P.want_gc = j->gc != NULL; j->P.want_lc = j->lc != NULL;
     j->P.pf_from = j->calc_pf ? (j->calc_gc ? 1 : 2) : 0;
     j->P.n_angles = j->calc_pf ? j->n_angles : 0;
     j->P.mu_user = mu_user;
     j->P.accuracy = j->accuracy;
     j->P.save_control = j->save_control;
     j->P.acc_mode = j->acc_mode;
     j->P.acc_in = j->acc_in;
     if (j->save_control == 2) {
          j->P.save1_rows = (const double *const *) *j->save1;
          j->P.save2_rows = n_qang > 0 ? (const double *const *const *) *j->save2 : NULL;
          j->P.w2 = j->w2;
     }
     /* results: the scalars in a small staging array, the expansions and the
        phase matrix straight into the caller's rows */
     ncol = 1 + nd;
     j->dev_out = (double *) job_take(j, (size_t) ncol * 4 * 8);
     memset(&j->R, 0, sizeof(j->R));
     j->R.scal = j->dev_out;
     j->rows = (double **) job_take(j, (size_t) 3 * ncol * 6 * sizeof(double *));
     for (k = 0; k < ncol * 6; ++k) {
          const int col = k / 6, e = k % 6;
          if (j->P.want_gc)
               j->rows[k] = col == 0 ? j->gc[e] : j->gc_l[col - 1][e];
          if (j->P.want_lc)
               j->rows[ncol * 6 + k] = col == 0 ? j->lc[e] : j->lc_l[col - 1][e];
          if (j->P.n_angles > 0)
               j->rows[2 * ncol * 6 + k] = col == 0 ? j->pf[e] : j->pf_l[col - 1][e];
     }
     if (j->acc_mode != LMIEB_ACC_PARTIAL) {
          j->R.gc_rows = j->P.want_gc ? j->rows : NULL;
          j->R.lc_rows = j->P.want_lc ? j->rows + ncol * 6 : NULL;
          j->R.pf_rows = j->P.n_angles > 0 ? j->rows + 2 * ncol * 6 : NULL;
     }
     j->R.acc = j->acc_out;
     if (j->save_control == 1) {
          j->R.save1 = (*j->save1)[0];
          j->R.save2 = (*j->save2)[0][0];
     }
     if (j->verbose)
          fprintf(stderr, "lmie_b200: n_radii = %d, n1 = %d, n_qang = %d, n_derivs = %d (%d Mie, %d shape)\n",
                  n, n1, n_qang, nd, nd1, nd2);
     return 0;
}

/* Copies a solved case's results into the caller's arrays. */
static void job_finish(case_job *j) {
     int nd = j->nd, k;
     const double *scal = j->R.scal;
     *j->cext = scal[0];
     *j->csca = scal[1];
     *j->cbak = scal[2];
     *j->g = scal[3];
     for (k = 0; k < nd; ++k) {
          j->cext_l[k] = scal[(1 + k) * 4 + 0];
          j->csca_l[k] = scal[(1 + k) * 4 + 1];
          j->cbak_l[k] = scal[(1 + k) * 4 + 2];
          j->g_l[k] = scal[(1 + k) * 4 + 3];
     }
     /* gc, lc and pf were written into the caller's rows when unpacked */
     *j->n_coef = j->R.n_coef_out;
}

int lmie_solution2_l(int calc_gc, int calc_lc, int calc_pf,
                     enum size_dist_type dist_type,
                     int n_int1, int n_int2, int n_quad,
                     int n_angles, int n_derivs, int save_control,
                     double lambda, double mr, double mi,
                     double a1, double a2, double a3, double a4, double a5,
                     double r1, double r2,
                     double *lambda_l, double *mr_l, double *mi_l,
                     double *a1_l, double *a2_l, double *a3_l, double *a4_l, double *a5_l,
                     double *r1_l, double *r2_l,
                     double accuracy, int *n_coef,
                     double *r21, double *r22,
                     double *norm, double *reff, double *veff,
                     double *gavg, double *vavg, double *ravg, double *rvw,
                     double *cext, double *csca, double *cbak, double *g,
                     double **gc, double **lc, double *theta, double **pf,
                     double *r21_l, double *r22_l,
                     double *norm_l, double *reff_l, double *veff_l,
                     double *gavg_l, double *vavg_l, double *ravg_l, double *rvw_l,
                     double *cext_l, double *csca_l, double *cbak_l, double *g_l,
                     double ***gc_l, double ***lc_l, double ***pf_l,
                     double ***save1, double ****save2,
                     int verbose, int n_threads, int use_mpi) {
     case_job j;
     int rc;
     (void) n_threads;
     memset(&j, 0, sizeof(j));
     /* use_mpi: the radii are shared with the registered group (the
        reference's MPI path, src/lmie_schedule.c:1125-1152) */
     if (use_mpi && lmieb_get_radius_group(&j.share_rank, &j.share_world))
          j.acc_mode = LMIEB_ACC_GROUP;
     j.calc_gc = calc_gc; j.calc_lc = calc_lc; j.calc_pf = calc_pf; j.dist_type = dist_type;
     j.n_int1 = n_int1; j.n_int2 = n_int2; j.n_quad = n_quad; j.n_angles = n_angles;
     j.n_derivs = n_derivs; j.save_control = save_control;
     j.lambda = lambda; j.mr = mr; j.mi = mi; j.a1 = a1; j.a2 = a2; j.a3 = a3; j.a4 = a4; j.a5 = a5;
     j.r1 = r1; j.r2 = r2; j.accuracy = accuracy;
     j.lambda_l = lambda_l; j.mr_l = mr_l; j.mi_l = mi_l; j.a1_l = a1_l; j.a2_l = a2_l;
     j.a3_l = a3_l; j.a4_l = a4_l; j.a5_l = a5_l; j.r1_l = r1_l; j.r2_l = r2_l;
     j.verbose = verbose;
     j.n_coef = n_coef; j.r21 = r21; j.r22 = r22; j.norm = norm; j.reff = reff; j.veff = veff;
     j.gavg = gavg; j.vavg = vavg; j.ravg = ravg; j.rvw = rvw;
     j.cext = cext; j.csca = csca; j.cbak = cbak; j.g = g;
     j.gc = gc; j.lc = lc; j.theta = theta; j.pf = pf;
     j.r21_l = r21_l; j.r22_l = r22_l; j.norm_l = norm_l; j.reff_l = reff_l; j.veff_l = veff_l;
     j.gavg_l = gavg_l; j.vavg_l = vavg_l; j.ravg_l = ravg_l; j.rvw_l = rvw_l;
     j.cext_l = cext_l; j.csca_l = csca_l; j.cbak_l = cbak_l; j.g_l = g_l;
     j.gc_l = gc_l; j.lc_l = lc_l; j.pf_l = pf_l;
     j.save1 = save1; j.save2 = save2;
     rc = lmieb_fault_injected("prepare") ? -1 : job_prepare(&j);
     if (rc != 0 && j.acc_mode == LMIEB_ACC_GROUP)
          /* the other processes of the group must not wait for this one */
          lmieb_group_abort(n_derivs, (calc_gc || calc_lc) ?
                            lmie_calc_max_coef(lambda, dist_type, a1, a2, a3, r1, r2) : 0);
     if (rc == 0 && lmieb_device_solve(&j.P, &j.R)) {
          fprintf(stderr, "ERROR: lmie_core_solution()\n");
          rc = -1;
     }
     if (rc == 0)
          job_finish(&j);
     job_free(&j);
     return rc;
}

/* ---- batches -------------------------------------------------------------- */

static double wall_ms(void) {
     struct timespec ts;
     clock_gettime(CLOCK_MONOTONIC, &ts);
     return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

static void job_from_struct(case_job *j, lmie_in_data *in, lmie_out_data *out, int verbose) {
     memset(j, 0, sizeof(*j));
     j->calc_gc = in->calc_gc; j->calc_lc = in->calc_lc; j->calc_pf = in->calc_pf;
     j->dist_type = in->dist_type; j->n_int1 = in->n_int1; j->n_int2 = in->n_int2;
     j->n_quad = in->n_quad; j->n_angles = in->n_angles; j->n_derivs = in->n_derivs;
     j->save_control = in->save_control;
     j->lambda = in->lambda; j->mr = in->mr; j->mi = in->mi;
     j->a1 = in->a1; j->a2 = in->a2; j->a3 = in->a3; j->a4 = in->a4; j->a5 = in->a5;
     j->r1 = in->r1; j->r2 = in->r2; j->accuracy = in->accuracy;
     j->lambda_l = in->lambda_l; j->mr_l = in->mr_l; j->mi_l = in->mi_l; j->a1_l = in->a1_l;
     j->a2_l = in->a2_l; j->a3_l = in->a3_l; j->a4_l = in->a4_l; j->a5_l = in->a5_l;
     j->r1_l = in->r1_l; j->r2_l = in->r2_l;
     j->verbose = verbose;
     j->n_coef = &out->n_coef; j->r21 = &out->r1; j->r22 = &out->r2; j->norm = &out->norm;
     j->reff = &out->reff; j->veff = &out->veff; j->gavg = &out->gavg; j->vavg = &out->vavg;
     j->ravg = &out->ravg; j->rvw = &out->rvw; j->cext = &out->cext; j->csca = &out->csca;
     j->cbak = &out->cbak; j->g = &out->g;
     j->gc = out->gc; j->lc = out->lc; j->theta = out->theta; j->pf = out->pf;
     j->r21_l = out->r1_l; j->r22_l = out->r2_l; j->norm_l = out->norm_l; j->reff_l = out->reff_l;
     j->veff_l = out->veff_l; j->gavg_l = out->gavg_l; j->vavg_l = out->vavg_l;
     j->ravg_l = out->ravg_l; j->rvw_l = out->rvw_l; j->cext_l = out->cext_l;
     j->csca_l = out->csca_l; j->cbak_l = out->cbak_l; j->g_l = out->g_l;
     j->gc_l = out->gc_l; j->lc_l = out->lc_l; j->pf_l = out->pf_l;
     j->save1 = &out->save1; j->save2 = &out->save2;
}

typedef struct {
     case_job *jobs;
     lmie_in_data *in;          /* stage 0: the cases' inputs and outputs */
     lmie_out_data *out;
     int n, stage, verbose;
} job_pool;

static void job_stage(void *arg, int i) {
     job_pool *p = (job_pool *) arg;
     if (p->stage == 0) {
          job_from_struct(&p->jobs[i], &p->in[i], &p->out[i], p->verbose);
          p->jobs[i].rc = job_prepare(&p->jobs[i]);
     } else if (p->jobs[i].rc == 0) {
          job_finish(&p->jobs[i]);
     }
}

/* Runs stage 0 (set up from in/out and prepare) or 1 (finish) of every job
 * on up to n_threads host threads. */
static void run_jobs_io(case_job *jobs, lmie_in_data *in, lmie_out_data *out, int verbose, int n, int stage,
                        int n_threads) {
     job_pool p;
     p.jobs = jobs; p.in = in; p.out = out; p.verbose = verbose; p.n = n; p.stage = stage;
     lmieb_host_parallel(n, n_threads > 0 ? n_threads : 1, job_stage, &p);
}

static void run_jobs(case_job *jobs, int n, int stage, int n_threads) {
     run_jobs_io(jobs, NULL, NULL, 0, n, stage, n_threads);
}

/* Releases the host scratch of jobs[0..n) on the calling thread: the blocks
 * go to the pool under one lock (job_free is idempotent). */
static void jobs_release(case_job *jobs, int n) {
     int i;
     pthread_mutex_lock(&blk_mu);
     for (i = 0; i < n; ++i)
          if (jobs[i].blk && blk_keep(jobs[i].blk, jobs[i].blk_size))
               jobs[i].blk = NULL;
     pthread_mutex_unlock(&blk_mu);
     for (i = 0; i < n; ++i)
          job_free(&jobs[i]);
}

/* Two prepared cases can share a device batch when their derivative layout
 * and requested outputs agree. */
static int jobs_compatible(const case_job *a, const case_job *b) {
     int q;
     if (a->P.save_control != 0 || b->P.save_control != 0)
          return 0;
     if (a->P.nd != b->P.nd || a->P.nd1 != b->P.nd1 || a->P.nd2 != b->P.nd2 ||
         a->P.want_gc != b->P.want_gc || a->P.want_lc != b->P.want_lc || a->P.pf_from != b->P.pf_from)
          return 0;
     for (q = 0; q < a->P.nd1; ++q)
          if (a->P.idx1[q] != b->P.idx1[q])
               return 0;
     for (q = 0; q < a->P.nd2; ++q)
          if (a->P.idx2[q] != b->P.idx2[q])
               return 0;
     return 1;
}

/* ---- radius sharing, two-call form ---------------------------------------- */

long long lmieb_partial_size(const lmie_in_data *in) {
     const int nd = in->n_derivs > 0 ? in->n_derivs : 0;
     const int nq = (in->calc_gc || in->calc_lc) ?
                    lmie_calc_max_coef(in->lambda, in->dist_type, in->a1, in->a2, in->a3, in->r1, in->r2) : 0;
     return 4LL * (1 + nd) * (1 + nq);
}

/* One device solve of `in` into `out` in radius-sharing mode acc_mode. */
static int share_solve(lmie_in_data *in, lmie_out_data *out, int acc_mode, int rank, int world,
                       const double *acc_in, double *acc_out, int verbose) {
     case_job j;
     int rc;
     job_from_struct(&j, in, out, verbose);
     j.acc_mode = acc_mode;
     j.share_rank = rank;
     j.share_world = world;
     j.acc_in = acc_in;
     j.acc_out = acc_out;
     rc = job_prepare(&j);
     if (rc == 0 && 4LL * (1 + j.P.nd) * (1 + j.P.n_qang) != lmieb_partial_size(in)) {
          fprintf(stderr, "ERROR: radius sharing: the integrals of this case are not "
                  "lmieb_partial_size() doubles (were out's gc / lc arrays set by hand?)\n");
          rc = -1;
     }
     if (rc == 0 && lmieb_device_solve(&j.P, &j.R)) {
          fprintf(stderr, "ERROR: lmie_core_solution()\n");
          rc = -1;
     }
     if (rc == 0 && acc_mode == LMIEB_ACC_FINISH)
          job_finish(&j);
     job_free(&j);
     return rc;
}

int lmieb_solution_partial(lmie_in_data *in, int rank, int world, double *acc, int verbose) {
     lmie_out_data out;
     int rc;
     if (world < 1 || rank < 0 || rank >= world || !acc) {
          fprintf(stderr, "ERROR: lmieb_solution_partial(): rank %d of %d%s\n", rank, world,
                  acc ? "" : ", acc NULL");
          return -1;
     }
     /* scratch for the host-side outputs (moments, r1, r2, ...) */
     memset(&out, 0, sizeof(out));
     if (lmie_out_alloc(in, &out, lmie_calc_max_coef(in->lambda, in->dist_type, in->a1, in->a2,
                                                     in->a3, in->r1, in->r2))) {
          fprintf(stderr, "ERROR: lmie_out_alloc()\n");
          return -1;
     }
     rc = share_solve(in, &out, LMIEB_ACC_PARTIAL, rank, world, NULL, acc, verbose);
     lmie_out_free(&out, in->n_derivs > 0);
     return rc;
}

int lmieb_solution_finish(lmie_in_data *in, lmie_out_data *out, int alloc_out, const double *acc,
                          int verbose) {
     if (!acc) {
          fprintf(stderr, "ERROR: lmieb_solution_finish(): acc NULL\n");
          return -1;
     }
     if (alloc_out && lmie_out_alloc(in, out, lmie_calc_max_coef(in->lambda, in->dist_type, in->a1,
                                                                 in->a2, in->a3, in->r1, in->r2))) {
          fprintf(stderr, "ERROR: lmie_out_alloc()\n");
          return -1;
     }
     return share_solve(in, out, LMIEB_ACC_FINISH, 0, 1, acc, NULL, verbose);
}

int lmie_solution_batch(int n_cases, lmie_in_data *in, lmie_out_data *out, int alloc_out,
                        int verbose, int n_threads) {
     return lmie_solution_batch2(n_cases, in, out, alloc_out, verbose, n_threads, LMIEB_PRECISION_FP64);
}

static int g_pipeline = 0;

int lmieb_set_pipeline(int chunks) {
     if (chunks < 0)
          return -1;
     g_pipeline = chunks;
     return 0;
}

/* Submitted device work of one chunk of cases: tickets with their ranges in
 * the P/R arrays. */
typedef struct {
     long long *ticket;
     int n;
} chunk_tickets;

/* Waits for a chunk's tickets, copies the results back to their jobs and
 * scatters them into the callers' outputs. */
static int finish_chunk(chunk_tickets *ct, case_job *jobs, int j0, int j1, const int *pos2job,
                        const int *pbeg, const int *pend, lmieb_result *R, int n_threads, int ok,
                        double *t_finish) {
     int rc = ok ? 0 : -1, q, i;
     double t0;
     for (q = 0; q < ct->n; ++q)
          if (lmieb_device_collect(ct->ticket[q])) {
               fprintf(stderr, "ERROR: lmie_solution_batch(): device solve\n");
               rc = -1;
          }
     if (rc == 0) {
          for (q = 0; q < ct->n; ++q)
               for (i = pbeg[q]; i < pend[q]; ++i)
                    jobs[pos2job[i]].R = R[i];
          t0 = wall_ms();
          run_jobs(jobs + j0, j1 - j0, 1, n_threads);
          *t_finish += wall_ms() - t0;
     }
     /* the chunk's host scratch is no longer referenced: released here, while
        the device still works on the next chunk */
     jobs_release(jobs + j0, j1 - j0);
     ct->n = 0;
     return rc;
}

/* relative size of chunk c of `chunks` (see lmie_solution_batch2) */
static double chunk_weight(int c, int chunks) {
     if (chunks < 3)
          return 1.;
     return c == 0 ? 0.25 : (c == chunks - 1 ? 0.5 : 1.);
}

int lmie_solution_batch2(int n_cases, lmie_in_data *in, lmie_out_data *out, int alloc_out,
                         int verbose, int n_threads, int precision) {
     case_job *jobs;
     lmieb_problem *P;
     lmieb_result *R;
     int *done, *pos2job, *bnd, i, k, c, rc = 0, np = 0, chunks, first = 1, n_last = 0, prepared = 0;
     long long *tk[2];
     int *tb[2], *te[2];
     chunk_tickets ct[2];
     int cj0[2] = {0, 0}, cj1[2] = {0, 0};
     double t0, t_prep = 0., t_fin = 0.;
     if (n_cases <= 0)
          return 0;
     if (precision != LMIEB_PRECISION_FP64 && precision != LMIEB_PRECISION_TF32X3 &&
         precision != LMIEB_PRECISION_INT8) {
          fprintf(stderr, "ERROR: lmie_solution_batch2(): unknown precision %d\n", precision);
          return -1;
     }
     if (alloc_out) {
          for (i = 0; i < n_cases; ++i) {
               int max_coef = lmie_calc_max_coef(in[i].lambda, in[i].dist_type, in[i].a1, in[i].a2,
                                                 in[i].a3, in[i].r1, in[i].r2);
               if (lmie_out_alloc(&in[i], &out[i], max_coef)) {
                    fprintf(stderr, "ERROR: lmie_out_alloc()\n");
                    return -1;
               }
          }
     }
     /* every job is set up (zeroed first) by its chunk's preparation */
     jobs = (case_job *) malloc((size_t) n_cases * sizeof(case_job));
     P = (lmieb_problem *) calloc(n_cases, sizeof(lmieb_problem));
     R = (lmieb_result *) calloc(n_cases, sizeof(lmieb_result));
     done = (int *) calloc(n_cases, sizeof(int));
     pos2job = (int *) calloc(n_cases, sizeof(int));
     for (c = 0; c < 2; ++c) {
          tk[c] = (long long *) calloc(n_cases, sizeof(long long));
          tb[c] = (int *) calloc(n_cases, sizeof(int));
          te[c] = (int *) calloc(n_cases, sizeof(int));
          ct[c].ticket = tk[c];
          ct[c].n = 0;
     }
     /* chunks of cases: chunk c is prepared and packed while the device works
        on chunk c - 1, whose results are then unpacked and scattered */
     chunks = g_pipeline > 0 ? g_pipeline : (n_cases / 640 < 6 ? (n_cases / 640 > 1 ? n_cases / 640 : 1) : 6);
     if (chunks > n_cases)
          chunks = n_cases;
     /* chunk boundaries: with three or more chunks the first is a quarter and
        the last half the size of the others, so that the device starts after a
        short preparation and the last results are unpacked soon after it ends */
     bnd = (int *) calloc((size_t) chunks + 1, sizeof(int));
     {
          double wsum = 0., acc = 0.;
          for (c = 0; c < chunks; ++c)
               wsum += chunk_weight(c, chunks);
          for (c = 0; c < chunks; ++c) {
               acc += chunk_weight(c, chunks);
               bnd[c + 1] = c + 1 == chunks ? n_cases : (int) (n_cases * (acc / wsum) + 0.5);
               if (bnd[c + 1] < bnd[c] + 1)
                    bnd[c + 1] = bnd[c] + 1;
          }
     }
     for (c = 0; c < chunks && bnd[c] < n_cases; ++c) {
          const int j0 = bnd[c], j1 = bnd[c + 1] < n_cases ? bnd[c + 1] : n_cases, s = c & 1, o = s ^ 1;
          n_last = c;
          int q = 0;
          t0 = wall_ms();
          run_jobs_io(jobs + j0, in + j0, out + j0, verbose, j1 - j0, 0, n_threads);
          prepared = j1;
          t_prep += wall_ms() - t0;
          for (i = j0; i < j1; ++i)
               if (jobs[i].rc) {
                    fprintf(stderr, "ERROR: lmie_solution_batch(): case %d\n", i);
                    rc = -1;
               }
          /* device batches of compatible cases of the chunk, in input order */
          for (i = j0; rc == 0 && i < j1; ++i) {
               int m = 0, base = np, off = 0;
               if (done[i])
                    continue;
               for (k = i; k < j1; ++k) {
                    if (done[k] || (k != i && !jobs_compatible(&jobs[i], &jobs[k])))
                         continue;
                    P[np] = jobs[k].P;
                    P[np].precision = precision;
                    R[np] = jobs[k].R;
                    pos2job[np] = k;
                    done[k] = 1;
                    ++np;
                    ++m;
                    if (jobs[i].P.save_control != 0)
                         break;
               }
               while (rc == 0 && off < m) {
                    const int f = lmieb_device_fit(m - off, P + base + off);
                    const long long t = lmieb_device_submit(f, P + base + off, R + base + off, first);
                    first = 0;
                    if (t < 0) {
                         fprintf(stderr, "ERROR: lmie_solution_batch(): device solve\n");
                         rc = -1;
                         break;
                    }
                    tk[s][q] = t;
                    tb[s][q] = base + off;
                    te[s][q] = base + off + f;
                    ++q;
                    off += f;
               }
          }
          ct[s].n = q;
          cj0[s] = j0;
          cj1[s] = j1;
          /* the previous chunk's results */
          if (ct[o].n && finish_chunk(&ct[o], jobs, cj0[o], cj1[o], pos2job, tb[o], te[o], R, n_threads,
                                      rc == 0, &t_fin))
               rc = -1;
          if (rc != 0)
               break;
     }
     for (c = 0; c < 2; ++c) {
          const int s = (n_last + c) & 1;   /* the last chunk, then any other left */
          if (ct[s].n && finish_chunk(&ct[s], jobs, cj0[s], cj1[s], pos2job, tb[s], te[s], R, n_threads,
                                      rc == 0, &t_fin))
               rc = -1;
     }
     lmieb_host_phase(0, t_prep);
     lmieb_host_phase(4, t_fin);
     if (rc != 0)      /* chunks given up before their finish (job_free is idempotent) */
          jobs_release(jobs, prepared);
     free(bnd);
     for (c = 0; c < 2; ++c) {
          free(tk[c]); free(tb[c]); free(te[c]);
     }
     free(jobs); free(P); free(R); free(done); free(pos2job);
     return rc;
}


/* ---- autotuner ------------------------------------------------------------ */

int lmie_solution_autotune(int n_cases, lmie_in_data *in, lmie_out_data *out, int n_threads, int precision,
                           int *best_chunks, double *best_items, double *best_ms) {
     static const int chunk_c[] = {1, 2, 3, 4, 6};
     static const double items_fp64[] = {32., 64., 128., 256.}, items_tc[] = {1., 2., 4.};
     const int tensor = precision == LMIEB_PRECISION_TF32X3 || precision == LMIEB_PRECISION_INT8;
     const double *items = tensor ? items_tc : items_fp64;
     const int n_items = tensor ? 3 : 4;
     const int keep = g_pipeline, keep_timing = lmieb_timing_state();
     const double keep_items = lmieb_get_work_granularity(precision);
     int a, b, r, bc = keep, rc = 0;
     double bi = keep_items, bd = -1., bt = -1.;
     if (n_cases < 1 || (precision != LMIEB_PRECISION_FP64 && precision != LMIEB_PRECISION_TF32X3 &&
                         precision != LMIEB_PRECISION_INT8)) {
          fprintf(stderr, "ERROR: lmie_solution_autotune(): invalid arguments\n");
          return -1;
     }
     /* 1. work granularity: it sets the device work and the host's packing
      *    of the work items (finer items, longer lists), so it is chosen by
      *    the kernels' device time (per-stage CUDA events, one sub-batch,
      *    undisturbed by the host's load) plus the packing time */
     g_pipeline = 1;
     lmieb_set_timing(1);
     for (b = 0; b < n_items && rc == 0; ++b) {
          double d = -1.;
          lmieb_set_work_granularity(precision, items[b]);
          for (r = 0; r < 3 && rc == 0; ++r) {
               double st[LMIEB_N_STAGES], dt = 0.;
               int s;
               double hm[LMIEB_N_HOST];
               rc = lmie_solution_batch2(n_cases, in, out, 0, 0, n_threads, precision);
               lmieb_last_timing(st, LMIEB_N_STAGES);
               for (s = 1; s < LMIEB_N_STAGES - 1; ++s)      /* kernels: stages between the copies */
                    dt += st[s];
               lmieb_last_host_timing(hm, LMIEB_N_HOST);
               dt += hm[1];                                   /* packing */
               if (r > 0 && (d < 0. || dt < d))
                    d = dt;
          }
          if (rc == 0 && (bd < 0. || d < bd)) {
               bd = d;
               bi = items[b];
          }
     }
     lmieb_set_timing(keep_timing);
     lmieb_set_work_granularity(precision, bi);
     /* 2. orders per block of the phase matrix at the user angles (its tile
      *    along the orders), by that stage's device time */
     {
          static const int part_c[] = {128, 256, 512};
          int bp = lmieb_get_user_angle_part();
          double bu = -1.;
          g_pipeline = 1;
          lmieb_set_timing(1);
          for (b = 0; b < 3 && rc == 0; ++b) {
               double d = -1.;
               lmieb_set_user_angle_part(part_c[b]);
               for (r = 0; r < 3 && rc == 0; ++r) {
                    double st[LMIEB_N_STAGES];
                    rc = lmie_solution_batch2(n_cases, in, out, 0, 0, n_threads, precision);
                    lmieb_last_timing(st, LMIEB_N_STAGES);
                    if (r > 0 && (d < 0. || st[7] < d))       /* stage 7: user angles */
                         d = st[7];
               }
               if (rc == 0 && (bu < 0. || d < bu)) {
                    bu = d;
                    bp = part_c[b];
               }
          }
          lmieb_set_timing(keep_timing);
          lmieb_set_user_angle_part(bp);
     }
     /* 3. pipeline depth: the overlap of host work with the device, by the
      *    wall time of the public batch call (one call to settle the buffers,
      *    then the faster of two) */
     for (a = 0; a < 5 && rc == 0; ++a) {
          double t = -1.;
          if (chunk_c[a] > 1 && n_cases < 2 * chunk_c[a])
               continue;
          g_pipeline = chunk_c[a];
          for (r = 0; r < 3 && rc == 0; ++r) {
               const double t0 = wall_ms();
               rc = lmie_solution_batch2(n_cases, in, out, 0, 0, n_threads, precision);
               const double dt = wall_ms() - t0;
               if (r > 0 && (t < 0. || dt < t))
                    t = dt;
          }
          if (rc == 0 && (bt < 0. || t < bt)) {
               bt = t;
               bc = chunk_c[a];
          }
     }
     g_pipeline = rc == 0 ? bc : keep;
     lmieb_set_work_granularity(precision, rc == 0 ? bi : keep_items);
     if (best_chunks)
          *best_chunks = g_pipeline;
     if (best_items)
          *best_items = lmieb_get_work_granularity(precision);
     if (best_ms)
          *best_ms = bt;
     return rc;
}
