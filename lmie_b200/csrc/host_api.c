/*
 * host_api.c -- the drop-in C interface of liblmie_b200 (include/lmie_interface.h).
 *
 * Same entry points, argument meaning, output layout and error behaviour as
 * the reference's src/lmie_interface.c; the Mie work itself is done on the
 * GPU by lmieb_device_solve (driver.cu).  There is no CPU fallback: without a
 * usable GPU every solve returns -1 with an ERROR line.
 */
#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

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

int lmie_solution_slave(void) {
     fprintf(stderr, "ERROR: lmie_solution_slave(): this library is built without MPI; "
             "distribute cases over GPUs with lmie_solution_batch instead\n");
     return -1;
}

/* Scratch owned by one lmie_solution2_l call. */
typedef struct {
     double *qx, *qw, *nr, *qx_l, *qw_l, *nr_l;
     double *x, *xl, *w, *w2, *mu_user, *sv1, *sv2;
     int *n1r, *n2r, *idx1, *idx2;
     double *dev_out;
} call_scratch;

static void scratch_free(call_scratch *s) {
     free(s->qx); free(s->qw); free(s->nr); free(s->qx_l); free(s->qw_l); free(s->nr_l);
     free(s->x); free(s->xl); free(s->w); free(s->w2); free(s->mu_user);
     free(s->n1r); free(s->n2r); free(s->idx1); free(s->idx2); free(s->dev_out);
     free(s->sv1); free(s->sv2);
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
     int n, nd = n_derivs > 0 ? n_derivs : 0, nd1 = 0, nd2 = 0, i, k, e;
     int n1, n_qang, n_coef_all, ncol;
     double x2;
     double complex m, z2;
     call_scratch s;
     lmieb_dist_in din;
     lmieb_dist_out dout;
     lmieb_moments_out mom;
     lmieb_problem P;
     lmieb_result R;
     double *scal, *dgc, *dlc, *dpf;
     size_t n_out;
     (void) n_threads;
     (void) use_mpi;

     memset(&s, 0, sizeof(s));

     /* input check (reference src/lmie_interface.c:404-408) */
     if (calc_pf && (!calc_gc && !calc_lc)) {
          fprintf(stderr, "ERROR: either calc_gc or calc_lc must be set to true when "
                  "calc_pf is true\n");
          return -1;
     }
     if (save_control < 0 || save_control > 2) {
          fprintf(stderr, "ERROR: invalid save_control: %d\n", save_control);
          return -1;
     }
     if (calc_pf && n_angles < 1) {
          fprintf(stderr, "ERROR: n_angles must be >= 1 when calc_pf is true\n");
          return -1;
     }

     n = lmieb_dist_count(dist_type, n_int1, n_int2, n_quad);
     if (n <= 0) {
          if (n == 0)
               fprintf(stderr, "ERROR: size distribution has no quadrature points\n");
          return -1;
     }

     /* ---- size distribution quadrature and moments ---- */
     s.qx = lmieb_arr1(n);
     s.qw = lmieb_arr1(n);
     s.nr = lmieb_arr1(n);
     s.qx_l = lmieb_arr1((size_t) n * nd);
     s.qw_l = lmieb_arr1((size_t) n * nd);
     s.nr_l = lmieb_arr1((size_t) n * nd);
     memset(&din, 0, sizeof(din));
     din.dist_type = dist_type; din.n_int1 = n_int1; din.n_int2 = n_int2; din.n_quad = n_quad;
     din.nd = nd;
     din.a1 = a1; din.a2 = a2; din.a3 = a3; din.a4 = a4; din.a5 = a5; din.r1 = r1; din.r2 = r2;
     din.a1_l = a1_l; din.a2_l = a2_l; din.a3_l = a3_l; din.a4_l = a4_l; din.a5_l = a5_l;
     din.r1_l = r1_l; din.r2_l = r2_l;
     dout.qx = s.qx; dout.qw = s.qw; dout.nr = s.nr;
     dout.qx_l = s.qx_l; dout.qw_l = s.qw_l; dout.nr_l = s.nr_l;
     dout.r1_l = r21_l; dout.r2_l = r22_l; dout.norm_l = norm_l;
     if (lmieb_particle_dist(&din, &dout) < 0) {
          fprintf(stderr, "ERROR: get_particle_dist()\n");
          scratch_free(&s);
          return -1;
     }
     *r21 = dout.r1;
     *r22 = dout.r2;
     *norm = dout.norm;
     mom.reff_l = reff_l; mom.veff_l = veff_l; mom.gavg_l = gavg_l;
     mom.vavg_l = vavg_l; mom.ravg_l = ravg_l; mom.rvw_l = rvw_l;
     lmieb_moments(n, nd, s.qx, s.qw, s.nr, s.qx_l, s.qw_l, s.nr_l, &mom);
     *reff = mom.reff; *veff = mom.veff; *gavg = mom.gavg;
     *vavg = mom.vavg; *ravg = mom.ravg; *rvw = mom.rvw;

     /* ---- derivative split (reference src/lmie_interface.c:304-353) ---- */
     s.idx1 = (int *) calloc(nd > 0 ? nd : 1, sizeof(int));
     s.idx2 = (int *) calloc(nd > 0 ? nd : 1, sizeof(int));
     for (i = 0; i < nd; ++i) {
          if (lambda_l[i] != 0. || mr_l[i] != 0. || mi_l[i] != 0. ||
              r21_l[i] != 0. || r22_l[i] != 0.)
               s.idx1[nd1++] = i;
          else
               s.idx2[nd2++] = i;
     }

     /* ---- global truncation (reference src/lmie_schedule.c:1004-1017) ---- */
     m = mr - I * mi;
     x2 = 2. * M_PI * *r22 / lambda;
     z2 = m * x2;
     n1 = lmieb_calc_n1(x2);
     (void) z2;
     n_qang = (!gc && !lc) ? 0 : 2 * n1;
     n_coef_all = 2 * n1;

     /* ---- per-radius size parameters, truncation and weights
      *      (reference src/lmie_core.c:263-292) ---- */
     s.x = lmieb_arr1(n);
     s.xl = lmieb_arr1((size_t) n * (nd1 > 0 ? nd1 : 1));
     s.w = lmieb_arr1((size_t) n * (1 + nd));
     s.n1r = (int *) calloc(n, sizeof(int));
     s.n2r = (int *) calloc(n, sizeof(int));
     for (i = 0; i < n; ++i) {
          double x = 2. * M_PI * s.qx[i] / lambda;
          double complex z = m * x;
          s.x[i] = x;
          s.n1r[i] = lmieb_calc_n1(x);
          s.n2r[i] = lmieb_calc_n2(s.n1r[i], creal(z), cimag(z));
          s.w[i] = s.nr[i] * s.qw[i];
          for (k = 0; k < nd1; ++k) {
               int kk = s.idx1[k];
               s.xl[(size_t) k * n + i] = 2. * M_PI * (s.qx_l[(size_t) i * nd + kk] -
                                        s.qx[i] * lambda_l[kk] / lambda) / lambda;
               s.w[(size_t) (1 + kk) * n + i] = s.nr_l[(size_t) i * nd + kk] * s.qw[i] +
                                                s.nr[i] * s.qw_l[(size_t) i * nd + kk];
          }
          for (k = 0; k < nd2; ++k) {
               int kk = s.idx2[k];
               s.w[(size_t) (1 + kk) * n + i] = s.nr_l[(size_t) i * nd + kk] * s.qw[i];
          }
     }
     if (n1 < 1 || s.n1r[n - 1] < 1) {
          fprintf(stderr, "ERROR: invalid size parameter (lambda = %g, r2 = %g)\n", lambda, *r22);
          scratch_free(&s);
          return -1;
     }
     for (i = 0; i < n; ++i) {
          if (s.n1r[i] > n1) {
               fprintf(stderr, "ERROR: radius %d (r = %g) lies above r2 = %g\n", i, s.qx[i], *r22);
               scratch_free(&s);
               return -1;
          }
     }

     /* ---- save_control: allocate / gather the per-radius kernels ---- */
     if (save_control == 1) {
          *save1 = lmieb_arr2(4, n);
          *save2 = lmieb_arr3(4, n, n_qang > 0 ? n_qang : 1);
     }
     if (save_control == 2) {
          s.w2 = lmieb_arr1((size_t) n * (nd > 0 ? nd : 1));
          for (i = 0; i < n; ++i)
               for (k = 0; k < nd2; ++k) {
                    int kk = s.idx2[k];
                    s.w2[(size_t) kk * n + i] = s.nr_l[(size_t) i * nd + kk] * s.qw[i] +
                                                s.nr[i] * s.qw_l[(size_t) i * nd + kk];
               }
     }

     /* ---- user angles (reference misc/rtutil_scat_int.c:487-503,580) ---- */
     if (calc_pf) {
          double d = 180. / (n_angles - 1);
          s.mu_user = lmieb_arr1(n_angles);
          for (i = 0; i < n_angles; ++i) {
               theta[i] = i * d;
               s.mu_user[i] = cos(theta[i] * (M_PI / 180.0));
          }
     }

     /* ---- device solve ---- */
     memset(&P, 0, sizeof(P));
     P.n = n; P.nd = nd; P.nd1 = nd1; P.nd2 = nd2; P.idx1 = s.idx1; P.idx2 = s.idx2;
     P.lambda = lambda; P.mr = mr; P.mi = mi;
     P.lambda_l = lambda_l; P.mr_l = mr_l; P.mi_l = mi_l;
     P.x = s.x; P.xl = s.xl; P.w = s.w; P.n1r = s.n1r; P.n2r = s.n2r;
     P.n1 = n1; P.n_qang = n_qang; P.n_coef = n_coef_all;
     P.want_gc = gc != NULL; P.want_lc = lc != NULL;
     P.pf_from = calc_pf ? (calc_gc ? 1 : 2) : 0;
     P.n_angles = calc_pf ? n_angles : 0;
     P.mu_user = s.mu_user;
     P.accuracy = accuracy;
     P.save_control = save_control;
     if (save_control == 2) {
          /* gather the caller's kernels through their row pointers */
          int q, r;
          if (!save1 || !*save1 || (n_qang > 0 && (!save2 || !*save2))) {
               fprintf(stderr, "ERROR: save_control = 2 needs save1 and save2 from a "
                       "save_control = 1 call\n");
               scratch_free(&s);
               return -1;
          }
          s.sv1 = lmieb_arr1((size_t) 4 * n);
          s.sv2 = lmieb_arr1((size_t) 4 * n * (n_qang > 0 ? n_qang : 1));
          for (q = 0; q < 4; ++q) {
               memcpy(s.sv1 + (size_t) q * n, (*save1)[q], sizeof(double) * n);
               if (n_qang > 0)
                    for (r = 0; r < n; ++r)
                         memcpy(s.sv2 + ((size_t) q * n + r) * n_qang, (*save2)[q][r],
                                sizeof(double) * n_qang);
          }
          P.save1_in = s.sv1;
          P.save2_in = s.sv2;
          P.w2 = s.w2;
     }

     ncol = 1 + nd;
     n_out = (size_t) ncol * 4 + (P.want_gc ? (size_t) ncol * 6 * n_coef_all : 0) +
             (P.want_lc ? (size_t) ncol * 6 * n_coef_all : 0) +
             (size_t) ncol * 6 * P.n_angles;
     s.dev_out = lmieb_arr1(n_out);
     scal = s.dev_out;
     dgc = scal + ncol * 4;
     dlc = dgc + (P.want_gc ? (size_t) ncol * 6 * n_coef_all : 0);
     dpf = dlc + (P.want_lc ? (size_t) ncol * 6 * n_coef_all : 0);
     memset(&R, 0, sizeof(R));
     R.scal = scal;
     R.gc = P.want_gc ? dgc : NULL;
     R.lc = P.want_lc ? dlc : NULL;
     R.pf = P.n_angles > 0 ? dpf : NULL;
     if (save_control == 1) {
          R.save1 = (*save1)[0];
          R.save2 = (*save2)[0][0];
     }
     if (verbose)
          fprintf(stderr, "lmie_b200: n_radii = %d, n1 = %d, n_qang = %d, n_derivs = %d (%d Mie, %d shape)\n",
                  n, n1, n_qang, nd, nd1, nd2);
     if (lmieb_device_solve(&P, &R)) {
          fprintf(stderr, "ERROR: lmie_core_solution()\n");
          scratch_free(&s);
          return -1;
     }

     /* ---- scatter into the caller's arrays ---- */
     *cext = scal[0];
     *csca = scal[1];
     *cbak = scal[2];
     *g = scal[3];
     for (k = 0; k < nd; ++k) {
          cext_l[k] = scal[(1 + k) * 4 + 0];
          csca_l[k] = scal[(1 + k) * 4 + 1];
          cbak_l[k] = scal[(1 + k) * 4 + 2];
          g_l[k] = scal[(1 + k) * 4 + 3];
     }
     if (gc) {
          for (e = 0; e < 6; ++e)
               memcpy(gc[e], dgc + (size_t) e * n_coef_all, sizeof(double) * n_coef_all);
          for (k = 0; k < nd; ++k)
               for (e = 0; e < 6; ++e)
                    memcpy(gc_l[k][e], dgc + ((size_t) (1 + k) * 6 + e) * n_coef_all,
                           sizeof(double) * n_coef_all);
     }
     if (lc) {
          for (e = 0; e < 6; ++e)
               memcpy(lc[e], dlc + (size_t) e * n_coef_all, sizeof(double) * n_coef_all);
          for (k = 0; k < nd; ++k)
               for (e = 0; e < 6; ++e)
                    memcpy(lc_l[k][e], dlc + ((size_t) (1 + k) * 6 + e) * n_coef_all,
                           sizeof(double) * n_coef_all);
     }
     if (calc_pf) {
          for (e = 0; e < 6; ++e)
               memcpy(pf[e], dpf + (size_t) e * n_angles, sizeof(double) * n_angles);
          for (k = 0; k < nd; ++k)
               for (e = 0; e < 6; ++e)
                    memcpy(pf_l[k][e], dpf + ((size_t) (1 + k) * 6 + e) * n_angles,
                           sizeof(double) * n_angles);
     }
     *n_coef = R.n_coef_out;

     scratch_free(&s);
     return 0;
}
