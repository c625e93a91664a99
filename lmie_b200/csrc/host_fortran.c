/*
 * host_fortran.c -- the `_`-suffixed entry points the reference's Fortran 77
 * and Fortran 90 wrappers call (reference interfaces/lmie_int_util.c:21-241;
 * interfaces/lmie_int_f77.f and lmie_int_f90.f90 call these unchanged).
 *
 * All arguments arrive by reference.  Fortran arrays are column-major, so
 * gc(max_coef,6) is C gc[6][max_coef], gc_l(max_coef,6,n_derivs) is
 * gc_l[n_derivs][6][max_coef] and pf(n_angles,6) is pf[6][n_angles]; the shim
 * builds row-pointer views over the caller's memory and calls
 * lmie_solution2_l.
 *
 * Deviation: the reference's lmie_solution2_ passes a null pointer for
 * n_derivs to lmie_solution2_l_, which then dereferences it
 * (interfaces/lmie_int_util.c:109-113,176); here it passes a pointer to 0.
 */
#include <stdio.h>
#include <stdlib.h>

#include "host.h"

static double **view2(double *mem, size_t m, size_t n) {
     size_t i;
     double **p = (double **) malloc(sizeof(double *) * (m ? m : 1));
     for (i = 0; i < m; ++i)
          p[i] = mem + i * n;
     return p;
}

static double ***view3(double *mem, size_t a, size_t b, size_t c) {
     size_t i;
     size_t na = a > 0 ? a : 1, nab = a * b > 0 ? a * b : 1;
     double ***p = (double ***) malloc(sizeof(double **) * na + sizeof(double *) * nab);
     double **q = (double **) (p + na);
     for (i = 0; i < a; ++i)
          p[i] = q + i * b;
     for (i = 0; i < a * b; ++i)
          q[i] = mem + i * c;
     return p;
}

int size_dist_code_(char *name) {
     return (int) size_dist_code(name);
}

int lmie_calc_max_coef_(double *lambda, enum size_dist_type *dist_type,
                        double *a1, double *a2, double *a3, double *r1, double *r2) {
     return lmie_calc_max_coef(*lambda, *dist_type, *a1, *a2, *a3, *r1, *r2);
}

int lmie_solution2_l_(int *calc_gc, int *calc_lc, int *calc_pf,
                      enum size_dist_type *dist_type,
                      int *n_int1, int *n_int2, int *n_quad,
                      int *n_angles, int *n_derivs, int *save_control,
                      double *lambda, double *mr, double *mi,
                      double *a1, double *a2, double *a3, double *a4, double *a5,
                      double *r1, double *r2,
                      double *lambda_l, double *mr_l, double *mi_l,
                      double *a1_l, double *a2_l, double *a3_l, double *a4_l, double *a5_l,
                      double *r1_l, double *r2_l,
                      double *accuracy, int *n_coef,
                      double *r21, double *r22,
                      double *norm, double *reff, double *veff,
                      double *gavg, double *vavg, double *ravg, double *rvw,
                      double *cext, double *csca, double *cbak, double *g,
                      double *gc, double *lc, double *theta, double *pf,
                      double *r21_l, double *r22_l,
                      double *norm_l, double *reff_l, double *veff_l,
                      double *gavg_l, double *vavg_l, double *ravg_l, double *rvw_l,
                      double *cext_l, double *csca_l, double *cbak_l, double *g_l,
                      double *gc_l, double *lc_l, double *pf_l,
                      double ***save1, double ****save2,
                      int *max_coef, int *verbose, int *n_threads, int *use_mpi) {
     int nd = n_derivs ? *n_derivs : 0, rc;
     double **gc2 = NULL, **lc2 = NULL, **pf2 = NULL;
     double ***gc_l2 = NULL, ***lc_l2 = NULL, ***pf_l2 = NULL;

     if (*calc_gc) {
          gc2 = view2(gc, 6, *max_coef);
          if (nd > 0)
               gc_l2 = view3(gc_l, nd, 6, *max_coef);
     }
     if (*calc_lc) {
          lc2 = view2(lc, 6, *max_coef);
          if (nd > 0)
               lc_l2 = view3(lc_l, nd, 6, *max_coef);
     }
     if (*calc_pf) {
          pf2 = view2(pf, 6, *n_angles);
          if (nd > 0)
               pf_l2 = view3(pf_l, nd, 6, *n_angles);
     }

     rc = lmie_solution2_l(*calc_gc, *calc_lc, *calc_pf, *dist_type, *n_int1, *n_int2, *n_quad,
                           *n_angles, nd, *save_control, *lambda, *mr, *mi,
                           *a1, *a2, *a3, *a4, *a5, *r1, *r2,
                           lambda_l, mr_l, mi_l, a1_l, a2_l, a3_l, a4_l, a5_l, r1_l, r2_l,
                           *accuracy, n_coef, r21, r22, norm, reff, veff, gavg, vavg, ravg, rvw,
                           cext, csca, cbak, g, gc2, lc2, theta, pf2,
                           r21_l, r22_l, norm_l, reff_l, veff_l, gavg_l, vavg_l, ravg_l, rvw_l,
                           cext_l, csca_l, cbak_l, g_l, gc_l2, lc_l2, pf_l2,
                           save1, save2, *verbose, *n_threads, *use_mpi);

     free(gc2); free(gc_l2);
     free(lc2); free(lc_l2);
     free(pf2); free(pf_l2);

     if (rc) {
          fprintf(stderr, "ERROR: lmie_solution2_l()\n");
          return -1;
     }
     return 0;
}

int lmie_solution2_(int *calc_gc, int *calc_lc, int *calc_pf,
                    enum size_dist_type *dist_type,
                    int *n_int1, int *n_int2,
                    int *n_quad, int *n_angles, int *save_control,
                    double *lambda, double *mr, double *mi,
                    double *a1, double *a2, double *a3, double *a4, double *a5,
                    double *r1, double *r2,
                    double *accuracy, int *n_coef,
                    double *r21, double *r22,
                    double *norm, double *reff, double *veff,
                    double *gavg, double *vavg, double *ravg, double *rvw,
                    double *cext, double *csca, double *cbak, double *g,
                    double *gc, double *lc, double *theta, double *pf,
                    double ***save1, double ****save2,
                    int *max_coef, int *verbose, int *n_threads, int *use_mpi) {
     int zero = 0;
     return lmie_solution2_l_(calc_gc, calc_lc, calc_pf, dist_type, n_int1, n_int2, n_quad,
                              n_angles, &zero, save_control, lambda, mr, mi,
                              a1, a2, a3, a4, a5, r1, r2,
                              NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL,
                              accuracy, n_coef, r21, r22, norm, reff, veff, gavg, vavg, ravg, rvw,
                              cext, csca, cbak, g, gc, lc, theta, pf,
                              NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL,
                              NULL, NULL, NULL, NULL, NULL, NULL, NULL,
                              save1, save2, max_coef, verbose, n_threads, use_mpi);
}
