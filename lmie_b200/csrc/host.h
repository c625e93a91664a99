/*
 * host.h -- internal declarations of the C host layer of liblmie_b200.
 */
#ifndef LMIEB_HOST_H
#define LMIEB_HOST_H

#include "../../include/lmie_interface.h"
#include "../../include/lmie_b200.h"
#include "lmieb.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
     int dist_type, n_int1, n_int2, n_quad, nd;
     double a1, a2, a3, a4, a5, r1, r2;
     const double *a1_l, *a2_l, *a3_l, *a4_l, *a5_l, *r1_l, *r2_l;   /* [nd] */
} lmieb_dist_in;

typedef struct {
     double *qx, *qw, *nr;           /* [n] */
     double *qx_l, *qw_l, *nr_l;     /* [n*nd], radius-major */
     double r1, r2, norm;
     double *r1_l, *r2_l, *norm_l;   /* [nd] */
} lmieb_dist_out;

typedef struct {
     double reff, veff, gavg, vavg, ravg, rvw;
     double *reff_l, *veff_l, *gavg_l, *vavg_l, *ravg_l, *rvw_l;   /* [nd] */
} lmieb_moments_out;

int lmieb_dist_count(int dist_type, int n_int1, int n_int2, int n_quad);
void lmieb_power_law_range(double a1, double a2, double *r1, double *r2);
void lmieb_gauss_leg(int n, double x1, double x2, double *x, double *w);
int lmieb_particle_dist(const lmieb_dist_in *in, lmieb_dist_out *out);
void lmieb_moments(int n, int nd, const double *qx, const double *qw, const double *nr,
                   const double *qx_l, const double *qw_l, const double *nr_l,
                   lmieb_moments_out *m);

/* truncation integers (reference src/lmie_core.c:18-38) */
int lmieb_calc_n1(double x);
int lmieb_calc_n2(int n1, double zr, double zi);

/* row-pointer arrays in the reference's single-block layout */
double *lmieb_arr1(size_t n);
double **lmieb_arr2(size_t m, size_t n);
double ***lmieb_arr3(size_t a, size_t b, size_t c);

#ifdef __cplusplus
}
#endif

#endif
