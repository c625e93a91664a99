/*
 * lmie_oracle.c -- CPU FP64 restatement of LMie's polydisperse Mie solve.
 *
 * TEST INFRASTRUCTURE ONLY (see lmie_oracle.h).  Single-threaded, plain C99,
 * written for readability rather than speed.  Each function names the
 * reference file:line whose algorithm it restates; the arithmetic follows the
 * reference's operation order so the two agree to a few ulps.
 */
#include <complex.h>
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "lmie_oracle.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef double complex cplx;

/* ------------------------------------------------------------------------ */
/* Row-pointer arrays: pointer table followed by contiguous data in one block
 * (reference misc/gutil_alloc.c:18-70,214-226).                            */
/* ------------------------------------------------------------------------ */
static double *arr1(size_t n) {
     return (double *) calloc(n ? n : 1, sizeof(double));
}

static double **arr2(size_t m, size_t n) {
     size_t i;
     double **p = (double **) calloc(1, m * sizeof(double *) + m * n * sizeof(double) + 8);
     double *d = (double *) (p + m);
     for (i = 0; i < m; ++i)
          p[i] = d + i * n;
     return p;
}

static double ***arr3(size_t a, size_t b, size_t c) {
     size_t i, j;
     double ***p = (double ***) calloc(1, a * sizeof(double **) + a * b * sizeof(double *) +
                                          a * b * c * sizeof(double) + 8);
     double **q = (double **) (p + a);
     double *d = (double *) (q + a * b);
     for (i = 0; i < a; ++i) {
          p[i] = q + i * b;
          for (j = 0; j < b; ++j)
               q[i * b + j] = d + (i * b + j) * c;
     }
     return p;
}

/* ------------------------------------------------------------------------ */
/* Truncation integers (reference src/lmie_core.c:18-38, Mishchenko 2002).  */
/* ------------------------------------------------------------------------ */
int oracle_calc_n1(double x) {
     return (int) (x + 4.05 * pow(x, 1. / 3.) + 8);
}

int oracle_calc_n2(int n1, double zr, double zi) {
     double az = cabs(zr + I * zi);
     double t = n1 > az ? n1 : az;
     return (int) (t + 6.40 * pow(t, 1. / 3.) + 8);
}

/* ------------------------------------------------------------------------ */
/* Brent/Dekker root finder on [ax,bx] (Forsythe, Malcolm & Moler 1977,
 * "zeroin"), used for the power-law radius range (reference misc/zeroin.c,
 * called from misc/rtutil_size_dist.c:106-121).                            */
/* ------------------------------------------------------------------------ */
static double brent_root(double ax, double bx, double (*f)(double, const double *),
                         const double *data, double tol) {
     double a = ax, b = bx, c, fa = f(a, data), fb = f(b, data), fc;
     c = a; fc = fa;
     for (;;) {
          double prev = b - a, tol_act, p, q, step;
          if (fabs(fc) < fabs(fb)) {
               a = b; b = c; c = a;
               fa = fb; fb = fc; fc = fa;
          }
          tol_act = 2 * DBL_EPSILON * fabs(b) + tol / 2;
          step = (c - b) / 2;
          if (fabs(step) <= tol_act || fb == 0.)
               return b;
          if (fabs(prev) >= tol_act && fabs(fa) > fabs(fb)) {
               double t1, cb = c - b, t2;
               if (a == c) {
                    t1 = fb / fa;
                    p = cb * t1;
                    q = 1.0 - t1;
               } else {
                    q = fa / fc; t1 = fb / fc; t2 = fb / fa;
                    p = t2 * (cb * q * (q - t1) - (b - a) * (t1 - 1.0));
                    q = (q - 1.0) * (t1 - 1.0) * (t2 - 1.0);
               }
               if (p > 0) q = -q; else p = -p;
               if (p < (0.75 * cb * q - fabs(tol_act * q) / 2) && p < fabs(prev * q / 2))
                    step = p / q;
          }
          if (fabs(step) < tol_act)
               step = step > 0 ? tol_act : -tol_act;
          a = b; fa = fb;
          b += step; fb = f(b, data);
          if ((fb > 0 && fc > 0) || (fb < 0 && fc < 0)) {
               c = a; fc = fa;
          }
     }
}

/* Power law with effective radius a1 and variance a2: r2 = 2 a1 (1+a2) - r1
 * and (r2-r1)/ln(r2/r1) = a1 (reference misc/rtutil_size_dist.c:95-121). */
static double power_law_f(double r1, const double *d) {
     double r2 = (1. + d[1]) * 2. * d[0] - r1;
     return (r2 - r1) / log(r2 / r1) - d[0];
}

static void power_law_range(double a1, double a2, double *r1, double *r2) {
     double d[2] = {a1, a2};
     *r1 = brent_root(DBL_EPSILON, a1, power_law_f, d, 0.);
     *r2 = (1. + a2) * 2. * a1 - *r1;
}

/* ------------------------------------------------------------------------ */
/* Gauss-Legendre (Davis & Rabinowitz 1975): Newton with a second-order
 * correction on P_n, initial guess cos(t + da/tan t)
 * (reference misc/rtutil_math.c:73-129).                                   */
/* ------------------------------------------------------------------------ */
static void gl_node(int n, int i, int ia, int ib, double da, double *y_out, double *pn1_out) {
     double t = (4. * i + 3.) / ia * M_PI;
     double y = cos(t + da / tan(t)), y_old, pn = 1., pm = 0., pmm, s, dp, ddp;
     int j;
     do {
          pm = 0.;
          pn = 1.;
          for (j = 0; j < n; ++j) {
               pmm = pm;
               pm = pn;
               s = y * pm;
               pn = j / (j + 1.) * (s - pmm) + s;
          }
          s = 1. - y * y;
          dp = n * (pm - y * pn) / s;
          ddp = (2. * y * dp - ib * pn) / s;
          y_old = y;
          s = pn / dp;
          y = y_old - s * (1. + s * ddp / (2. * dp));
     } while (fabs(y - y_old) > DBL_EPSILON);
     *y_out = y;
     *pn1_out = pm;
}

/* Nodes ascending on [x1,x2] with endpoint derivatives
 * (reference misc/rtutil_math.c:231-316). */
static void gl_quad_l(int n, int nd, double x1, double x2, const double *x1_l, const double *x2_l,
                      double *x, double *w, double *x_l, double *w_l) {
     int i, k, ii = n - 1, half = (n + 1) / 2;
     int ia = 4 * n + 2, ib = n * (n + 1);
     double da = (n - 1) / (8. * pow((double) n, 3));
     double mid = (x1 + x2) / 2., hw = (x2 - x1) / 2.;
     for (i = 0; i < half; ++i, --ii) {
          double y, pn1, dd, de;
          gl_node(n, i, ia, ib, da, &y, &pn1);
          dd = hw * y;
          x[i] = mid - dd;
          x[ii] = mid + dd;
          de = n * pn1;
          de = 2. / (de * de);
          w[i] = (hw - dd * y) * de;
          w[ii] = w[i];
          for (k = 0; k < nd; ++k) {
               double mid_l = (x1_l[k] + x2_l[k]) / 2., hw_l = (x2_l[k] - x1_l[k]) / 2.;
               double dd_l = hw_l * y;
               x_l[i * nd + k] = mid_l - dd_l;
               x_l[ii * nd + k] = mid_l + dd_l;
               w_l[i * nd + k] = (hw_l - dd_l * y) * de;
               w_l[ii * nd + k] = w_l[i * nd + k];
          }
     }
}

void oracle_gauss_leg(int n, double x1, double x2, double *x, double *w) {
     gl_quad_l(n, 0, x1, x2, NULL, NULL, x, w, NULL, NULL);
}

/* n_int equal sub-intervals of [r1,r2], n_quad GL points each, with
 * derivatives of nodes/weights w.r.t. r1, r2
 * (reference misc/rtutil_size_dist.c:128-193, misc/rtutil_math.c:329-387). */
static void dist_quad(int n_int, int n_quad, int nd, double r1, double r2,
                      const double *r1_l, const double *r2_l,
                      double *qx, double *qw, double *qx_l, double *qw_l) {
     int i, j, k, ii, half = (n_quad + 1) / 2;
     double *tx = arr1(n_quad), *tw = arr1(n_quad);
     double a = (r2 - r1) / n_int;
     double *zero = arr1(nd ? nd : 1);
     gl_quad_l(n_quad, 0, -1., 1., NULL, NULL, tx, tw, NULL, NULL);
     for (i = 0; i < n_int; ++i) {
          int off = i * n_quad;
          double b = r1 + i * a;
          double mid = (b + (b + a)) / 2., hw = ((b + a) - b) / 2.;
          for (j = 0, ii = n_quad - 1; j < half; ++j, --ii) {
               double dd = hw * tx[ii];
               qx[off + j] = mid - dd;
               qx[off + ii] = mid + dd;
               qw[off + j] = tw[j] * hw;
               qw[off + ii] = qw[off + j];
               for (k = 0; k < nd; ++k) {
                    double a_l = (r2_l[k] - (r1_l ? r1_l[k] : 0.)) / n_int;
                    double b_l = (r1_l ? r1_l[k] : 0.) + i * a_l;
                    double c_l = b_l + a_l;
                    double mid_l = (b_l + c_l) / 2., hw_l = (c_l - b_l) / 2.;
                    double dd_l = hw_l * tx[ii];
                    qx_l[(off + j) * nd + k] = mid_l - dd_l;
                    qx_l[(off + ii) * nd + k] = mid_l + dd_l;
                    qw_l[(off + j) * nd + k] = 0. * hw + tw[j] * hw_l;
                    qw_l[(off + ii) * nd + k] = qw_l[(off + j) * nd + k];
               }
          }
     }
     free(tx); free(tw); free(zero);
}

/* ------------------------------------------------------------------------ */
/* Size distributions and their derivatives
 * (reference misc/rtutil_size_dist.c:20-49,200-646).                       */
/* ------------------------------------------------------------------------ */
static int dist_count(const lmie_in_data *in) {
     switch (in->dist_type) {
     case SIZE_DIST_MONO: return 1;
     case SIZE_DIST_MODIFIED_POWER_LAW: return in->n_int1 * in->n_quad + in->n_int2 * in->n_quad;
     case SIZE_DIST_MODIFIED_GAMMA: case SIZE_DIST_LOG_NORMAL: case SIZE_DIST_POWER_LAW:
     case SIZE_DIST_GAMMA: case SIZE_DIST_MODIFIED_BIMODAL_LOG_NORMAL: case SIZE_DIST_EXPONENTIAL:
          return in->n_int2 * in->n_quad;
     default:
          fprintf(stderr, "ERROR: Invalid distribution type: %d\n", in->dist_type);
          return -1;
     }
}

#define D(p, k) ((p) ? (p)[k] : 0.)

int oracle_particle_dist(const lmie_in_data *in,
                         double *qx, double *qw, double *nr,
                         double *qx_l, double *qw_l, double *nr_l,
                         double *r1o, double *r2o, double *r1o_l, double *r2o_l,
                         double *norm, double *norm_l) {
     int n = dist_count(in), nd = in->n_derivs, i, k;
     double a1 = in->a1, a2 = in->a2, a3 = in->a3, a4 = in->a4, a5 = in->a5;
     double sum = 0.;
     double *sum_l;
     if (n < 0)
          return -1;
     sum_l = arr1(nd);

     switch (in->dist_type) {
     case SIZE_DIST_MONO:
          *r1o = a1; *r2o = a1;
          for (k = 0; k < nd; ++k) { r1o_l[k] = 0.; r2o_l[k] = 0.; }
          qx[0] = a1; qw[0] = 1.; nr[0] = 1.;
          for (k = 0; k < nd; ++k) { qx_l[k] = in->a1_l[k]; qw_l[k] = 0.; nr_l[k] = 0.; }
          sum = 1.;
          break;

     case SIZE_DIST_MODIFIED_GAMMA: {
          /* n(r) = r^a1 exp(-a1/(a3 rc^a3) r^a3), rc = a2 */
          double b = pow(a2, a3), c = a3 * b, d = b / c, e = a3 / a2, f = log(a2), g = a1 / c;
          double *c_l = arr1(nd);
          *r1o = in->r1; *r2o = in->r2;
          for (k = 0; k < nd; ++k) { r1o_l[k] = in->r1_l[k]; r2o_l[k] = in->r2_l[k]; }
          dist_quad(in->n_int2, in->n_quad, nd, *r1o, *r2o, r1o_l, r2o_l, qx, qw, qx_l, qw_l);
          for (k = 0; k < nd; ++k)
               c_l[k] = in->a3_l[k] * d + (in->a2_l[k] * e + in->a3_l[k] * f);
          for (i = 0; i < n; ++i) {
               double h = pow(qx[i], a3), o = 0.;
               nr[i] = pow(qx[i], a1) * exp(-g * h);
               sum += nr[i] * qw[i];
               if (nd > 0)
                    o = log(qx[i]);
               for (k = 0; k < nd; ++k) {
                    double p = qx_l[i * nd + k] / qx[i];
                    nr_l[i * nd + k] = nr[i] * ((p * a1 + in->a1_l[k] * o) + h * ((-in->a1_l[k] +
                                       a1 * (-(p * a3 + in->a3_l[k] * o) + c_l[k])) / c));
                    sum_l[k] += nr_l[i * nd + k] * qw[i] + nr[i] * qw_l[i * nd + k];
               }
          }
          free(c_l);
          break;
     }

     case SIZE_DIST_LOG_NORMAL: {
          double b = log(a1), c = 2. * a2;
          *r1o = in->r1; *r2o = in->r2;
          for (k = 0; k < nd; ++k) { r1o_l[k] = in->r1_l[k]; r2o_l[k] = in->r2_l[k]; }
          dist_quad(in->n_int2, in->n_quad, nd, *r1o, *r2o, r1o_l, r2o_l, qx, qw, qx_l, qw_l);
          for (i = 0; i < n; ++i) {
               double d = log(qx[i]) - b, e = d * d / c;
               nr[i] = exp(-e) / qx[i];
               sum += nr[i] * qw[i];
               for (k = 0; k < nd; ++k) {
                    double f = qx_l[i * nd + k] / qx[i];
                    double b_l = in->a1_l[k] / a1, c_l = 2. * in->a2_l[k];
                    nr_l[i * nd + k] = nr[i] * (-f - ((2. * d * (f - b_l) - e * c_l) / c));
                    sum_l[k] += nr_l[i * nd + k] * qw[i] + nr[i] * qw_l[i * nd + k];
               }
          }
          break;
     }

     case SIZE_DIST_POWER_LAW: {
          power_law_range(a1, a2, r1o, r2o);
          for (k = 0; k < nd; ++k) {
               /* implicit differentiation of the two range equations */
               double L = log(*r2o) - log(*r1o);
               double b = -L + (*r2o - *r1o) / *r1o;
               double c = L - (*r2o - *r1o) / *r2o;
               double a = in->a1_l[k] * L * L;
               double d = in->a2_l[k] * 2. * a1 + (1. + a2) * 2. * in->a1_l[k];
               r1o_l[k] = (c * d - a) / (c - b);
               r2o_l[k] = (b * d - a) / (b - c);
          }
          dist_quad(in->n_int2, in->n_quad, nd, *r1o, *r2o, r1o_l, r2o_l, qx, qw, qx_l, qw_l);
          for (i = 0; i < n; ++i) {
               nr[i] = 1. / pow(qx[i], 3);
               sum += nr[i] * qw[i];
               for (k = 0; k < nd; ++k) {
                    nr_l[i * nd + k] = -nr[i] * 3. * qx_l[i * nd + k] / qx[i];
                    sum_l[k] += nr_l[i * nd + k] * qw[i] + nr[i] * qw_l[i * nd + k];
               }
          }
          break;
     }

     case SIZE_DIST_GAMMA: {
          /* n(r) = r^((1-3b)/b) exp(-r/(a b)), a = r_eff, b = v_eff */
          double b = a1 * a2, c = (1. - 3. * a2) / a2;
          *r1o = in->r1; *r2o = in->r2;
          for (k = 0; k < nd; ++k) { r1o_l[k] = in->r1_l[k]; r2o_l[k] = in->r2_l[k]; }
          dist_quad(in->n_int2, in->n_quad, nd, *r1o, *r2o, r1o_l, r2o_l, qx, qw, qx_l, qw_l);
          for (i = 0; i < n; ++i) {
               double d = pow(qx[i], c), e = qx[i] / b, f = exp(-e), g = 0., h = 0.;
               nr[i] = d * f;
               sum += nr[i] * qw[i];
               if (nd > 0) { g = c / qx[i]; h = log(qx[i]); }
               for (k = 0; k < nd; ++k) {
                    double b_l = in->a1_l[k] * a2 + a1 * in->a2_l[k];
                    double c_l = (-3. * in->a2_l[k] - c * in->a2_l[k]) / a2;
                    nr_l[i * nd + k] = d * ((qx_l[i * nd + k] * g + c_l * h) +
                                       (-qx_l[i * nd + k] + e * b_l) / b) * f;
                    sum_l[k] += nr_l[i * nd + k] * qw[i] + nr[i] * qw_l[i * nd + k];
               }
          }
          break;
     }

     case SIZE_DIST_MODIFIED_POWER_LAW: {
          int n1q = in->n_int1 * in->n_quad;
          *r1o = in->r1; *r2o = in->r2;
          for (k = 0; k < nd; ++k) { r1o_l[k] = in->r1_l[k]; r2o_l[k] = in->r2_l[k]; }
          dist_quad(in->n_int1, in->n_quad, nd, 0., *r1o, NULL, r1o_l, qx, qw, qx_l, qw_l);
          dist_quad(in->n_int2, in->n_quad, nd, *r1o, *r2o, r1o_l, r2o_l,
                    qx + n1q, qw + n1q, qx_l + (size_t) n1q * nd, qw_l + (size_t) n1q * nd);
          for (i = 0; i < n1q; ++i) {
               nr[i] = 1.;
               sum += nr[i] * qw[i];
               for (k = 0; k < nd; ++k) {
                    nr_l[i * nd + k] = 0.;
                    sum_l[k] += nr_l[i * nd + k] * qw[i] + nr[i] * qw_l[i * nd + k];
               }
          }
          for (; i < n; ++i) {
               double b = qx[i] / *r1o;
               nr[i] = pow(b, a1);
               sum += nr[i] * qw[i];
               for (k = 0; k < nd; ++k) {
                    nr_l[i * nd + k] = nr[i] * ((qx_l[i * nd + k] - b * r1o_l[k]) / *r1o *
                                       a1 / b + in->a1_l[k] * log(b));
                    sum_l[k] += nr_l[i * nd + k] * qw[i] + nr[i] * qw_l[i * nd + k];
               }
          }
          break;
     }

     case SIZE_DIST_MODIFIED_BIMODAL_LOG_NORMAL: {
          double b1 = log(a1), c1 = 2. * a2, b2 = log(a3), c2 = 2. * a4;
          *r1o = in->r1; *r2o = in->r2;
          for (k = 0; k < nd; ++k) { r1o_l[k] = in->r1_l[k]; r2o_l[k] = in->r2_l[k]; }
          dist_quad(in->n_int2, in->n_quad, nd, *r1o, *r2o, r1o_l, r2o_l, qx, qw, qx_l, qw_l);
          for (i = 0; i < n; ++i) {
               double d1 = log(qx[i]) - b1, e1 = d1 * d1 / c1;
               double d2 = log(qx[i]) - b2, e2 = d2 * d2 / c2;
               double o1 = exp(-e1), o2 = exp(-e2);
               double f = qx[i] * qx[i], f2 = f * f, p;
               nr[i] = (o1 + a5 * o2) / f2;
               sum += nr[i] * qw[i];
               d1 *= 2.; d2 *= 2.;
               o1 /= c1; o2 /= c2;
               p = nr[i] * 4. * qx[i] * f;
               for (k = 0; k < nd; ++k) {
                    double g = qx_l[i * nd + k] / qx[i];
                    double b1_l = in->a1_l[k] / a1, c1_l = 2. * in->a2_l[k];
                    double b2_l = in->a3_l[k] / a3, c2_l = 2. * in->a4_l[k];
                    double h1 = ((-g + b1_l) * d1 + e1 * c1_l) * o1;
                    double h2 = ((-g + b2_l) * d2 + e2 * c2_l) * o2;
                    nr_l[i * nd + k] = (h1 + in->a5_l[k] * exp(-e2) + a5 * h2 -
                                        p * qx_l[i * nd + k]) / f2;
                    sum_l[k] += nr_l[i * nd + k] * qw[i] + nr[i] * qw_l[i * nd + k];
               }
          }
          break;
     }

     case SIZE_DIST_EXPONENTIAL:
          /* n(D) = exp(-a1 D), D = 2r; no derivatives in the reference
           * (misc/rtutil_size_dist.c:607-613): nr_l stays zero. */
          *r1o = in->r1; *r2o = in->r2;
          for (k = 0; k < nd; ++k) { r1o_l[k] = in->r1_l[k]; r2o_l[k] = in->r2_l[k]; }
          dist_quad(in->n_int2, in->n_quad, nd, *r1o, *r2o, r1o_l, r2o_l, qx, qw, qx_l, qw_l);
          for (i = 0; i < n; ++i) {
               nr[i] = 2. * exp(-a1 * 2. * qx[i]);
               sum += nr[i] * qw[i];
               for (k = 0; k < nd; ++k)
                    nr_l[i * nd + k] = 0.;
          }
          break;

     default:
          free(sum_l);
          return -1;
     }

     /* normalisation (reference misc/rtutil_size_dist.c:621-631) */
     *norm = sum;
     for (k = 0; k < nd; ++k)
          norm_l[k] = sum_l[k];
     for (i = 0; i < n; ++i) {
          nr[i] /= sum;
          for (k = 0; k < nd; ++k)
               nr_l[i * nd + k] = (nr_l[i * nd + k] - nr[i] * sum_l[k]) / sum;
     }
     free(sum_l);
     return n;
}

/* Moments reff, veff, gavg, vavg, ravg, rvw and derivatives
 * (reference misc/rtutil_size_dist.c:653-794). */
static void dist_moments(int n, int nd, const double *qx, const double *qw, const double *nr,
                         const double *qx_l, const double *qw_l, const double *nr_l,
                         lmie_out_data *o) {
     int i, k;
     double m1 = 0., m2 = 0., m3 = 0., m4 = 0., v = 0.;
     double *m1_l = arr1(nd), *m2_l = arr1(nd), *m3_l = arr1(nd), *m4_l = arr1(nd), *v_l = arr1(nd);
     for (i = 0; i < n; ++i) {
          double e = nr[i] * qx[i] * qw[i], r0 = qx[i], r1 = r0 * qx[i], r2 = r1 * qx[i];
          double ew = qx[i] * qw[i], fw = nr[i] * qw[i], gw = nr[i] * qx[i];
          m1 += e; e *= qx[i]; m2 += e; e *= qx[i]; m3 += e; e *= qx[i]; m4 += e;
          for (k = 0; k < nd; ++k) {
               double h = ew * nr_l[i * nd + k], p = fw * qx_l[i * nd + k], q = gw * qw_l[i * nd + k];
               m1_l[k] += h + p + q;
               m2_l[k] += (h + 2. * p + q) * r0;
               m3_l[k] += (h + 3. * p + q) * r1;
               m4_l[k] += (h + 4. * p + q) * r2;
          }
     }
     o->gavg = m2 * M_PI;
     o->vavg = 4. / 3. * M_PI * m3;
     o->ravg = m1;
     o->rvw = 4. / 3. * M_PI * m4 / o->vavg;
     o->reff = m3 / m2;
     for (k = 0; k < nd; ++k) {
          o->gavg_l[k] = m2_l[k] * M_PI;
          o->vavg_l[k] = 4. / 3. * M_PI * m3_l[k];
          o->ravg_l[k] = m1_l[k];
          o->rvw_l[k] = 4. / 3. * M_PI * (m4_l[k] / o->vavg - m4 * o->vavg_l[k] / (o->vavg * o->vavg));
          o->reff_l[k] = m3_l[k] / m2 - m3 * m2_l[k] / (m2 * m2);
     }
     for (i = 0; i < n; ++i) {
          double b = qx[i] - o->reff, c = b * b, d = qx[i] * qx[i], e = d * qw[i], f = c * e;
          double g = 2. * b * e, h = 2. * qx[i] * qw[i];
          v += nr[i] * f;
          for (k = 0; k < nd; ++k) {
               double p = qx_l[i * nd + k] - o->reff_l[k];
               v_l[k] += nr_l[i * nd + k] * f + nr[i] *
                         (g * p + c * (h * qx_l[i * nd + k] + d * qw_l[i * nd + k]));
          }
     }
     {
          double b = o->gavg * o->reff * o->reff;
          double c, d, e, f;
          o->veff = v * M_PI / b;
          c = M_PI / b; d = o->veff * o->reff / b; e = d * o->reff; f = d * o->gavg * 2.;
          for (k = 0; k < nd; ++k)
               o->veff_l[k] = v_l[k] * c - (o->gavg_l[k] * e + f * o->reff_l[k]);
     }
     free(m1_l); free(m2_l); free(m3_l); free(m4_l); free(v_l);
}

/* ------------------------------------------------------------------------ */
/* Per-radius Mie solution (reference src/lmie_core.c:252-791).             */
/* ------------------------------------------------------------------------ */
typedef struct {
     int n_qang, nd, nd1, nd2;
     const int *idx1, *idx2;
     double lambda;
     const double *lambda_l;
     cplx m, m2;
     const cplx *m_l;                /* [nd] */
     const double *fv1, *fv2, *fv3, *fv4;
     const double *mu;               /* Gauss nodes, ascending on [-1,1] */
     int save_control;
     /* accumulators */
     double cext, csca, cbak, g;
     double *cext_l, *csca_l, *cbak_l, *g_l;   /* [nd] */
     double **pf;                    /* [4][n_qang] */
     double ***pf_l;                 /* [nd][4][n_qang] */
     double **save1;                 /* [4][n_qsize] */
     double ***save2;                /* [4][n_qsize][n_qang] */
} core_ctx;

static void mie_radius(core_ctx *C, int ir, double qx, double qw, double nr,
                       const double *qx_l, const double *qw_l, const double *nr_l) {
     int nd1 = C->nd1, nd2 = C->nd2, j, k, l;
     double x = 2. * M_PI * qx / C->lambda;
     cplx z = C->m * x;
     double f = nr * qw;
     int n1 = oracle_calc_n1(x);
     int n2 = oracle_calc_n2(n1, creal(z), cimag(z));
     double *x_l = arr1(nd1), *f_l = arr1(nd1), *f_l2 = arr1(nd2);
     cplx *z_l = (cplx *) calloc(nd1 + 1, sizeof(cplx));
     double *rn = arr1(n1 + 1), *psi = arr1(n1 + 1);
     double *rn_l = arr1((size_t) (n1 + 1) * (nd1 + 1)), *psi_l = arr1((size_t) (n1 + 1) * (nd1 + 1));
     cplx *zeta = (cplx *) calloc(n1 + 1, sizeof(cplx));
     cplx *zeta_l = (cplx *) calloc((size_t) (n1 + 1) * (nd1 + 1), sizeof(cplx));
     cplx *Dn = (cplx *) calloc(n2 + 1, sizeof(cplx));
     cplx *Dn_l = (cplx *) calloc((size_t) (n2 + 1) * (nd1 + 1), sizeof(cplx));
     cplx *a = (cplx *) calloc(n1 + 2, sizeof(cplx)), *b = (cplx *) calloc(n1 + 2, sizeof(cplx));
     cplx *a_l = (cplx *) calloc((size_t) (n1 + 2) * (nd1 + 1), sizeof(cplx));
     cplx *b_l = (cplx *) calloc((size_t) (n1 + 2) * (nd1 + 1), sizeof(cplx));
     double cosx = cos(x), sinx = sin(x);
#define L1(arr, n, k) (arr)[(size_t) (n) * (nd1 + 1) + (k)]

     for (k = 0; k < nd1; ++k) {
          int kk = C->idx1[k];
          x_l[k] = 2. * M_PI * (qx_l[kk] - qx * D(C->lambda_l, kk) / C->lambda) / C->lambda;
          z_l[k] = C->m_l[kk] * x + C->m * x_l[k];
          f_l[k] = nr_l[kk] * qw + nr * qw_l[kk];
     }
     for (k = 0; k < nd2; ++k)
          f_l2[k] = nr_l[C->idx2[k]] * qw;

     /* psi_n by the downward ratio r_n = psi_n/psi_{n-1} (src/lmie_core.c:298-330) */
     rn[n1] = 0.;
     for (k = 0; k < nd1; ++k) L1(rn_l, n1, k) = 0.;
     for (j = n1 - 1; j >= 0; --j) {
          double t = C->fv1[j] / x;
          rn[j] = 1. / (t - rn[j + 1]);
          for (k = 0; k < nd1; ++k)
               L1(rn_l, j, k) = -((-t / x) * x_l[k] - L1(rn_l, j + 1, k)) * (rn[j] * rn[j]);
     }
     psi[0] = sinx;
     psi[1] = rn[1] * psi[0];
     for (k = 0; k < nd1; ++k) {
          L1(psi_l, 0, k) = x_l[k] * cosx;
          L1(psi_l, 1, k) = L1(rn_l, 1, k) * psi[0] + rn[1] * L1(psi_l, 0, k);
     }
     for (j = 1; j < n1; ++j) {
          psi[j + 1] = rn[j + 1] * psi[j];
          for (k = 0; k < nd1; ++k)
               L1(psi_l, j + 1, k) = L1(rn_l, j + 1, k) * psi[j] + rn[j + 1] * L1(psi_l, j, k);
     }

     /* chi_n upward, zeta = psi + i chi (src/lmie_core.c:336-380) */
     {
          double t = 1. / x, c0 = cosx, c1 = t * c0 + sinx, c2;
          double *c0_l = arr1(nd1), *c1_l = arr1(nd1);
          zeta[0] = psi[0] + I * c0;
          zeta[1] = psi[1] + I * c1;
          for (k = 0; k < nd1; ++k) {
               c0_l[k] = x_l[k] * -sinx;
               c1_l[k] = (-t / x) * x_l[k] * c0 + t * c0_l[k] + x_l[k] * cosx;
               L1(zeta_l, 0, k) = L1(psi_l, 0, k) + I * c0_l[k];
               L1(zeta_l, 1, k) = L1(psi_l, 1, k) + I * c1_l[k];
          }
          for (j = 1; j < n1; ++j) {
               t = C->fv1[j] / x;
               c2 = t * c1 - c0;
               zeta[j + 1] = psi[j + 1] + I * c2;
               for (k = 0; k < nd1; ++k) {
                    double t_l = -t * x_l[k] / x;
                    double c2_l = t_l * c1 + t * c1_l[k] - c0_l[k];
                    L1(zeta_l, j + 1, k) = L1(psi_l, j + 1, k) + I * c2_l;
                    c0_l[k] = c1_l[k];
                    c1_l[k] = c2_l;
               }
               c0 = c1;
               c1 = c2;
          }
          free(c0_l); free(c1_l);
     }

     /* D_n(z) downward from D_{n2} = 0 (src/lmie_core.c:386-405) */
     Dn[n2] = 0.;
     for (k = 0; k < nd1; ++k) L1(Dn_l, n2, k) = 0.;
     for (j = n2 - 1; j >= 0; --j) {
          cplx c1 = (j + 1.) / z, c2 = Dn[j + 1] + c1;
          Dn[j] = c1 - 1. / c2;
          for (k = 0; k < nd1; ++k) {
               cplx c5 = (-c1 / z) * z_l[k];
               L1(Dn_l, j, k) = c5 + (L1(Dn_l, j + 1, k) + c5) / (c2 * c2);
          }
     }

     /* a_n, b_n and their tangent-linear forms (src/lmie_core.c:453-498) */
     for (j = 1; j <= n1; ++j) {
          double t = j / x;
          cplx c1 = Dn[j] / C->m + t;
          cplx num = c1 * psi[j] - psi[j - 1];
          cplx den = c1 * zeta[j] - zeta[j - 1];
          a[j] = num / den;
          for (k = 0; k < nd1; ++k) {
               int kk = C->idx1[k];
               double t_l = -t * x_l[k] / x;
               cplx c6 = L1(Dn_l, j, k) / C->m - Dn[j] / C->m2 * C->m_l[kk] + t_l;
               L1(a_l, j, k) = (c6 * psi[j] + c1 * L1(psi_l, j, k) - L1(psi_l, j - 1, k)) / den - num *
                               (c6 * zeta[j] + c1 * L1(zeta_l, j, k) - L1(zeta_l, j - 1, k)) / (den * den);
          }
          c1 = C->m * Dn[j] + t;
          num = c1 * psi[j] - psi[j - 1];
          den = c1 * zeta[j] - zeta[j - 1];
          b[j] = num / den;
          for (k = 0; k < nd1; ++k) {
               int kk = C->idx1[k];
               double t_l = -t * x_l[k] / x;
               cplx c4 = C->m_l[kk] * Dn[j] + C->m * L1(Dn_l, j, k) + t_l;
               L1(b_l, j, k) = (c4 * psi[j] + c1 * L1(psi_l, j, k) - L1(psi_l, j - 1, k)) / den - num *
                               (c4 * zeta[j] + c1 * L1(zeta_l, j, k) - L1(zeta_l, j - 1, k)) / (den * den);
          }
     }

     /* Cext, Csca, Cbak kernels (src/lmie_core.c:504-566) */
     {
          double se = 0., ss = 0., sgn = -1.;
          cplx sb = 0.;
          double *se_l = arr1(nd1), *ss_l = arr1(nd1);
          cplx *sb_l = (cplx *) calloc(nd1 + 1, sizeof(cplx));
          double bak;
          for (j = 1; j <= n1; ++j) {
               se += C->fv1[j] * creal(a[j] + b[j]);
               ss += C->fv1[j] * (creal(a[j] * conj(a[j])) + creal(b[j] * conj(b[j])));
               sb += C->fv1[j] * (a[j] - b[j]) * sgn;
               for (k = 0; k < nd1; ++k) {
                    se_l[k] += C->fv1[j] * creal(L1(a_l, j, k) + L1(b_l, j, k));
                    ss_l[k] += C->fv1[j] * 2. * (creal(a[j] * conj(L1(a_l, j, k))) +
                                                creal(b[j] * conj(L1(b_l, j, k))));
                    sb_l[k] += C->fv1[j] * (L1(a_l, j, k) - L1(b_l, j, k)) * sgn;
               }
               sgn = -sgn;
          }
          bak = creal(sb * conj(sb));
          C->cext += f * se;
          C->csca += f * ss;
          C->cbak += f * bak;
          if (C->save_control == 1) {
               C->save1[0][ir] = se;
               C->save1[1][ir] = ss;
               C->save1[2][ir] = bak;
          }
          for (k = 0; k < nd1; ++k) {
               int kk = C->idx1[k];
               C->cext_l[kk] += f_l[k] * se + f * se_l[k];
               C->csca_l[kk] += f_l[k] * ss + f * ss_l[k];
               C->cbak_l[kk] += f_l[k] * bak + f * 2. * creal(sb * conj(sb_l[k]));
          }
          for (k = 0; k < nd2; ++k) {
               int kk = C->idx2[k];
               C->cext_l[kk] += f_l2[k] * se;
               C->csca_l[kk] += f_l2[k] * ss;
               C->cbak_l[kk] += f_l2[k] * bak;
          }
          free(se_l); free(ss_l); free(sb_l);
     }

     /* asymmetry kernel (src/lmie_core.c:572-611) */
     {
          double sg = 0.;
          double *sg_l = arr1(nd1);
          for (j = 1; j < n1; ++j) {
               sg += C->fv3[j] * creal(a[j] * conj(a[j + 1]) + b[j] * conj(b[j + 1])) +
                     C->fv4[j] * creal(a[j] * conj(b[j]));
               for (k = 0; k < nd1; ++k)
                    sg_l[k] += C->fv3[j] * creal(L1(a_l, j, k) * conj(a[j + 1]) + a[j] * conj(L1(a_l, j + 1, k)) +
                                                 L1(b_l, j, k) * conj(b[j + 1]) + b[j] * conj(L1(b_l, j + 1, k))) +
                               C->fv4[j] * creal(L1(a_l, j, k) * conj(b[j]) + a[j] * conj(L1(b_l, j, k)));
          }
          C->g += f * sg;
          if (C->save_control == 1)
               C->save1[3][ir] = sg;
          for (k = 0; k < nd1; ++k)
               C->g_l[C->idx1[k]] += f_l[k] * sg + f * sg_l[k];
          for (k = 0; k < nd2; ++k)
               C->g_l[C->idx2[k]] += f_l2[k] * sg;
          free(sg_l);
     }

     /* angular accumulation (src/lmie_core.c:617-791) */
     if (C->n_qang > 0) {
          int nh = C->n_qang / 2;
          cplx *cs = (cplx *) calloc((size_t) (n1 + 1) * (nd1 + 1), sizeof(cplx));   /* fv4 (a+b) */
          cplx *cd = (cplx *) calloc((size_t) (n1 + 1) * (nd1 + 1), sizeof(cplx));   /* fv4 (a-b) */
          cplx *sp = (cplx *) calloc(2 * (nd1 + 1), sizeof(cplx));
          cplx *sm = (cplx *) calloc(2 * (nd1 + 1), sizeof(cplx));
          double half_f = f * .5;
          for (j = 1; j <= n1; ++j) {
               L1(cs, j, 0) = C->fv4[j] * (a[j] + b[j]);
               L1(cd, j, 0) = C->fv4[j] * (a[j] - b[j]);
               for (k = 0; k < nd1; ++k) {
                    L1(cs, j, k + 1) = C->fv4[j] * (L1(a_l, j, k) + L1(b_l, j, k));
                    L1(cd, j, k + 1) = C->fv4[j] * (L1(a_l, j, k) - L1(b_l, j, k));
               }
          }
          for (j = 0; j < nh; ++j) {
               double p0 = 0., p1 = 1., par = 1.;
               for (k = 0; k < 2 * (nd1 + 1); ++k) sp[k] = sm[k] = 0.;
               /* sp/sm[0..nd1]: node j; sp/sm[nd1+1..]: its mirror n_qang-1-j
                * (pi_n(-mu) = (-1)^(n+1) pi_n(mu), tau_n(-mu) = (-1)^n tau_n(mu)) */
               for (k = 1; k <= n1; ++k) {
                    double t1 = C->mu[j] * p1, t2 = t1 - p0, tau = k * t2 - p0;
                    double tp = p1 + tau, tm = p1 - tau;
                    for (l = 0; l <= nd1; ++l) {
                         sp[l] += tp * L1(cs, k, l);
                         sm[l] += tm * L1(cd, k, l);
                         sp[nd1 + 1 + l] += tm * (L1(cs, k, l) * par);
                         sm[nd1 + 1 + l] += tp * (L1(cd, k, l) * par);
                    }
                    par = -par;
                    p0 = p1;
                    p1 = t1 + C->fv2[k] * t2;
               }
               for (l = 0; l < 2; ++l) {
                    int jj = l == 0 ? j : C->n_qang - j - 1;
                    cplx s1 = .5 * (sp[l * (nd1 + 1)] + sm[l * (nd1 + 1)]);
                    cplx s2 = .5 * (sp[l * (nd1 + 1)] - sm[l * (nd1 + 1)]);
                    double e1 = creal(s1) * creal(s1) + cimag(s1) * cimag(s1);
                    cplx c12 = s1 * conj(s2);
                    double e3 = creal(s2) * creal(s2) + cimag(s2) * cimag(s2);
                    cplx c21 = s2 * conj(s1);
                    double p5 = (e1 + e3) * .5;
                    double p6 = (creal(c12) + creal(c21)) * .5;
                    double p7 = -(e1 - e3) * .5;
                    double p8 = -creal((c12 - c21) * .5 * I);
                    C->pf[0][jj] += f * p5;
                    C->pf[1][jj] += f * p6;
                    C->pf[2][jj] += f * p7;
                    C->pf[3][jj] += f * p8;
                    if (C->save_control == 1) {
                         C->save2[0][ir][jj] = p5;
                         C->save2[1][ir][jj] = p6;
                         C->save2[2][ir][jj] = p7;
                         C->save2[3][ir][jj] = p8;
                    }
                    for (k = 0; k < nd1; ++k) {
                         int kk = C->idx1[k];
                         cplx s1l = .5 * (sp[l * (nd1 + 1) + k + 1] + sm[l * (nd1 + 1) + k + 1]);
                         cplx s2l = .5 * (sp[l * (nd1 + 1) + k + 1] - sm[l * (nd1 + 1) + k + 1]);
                         double q1 = 2. * (creal(s1l) * creal(s1) + cimag(s1l) * cimag(s1));
                         cplx d12 = 2. * s1l * conj(s2);
                         double q3 = 2. * (creal(s2l) * creal(s2) + cimag(s2l) * cimag(s2));
                         cplx d21 = 2. * s2l * conj(s1);
                         C->pf_l[kk][0][jj] += f_l[k] * p5 + half_f * (q1 + q3);
                         C->pf_l[kk][1][jj] += f_l[k] * p6 + half_f * (creal(d12) + creal(d21));
                         C->pf_l[kk][2][jj] += f_l[k] * p7 + half_f * -(q1 - q3);
                         C->pf_l[kk][3][jj] += f_l[k] * p8 + half_f * -creal((d12 - d21) * I);
                    }
                    for (k = 0; k < nd2; ++k) {
                         int kk = C->idx2[k];
                         C->pf_l[kk][0][jj] += p5 * f_l2[k];
                         C->pf_l[kk][1][jj] += p6 * f_l2[k];
                         C->pf_l[kk][2][jj] += p7 * f_l2[k];
                         C->pf_l[kk][3][jj] += p8 * f_l2[k];
                    }
               }
          }
          free(cs); free(cd); free(sp); free(sm);
     }
#undef L1
     free(x_l); free(f_l); free(f_l2); free(z_l);
     free(rn); free(psi); free(rn_l); free(psi_l);
     free(zeta); free(zeta_l); free(Dn); free(Dn_l);
     free(a); free(b); free(a_l); free(b_l);
}

int oracle_mie_ab(double x, double mr, double mi, double *ab) {
     /* Standalone a_n/b_n via the same recurrences, no derivatives. */
     int n1 = oracle_calc_n1(x), j;
     cplx m = mr - I * mi, z = m * x;
     int n2 = oracle_calc_n2(n1, creal(z), cimag(z));
     double *rn = arr1(n1 + 1), *psi = arr1(n1 + 1);
     cplx *zeta = (cplx *) calloc(n1 + 1, sizeof(cplx)), *Dn = (cplx *) calloc(n2 + 1, sizeof(cplx));
     double c0 = cos(x), c1, c2;
     rn[n1] = 0.;
     for (j = n1 - 1; j >= 0; --j)
          rn[j] = 1. / ((2. * j + 1.) / x - rn[j + 1]);
     psi[0] = sin(x);
     for (j = 0; j < n1; ++j)
          psi[j + 1] = rn[j + 1] * psi[j];
     c1 = 1. / x * c0 + sin(x);
     zeta[0] = psi[0] + I * c0;
     zeta[1] = psi[1] + I * c1;
     for (j = 1; j < n1; ++j) {
          c2 = (2. * j + 1.) / x * c1 - c0;
          zeta[j + 1] = psi[j + 1] + I * c2;
          c0 = c1; c1 = c2;
     }
     Dn[n2] = 0.;
     for (j = n2 - 1; j >= 0; --j) {
          cplx t = (j + 1.) / z;
          Dn[j] = t - 1. / (Dn[j + 1] + t);
     }
     for (j = 1; j <= n1; ++j) {
          cplx ca = Dn[j] / m + j / x, cb = m * Dn[j] + j / x;
          cplx an = (ca * psi[j] - psi[j - 1]) / (ca * zeta[j] - zeta[j - 1]);
          cplx bn = (cb * psi[j] - psi[j - 1]) / (cb * zeta[j] - zeta[j - 1]);
          ab[2 * (j - 1)] = creal(an);
          ab[2 * (j - 1) + 1] = cimag(an);
          ab[2 * (n1 + j - 1)] = creal(bn);
          ab[2 * (n1 + j - 1) + 1] = cimag(bn);
     }
     free(rn); free(psi); free(zeta); free(Dn);
     return n1;
}

/* ------------------------------------------------------------------------ */
/* Generalized spherical functions P00, P0+2, P2+2, P2-2 by 3-term
 * recurrences in l (reference misc/rtutil_math.c:936-1017).               */
/* ------------------------------------------------------------------------ */
static void gsf_prt(int nl, double mu, double *p00, double *p02, double *p22, double *p2m) {
     int j;
     double mu2 = mu * mu;
     if (nl > 0) { p00[0] = 1.; p02[0] = 0.; p22[0] = 0.; p2m[0] = 0.; }
     if (nl > 1) { p00[1] = mu; p02[1] = 0.; p22[1] = 0.; p2m[1] = 0.; }
     if (nl > 2) {
          double t;
          p00[2] = (3. * mu2 - 1.) / 2.;
          p02[2] = .25 * sqrt(6.) * (mu2 - 1.);
          t = 1. + mu; p22[2] = .25 * t * t;
          t = 1. - mu; p2m[2] = .25 * t * t;
     }
     for (j = 2; j < nl - 1; ++j) {
          double jj = (double) j * j, jp1 = j + 1., jjp1 = j * jp1, jp1s = jp1 * jp1, tj1 = 2 * j + 1;
          double a02 = sqrt(jj - 4), b02 = sqrt(jp1s - 4);
          double a22 = tj1 * 4, b22 = jp1 * (jj - 4), c22 = j * (jp1s - 4);
          double t = tj1 * mu;
          p00[j + 1] = (t * p00[j] - j * p00[j - 1]) / jp1;
          p02[j + 1] = (t * p02[j] - a02 * p02[j - 1]) / b02;
          t = tj1 * jjp1 * mu;
          p22[j + 1] = ((t - a22) * p22[j] - b22 * p22[j - 1]) / c22;
          p2m[j + 1] = ((t + a22) * p2m[j] - b22 * p2m[j - 1]) / c22;
     }
}

/* Legendre polynomials (reference misc/rtutil_math.c:477-513). */
static void legendre(int nl, double mu, double *p) {
     int j;
     p[0] = 1.;
     if (nl > 1) p[1] = mu;
     for (j = 1; j < nl - 1; ++j) {
          double a = j / (j + 1.), b = mu * p[j];
          p[j + 1] = a * (b - p[j - 1]) + b;
     }
}

/* pf4 rows -> the 6 expansion inputs (reference src/lmie_schedule.c:927-935). */
static void pf4_to_6(double **pf4, double *pf6[6]) {
     pf6[0] = pf4[0]; pf6[1] = pf4[0]; pf6[2] = pf4[1];
     pf6[3] = pf4[1]; pf6[4] = pf4[2]; pf6[5] = pf4[3];
}

/* GSF projection with mu-parity folding (reference misc/rtutil_scat_int.c:20-56,63-230). */
static int gsf_project(int n_coef, int n_qang, double **pf4, const double *mu, const double *w,
                       double ***P, double **coefs, double accuracy) {
     int i, j, k, i1 = n_qang / 2 - 1, i2 = n_qang / 2;
     double *pf[6];
     pf4_to_6(pf4, pf);
     for (k = 0; k < 6; ++k)
          for (j = 0; j < n_coef; ++j)
               coefs[k][j] = 0.;
     for (i = 0; i < n_qang / 2; ++i, --i1, ++i2) {
          double b1[6], b2[6], t, s = 1.;
          for (k = 0; k < 6; ++k) { b1[k] = pf[k][i1] * w[i2]; b2[k] = pf[k][i2] * w[i2]; }
          t = b1[1]; b1[1] = t + b1[2]; b1[2] = t - b1[2];
          t = b2[1]; b2[1] = t + b2[2]; b2[2] = t - b2[2];
          for (j = 0; j < n_coef; ++j) {
               coefs[0][j] += P[0][i][j] * (b1[0] * s + b2[0]);
               coefs[1][j] += P[3][i][j] * b1[1] * s + P[2][i][j] * b2[1];
               coefs[2][j] += P[2][i][j] * b1[2] * s + P[3][i][j] * b2[2];
               coefs[3][j] += P[0][i][j] * (b1[3] * s + b2[3]);
               coefs[4][j] += P[1][i][j] * (b1[4] * s + b2[4]);
               coefs[5][j] += P[1][i][j] * (b1[5] * s + b2[5]);
               s = -s;
          }
     }
     for (j = 0; j < n_coef; ++j) {
          double t = coefs[1][j];
          coefs[1][j] = (t + coefs[2][j]) / 2.;
          coefs[2][j] = (t - coefs[2][j]) / 2.;
     }
     for (j = 0; j < n_coef; ++j) {
          double t = (2 * j + 1) / 2.;
          for (k = 0; k < 6; ++k)
               coefs[k][j] *= t;
     }
     for (j = 0; j < n_coef; ++j)
          if (fabs(coefs[0][j]) <= accuracy)
               return j + 1;
     return n_coef;
}

/* Legendre projection (reference misc/rtutil_scat_int.c:353-480). */
static int leg_project(int n_coef, int n_qang, double **pf4, const double *w,
                       double **Y, double **coefs, double accuracy) {
     int i, j, k, i1 = n_qang / 2 - 1, i2 = n_qang / 2;
     double *pf[6];
     pf4_to_6(pf4, pf);
     for (k = 0; k < 6; ++k)
          for (j = 0; j < n_coef; ++j)
               coefs[k][j] = 0.;
     for (i = 0; i < n_qang / 2; ++i, --i1, ++i2) {
          double b1[6], b2[6], s = 1.;
          for (k = 0; k < 6; ++k) { b1[k] = pf[k][i1] * w[i2]; b2[k] = pf[k][i2] * w[i2]; }
          for (j = 0; j < n_coef; ++j) {
               for (k = 0; k < 6; ++k)
                    coefs[k][j] += Y[i][j] * (b1[k] * s + b2[k]);
               s = -s;
          }
     }
     for (j = 0; j < n_coef; ++j)
          coefs[5][j] = -coefs[5][j];
     for (j = 0; j < n_coef; ++j) {
          double t = (2. * j + 1.) / 2.;
          for (k = 0; k < 6; ++k)
               coefs[k][j] *= t;
     }
     for (j = 0; j < n_coef; ++j)
          if (fabs(coefs[0][j]) <= accuracy)
               return j + 1;
     return n_coef;
}

/* Phase matrix at theta_i = i*180/(n-1) from the expansion
 * (reference misc/rtutil_scat_int.c:487-589,662-710,771-797). */
static void expand_pf(int n_coef, int n_theta, double **coefs, double *theta, double **pf, int gc) {
     int i, j;
     double d = 180. / (n_theta - 1);
     double *p00 = arr1(n_coef), *p02 = arr1(n_coef), *p22 = arr1(n_coef), *p2m = arr1(n_coef);
     for (i = 0; i < n_theta; ++i)
          theta[i] = i * d;
     for (i = 0; i < n_theta; ++i) {
          double mu = cos(theta[i] * (M_PI / 180.0));
          double s[6] = {0., 0., 0., 0., 0., 0.};
          if (gc) {
               gsf_prt(n_coef, mu, p00, p02, p22, p2m);
               for (j = 0; j < 2 && j < n_coef; ++j) {
                    s[0] += coefs[0][j] * p00[j];
                    s[3] += coefs[3][j] * p00[j];
               }
               for (; j < n_coef; ++j) {
                    s[0] += coefs[0][j] * p00[j];
                    s[3] += coefs[3][j] * p00[j];
                    s[4] += coefs[4][j] * p02[j];
                    s[5] += coefs[5][j] * p02[j];
                    s[1] += (coefs[1][j] + coefs[2][j]) * p22[j];
                    s[2] += (coefs[1][j] - coefs[2][j]) * p2m[j];
               }
               pf[0][i] = s[0];
               pf[3][i] = s[3];
               pf[4][i] = s[4];
               pf[5][i] = s[5];
               pf[1][i] = (s[1] + s[2]) / 2.;
               pf[2][i] = (s[1] - s[2]) / 2.;
          } else {
               int k;
               legendre(n_coef, mu, p00);
               for (k = 0; k < 6; ++k) {
                    double t = 0.;
                    for (j = 0; j < n_coef; ++j)
                         t += coefs[k][j] * p00[j];
                    pf[k][i] = t;
               }
               pf[5][i] = -pf[5][i];
          }
     }
     free(p00); free(p02); free(p22); free(p2m);
}

/* ------------------------------------------------------------------------ */
/* Driver (reference src/lmie_interface.c:199-507, src/lmie_schedule.c:942-1268). */
/* ------------------------------------------------------------------------ */
int oracle_calc_max_coef(double lambda, enum size_dist_type dist_type,
                         double a1, double a2, double a3, double r1, double r2) {
     (void) a3;
     if (dist_type == SIZE_DIST_POWER_LAW)
          power_law_range(a1, a2, &r1, &r2);
     return 2 * oracle_calc_n1(2. * M_PI * r2 / lambda);
}

static int out_alloc(const lmie_in_data *in, lmie_out_data *out, int max_coef) {
     int nd = in->n_derivs;
     if (nd > 0) {
          out->r1_l = arr1(nd); out->r2_l = arr1(nd); out->norm_l = arr1(nd);
          out->reff_l = arr1(nd); out->veff_l = arr1(nd); out->gavg_l = arr1(nd);
          out->vavg_l = arr1(nd); out->ravg_l = arr1(nd); out->rvw_l = arr1(nd);
          out->cext_l = arr1(nd); out->csca_l = arr1(nd); out->cbak_l = arr1(nd);
          out->g_l = arr1(nd);
     }
     out->gc = NULL; out->gc_l = NULL;
     if (in->calc_gc) {
          out->gc = arr2(6, max_coef);
          if (nd > 0) out->gc_l = arr3(nd, 6, max_coef);
     }
     out->lc = NULL; out->lc_l = NULL;
     if (in->calc_lc) {
          out->lc = arr2(6, max_coef);
          if (nd > 0) out->lc_l = arr3(nd, 6, max_coef);
     }
     out->pf = NULL; out->pf_l = NULL; out->theta = NULL;
     if (in->calc_pf) {
          out->theta = arr1(in->n_angles);
          out->pf = arr2(6, in->n_angles);
          if (nd > 0) out->pf_l = arr3(nd, 6, in->n_angles);
     }
     if (in->save_control != 2) {
          out->save1 = NULL;
          out->save2 = NULL;
     }
     return 0;
}

void oracle_out_free(lmie_out_data *out, int flag) {
     if (flag) {
          free(out->r1_l); free(out->r2_l); free(out->norm_l); free(out->reff_l);
          free(out->veff_l); free(out->gavg_l); free(out->vavg_l); free(out->ravg_l);
          free(out->rvw_l); free(out->cext_l); free(out->csca_l); free(out->cbak_l);
          free(out->g_l);
     }
     if (out->gc) { free(out->gc); if (flag) free(out->gc_l); }
     if (out->lc) { free(out->lc); if (flag) free(out->lc_l); }
     if (out->pf) { free(out->theta); free(out->pf); if (flag) free(out->pf_l); }
}

void oracle_free_save(lmie_out_data *out) {
     free(out->save1); out->save1 = NULL;
     free(out->save2); out->save2 = NULL;
}

int oracle_solution(lmie_in_data *in, lmie_out_data *out, int alloc_out) {
     int n, nd = in->n_derivs, nd1 = 0, nd2 = 0, i, j, k;
     int n1, n2, n_qang, n_coef, n_coef2 = 0;
     int *idx1 = NULL, *idx2 = NULL;
     double *qx, *qw, *nr, *qx_l, *qw_l, *nr_l;
     double x, *fv1, *fv2, *fv3, *fv4, *mu = NULL, *w = NULL;
     double **pf = NULL, ***pf_l = NULL;
     cplx m, m2 = 0., *m_l;
     double **gc, **lc;
     core_ctx C;

     if (alloc_out)
          out_alloc(in, out, oracle_calc_max_coef(in->lambda, in->dist_type, in->a1, in->a2,
                                                  in->a3, in->r1, in->r2));
     gc = out->gc;
     lc = out->lc;

     /* input check (reference src/lmie_interface.c:404-408) */
     if (in->calc_pf && !in->calc_gc && !in->calc_lc) {
          fprintf(stderr, "ERROR: either calc_gc or calc_lc must be set to true when "
                  "calc_pf is true\n");
          return -1;
     }

     n = dist_count(in);
     if (n < 0)
          return -1;
     qx = arr1(n); qw = arr1(n); nr = arr1(n);
     qx_l = arr1((size_t) n * nd); qw_l = arr1((size_t) n * nd); nr_l = arr1((size_t) n * nd);
     if (oracle_particle_dist(in, qx, qw, nr, qx_l, qw_l, nr_l, &out->r1, &out->r2,
                              out->r1_l, out->r2_l, &out->norm, out->norm_l) < 0)
          return -1;
     dist_moments(n, nd, qx, qw, nr, qx_l, qw_l, nr_l, out);

     /* derivative split (reference src/lmie_interface.c:304-353): index1 when
      * lambda, mr, mi or the (output) r1/r2 derivative is non-zero */
     if (nd > 0) {
          idx1 = (int *) calloc(nd, sizeof(int));
          idx2 = (int *) calloc(nd, sizeof(int));
          for (i = 0; i < nd; ++i) {
               if (in->lambda_l[i] != 0. || in->mr_l[i] != 0. || in->mi_l[i] != 0. ||
                   out->r1_l[i] != 0. || out->r2_l[i] != 0.)
                    idx1[nd1++] = i;
               else
                    idx2[nd2++] = i;
          }
     }

     /* global truncation, angles, order tables (reference src/lmie_schedule.c:1004-1072) */
     x = 2. * M_PI * out->r2 / in->lambda;
     m = in->mr - I * in->mi;
     n1 = oracle_calc_n1(x);
     n2 = oracle_calc_n2(n1, creal(m * x), cimag(m * x));
     (void) n2;
     n_qang = (!gc && !lc) ? 0 : 2 * n1;
     n_coef = 2 * n1;
     if (nd > 0)
          m2 = m * m;
     m_l = (cplx *) calloc(nd + 1, sizeof(cplx));
     for (i = 0; i < nd; ++i)
          m_l[i] = in->mr_l[i] - I * in->mi_l[i];
     fv1 = arr1(n1 + 1); fv2 = arr1(n1 + 1); fv3 = arr1(n1 + 1); fv4 = arr1(n1 + 1);
     fv1[0] = 1.;
     for (i = 1; i <= n1; ++i) {
          fv1[i] = 2. * i + 1.;
          fv2[i] = (i + 1.) / i;
          fv3[i] = (i + 2.) / fv2[i];
          fv4[i] = fv1[i] / (i * (i + 1.));
     }
     if (n_qang > 0) {
          mu = arr1(n_qang); w = arr1(n_qang);
          oracle_gauss_leg(n_qang, -1., 1., mu, w);
     }
     pf = arr2(4, n_qang ? n_qang : 1);
     pf_l = arr3(nd ? nd : 1, 4, n_qang ? n_qang : 1);

     memset(&C, 0, sizeof(C));
     C.n_qang = n_qang; C.nd = nd; C.nd1 = nd1; C.nd2 = nd2; C.idx1 = idx1; C.idx2 = idx2;
     C.lambda = in->lambda; C.lambda_l = in->lambda_l; C.m = m; C.m2 = m2; C.m_l = m_l;
     C.fv1 = fv1; C.fv2 = fv2; C.fv3 = fv3; C.fv4 = fv4; C.mu = mu;
     C.save_control = in->save_control;
     C.cext_l = out->cext_l; C.csca_l = out->csca_l; C.cbak_l = out->cbak_l; C.g_l = out->g_l;
     C.pf = pf; C.pf_l = pf_l;
     for (i = 0; i < nd; ++i)
          C.cext_l[i] = C.csca_l[i] = C.cbak_l[i] = C.g_l[i] = 0.;

     if (in->save_control == 1) {
          out->save1 = arr2(4, n);
          out->save2 = arr3(4, n, n_qang ? n_qang : 1);
          C.save1 = out->save1; C.save2 = out->save2;
     }

     if (in->save_control == 2) {
          /* re-weight stored per-radius kernels (reference src/lmie_schedule.c:1087-1124) */
          for (i = 0; i < n; ++i) {
               double a = nr[i] * qw[i];
               C.cext += out->save1[0][i] * a;
               C.csca += out->save1[1][i] * a;
               C.cbak += out->save1[2][i] * a;
               C.g += out->save1[3][i] * a;
               for (j = 0; j < n_qang; ++j)
                    for (k = 0; k < 4; ++k)
                         pf[k][j] += out->save2[k][i][j] * a;
               for (j = 0; j < nd2; ++j) {
                    int jj = idx2[j];
                    double a_l = nr_l[i * nd + jj] * qw[i] + nr[i] * qw_l[i * nd + jj];
                    C.cext_l[jj] += out->save1[0][i] * a_l;
                    C.csca_l[jj] += out->save1[1][i] * a_l;
                    C.cbak_l[jj] += out->save1[2][i] * a_l;
                    C.g_l[jj] += out->save1[3][i] * a_l;
                    for (k = 0; k < n_qang; ++k) {
                         int e;
                         for (e = 0; e < 4; ++e)
                              pf_l[jj][e][k] += out->save2[e][i][k] * a_l;
                    }
               }
          }
     } else {
          for (i = 0; i < n; ++i)
               mie_radius(&C, i, qx[i], qw[i], nr[i],
                          nd ? qx_l + (size_t) i * nd : NULL,
                          nd ? qw_l + (size_t) i * nd : NULL,
                          nd ? nr_l + (size_t) i * nd : NULL);
     }

     /* normalisation (reference src/lmie_schedule.c:1155-1199) */
     {
          double a = 2. / C.csca, a_l;
          for (i = 0; i < nd; ++i) {
               a_l = -a * C.csca_l[i] / C.csca;
               C.g_l[i] = C.g_l[i] * a + C.g * a_l;
               for (j = 0; j < n_qang; ++j)
                    for (k = 0; k < 4; ++k)
                         pf_l[i][k][j] = pf_l[i][k][j] * a + pf[k][j] * a_l;
          }
          C.g = C.g / C.csca * 2.;
          for (j = 0; j < n_qang; ++j)
               for (k = 0; k < 4; ++k)
                    pf[k][j] *= a;
          a = in->lambda * in->lambda / (2. * M_PI);
          for (i = 0; i < nd; ++i) {
               a_l = 2. * in->lambda_l[i] * in->lambda / (2. * M_PI);
               C.cext_l[i] = C.cext_l[i] * a + C.cext * a_l;
               C.csca_l[i] = C.csca_l[i] * a + C.csca * a_l;
               C.cbak_l[i] = (C.cbak_l[i] * a + C.cbak * a_l) / (2. * 4. * M_PI);
          }
          out->cext = C.cext * a;
          out->csca = C.csca * a;
          out->cbak = C.cbak * a / (2. * 4. * M_PI);
          out->g = C.g;
     }

     /* expansions (reference src/lmie_schedule.c:1205-1241) */
     if (gc) {
          double ***P = arr3(4, n_qang / 2 > 0 ? n_qang / 2 : 1, n_coef);
          for (i = 0; i < n_qang / 2; ++i)
               gsf_prt(n_coef, mu[n_qang / 2 + i], P[0][i], P[1][i], P[2][i], P[3][i]);
          n_coef2 = gsf_project(n_coef, n_qang, pf, mu, w, P, gc, in->accuracy);
          for (i = 0; i < nd; ++i) {
               gsf_project(n_coef, n_qang, pf_l[i], mu, w, P, out->gc_l[i], in->accuracy);
               out->gc_l[i][0][0] = 0.;
          }
          free(P);
     }
     if (lc) {
          double **Y = arr2(n_qang / 2 > 0 ? n_qang / 2 : 1, n_coef);
          for (i = 0; i < n_qang / 2; ++i)
               legendre(n_coef, mu[n_qang / 2 + i], Y[i]);
          n_coef2 = leg_project(n_coef, n_qang, pf, w, Y, lc, in->accuracy);
          for (i = 0; i < nd; ++i) {
               leg_project(n_coef, n_qang, pf_l[i], w, Y, out->lc_l[i], in->accuracy);
               out->lc_l[i][0][0] = 0.;
          }
          free(Y);
     }
     out->n_coef = n_coef2;

     /* phase matrix at user angles (reference src/lmie_interface.c:468-483) */
     if (in->calc_pf) {
          if (in->calc_gc) {
               expand_pf(n_coef2, in->n_angles, gc, out->theta, out->pf, 1);
               for (i = 0; i < nd; ++i)
                    expand_pf(n_coef2, in->n_angles, out->gc_l[i], out->theta, out->pf_l[i], 1);
          } else {
               expand_pf(n_coef2, in->n_angles, lc, out->theta, out->pf, 0);
               for (i = 0; i < nd; ++i)
                    expand_pf(n_coef2, in->n_angles, out->lc_l[i], out->theta, out->pf_l[i], 0);
          }
     }

     free(qx); free(qw); free(nr); free(qx_l); free(qw_l); free(nr_l);
     free(idx1); free(idx2); free(m_l);
     free(fv1); free(fv2); free(fv3); free(fv4); free(mu); free(w);
     free(pf); free(pf_l);
     return 0;
}
