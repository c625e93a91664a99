/*
 * host_dist.c -- size-distribution quadrature, moments and Gauss-Legendre
 * nodes for the host side of liblmie_b200.
 *
 * These are the host steps the reference runs before its Mie core; they cost
 * O(n_radii) and stay on the CPU.  Arithmetic follows the reference's
 * operation order so that the radius nodes -- and with them the truncation
 * integers n1(r), n2(r) -- are the reference's to the last bit.
 *
 *   dist_count      <- misc/rtutil_size_dist.c:20-49
 *   power-law range <- misc/rtutil_size_dist.c:95-121 (Brent's method, as in
 *                      misc/zeroin.c: Forsythe, Malcolm & Moler 1977)
 *   gl_nodes        <- misc/rtutil_math.c:73-129,231-316 (Davis & Rabinowitz)
 *   interval quad   <- misc/rtutil_size_dist.c:128-193, misc/rtutil_math.c:329-387
 *   distributions   <- misc/rtutil_size_dist.c:200-646
 *   moments         <- misc/rtutil_size_dist.c:653-794
 */
#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "host.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

int lmieb_dist_count(int dist_type, int n_int1, int n_int2, int n_quad) {
     switch (dist_type) {
     case SIZE_DIST_MONO:
          return 1;
     case SIZE_DIST_MODIFIED_POWER_LAW:
          return n_int1 * n_quad + n_int2 * n_quad;
     case SIZE_DIST_MODIFIED_GAMMA:
     case SIZE_DIST_LOG_NORMAL:
     case SIZE_DIST_POWER_LAW:
     case SIZE_DIST_GAMMA:
     case SIZE_DIST_MODIFIED_BIMODAL_LOG_NORMAL:
     case SIZE_DIST_EXPONENTIAL:
          return n_int2 * n_quad;
     default:
          fprintf(stderr, "ERROR: Invalid distribution type: %d\n", dist_type);
          return -1;
     }
}

/* ---- power-law range: Brent's root finder --------------------------------- */
typedef double (*root_fn)(double, const double *);

static double brent(double lo, double hi, root_fn f, const double *par, double tol) {
     double a = lo, b = hi, c, fa = f(a, par), fb = f(b, par), fc;
     c = a;
     fc = fa;
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
               double cb = c - b, s1, s2;
               if (a == c) {
                    s1 = fb / fa;
                    p = cb * s1;
                    q = 1.0 - s1;
               } else {
                    q = fa / fc;
                    s1 = fb / fc;
                    s2 = fb / fa;
                    p = s2 * (cb * q * (q - s1) - (b - a) * (s1 - 1.0));
                    q = (q - 1.0) * (s1 - 1.0) * (s2 - 1.0);
               }
               if (p > 0)
                    q = -q;
               else
                    p = -p;
               if (p < (0.75 * cb * q - fabs(tol_act * q) / 2) && p < fabs(prev * q / 2))
                    step = p / q;
          }
          if (fabs(step) < tol_act)
               step = step > 0 ? tol_act : -tol_act;
          a = b;
          fa = fb;
          b += step;
          fb = f(b, par);
          if ((fb > 0 && fc > 0) || (fb < 0 && fc < 0)) {
               c = a;
               fc = fa;
          }
     }
}

static double power_law_eq(double r1, const double *par) {
     double r2 = (1. + par[1]) * 2. * par[0] - r1;
     return (r2 - r1) / log(r2 / r1) - par[0];
}

void lmieb_power_law_range(double a1, double a2, double *r1, double *r2) {
     double par[2];
     par[0] = a1;
     par[1] = a2;
     *r1 = brent(DBL_EPSILON, a1, power_law_eq, par, 0.);
     *r2 = (1. + a2) * 2. * a1 - *r1;
}

/* ---- Gauss-Legendre ------------------------------------------------------- */
static void gl_root(int n, int i, int ia, int ib, double da, double *root, double *p_nm1) {
     double th = (4. * i + 3.) / ia * M_PI;
     double y = cos(th + da / tan(th)), y_prev;
     double p_n, p_m, p_mm, t, d1, d2;
     int j;
     do {
          p_m = 0.;
          p_n = 1.;
          for (j = 0; j < n; ++j) {
               p_mm = p_m;
               p_m = p_n;
               t = y * p_m;
               p_n = j / (j + 1.) * (t - p_mm) + t;
          }
          t = 1. - y * y;
          d1 = n * (p_m - y * p_n) / t;
          d2 = (2. * y * d1 - ib * p_n) / t;
          y_prev = y;
          t = p_n / d1;
          y = y_prev - t * (1. + t * d2 / (2. * d1));
     } while (fabs(y - y_prev) > DBL_EPSILON);
     *root = y;
     *p_nm1 = p_m;
}

void lmieb_gauss_leg(int n, double x1, double x2, double *x, double *w) {
     int i, ii = n - 1, half = (n + 1) / 2;
     int ia = 4 * n + 2, ib = n * (n + 1);
     double da = (n - 1) / (8. * pow((double) n, 3));
     double mid = (x1 + x2) / 2., hw = (x2 - x1) / 2.;
     for (i = 0; i < half; ++i, --ii) {
          double y, pm, dd, de;
          gl_root(n, i, ia, ib, da, &y, &pm);
          dd = hw * y;
          x[i] = mid - dd;
          x[ii] = mid + dd;
          de = n * pm;
          de = 2. / (de * de);
          w[i] = (hw - dd * y) * de;
          w[ii] = w[i];
     }
}

/* Gauss-Legendre nodes and weights on [-1, 1] ([x | w]), computed once per n
 * up to GL_CACHE_MAX and kept: every case with the same n_quad reuses them. */
#define GL_CACHE_MAX 4096
static pthread_mutex_t gl_cache_mu = PTHREAD_MUTEX_INITIALIZER;
static double *gl_cache[GL_CACHE_MAX + 1];

static const double *gl_unit(int n) {
     double *p;
     if (n < 1 || n > GL_CACHE_MAX) return NULL;
     pthread_mutex_lock(&gl_cache_mu);
     p = gl_cache[n];
     if (!p && (p = (double *) malloc(sizeof(double) * (size_t) n * 2)) != NULL) {
          lmieb_gauss_leg(n, -1., 1., p, p + n);
          gl_cache[n] = p;
     }
     pthread_mutex_unlock(&gl_cache_mu);
     return p;
}

/* n_int equal sub-intervals of [r1, r2], n_quad nodes each; derivatives of
 * nodes and weights follow from those of the end points (r1_l may be NULL:
 * the lower end is fixed). */
static void interval_quad(int n_int, int n_quad, int nd, double r1, double r2,
                          const double *r1_l, const double *r2_l,
                          double *qx, double *qw, double *qx_l, double *qw_l) {
     int i, j, k, half = (n_quad + 1) / 2;
     const double *unit = gl_unit(n_quad);
     double *own = NULL;
     const double *tx, *tw;
     double step = (r2 - r1) / n_int;
     if (!unit) {
          own = (double *) malloc(sizeof(double) * (size_t) n_quad * 2);
          lmieb_gauss_leg(n_quad, -1., 1., own, own + n_quad);
          unit = own;
     }
     tx = unit;
     tw = unit + n_quad;
     for (i = 0; i < n_int; ++i) {
          size_t base = (size_t) i * n_quad;
          double lo = r1 + i * step, hi = lo + step;
          double mid = (lo + hi) / 2., hw = (hi - lo) / 2.;
          int jj = n_quad - 1;
          for (j = 0; j < half; ++j, --jj) {
               double dd = hw * tx[jj];
               qx[base + j] = mid - dd;
               qx[base + jj] = mid + dd;
               qw[base + j] = tw[j] * hw;
               qw[base + jj] = qw[base + j];
               for (k = 0; k < nd; ++k) {
                    double r1k = r1_l ? r1_l[k] : 0.;
                    double step_l = (r2_l[k] - r1k) / n_int;
                    double lo_l = r1k + i * step_l, hi_l = lo_l + step_l;
                    double mid_l = (lo_l + hi_l) / 2., hw_l = (hi_l - lo_l) / 2.;
                    double dd_l = hw_l * tx[jj];
                    qx_l[(base + j) * nd + k] = mid_l - dd_l;
                    qx_l[(base + jj) * nd + k] = mid_l + dd_l;
                    qw_l[(base + j) * nd + k] = tw[j] * hw_l;
                    qw_l[(base + jj) * nd + k] = qw_l[(base + j) * nd + k];
               }
          }
     }
     free(own);
}

/* ---- distributions ---------------------------------------------------------
 * Each evaluator fills nr[i] (unnormalised) and nr_l[i*nd+k], and adds to the
 * normalisation integral s and its derivatives s_l. */
typedef struct {
     const lmieb_dist_in *in;
     int n, nd;
     const double *qx, *qw, *qx_l, *qw_l;
     double *nr, *nr_l;
     double s, *s_l;
} dist_eval;

static void acc_norm(dist_eval *e, int i) {
     int k, nd = e->nd;
     e->s += e->nr[i] * e->qw[i];
     for (k = 0; k < nd; ++k)
          e->s_l[k] += e->nr_l[(size_t) i * nd + k] * e->qw[i] + e->nr[i] * e->qw_l[(size_t) i * nd + k];
}

static void eval_modified_gamma(dist_eval *e) {
     const lmieb_dist_in *p = e->in;
     int i, k, nd = e->nd;
     double b = pow(p->a2, p->a3), c = p->a3 * b, d = b / c, ee = p->a3 / p->a2, f = log(p->a2);
     double g = p->a1 / c;
     for (i = 0; i < e->n; ++i) {
          double h = pow(e->qx[i], p->a3), o = nd > 0 ? log(e->qx[i]) : 0.;
          e->nr[i] = pow(e->qx[i], p->a1) * exp(-g * h);
          for (k = 0; k < nd; ++k) {
               double pk = e->qx_l[(size_t) i * nd + k] / e->qx[i];
               double c_l = p->a3_l[k] * d + (p->a2_l[k] * ee + p->a3_l[k] * f);
               e->nr_l[(size_t) i * nd + k] = e->nr[i] * ((pk * p->a1 + p->a1_l[k] * o) + h * ((-p->a1_l[k] +
                    p->a1 * (-(pk * p->a3 + p->a3_l[k] * o) + c_l)) / c));
          }
          acc_norm(e, i);
     }
}

static void eval_log_normal(dist_eval *e) {
     const lmieb_dist_in *p = e->in;
     int i, k, nd = e->nd;
     double b = log(p->a1), c = 2. * p->a2;
     for (i = 0; i < e->n; ++i) {
          double d = log(e->qx[i]) - b, ee = d * d / c;
          e->nr[i] = exp(-ee) / e->qx[i];
          for (k = 0; k < nd; ++k) {
               double f = e->qx_l[(size_t) i * nd + k] / e->qx[i];
               double b_l = p->a1_l[k] / p->a1, c_l = 2. * p->a2_l[k];
               e->nr_l[(size_t) i * nd + k] = e->nr[i] * (-f - ((2. * d * (f - b_l) - ee * c_l) / c));
          }
          acc_norm(e, i);
     }
}

static void eval_power_law(dist_eval *e) {
     int i, k, nd = e->nd;
     for (i = 0; i < e->n; ++i) {
          e->nr[i] = 1. / pow(e->qx[i], 3);
          for (k = 0; k < nd; ++k)
               e->nr_l[(size_t) i * nd + k] = -e->nr[i] * 3. * e->qx_l[(size_t) i * nd + k] / e->qx[i];
          acc_norm(e, i);
     }
}

static void eval_gamma(dist_eval *e) {
     const lmieb_dist_in *p = e->in;
     int i, k, nd = e->nd;
     double b = p->a1 * p->a2, c = (1. - 3. * p->a2) / p->a2;
     for (i = 0; i < e->n; ++i) {
          double d = pow(e->qx[i], c), ee = e->qx[i] / b, f = exp(-ee), g = 0., h = 0.;
          e->nr[i] = d * f;
          if (nd > 0) {
               g = c / e->qx[i];
               h = log(e->qx[i]);
          }
          for (k = 0; k < nd; ++k) {
               double b_l = p->a1_l[k] * p->a2 + p->a1 * p->a2_l[k];
               double c_l = (-3. * p->a2_l[k] - c * p->a2_l[k]) / p->a2;
               double xl = e->qx_l[(size_t) i * nd + k];
               e->nr_l[(size_t) i * nd + k] = d * ((xl * g + c_l * h) + (-xl + ee * b_l) / b) * f;
          }
          acc_norm(e, i);
     }
}

static void eval_bimodal(dist_eval *e) {
     const lmieb_dist_in *p = e->in;
     int i, k, nd = e->nd;
     double b1 = log(p->a1), c1 = 2. * p->a2, b2 = log(p->a3), c2 = 2. * p->a4;
     for (i = 0; i < e->n; ++i) {
          double d1 = log(e->qx[i]) - b1, e1 = d1 * d1 / c1;
          double d2 = log(e->qx[i]) - b2, e2 = d2 * d2 / c2;
          double o1 = exp(-e1), o2 = exp(-e2);
          double f = e->qx[i] * e->qx[i], f2 = f * f, q;
          e->nr[i] = (o1 + p->a5 * o2) / f2;
          d1 *= 2.;
          d2 *= 2.;
          o1 /= c1;
          o2 /= c2;
          q = e->nr[i] * 4. * e->qx[i] * f;
          for (k = 0; k < nd; ++k) {
               double g = e->qx_l[(size_t) i * nd + k] / e->qx[i];
               double h1 = ((-g + p->a1_l[k] / p->a1) * d1 + e1 * (2. * p->a2_l[k])) * o1;
               double h2 = ((-g + p->a3_l[k] / p->a3) * d2 + e2 * (2. * p->a4_l[k])) * o2;
               e->nr_l[(size_t) i * nd + k] = (h1 + p->a5_l[k] * exp(-e2) + p->a5 * h2 -
                                               q * e->qx_l[(size_t) i * nd + k]) / f2;
          }
          acc_norm(e, i);
     }
}

static void eval_exponential(dist_eval *e) {
     /* n(D) = exp(-a1 D), D = 2 r.  The reference leaves these derivatives
      * uninitialised (misc/rtutil_size_dist.c:607-613); they are defined as
      * zero here, and the normalisation derivative likewise. */
     int i, k, nd = e->nd;
     for (i = 0; i < e->n; ++i) {
          e->nr[i] = 2. * exp(-e->in->a1 * 2. * e->qx[i]);
          e->s += e->nr[i] * e->qw[i];
          for (k = 0; k < nd; ++k)
               e->nr_l[(size_t) i * nd + k] = 0.;
     }
}

int lmieb_particle_dist(const lmieb_dist_in *in, lmieb_dist_out *o) {
     int n = lmieb_dist_count(in->dist_type, in->n_int1, in->n_int2, in->n_quad);
     int nd = in->nd, i, k;
     dist_eval e;
     if (n < 0)
          return -1;
     memset(&e, 0, sizeof(e));
     e.in = in;
     e.n = n;
     e.nd = nd;
     e.qx = o->qx;
     e.qw = o->qw;
     e.qx_l = o->qx_l;
     e.qw_l = o->qw_l;
     e.nr = o->nr;
     e.nr_l = o->nr_l;
     e.s_l = o->norm_l;
     for (k = 0; k < nd; ++k)
          o->norm_l[k] = 0.;

     if (in->dist_type == SIZE_DIST_MONO) {
          o->r1 = o->r2 = in->a1;
          for (k = 0; k < nd; ++k) {
               o->r1_l[k] = 0.;
               o->r2_l[k] = 0.;
               o->qx_l[k] = in->a1_l[k];
               o->qw_l[k] = 0.;
               o->nr_l[k] = 0.;
          }
          o->qx[0] = in->a1;
          o->qw[0] = 1.;
          o->nr[0] = 1.;
          e.s = 1.;
     } else if (in->dist_type == SIZE_DIST_POWER_LAW) {
          lmieb_power_law_range(in->a1, in->a2, &o->r1, &o->r2);
          for (k = 0; k < nd; ++k) {
               /* implicit derivatives of the two range equations */
               double L = log(o->r2) - log(o->r1);
               double b = -L + (o->r2 - o->r1) / o->r1;
               double c = L - (o->r2 - o->r1) / o->r2;
               double a = in->a1_l[k] * L * L;
               double d = in->a2_l[k] * 2. * in->a1 + (1. + in->a2) * 2. * in->a1_l[k];
               o->r1_l[k] = (c * d - a) / (c - b);
               o->r2_l[k] = (b * d - a) / (b - c);
          }
          interval_quad(in->n_int2, in->n_quad, nd, o->r1, o->r2, o->r1_l, o->r2_l,
                        o->qx, o->qw, o->qx_l, o->qw_l);
          eval_power_law(&e);
     } else {
          o->r1 = in->r1;
          o->r2 = in->r2;
          for (k = 0; k < nd; ++k) {
               o->r1_l[k] = in->r1_l[k];
               o->r2_l[k] = in->r2_l[k];
          }
          if (in->dist_type == SIZE_DIST_MODIFIED_POWER_LAW) {
               int n1q = in->n_int1 * in->n_quad;
               interval_quad(in->n_int1, in->n_quad, nd, 0., o->r1, NULL, o->r1_l,
                             o->qx, o->qw, o->qx_l, o->qw_l);
               interval_quad(in->n_int2, in->n_quad, nd, o->r1, o->r2, o->r1_l, o->r2_l,
                             o->qx + n1q, o->qw + n1q, o->qx_l + (size_t) n1q * nd,
                             o->qw_l + (size_t) n1q * nd);
               for (i = 0; i < n; ++i) {
                    if (i < n1q) {
                         o->nr[i] = 1.;
                         for (k = 0; k < nd; ++k)
                              o->nr_l[(size_t) i * nd + k] = 0.;
                    } else {
                         double b = o->qx[i] / o->r1;
                         o->nr[i] = pow(b, in->a1);
                         for (k = 0; k < nd; ++k)
                              o->nr_l[(size_t) i * nd + k] = o->nr[i] * ((o->qx_l[(size_t) i * nd + k] -
                                   b * o->r1_l[k]) / o->r1 * in->a1 / b + in->a1_l[k] * log(b));
                    }
                    acc_norm(&e, i);
               }
          } else {
               interval_quad(in->n_int2, in->n_quad, nd, o->r1, o->r2, o->r1_l, o->r2_l,
                             o->qx, o->qw, o->qx_l, o->qw_l);
               switch (in->dist_type) {
               case SIZE_DIST_MODIFIED_GAMMA: eval_modified_gamma(&e); break;
               case SIZE_DIST_LOG_NORMAL: eval_log_normal(&e); break;
               case SIZE_DIST_GAMMA: eval_gamma(&e); break;
               case SIZE_DIST_MODIFIED_BIMODAL_LOG_NORMAL: eval_bimodal(&e); break;
               case SIZE_DIST_EXPONENTIAL: eval_exponential(&e); break;
               default:
                    fprintf(stderr, "ERROR: Invalid distribution type: %d\n", in->dist_type);
                    return -1;
               }
          }
     }

     /* normalise n(r) to unit integral */
     o->norm = e.s;
     for (i = 0; i < n; ++i) {
          o->nr[i] /= e.s;
          for (k = 0; k < nd; ++k)
               o->nr_l[(size_t) i * nd + k] = (o->nr_l[(size_t) i * nd + k] - o->nr[i] * o->norm_l[k]) / e.s;
     }
     return n;
}

/* ---- moments --------------------------------------------------------------- */
void lmieb_moments(int n, int nd, const double *qx, const double *qw, const double *nr,
                   const double *qx_l, const double *qw_l, const double *nr_l,
                   lmieb_moments_out *m) {
     int i, k;
     double s1 = 0., s2 = 0., s3 = 0., s4 = 0., v = 0.;
     double *t = (double *) calloc((size_t) (nd > 0 ? nd : 1) * 5, sizeof(double));
     double *s1_l = t, *s2_l = t + nd, *s3_l = t + 2 * nd, *s4_l = t + 3 * nd, *v_l = t + 4 * nd;
     for (i = 0; i < n; ++i) {
          double e = nr[i] * qx[i] * qw[i];
          double r0 = qx[i], r1 = r0 * qx[i], r2 = r1 * qx[i];
          double xw = qx[i] * qw[i], nw = nr[i] * qw[i], nx = nr[i] * qx[i];
          s1 += e;
          e *= qx[i];
          s2 += e;
          e *= qx[i];
          s3 += e;
          e *= qx[i];
          s4 += e;
          for (k = 0; k < nd; ++k) {
               size_t ik = (size_t) i * nd + k;
               double h = xw * nr_l[ik], p = nw * qx_l[ik], q = nx * qw_l[ik];
               s1_l[k] += h + p + q;
               s2_l[k] += (h + 2. * p + q) * r0;
               s3_l[k] += (h + 3. * p + q) * r1;
               s4_l[k] += (h + 4. * p + q) * r2;
          }
     }
     m->gavg = s2 * M_PI;
     m->vavg = 4. / 3. * M_PI * s3;
     m->ravg = s1;
     m->rvw = 4. / 3. * M_PI * s4 / m->vavg;
     m->reff = s3 / s2;
     for (k = 0; k < nd; ++k) {
          m->gavg_l[k] = s2_l[k] * M_PI;
          m->vavg_l[k] = 4. / 3. * M_PI * s3_l[k];
          m->ravg_l[k] = s1_l[k];
          m->rvw_l[k] = 4. / 3. * M_PI * (s4_l[k] / m->vavg - s4 * m->vavg_l[k] / (m->vavg * m->vavg));
          m->reff_l[k] = s3_l[k] / s2 - s3 * s2_l[k] / (s2 * s2);
     }
     for (i = 0; i < n; ++i) {
          double b = qx[i] - m->reff, c = b * b, d = qx[i] * qx[i], e = d * qw[i], f = c * e;
          double g = 2. * b * e, h = 2. * qx[i] * qw[i];
          v += nr[i] * f;
          for (k = 0; k < nd; ++k) {
               size_t ik = (size_t) i * nd + k;
               double p = qx_l[ik] - m->reff_l[k];
               v_l[k] += nr_l[ik] * f + nr[i] * (g * p + c * (h * qx_l[ik] + d * qw_l[ik]));
          }
     }
     {
          double b = m->gavg * m->reff * m->reff, c, d, e, f;
          m->veff = v * M_PI / b;
          c = M_PI / b;
          d = m->veff * m->reff / b;
          e = d * m->reff;
          f = d * m->gavg * 2.;
          for (k = 0; k < nd; ++k)
               m->veff_l[k] = v_l[k] * c - (m->gavg_l[k] * e + f * m->reff_l[k]);
     }
     free(t);
}
