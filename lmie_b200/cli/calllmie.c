/*
 * calllmie.c -- command-line driver of liblmie_b200: one polydisperse solve
 * described by flags, written as LMie's text scattering files.
 *
 * It keeps the reference tool's command line and output (utils/calllmie.c):
 *
 *   -dist <name> <values...>     size distribution and its parameters, the
 *                                values each type takes per
 *                                misc/rtutil_support.c:580-673 (mono: r;
 *                                modified_gamma: a1 a2 a3 r1 r2; log_normal,
 *                                gamma: a1 a2 r1 r2; power_law: a1 a2;
 *                                modified_power_law: a1 r1 r2;
 *                                modified_bimodal_log_normal: a1..a5 r1 r2;
 *                                exponential: a1 r1 r2)
 *   -lambda <l>  -m <mr> <mi>  -n_int1 <n>  -n_int2 <n>  -n_quad <n>
 *   -n_angles <n> (default 18001)  -accuracy <a> (default 1e-7)
 *   -derivs <n>                  number of derivative inputs; then
 *   -lambda_l <list>  -m_l <mr list> <mi list>  -dist_l <lists...>
 *                                comma-separated lists of n values
 *                                (misc/rtutil_support.c:449-500,676-756)
 *   -total <file> [<files>]      header: inputs, integrated quantities
 *   -gc <file> [<files>]         generalized-spherical-function coefficients
 *   -lc <file> [<files>]         Legendre coefficients
 *   -pf <file> [<files>]         phase matrix at n_angles angles
 *                                ("-" writes to stdout; with -derivs a second
 *                                argument lists one file per derivative)
 *   -check_cbak <tol>  -check_g <tol>   self-consistency checks
 *                                (utils/calllmie.c:731-755)
 *   -save_dist                   solve once with save_control 1, then again
 *                                from the saved per-radius quantities
 *   -n_threads <n>  -timing <n>  -verbose  -findif <x>  -help  -version
 *                                (-timing times n full solves, save_control 0)
 *
 * File formats follow misc/rtutil_scat_io.c:250-289 (header),
 * 636-697 (phase matrix) and 823-877 (coefficients).  -timing repeats the
 * solve n times and prints the elapsed wall-clock seconds (the work runs on
 * the GPU, so host CPU time would not measure it).  Errors print an
 * "ERROR: ..." line and exit with status 1, as the reference does.
 */
#define _POSIX_C_SOURCE 200809L

#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <lmie_interface.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define TOOL "calllmie"
#define TOOL_VERSION "lmie_b200"

static void die(const char *fmt, const char *a, const char *b) {
     fprintf(stderr, "ERROR: ");
     fprintf(stderr, fmt, a, b);
     fprintf(stderr, "\n");
     exit(1);
}

/* the next n arguments after argv[i] must exist */
static void need(int i, int argc, int n, const char *opt) {
     if (i + n >= argc) die("not enough arguments for %s%s", opt, "");
}

static double num(const char *s, const char *opt) {
     char *end;
     double v;
     errno = 0;
     v = strtod(s, &end);
     if (errno || end == s || *end != '\0') die("invalid value for %s: %s", opt, s);
     return v;
}

static int inum(const char *s, const char *opt) {
     char *end;
     long v;
     errno = 0;
     v = strtol(s, &end, 10);
     if (errno || end == s || *end != '\0') die("invalid value for %s: %s", opt, s);
     return (int) v;
}

/* split a list at commas, spaces or newlines into *out (malloc'd, strdup'd) */
static int split_list(const char *list, char ***out) {
     char *tmp = strdup(list), *save = NULL, *tok;
     int n = 0, cap = 8;
     char **v = malloc(cap * sizeof(char *));
     for (tok = strtok_r(tmp, " \n,", &save); tok; tok = strtok_r(NULL, " \n,", &save)) {
          if (n == cap) v = realloc(v, (cap *= 2) * sizeof(char *));
          v[n++] = strdup(tok);
     }
     free(tmp);
     *out = v;
     return n;
}

/* one entry per derivative: strings */
static char **deriv_names(int n_derivs, const char *opt, const char *list) {
     char **v;
     int n;
     if (n_derivs <= 0) die("Must specifiy -derivs <n_derivs> option before %s%s", opt, "");
     n = split_list(list, &v);
     if (n != n_derivs) {
          fprintf(stderr, "ERROR: Number of values in %s list is not consistent with the specified "
                  "number of derivs: %d\n", opt, n_derivs);
          exit(1);
     }
     return v;
}

/* one entry per derivative: numbers */
static double *deriv_values(int n_derivs, const char *opt, const char *list) {
     char **s = deriv_names(n_derivs, opt, list);
     double *v = malloc(n_derivs * sizeof(double));
     int i;
     for (i = 0; i < n_derivs; ++i) {
          v[i] = num(s[i], opt);
          free(s[i]);
     }
     free(s);
     return v;
}

/* which of (a1, a2, a3, a4, a5, r1, r2) a distribution takes, in command-line
 * order; mono's single value is both a1 and the radius range */
static const char *dist_slots(enum size_dist_type t) {
     switch (t) {
          case SIZE_DIST_MONO:                        return "0";
          case SIZE_DIST_MODIFIED_GAMMA:              return "01256";
          case SIZE_DIST_LOG_NORMAL:                  return "0156";
          case SIZE_DIST_POWER_LAW:                   return "01";
          case SIZE_DIST_GAMMA:                       return "0156";
          case SIZE_DIST_MODIFIED_POWER_LAW:          return "056";
          case SIZE_DIST_MODIFIED_BIMODAL_LOG_NORMAL: return "0123456";
          case SIZE_DIST_EXPONENTIAL:                 return "056";
          default:                                    return NULL;
     }
}

typedef struct {
     /* inputs */
     enum size_dist_type dist;
     int have_dist, have_lambda, have_m, have_int1, have_int2, have_quad;
     int n_int1, n_int2, n_quad, n_angles, n_derivs, n_threads, n_timing;
     int verbose, save_dist, check_cbak, check_g, timing;
     double lambda, mr, mi, p[7], accuracy, tol_cbak, tol_g;
     double *lambda_l, *mr_l, *mi_l, *p_l[7];
     /* outputs: file names (value, then one per derivative) */
     const char *fn[4];
     char **fn_l[4];
} cli;

enum { OUT_TOTAL, OUT_GC, OUT_LC, OUT_PF };

static void usage(void) {
     printf("%s <flags ...>\n\n", TOOL);
     printf("Flags as for LMie's calllmie: -dist, -lambda, -m, -n_int1, -n_int2, -n_quad,\n"
            "-n_angles, -accuracy, -derivs, -lambda_l, -m_l, -dist_l, -total, -gc, -lc, -pf,\n"
            "-check_cbak, -check_g, -save_dist, -n_threads, -timing, -verbose, -help, -version.\n");
}

static void parse(cli *c, int argc, char **argv) {
     static const char *outs[4] = {"-total", "-gc", "-lc", "-pf"};
     double *zeros = NULL;
     int i, k;
     for (i = 1; i < argc; ++i) {
          const char *a = argv[i];
          if (a[0] != '-') {
               printf("Too many arguments, use -help for more information\n");
               exit(1);
          }
          for (k = 0; k < 4; ++k)
               if (strcmp(a, outs[k]) == 0) break;
          if (k < 4) {
               need(i, argc, c->n_derivs > 0 ? 2 : 1, a);
               c->fn[k] = argv[++i];
               if (c->n_derivs > 0) c->fn_l[k] = deriv_names(c->n_derivs, a, argv[++i]);
          } else if (strcmp(a, "-accuracy") == 0) {
               need(i, argc, 1, a);
               c->accuracy = num(argv[++i], a);
          } else if (strcmp(a, "-check_cbak") == 0) {
               need(i, argc, 1, a);
               c->check_cbak = 1;
               c->tol_cbak = num(argv[++i], a);
          } else if (strcmp(a, "-check_g") == 0) {
               need(i, argc, 1, a);
               c->check_g = 1;
               c->tol_g = num(argv[++i], a);
          } else if (strcmp(a, "-derivs") == 0) {
               need(i, argc, 1, a);
               c->n_derivs = inum(argv[++i], a);
               if (c->n_derivs < 0) die("invalid value for %s: %s", a, argv[i]);
               zeros = calloc(c->n_derivs > 0 ? c->n_derivs : 1, sizeof(double));
               c->lambda_l = c->mr_l = c->mi_l = zeros;
               for (k = 0; k < 7; ++k) c->p_l[k] = zeros;
          } else if (strcmp(a, "-findif") == 0) {
               /* accepted for compatibility; the reference ignores its value too */
               need(i, argc, 1, a);
               ++i;
          } else if (strcmp(a, "-dist") == 0) {
               const char *slots;
               int s;
               need(i, argc, 1, a);
               c->dist = size_dist_code(argv[++i]);
               if ((int) c->dist < 0) die("(-dist) invalid distribution name: %s%s", argv[i], "");
               c->have_dist = 1;
               slots = dist_slots(c->dist);
               if (!slots) continue;
               need(i, argc, (int) strlen(slots), a);
               for (s = 0; slots[s]; ++s) c->p[slots[s] - '0'] = num(argv[++i], a);
               if (c->dist == SIZE_DIST_MONO) c->p[5] = c->p[6] = c->p[0];
          } else if (strcmp(a, "-dist_l") == 0) {
               const char *slots;
               int s;
               if (!c->have_dist) die("must specify -dist before -dist_l%s%s", "", "");
               slots = dist_slots(c->dist);
               if (!slots) die("(-dist) invalid distribution type: %s%s", size_dist_name(c->dist), "");
               need(i, argc, (int) strlen(slots), a);
               for (s = 0; slots[s]; ++s) c->p_l[slots[s] - '0'] = deriv_values(c->n_derivs, a, argv[++i]);
          } else if (strcmp(a, "-help") == 0) {
               usage();
               exit(0);
          } else if (strcmp(a, "-lambda") == 0) {
               need(i, argc, 1, a);
               c->have_lambda = 1;
               c->lambda = num(argv[++i], a);
          } else if (strcmp(a, "-lambda_l") == 0) {
               need(i, argc, 1, a);
               c->lambda_l = deriv_values(c->n_derivs, a, argv[++i]);
          } else if (strcmp(a, "-m") == 0) {
               need(i, argc, 2, a);
               c->have_m = 1;
               c->mr = num(argv[++i], a);
               c->mi = num(argv[++i], a);
          } else if (strcmp(a, "-m_l") == 0) {
               need(i, argc, 2, a);
               c->mr_l = deriv_values(c->n_derivs, a, argv[++i]);
               c->mi_l = deriv_values(c->n_derivs, a, argv[++i]);
          } else if (strcmp(a, "-n_int1") == 0) {
               need(i, argc, 1, a);
               c->have_int1 = 1;
               c->n_int1 = inum(argv[++i], a);
          } else if (strcmp(a, "-n_int2") == 0) {
               need(i, argc, 1, a);
               c->have_int2 = 1;
               c->n_int2 = inum(argv[++i], a);
          } else if (strcmp(a, "-n_quad") == 0) {
               need(i, argc, 1, a);
               c->have_quad = 1;
               c->n_quad = inum(argv[++i], a);
          } else if (strcmp(a, "-n_angles") == 0) {
               need(i, argc, 1, a);
               c->n_angles = inum(argv[++i], a);
          } else if (strcmp(a, "-n_threads") == 0) {
               need(i, argc, 1, a);
               c->n_threads = inum(argv[++i], a);
          } else if (strcmp(a, "-timing") == 0) {
               need(i, argc, 1, a);
               c->timing = 1;
               c->n_timing = inum(argv[++i], a);
          } else if (strcmp(a, "-save_dist") == 0) {
               c->save_dist = 1;
          } else if (strcmp(a, "-verbose") == 0) {
               c->verbose = 1;
          } else if (strcmp(a, "-version") == 0) {
               printf("%s version %s\n", TOOL, TOOL_VERSION);
               exit(0);
          } else {
               printf("Invalid option: %s, use -help for more information\n", a);
               exit(1);
          }
     }
     if (!c->have_dist) die("must specify a size distribution with -dist%s%s", "", "");
     if (!c->have_lambda) die("must specify the wavelength with -lambda%s%s", "", "");
     if (!c->have_m) die("must specify the index of refraction with -m%s%s", "", "");
     if (c->dist == SIZE_DIST_MODIFIED_POWER_LAW && !c->have_int1)
          die("must specify the # of integration subintervals from r0 to r1 with -n_int1%s%s", "", "");
     if (!c->have_int2) die("must specify the # of integration subintervals from r1 to r2 with -n_int2%s%s", "", "");
     if (!c->have_quad) die("must specify the # of quadrature points on each interval with -n_quad%s%s", "", "");
     if (c->check_cbak && !c->fn[OUT_PF]) die("must use -pf when using -check_cbak%s%s", "", "");
     if (c->check_g && !c->fn[OUT_PF]) die("must use -pf when using -check_g%s%s", "", "");
}

/* the text header of misc/rtutil_scat_io.c:250-289: inputs, then integrated
 * quantities (value or one derivative) */
static int write_header(FILE *fp, const cli *c, int d, const lmie_out_data *o) {
     const int v = d < 0;
     const double lam = v ? c->lambda : c->lambda_l[d], mr = v ? c->mr : c->mr_l[d], mi = v ? c->mi : c->mi_l[d];
     double p[5];
     int k;
     for (k = 0; k < 5; ++k) p[k] = v ? c->p[k] : c->p_l[k][d];
     if (fprintf(fp, "lambda    = %e\n", lam) < 1) return -1;
     fprintf(fp, "mr        = %e\n", mr);
     fprintf(fp, "mi        = %e\n", mi);
     fprintf(fp, "dist_type = %s\n", size_dist_name(c->dist));
     fprintf(fp, "a1        = %e\n", p[0]);
     fprintf(fp, "a2        = %e\n", p[1]);
     fprintf(fp, "a3        = %e\n", p[2]);
     fprintf(fp, "a4        = %e\n", p[3]);
     fprintf(fp, "a5        = %e\n", p[4]);
     fprintf(fp, "r1        = %e\n", v ? o->r1 : o->r1_l[d]);
     fprintf(fp, "r2        = %e\n", v ? o->r2 : o->r2_l[d]);
     fprintf(fp, "n_int1    = %d\n", c->n_int1);
     fprintf(fp, "n_int2    = %d\n", c->n_int2);
     fprintf(fp, "n_quad    = %d\n", c->n_quad);
     fprintf(fp, "norm      = %e\n", v ? o->norm : o->norm_l[d]);
     fprintf(fp, "reff      = %e\n", v ? o->reff : o->reff_l[d]);
     fprintf(fp, "veff      = %e\n", v ? o->veff : o->veff_l[d]);
     fprintf(fp, "gavg      = %e\n", v ? o->gavg : o->gavg_l[d]);
     fprintf(fp, "vavg      = %e\n", v ? o->vavg : o->vavg_l[d]);
     fprintf(fp, "ravg      = %e\n", v ? o->ravg : o->ravg_l[d]);
     fprintf(fp, "rvw       = %e\n", v ? o->rvw : o->rvw_l[d]);
     fprintf(fp, "cext      = %e\n", v ? o->cext : o->cext_l[d]);
     fprintf(fp, "csca      = %e\n", v ? o->csca : o->csca_l[d]);
     fprintf(fp, "cbak      = %e\n", v ? o->cbak : o->cbak_l[d]);
     if (fprintf(fp, "g         = %e\n", v ? o->g : o->g_l[d]) < 1) return -1;
     return 0;
}

/* one output file (kind k) for the value (d < 0) or derivative d */
static void write_output(const cli *c, int k, int d, const lmie_out_data *o) {
     const char *fn = d < 0 ? c->fn[k] : c->fn_l[k][d];
     FILE *fp = fn[0] == '-' ? stdout : fopen(fn, "w");
     int i, bad;
     if (!fp) {
          fprintf(stderr, "ERROR: Error opening file for writing: %s ... %s\n", fn, strerror(errno));
          exit(1);
     }
     bad = write_header(fp, c, d, o);
     if (!bad && k == OUT_GC) {
          double **gc = d < 0 ? o->gc : o->gc_l[d];
          fprintf(fp, "%d\n", o->n_coef);
          for (i = 0; i < o->n_coef; ++i)
               fprintf(fp, "%e %e %e %e %e %e\n", gc[0][i], gc[1][i], gc[2][i], gc[3][i], gc[4][i], gc[5][i]);
     } else if (!bad && k == OUT_LC) {
          double **lc = d < 0 ? o->lc : o->lc_l[d];
          fprintf(fp, "%d\n", o->n_coef);
          for (i = 0; i < o->n_coef; ++i)
               fprintf(fp, "%e %e %e %e %e %e\n", lc[0][i], lc[1][i], lc[2][i], lc[3][i], lc[4][i], lc[5][i]);
     } else if (!bad && k == OUT_PF) {
          double **pf = d < 0 ? o->pf : o->pf_l[d];
          fprintf(fp, "%d\n", c->n_angles);
          for (i = 0; i < c->n_angles; ++i)
               fprintf(fp, "%e %e %e %e %e %e %e\n", o->theta[i], pf[0][i], pf[1][i], pf[2][i], pf[3][i],
                       pf[4][i], pf[5][i]);
     }
     if (bad || ferror(fp)) {
          fprintf(stderr, "ERROR: Problem writing to file: %s\n", fn);
          exit(1);
     }
     if (fp != stdout) fclose(fp);
     else fflush(fp);
}

static double now_s(void) {
     struct timespec t;
     clock_gettime(CLOCK_MONOTONIC, &t);
     return (double) t.tv_sec + 1e-9 * (double) t.tv_nsec;
}

int main(int argc, char **argv) {
     cli c;
     lmie_in_data in;
     lmie_out_data out;
     int i, k;
     double t0 = 0., t1 = 0.;

     memset(&c, 0, sizeof(c));
     c.n_angles = 18001;
     c.n_threads = 1;
     c.n_timing = 1;
     c.accuracy = 1e-7;
     c.tol_cbak = 1e-5;
     c.tol_g = 1e-5;
     parse(&c, argc, argv);

     if (lmie_in_alloc(&in, c.n_derivs)) die("lmie_in_alloc()%s%s", "", "");
     in.save_control = c.save_dist ? 1 : 0;
     in.calc_gc = c.fn[OUT_GC] || c.fn[OUT_PF];
     in.calc_lc = c.fn[OUT_LC] != NULL;
     in.calc_pf = c.fn[OUT_PF] != NULL;
     in.dist_type = c.dist;
     in.n_int1 = c.n_int1;
     in.n_int2 = c.n_int2;
     in.n_quad = c.n_quad;
     in.n_angles = c.n_angles;
     in.n_derivs = c.n_derivs;
     in.lambda = c.lambda;
     in.mr = c.mr;
     in.mi = c.mi;
     in.a1 = c.p[0];
     in.a2 = c.p[1];
     in.a3 = c.p[2];
     in.a4 = c.p[3];
     in.a5 = c.p[4];
     in.r1 = c.p[5];
     in.r2 = c.p[6];
     for (i = 0; i < c.n_derivs; ++i) {
          in.lambda_l[i] = c.lambda_l[i];
          in.mr_l[i] = c.mr_l[i];
          in.mi_l[i] = c.mi_l[i];
          in.a1_l[i] = c.p_l[0][i];
          in.a2_l[i] = c.p_l[1][i];
          in.a3_l[i] = c.p_l[2][i];
          in.a4_l[i] = c.p_l[3][i];
          in.a5_l[i] = c.p_l[4][i];
          in.r1_l[i] = c.p_l[5][i];
          in.r2_l[i] = c.p_l[6][i];
     }
     in.accuracy = c.accuracy;

     if (lmie_solution(&in, &out, 1, c.verbose, c.n_threads, 0)) die("lmie_solution()%s%s", "", "");

     if (c.save_dist) {
          /* second solve from the saved per-radius quantities into the same
           * arrays (the reference clears them to -999 first) */
          const int max_coef = lmie_calc_max_coef(in.lambda, in.dist_type, in.a1, in.a2, in.a3, in.r1, in.r2);
          in.save_control = 2;
          if (in.calc_gc)
               for (i = 0; i < 6 * max_coef; ++i) out.gc[0][i] = -999.;
          if (in.calc_lc)
               for (i = 0; i < 6 * max_coef; ++i) out.lc[0][i] = -999.;
          if (in.calc_pf)
               for (i = 0; i < 6 * c.n_angles; ++i) out.pf[0][i] = -999.;
          if (lmie_solution(&in, &out, 0, c.verbose, c.n_threads, 0)) die("lmie_solution()%s%s", "", "");
     }

     if (c.timing) {
          /* timed: full solves (save_control 0), each into fresh arrays */
          lmie_out_data tmp;
          in.save_control = 0;
          t0 = now_s();
          for (i = 0; i < c.n_timing; ++i) {
               if (lmie_solution(&in, &tmp, 1, c.verbose, c.n_threads, 0)) die("lmie_solution()%s%s", "", "");
               lmie_out_free(&tmp, c.n_derivs > 0);
          }
          t1 = now_s();
     }

     if (c.check_cbak) {
          const double cbak2 = out.pf[0][c.n_angles - 1] * out.csca / (4. * M_PI);
          if (fabs(out.cbak - cbak2) > c.tol_cbak) {
               fprintf(stderr, "ERROR: check_cbak failed: cbak = %.6e and pf[0][n_angles - 1] * csca / (4. * PI) = "
                       "%.6e\n", out.cbak, cbak2);
               exit(1);
          }
     }
     if (c.check_g) {
          const double g2 = (in.calc_gc ? out.gc[0][1] : out.lc[0][1]) / 3.;
          if (fabs(out.g - g2) > c.tol_g) {
               fprintf(stderr, "ERROR: check_g failed: g = %.6e and gc[0][1] / 3. = %.6e\n", out.g, g2);
               exit(1);
          }
     }

     for (k = 0; k < 4; ++k)
          if (c.fn[k]) write_output(&c, k, -1, &out);
     for (i = 0; i < c.n_derivs; ++i)
          for (k = 0; k < 4; ++k)
               if (c.fn[k]) write_output(&c, k, i, &out);

     if (c.timing) printf("%.2f\n", t1 - t0);

     lmie_in_free(&in, c.n_derivs > 0);
     lmie_out_free(&out, c.n_derivs > 0);
     return 0;
}
