/*
 * lmie_interface.h -- drop-in C interface of the B200 polydisperse Mie solver.
 *
 * Existing LMie callers (C, and Fortran 77/90 through the `_` shims) compile
 * against this header and link liblmie_b200.so instead of liblmie.a.  The two
 * structs below keep the field order and types of the reference structs byte
 * for byte, because callers fill and read them directly:
 *   lmie_in_data   <- reference src/lmie_interface.h:20-57
 *   lmie_out_data  <- reference src/lmie_interface.h:60-101
 * and every prototype keeps the reference signature and meaning:
 *   lmie_calc_max_coef  <- src/lmie_interface.h:104-105 (impl. src/lmie_interface.c:24-31)
 *   lmie_in_alloc/free  <- src/lmie_interface.h:107-108 (impl. src/lmie_interface.c:38-72)
 *   lmie_out_alloc/free <- src/lmie_interface.h:109-110 (impl. src/lmie_interface.c:79-169)
 *   lmie_in_zero_derivs <- src/lmie_interface.h:112     (impl. src/lmie_interface.c:176-192)
 *   lmie_solution       <- src/lmie_interface.h:114-115 (impl. src/lmie_interface.c:199-250)
 *   lmie_solution2      <- src/lmie_interface.h:117-133 (impl. src/lmie_interface.c:257-297)
 *   lmie_solution2_l    <- src/lmie_interface.h:135-155 (impl. src/lmie_interface.c:360-507)
 *   lmie_solution_slave <- src/lmie_interface.h:157     (impl. src/lmie_interface.c:514-526)
 *   size_dist_code/name <- misc/rtutil_support.h:54-56  (impl. misc/rtutil_support.c:508-535)
 *   enum size_dist_type <- misc/rtutil_size_dist.h:22-34 (numeric order is ABI)
 *
 * Return convention (reference src/lmie_interface.c:212-214,244-246): 0 on
 * success, -1 on failure with an "ERROR: ..." line on stderr.  There is no CPU
 * fallback: when no usable sm_100 GPU is present the solve returns -1.
 *
 * Output arrays are "row-pointer" arrays: one malloc block holding the row
 * pointer table followed by the contiguous data (reference
 * misc/gutil_alloc.c:18-70,214-226), so gc[0] points at all 6*max_coef
 * doubles and free(gc) releases everything.
 */
#ifndef LMIE_INTERFACE_H
#define LMIE_INTERFACE_H

#ifdef __cplusplus
extern "C" {
#endif

#ifndef LMIE_SIZE_DIST_TYPE_DEFINED
#define LMIE_SIZE_DIST_TYPE_DEFINED
#define SIZE_DIST_MAX_PARAMS 5

enum size_dist_type {
     SIZE_DIST_NONE,
     SIZE_DIST_MODIFIED_GAMMA,
     SIZE_DIST_LOG_NORMAL,
     SIZE_DIST_POWER_LAW,
     SIZE_DIST_GAMMA,
     SIZE_DIST_MODIFIED_POWER_LAW,
     SIZE_DIST_MODIFIED_BIMODAL_LOG_NORMAL,
     SIZE_DIST_EXPONENTIAL,
     SIZE_DIST_MONO,

     N_SIZE_DIST_TYPES
};
#endif

typedef struct {
     int save_control;          /* 0: normal, 1: also return save1/save2, 2: re-weight save1/save2 */

     int calc_gc;               /* generalized-spherical-function coefficients */
     int calc_lc;               /* Legendre coefficients */
     int calc_pf;               /* phase matrix at n_angles uniform angles */

     enum size_dist_type dist_type;

     int n_int1;
     int n_int2;
     int n_quad;
     int n_angles;
     int n_derivs;

     double lambda;
     double mr;                 /* m = mr - i*mi, mi >= 0 */
     double mi;
     double a1;
     double a2;
     double a3;
     double a4;
     double a5;
     double r1;
     double r2;

     double *lambda_l;
     double *mr_l;
     double *mi_l;
     double *a1_l;
     double *a2_l;
     double *a3_l;
     double *a4_l;
     double *a5_l;
     double *r1_l;
     double *r2_l;

     double accuracy;
} lmie_in_data;


typedef struct {
     int n_coef;

     double r1;
     double r2;
     double norm;
     double reff;
     double veff;
     double gavg;
     double vavg;
     double ravg;
     double rvw;
     double cext;
     double csca;
     double cbak;
     double g;
     double **gc;               /* [6][max_coef] */
     double **lc;               /* [6][max_coef] */
     double *theta;             /* [n_angles] */
     double **pf;               /* [6][n_angles] */

     double *r1_l;
     double *r2_l;
     double *norm_l;
     double *reff_l;
     double *veff_l;
     double *gavg_l;
     double *vavg_l;
     double *ravg_l;
     double *rvw_l;
     double *cext_l;
     double *csca_l;
     double *cbak_l;
     double *g_l;
     double ***gc_l;            /* [n_derivs][6][max_coef] */
     double ***lc_l;            /* [n_derivs][6][max_coef] */
     double ***pf_l;            /* [n_derivs][6][n_angles] */

     double **save1;            /* [4][n_qsize]          (save_control 1/2) */
     double ***save2;           /* [4][n_qsize][n_qang]  (save_control 1/2) */
} lmie_out_data;


int lmie_calc_max_coef(double lambda, enum size_dist_type dist_type,
                       double a1, double a2, double a3, double r1, double r2);

int lmie_in_alloc(lmie_in_data *in, int n_derivs);
void lmie_in_free(lmie_in_data *in, int flag);
int lmie_out_alloc(lmie_in_data *in, lmie_out_data *out, int max_coef);
void lmie_out_free(lmie_out_data *out, int flag);

void lmie_in_zero_derivs(lmie_in_data *in, int n_derivs);

int lmie_solution(lmie_in_data *in, lmie_out_data *out, int alloc_out, int verbose,
                  int n_threads, int use_mpi);

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
                   int verbose, int n_threads, int use_mpi);

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
                     int verbose, int n_threads, int use_mpi);

/* MPI worker loop of the reference.  This library has no MPI: it prints an
 * ERROR line and returns -1 (multi-device work goes through
 * lmie_solution_batch on one process per GPU instead). */
int lmie_solution_slave(void);

/* Size distribution name <-> code (reference misc/rtutil_support.c:508-535).
 * size_dist_code returns -1 for an unknown name, size_dist_name NULL for an
 * unknown code; both print an ERROR line. */
enum size_dist_type size_dist_code(const char *name);
const char *size_dist_name(enum size_dist_type code);

/* Fortran-facing shims (all arguments by reference; max_coef is the leading
 * dimension of gc/lc in the caller's column-major arrays) -- reference
 * interfaces/lmie_int_util.c:21-61,72-241. */
int size_dist_code_(char *name);
int lmie_calc_max_coef_(double *lambda, enum size_dist_type *dist_type,
                        double *a1, double *a2, double *a3, double *r1, double *r2);
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
                    int *max_coef, int *verbose, int *n_threads, int *use_mpi);
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
                      int *max_coef, int *verbose, int *n_threads, int *use_mpi);

#ifdef __cplusplus
}
#endif

#endif /* LMIE_INTERFACE_H */
