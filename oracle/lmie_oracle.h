/*
 * lmie_oracle.h -- CPU FP64 restatement of LMie's polydisperse Mie solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker that tests/, the smoke test
 * and the CPU-baseline leg of bench.py compare the CUDA product against.  The
 * product (lmie_b200/) never links, loads or calls it.
 *
 * Parity is pinned: tests/test_oracle_pins.py checks this restatement against
 * (a) the reference's golden output examples/example.out (7 significant
 * digits, committed as tests/golden/example_out.npz) and (b) full-precision
 * outputs of the reference library itself, compiled from the reference
 * sources by `make -C oracle ref` (committed as tests/golden/ref_*.npz by
 * tests/golden/make_golden.py).
 *
 * The structs are the public ones of include/lmie_interface.h (same byte
 * layout as the reference's src/lmie_interface.h:20-101).
 */
#ifndef LMIE_ORACLE_H
#define LMIE_ORACLE_H

#include "../include/lmie_interface.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Same contract as lmie_solution (reference src/lmie_interface.c:199-250),
 * single-threaded; n_threads/verbose/use_mpi do not exist here. */
int oracle_solution(lmie_in_data *in, lmie_out_data *out, int alloc_out);

/* Same as lmie_calc_max_coef (reference src/lmie_interface.c:24-31). */
int oracle_calc_max_coef(double lambda, enum size_dist_type dist_type,
                         double a1, double a2, double a3, double r1, double r2);

/* Frees what oracle_solution(alloc_out=1) allocated (reference
 * src/lmie_interface.c:129-169). */
void oracle_out_free(lmie_out_data *out, int flag);

/* Frees save1/save2 returned by save_control == 1. */
void oracle_free_save(lmie_out_data *out);

/* Size-distribution quadrature (reference misc/rtutil_size_dist.c:200-646):
 * fills qx, qw, nr [n] and, when n_derivs > 0, qx_l, qw_l, nr_l [n*n_derivs]
 * (row-major, radius-major) plus r1_out/r2_out (+_l) and norm (+_l).
 * Returns the number of radii or -1. */
int oracle_particle_dist(const lmie_in_data *in,
                         double *qx, double *qw, double *nr,
                         double *qx_l, double *qw_l, double *nr_l,
                         double *r1_out, double *r2_out,
                         double *r1_l_out, double *r2_l_out,
                         double *norm, double *norm_l);

/* Gauss-Legendre nodes/weights on [x1,x2] (reference
 * misc/rtutil_math.c:73-129,224-316). */
void oracle_gauss_leg(int n, double x1, double x2, double *x, double *w);

/* Truncation integers (reference src/lmie_core.c:18-38). */
int oracle_calc_n1(double x);
int oracle_calc_n2(int n1, double zr, double zi);

/* Per-radius Mie coefficients a_n, b_n (n = 1..n1), for unit tests of the
 * recurrences: writes 2*(n1) complex values as interleaved re/im doubles,
 * a first then b.  Returns n1. */
int oracle_mie_ab(double x, double mr, double mi, double *ab);

#ifdef __cplusplus
}
#endif

#endif
