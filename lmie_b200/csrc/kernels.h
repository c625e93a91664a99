// kernels.h -- launch interface of the FP64 kernels of liblmie_b200 (k_fp64.cu),
// used by the driver (driver.cu).
#pragma once

#include "dev_common.cuh"

// Device view of one polydisperse problem (all pointers are device memory).
struct DevProblem {
    int n;                      // radii
    int nd, nd1, nd2;
    int n1;                     // global truncation
    int n_qang, nh, n_coef;
    int n_angles;
    int save_control;
    double lambda;
    cplx m, minv, m2;
    const cplx *m_l;            // [nd]
    const double *lambda_l;     // [nd]
    const int *idx1, *idx2;     // [nd1], [nd2]
    const double *x;            // [n]
    const double *xl;           // [nd1*n]
    const double *w;            // [(1+nd)*n]
    const int *n1r, *n2r;       // [n]
    const long long *off;       // [n+1] prefix sums of n1r
    long long tot;              // off[n]
    const long long *offp;      // [n+1] prefix sums of n1r + 1 (orders 0..n1 per radius)
    long long totp;             // offp[n]
    int ntiles;                 // order tiles of K1b over all radii
    const double *fv;           // [4*(n1+2)]: fv1 | fv2 | fv3 | fv4
    const double *mu, *wq;      // [n_qang] Gauss nodes (ascending) and weights
    const double *gl_guess;     // [(n_qang+1)/2] Newton starting points for the nodes
    const double *gl_jr;        // [n_qang] j / (j + 1.) for the Legendre recurrence of the nodes
    const double *rc;           // [8*n_coef] per-order GSF/Legendre recurrence coefficients
};

// Coefficient columns: column 0 = value, column 1+k = index1 slot k.  Entry
// (col, off[r] + j - 1) holds {Re cs, Im cs, Re cd, Im cd} with
// cs = fv4_j (a_j + b_j), cd = fv4_j (a_j - b_j).
// Per-radius sums rs[(col*5 + q)*n + r], q: se, ss, Re sb, Im sb, sg.

// guess[i]: cos(t_i + da / tan t_i), t_i = (4i+3) pi / (4n+2), computed on the host
int launch_gauss(cudaStream_t s, int n, const double *guess, const double *jr, double *mu, double *wq);

// K1 for one chunk of nc tangent-linear columns starting at index1 slot c0:
// sequential recurrences into rec, then a_n/b_n tiles (tiles[i] = {radius,
// first order}) into coef and the tile partial sums rsp[(col*5+q)*ntiles + tile].
int launch_coef(cudaStream_t s, const DevProblem &P, int nc, int c0, int write_value, const int2 *tiles,
                double4 *rec, double *coef, double *rsp);
// rs[(col*5+q)*n + r] = sum of the tile partials of radius r (tiles tstart[r]..tstart[r+1]-1)
int launch_tile_reduce(cudaStream_t s, const DevProblem &P, const int *tstart, const double *rsp, double *rs);

int launch_reduce_scalars(cudaStream_t s, const DevProblem &P, const double *rs,
                          double *sums, double *save1);

int launch_angular(cudaStream_t s, const DevProblem &P, int nc1, int c1base, int nc2,
                   int c2base, int first, int n_groups, const int *gstart,
                   const double *coef, double *part, double *save2);

// half-angles one K3 block covers for a chunk of nc1 index1 columns
int angular_angles_per_block(int nc1);

int launch_reduce_pf(cudaStream_t s, const DevProblem &P, int n_groups, const double *part,
                     double *pfacc);

int launch_save_reweight(cudaStream_t s, const DevProblem &P, const double *save1,
                         const double *save2, const double *w2, double *sums, double *pfacc);

int launch_normalize(cudaStream_t s, const DevProblem &P, const double *sums,
                     const double *pfacc, double *scal_out, double *pfn);

// Expansion of the normalised phase matrix over Gauss angles.  kind 0: GSF
// (alpha/beta coefficients), kind 1: Legendre.
int launch_expand(cudaStream_t s, const DevProblem &P, int kind, int lchunk, double accuracy,
                  const double *pfn, double *state, double *tab, double *raw, double *coefs,
                  int *trunc);

int launch_phase_user(cudaStream_t s, const DevProblem &P, int kind, const double *coefs,
                      const int *trunc, const double *mu_user, double *pf_out);
