// kernels.h -- launch interface of the FP64 kernels of liblmie_b200
// (k_fp64.cu), used by the driver (driver.cu).
//
// Every kernel works on a batch of independent polydisperse cases: all radii
// of all cases form one list, and a device case table gives each case its
// parameters and its offsets into the concatenated arrays.  A single
// lmie_solution() is a batch of one.
#pragma once

#include "dev_common.cuh"

// limit of every bounded wait of the tensor-core kernels (~1 s at 1.96 GHz), in SM clock cycles
constexpr long long LMIEB_WAIT_CYCLES = 1LL << 31;

// One contiguous copy of a sub-batch whose coefficients were computed by an
// earlier sub-batch: n doubles from src (that sub-batch's arena) to the
// coefficient columns (which = 0) or per-radius sums (which = 1) at dst_off.
struct GatherSeg {
    const double *src;
    long long dst_off, n;
    int which;
};
// K1 keeps its downward recurrences at the top of every block of K1_B orders
// and replays a block into per-thread arrays of K1_B entries: with 8 they stay
// in L1 at four blocks of 64 threads per SM (16: 3.9 ms of K1 on the
// 4096-case batch, 8: 3.7 ms, 4: 3.7 ms).
constexpr int K1_B = 8;
// doubles per checkpoint block of a chunk of nc tangent-linear columns
__host__ __device__ constexpr int k1_ck_width(int nc) { return 3 + 3 * nc; }

// One case of a batch (device copy).  Offsets index the batch-wide arrays.
struct DevCase {
    double lambda;
    cplx m, minv;
    double accuracy;            // expansion truncation threshold
    int r0, nr;                 // radius range [r0, r0 + nr) in the batch lists
    long long o0;               // its first order in the coefficient columns (sum of n1 of the radii before)
    int n1, n_qang, nh, n_coef, n_angles;
    int ml_off;                 // m_l / lambda_l of this case at [ml_off, ml_off + nd)
    long long mu_off;           // Gauss nodes/weights in the node pool
    long long pf_off;           // [Q][n_qang] block in pfacc / pfn (Q = 4 (1 + nd))
    long long part_off;         // [G][Q][n_qang] block of angular partials
    long long ck_off;           // recurrence checkpoints of the expansion
    long long ex_off;           // [n_atile][ncol][6][n_coef] expansion partials
    long long gc_off, lc_off;   // [ncol][6][n_coef] outputs
    long long pf_out_off;       // [ncol][6][n_angles] output (user angles)
    long long mu_user_off;      // user-angle cosines
    int pu_parts;               // K5: parts of pu_lp orders (each angle tile's blocks)
    long long pu_scr_off;       // K5 with more than one part: its [part][ncol][6][n_angles] partial sums
    int scal_off;               // [ncol][4] normalised cross sections and g
    int G;                      // angular radius groups
    int nkx;                    // int8 K3: chunks of OZ_KC orders its row exponents cover
    long long rx_off;           // int8 K3: its row exponents ([nh][nkx][2] bytes)
    long long a_off;            // int8 K3: its A operand digits ([tile][nkx][OZ_AROW / 16 pieces][OZ_M rows][16 bytes])
    double trunc_band;          // > 0: K4 records where |beta_l| comes within trunc_band (2l + 1)
                                // of `accuracy` (band[2c], band[2c + 1]; see launch_expand)
};

struct DevBatch {
    int ncase;
    int R;                      // radii over all cases
    int nd, nd1, nd2;           // derivative layout (uniform over the batch)
    int n1max, ncmax;           // largest n1 and n_coef (table lengths)
    int pu_lp;                  // K5: orders per block (a multiple of PU_T)
    const DevCase *cs;          // [ncase]
    const int *idx1, *idx2;     // [nd1], [nd2]
    const cplx *m_l;            // [ncase * nd]
    const double *lambda_l;     // [ncase * nd]
    const int *rcase;           // [R] case of each radius
    const int *k1ord;           // [ncase] K1's order of the cases (largest n1 first)
    const long long *k1pre;     // [ncase + 1] radii of the cases before each in that order
    const double *x;            // [R] size parameters
    const double *xl;           // [nd1][R] d x / d p for index1 slot k
    const double *w;            // [(1 + nd)][R] row 0: f = nr qw; row 1+kk: f_l (index1) or f_l2 (index2)
    const int *n1r, *n2r;       // [R]
    const long long *off;       // [R+1] prefix sums of n1r (coefficient storage)
    const long long *ckoff;     // [R+1] prefix sums of ceil(n1r / K1_B) (K1 checkpoint blocks)
    long long tot, ckn;
    const double *fv;           // [4][n1max + 2]: fv1 | fv2 | fv3 | fv4
    const double *rc;           // [8 * ncmax] GSF/Legendre recurrence coefficients per order
    const double *mu_pool;      // Gauss pool: n nodes then n weights at DevCase.mu_off
    const double *mu_user;      // user-angle cosines (DevCase.mu_user_off)
    // split-precision K3 (tc_layout.cuh); null in the FP64 form
    const int *tc_pos;          // [R] position of the radius in its group + 256 * the group's chunks
                                //     (-1: the radius' case keeps the FP64 angular stage)
    const long long *tc_roff;   // [R] float offset of the radius' group in the B operand
    const int *tg_r0, *tg_n, *tg_nk;   // per group: first radius, radii, chunks of TC_KC orders
    const long long *tg_off;    // per group: float offset of its B operand block (int8 K3: byte offset)
    // int8 fixed-point K3 (oz_layout.cuh); null in the other forms
    const double *oz_f2;        // [OZ_KC * max chunks + 2]: (k + 1) / k
    const signed char *oz_rowexp;   // row exponents (DevCase.rx_off)
    const int *oz_colexp;       // [group][OZ_NP] column exponents
    const unsigned char *oz_aop;   // A operand digits of every angle tile (DevCase.a_off)
    int *oz_radexp;             // [1 + nd1][R][4]: per radius, coefficient column and component, the
                                //     largest (biased exponent + e_k) over the orders, 0 if no normal
                                //     value (written by K1)
};

// Coefficient columns: column 0 = value, column 1+k = index1 slot k.  Entry
// (col, off[r] + j - 1) holds {Re cs, Im cs, Re cd, Im cd} with
// cs = fv4_j (a_j + b_j), cd = fv4_j (a_j - b_j).
// Per-radius sums rs[(col*5 + q)*R + r], q: se, ss, Re sb, Im sb, sg.

// Gauss-Legendre nodes of npairs root pairs: pair p belongs to order
// n = ns[pt[p]] and is root pi[p]; that order's n nodes and then n weights
// start at pool + mo[pt[p]], its host starting points at guess + go[pt[p]].
int launch_gauss(cudaStream_t s, int npairs, const int *pt, const int *pi, const int *ns,
                 const long long *mo, const long long *go, const double *guess, const double *jr,
                 double *pool);

// K1 for one chunk of nc tangent-linear columns starting at index1 slot c0.
// With bop set, the coefficients go to the tensor-core B operand
// (tc_layout.cuh) instead of coef.
int launch_coef(cudaStream_t s, const DevBatch &B, int nc, int c0, int write_value, double *ck, double *coef,
                float *bop, double *rs);

// K2: sums[case][(1+nd)][4] (unnormalised), save1 [4][R] for save_control 1
int launch_reduce_scalars(cudaStream_t s, const DevBatch &B, const double *rs, double *sums, double *save1);

// K3 work item: one block of half-angles of one case over a radius range.
struct AngItem {
    int c, xt, g, rbeg, rend;
};
int angular_angles_per_block(int nc1);
int launch_angular(cudaStream_t s, const DevBatch &B, int nc1, int c1base, int nc2, int c2base, int first,
                   int nitems, const AngItem *items, const double *coef, double *part, double *save2);
// K3 in split precision on the tensor cores (k_tc.cu).  An item is one case
// (c), 64 half-angles (xt), a partial slot (g) and the radius groups
// [rbeg, rend).  err is set when a block gave up waiting.
int launch_angular_tc(cudaStream_t s, const DevBatch &B, int nitems, const AngItem *items, const float *bop,
                      double *part, int seg, int *err);
// D[128 x 240] = A[128 x K] B[240 x K]^T through the same tensor-core path
int launch_tc_selftest(cudaStream_t s, int K, const double *A, const double *Bm, double *D, int *err);
// K3 as an exact fixed-point contraction on the int8 tensor cores (k_oz.cu):
// the row exponents (thread per (case, half-angle) of the flat index space
// row_start), the A operand digits (thread per product row of every angle
// tile, arow_start) and the B operand digits and column exponents (block per
// radius group) from K1's FP64 coefficient columns, then the products; items
// as for launch_angular_tc.
int launch_oz_operands(cudaStream_t s, const DevBatch &B, long long nrow, const long long *row_start,
                       signed char *rowexp, long long narow, const long long *arow_start, unsigned char *aop,
                       int ngroups, const double *coef, unsigned char *bop, int *colexp);
int launch_angular_oz(cudaStream_t s, const DevBatch &B, int nitems, const AngItem *items, const unsigned char *bop,
                      double *part, int *err);
// D[128 x OZ_NP] = A[128 x K] B[OZ_NP x K]^T through the same fixed-point path
// *err = 2 if the radius group's failure count *failed is not zero
int launch_group_flag(cudaStream_t s, const double *failed, int *err);
int launch_oz_selftest(cudaStream_t s, int K, const double *A, const double *Bm, double *D, int *err,
                       long long wait_cycles, int withhold);
// per-case element lists: element e of the flat index space belongs to the
// case c with start[c] <= e < start[c+1] (start has ncase + 1 entries)
int launch_reduce_pf(cudaStream_t s, const DevBatch &B, long long total, const long long *start,
                     const double *part, double *pfacc);
// save_control 2, batch of one case with n_qang angles
int launch_save_reweight(cudaStream_t s, const DevBatch &B, int n_qang, const double *save1,
                         const double *save2, const double *w2, double *sums, double *pfacc);
int launch_normalize(cudaStream_t s, const DevBatch &B, long long total, const long long *start,
                     const double *sums, const double *pfacc, double *scal, double *pfn);

// K4: expansion over Gauss angles.  kind 0: GSF, 1: Legendre.  trunc[c] gets
// n_coef - l for the first l with |beta_l| <= accuracy (0: none); for cases
// with a truncation band d_l = C.trunc_band (2l + 1), band[2c] and band[2c+1]
// get n_coef - l for the first l with |beta_l| <= accuracy + d_l and
// <= accuracy - d_l.
constexpr int PU_LP = 256;     // default orders per K5 block (a multiple of PU_T)
constexpr int PU_T = 64;       // user angles per K5 block (and orders staged per step)
constexpr int EX_LT = 32;       // orders per tile
constexpr int EX_AT = 32;       // half-angles per tile
struct ExpItem {
    int c, lt, at;              // case, order tile, angle tile
};
// ck_start: flat (case, half-angle, function) checkpoint-thread index space;
// fin_start: flat (case, column, order) index space of the finalisation.
// runs: (case, 0, angle tile) items of the GSF expansion on the FP64 tensor
// cores, one block each over all the case's orders (used with kind 0 when the
// columns fit it, see expand_gsf_launches; else the items and checkpoints).
// K1's outputs (coefficient columns, per-radius sums) copied in instead of
// computed: one block per segment
int launch_gather(cudaStream_t s, int nseg, const GatherSeg *segs, double *coef, double *rs);
int launch_expand(cudaStream_t s, const DevBatch &B, int kind, long long nck,
                  const long long *ck_start, int nitems, const ExpItem *items, int nruns, const ExpItem *runs,
                  long long nfin, const long long *fin_start, const double *pfn, double *ckpt, double *exq,
                  double *coefs, int *trunc, int *band);
// kernels the GSF expansion launches before its finalisation for ncol columns
int expand_gsf_launches(int ncol);

// K5: block per (case, tile of PU_T user angles, part of B.pu_lp orders),
// cases in K1's launch order (start: the blocks before each case in that
// order); cases of several parts add them up from scr (red_start: flat
// (case, column, element, angle) index space of those cases).
int launch_phase_user(cudaStream_t s, const DevBatch &B, int kind, long long total, const long long *start,
                      const double *coefs, const int *trunc, double *pf_out, double *scr, long long nred,
                      const long long *red_start);
