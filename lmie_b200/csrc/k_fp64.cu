// k_fp64.cu -- the FP64 kernels of the polydisperse solve (sm_100a), over a
// batch of independent cases (one lmie_solution() is a batch of one).
//
//   k_gauss          Gauss-Legendre angles on [-1,1]        <- misc/rtutil_math.c:73-129,231-316
//   k_mie<NC>        per radius: D_n, psi, chi recurrences (checkpointed
//                    downward sweeps, replayed per block), a_n, b_n, their
//                    tangent-linear forms, expansion coefficients and the
//                    per-radius sums                        <- src/lmie_core.c:263-652
//   k_reduce_scalars radius reduction of Cext/Csca/Cbak/g    <- src/lmie_core.c:537-611,
//                                                              src/lmie_schedule.c:334-338
//   k_angular<..>    S1/S2 accumulation over orders and the phase-matrix
//                    quadratic forms, reduced over a radius group
//                                                           <- src/lmie_core.c:658-791
//   k_reduce_pf      fixed-order sum over radius groups
//   k_normalize_*    2/Csca and lambda^2/2pi normalisation   <- src/lmie_schedule.c:1155-1199
//   k_exp_*          expansion coefficients over Gauss angles as a contraction
//                    over (order tile x angle tile), basis functions generated
//                    per tile from recurrence checkpoints  <- misc/rtutil_scat_int.c:20-230,353-480,
//                                                              misc/rtutil_math.c:477-513,936-1017
//   k_phase_user     phase matrix at the user's angles       <- misc/rtutil_scat_int.c:510-589,662-710
//
// All reductions run in a fixed order, so a solve is bit-reproducible.
#include <cstdio>

#include "kernels.h"
#include "tc_layout.cuh"

namespace {

// ---------------------------------------------------------------------------
// Gauss-Legendre nodes: one thread per root pair, Newton with the
// second-order correction of Davis & Rabinowitz.  The initial guesses come
// from the host (libm cos/tan) and every operation is an explicit
// round-to-nearest intrinsic (no FMA contraction), so the nodes are the
// reference's to the last bit -- at size parameters ~1000 the phase matrix
// changes by ~1e-10 per ulp of a node.
// ---------------------------------------------------------------------------
__global__ void k_gauss(int npairs, const int *__restrict__ pt, const int *__restrict__ pi,
                        const int *__restrict__ ns, const long long *__restrict__ mo,
                        const long long *__restrict__ go, const double *__restrict__ guess,
                        const double *__restrict__ jr, double *mu, double *wq) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    const int t = pt[p], i = pi[p], n = ns[t];
    const double dn = (double) n;
    const double ib = (double) (n * (n + 1));
    double y = guess[go[t] + i], y_prev, pn, pm, pmm, u, d1, d2;
    int it = 0;
    do {
        pm = 0.;
        pn = 1.;
        for (int j = 0; j < n; ++j) {
            pmm = pm;
            pm = pn;
            u = __dmul_rn(y, pm);
            pn = __dadd_rn(__dmul_rn(jr[j], __dsub_rn(u, pmm)), u);   // jr[j] = j / (j + 1.)
        }
        u = __dsub_rn(1., __dmul_rn(y, y));
        d1 = __ddiv_rn(__dmul_rn(dn, __dsub_rn(pm, __dmul_rn(y, pn))), u);
        d2 = __ddiv_rn(__dsub_rn(__dmul_rn(__dmul_rn(2., y), d1), __dmul_rn(ib, pn)), u);
        y_prev = y;
        u = __ddiv_rn(pn, d1);
        y = __dsub_rn(y_prev, __dmul_rn(u, __dadd_rn(1., __ddiv_rn(__dmul_rn(u, d2), __dmul_rn(2., d1)))));
    } while (fabs(__dsub_rn(y, y_prev)) > 2.220446049250313e-16 && ++it < 100);
    double de = __dmul_rn(dn, pm);
    de = __ddiv_rn(2., __dmul_rn(de, de));
    double *m = mu + mo[t], *w = m + n;   // pool entry: n nodes then n weights
    m[i] = -y;
    m[n - 1 - i] = y;
    w[i] = __dmul_rn(__dsub_rn(1., __dmul_rn(y, y)), de);
    w[n - 1 - i] = w[i];
}

// ---------------------------------------------------------------------------
// K1: one thread per radius.  The downward recurrences -- D_n(mx) from n2 and
// the psi ratio from n1, each with its tangent-linear columns -- keep only
// their values at the top of every block of K1_B orders (checkpoints in ck);
// the ascending pass replays each block from its checkpoint into local
// arrays (the same operations, so the same values), runs psi and chi upward,
// forms a_n, b_n and their tangent-linear columns, writes the expansion
// coefficients fv4 (a +- b) (coef, or the tensor-core B operand) and sums the
// per-radius cross sections rs[(col*5 + q)*R + r], q: se, ss, Re sb, Im sb, sg,
// in order.  Follows src/lmie_core.c:298-370 (psi ratio, psi, chi), 386-440
// (D), 455-510 (a, b and tangents), 515-590 (cross-section and asymmetry
// sums per radius).
// ---------------------------------------------------------------------------

// Split-precision operand of K1's radius.  The 8 floats of order j and column
// slot cc -- e = 0..7: S hi re, S hi im, S lo re, S lo im, D' hi re, D' hi im,
// D' lo re, D' lo im, with D' = s_j (a - b) fv4 -- are staged in the thread's
// slot u = (j - 1) % 4 of shared memory, tcbuf[((u * CC + cc) * 8 + e) * T +
// thread] (a warp's accesses hit consecutive banks); every 4 orders (and after
// the last) they go out as 16-byte pieces of the K-major core-matrix layout of
// tc_layout.cuh instead of 4-byte stores per order.
template <int CC>
__device__ __forceinline__ void tc_stage(float *tcbuf, int j, int cc, double sre, double sim, double dre,
                                         double dim) {
    const int T = blockDim.x, u = (j - 1) & 3;
    const double sg = (j & 1) ? 1. : -1.;             // s_j of D'
    float *p = tcbuf + (size_t) ((u * CC + cc) * 8) * T + threadIdx.x;
    float h, l;
    tc_split(sre, h, l); p[0] = h; p[2 * T] = l;
    tc_split(sim, h, l); p[1 * T] = h; p[3 * T] = l;
    tc_split(sg * dre, h, l); p[4 * T] = h; p[6 * T] = l;
    tc_split(sg * dim, h, l); p[5 * T] = h; p[7 * T] = l;
}

// Writes the group of 4 orders that holds order j (orders after j in it are
// zero) for the column slots this launch produces: slot 0 (the value) when
// write_value, slots 1.. the tangent-linear columns c0 + 1...
template <int CC>
__device__ __forceinline__ void tc_flush(const float *tcbuf, float *__restrict__ rbase, int j, int pos, int c1,
                                         int c0, int write_value, int gnk) {
    const int T = blockDim.x, last = (j - 1) & 3, k0 = (j - 1) - last;
    constexpr int P = TC_BPART / 4;
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int cc = 0; cc < CC; ++cc) {
        if (cc == 0 && !write_value) continue;
        const int col = cc == 0 ? 0 : c0 + cc;
        const int n = (pos * c1 + col) * 2;
        {
            const int kc = k0 / TC_KC, kk = k0 - kc * TC_KC;
            float *base = rbase + (size_t) kc * (TC_BSTAGE / 4);
            const int i0 = tc_idx(n, kk, TC_NP), d0 = tc_idx(TC_NHALF + n, kk, TC_NP);
            float v[8][4];
#pragma unroll
            for (int e = 0; e < 8; ++e)
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    v[e][u] = u <= last ? tcbuf[(size_t) ((u * CC + cc) * 8 + e) * T + threadIdx.x] : 0.f;
            *(float4 *) (base + i0) = make_float4(v[0][0], v[0][1], v[0][2], v[0][3]);
            *(float4 *) (base + i0 + 4) = make_float4(v[1][0], v[1][1], v[1][2], v[1][3]);
            *(float4 *) (base + P + i0) = make_float4(v[2][0], v[2][1], v[2][2], v[2][3]);
            *(float4 *) (base + P + i0 + 4) = make_float4(v[3][0], v[3][1], v[3][2], v[3][3]);
            *(float4 *) (base + d0) = make_float4(v[4][0], v[4][1], v[4][2], v[4][3]);
            *(float4 *) (base + d0 + 4) = make_float4(v[5][0], v[5][1], v[5][2], v[5][3]);
            *(float4 *) (base + P + d0) = make_float4(v[6][0], v[6][1], v[6][2], v[6][3]);
            *(float4 *) (base + P + d0 + 4) = make_float4(v[7][0], v[7][1], v[7][2], v[7][3]);
        }
        // after the radius' last order: zeros up to the end of its group's chunks
        // (the operand buffer is not cleared between solves)
        for (int k = k0 + 4; k < gnk * TC_KC; k += 4) {
            const int kc = k / TC_KC, kk = k - kc * TC_KC;
            float *base = rbase + (size_t) kc * (TC_BSTAGE / 4);
            const int i0 = tc_idx(n, kk, TC_NP), d0 = tc_idx(TC_NHALF + n, kk, TC_NP);
            *(float4 *) (base + i0) = z;
            *(float4 *) (base + i0 + 4) = z;
            *(float4 *) (base + P + i0) = z;
            *(float4 *) (base + P + i0 + 4) = z;
            *(float4 *) (base + d0) = z;
            *(float4 *) (base + d0 + 4) = z;
            *(float4 *) (base + P + d0) = z;
            *(float4 *) (base + P + d0 + 4) = z;
        }
    }
}

// m[c] = max(m[c], biased exponent of component c + ek) over the normal
// values among (Re cs, Im cs, Re cd, Im cd)
__device__ __forceinline__ void oz_track(int (&m)[4], cplx cs, cplx cd, int ek) {
    const double v[4] = {cs.re, cs.im, cd.re, cd.im};
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int ex = (__double2hiint(v[c]) >> 20) & 0x7FF;
        m[c] = max(m[c], ex ? ex + ek : 0);
    }
}

template <int NC>
__global__ void __launch_bounds__(64) k_mie(DevBatch B, int c0, int write_value, double *__restrict__ ck,
                                            double *__restrict__ coef, float *__restrict__ bop,
                                            double *__restrict__ rs) {
    constexpr int CC = 1 + NC;
    constexpr int CW = k1_ck_width(NC);               // D (2), D_l (2 NC), ratio (1), ratio_l (NC)
    // thread t takes the radius of rank t in the launch order: cases in the
    // order k1ord, each from its largest radius down
    const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= B.R) return;
    const int kc = find_case(B.k1pre, B.ncase, t);
    const int r = [&] {
        const DevCase &Ck = B.cs[B.k1ord[kc]];
        return Ck.r0 + Ck.nr - 1 - (int) (t - B.k1pre[kc]);
    }();
    const int R = B.R;
    const DevCase &C = B.cs[B.rcase[r]];
    const int n1 = B.n1r[r], n2 = B.n2r[r];
    const double x = B.x[r];
    const double xinv = 1. / x;
    const cplx m = C.m, minv = C.minv;
    const cplx z = mk(m.re * x, m.im * x);
    const cplx zinv = cinv(z);
    const int nb = (n1 + K1_B - 1) / K1_B;
    double *ckr = ck + (size_t) B.ckoff[r] * CW;     // nb blocks of CW doubles
    const double *fv1 = B.fv, *fv3 = B.fv + 2 * (B.n1max + 2), *fv4 = B.fv + 3 * (B.n1max + 2);

    double xl[NC > 0 ? NC : 1];
    cplx zl[NC > 0 ? NC : 1], ml[NC > 0 ? NC : 1];
#pragma unroll
    for (int k = 0; k < NC; ++k) {
        const int kk = B.idx1[c0 + k];
        xl[k] = B.xl[(size_t) (c0 + k) * R + r];
        ml[k] = B.m_l[C.ml_off + kk];
        zl[k] = ml[k] * x + m * xl[k];
    }

    // ---- downward sweeps: checkpoints only ----
    // Two independent chains: D_n from n2 and the psi ratio from n1 (n2 > n1).
    // Below n1 they advance in the same loop, so that the dependent steps of
    // one fill the latency of the other; each chain's arithmetic and order
    // are those of a sweep of its own.
    {
        cplx D = mk(0., 0.), Dl[NC > 0 ? NC : 1];
        double rn = 0., rl[NC > 0 ? NC : 1];
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            Dl[k] = mk(0., 0.);
            rl[k] = 0.;
        }
        for (int c = 0; c < nb; ++c) {
            double *q = ckr + (size_t) c * CW;
            if (c * K1_B + K1_B >= n2) {
                q[0] = q[1] = 0.;
#pragma unroll
                for (int k = 0; k < NC; ++k) q[2 + 2 * k] = q[3 + 2 * k] = 0.;
            }
            if (c * K1_B + K1_B >= n1) {
                q[2 + 2 * NC] = 0.;
#pragma unroll
                for (int k = 0; k < NC; ++k) q[3 + 2 * NC + k] = 0.;
            }
        }
        auto d_step = [&](int j) {
            const cplx c1 = (j + 1.) * zinv;
            const cplx ic2 = cinv(D + c1);
            D = c1 - ic2;
            if (NC > 0) {
                const cplx c3 = -c1 * zinv;
                const cplx ic4 = ic2 * ic2;
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    const cplx c5 = c3 * zl[k];
                    Dl[k] = c5 + (Dl[k] + c5) * ic4;
                }
            }
            if (j % K1_B == 0 && j / K1_B - 1 < nb) {
                double *q = ckr + (size_t) (j / K1_B - 1) * CW;
                q[0] = D.re;
                q[1] = D.im;
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    q[2 + 2 * k] = Dl[k].re;
                    q[3 + 2 * k] = Dl[k].im;
                }
            }
        };
        auto r_step = [&](int j) {
            const double a1 = (2. * j + 1.) * xinv;
            const double rnew = 1. / (a1 - rn);
            if (NC > 0) {
                const double a2 = -a1 * xinv, a3 = rnew * rnew;
#pragma unroll
                for (int k = 0; k < NC; ++k) rl[k] = -(a2 * xl[k] - rl[k]) * a3;
            }
            rn = rnew;
            if (j % K1_B == 0 && j / K1_B - 1 < nb) {
                double *q = ckr + (size_t) (j / K1_B - 1) * CW + 2 + 2 * NC;
                q[0] = rn;
#pragma unroll
                for (int k = 0; k < NC; ++k) q[1 + k] = rl[k];
            }
        };
        for (int j = n2 - 1; j >= n1; --j) d_step(j);
        for (int j = n1 - 1; j >= 1; --j) {
            d_step(j);
            r_step(j);
        }
    }

    // ---- ascending pass ----
    double sinx, cosx;
    sincos(x, &sinx, &cosx);
    double psi_p = sinx, chi_p = cosx, chi_c = xinv * cosx + sinx;     // psi_0, chi_0, chi_1
    double psil_p[NC > 0 ? NC : 1], chil_p[NC > 0 ? NC : 1], chil_c[NC > 0 ? NC : 1];
#pragma unroll
    for (int k = 0; k < NC; ++k) {
        psil_p[k] = xl[k] * cosx;
        chil_p[k] = xl[k] * -sinx;
        chil_c[k] = (-xinv * xinv) * xl[k] * cosx + xinv * chil_p[k] + xl[k] * cosx;
    }
    double acc[5 * CC];
#pragma unroll
    for (int q = 0; q < 5 * CC; ++q) acc[q] = 0.;
    cplx ap = mk(0., 0.), bp = mk(0., 0.), alp[NC > 0 ? NC : 1], blp[NC > 0 ? NC : 1];
#pragma unroll
    for (int k = 0; k < NC; ++k) alp[k] = blp[k] = mk(0., 0.);
    const cplx Dm2f = minv * minv;
    const size_t tot = (size_t) B.tot, off = (size_t) B.off[r];
    // split precision: the radii of tensor-core cases write the B operand
    const int tcode = bop ? B.tc_pos[r] : -1;
    const bool to_tc = tcode >= 0;
    const int tpos = tcode & 255, tgnk = tcode >> 8;   // position in the group, the group's chunks
    const long long troff = to_tc ? B.tc_roff[r] : 0;
    extern __shared__ float tcbuf[];                  // [4][1 + NC][8][blockDim.x] when bop is set
    double4 *cf = (double4 *) coef;
    // int8 form: the largest (biased exponent + e_k) of each column and
    // component, the column exponents of the fixed-point B operand
    int *const rx = B.oz_radexp;
    int mxe[CC][4];
#pragma unroll
    for (int q = 0; q < 4 * CC; ++q) mxe[q / 4][q % 4] = 0;

    cplx Dloc[K1_B], Dlloc[NC > 0 ? NC : 1][K1_B];
    double rloc[K1_B], rlloc[NC > 0 ? NC : 1][K1_B];
    for (int c = 0; c < nb; ++c) {
        const int lo = c * K1_B + 1, hi = min(c * K1_B + K1_B, n1);
        const double *q = ckr + (size_t) c * CW;
        // replay D, D_l from the block's top (t <= n2) and the psi ratio and
        // its tangents from hi (t >= hi) down to lo: one loop below hi, as in
        // the downward sweeps
        {
            const int t = min(c * K1_B + K1_B, n2);
            cplx D = mk(q[0], q[1]), Dl[NC > 0 ? NC : 1];
#pragma unroll
            for (int k = 0; k < NC; ++k) Dl[k] = mk(q[2 + 2 * k], q[3 + 2 * k]);
            if (t <= hi) {
                Dloc[t - lo] = D;
#pragma unroll
                for (int k = 0; k < NC; ++k) Dlloc[k][t - lo] = Dl[k];
            }
            const double *qr = q + 2 + 2 * NC;
            double rn = qr[0], rl[NC > 0 ? NC : 1];
#pragma unroll
            for (int k = 0; k < NC; ++k) rl[k] = qr[1 + k];
            rloc[hi - lo] = rn;
#pragma unroll
            for (int k = 0; k < NC; ++k) rlloc[k][hi - lo] = rl[k];
            auto d_step = [&](int j) {
                const cplx c1 = (j + 1.) * zinv;
                const cplx ic2 = cinv(D + c1);
                D = c1 - ic2;
                if (NC > 0) {
                    const cplx c3 = -c1 * zinv;
                    const cplx ic4 = ic2 * ic2;
#pragma unroll
                    for (int k = 0; k < NC; ++k) {
                        const cplx c5 = c3 * zl[k];
                        Dl[k] = c5 + (Dl[k] + c5) * ic4;
                    }
                }
                if (j <= hi) {
                    Dloc[j - lo] = D;
#pragma unroll
                    for (int k = 0; k < NC; ++k) Dlloc[k][j - lo] = Dl[k];
                }
            };
            auto r_step = [&](int j) {
                const double a1 = (2. * j + 1.) * xinv;
                const double rnew = 1. / (a1 - rn);
                if (NC > 0) {
                    const double a2 = -a1 * xinv, a3 = rnew * rnew;
#pragma unroll
                    for (int k = 0; k < NC; ++k) rl[k] = -(a2 * xl[k] - rl[k]) * a3;
                }
                rn = rnew;
                rloc[j - lo] = rn;
#pragma unroll
                for (int k = 0; k < NC; ++k) rlloc[k][j - lo] = rl[k];
            };
            for (int j = t - 1; j >= hi; --j) d_step(j);
            for (int j = hi - 1; j >= lo; --j) {
                d_step(j);
                r_step(j);
            }
        }
        for (int j = lo; j <= hi; ++j) {
            const double rj = rloc[j - lo];
            const double psi = rj * psi_p;
            double psil[NC > 0 ? NC : 1];
#pragma unroll
            for (int k = 0; k < NC; ++k) psil[k] = rlloc[k][j - lo] * psi_p + rj * psil_p[k];
            const cplx D = Dloc[j - lo];
            const cplx zeta = mk(psi, chi_c), zeta_p = mk(psi_p, chi_p);
            const double tt = j * xinv;
            const cplx ca = D * minv + tt;
            const cplx na = ca * psi - psi_p;
            const cplx ida = cinv(ca * zeta - zeta_p);
            const cplx a = na * ida;
            const cplx cb = m * D + tt;
            const cplx nbq = cb * psi - psi_p;
            const cplx idb = cinv(cb * zeta - zeta_p);
            const cplx b = nbq * idb;
            cplx al[NC > 0 ? NC : 1], bl[NC > 0 ? NC : 1];
            if (NC > 0) {
                const cplx Dm2 = D * Dm2f;
                const double tx = -tt * xinv;
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    const cplx Dl = Dlloc[k][j - lo];
                    const cplx zetal = mk(psil[k], chil_c[k]), zetal_p = mk(psil_p[k], chil_p[k]);
                    const double tl = tx * xl[k];
                    const cplx c6 = Dl * minv - Dm2 * ml[k] + tl;
                    al[k] = (c6 * psi + ca * psil[k] - psil_p[k]) * ida -
                            na * ((c6 * zeta + ca * zetal - zetal_p) * (ida * ida));
                    const cplx c4 = ml[k] * D + m * Dl + tl;
                    bl[k] = (c4 * psi + cb * psil[k] - psil_p[k]) * idb -
                            nbq * ((c4 * zeta + cb * zetal - zetal_p) * (idb * idb));
                }
            }
            // sums of order j, and the asymmetry term of order j - 1 (it needs a_j, b_j)
            const double f1 = fv1[j], f4 = fv4[j];
            const double sgn = (j & 1) ? -1. : 1.;
            acc[0] += f1 * (a.re + b.re);
            acc[1] += f1 * (norm2(a) + norm2(b));
            acc[2] += f1 * sgn * (a.re - b.re);
            acc[3] += f1 * sgn * (a.im - b.im);
            if (j >= 2) acc[4] += fv3[j - 1] * (re_mulc(ap, a) + re_mulc(bp, b)) + fv4[j - 1] * re_mulc(ap, bp);
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                double *qq = acc + 5 * (1 + k);
                qq[0] += f1 * (al[k].re + bl[k].re);
                qq[1] += f1 * 2. * (re_mulc(a, al[k]) + re_mulc(b, bl[k]));
                qq[2] += f1 * sgn * (al[k].re - bl[k].re);
                qq[3] += f1 * sgn * (al[k].im - bl[k].im);
                if (j >= 2)
                    qq[4] += fv3[j - 1] * (re_mulc(alp[k], a) + re_mulc(ap, al[k]) + re_mulc(blp[k], b) +
                                           re_mulc(bp, bl[k])) +
                             fv4[j - 1] * (re_mulc(alp[k], bp) + re_mulc(ap, blp[k]));
            }
            // expansion coefficients of order j
            const int ek = 32 - __clz(2 * j - 1);
            if (write_value) {
                const cplx cs = (a + b) * f4, cd = (a - b) * f4;
                if (to_tc) tc_stage<CC>(tcbuf, j, 0, cs.re, cs.im, cd.re, cd.im);
                else cf[off + j - 1] = make_double4(cs.re, cs.im, cd.re, cd.im);
                if (rx) oz_track(mxe[0], cs, cd, ek);
            }
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                const cplx cs = (al[k] + bl[k]) * f4, cd = (al[k] - bl[k]) * f4;
                if (to_tc) tc_stage<CC>(tcbuf, j, 1 + k, cs.re, cs.im, cd.re, cd.im);
                else cf[(size_t) (1 + c0 + k) * tot + off + j - 1] = make_double4(cs.re, cs.im, cd.re, cd.im);
                if (rx) oz_track(mxe[1 + k], cs, cd, ek);
            }
            if (to_tc && (((j - 1) & 3) == 3 || j == n1))
                tc_flush<CC>(tcbuf, bop + troff, j, tpos, 1 + B.nd1, c0, write_value, j == n1 ? tgnk : 0);
            // upward: chi_{j+1} and its tangents; shift the previous order
            const double a1 = (2. * j + 1.) * xinv;
            const double chi_n = a1 * chi_c - chi_p;
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                const double a2l = -a1 * xl[k] * xinv;
                const double chil_n = a2l * chi_c + a1 * chil_c[k] - chil_p[k];
                chil_p[k] = chil_c[k];
                chil_c[k] = chil_n;
                psil_p[k] = psil[k];
                alp[k] = al[k];
                blp[k] = bl[k];
            }
            chi_p = chi_c;
            chi_c = chi_n;
            psi_p = psi;
            ap = a;
            bp = b;
        }
    }
#pragma unroll
    for (int q = 0; q < 5 * CC; ++q) {
        const int cc = q / 5, qq = q % 5;
        if (cc == 0 && !write_value) continue;
        const size_t col = cc == 0 ? 0 : (size_t) (1 + c0 + cc - 1);
        rs[(col * 5 + qq) * R + r] = acc[q];
    }
    if (rx) {
#pragma unroll
        for (int cc = 0; cc < CC; ++cc) {
            if (cc == 0 && !write_value) continue;
            const size_t col = cc == 0 ? 0 : (size_t) (1 + c0 + cc - 1);
            *(int4 *) (rx + (col * R + r) * 4) = make_int4(mxe[cc][0], mxe[cc][1], mxe[cc][2], mxe[cc][3]);
        }
    }
}

// ---------------------------------------------------------------------------
// K2: one block per (case, output column); fixed-order block reduction over
// the case's radii.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double block_sum(double v, double *sh) {
    const int t = threadIdx.x;
    sh[t] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (t < s) sh[t] += sh[t + s];
        __syncthreads();
    }
    double r = sh[0];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(256) k_reduce_scalars(DevBatch B, const double *__restrict__ rs,
                                                        double *__restrict__ sums,
                                                        double *__restrict__ save1) {
    __shared__ double sh[256];
    const int cidx = blockIdx.x;
    const int col = blockIdx.y;           // 0 = value, 1+kk = slot kk
    const DevCase &C = B.cs[cidx];
    const int R = B.R;
    int kind = 0, c1 = 0;                 // 0 value, 1 index1, 2 index2
    if (col > 0) {
        const int kk = col - 1;
        for (int k = 0; k < B.nd1; ++k)
            if (B.idx1[k] == kk) { kind = 1; c1 = 1 + k; }
        if (kind == 0) kind = 2;
    }
    double acc[4] = {0., 0., 0., 0.};
    for (int r = C.r0 + threadIdx.x; r < C.r0 + C.nr; r += blockDim.x) {
        const double f = B.w[r];
        const double se = rs[r], ss = rs[(size_t) R + r];
        const double sbr = rs[(size_t) 2 * R + r], sbi = rs[(size_t) 3 * R + r];
        const double sg = rs[(size_t) 4 * R + r];
        const double bak = sbr * sbr + sbi * sbi;
        if (kind == 0) {
            acc[0] += f * se;
            acc[1] += f * ss;
            acc[2] += f * bak;
            acc[3] += f * sg;
            if (save1) {
                save1[r] = se;
                save1[(size_t) R + r] = ss;
                save1[(size_t) 2 * R + r] = bak;
                save1[(size_t) 3 * R + r] = sg;
            }
        } else if (kind == 1) {
            const double fl = B.w[(size_t) col * R + r];
            const double *q = rs + (size_t) c1 * 5 * R;
            acc[0] += fl * se + f * q[r];
            acc[1] += fl * ss + f * q[(size_t) R + r];
            acc[2] += fl * bak + f * 2. * (sbr * q[(size_t) 2 * R + r] + sbi * q[(size_t) 3 * R + r]);
            acc[3] += fl * sg + f * q[(size_t) 4 * R + r];
        } else {
            const double fl = B.w[(size_t) col * R + r];
            acc[0] += fl * se;
            acc[1] += fl * ss;
            acc[2] += fl * bak;
            acc[3] += fl * sg;
        }
    }
    const int ncol = 1 + B.nd;
    for (int q = 0; q < 4; ++q) {
        double v = block_sum(acc[q], sh);
        if (threadIdx.x == 0) sums[((size_t) cidx * ncol + col) * 4 + q] = v;
    }
}

// ---------------------------------------------------------------------------
// K3: one thread per half-angle (mu_j < 0) and its mirror (-mu_j); a block
// covers AP * ANG_T half-angles of one case and one radius group of it.  For
// every radius the pi_n/tau_n recurrence runs in registers, the coefficient
// columns are staged through shared memory ANG_KT orders at a time (the next
// chunk prefetched into registers), and the quadratic forms of S1, S2 are
// accumulated per thread in shared memory.  One half-angle per thread (AP 1)
// keeps the registers low enough for 12 resident warps per SM, which hides
// the FP64 latencies better than two half-angles sharing coefficient loads.
// ---------------------------------------------------------------------------
constexpr int ANG_T = 128;
constexpr int ANG_KT = 64;

template <int NC1, int NC2, int AP>
__global__ void __launch_bounds__(ANG_T) k_angular(DevBatch B, int c1base, int c2base, int first,
                                                   const AngItem *__restrict__ items,
                                                   const double *__restrict__ coef,
                                                   double *__restrict__ part, double *__restrict__ save2) {
    constexpr int C1 = 1 + NC1;
    constexpr int NS = 1 + NC1 + NC2;
    extern __shared__ double4 smem4[];
    double4 *cbuf = smem4;                                   // [ANG_KT][C1] {cs, cd}
    double *gks = (double *) (cbuf + ANG_KT * C1);           // [ANG_KT] (2k+1)/k
    double *acc = gks + ANG_KT;                              // [AP][NS*2*4][ANG_T]

    const AngItem it = items[blockIdx.x];
    const DevCase &C = B.cs[it.c];
    const int tid = threadIdx.x;
    const int R = B.R;
    const int nh = C.nh, n_qang = C.n_qang;
    const size_t tot = (size_t) B.tot;
    const double *fv2 = B.fv + (B.n1max + 2);
    const double *mup = B.mu_pool + C.mu_off;
    const double4 *cf = (const double4 *) coef;
    int jh[AP];
    bool act[AP];
    double mu[AP];
#pragma unroll
    for (int a = 0; a < AP; ++a) {
        jh[a] = (it.xt * AP + a) * ANG_T + tid;
        act[a] = jh[a] < nh;
        mu[a] = act[a] ? mup[jh[a]] : 0.;
    }
    const bool any = act[0];

    for (int q = 0; q < AP * NS * 8; ++q) acc[q * ANG_T + tid] = 0.;

    int slot1[NC1 > 0 ? NC1 : 1], slot2[NC2 > 0 ? NC2 : 1];
#pragma unroll
    for (int k = 0; k < NC1; ++k) slot1[k] = 1 + B.idx1[c1base + k];
#pragma unroll
    for (int k = 0; k < NC2; ++k) slot2[k] = 1 + B.idx2[c2base + k];

    // The next chunk's coefficients are loaded into registers while the
    // current chunk is consumed from shared memory.
    constexpr int PF = (ANG_KT * C1 + ANG_T - 1) / ANG_T;
    double4 pre[PF];
    double pre_fv = 0.;
    auto fetch = [&](size_t off, int n1, int k0) {
        const int kt = min(ANG_KT, n1 - k0);
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int idx = tid + u * ANG_T;
            if (idx < kt * C1) {
                const int t = idx / C1, c = idx - t * C1;
                const size_t col = c == 0 ? 0 : (size_t) (c1base + c);
                pre[u] = cf[col * tot + off + k0 + t];
            }
        }
        if (tid < kt) pre_fv = fv2[k0 + tid + 1];
    };

    for (int r = it.rbeg; r < it.rend; ++r) {
        const int n1 = B.n1r[r];
        const size_t off = (size_t) B.off[r];
        cplx spA[AP][C1], smA[AP][C1], spB[AP][C1], smB[AP][C1];
        double p0[AP], p1[AP];
#pragma unroll
        for (int a = 0; a < AP; ++a) {
            p0[a] = 0.;
            p1[a] = 1.;
#pragma unroll
            for (int c = 0; c < C1; ++c) spA[a][c] = smA[a][c] = spB[a][c] = smB[a][c] = mk(0., 0.);
        }
        double kd = 1.;
        fetch(off, n1, 0);
        for (int k0 = 0; k0 < n1; k0 += ANG_KT) {
            const int kt = min(ANG_KT, n1 - k0);
            __syncthreads();
#pragma unroll
            for (int u = 0; u < PF; ++u) {
                const int idx = tid + u * ANG_T;
                if (idx < kt * C1) cbuf[idx] = pre[u];
            }
            if (tid < kt) gks[tid] = 1. + pre_fv;
            __syncthreads();
            if (k0 + ANG_KT < n1) fetch(off, n1, k0 + ANG_KT);
            if (!any) continue;
            // orders k = k0 + t + 1: t even <-> k odd <-> mirror sign +1.  With
            // t2 = mu pi_k - pi_{k-1}: tau_k = k t2 - pi_{k-1} and
            // pi_{k+1} = mu pi_k + (k+1)/k t2 = (2k+1)/k t2 + pi_{k-1}
            // (the reference's a1 + fv2 a2, src/lmie_core.c:674-689, in three FMAs)
            auto step = [&](int t, bool odd) {
                const double gk = gks[t];
#pragma unroll
                for (int a = 0; a < AP; ++a) {
                    const double t2 = fma(mu[a], p1[a], -p0[a]), tau = fma(kd, t2, -p0[a]);
                    const double tp = p1[a] + tau, tm = p1[a] - tau;
                    const double pn = fma(gk, t2, p0[a]);
                    p0[a] = p1[a];
                    p1[a] = pn;
#pragma unroll
                    for (int c = 0; c < C1; ++c) {
                        const double4 v = cbuf[t * C1 + c];
                        spA[a][c].re += tp * v.x;  spA[a][c].im += tp * v.y;
                        smA[a][c].re += tm * v.z;  smA[a][c].im += tm * v.w;
                        if (odd) {
                            spB[a][c].re += tm * v.x;  spB[a][c].im += tm * v.y;
                            smB[a][c].re += tp * v.z;  smB[a][c].im += tp * v.w;
                        } else {
                            spB[a][c].re -= tm * v.x;  spB[a][c].im -= tm * v.y;
                            smB[a][c].re -= tp * v.z;  smB[a][c].im -= tp * v.w;
                        }
                    }
                }
                kd += 1.;
            };
            int t = 0;
            for (; t + 1 < kt; t += 2) {
                step(t, true);
                step(t + 1, false);
            }
            if (t < kt) step(t, true);
        }
        if (!any) continue;
        const double f = B.w[r], half_f = f * .5;
        double fl1[NC1 > 0 ? NC1 : 1], fl2[NC2 > 0 ? NC2 : 1];
#pragma unroll
        for (int k = 0; k < NC1; ++k) fl1[k] = B.w[(size_t) slot1[k] * R + r];
#pragma unroll
        for (int k = 0; k < NC2; ++k) fl2[k] = B.w[(size_t) slot2[k] * R + r];
#pragma unroll
        for (int a = 0; a < AP; ++a) {
            if (!act[a]) continue;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const cplx *sp = h ? spB[a] : spA[a];
                const cplx *sm = h ? smB[a] : smA[a];
                const cplx s1 = (sp[0] + sm[0]) * .5, s2 = (sp[0] - sm[0]) * .5;
                const double e1 = norm2(s1), e3 = norm2(s2);
                const cplx c12 = s1 * conjg(s2), c21 = s2 * conjg(s1);
                const double pv[4] = {(e1 + e3) * .5, (c12.re + c21.re) * .5, -(e1 - e3) * .5,
                                      .5 * (c12.im - c21.im)};
                double *accA = acc + (size_t) a * NS * 8 * ANG_T;
                double *av = accA + (h * 4) * ANG_T + tid;
                if (first) {
#pragma unroll
                    for (int e = 0; e < 4; ++e) av[e * ANG_T] += f * pv[e];
                    if (save2) {
                        const int jj = h ? n_qang - 1 - jh[a] : jh[a];
#pragma unroll
                        for (int e = 0; e < 4; ++e) save2[((size_t) e * R + r) * n_qang + jj] = pv[e];
                    }
                }
#pragma unroll
                for (int k = 0; k < NC1; ++k) {
                    const cplx s1l = (sp[1 + k] + sm[1 + k]) * .5, s2l = (sp[1 + k] - sm[1 + k]) * .5;
                    const double q1 = 2. * (s1l.re * s1.re + s1l.im * s1.im);
                    const double q3 = 2. * (s2l.re * s2.re + s2l.im * s2.im);
                    const cplx d12 = (s1l * conjg(s2)) * 2., d21 = (s2l * conjg(s1)) * 2.;
                    double *al = accA + ((1 + k) * 8 + h * 4) * ANG_T + tid;
                    al[0] += fl1[k] * pv[0] + half_f * (q1 + q3);
                    al[ANG_T] += fl1[k] * pv[1] + half_f * (d12.re + d21.re);
                    al[2 * ANG_T] += fl1[k] * pv[2] + half_f * -(q1 - q3);
                    al[3 * ANG_T] += fl1[k] * pv[3] + half_f * (d12.im - d21.im);
                }
#pragma unroll
                for (int k = 0; k < NC2; ++k) {
                    double *al = accA + ((1 + NC1 + k) * 8 + h * 4) * ANG_T + tid;
#pragma unroll
                    for (int e = 0; e < 4; ++e) al[e * ANG_T] += pv[e] * fl2[k];
                }
            }
        }
    }
    const int Q = 4 * (1 + B.nd);
    double *pc = part + C.part_off + (size_t) it.g * Q * n_qang;
#pragma unroll
    for (int a = 0; a < AP; ++a) {
        if (!act[a]) continue;
        const double *accA = acc + (size_t) a * NS * 8 * ANG_T;
        for (int s = 0; s < NS; ++s) {
            if (s == 0 && !first) continue;
            const int slot = s == 0 ? 0 : (s <= NC1 ? slot1[s - 1] : slot2[s - 1 - NC1]);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int jj = h ? n_qang - 1 - jh[a] : jh[a];
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    pc[(size_t) (slot * 4 + e) * n_qang + jj] = accA[(s * 8 + h * 4 + e) * ANG_T + tid];
            }
        }
    }
}

// pfacc[case][q][jj] = sum over the case's radius groups, in group order
__global__ void k_reduce_pf(DevBatch B, long long total, const long long *__restrict__ start,
                            const double *__restrict__ part, double *__restrict__ pfacc) {
    const long long e = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const int c = find_case(start, B.ncase, e);
    const DevCase &C = B.cs[c];
    const long long local = e - start[c];
    const size_t span = (size_t) 4 * (1 + B.nd) * C.n_qang;
    double s = 0.;
    for (int g = 0; g < C.G; ++g) s += part[C.part_off + (size_t) g * span + local];
    pfacc[C.pf_off + local] = s;
}

// save_control 2 (single case): re-weight stored per-radius kernels
// (src/lmie_schedule.c:1087-1124)
__global__ void k_save_reweight_pf(DevBatch B, int n_qang, const double *__restrict__ save2,
                                   const double *__restrict__ w2, double *__restrict__ pfacc) {
    const size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;   // e*n_qang + jj
    if (i >= (size_t) 4 * n_qang) return;
    const int e = (int) (i / n_qang), jj = (int) (i % n_qang);
    const int n = B.R;
    double s = 0.;
    for (int r = 0; r < n; ++r) s += save2[((size_t) e * n + r) * n_qang + jj] * B.w[r];
    pfacc[(size_t) e * n_qang + jj] = s;
    for (int k = 0; k < B.nd; ++k) {
        double v = 0.;
        bool idx2 = false;
        for (int q = 0; q < B.nd2; ++q) idx2 |= B.idx2[q] == k;
        if (idx2)
            for (int r = 0; r < n; ++r) v += save2[((size_t) e * n + r) * n_qang + jj] * w2[(size_t) k * n + r];
        pfacc[((size_t) (1 + k) * 4 + e) * n_qang + jj] = v;
    }
}

__global__ void k_save_reweight_scal(DevBatch B, const double *__restrict__ save1, const double *__restrict__ w2,
                                     double *__restrict__ sums) {
    const int col = threadIdx.x;    // 0..nd
    if (col > B.nd) return;
    const int n = B.R;
    double acc[4] = {0., 0., 0., 0.};
    bool on = col == 0;
    if (col > 0)
        for (int q = 0; q < B.nd2; ++q) on |= B.idx2[q] == col - 1;
    if (on)
        for (int r = 0; r < n; ++r) {
            const double a = col == 0 ? B.w[r] : w2[(size_t) (col - 1) * n + r];
            for (int q = 0; q < 4; ++q) acc[q] += save1[(size_t) q * n + r] * a;
        }
    for (int q = 0; q < 4; ++q) sums[col * 4 + q] = acc[q];
}

// ---------------------------------------------------------------------------
// Normalisation: g and the phase matrix by 2/Csca, cross sections by
// lambda^2/(2 pi), Cbak additionally by 1/(8 pi), with the chain rule for
// every derivative slot.
// ---------------------------------------------------------------------------
__global__ void k_normalize_pf(DevBatch B, long long total, const long long *__restrict__ start,
                               const double *__restrict__ sums, const double *__restrict__ pfacc,
                               double *__restrict__ pfn) {
    const long long e = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const int c = find_case(start, B.ncase, e);
    const DevCase &C = B.cs[c];
    const long long local = e - start[c];
    const int q = (int) (local / C.n_qang), jj = (int) (local % C.n_qang);
    const int slot = q / 4, el = q % 4;
    const double *sm = sums + (size_t) c * (1 + B.nd) * 4;
    const double csca = sm[1];
    const double a = 2. / csca;
    const double *pa = pfacc + C.pf_off;
    if (slot == 0) {
        pfn[C.pf_off + local] = pa[local] * a;
    } else {
        const double a_l = -a * sm[slot * 4 + 1] / csca;
        pfn[C.pf_off + local] = pa[local] * a + pa[(size_t) el * C.n_qang + jj] * a_l;
    }
}

__global__ void k_normalize_scal(DevBatch B, const double *__restrict__ sums, double *__restrict__ scal) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= B.ncase) return;
    const DevCase &C = B.cs[c];
    const int ncol = 1 + B.nd;
    const double *sm = sums + (size_t) c * ncol * 4;
    double *o = scal + C.scal_off;
    const double csca = sm[1];
    const double a = 2. / csca;
    const double lam = C.lambda;
    const double b = lam * lam / (2. * LMIEB_PI);
    const double g = sm[3];
    for (int k = 0; k < B.nd; ++k) {
        const double *s = sm + (1 + k) * 4;
        const double a_l = -a * s[1] / csca;
        const double b_l = 2. * B.lambda_l[C.ml_off + k] * lam / (2. * LMIEB_PI);
        double *ok = o + (1 + k) * 4;
        ok[0] = s[0] * b + sm[0] * b_l;
        ok[1] = s[1] * b + sm[1] * b_l;
        ok[2] = (s[2] * b + sm[2] * b_l) / (2. * 4. * LMIEB_PI);
        ok[3] = s[3] * a + g * a_l;
    }
    o[0] = sm[0] * b;
    o[1] = sm[1] * b;
    o[2] = sm[2] * b / (2. * 4. * LMIEB_PI);
    o[3] = g / csca * 2.;
}

// ---------------------------------------------------------------------------
// GSF / Legendre basis recurrences.  rc[8*l + q] (host-computed, l >= 3,
// j = l - 1): p00_l = q0 mu p00_{l-1} - q1 p00_{l-2};
// p02_l = q2 mu p02_{l-1} - q3 p02_{l-2};
// p22_l = (q4 mu - q5) p22_{l-1} - q6 p22_{l-2}; p2m_l = (q4 mu + q5) p2m_{l-1} - q6 p2m_{l-2};
// Legendre: p_l = q1 (mu p_{l-1} - p_{l-2}) + mu p_{l-1} (q1 = 1/2 at l = 2).
// Function f of the GSF set: 0 p00, 1 p0+2, 2 p2+2, 3 p2-2; Legendre: f = 0.
// ---------------------------------------------------------------------------
template <int KIND>
__device__ __forceinline__ double basis_first(int f, int l, double x) {
    if (KIND == 1) return l == 0 ? 1. : x;
    if (l == 0) return f == 0 ? 1. : 0.;
    if (l == 1) return f == 0 ? x : 0.;
    const double x2 = x * x;
    if (f == 0) return (3. * x2 - 1.) / 2.;
    if (f == 1) return .25 * sqrt(6.) * (x2 - 1.);
    double t = f == 2 ? 1. + x : 1. - x;
    return .25 * t * t;
}

template <int KIND>
__device__ __forceinline__ double basis_step(int f, const double *c, double x, double cur, double prev) {
    if (KIND == 1) {
        const double b = x * cur;
        return c[1] * (b - prev) + b;
    }
    if (f == 0) return c[0] * x * cur - c[1] * prev;
    if (f == 1) return c[2] * x * cur - c[3] * prev;
    const double e = c[4] * x;
    return (f == 2 ? e - c[5] : e + c[5]) * cur - c[6] * prev;
}

// advance one basis function from order l-1 to l
template <int KIND>
__device__ __forceinline__ double basis_next(int f, int l, const double *rc, double x, double cur, double prev) {
    const int first = KIND == 1 ? 2 : 3;
    return l < first ? basis_first<KIND>(f, l, x) : basis_step<KIND>(f, rc + 8 * (size_t) l, x, cur, prev);
}

// ---------------------------------------------------------------------------
// K4a: one thread per (case, basis function, positive node) runs the
// recurrence over all orders and checkpoints (p_{l-2}, p_{l-1}) at the start
// of every EX_LT-order tile.
// ---------------------------------------------------------------------------
// one chain: function F of the set at node x over all n_coef orders
template <int KIND, int F>
__device__ __forceinline__ void ckpt_chain(const DevCase &C, int i, double x, const double *__restrict__ rc,
                                           double *__restrict__ ck) {
    constexpr int NF = KIND == 0 ? 4 : 1;
    constexpr int first = KIND == 1 ? 2 : 3;
    double prev = 0., cur = 0.;
    for (int lb = 0; lb < C.n_coef; lb += EX_LT) {
        const size_t o = (((size_t) (lb / EX_LT) * NF + F) * C.nh + i) * 2;
        ck[o] = prev;
        ck[o + 1] = cur;
        const int le = min(C.n_coef, lb + EX_LT);
        int l = lb;
        for (; l < le && l < first; ++l) {
            const double v = basis_first<KIND>(F, l, x);
            prev = cur;
            cur = v;
        }
        // the recurrence coefficients do not depend on the chain: unrolled,
        // with the function fixed, their loads are issued ahead of the
        // dependent steps
#pragma unroll 8
        for (; l < le; ++l) {
            const double v = basis_step<KIND>(F, rc + 8 * (size_t) l, x, cur, prev);
            prev = cur;
            cur = v;
        }
    }
}

template <int KIND>
__global__ void k_exp_ckpt(DevBatch B, long long total, const long long *__restrict__ start,
                           double *__restrict__ ckpt) {
    const long long e = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const int c = find_case(start, B.ncase, e);
    const DevCase &C = B.cs[c];
    const long long local = e - start[c];
    const int f = (int) (local / C.nh), i = (int) (local % C.nh);
    const double x = B.mu_pool[C.mu_off + C.nh + i];
    double *ck = ckpt + C.ck_off;
    if (KIND == 1) ckpt_chain<KIND, 0>(C, i, x, B.rc, ck);
    else if (f == 0) ckpt_chain<KIND, 0>(C, i, x, B.rc, ck);
    else if (f == 1) ckpt_chain<KIND, 1>(C, i, x, B.rc, ck);
    else if (f == 2) ckpt_chain<KIND, 2>(C, i, x, B.rc, ck);
    else ckpt_chain<KIND, 3>(C, i, x, B.rc, ck);
}

// ---------------------------------------------------------------------------
// K4b: one block per (case, order tile, angle tile).  The basis functions of
// the tile are generated into shared memory from the checkpoints, the
// weighted phase-matrix moments of the tile's node pairs (mu-parity folding)
// are staged next to them, and each output (order, column) is contracted
// over the tile's EX_AT node pairs.  Raw per-tile sums go to exq.
// ---------------------------------------------------------------------------
// threads of a K4b block: one per (order, column) of the contraction, at
// least 128 (the basis phase) and at most EX_TMAX
constexpr int EX_TMAX = 256;

// D (8 x 8, two values per thread) += A (8 x 4, one value) B (4 x 8, one value)
// in FP64 on the tensor cores
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// ---------------------------------------------------------------------------
// K4 of the GSF expansion on the FP64 tensor cores (k_exp_gsf): one block of
// 4 warps per (case, angle tile) runs over all the case's orders, a tile of
// EX_LT orders at a time.  Thread (function f, node pair ia) continues its
// basis recurrence from tile to tile in registers (no checkpoints), writing
// the tile's values into shared memory; the weighted phase-matrix moments of
// the block's node pairs are staged once; the recurrence coefficients of the
// next tile are loaded while the current one's are used.  For each order
// parity the 16 orders of that parity form an M = 16 product over K = the
// EX_AT node pairs (mma.sync m8n8k4 f64), the basis functions against the
// folded moments of that parity, whose raw sums go to exq per angle tile
// (the sums of the FP64 kernel, k_exp_tile<0>, in another order).  Basis and
// moments are staged in the m8n8k4 fragment order, so every operand load of
// a warp reads 32 consecutive doubles.
// ---------------------------------------------------------------------------
constexpr int EX_NB = 4;                 // n-blocks of 8 outputs: up to 16 columns
constexpr int EX_KS = EX_AT / 4;         // k-steps of 4 node pairs
// one fragment (32 lanes) every EX_SEG doubles: a warp's fragment load reads
// 32 consecutive doubles, and the staging stores of a warp (4 lanes of each
// of 8 k-steps) fall on distinct bank pairs
constexpr int EX_SEG = 36;
constexpr int EX_AF = 4 * 2 * 2 * EX_KS * EX_SEG;   // basis fragments: [f][parity][m-block][k-step]

// GSF function F of one node pair over the orders of a tile (u < lt, zeros
// after), into its fragment positions (order u = par + 2 m: block par,
// m >> 3, row m & 7), continuing the chain (prev, cur) from the previous
// tile; the recurrence coefficients' loads of the fully unrolled steps do not
// depend on the chain and go ahead of it.
template <int F>
__device__ __forceinline__ void gsf_tile_chain(double *af, const double *rcs, double x, double &prev, double &cur,
                                               int l0, int lt) {
    if (lt == EX_LT && l0 >= 3) {
#pragma unroll
        for (int u = 0; u < EX_LT; ++u) {
            const double v = basis_step<0>(F, rcs + 8 * u, x, cur, prev);
            prev = cur;
            cur = v;
            af[(((u & 1) * 2 + (u >> 4)) * EX_KS) * EX_SEG + (((u >> 1) & 7) << 2)] = v;
        }
        return;
    }
    for (int u = 0; u < EX_LT; ++u) {
        double v = 0.;
        if (u < lt) {
            const int l = l0 + u;
            v = l < 3 ? basis_first<0>(F, l, x) : basis_step<0>(F, rcs + 8 * u, x, cur, prev);
            prev = cur;
            cur = v;
        }
        af[(((u & 1) * 2 + (u >> 4)) * EX_KS) * EX_SEG + (((u >> 1) & 7) << 2)] = v;
    }
}

// doubles between the k-steps of the moment fragments (staged once per
// block: no padding)
constexpr int EX_BSEG = 32;

__host__ __device__ inline int ex_bf_run_size(int ncol) { return 2 * 4 * ((2 * ncol + 7) / 8) * EX_KS * EX_BSEG; }

__global__ void __launch_bounds__(128) k_exp_gsf(DevBatch B, const ExpItem *__restrict__ items,
                                                const double *__restrict__ pfn, double *__restrict__ exq) {
    extern __shared__ double sm[];
    const ExpItem it = items[blockIdx.x];
    const DevCase &C = B.cs[it.c];
    const int nh = C.nh, nq = C.n_qang, ncf = C.n_coef;
    const int ncol = 1 + B.nd, nbn = (2 * ncol + 7) >> 3;
    const int i0 = it.at * EX_AT;
    const double *mup = B.mu_pool + C.mu_off, *wqp = mup + nq;
    double *Af = sm;                                       // basis fragments of the current tile
    double *Bf = Af + EX_AF;                               // moment fragments of the block's node pairs
    double *rcs = Bf + ex_bf_run_size(ncol);               // [2][8 EX_LT] recurrence coefficients of a tile
    // weighted moments of the node pairs, folded for either order parity
    // (s = (-1)^l multiplies the mirror node's terms), into the fragment of
    // each (function slot, output): slot 0 p00 (m0, m5), 1 p2+2 (m2, m3),
    // 2 p2-2 (m1, m4), 3 p0+2 (m6, m7); column n = 2 col + output (columns
    // past ncol only reach outputs that are not kept: zeros; node pairs past
    // the case's angles get zeros)
    for (int t = threadIdx.x; t < 8 * nbn * EX_KS * EX_BSEG; t += blockDim.x) Bf[t] = 0.;
    __syncthreads();
    for (int t = threadIdx.x; t < ncol * EX_AT; t += blockDim.x) {
        const int col = t / EX_AT, ia = t % EX_AT, i = i0 + ia;
        double u0 = 0., u1 = 0., u2 = 0., u3 = 0., v0 = 0., v1 = 0., v2 = 0., v3 = 0.;
        if (i < nh) {
            const int i1 = nh - 1 - i, i2 = nh + i;
            const double w = wqp[i2];
            const double *F = pfn + C.pf_off + (size_t) col * 4 * nq;
            u0 = F[i1] * w; u1 = F[nq + i1] * w; u2 = F[2 * nq + i1] * w; u3 = F[3 * nq + i1] * w;
            v0 = F[i2] * w; v1 = F[nq + i2] * w; v2 = F[2 * nq + i2] * w; v3 = F[3 * nq + i2] * w;
        }
        const int ks = ia >> 2, k = ia & 3;
#pragma unroll
        for (int par = 0; par < 2; ++par) {
            const double sg = par ? -1. : 1.;
            const double m[8] = {sg * u0 + v0, sg * (u0 + u1), v0 + v1, sg * (u0 - u1),
                                 v0 - v1,      sg * u1 + v1,   sg * u2 + v2, sg * u3 + v3};
            // (slot, output) -> moment
            const int mom[4][2] = {{0, 5}, {2, 3}, {1, 4}, {6, 7}};
#pragma unroll
            for (int slot = 0; slot < 4; ++slot)
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const int n = 2 * col + j, nb = n >> 3, nl = n & 7;
                    Bf[(((par * 4 + slot) * nbn + nb) * EX_KS + ks) * EX_BSEG + (nl << 2) + k] = m[mom[slot][j]];
                }
        }
    }
    // the chain of this thread: function f at node pair ia, from order 0
    const int f = threadIdx.x >> 5, ia = threadIdx.x & 31, i = i0 + ia;
    double *af = Af + (size_t) f * (2 * 2 * EX_KS * EX_SEG) + (ia >> 2) * EX_SEG + (ia & 3);
    const double x = i < nh ? mup[nh + i] : 0.;
    double prev = 0., cur = 0.;
    // the first tile's recurrence coefficients
    const int nlt = (ncf + EX_LT - 1) / EX_LT;
    for (int t = threadIdx.x; t < 8 * min(EX_LT, ncf); t += blockDim.x) rcs[t] = B.rc[t];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int par = warp & 1, mb = warp >> 1;
    const double *a0 = Af + ((0 * 2 + par) * 2 + mb) * EX_KS * EX_SEG + lane;   // function 0 (p00)
    constexpr int AF = 2 * 2 * EX_KS * EX_SEG;                                   // stride of a function
    const double *b0 = Bf + (size_t) par * 4 * nbn * EX_KS * EX_BSEG + lane;
    const int BS = nbn * EX_KS * EX_BSEG;                                         // stride of a slot
    double *out = exq + C.ex_off + (size_t) it.at * ncol * 6 * ncf;
    for (int lt = 0; lt < nlt; ++lt) {
        const int l0 = lt * EX_LT, lc = min(EX_LT, ncf - l0);
        const double *rc = rcs + (lt & 1) * 8 * EX_LT;
        // the next tile's coefficients, loaded now and stored after the chain
        const int l1 = l0 + EX_LT, lc1 = min(EX_LT, ncf - l1);
        const int t0 = threadIdx.x, t1 = threadIdx.x + 128;
        double r0 = 0., r1 = 0.;
        if (lc1 > 0) {
            if (t0 < 8 * lc1) r0 = B.rc[8 * (size_t) l1 + t0];
            if (t1 < 8 * lc1) r1 = B.rc[8 * (size_t) l1 + t1];
        }
        // basis functions of the tile (warp-uniform function: one specialised chain each)
        const int lct = i < nh ? lc : 0;
        if (f == 0) gsf_tile_chain<0>(af, rc, x, prev, cur, l0, lct);
        else if (f == 1) gsf_tile_chain<1>(af, rc, x, prev, cur, l0, lct);
        else if (f == 2) gsf_tile_chain<2>(af, rc, x, prev, cur, l0, lct);
        else gsf_tile_chain<3>(af, rc, x, prev, cur, l0, lct);
        if (lc1 > 0) {
            double *rn = rcs + ((lt + 1) & 1) * 8 * EX_LT;
            if (t0 < 8 * lc1) rn[t0] = r0;
            if (t1 < 8 * lc1) rn[t1] = r1;
        }
        __syncthreads();
        // For each order parity the 16 orders of that parity form an M = 16
        // product over K = the tile's EX_AT node pairs: the basis functions
        // against the folded moments of that parity.  Each function feeds
        // two outputs per column (N = 2 ncol): p00 -> (e0: m0, e3: m5), p0+2
        // -> (e4: m6, e5: m7), p2+2 -> (e1: m2, e2: m3) and p2-2 -> (e1: m1,
        // e2: m4), the last two into the same accumulators.  Warp w takes
        // parity w & 1 and the orders 8 (w >> 1) .. + 7 of it.
        double acc[3][EX_NB][2];
#pragma unroll
        for (int g = 0; g < 3; ++g)
#pragma unroll
            for (int nb = 0; nb < EX_NB; ++nb) acc[g][nb][0] = acc[g][nb][1] = 0.;
#pragma unroll 2
        for (int ks = 0; ks < EX_KS; ++ks) {
            const double a00 = a0[ks * EX_SEG], a02 = a0[AF + ks * EX_SEG];
            const double a22 = a0[2 * AF + ks * EX_SEG], a2m = a0[3 * AF + ks * EX_SEG];
#pragma unroll
            for (int nb = 0; nb < EX_NB; ++nb) {
                if (nb >= nbn) break;
                const double *bb = b0 + (nb * EX_KS + ks) * EX_BSEG;
                dmma(acc[0][nb][0], acc[0][nb][1], a00, bb[0]);
                dmma(acc[1][nb][0], acc[1][nb][1], a22, bb[BS]);
                dmma(acc[1][nb][0], acc[1][nb][1], a2m, bb[2 * BS]);
                dmma(acc[2][nb][0], acc[2][nb][1], a02, bb[3 * BS]);
            }
        }
        // accumulators: row m = lane >> 2 (order), columns 2 (lane & 3) + {0, 1}:
        // one column, its two outputs; raw sums of the angle tile to exq
        const int u = par + 2 * (8 * mb + (lane >> 2));
        if (u < lc) {
#pragma unroll
            for (int nb = 0; nb < EX_NB; ++nb) {
                if (nb >= nbn) break;
                const int col = 4 * nb + (lane & 3);
                if (col < ncol) {
                    double *oc = out + (size_t) col * 6 * ncf + l0 + u;
                    oc[0 * (size_t) ncf] = acc[0][nb][0];
                    oc[3 * (size_t) ncf] = acc[0][nb][1];
                    oc[1 * (size_t) ncf] = acc[1][nb][0];
                    oc[2 * (size_t) ncf] = acc[1][nb][1];
                    oc[4 * (size_t) ncf] = acc[2][nb][0];
                    oc[5 * (size_t) ncf] = acc[2][nb][1];
                }
            }
        }
        // the tile's basis has been read before the next tile's chains overwrite it
        __syncthreads();
    }
}

template <int KIND>
__global__ void __launch_bounds__(EX_TMAX) k_exp_tile(DevBatch B, const ExpItem *__restrict__ items,
                                                   const double *__restrict__ pfn,
                                                   const double *__restrict__ ckpt,
                                                   double *__restrict__ exq) {
    constexpr int NF = KIND == 0 ? 4 : 1;
    extern __shared__ double sm[];
    constexpr int NM = KIND == 0 ? 8 : 6;                  // folded moments per column and node pair
    double *P = sm;                                        // [NF][EX_LT][EX_AT + 1]
    double *Bv = P + NF * EX_LT * (EX_AT + 1);             // [ncol][NM][EX_AT][2 order parities]
    const ExpItem it = items[blockIdx.x];
    const DevCase &C = B.cs[it.c];
    const int nh = C.nh, nq = C.n_qang, ncf = C.n_coef;
    const int ncol = 1 + B.nd;
    const int l0 = it.lt * EX_LT, lt = min(EX_LT, ncf - l0);
    const int i0 = it.at * EX_AT;
    const double *mup = B.mu_pool + C.mu_off, *wqp = mup + nq;
    double *rcs = Bv + (size_t) ncol * NM * EX_AT * 2;     // [8 EX_LT] recurrence coefficients of the tile
    for (int t = threadIdx.x; t < 8 * lt; t += blockDim.x) rcs[t] = B.rc[8 * (size_t) l0 + t];
    __syncthreads();

    // basis functions of the tile
    for (int t = threadIdx.x; t < NF * EX_AT; t += blockDim.x) {
        const int f = t / EX_AT, ia = t % EX_AT, i = i0 + ia;
        double *Pf = P + (size_t) f * EX_LT * (EX_AT + 1) + ia;
        if (i < nh) {
            const double x = mup[nh + i];
            const size_t o = (((size_t) it.lt * NF + f) * nh + i) * 2;
            double prev = ckpt[C.ck_off + o], cur = ckpt[C.ck_off + o + 1];
            constexpr int first = KIND == 1 ? 2 : 3;
            for (int u = 0; u < lt; ++u) {
                const int l = l0 + u;
                const double v = l < first ? basis_first<KIND>(f, l, x) : basis_step<KIND>(f, rcs + 8 * u, x, cur, prev);
                prev = cur;
                cur = v;
                Pf[u * (EX_AT + 1)] = v;
            }
            for (int u = lt; u < EX_LT; ++u) Pf[u * (EX_AT + 1)] = 0.;
        } else {
            for (int u = 0; u < EX_LT; ++u) Pf[u * (EX_AT + 1)] = 0.;
        }
    }
    // weighted moments of the node pairs (u* at the mirror node -mu_i, v* at
    // +mu_i), folded for either order parity: s = (-1)^l multiplies the mirror
    // node's terms.  The two parities sit side by side, so the lanes of a warp
    // (consecutive orders) read one 16-byte pair.
    for (int t = threadIdx.x; t < ncol * EX_AT; t += blockDim.x) {
        const int col = t / EX_AT, ia = t % EX_AT, i = i0 + ia;
        double u0 = 0., u1 = 0., u2 = 0., u3 = 0., v0 = 0., v1 = 0., v2 = 0., v3 = 0.;
        if (i < nh) {
            const int i1 = nh - 1 - i, i2 = nh + i;
            const double w = wqp[i2];
            const double *F = pfn + C.pf_off + (size_t) col * 4 * nq;
            u0 = F[i1] * w; u1 = F[nq + i1] * w; u2 = F[2 * nq + i1] * w; u3 = F[3 * nq + i1] * w;
            v0 = F[i2] * w; v1 = F[nq + i2] * w; v2 = F[2 * nq + i2] * w; v3 = F[3 * nq + i2] * w;
        }
        double *bv = Bv + ((size_t) col * NM * EX_AT + ia) * 2;
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            const double sg = p ? -1. : 1.;
            if (KIND == 0) {
                // acc0 = p00 m0; acc1 = p2-2 m1 + p2+2 m2; acc2 = p2+2 m3 + p2-2 m4;
                // acc3 = p00 m5; acc4 = p0+2 m6; acc5 = p0+2 m7
                bv[(0 * EX_AT) * 2 + p] = sg * u0 + v0;
                bv[(1 * EX_AT) * 2 + p] = sg * (u0 + u1);
                bv[(2 * EX_AT) * 2 + p] = v0 + v1;
                bv[(3 * EX_AT) * 2 + p] = sg * (u0 - u1);
                bv[(4 * EX_AT) * 2 + p] = v0 - v1;
                bv[(5 * EX_AT) * 2 + p] = sg * u1 + v1;
                bv[(6 * EX_AT) * 2 + p] = sg * u2 + v2;
                bv[(7 * EX_AT) * 2 + p] = sg * u3 + v3;
            } else {
                bv[(0 * EX_AT) * 2 + p] = sg * u0 + v0;
                bv[(1 * EX_AT) * 2 + p] = sg * u0 + v0;
                bv[(2 * EX_AT) * 2 + p] = sg * u1 + v1;
                bv[(3 * EX_AT) * 2 + p] = sg * u1 + v1;
                bv[(4 * EX_AT) * 2 + p] = sg * u2 + v2;
                bv[(5 * EX_AT) * 2 + p] = sg * u3 + v3;
            }
        }
    }
    __syncthreads();
    // contraction over the tile's node pairs
    for (int t = threadIdx.x; t < ncol * lt; t += blockDim.x) {
        const int col = t / lt, u = t % lt;
        const int l = l0 + u;
        const double *bv = Bv + (size_t) col * NM * EX_AT * 2 + (l & 1);
        double acc[6] = {0., 0., 0., 0., 0., 0.};
        if (KIND == 0) {
            const double *P00 = P + (size_t) (0 * EX_LT + u) * (EX_AT + 1);
            const double *P02 = P + (size_t) (1 * EX_LT + u) * (EX_AT + 1);
            const double *P22 = P + (size_t) (2 * EX_LT + u) * (EX_AT + 1);
            const double *P2m = P + (size_t) (3 * EX_LT + u) * (EX_AT + 1);
#pragma unroll 4
            for (int ia = 0; ia < EX_AT; ++ia) {
                const double p00 = P00[ia], p02 = P02[ia], p22 = P22[ia], p2m = P2m[ia];
                const double *m = bv + 2 * ia;
                acc[0] += p00 * m[0 * EX_AT * 2];
                acc[1] += p2m * m[1 * EX_AT * 2];
                acc[1] += p22 * m[2 * EX_AT * 2];
                acc[2] += p22 * m[3 * EX_AT * 2];
                acc[2] += p2m * m[4 * EX_AT * 2];
                acc[3] += p00 * m[5 * EX_AT * 2];
                acc[4] += p02 * m[6 * EX_AT * 2];
                acc[5] += p02 * m[7 * EX_AT * 2];
            }
        } else {
            const double *Y = P + (size_t) u * (EX_AT + 1);
#pragma unroll 4
            for (int ia = 0; ia < EX_AT; ++ia) {
                const double y = Y[ia];
                const double *m = bv + 2 * ia;
#pragma unroll
                for (int e = 0; e < 6; ++e) acc[e] += y * m[e * EX_AT * 2];
            }
        }
        double *o = exq + C.ex_off + ((size_t) it.at * ncol + col) * 6 * ncf + l;
#pragma unroll
        for (int e = 0; e < 6; ++e) o[(size_t) e * ncf] = acc[e];
    }
}

// K4c: sum of the angle tiles in order, recombination, (2l+1)/2 scaling,
// zeroed beta_0 derivative and the truncation search (first l with
// |coef_0(l)| <= accuracy).
template <int KIND>
__global__ void k_exp_final(DevBatch B, long long total, const long long *__restrict__ start,
                            const double *__restrict__ exq, double *__restrict__ coefs, int *__restrict__ trunc,
                            int *__restrict__ band) {
    const long long e = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const int c = find_case(start, B.ncase, e);
    const DevCase &C = B.cs[c];
    const long long local = e - start[c];
    const int ncf = C.n_coef, ncol = 1 + B.nd;
    const int col = (int) (local / ncf), l = (int) (local % ncf);
    const int nat = (C.nh + EX_AT - 1) / EX_AT;
    double v[6] = {0., 0., 0., 0., 0., 0.};
    for (int at = 0; at < nat; ++at) {
        const double *q = exq + C.ex_off + ((size_t) at * ncol + col) * 6 * ncf + l;
#pragma unroll
        for (int k = 0; k < 6; ++k) v[k] += q[(size_t) k * ncf];
    }
    if (KIND == 0) {
        const double t = v[1];
        v[1] = (t + v[2]) / 2.;
        v[2] = (t - v[2]) / 2.;
    } else {
        v[5] = -v[5];
    }
    const double sc = (2. * l + 1.) / 2.;
#pragma unroll
    for (int k = 0; k < 6; ++k) v[k] *= sc;
    if (col > 0 && l == 0) v[0] = 0.;
    double *o = coefs + (KIND == 0 ? C.gc_off : C.lc_off) + (size_t) col * 6 * ncf;
#pragma unroll
    for (int k = 0; k < 6; ++k) o[(size_t) k * ncf + l] = v[k];
    if (col == 0 && fabs(v[0]) <= C.accuracy) atomicMax(trunc + c, ncf - l);
    if (col == 0 && C.trunc_band > 0.) {
        // where |beta_l| first comes within the band of `accuracy` from above and
        // from below: the truncation is certain when neither lies on another l
        const double d = C.trunc_band * (2. * l + 1.);
        if (fabs(v[0]) <= C.accuracy + d) atomicMax(band + 2 * c, ncf - l);
        if (fabs(v[0]) <= C.accuracy - d) atomicMax(band + 2 * c + 1, ncf - l);
    }
}

// ---------------------------------------------------------------------------
// K5: phase matrix at the user's angles from the truncated expansion; one
// block per (case, tile of PU_T user angles, part of B.pu_lp orders), one
// thread per angle, cases with the most orders first.  A block runs the basis
// recurrences from order 0 and sums the terms of its part's orders, so that a
// case with many orders is spread over several blocks instead of one long
// chain; a case of several parts writes their sums to scr, added up in order
// by k_phase_user_sum.  The basis functions of an order are generated once
// per angle and used by up to CG columns at a time; the expansion
// coefficients of those columns (GSF: with the a2 +- a3 pair combined) and the
// recurrence coefficients of PU_T orders at a time are staged in shared
// memory, which all threads read.
// ---------------------------------------------------------------------------
template <int KIND, int CG>
__global__ void __launch_bounds__(PU_T) k_phase_user(DevBatch B, const long long *__restrict__ start,
                                                     const double *__restrict__ coefs,
                                                     const int *__restrict__ trunc, double *__restrict__ out,
                                                     double *__restrict__ scr) {
    __shared__ double cfs[CG][6][PU_T], rcs[8 * PU_T];
    const int kr = find_case(start, B.ncase, blockIdx.x);
    const int c = B.k1ord[kr];
    const DevCase &C = B.cs[c];
    const int na = C.n_angles, ncf = C.n_coef, ncol = 1 + B.nd;
    const int ntile = (na + PU_T - 1) / PU_T;
    const int local = (int) (blockIdx.x - start[kr]);
    const int part = local / ntile, tile = local - part * ntile;
    const int a = tile * PU_T + threadIdx.x;
    const bool act = a < na;
    const int nt = trunc[c] > 0 ? ncf - trunc[c] + 1 : ncf;
    // this block's orders [lbeg, lend); the tiles of PU_T orders before lbeg
    // only advance the recurrences (pu_lp is a multiple of PU_T)
    const int lbeg = part * B.pu_lp, lend = min(nt, lbeg + B.pu_lp);
    const double x = act ? B.mu_user[C.mu_user_off + a] : 0.;
    const double *cf0 = coefs + (KIND == 0 ? C.gc_off : C.lc_off);
    for (int g0 = 0; g0 < ncol; g0 += CG) {
        const int ng = min(CG, ncol - g0);
        double s[CG][6];
#pragma unroll
        for (int g = 0; g < CG; ++g)
#pragma unroll
            for (int e = 0; e < 6; ++e) s[g][e] = 0.;
        double q[4] = {0., 0., 0., 0.}, p[4] = {0., 0., 0., 0.};
        for (int l0 = 0; l0 < lend; l0 += PU_T) {
            const int lt = min(PU_T, lend - l0);
            const bool sum = l0 >= lbeg;
            __syncthreads();
            for (int t = threadIdx.x; sum && t < ng * PU_T; t += PU_T) {
                const int g = t / PU_T, u = t % PU_T;
                const double *cf = cf0 + (size_t) (g0 + g) * 6 * ncf + l0 + u;
                double v[6] = {0., 0., 0., 0., 0., 0.};
                if (u < lt)
#pragma unroll
                    for (int e = 0; e < 6; ++e) v[e] = cf[(size_t) e * ncf];
                if (KIND == 0) {
                    const double a2 = v[1], a3 = v[2];
                    v[1] = a2 + a3;
                    v[2] = a2 - a3;
                }
#pragma unroll
                for (int e = 0; e < 6; ++e) cfs[g][e][u] = v[e];
            }
            for (int t = threadIdx.x; t < 8 * lt; t += PU_T) rcs[t] = B.rc[8 * (size_t) l0 + t];
            __syncthreads();
            for (int u = 0; u < lt; ++u) {
                const int l = l0 + u;
                const double *rl = rcs + 8 * u;                       // recurrence coefficients of order l
                if (KIND == 0) {
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        const double v = l < 3 ? basis_first<0>(f, l, x) : basis_step<0>(f, rl, x, p[f], q[f]);
                        q[f] = p[f];
                        p[f] = v;
                    }
                    if (!sum) continue;
#pragma unroll
                    for (int g = 0; g < CG; ++g) {
                        s[g][0] += cfs[g][0][u] * p[0];
                        s[g][3] += cfs[g][3][u] * p[0];
                        if (l >= 2) {
                            s[g][4] += cfs[g][4][u] * p[1];
                            s[g][5] += cfs[g][5][u] * p[1];
                            s[g][1] += cfs[g][1][u] * p[2];
                            s[g][2] += cfs[g][2][u] * p[3];
                        }
                    }
                } else {
                    const double v = l < 2 ? basis_first<1>(0, l, x) : basis_step<1>(0, rl, x, p[0], q[0]);
                    q[0] = p[0];
                    p[0] = v;
                    if (!sum) continue;
#pragma unroll
                    for (int g = 0; g < CG; ++g)
#pragma unroll
                        for (int e = 0; e < 6; ++e) s[g][e] += cfs[g][e][u] * v;
                }
            }
        }
        if (act) {
#pragma unroll
            for (int g = 0; g < CG; ++g) {
                if (g >= ng) break;
                double *o = (C.pu_parts > 1 ? scr + C.pu_scr_off + (size_t) part * ncol * 6 * na
                                            : out + C.pf_out_off) + (size_t) (g0 + g) * 6 * na;
                if (KIND == 0) {
                    o[a] = s[g][0];
                    o[(size_t) 3 * na + a] = s[g][3];
                    o[(size_t) 4 * na + a] = s[g][4];
                    o[(size_t) 5 * na + a] = s[g][5];
                    o[(size_t) 1 * na + a] = (s[g][1] + s[g][2]) / 2.;
                    o[(size_t) 2 * na + a] = (s[g][1] - s[g][2]) / 2.;
                } else {
                    o[a] = s[g][0];
                    o[(size_t) 1 * na + a] = s[g][1];
                    o[(size_t) 2 * na + a] = s[g][2];
                    o[(size_t) 3 * na + a] = s[g][3];
                    o[(size_t) 4 * na + a] = s[g][4];
                    o[(size_t) 5 * na + a] = -s[g][5];
                }
            }
        }
    }
}

// The phase matrix of cases of several K5 parts: thread per (case, column,
// element, angle) of the flat space `start`, the parts' sums added in order.
__global__ void k_phase_user_sum(DevBatch B, long long total, const long long *__restrict__ start,
                                 const double *__restrict__ scr, double *__restrict__ out) {
    const long long e = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const int c = find_case(start, B.ncase, e);
    const DevCase &C = B.cs[c];
    const long long local = e - start[c], n = (long long) (1 + B.nd) * 6 * C.n_angles;
    const double *sp = scr + C.pu_scr_off + local;
    double v = sp[0];
    for (int p = 1; p < C.pu_parts; ++p) v += sp[(size_t) p * n];
    out[C.pf_out_off + local] = v;
}

template <int NC1, int NC2>
constexpr int angular_ap() { return 1; }

template <int NC1, int NC2>
size_t angular_smem() {
    return sizeof(double4) * ANG_KT * (1 + NC1) + sizeof(double) * ANG_KT +
           sizeof(double) * angular_ap<NC1, NC2>() * (1 + NC1 + NC2) * 8 * ANG_T;
}

template <int NC1, int NC2>
int run_angular(cudaStream_t s, const DevBatch &B, int c1base, int c2base, int first, int nitems,
                const AngItem *items, const double *coef, double *part, double *save2) {
    constexpr int AP = angular_ap<NC1, NC2>();
    const size_t sm = angular_smem<NC1, NC2>();
    static bool attr = false;
    if (!attr) {
        LMIEB_CUDA_TRY(cudaFuncSetAttribute(k_angular<NC1, NC2, AP>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm));
        attr = true;
    }
    k_angular<NC1, NC2, AP><<<nitems, ANG_T, sm, s>>>(B, c1base, c2base, first, items, coef, part, save2);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}

template <int NC1>
int run_angular_nc2(cudaStream_t s, const DevBatch &B, int nc2, int c1base, int c2base, int first, int nitems,
                    const AngItem *items, const double *coef, double *part, double *save2) {
    switch (nc2) {
    case 0: return run_angular<NC1, 0>(s, B, c1base, c2base, first, nitems, items, coef, part, save2);
    case 1: return run_angular<NC1, 1>(s, B, c1base, c2base, first, nitems, items, coef, part, save2);
    case 2: return run_angular<NC1, 2>(s, B, c1base, c2base, first, nitems, items, coef, part, save2);
    case 3: return run_angular<NC1, 3>(s, B, c1base, c2base, first, nitems, items, coef, part, save2);
    case 4: return run_angular<NC1, 4>(s, B, c1base, c2base, first, nitems, items, coef, part, save2);
    }
    return -1;
}

template <int KIND>
int run_expand(cudaStream_t s, const DevBatch &B, long long nck, const long long *ck_start,
               int nitems, const ExpItem *items, int nruns, const ExpItem *runs, long long nfin,
               const long long *fin_start, const double *pfn, double *ckpt, double *exq, double *coefs,
               int *trunc, int *band) {
    constexpr int NF = KIND == 0 ? 4 : 1;
    constexpr int SMAX = 200 * 1024;
    constexpr int NM = KIND == 0 ? 8 : 6;
    const size_t sm = sizeof(double) * ((size_t) NF * EX_LT * (EX_AT + 1) + (size_t) (1 + B.nd) * NM * EX_AT * 2 +
                                        (size_t) 8 * EX_LT);
    if (sm > (size_t) SMAX) {
        fprintf(stderr, "ERROR: expansion tile needs %zu bytes of shared memory (too many derivatives)\n", sm);
        return -1;
    }
    static bool attr = false;
    if (!attr) {
        LMIEB_CUDA_TRY(cudaFuncSetAttribute(k_exp_tile<KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMAX));
        attr = true;
    }
    const int ncol = 1 + B.nd;
    if (KIND == 0 && expand_gsf_launches(ncol) == 1) {
        // the GSF contraction on the FP64 tensor cores, one block per (case, angle tile)
        const size_t smm = sizeof(double) * ((size_t) EX_AF + ex_bf_run_size(ncol) + (size_t) 2 * 8 * EX_LT);
        static bool attr_mma = false;
        if (!attr_mma) {
            LMIEB_CUDA_TRY(cudaFuncSetAttribute(k_exp_gsf, cudaFuncAttributeMaxDynamicSharedMemorySize, SMAX));
            attr_mma = true;
        }
        if (nruns > 0) k_exp_gsf<<<nruns, 128, smm, s>>>(B, runs, pfn, exq);
    } else {
        k_exp_ckpt<KIND><<<ceil_div(nck, 128), 128, 0, s>>>(B, nck, ck_start, ckpt);
        LMIEB_CUDA_TRY(cudaGetLastError());
        const int nt = std::min(EX_TMAX, std::max(128, (ncol * EX_LT + 31) / 32 * 32));
        k_exp_tile<KIND><<<nitems, nt, sm, s>>>(B, items, pfn, ckpt, exq);
    }
    LMIEB_CUDA_TRY(cudaGetLastError());
    k_exp_final<KIND><<<ceil_div(nfin, 256), 256, 0, s>>>(B, nfin, fin_start, exq, coefs, trunc, band);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
int launch_gauss(cudaStream_t s, int npairs, const int *pt, const int *pi, const int *ns, const long long *mo,
                 const long long *go, const double *guess, const double *jr, double *pool) {
    if (npairs <= 0) return 0;
    k_gauss<<<ceil_div(npairs, 32), 32, 0, s>>>(npairs, pt, pi, ns, mo, go, guess, jr, pool, pool);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}

namespace {
// the radius group's failure count after its sum: nonzero -> error word 2
__global__ void k_group_flag(const double *__restrict__ failed, int *__restrict__ err) {
    if (*failed != 0.) *err = 2;
}
}  // namespace

int launch_group_flag(cudaStream_t s, const double *failed, int *err) {
    k_group_flag<<<1, 1, 0, s>>>(failed, err);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int launch_coef(cudaStream_t s, const DevBatch &B, int nc, int c0, int write_value, double *ck, double *coef,
                float *bop, double *rs) {
    const unsigned rb = ceil_div(B.R, 64);
    switch (nc) {
#define LMIEB_K1(NC_)                                                                                    \
    case NC_:                                                                                            \
        k_mie<NC_><<<rb, 64, bop ? 4 * 8 * (1 + NC_) * 64 * sizeof(float) : 0, s>>>(B, c0, write_value, ck,   \
                                                                                  coef, bop, rs);        \
        break;
    LMIEB_K1(0)
    LMIEB_K1(1)
    LMIEB_K1(2)
    LMIEB_K1(3)
    LMIEB_K1(4)
#undef LMIEB_K1
    default:
        fprintf(stderr, "ERROR: launch_coef: bad chunk width %d\n", nc);
        return -1;
    }
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}

namespace {
__global__ void __launch_bounds__(256) k_gather(const GatherSeg *__restrict__ segs, double *__restrict__ coef,
                                               double *__restrict__ rs) {
    const GatherSeg g = segs[blockIdx.x];
    double *dst = (g.which ? rs : coef) + g.dst_off;
    for (long long i = threadIdx.x; i < g.n; i += blockDim.x) dst[i] = g.src[i];
}
}  // namespace

int launch_gather(cudaStream_t s, int nseg, const GatherSeg *segs, double *coef, double *rs) {
    if (nseg <= 0) return 0;
    k_gather<<<nseg, 256, 0, s>>>(segs, coef, rs);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int launch_reduce_scalars(cudaStream_t s, const DevBatch &B, const double *rs, double *sums, double *save1) {
    dim3 grid(B.ncase, 1 + B.nd);
    k_reduce_scalars<<<grid, 256, 0, s>>>(B, rs, sums, save1);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int angular_angles_per_block(int) { return ANG_T; }

int launch_angular(cudaStream_t s, const DevBatch &B, int nc1, int c1base, int nc2, int c2base, int first,
                   int nitems, const AngItem *items, const double *coef, double *part, double *save2) {
    if (nitems <= 0) return 0;
    switch (nc1) {
    case 0: return run_angular_nc2<0>(s, B, nc2, c1base, c2base, first, nitems, items, coef, part, save2);
    case 1: return run_angular_nc2<1>(s, B, nc2, c1base, c2base, first, nitems, items, coef, part, save2);
    case 2: return run_angular_nc2<2>(s, B, nc2, c1base, c2base, first, nitems, items, coef, part, save2);
    case 3: return run_angular_nc2<3>(s, B, nc2, c1base, c2base, first, nitems, items, coef, part, save2);
    case 4: return run_angular_nc2<4>(s, B, nc2, c1base, c2base, first, nitems, items, coef, part, save2);
    }
    fprintf(stderr, "ERROR: launch_angular: bad chunk width %d\n", nc1);
    return -1;
}

int launch_reduce_pf(cudaStream_t s, const DevBatch &B, long long total, const long long *start,
                     const double *part, double *pfacc) {
    if (total <= 0) return 0;
    k_reduce_pf<<<ceil_div(total, 256), 256, 0, s>>>(B, total, start, part, pfacc);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int launch_save_reweight(cudaStream_t s, const DevBatch &B, int n_qang, const double *save1, const double *save2,
                         const double *w2, double *sums, double *pfacc) {
    k_save_reweight_scal<<<1, 32 * ceil_div(1 + B.nd, 32), 0, s>>>(B, save1, w2, sums);
    LMIEB_CUDA_TRY(cudaGetLastError());
    if (n_qang > 0) {
        k_save_reweight_pf<<<ceil_div((size_t) 4 * n_qang, 128), 128, 0, s>>>(B, n_qang, save2, w2, pfacc);
        LMIEB_CUDA_TRY(cudaGetLastError());
    }
    return 0;
}

int launch_normalize(cudaStream_t s, const DevBatch &B, long long total, const long long *start,
                     const double *sums, const double *pfacc, double *scal, double *pfn) {
    if (total > 0) {
        k_normalize_pf<<<ceil_div(total, 256), 256, 0, s>>>(B, total, start, sums, pfacc, pfn);
        LMIEB_CUDA_TRY(cudaGetLastError());
    }
    k_normalize_scal<<<ceil_div(B.ncase, 128), 128, 0, s>>>(B, sums, scal);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int expand_gsf_launches(int ncol) { return 2 * ncol <= 8 * EX_NB ? 1 : 2; }

int launch_expand(cudaStream_t s, const DevBatch &B, int kind, long long nck,
                  const long long *ck_start, int nitems, const ExpItem *items, int nruns, const ExpItem *runs,
                  long long nfin, const long long *fin_start, const double *pfn, double *ckpt, double *exq,
                  double *coefs, int *trunc, int *band) {
    if (nitems <= 0) return 0;
    if (kind == 0)
        return run_expand<0>(s, B, nck, ck_start, nitems, items, nruns, runs, nfin, fin_start, pfn, ckpt, exq,
                             coefs, trunc, band);
    return run_expand<1>(s, B, nck, ck_start, nitems, items, 0, nullptr, nfin, fin_start, pfn, ckpt, exq, coefs,
                         trunc, band);
}

int launch_phase_user(cudaStream_t s, const DevBatch &B, int kind, long long total, const long long *start,
                      const double *coefs, const int *trunc, double *pf_out, double *scr, long long nred,
                      const long long *red_start) {
    if (total <= 0) return 0;
    const int ncol = 1 + B.nd;
    const unsigned nb = (unsigned) total;
    if (kind == 0) {
        if (ncol == 1) k_phase_user<0, 1><<<nb, PU_T, 0, s>>>(B, start, coefs, trunc, pf_out, scr);
        else if (ncol <= 3) k_phase_user<0, 3><<<nb, PU_T, 0, s>>>(B, start, coefs, trunc, pf_out, scr);
        else k_phase_user<0, 5><<<nb, PU_T, 0, s>>>(B, start, coefs, trunc, pf_out, scr);
    } else {
        if (ncol == 1) k_phase_user<1, 1><<<nb, PU_T, 0, s>>>(B, start, coefs, trunc, pf_out, scr);
        else if (ncol <= 3) k_phase_user<1, 3><<<nb, PU_T, 0, s>>>(B, start, coefs, trunc, pf_out, scr);
        else k_phase_user<1, 5><<<nb, PU_T, 0, s>>>(B, start, coefs, trunc, pf_out, scr);
    }
    LMIEB_CUDA_TRY(cudaGetLastError());
    if (nred > 0) {
        k_phase_user_sum<<<ceil_div(nred, 256), 256, 0, s>>>(B, nred, red_start, scr, pf_out);
        LMIEB_CUDA_TRY(cudaGetLastError());
    }
    return 0;
}
