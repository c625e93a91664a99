// k_fp64.cu -- the FP64 kernels of the drop-in solve (sm_100a).
//
//   k_gauss          Gauss-Legendre angles on [-1,1]        <- misc/rtutil_math.c:73-129,231-316
//   k_coef<NC>       per-radius recurrences, a_n, b_n, their tangent-linear
//                    forms, expansion coefficients and per-radius sums
//                                                           <- src/lmie_core.c:263-652
//   k_reduce_scalars radius reduction of Cext/Csca/Cbak/g    <- src/lmie_core.c:537-611,
//                                                              src/lmie_schedule.c:334-338
//   k_angular<..>    S1/S2 accumulation over orders and the phase-matrix
//                    quadratic forms, reduced over a radius group
//                                                           <- src/lmie_core.c:658-791
//   k_reduce_pf      fixed-order sum over radius groups
//   k_normalize      2/Csca and lambda^2/2pi normalisation   <- src/lmie_schedule.c:1155-1199
//   k_gsf_* / k_leg_* expansion coefficients over Gauss angles
//                                                           <- misc/rtutil_scat_int.c:20-230,353-480,
//                                                              misc/rtutil_math.c:477-513,936-1017
//   k_phase_user     phase matrix at the user's angles       <- misc/rtutil_scat_int.c:510-589,662-710
//
// All reductions run in a fixed order, so a solve is bit-reproducible.
#include <cstdio>

#include "kernels.h"

namespace {

// ---------------------------------------------------------------------------
// Gauss-Legendre nodes: one thread per root pair, Newton with the
// second-order correction of Davis & Rabinowitz.  The initial guesses come
// from the host (libm cos/tan) and every operation is an explicit
// round-to-nearest intrinsic (no FMA contraction), so the nodes are the
// reference's to the last bit -- at size parameters ~1000 the phase matrix
// changes by ~1e-10 per ulp of a node.
// ---------------------------------------------------------------------------
__global__ void k_gauss(int n, const double *__restrict__ guess, double *mu, double *wq) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int half = (n + 1) / 2;
    if (i >= half) return;
    const double dn = (double) n;
    const double ib = (double) (n * (n + 1));
    double y = guess[i], y_prev, pn, pm, pmm, t, d1, d2;
    int it = 0;
    do {
        pm = 0.;
        pn = 1.;
        for (int j = 0; j < n; ++j) {
            pmm = pm;
            pm = pn;
            t = __dmul_rn(y, pm);
            pn = __dadd_rn(__dmul_rn(__ddiv_rn((double) j, (double) j + 1.), __dsub_rn(t, pmm)), t);
        }
        t = __dsub_rn(1., __dmul_rn(y, y));
        d1 = __ddiv_rn(__dmul_rn(dn, __dsub_rn(pm, __dmul_rn(y, pn))), t);
        d2 = __ddiv_rn(__dsub_rn(__dmul_rn(__dmul_rn(2., y), d1), __dmul_rn(ib, pn)), t);
        y_prev = y;
        t = __ddiv_rn(pn, d1);
        y = __dsub_rn(y_prev, __dmul_rn(t, __dadd_rn(1., __ddiv_rn(__dmul_rn(t, d2), __dmul_rn(2., d1)))));
    } while (fabs(__dsub_rn(y, y_prev)) > 2.220446049250313e-16 && ++it < 100);
    double de = __dmul_rn(dn, pm);
    de = __ddiv_rn(2., __dmul_rn(de, de));
    mu[i] = -y;
    mu[n - 1 - i] = y;
    wq[i] = __dmul_rn(__dsub_rn(1., __dmul_rn(y, y)), de);
    wq[n - 1 - i] = wq[i];
}

// ---------------------------------------------------------------------------
// K1: one thread per radius.  Downward passes (D_n from n2, psi ratio from
// n1) store their values for orders 1..n1 in order-major scratch (coalesced
// across the radii of a warp); one upward pass then forms psi, chi, zeta,
// a_n, b_n, the NC tangent-linear columns, the expansion coefficients and
// the per-radius cross-section and asymmetry sums.
// ---------------------------------------------------------------------------
template <int NC>
__global__ void __launch_bounds__(128) k_coef(DevProblem P, int c0, int write_value, int r0, int nb,
                                              int jmax, double *__restrict__ scr_r,
                                              double *__restrict__ scr_d, double *__restrict__ coef,
                                              double *__restrict__ rs) {
    const int rb = blockIdx.x * blockDim.x + threadIdx.x;
    if (rb >= nb) return;
    const int r = r0 + rb;
    const int n = P.n;
    const int n1 = P.n1r[r], n2 = P.n2r[r];
    const double x = P.x[r];
    const double xinv = 1. / x;
    const cplx m = P.m, minv = P.minv, m2 = P.m2;
    const cplx z = mk(m.re * x, m.im * x);
    const cplx zinv = 1. / z;
    const double *fv1 = P.fv, *fv3 = P.fv + 2 * (P.n1 + 2), *fv4 = P.fv + 3 * (P.n1 + 2);

    double xl[NC > 0 ? NC : 1];
    cplx zl[NC > 0 ? NC : 1], ml[NC > 0 ? NC : 1];
#pragma unroll
    for (int k = 0; k < NC; ++k) {
        int kk = P.idx1[c0 + k];
        xl[k] = P.xl[(size_t) (c0 + k) * n + r];
        ml[k] = P.m_l[kk];
        zl[k] = ml[k] * x + m * xl[k];
    }

    // scratch column c (0 = value, 1+k = derivative k) at order j
#define SCR_R(c, j) scr_r[((size_t) (c) * jmax + (j)) * nb + rb]
#define SCR_D(c, j) (((double2 *) scr_d)[((size_t) (c) * jmax + (j)) * nb + rb])

    // D_n(z) downward from D_{n2} = 0; orders 1..n1 are kept
    {
        cplx D = mk(0., 0.);
        cplx Dl[NC > 0 ? NC : 1];
#pragma unroll
        for (int k = 0; k < NC; ++k) Dl[k] = mk(0., 0.);
        for (int j = n2 - 1; j >= 1; --j) {
            cplx c1 = (j + 1.) * zinv;
            cplx c2 = D + c1;
            cplx ic2 = 1. / c2;
            D = c1 - ic2;
            if (NC > 0) {
                cplx c3 = -c1 * zinv;
                cplx ic4 = ic2 * ic2;
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    cplx c5 = c3 * zl[k];
                    Dl[k] = c5 + (Dl[k] + c5) * ic4;
                }
            }
            if (j <= n1) {
                SCR_D(0, j) = make_double2(D.re, D.im);
#pragma unroll
                for (int k = 0; k < NC; ++k) SCR_D(1 + k, j) = make_double2(Dl[k].re, Dl[k].im);
            }
        }
    }
    // psi_j / psi_{j-1} downward from r_{n1} = 0
    {
        double rn = 0., rl[NC > 0 ? NC : 1];
#pragma unroll
        for (int k = 0; k < NC; ++k) rl[k] = 0.;
        SCR_R(0, n1) = 0.;
#pragma unroll
        for (int k = 0; k < NC; ++k) SCR_R(1 + k, n1) = 0.;
        for (int j = n1 - 1; j >= 1; --j) {
            double a1 = fv1[j] * xinv;
            double rnew = 1. / (a1 - rn);
            if (NC > 0) {
                double a2 = -a1 * xinv, a3 = rnew * rnew;
#pragma unroll
                for (int k = 0; k < NC; ++k) rl[k] = -(a2 * xl[k] - rl[k]) * a3;
            }
            rn = rnew;
            SCR_R(0, j) = rn;
#pragma unroll
            for (int k = 0; k < NC; ++k) SCR_R(1 + k, j) = rl[k];
        }
    }

    // upward pass
    double sinx, cosx;
    sincos(x, &sinx, &cosx);
    double psi_p = sinx, chi_p = cosx, chi_c = xinv * cosx + sinx;
    double psil_p[NC > 0 ? NC : 1], chil_p[NC > 0 ? NC : 1], chil_c[NC > 0 ? NC : 1];
#pragma unroll
    for (int k = 0; k < NC; ++k) {
        psil_p[k] = xl[k] * cosx;
        chil_p[k] = xl[k] * -sinx;
        chil_c[k] = (-xinv * xinv) * xl[k] * cosx + xinv * chil_p[k] + xl[k] * cosx;
    }
    double se = 0., ss = 0., sg = 0., sgn = -1.;
    cplx sb = mk(0., 0.), a_p = mk(0., 0.), b_p = mk(0., 0.);
    double sel[NC > 0 ? NC : 1], ssl[NC > 0 ? NC : 1], sgl[NC > 0 ? NC : 1];
    cplx sbl[NC > 0 ? NC : 1], al_p[NC > 0 ? NC : 1], bl_p[NC > 0 ? NC : 1];
#pragma unroll
    for (int k = 0; k < NC; ++k) {
        sel[k] = ssl[k] = sgl[k] = 0.;
        sbl[k] = al_p[k] = bl_p[k] = mk(0., 0.);
    }
    const size_t tot = (size_t) P.tot;
    double2 *cf = (double2 *) coef;
    const size_t obase = (size_t) P.off[r];

    for (int j = 1; j <= n1; ++j) {
        const double rj = SCR_R(0, j);
        const double2 Dv = SCR_D(0, j);
        const cplx D = mk(Dv.x, Dv.y);
        const double psi = rj * psi_p;
        const cplx zeta = mk(psi, chi_c), zeta_p = mk(psi_p, chi_p);
        const double t = j * xinv;

        const cplx ca = D * minv + t;
        const cplx na = ca * psi - psi_p;
        const cplx da = ca * zeta - zeta_p;
        const cplx ida = 1. / da;
        const cplx a = na * ida;
        const cplx cb = m * D + t;
        const cplx nbv = cb * psi - psi_p;
        const cplx db = cb * zeta - zeta_p;
        const cplx idb = 1. / db;
        const cplx b = nbv * idb;

        const double f4 = fv4[j], f1 = fv1[j];
        se += f1 * (a.re + b.re);
        ss += f1 * (norm2(a) + norm2(b));
        sb = sb + (a - b) * (f1 * sgn);
        if (j >= 2) sg += fv3[j - 1] * (re_mulc(a_p, a) + re_mulc(b_p, b)) + fv4[j - 1] * re_mulc(a_p, b_p);

        if (write_value) {
            const cplx cs = (a + b) * f4, cd = (a - b) * f4;
            const size_t o = obase + j - 1;
            cf[o * 2] = make_double2(cs.re, cs.im);
            cf[o * 2 + 1] = make_double2(cd.re, cd.im);
        }

        const cplx Dm2 = D * (minv * minv);
        const double tx = -t * xinv;
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            const double rl = SCR_R(1 + k, j);
            const double2 Dlv = SCR_D(1 + k, j);
            const cplx Dl = mk(Dlv.x, Dlv.y);
            const double psil = rl * psi_p + rj * psil_p[k];
            const cplx zetal = mk(psil, chil_c[k]), zetal_p = mk(psil_p[k], chil_p[k]);
            const double tl = tx * xl[k];
            const cplx c6 = Dl * minv - Dm2 * ml[k] + tl;
            const cplx al = (c6 * psi + ca * psil - psil_p[k]) * ida -
                            na * ((c6 * zeta + ca * zetal - zetal_p) * (ida * ida));
            const cplx c4 = ml[k] * D + m * Dl + tl;
            const cplx bl = (c4 * psi + cb * psil - psil_p[k]) * idb -
                            nbv * ((c4 * zeta + cb * zetal - zetal_p) * (idb * idb));
            sel[k] += f1 * (al.re + bl.re);
            ssl[k] += f1 * 2. * (re_mulc(a, al) + re_mulc(b, bl));
            sbl[k] = sbl[k] + (al - bl) * (f1 * sgn);
            if (j >= 2)
                sgl[k] += fv3[j - 1] * (re_mulc(al_p[k], a) + re_mulc(a_p, al) + re_mulc(bl_p[k], b) +
                                        re_mulc(b_p, bl)) +
                          fv4[j - 1] * (re_mulc(al_p[k], b_p) + re_mulc(a_p, bl_p[k]));
            const cplx cs = (al + bl) * f4, cd = (al - bl) * f4;
            const size_t o = ((size_t) (1 + c0 + k) * tot + obase + j - 1) * 2;
            cf[o] = make_double2(cs.re, cs.im);
            cf[o + 1] = make_double2(cd.re, cd.im);
            al_p[k] = al;
            bl_p[k] = bl;
            psil_p[k] = psil;
        }
        // advance chi to order j+1
        if (j < n1) {
            const double a1 = fv1[j] * xinv;
            const double chi_n = a1 * chi_c - chi_p;
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                const double a2l = -a1 * xl[k] * xinv;
                const double chil_n = a2l * chi_c + a1 * chil_c[k] - chil_p[k];
                chil_p[k] = chil_c[k];
                chil_c[k] = chil_n;
            }
            chi_p = chi_c;
            chi_c = chi_n;
        }
        psi_p = psi;
        a_p = a;
        b_p = b;
        sgn = -sgn;
    }
#undef SCR_R
#undef SCR_D
    if (write_value) {
        rs[(size_t) 0 * n + r] = se;
        rs[(size_t) 1 * n + r] = ss;
        rs[(size_t) 2 * n + r] = sb.re;
        rs[(size_t) 3 * n + r] = sb.im;
        rs[(size_t) 4 * n + r] = sg;
    }
#pragma unroll
    for (int k = 0; k < NC; ++k) {
        const size_t c = 1 + c0 + k;
        rs[(c * 5 + 0) * n + r] = sel[k];
        rs[(c * 5 + 1) * n + r] = ssl[k];
        rs[(c * 5 + 2) * n + r] = sbl[k].re;
        rs[(c * 5 + 3) * n + r] = sbl[k].im;
        rs[(c * 5 + 4) * n + r] = sgl[k];
    }
}

// ---------------------------------------------------------------------------
// K2: one block per output column; fixed-order block reduction over radii.
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

__global__ void __launch_bounds__(256) k_reduce_scalars(DevProblem P, const double *__restrict__ rs,
                                                        double *__restrict__ sums,
                                                        double *__restrict__ save1) {
    __shared__ double sh[256];
    const int col = blockIdx.x;           // 0 = value, 1+kk = slot kk
    const int n = P.n;
    int kind = 0, c1 = 0;                 // 0 value, 1 index1, 2 index2
    if (col > 0) {
        const int kk = col - 1;
        for (int k = 0; k < P.nd1; ++k)
            if (P.idx1[k] == kk) { kind = 1; c1 = 1 + k; }
        if (kind == 0) kind = 2;
    }
    double acc[4] = {0., 0., 0., 0.};
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        const double f = P.w[r];
        const double se = rs[r], ss = rs[(size_t) n + r];
        const double sbr = rs[(size_t) 2 * n + r], sbi = rs[(size_t) 3 * n + r];
        const double sg = rs[(size_t) 4 * n + r];
        const double bak = sbr * sbr + sbi * sbi;
        if (kind == 0) {
            acc[0] += f * se;
            acc[1] += f * ss;
            acc[2] += f * bak;
            acc[3] += f * sg;
            if (save1) {
                save1[r] = se;
                save1[(size_t) n + r] = ss;
                save1[(size_t) 2 * n + r] = bak;
                save1[(size_t) 3 * n + r] = sg;
            }
        } else if (kind == 1) {
            const double fl = P.w[(size_t) col * n + r];
            const double *q = rs + (size_t) c1 * 5 * n;
            acc[0] += fl * se + f * q[r];
            acc[1] += fl * ss + f * q[(size_t) n + r];
            acc[2] += fl * bak + f * 2. * (sbr * q[(size_t) 2 * n + r] + sbi * q[(size_t) 3 * n + r]);
            acc[3] += fl * sg + f * q[(size_t) 4 * n + r];
        } else {
            const double fl = P.w[(size_t) col * n + r];
            acc[0] += fl * se;
            acc[1] += fl * ss;
            acc[2] += fl * bak;
            acc[3] += fl * sg;
        }
    }
    for (int q = 0; q < 4; ++q) {
        double v = block_sum(acc[q], sh);
        if (threadIdx.x == 0) sums[col * 4 + q] = v;
    }
}

// ---------------------------------------------------------------------------
// K3: one thread per half-angle (mu_j < 0) and its mirror (-mu_j); a block
// covers ANG_T half-angles and one radius group.  For every radius the
// pi_n/tau_n recurrence runs in registers, the coefficient columns are
// staged through shared memory ANG_KT orders at a time, and the quadratic
// forms of S1, S2 are accumulated per thread in shared memory.
// ---------------------------------------------------------------------------
constexpr int ANG_T = 64;
constexpr int ANG_KT = 64;

template <int NC1, int NC2>
__global__ void __launch_bounds__(ANG_T) k_angular(DevProblem P, int c1base, int c2base, int first,
                                                   const int *__restrict__ gstart,
                                                   const double *__restrict__ coef,
                                                   double *__restrict__ part, double *__restrict__ save2) {
    constexpr int C1 = 1 + NC1;
    constexpr int NS = 1 + NC1 + NC2;
    extern __shared__ double4 smem4[];
    double4 *cbuf = smem4;                                   // [ANG_KT][C1] {cs, cd}
    double *fv2s = (double *) (cbuf + ANG_KT * C1);          // [ANG_KT]
    double *acc = fv2s + ANG_KT;                             // [NS*2*4][ANG_T]

    const int tid = threadIdx.x;
    const int jh = blockIdx.x * ANG_T + tid;
    const int g = blockIdx.y;
    const bool act = jh < P.nh;
    const double mu = act ? P.mu[jh] : 0.;
    const int n = P.n;
    const size_t tot = (size_t) P.tot;
    const double *fv2 = P.fv + (P.n1 + 2);
    const double4 *cf = (const double4 *) coef;

    for (int q = 0; q < NS * 8; ++q) acc[q * ANG_T + tid] = 0.;

    int slot1[NC1 > 0 ? NC1 : 1], slot2[NC2 > 0 ? NC2 : 1];
#pragma unroll
    for (int k = 0; k < NC1; ++k) slot1[k] = 1 + P.idx1[c1base + k];
#pragma unroll
    for (int k = 0; k < NC2; ++k) slot2[k] = 1 + P.idx2[c2base + k];

    const int rbeg = gstart[g], rend = gstart[g + 1];
    for (int r = rbeg; r < rend; ++r) {
        const int n1 = P.n1r[r];
        const size_t off = (size_t) P.off[r];
        cplx spA[C1], smA[C1], spB[C1], smB[C1];
#pragma unroll
        for (int c = 0; c < C1; ++c) spA[c] = smA[c] = spB[c] = smB[c] = mk(0., 0.);
        double p0 = 0., p1 = 1., par = 1.;
        for (int k0 = 0; k0 < n1; k0 += ANG_KT) {
            const int kt = min(ANG_KT, n1 - k0);
            __syncthreads();
            for (int idx = tid; idx < kt * C1; idx += ANG_T) {
                const int t = idx / C1, c = idx - t * C1;
                const size_t col = c == 0 ? 0 : (size_t) (c1base + c);
                cbuf[t * C1 + c] = cf[col * tot + off + k0 + t];
            }
            for (int t = tid; t < kt; t += ANG_T) fv2s[t] = fv2[k0 + t + 1];
            __syncthreads();
            if (act) {
                for (int t = 0; t < kt; ++t) {
                    const double kd = (double) (k0 + t + 1);
                    const double t1 = mu * p1, t2 = t1 - p0, tau = kd * t2 - p0;
                    const double tp = p1 + tau, tm = p1 - tau;
                    const double tpB = par * tp, tmB = par * tm;
#pragma unroll
                    for (int c = 0; c < C1; ++c) {
                        const double4 v = cbuf[t * C1 + c];
                        spA[c].re += tp * v.x;  spA[c].im += tp * v.y;
                        smA[c].re += tm * v.z;  smA[c].im += tm * v.w;
                        spB[c].re += tmB * v.x; spB[c].im += tmB * v.y;
                        smB[c].re += tpB * v.z; smB[c].im += tpB * v.w;
                    }
                    par = -par;
                    p0 = p1;
                    p1 = t1 + fv2s[t] * t2;
                }
            }
        }
        if (!act) continue;
        const double f = P.w[r], half_f = f * .5;
        double fl1[NC1 > 0 ? NC1 : 1], fl2[NC2 > 0 ? NC2 : 1];
#pragma unroll
        for (int k = 0; k < NC1; ++k) fl1[k] = P.w[(size_t) slot1[k] * n + r];
#pragma unroll
        for (int k = 0; k < NC2; ++k) fl2[k] = P.w[(size_t) slot2[k] * n + r];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const cplx *sp = h ? spB : spA;
            const cplx *sm = h ? smB : smA;
            const cplx s1 = (sp[0] + sm[0]) * .5, s2 = (sp[0] - sm[0]) * .5;
            const double e1 = norm2(s1), e3 = norm2(s2);
            const cplx c12 = s1 * conjg(s2), c21 = s2 * conjg(s1);
            const double pv[4] = {(e1 + e3) * .5, (c12.re + c21.re) * .5, -(e1 - e3) * .5,
                                  .5 * (c12.im - c21.im)};
            double *a = acc + (h * 4) * ANG_T + tid;
            if (first) {
#pragma unroll
                for (int e = 0; e < 4; ++e) a[e * ANG_T] += f * pv[e];
                if (save2) {
                    const int jj = h ? P.n_qang - 1 - jh : jh;
#pragma unroll
                    for (int e = 0; e < 4; ++e) save2[((size_t) e * n + r) * P.n_qang + jj] = pv[e];
                }
            }
#pragma unroll
            for (int k = 0; k < NC1; ++k) {
                const cplx s1l = (sp[1 + k] + sm[1 + k]) * .5, s2l = (sp[1 + k] - sm[1 + k]) * .5;
                const double q1 = 2. * (s1l.re * s1.re + s1l.im * s1.im);
                const double q3 = 2. * (s2l.re * s2.re + s2l.im * s2.im);
                const cplx d12 = (s1l * conjg(s2)) * 2., d21 = (s2l * conjg(s1)) * 2.;
                double *al = acc + ((1 + k) * 8 + h * 4) * ANG_T + tid;
                al[0] += fl1[k] * pv[0] + half_f * (q1 + q3);
                al[ANG_T] += fl1[k] * pv[1] + half_f * (d12.re + d21.re);
                al[2 * ANG_T] += fl1[k] * pv[2] + half_f * -(q1 - q3);
                al[3 * ANG_T] += fl1[k] * pv[3] + half_f * (d12.im - d21.im);
            }
#pragma unroll
            for (int k = 0; k < NC2; ++k) {
                double *al = acc + ((1 + NC1 + k) * 8 + h * 4) * ANG_T + tid;
#pragma unroll
                for (int e = 0; e < 4; ++e) al[e * ANG_T] += pv[e] * fl2[k];
            }
        }
    }
    if (!act) return;
    const int Q = 4 * (1 + P.nd);
    for (int s = 0; s < NS; ++s) {
        if (s == 0 && !first) continue;
        const int slot = s == 0 ? 0 : (s <= NC1 ? slot1[s - 1] : slot2[s - 1 - NC1]);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int jj = h ? P.n_qang - 1 - jh : jh;
#pragma unroll
            for (int e = 0; e < 4; ++e)
                part[((size_t) g * Q + slot * 4 + e) * P.n_qang + jj] = acc[(s * 8 + h * 4 + e) * ANG_T + tid];
        }
    }
}

__global__ void k_reduce_pf(int n_groups, int Q, int n_qang, const double *__restrict__ part,
                            double *__restrict__ pfacc) {
    const size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t) Q * n_qang) return;
    double s = 0.;
    for (int g = 0; g < n_groups; ++g) s += part[(size_t) g * Q * n_qang + i];
    pfacc[i] = s;
}

// save_control 2: re-weight stored per-radius kernels (src/lmie_schedule.c:1087-1124)
__global__ void k_save_reweight_pf(DevProblem P, const double *__restrict__ save2,
                                   const double *__restrict__ w2, double *__restrict__ pfacc) {
    const size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;   // e*n_qang + jj
    if (i >= (size_t) 4 * P.n_qang) return;
    const int e = (int) (i / P.n_qang), jj = (int) (i % P.n_qang);
    const int n = P.n;
    double s = 0.;
    for (int r = 0; r < n; ++r) s += save2[((size_t) e * n + r) * P.n_qang + jj] * P.w[r];
    pfacc[(size_t) e * P.n_qang + jj] = s;
    for (int k = 0; k < P.nd; ++k) {
        double v = 0.;
        bool idx2 = false;
        for (int q = 0; q < P.nd2; ++q) idx2 |= P.idx2[q] == k;
        if (idx2)
            for (int r = 0; r < n; ++r) v += save2[((size_t) e * n + r) * P.n_qang + jj] * w2[(size_t) k * n + r];
        pfacc[((size_t) (1 + k) * 4 + e) * P.n_qang + jj] = v;
    }
}

__global__ void k_save_reweight_scal(DevProblem P, const double *__restrict__ save1,
                                     const double *__restrict__ w2, double *__restrict__ sums) {
    const int col = threadIdx.x;    // 0..nd
    if (col > P.nd) return;
    const int n = P.n;
    double acc[4] = {0., 0., 0., 0.};
    bool on = col == 0;
    if (col > 0)
        for (int q = 0; q < P.nd2; ++q) on |= P.idx2[q] == col - 1;
    if (on)
        for (int r = 0; r < n; ++r) {
            const double a = col == 0 ? P.w[r] : w2[(size_t) (col - 1) * n + r];
            for (int q = 0; q < 4; ++q) acc[q] += save1[(size_t) q * n + r] * a;
        }
    for (int q = 0; q < 4; ++q) sums[col * 4 + q] = acc[q];
}

// ---------------------------------------------------------------------------
// Normalisation: g and the phase matrix by 2/Csca, cross sections by
// lambda^2/(2 pi), Cbak additionally by 1/(8 pi), with the chain rule for
// every derivative slot.
// ---------------------------------------------------------------------------
__global__ void k_normalize(DevProblem P, const double *__restrict__ sums, const double *__restrict__ pfacc,
                            double *__restrict__ scal, double *__restrict__ pfn) {
    const double csca = sums[1];
    const double a = 2. / csca;
    const size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    const size_t npf = (size_t) 4 * (1 + P.nd) * P.n_qang;
    if (i < npf) {
        const int q = (int) (i / P.n_qang), jj = (int) (i % P.n_qang);
        const int slot = q / 4, e = q % 4;
        if (slot == 0) {
            pfn[i] = pfacc[i] * a;
        } else {
            const double a_l = -a * sums[slot * 4 + 1] / csca;
            pfn[i] = pfacc[i] * a + pfacc[(size_t) e * P.n_qang + jj] * a_l;
        }
    }
    if (i == 0) {
        const double lam = P.lambda;
        const double b = lam * lam / (2. * LMIEB_PI);
        const double g = sums[3];
        for (int k = 0; k < P.nd; ++k) {
            const double *s = sums + (1 + k) * 4;
            const double a_l = -a * s[1] / csca;
            const double b_l = 2. * P.lambda_l[k] * lam / (2. * LMIEB_PI);
            double *o = scal + (1 + k) * 4;
            o[0] = s[0] * b + sums[0] * b_l;
            o[1] = s[1] * b + sums[1] * b_l;
            o[2] = (s[2] * b + sums[2] * b_l) / (2. * 4. * LMIEB_PI);
            o[3] = s[3] * a + g * a_l;
        }
        scal[0] = sums[0] * b;
        scal[1] = sums[1] * b;
        scal[2] = sums[2] * b / (2. * 4. * LMIEB_PI);
        scal[3] = g / csca * 2.;
    }
}

// ---------------------------------------------------------------------------
// K4: expansion of the normalised phase matrix over the Gauss angles, with
// the mu-parity folding: the basis functions are tabulated at the positive
// nodes in chunks of orders (state carried between chunks), then one warp per
// (order, column) contracts over the nh node pairs.
// ---------------------------------------------------------------------------
__global__ void k_gsf_table(int nh, const double *__restrict__ mu, int l0, int l1, int lc,
                            double *__restrict__ st, double *__restrict__ tab) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nh) return;
    const double x = mu[nh + i];
    double q[8];     // rows l-1 and l of p00, p0p2, p2p2, p2m2
    if (l0 > 0)
        for (int v = 0; v < 8; ++v) q[v] = st[(size_t) v * nh + i];
    for (int l = l0; l < l1; ++l) {
        double p00, p02, p22, p2m;
        if (l == 0) {
            p00 = 1.; p02 = 0.; p22 = 0.; p2m = 0.;
        } else if (l == 1) {
            p00 = x; p02 = 0.; p22 = 0.; p2m = 0.;
        } else if (l == 2) {
            const double x2 = x * x;
            p00 = (3. * x2 - 1.) / 2.;
            p02 = .25 * sqrt(6.) * (x2 - 1.);
            double t = 1. + x;
            p22 = .25 * t * t;
            t = 1. - x;
            p2m = .25 * t * t;
        } else {
            const int j = l - 1;
            const double jj = (double) j * j, jp1 = j + 1., jjp1 = j * jp1, jp1s = jp1 * jp1;
            const double tj1 = 2 * j + 1;
            const double a02 = sqrt(jj - 4), b02 = sqrt(jp1s - 4);
            const double a22 = tj1 * 4, b22 = jp1 * (jj - 4), c22 = j * (jp1s - 4);
            double t = tj1 * x;
            p00 = (t * q[4] - j * q[0]) / jp1;
            p02 = (t * q[5] - a02 * q[1]) / b02;
            t = tj1 * jjp1 * x;
            p22 = ((t - a22) * q[6] - b22 * q[2]) / c22;
            p2m = ((t + a22) * q[7] - b22 * q[3]) / c22;
        }
        q[0] = q[4]; q[1] = q[5]; q[2] = q[6]; q[3] = q[7];
        q[4] = p00; q[5] = p02; q[6] = p22; q[7] = p2m;
        const size_t row = (size_t) (l - l0);
        tab[(0 * (size_t) lc + row) * nh + i] = p00;
        tab[(1 * (size_t) lc + row) * nh + i] = p02;
        tab[(2 * (size_t) lc + row) * nh + i] = p22;
        tab[(3 * (size_t) lc + row) * nh + i] = p2m;
    }
    for (int v = 0; v < 8; ++v) st[(size_t) v * nh + i] = q[v];
}

__global__ void k_leg_table(int nh, const double *__restrict__ mu, int l0, int l1, int lc,
                            double *__restrict__ st, double *__restrict__ tab) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nh) return;
    const double x = mu[nh + i];
    double pm = 0., pc = 0.;
    if (l0 > 0) { pm = st[i]; pc = st[(size_t) nh + i]; }
    for (int l = l0; l < l1; ++l) {
        double p;
        if (l == 0) p = 1.;
        else if (l == 1) p = x;
        else {
            const int j = l - 1;
            const double a = j / (j + 1.), b = x * pc;
            p = a * (b - pm) + b;
        }
        pm = pc;
        pc = p;
        tab[(size_t) (l - l0) * nh + i] = p;
    }
    st[i] = pm;
    st[(size_t) nh + i] = pc;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// kind 0 (GSF) / 1 (Legendre): raw[(c*6+e)*n_coef + l] for l in [l0, l1)
template <int KIND>
__global__ void __launch_bounds__(256) k_expand_project(DevProblem P, int l0, int l1, int lc,
                                                        const double *__restrict__ pfn,
                                                        const double *__restrict__ tab,
                                                        double *__restrict__ raw) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int nl = l1 - l0;
    const int ncol = 1 + P.nd;
    if (warp >= nl * ncol) return;
    const int lr = warp % nl, c = warp / nl;
    const int l = l0 + lr;
    const int nh = P.nh, nq = P.n_qang;
    const double s = (l & 1) ? -1. : 1.;
    const double *F0 = pfn + ((size_t) c * 4 + 0) * nq, *F1 = pfn + ((size_t) c * 4 + 1) * nq;
    const double *F2 = pfn + ((size_t) c * 4 + 2) * nq, *F3 = pfn + ((size_t) c * 4 + 3) * nq;
    double acc[6] = {0., 0., 0., 0., 0., 0.};
    for (int i = lane; i < nh; i += 32) {
        const int i1 = nh - 1 - i, i2 = nh + i;
        const double w = P.wq[i2];
        const double u0 = F0[i1] * w, u1 = F1[i1] * w, u2 = F2[i1] * w, u3 = F3[i1] * w;
        const double v0 = F0[i2] * w, v1 = F1[i2] * w, v2 = F2[i2] * w, v3 = F3[i2] * w;
        if (KIND == 0) {
            const double P00 = tab[(0 * (size_t) lc + lr) * nh + i];
            const double P02 = tab[(1 * (size_t) lc + lr) * nh + i];
            const double P22 = tab[(2 * (size_t) lc + lr) * nh + i];
            const double P2m = tab[(3 * (size_t) lc + lr) * nh + i];
            acc[0] += P00 * (u0 * s + v0);
            acc[1] += P2m * (u0 + u1) * s + P22 * (v0 + v1);
            acc[2] += P22 * (u0 - u1) * s + P2m * (v0 - v1);
            acc[3] += P00 * (u1 * s + v1);
            acc[4] += P02 * (u2 * s + v2);
            acc[5] += P02 * (u3 * s + v3);
        } else {
            const double Y = tab[(size_t) lr * nh + i];
            acc[0] += Y * (u0 * s + v0);
            acc[1] += Y * (u0 * s + v0);
            acc[2] += Y * (u1 * s + v1);
            acc[3] += Y * (u1 * s + v1);
            acc[4] += Y * (u2 * s + v2);
            acc[5] += Y * (u3 * s + v3);
        }
    }
#pragma unroll
    for (int e = 0; e < 6; ++e) acc[e] = warp_sum(acc[e]);
    if (lane == 0) {
#pragma unroll
        for (int e = 0; e < 6; ++e) raw[((size_t) c * 6 + e) * P.n_coef + l] = acc[e];
    }
}

// Recombination, (2l+1)/2 scaling, zeroed beta_0 derivative and the
// truncation search (first l with |coef_0(l)| <= accuracy).
template <int KIND>
__global__ void k_expand_finalize(DevProblem P, double accuracy, const double *__restrict__ raw,
                                  double *__restrict__ coefs, int *__restrict__ trunc) {
    const size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    const int nc = P.n_coef;
    if (i >= (size_t) (1 + P.nd) * nc) return;
    const int c = (int) (i / nc), l = (int) (i % nc);
    const double *rw = raw + (size_t) c * 6 * nc;
    double v[6];
#pragma unroll
    for (int e = 0; e < 6; ++e) v[e] = rw[(size_t) e * nc + l];
    if (KIND == 0) {
        const double t = v[1];
        v[1] = (t + v[2]) / 2.;
        v[2] = (t - v[2]) / 2.;
    } else {
        v[5] = -v[5];
    }
    const double sc = (2. * l + 1.) / 2.;
#pragma unroll
    for (int e = 0; e < 6; ++e) v[e] *= sc;
    if (c > 0 && l == 0) v[0] = 0.;
    double *o = coefs + (size_t) c * 6 * nc;
#pragma unroll
    for (int e = 0; e < 6; ++e) o[(size_t) e * nc + l] = v[e];
    if (c == 0 && fabs(v[0]) <= accuracy) atomicMax(trunc, nc - l);
}

// ---------------------------------------------------------------------------
// K5: phase matrix at the user's angles from the truncated expansion; one
// thread per (angle, column).
// ---------------------------------------------------------------------------
template <int KIND>
__global__ void k_phase_user(DevProblem P, const double *__restrict__ coefs, const int *__restrict__ trunc,
                             const double *__restrict__ mu_user, double *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int na = P.n_angles, ncol = 1 + P.nd;
    if (i >= na * ncol) return;
    const int a = i % na, c = i / na;
    const int ncf = P.n_coef;
    const int nt = trunc[0] > 0 ? ncf - trunc[0] + 1 : ncf;
    const double x = mu_user[a];
    const double *cf = coefs + (size_t) c * 6 * ncf;
    double *o = out + (size_t) c * 6 * na;
    if (KIND == 0) {
        double s0 = 0., s1 = 0., s2 = 0., s3 = 0., s4 = 0., s5 = 0.;
        double q00 = 0., q02 = 0., q22 = 0., q2m = 0.;   // row l-1
        double p00 = 0., p02 = 0., p22 = 0., p2m = 0.;   // row l
        for (int l = 0; l < nt; ++l) {
            double n00, n02, n22, n2m;
            if (l == 0) { n00 = 1.; n02 = n22 = n2m = 0.; }
            else if (l == 1) { n00 = x; n02 = n22 = n2m = 0.; }
            else if (l == 2) {
                const double x2 = x * x;
                n00 = (3. * x2 - 1.) / 2.;
                n02 = .25 * sqrt(6.) * (x2 - 1.);
                double t = 1. + x;
                n22 = .25 * t * t;
                t = 1. - x;
                n2m = .25 * t * t;
            } else {
                const int j = l - 1;
                const double jj = (double) j * j, jp1 = j + 1., jjp1 = j * jp1, jp1s = jp1 * jp1;
                const double tj1 = 2 * j + 1;
                const double a02 = sqrt(jj - 4), b02 = sqrt(jp1s - 4);
                const double a22 = tj1 * 4, b22 = jp1 * (jj - 4), c22 = j * (jp1s - 4);
                double t = tj1 * x;
                n00 = (t * p00 - j * q00) / jp1;
                n02 = (t * p02 - a02 * q02) / b02;
                t = tj1 * jjp1 * x;
                n22 = ((t - a22) * p22 - b22 * q22) / c22;
                n2m = ((t + a22) * p2m - b22 * q2m) / c22;
            }
            q00 = p00; q02 = p02; q22 = p22; q2m = p2m;
            p00 = n00; p02 = n02; p22 = n22; p2m = n2m;
            s0 += cf[l] * p00;
            s3 += cf[(size_t) 3 * ncf + l] * p00;
            if (l >= 2) {
                s4 += cf[(size_t) 4 * ncf + l] * p02;
                s5 += cf[(size_t) 5 * ncf + l] * p02;
                s1 += (cf[(size_t) 1 * ncf + l] + cf[(size_t) 2 * ncf + l]) * p22;
                s2 += (cf[(size_t) 1 * ncf + l] - cf[(size_t) 2 * ncf + l]) * p2m;
            }
        }
        o[a] = s0;
        o[(size_t) 3 * na + a] = s3;
        o[(size_t) 4 * na + a] = s4;
        o[(size_t) 5 * na + a] = s5;
        o[(size_t) 1 * na + a] = (s1 + s2) / 2.;
        o[(size_t) 2 * na + a] = (s1 - s2) / 2.;
    } else {
        double s[6] = {0., 0., 0., 0., 0., 0.};
        double pm = 0., pc = 0.;
        for (int l = 0; l < nt; ++l) {
            double p;
            if (l == 0) p = 1.;
            else if (l == 1) p = x;
            else {
                const int j = l - 1;
                const double aa = j / (j + 1.), b = x * pc;
                p = aa * (b - pm) + b;
            }
            pm = pc;
            pc = p;
#pragma unroll
            for (int e = 0; e < 6; ++e) s[e] += cf[(size_t) e * ncf + l] * p;
        }
        for (int e = 0; e < 6; ++e) o[(size_t) e * na + a] = e == 5 ? -s[e] : s[e];
    }
}

template <int NC1, int NC2>
size_t angular_smem() {
    return sizeof(double4) * ANG_KT * (1 + NC1) + sizeof(double) * ANG_KT +
           sizeof(double) * (1 + NC1 + NC2) * 8 * ANG_T;
}

template <int NC1, int NC2>
int run_angular(cudaStream_t s, const DevProblem &P, int c1base, int c2base, int first, int G,
                const int *gstart, const double *coef, double *part, double *save2) {
    const size_t sm = angular_smem<NC1, NC2>();
    static bool attr = false;
    if (!attr) {
        LMIEB_CUDA_TRY(cudaFuncSetAttribute(k_angular<NC1, NC2>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm));
        attr = true;
    }
    dim3 grid(ceil_div(P.nh, ANG_T), G);
    k_angular<NC1, NC2><<<grid, ANG_T, sm, s>>>(P, c1base, c2base, first, gstart, coef, part, save2);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}

template <int NC1>
int run_angular_nc2(cudaStream_t s, const DevProblem &P, int nc2, int c1base, int c2base, int first,
                    int G, const int *gstart, const double *coef, double *part, double *save2) {
    switch (nc2) {
    case 0: return run_angular<NC1, 0>(s, P, c1base, c2base, first, G, gstart, coef, part, save2);
    case 1: return run_angular<NC1, 1>(s, P, c1base, c2base, first, G, gstart, coef, part, save2);
    case 2: return run_angular<NC1, 2>(s, P, c1base, c2base, first, G, gstart, coef, part, save2);
    case 3: return run_angular<NC1, 3>(s, P, c1base, c2base, first, G, gstart, coef, part, save2);
    case 4: return run_angular<NC1, 4>(s, P, c1base, c2base, first, G, gstart, coef, part, save2);
    }
    return -1;
}

}  // namespace

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
int launch_gauss(cudaStream_t s, int n, const double *guess, double *mu, double *wq) {
    k_gauss<<<ceil_div((n + 1) / 2, 64), 64, 0, s>>>(n, guess, mu, wq);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int launch_coef(cudaStream_t s, const DevProblem &P, int nc, int c0, int write_value, int r0, int nb,
                int jmax, double *scr_r, double *scr_d, double *coef, double *rs) {
    const unsigned blocks = ceil_div(nb, 128);
    switch (nc) {
    case 0: k_coef<0><<<blocks, 128, 0, s>>>(P, c0, write_value, r0, nb, jmax, scr_r, scr_d, coef, rs); break;
    case 1: k_coef<1><<<blocks, 128, 0, s>>>(P, c0, write_value, r0, nb, jmax, scr_r, scr_d, coef, rs); break;
    case 2: k_coef<2><<<blocks, 128, 0, s>>>(P, c0, write_value, r0, nb, jmax, scr_r, scr_d, coef, rs); break;
    case 3: k_coef<3><<<blocks, 128, 0, s>>>(P, c0, write_value, r0, nb, jmax, scr_r, scr_d, coef, rs); break;
    case 4: k_coef<4><<<blocks, 128, 0, s>>>(P, c0, write_value, r0, nb, jmax, scr_r, scr_d, coef, rs); break;
    default:
        fprintf(stderr, "ERROR: launch_coef: bad chunk width %d\n", nc);
        return -1;
    }
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int launch_reduce_scalars(cudaStream_t s, const DevProblem &P, const double *rs, double *sums,
                          double *save1) {
    k_reduce_scalars<<<1 + P.nd, 256, 0, s>>>(P, rs, sums, save1);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int launch_angular(cudaStream_t s, const DevProblem &P, int nc1, int c1base, int nc2, int c2base,
                   int first, int G, const int *gstart, const double *coef, double *part,
                   double *save2) {
    switch (nc1) {
    case 0: return run_angular_nc2<0>(s, P, nc2, c1base, c2base, first, G, gstart, coef, part, save2);
    case 1: return run_angular_nc2<1>(s, P, nc2, c1base, c2base, first, G, gstart, coef, part, save2);
    case 2: return run_angular_nc2<2>(s, P, nc2, c1base, c2base, first, G, gstart, coef, part, save2);
    case 3: return run_angular_nc2<3>(s, P, nc2, c1base, c2base, first, G, gstart, coef, part, save2);
    case 4: return run_angular_nc2<4>(s, P, nc2, c1base, c2base, first, G, gstart, coef, part, save2);
    }
    fprintf(stderr, "ERROR: launch_angular: bad chunk width %d\n", nc1);
    return -1;
}

int launch_reduce_pf(cudaStream_t s, const DevProblem &P, int G, const double *part, double *pfacc) {
    const int Q = 4 * (1 + P.nd);
    const size_t tot = (size_t) Q * P.n_qang;
    k_reduce_pf<<<ceil_div(tot, 256), 256, 0, s>>>(G, Q, P.n_qang, part, pfacc);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int launch_save_reweight(cudaStream_t s, const DevProblem &P, const double *save1, const double *save2,
                         const double *w2, double *sums, double *pfacc) {
    k_save_reweight_scal<<<1, 32 * ceil_div(1 + P.nd, 32), 0, s>>>(P, save1, w2, sums);
    LMIEB_CUDA_TRY(cudaGetLastError());
    if (P.n_qang > 0) {
        k_save_reweight_pf<<<ceil_div((size_t) 4 * P.n_qang, 128), 128, 0, s>>>(P, save2, w2, pfacc);
        LMIEB_CUDA_TRY(cudaGetLastError());
    }
    return 0;
}

int launch_normalize(cudaStream_t s, const DevProblem &P, const double *sums, const double *pfacc,
                     double *scal, double *pfn) {
    const size_t npf = (size_t) 4 * (1 + P.nd) * P.n_qang;
    k_normalize<<<ceil_div(npf > 0 ? npf : 1, 256), 256, 0, s>>>(P, sums, pfacc, scal, pfn);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int launch_expand(cudaStream_t s, const DevProblem &P, int kind, int lchunk, double accuracy,
                  const double *pfn, double *state, double *tab, double *raw, double *coefs, int *trunc) {
    const int nc = P.n_coef, ncol = 1 + P.nd;
    LMIEB_CUDA_TRY(cudaMemsetAsync(trunc, 0, sizeof(int), s));
    for (int l0 = 0; l0 < nc; l0 += lchunk) {
        const int l1 = l0 + lchunk < nc ? l0 + lchunk : nc;
        if (kind == 0)
            k_gsf_table<<<ceil_div(P.nh, 128), 128, 0, s>>>(P.nh, P.mu, l0, l1, lchunk, state, tab);
        else
            k_leg_table<<<ceil_div(P.nh, 128), 128, 0, s>>>(P.nh, P.mu, l0, l1, lchunk, state, tab);
        LMIEB_CUDA_TRY(cudaGetLastError());
        const size_t warps = (size_t) (l1 - l0) * ncol;
        if (kind == 0)
            k_expand_project<0><<<ceil_div(warps * 32, 256), 256, 0, s>>>(P, l0, l1, lchunk, pfn, tab, raw);
        else
            k_expand_project<1><<<ceil_div(warps * 32, 256), 256, 0, s>>>(P, l0, l1, lchunk, pfn, tab, raw);
        LMIEB_CUDA_TRY(cudaGetLastError());
    }
    const size_t nt = (size_t) ncol * nc;
    if (kind == 0)
        k_expand_finalize<0><<<ceil_div(nt, 256), 256, 0, s>>>(P, accuracy, raw, coefs, trunc);
    else
        k_expand_finalize<1><<<ceil_div(nt, 256), 256, 0, s>>>(P, accuracy, raw, coefs, trunc);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int launch_phase_user(cudaStream_t s, const DevProblem &P, int kind, const double *coefs, const int *trunc,
                      const double *mu_user, double *pf_out) {
    const size_t nt = (size_t) P.n_angles * (1 + P.nd);
    if (kind == 0)
        k_phase_user<0><<<ceil_div(nt, 64), 64, 0, s>>>(P, coefs, trunc, mu_user, pf_out);
    else
        k_phase_user<1><<<ceil_div(nt, 64), 64, 0, s>>>(P, coefs, trunc, mu_user, pf_out);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}
