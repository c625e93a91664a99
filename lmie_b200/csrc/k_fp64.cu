// k_fp64.cu -- the FP64 kernels of the drop-in solve (sm_100a).
//
//   k_gauss          Gauss-Legendre angles on [-1,1]        <- misc/rtutil_math.c:73-129,231-316
//   k_recur<NC>      per-radius sequential recurrences (D_n, psi, chi)
//                                                           <- src/lmie_core.c:263-405
//   k_abcoef<NC>     a_n, b_n, their tangent-linear forms, expansion
//                    coefficients and per-radius sums, per (radius, order tile)
//                                                           <- src/lmie_core.c:453-652
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
__global__ void k_gauss(int n, const double *__restrict__ guess, const double *__restrict__ jr,
                        double *mu, double *wq) {
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
            pn = __dadd_rn(__dmul_rn(jr[j], __dsub_rn(t, pmm)), t);   // jr[j] = j / (j + 1.)
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
// K1a: one thread per radius runs the three recurrences that are sequential
// in the order n -- D_n(mx) downward from n2, the psi ratio downward from n1,
// then psi and chi upward -- and stores psi_j, chi_j, D_j (j = 0..n1) for the
// value and the NC tangent-linear columns of this chunk.  Storage rec[col] is
// order-contiguous per radius ({psi, chi, Re D, Im D} per order), so K1b reads
// it coalesced.
// ---------------------------------------------------------------------------
template <int NC>
__global__ void __launch_bounds__(64) k_recur(DevProblem P, int c0, int write_value,
                                             double4 *__restrict__ rec) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= P.n) return;
    const int n = P.n;
    const int n1 = P.n1r[r], n2 = P.n2r[r];
    const double x = P.x[r];
    const double xinv = 1. / x;
    const cplx m = P.m;
    const cplx z = mk(m.re * x, m.im * x);
    const cplx zinv = cinv(z);
    const size_t totp = (size_t) P.totp;
    const size_t base = (size_t) P.offp[r];
    double4 *R0 = rec + base;                         // value column

    double xl[NC > 0 ? NC : 1];
    cplx zl[NC > 0 ? NC : 1];
#pragma unroll
    for (int k = 0; k < NC; ++k) {
        const int kk = P.idx1[c0 + k];
        xl[k] = P.xl[(size_t) (c0 + k) * n + r];
        zl[k] = P.m_l[kk] * x + m * xl[k];
    }
#define RC(k) (rec + (size_t) (1 + c0 + (k)) * totp + base)

    // D_n downward from D_{n2} = 0; orders 1..n1 kept
    {
        cplx D = mk(0., 0.), Dl[NC > 0 ? NC : 1];
#pragma unroll
        for (int k = 0; k < NC; ++k) Dl[k] = mk(0., 0.);
        for (int j = n2 - 1; j >= 1; --j) {
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
            if (j <= n1) {
                if (write_value) ((double2 *) (R0 + j))[1] = make_double2(D.re, D.im);
#pragma unroll
                for (int k = 0; k < NC; ++k) ((double2 *) (RC(k) + j))[1] = make_double2(Dl[k].re, Dl[k].im);
            }
        }
    }
    // psi ratio r_j = psi_j / psi_{j-1} downward from r_{n1} = 0.  The value
    // ratio is parked in the value's psi slot, or -- in chunks that do not
    // write the value column -- in the chi slot of the chunk's first column,
    // until the upward pass replaces it.
    double *park = write_value ? &R0[0].x : &(rec + (size_t) (1 + c0) * totp + base)[0].y;
    {
        double rn = 0., rl[NC > 0 ? NC : 1];
#pragma unroll
        for (int k = 0; k < NC; ++k) rl[k] = 0.;
        park[(size_t) n1 * 4] = 0.;
#pragma unroll
        for (int k = 0; k < NC; ++k) RC(k)[n1].x = 0.;
        for (int j = n1 - 1; j >= 1; --j) {
            const double a1 = (2. * j + 1.) * xinv;
            const double rnew = 1. / (a1 - rn);
            if (NC > 0) {
                const double a2 = -a1 * xinv, a3 = rnew * rnew;
#pragma unroll
                for (int k = 0; k < NC; ++k) rl[k] = -(a2 * xl[k] - rl[k]) * a3;
            }
            rn = rnew;
            park[(size_t) j * 4] = rn;
#pragma unroll
            for (int k = 0; k < NC; ++k) RC(k)[j].x = rl[k];
        }
    }
    // psi, chi upward
    {
        double sinx, cosx;
        sincos(x, &sinx, &cosx);
        double psi = sinx, chi_p = cosx, chi_c = xinv * cosx + sinx;
        double psil[NC > 0 ? NC : 1], chil_p[NC > 0 ? NC : 1], chil_c[NC > 0 ? NC : 1];
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            psil[k] = xl[k] * cosx;
            chil_p[k] = xl[k] * -sinx;
            chil_c[k] = (-xinv * xinv) * xl[k] * cosx + xinv * chil_p[k] + xl[k] * cosx;
        }
        if (write_value) {
            R0[0].x = psi;
            R0[0].y = chi_p;
        }
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            RC(k)[0].x = psil[k];
            RC(k)[0].y = chil_p[k];
        }
        // the stored ratios are read back 8 orders at a time, so the loads of
        // a group overlap instead of serialising on L2 latency
        constexpr int G8 = 8;
        double rbuf[G8], rlbuf[NC > 0 ? NC : 1][G8];
        for (int j = 1; j <= n1; ++j) {
            const int u = (j - 1) & (G8 - 1);
            if (u == 0) {
#pragma unroll
                for (int v = 0; v < G8; ++v) {
                    const int jv = j + v <= n1 ? j + v : n1;
                    rbuf[v] = park[(size_t) jv * 4];
#pragma unroll
                    for (int k = 0; k < NC; ++k) rlbuf[k][v] = RC(k)[jv].x;
                }
            }
            double rj = rbuf[0];
#pragma unroll
            for (int v = 1; v < G8; ++v)
                if (u == v) rj = rbuf[v];
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                double rl = rlbuf[k][0];
#pragma unroll
                for (int v = 1; v < G8; ++v)
                    if (u == v) rl = rlbuf[k][v];
                psil[k] = rl * psi + rj * psil[k];
                RC(k)[j].x = psil[k];
                RC(k)[j].y = chil_c[k];
            }
            psi = rj * psi;
            if (write_value) {
                R0[j].x = psi;
                R0[j].y = chi_c;
            }
            if (j < n1) {
                const double a1 = (2. * j + 1.) * xinv;
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
        }
    }
#undef RC
}

// ---------------------------------------------------------------------------
// K1b: one block per (radius, tile of ABT-1 orders), one thread per order.
// Forms a_n, b_n and their tangent-linear columns from the stored
// recurrences, writes the expansion coefficients fv4 (a +- b) and reduces the
// tile's contributions to the extinction, scattering, backscatter and
// asymmetry sums (the last thread's order is the next tile's first; it is
// computed only as the neighbour a_{j+1}, b_{j+1} of the asymmetry term).
// ---------------------------------------------------------------------------
constexpr int ABT = 128;

template <int NC>
__global__ void __launch_bounds__(ABT) k_abcoef(DevProblem P, int c0, int write_value,
                                                const int2 *__restrict__ tiles,
                                                const double4 *__restrict__ rec,
                                                double *__restrict__ coef, double *__restrict__ rsp) {
    constexpr int C = 1 + NC;
    __shared__ cplx sab[2 * C][ABT];
    __shared__ double red[5 * C][ABT / 32];
    const int t = threadIdx.x;
    const int2 tile = tiles[blockIdx.x];
    const int r = tile.x, j0 = tile.y;
    const int n1 = P.n1r[r];
    const int j = j0 + t;
    const bool valid = j <= n1;
    const bool owned = valid && t < ABT - 1;
    const int n = P.n;
    const double x = P.x[r];
    const double xinv = 1. / x;
    const cplx m = P.m, minv = P.minv;
    const size_t totp = (size_t) P.totp, tot = (size_t) P.tot;
    const size_t base = (size_t) P.offp[r];
    const double *fv1 = P.fv, *fv3 = P.fv + 2 * (P.n1 + 2), *fv4 = P.fv + 3 * (P.n1 + 2);

    cplx a = mk(0., 0.), b = mk(0., 0.), al[NC > 0 ? NC : 1], bl[NC > 0 ? NC : 1];
    if (valid) {
        const double4 v = rec[base + j], vp = rec[base + j - 1];
        const cplx D = mk(v.z, v.w);
        const cplx zeta = mk(v.x, v.y), zeta_p = mk(vp.x, vp.y);
        const double psi = v.x, psi_p = vp.x;
        const double tt = j * xinv;
        const cplx ca = D * minv + tt;
        const cplx na = ca * psi - psi_p;
        const cplx ida = cinv(ca * zeta - zeta_p);
        a = na * ida;
        const cplx cb = m * D + tt;
        const cplx nb = cb * psi - psi_p;
        const cplx idb = cinv(cb * zeta - zeta_p);
        b = nb * idb;
        if (NC > 0) {
            const cplx Dm2 = D * (minv * minv);
            const double tx = -tt * xinv;
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                const size_t cb_ = (size_t) (1 + c0 + k) * totp + base;
                const double4 w = rec[cb_ + j], wp = rec[cb_ + j - 1];
                const cplx Dl = mk(w.z, w.w);
                const cplx zetal = mk(w.x, w.y), zetal_p = mk(wp.x, wp.y);
                const double psil = w.x, psil_p = wp.x;
                const double tl = tx * P.xl[(size_t) (c0 + k) * n + r];
                const cplx ml = P.m_l[P.idx1[c0 + k]];
                const cplx c6 = Dl * minv - Dm2 * ml + tl;
                al[k] = (c6 * psi + ca * psil - psil_p) * ida -
                        na * ((c6 * zeta + ca * zetal - zetal_p) * (ida * ida));
                const cplx c4 = ml * D + m * Dl + tl;
                bl[k] = (c4 * psi + cb * psil - psil_p) * idb -
                        nb * ((c4 * zeta + cb * zetal - zetal_p) * (idb * idb));
            }
        }
    } else {
#pragma unroll
        for (int k = 0; k < NC; ++k) al[k] = bl[k] = mk(0., 0.);
    }
    sab[0][t] = a;
    sab[1][t] = b;
#pragma unroll
    for (int k = 0; k < NC; ++k) {
        sab[2 + 2 * k][t] = al[k];
        sab[3 + 2 * k][t] = bl[k];
    }
    __syncthreads();

    double acc[5 * C];
#pragma unroll
    for (int q = 0; q < 5 * C; ++q) acc[q] = 0.;
    if (owned) {
        const double f1 = fv1[j], f4 = fv4[j];
        const double sgn = (j & 1) ? -1. : 1.;
        acc[0] = f1 * (a.re + b.re);
        acc[1] = f1 * (norm2(a) + norm2(b));
        acc[2] = f1 * sgn * (a.re - b.re);
        acc[3] = f1 * sgn * (a.im - b.im);
        const bool gterm = j < n1;
        cplx an = mk(0., 0.), bn = mk(0., 0.);
        if (gterm) {
            an = sab[0][t + 1];
            bn = sab[1][t + 1];
            acc[4] = fv3[j] * (re_mulc(a, an) + re_mulc(b, bn)) + fv4[j] * re_mulc(a, b);
        }
        double2 *cf = (double2 *) coef;
        if (write_value) {
            const cplx cs = (a + b) * f4, cd = (a - b) * f4;
            const size_t o = ((size_t) P.off[r] + j - 1) * 2;
            cf[o] = make_double2(cs.re, cs.im);
            cf[o + 1] = make_double2(cd.re, cd.im);
        }
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            double *q = acc + 5 * (1 + k);
            q[0] = f1 * (al[k].re + bl[k].re);
            q[1] = f1 * 2. * (re_mulc(a, al[k]) + re_mulc(b, bl[k]));
            q[2] = f1 * sgn * (al[k].re - bl[k].re);
            q[3] = f1 * sgn * (al[k].im - bl[k].im);
            if (gterm) {
                const cplx aln = sab[2 + 2 * k][t + 1], bln = sab[3 + 2 * k][t + 1];
                q[4] = fv3[j] * (re_mulc(al[k], an) + re_mulc(a, aln) + re_mulc(bl[k], bn) + re_mulc(b, bln)) +
                       fv4[j] * (re_mulc(al[k], b) + re_mulc(a, bl[k]));
            }
            const cplx cs = (al[k] + bl[k]) * f4, cd = (al[k] - bl[k]) * f4;
            const size_t o = (((size_t) (1 + c0 + k)) * tot + (size_t) P.off[r] + j - 1) * 2;
            cf[o] = make_double2(cs.re, cs.im);
            cf[o + 1] = make_double2(cd.re, cd.im);
        }
    }
    // block reduction of the 5*C tile sums (fixed order)
#pragma unroll
    for (int q = 0; q < 5 * C; ++q) {
        double v = acc[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((t & 31) == 0) red[q][t >> 5] = v;
    }
    __syncthreads();
    const int ntiles = P.ntiles;
    for (int q = t; q < 5 * C; q += ABT) {
        double v = 0.;
#pragma unroll
        for (int w = 0; w < ABT / 32; ++w) v += red[q][w];
        const int c = q / 5, qq = q % 5;
        if (c == 0 && !write_value) continue;
        const size_t col = c == 0 ? 0 : (size_t) (1 + c0 + c - 1);
        rsp[(col * 5 + qq) * ntiles + blockIdx.x] = v;
    }
}

// Sum the tile partials of every radius in tile order: rs[(col*5+q)*n + r].
__global__ void k_tile_reduce(int n, int ncol, int ntiles, const int *__restrict__ tstart,
                              const double *__restrict__ rsp, double *__restrict__ rs) {
    const size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t) ncol * 5 * n) return;
    const int r = (int) (i % n);
    const size_t cq = i / n;
    double v = 0.;
    for (int tt = tstart[r]; tt < tstart[r + 1]; ++tt) v += rsp[cq * ntiles + tt];
    rs[cq * n + r] = v;
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

// AP half-angle pairs per thread (AP = 2 when the accumulators fit), so one
// staged coefficient feeds 8*AP FMAs and the AP pi/tau chains interleave.
template <int NC1, int NC2, int AP>
__global__ void __launch_bounds__(ANG_T) k_angular(DevProblem P, int c1base, int c2base, int first,
                                                   const int *__restrict__ gstart,
                                                   const double *__restrict__ coef,
                                                   double *__restrict__ part, double *__restrict__ save2) {
    constexpr int C1 = 1 + NC1;
    constexpr int NS = 1 + NC1 + NC2;
    extern __shared__ double4 smem4[];
    double4 *cbuf = smem4;                                   // [ANG_KT][C1] {cs, cd}
    double *fv2s = (double *) (cbuf + ANG_KT * C1);          // [ANG_KT]
    double *acc = fv2s + ANG_KT;                             // [AP][NS*2*4][ANG_T]

    const int tid = threadIdx.x;
    const int g = blockIdx.y;
    const int n = P.n;
    const size_t tot = (size_t) P.tot;
    const double *fv2 = P.fv + (P.n1 + 2);
    const double4 *cf = (const double4 *) coef;
    int jh[AP];
    bool act[AP];
    double mu[AP];
#pragma unroll
    for (int a = 0; a < AP; ++a) {
        jh[a] = (blockIdx.x * AP + a) * ANG_T + tid;
        act[a] = jh[a] < P.nh;
        mu[a] = act[a] ? P.mu[jh[a]] : 0.;
    }
    const bool any = act[0];

    for (int q = 0; q < AP * NS * 8; ++q) acc[q * ANG_T + tid] = 0.;

    int slot1[NC1 > 0 ? NC1 : 1], slot2[NC2 > 0 ? NC2 : 1];
#pragma unroll
    for (int k = 0; k < NC1; ++k) slot1[k] = 1 + P.idx1[c1base + k];
#pragma unroll
    for (int k = 0; k < NC2; ++k) slot2[k] = 1 + P.idx2[c2base + k];

    const int rbeg = gstart[g], rend = gstart[g + 1];
    for (int r = rbeg; r < rend; ++r) {
        const int n1 = P.n1r[r];
        const size_t off = (size_t) P.off[r];
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
        // the next chunk's coefficients are loaded into registers while the
        // current chunk is consumed from shared memory
        constexpr int PF = (ANG_KT * C1 + ANG_T - 1) / ANG_T;
        double4 pre[PF];
        double pre_fv = 0.;
        auto fetch = [&](int k0) {
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
        fetch(0);
        for (int k0 = 0; k0 < n1; k0 += ANG_KT) {
            const int kt = min(ANG_KT, n1 - k0);
            __syncthreads();
#pragma unroll
            for (int u = 0; u < PF; ++u) {
                const int idx = tid + u * ANG_T;
                if (idx < kt * C1) cbuf[idx] = pre[u];
            }
            if (tid < kt) fv2s[tid] = pre_fv;
            __syncthreads();
            if (k0 + ANG_KT < n1) fetch(k0 + ANG_KT);
            if (!any) continue;
            // orders k = k0 + t + 1: t even <-> k odd <-> mirror sign +1
            auto step = [&](int t, bool odd) {
#pragma unroll
                for (int a = 0; a < AP; ++a) {
                    const double t1 = mu[a] * p1[a], t2 = t1 - p0[a], tau = kd * t2 - p0[a];
                    const double tp = p1[a] + tau, tm = p1[a] - tau;
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
                    p0[a] = p1[a];
                    p1[a] = t1 + fv2s[t] * t2;
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
        const double f = P.w[r], half_f = f * .5;
        double fl1[NC1 > 0 ? NC1 : 1], fl2[NC2 > 0 ? NC2 : 1];
#pragma unroll
        for (int k = 0; k < NC1; ++k) fl1[k] = P.w[(size_t) slot1[k] * n + r];
#pragma unroll
        for (int k = 0; k < NC2; ++k) fl2[k] = P.w[(size_t) slot2[k] * n + r];
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
                        const int jj = h ? P.n_qang - 1 - jh[a] : jh[a];
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
    const int Q = 4 * (1 + P.nd);
#pragma unroll
    for (int a = 0; a < AP; ++a) {
        if (!act[a]) continue;
        const double *accA = acc + (size_t) a * NS * 8 * ANG_T;
        for (int s = 0; s < NS; ++s) {
            if (s == 0 && !first) continue;
            const int slot = s == 0 ? 0 : (s <= NC1 ? slot1[s - 1] : slot2[s - 1 - NC1]);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int jj = h ? P.n_qang - 1 - jh[a] : jh[a];
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    part[((size_t) g * Q + slot * 4 + e) * P.n_qang + jj] = accA[(s * 8 + h * 4 + e) * ANG_T + tid];
            }
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
// Per-order recurrence coefficients rc[8*l + q] (host-computed, l >= 3,
// j = l - 1): p00_l = q0 mu p00_{l-1} - q1 p00_{l-2};
// p02_l = q2 mu p02_{l-1} - q3 p02_{l-2};
// p22_l = (q4 mu - q5) p22_{l-1} - q6 p22_{l-2}; p2m_l = (q4 mu + q5) p2m_{l-1} - q6 p2m_{l-2};
// Legendre: p_l = q1 (mu p_{l-1} - p_{l-2}) + mu p_{l-1}.
struct GsfRow {
    double p00, p02, p22, p2m;
};

__device__ __forceinline__ GsfRow gsf_first(int l, double x) {
    GsfRow o;
    if (l == 0) {
        o.p00 = 1.; o.p02 = 0.; o.p22 = 0.; o.p2m = 0.;
    } else if (l == 1) {
        o.p00 = x; o.p02 = 0.; o.p22 = 0.; o.p2m = 0.;
    } else {
        const double x2 = x * x;
        o.p00 = (3. * x2 - 1.) / 2.;
        o.p02 = .25 * sqrt(6.) * (x2 - 1.);
        double t = 1. + x;
        o.p22 = .25 * t * t;
        t = 1. - x;
        o.p2m = .25 * t * t;
    }
    return o;
}

__device__ __forceinline__ GsfRow gsf_next(const double *c, double x, const GsfRow &cur, const GsfRow &prev) {
    GsfRow o;
    o.p00 = c[0] * x * cur.p00 - c[1] * prev.p00;
    o.p02 = c[2] * x * cur.p02 - c[3] * prev.p02;
    const double e = c[4] * x;
    o.p22 = (e - c[5]) * cur.p22 - c[6] * prev.p22;
    o.p2m = (e + c[5]) * cur.p2m - c[6] * prev.p2m;
    return o;
}

// One thread per (positive node, basis function): the four recurrences are
// independent, so each runs on its own thread; the per-order coefficients
// are staged through shared memory GT_L orders at a time.
constexpr int GT_T = 64;
constexpr int GT_L = 128;

__global__ void __launch_bounds__(GT_T) k_gsf_table(int nh, const double *__restrict__ mu,
                                                    const double *__restrict__ rc, int l0, int l1, int lc,
                                                    double *__restrict__ st, double *__restrict__ tab) {
    __shared__ double src[GT_L][8];
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    const bool act = id < 4 * nh;
    const int f = act ? id / nh : 0, i = act ? id - f * nh : 0;
    const double x = act ? mu[nh + i] : 0.;
    double prev = 0., cur = 0.;
    if (act && l0 > 0) {
        prev = st[(size_t) f * nh + i];
        cur = st[(size_t) (4 + f) * nh + i];
    }
    double *out = tab + (size_t) f * lc * nh + i;
    // p_l = (A x + s C5) p_{l-1} - C p_{l-2}
    const int ia = f == 0 ? 0 : f == 1 ? 2 : 4;
    const int ic = f == 0 ? 1 : f == 1 ? 3 : 6;
    const double sb = f == 2 ? -1. : f == 3 ? 1. : 0.;
    for (int c0 = l0; c0 < l1; c0 += GT_L) {
        const int ct = min(GT_L, l1 - c0);
        __syncthreads();
        for (int q = threadIdx.x; q < 8 * ct; q += GT_T) src[q / 8][q % 8] = rc[8 * (size_t) c0 + q];
        __syncthreads();
        if (!act) continue;
        for (int t = 0; t < ct; ++t) {
            const int l = c0 + t;
            double v;
            if (l < 3) {
                const GsfRow g = gsf_first(l, x);
                v = f == 0 ? g.p00 : f == 1 ? g.p02 : f == 2 ? g.p22 : g.p2m;
            } else {
                v = (src[t][ia] * x + sb * src[t][5]) * cur - src[t][ic] * prev;
            }
            prev = cur;
            cur = v;
            out[(size_t) (l - l0) * nh] = v;
        }
    }
    if (!act) return;
    st[(size_t) f * nh + i] = prev;
    st[(size_t) (4 + f) * nh + i] = cur;
}

__global__ void k_leg_table(int nh, const double *__restrict__ mu, const double *__restrict__ rc, int l0,
                            int l1, int lc, double *__restrict__ st, double *__restrict__ tab) {
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
            const double b = x * pc;
            p = rc[8 * (size_t) l + 1] * (b - pm) + b;
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
// thread per user angle, one block column per output column.  The
// coefficients and recurrence constants are staged through shared memory
// PU_L orders at a time and read as broadcasts.
// ---------------------------------------------------------------------------
constexpr int PU_T = 64;
constexpr int PU_L = 256;

template <int KIND>
__global__ void __launch_bounds__(PU_T) k_phase_user(DevProblem P, const double *__restrict__ coefs,
                                                     const int *__restrict__ trunc, const double *__restrict__ rc,
                                                     const double *__restrict__ mu_user, double *__restrict__ out) {
    __shared__ double scf[6][PU_L];
    __shared__ double src[PU_L][8];
    const int a = blockIdx.x * PU_T + threadIdx.x;
    const int c = blockIdx.y;
    const int na = P.n_angles;
    const bool act = a < na;
    const int ncf = P.n_coef;
    const int nt = trunc[0] > 0 ? ncf - trunc[0] + 1 : ncf;
    const double x = act ? mu_user[a] : 0.;
    const double *cf = coefs + (size_t) c * 6 * ncf;
    double s0 = 0., s1 = 0., s2 = 0., s3 = 0., s4 = 0., s5 = 0.;
    GsfRow prev = {0., 0., 0., 0.}, cur = {0., 0., 0., 0.};
    double pm = 0., pc = 0.;
    for (int l0 = 0; l0 < nt; l0 += PU_L) {
        const int lt = min(PU_L, nt - l0);
        __syncthreads();
        for (int i = threadIdx.x; i < 6 * lt; i += PU_T) {
            const int e = i / lt, l = i - e * lt;
            scf[e][l] = cf[(size_t) e * ncf + l0 + l];
        }
        for (int i = threadIdx.x; i < 8 * lt; i += PU_T) src[i / 8][i % 8] = rc[8 * (size_t) l0 + i];
        __syncthreads();
        if (!act) continue;
        for (int t = 0; t < lt; ++t) {
            const int l = l0 + t;
            if (KIND == 0) {
                const GsfRow nx = l < 3 ? gsf_first(l, x) : gsf_next(src[t], x, cur, prev);
                prev = cur;
                cur = nx;
                s0 += scf[0][t] * cur.p00;
                s3 += scf[3][t] * cur.p00;
                if (l >= 2) {
                    s4 += scf[4][t] * cur.p02;
                    s5 += scf[5][t] * cur.p02;
                    s1 += (scf[1][t] + scf[2][t]) * cur.p22;
                    s2 += (scf[1][t] - scf[2][t]) * cur.p2m;
                }
            } else {
                double p;
                if (l == 0) p = 1.;
                else if (l == 1) p = x;
                else {
                    const double b = x * pc;
                    p = src[t][1] * (b - pm) + b;
                }
                pm = pc;
                pc = p;
                s0 += scf[0][t] * p;
                s1 += scf[1][t] * p;
                s2 += scf[2][t] * p;
                s3 += scf[3][t] * p;
                s4 += scf[4][t] * p;
                s5 += scf[5][t] * p;
            }
        }
    }
    if (!act) return;
    double *o = out + (size_t) c * 6 * na;
    if (KIND == 0) {
        o[a] = s0;
        o[(size_t) 3 * na + a] = s3;
        o[(size_t) 4 * na + a] = s4;
        o[(size_t) 5 * na + a] = s5;
        o[(size_t) 1 * na + a] = (s1 + s2) / 2.;
        o[(size_t) 2 * na + a] = (s1 - s2) / 2.;
    } else {
        o[a] = s0;
        o[(size_t) 1 * na + a] = s1;
        o[(size_t) 2 * na + a] = s2;
        o[(size_t) 3 * na + a] = s3;
        o[(size_t) 4 * na + a] = s4;
        o[(size_t) 5 * na + a] = -s5;
    }
}

template <int NC1, int NC2>
constexpr int angular_ap() { return NC1 <= 2 ? 2 : 1; }

template <int NC1, int NC2>
size_t angular_smem() {
    return sizeof(double4) * ANG_KT * (1 + NC1) + sizeof(double) * ANG_KT +
           sizeof(double) * angular_ap<NC1, NC2>() * (1 + NC1 + NC2) * 8 * ANG_T;
}

template <int NC1, int NC2>
int run_angular(cudaStream_t s, const DevProblem &P, int c1base, int c2base, int first, int G,
                const int *gstart, const double *coef, double *part, double *save2) {
    constexpr int AP = angular_ap<NC1, NC2>();
    const size_t sm = angular_smem<NC1, NC2>();
    static bool attr = false;
    if (!attr) {
        LMIEB_CUDA_TRY(cudaFuncSetAttribute(k_angular<NC1, NC2, AP>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm));
        attr = true;
    }
    dim3 grid(ceil_div(P.nh, ANG_T * AP), G);
    k_angular<NC1, NC2, AP><<<grid, ANG_T, sm, s>>>(P, c1base, c2base, first, gstart, coef, part, save2);
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
int launch_gauss(cudaStream_t s, int n, const double *guess, const double *jr, double *mu, double *wq) {
    k_gauss<<<ceil_div((n + 1) / 2, 32), 32, 0, s>>>(n, guess, jr, mu, wq);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int launch_coef(cudaStream_t s, const DevProblem &P, int nc, int c0, int write_value, const int2 *tiles,
                double4 *rec, double *coef, double *rsp) {
    const unsigned rb = ceil_div(P.n, 64);
    const unsigned tb = (unsigned) P.ntiles;
    switch (nc) {
#define LMIEB_K1(NC_)                                                                                    \
    case NC_:                                                                                            \
        k_recur<NC_><<<rb, 64, 0, s>>>(P, c0, write_value, rec);                                         \
        k_abcoef<NC_><<<tb, ABT, 0, s>>>(P, c0, write_value, tiles, rec, coef, rsp);                    \
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

int launch_tile_reduce(cudaStream_t s, const DevProblem &P, const int *tstart, const double *rsp, double *rs) {
    const size_t nt = (size_t) (1 + P.nd1) * 5 * P.n;
    k_tile_reduce<<<ceil_div(nt, 256), 256, 0, s>>>(P.n, 1 + P.nd1, P.ntiles, tstart, rsp, rs);
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

int angular_angles_per_block(int nc1) { return ANG_T * (nc1 <= 2 ? 2 : 1); }

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
    const double *rc = P.rc;
    const int nc = P.n_coef, ncol = 1 + P.nd;
    LMIEB_CUDA_TRY(cudaMemsetAsync(trunc, 0, sizeof(int), s));
    for (int l0 = 0; l0 < nc; l0 += lchunk) {
        const int l1 = l0 + lchunk < nc ? l0 + lchunk : nc;
        if (kind == 0)
            k_gsf_table<<<ceil_div((size_t) 4 * P.nh, GT_T), GT_T, 0, s>>>(P.nh, P.mu, rc, l0, l1, lchunk, state, tab);
        else
            k_leg_table<<<ceil_div(P.nh, 32), 32, 0, s>>>(P.nh, P.mu, rc, l0, l1, lchunk, state, tab);
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
    dim3 grid(ceil_div(P.n_angles, PU_T), 1 + P.nd);
    if (kind == 0)
        k_phase_user<0><<<grid, PU_T, 0, s>>>(P, coefs, trunc, P.rc, mu_user, pf_out);
    else
        k_phase_user<1><<<grid, PU_T, 0, s>>>(P, coefs, trunc, P.rc, mu_user, pf_out);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}
