// adjoint.cu -- lmie_solution_adjoint: reverse-mode gradient of an
// output-weighted scalar of many wavelengths sharing one binned size
// distribution (include/lmie_b200.h).  No counterpart in the reference; its
// forward model is the reference's Mie solution (src/lmie_core.c:263-790,
// src/lmie_schedule.c:1155-1199) for the per-radius SIZE_DIST_MONO solves
// combined with the bin weights.
//
// Per wavelength k (a "case") and quadrature radius r, with W_r = weight[b] q_r:
//   e_r = sum_n (2n+1) Re(a_n + b_n),  s_r = sum_n (2n+1)(|a_n|^2 + |b_n|^2),
//   g_r = sum_{n<n1} fv3_n Re(a_n a_{n+1}* + b_n b_{n+1}*) + fv4_n Re(a_n b_n*),
//   sp, sm at the user angles (sp = sum_n (pi_n + tau_n) fv4_n (a_n + b_n), sm
//   likewise with -), F11 = (|sp|^2 + |sm|^2)/4, F12 = -Re(sp sm*)/2,
//   phi_r = sum_i d11_i F11(theta_i) + d12_i F12(theta_i);
//   E = sum W e, S = sum W s, G = sum W g, Phi = sum W phi, N = sum W;
//   Cext = kappa E / N, Csca = kappa S / N (kappa = lambda^2 / 2 pi), g = 2 G / S,
//   P11 = 2 sum W F11 / S, P12 = 2 sum W F12 / S,
//   L_k = c_cext Cext + c_csca Csca + 2 (c_g G + Phi) / S.
// Reverse sweep: dL/dE, dL/dS, dL/dG, dL/dPhi, dL/dN per wavelength; per
// radius the adjoints of a_n, b_n (conj-gradient convention a_bar =
// dL/dRe a + i dL/dIm a) from the cross-section sums and, through the
// transposed angular contraction, from phi; then with the complex derivatives
// A_n = da_n/dm, B_n = db_n/dm,
//   dL/dmr = Re sum (conj(a_bar) A + conj(b_bar) B),  dL/dmi = Im sum (...)
// (m = mr - i mi).  A_n, B_n use dD_n/dz = n(n+1)/z^2 - 1 - D_n^2 (z = m x),
// so the D_n recurrence is never differentiated; the recurrences are re-run
// from checkpoints every ADJ_K orders, in both sweeps.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "dev_common.cuh"
#include "../../include/lmie_b200.h"

extern "C" int lmieb_calc_n1(double x);
extern "C" void lmieb_host_parallel(int n, int n_threads, void (*fn)(void *, int), void *arg);
extern "C" int lmieb_calc_n2(int n1, double zr, double zi);
extern "C" void lmieb_gauss_leg(int n, double x1, double x2, double *x, double *w);

namespace {

constexpr int ADJ_K = 64;          // orders per checkpoint block
constexpr int ADJ_T = 128;         // threads of the angular kernels (half-angles)
constexpr int ADJ_GR = 16;         // radii per block of the forward angular kernel

struct Adj {
    int L, R;                      // wavelengths, radii
    int na, nhu;                   // user angles, half-angles (theta <= 90 deg)
    int G;                         // radius groups of the forward angular kernel
    const double *lam;             // [L]
    const cplx *m;                 // [L]
    const double *W, *q;           // [R]
    const int *bin;                // [R]
    const double *x;               // [L*R]
    const int *n1, *n2;            // [L*R]
    const long long *off;          // [L*R+1] per-order offsets (n1 each)
    const long long *coff;         // [L*R+1] checkpoint offsets (ceil(n1/ADJ_K) each)
    const double *tab;             // [(n - 1) * nhu + h] -> {pi_n, tau_n}(mu_h), n = 1..n1max
    const double *tabt;            // [h * n1max + n - 1] -> {pi_n, tau_n}(mu_h) (orders contiguous)
    int n1max;
    const double *dw;              // [L][na][2] d11, d12
    const double *cw;              // [L][3] c_cext, c_csca, c_g
    cplx *cs, *cd;                 // per order: fv4 (a +- b)
    cplx *cbs, *cbd;               // per order: their adjoints (times W dL/dPhi)
    cplx *ckD;                     // checkpoints of D_n
    double *ckr;                   // checkpoints of psi_n / psi_{n-1}
    double *esg;                   // [L*R][4] e, s, g, phi
    double *pfp;                   // [L][G][na][2] partial sums of W F11, W F12
    double *lw;                    // [L][8] dL/dE, dL/dS, dL/dG, dL/dPhi, dL/dN, loss, Cext, Csca
    double *vals;                  // [L][3 + 2 na]
    double *zr;                    // [L*R][3] dL/dmr, dL/dmi, dL/dW of the radius
    double *gout;                  // [2 L + n_bins] gradient outputs
    int n_bins;
    const int *bstart;             // [n_bins + 1] radii of each bin
};

__device__ __forceinline__ double fv3d(int j) { return (j + 2.) * j / (j + 1.); }
__device__ __forceinline__ double fv4d(int j) { return (2. * j + 1.) / (j * (j + 1.)); }

// D_j for j in [lo, hi] (hi <= n2) by the downward recurrence from the
// checkpoint value at t (t >= hi): exact replay of the first sweep.
__device__ __forceinline__ void replay_D(cplx *Dl, int lo, int hi, int t, cplx Dt, cplx z) {
    cplx D = Dt;
    if (t <= hi) Dl[t - lo] = D;
    const cplx zi = cinv(z);
    for (int j = t - 1; j >= lo; --j) {
        const cplx u = (j + 1.) * zi;
        D = u - cinv(D + u);
        if (j <= hi) Dl[j - lo] = D;
    }
}

__device__ __forceinline__ void replay_r(double *rl, int lo, int hi, int t, double rt, double xinv) {
    double rr = rt;
    if (t <= hi) rl[t - lo] = rr;
    for (int j = t - 1; j >= lo; --j) {
        rr = 1. / ((2. * j + 1.) * xinv - rr);
        if (j <= hi) rl[j - lo] = rr;
    }
}

// First sweeps of one radius: checkpoints of D (from n2 down) and of the
// psi ratio (from n1 down); block c covers orders [c ADJ_K + 1, c ADJ_K + ADJ_K]
// and starts its replay at t_c = min(c ADJ_K + ADJ_K, n2) (D) or n1 (ratio).
__device__ void checkpoints(int n1, int n2, double x, cplx z, cplx *ckD, double *ckr) {
    const int nb = (n1 + ADJ_K - 1) / ADJ_K;
    const cplx zi = cinv(z);
    cplx D = mk(0., 0.);
    for (int c = 0; c < nb; ++c)
        if (c * ADJ_K + ADJ_K >= n2) ckD[c] = D;
    for (int j = n2 - 1; j >= 1; --j) {
        const cplx u = (j + 1.) * zi;
        D = u - cinv(D + u);
        if (j % ADJ_K == 0 && j / ADJ_K - 1 < nb && j < n2) ckD[j / ADJ_K - 1] = D;
    }
    const double xinv = 1. / x;
    double rr = 0.;
    for (int c = 0; c < nb; ++c)
        if (c * ADJ_K + ADJ_K >= n1) ckr[c] = 0.;
    for (int j = n1 - 1; j >= 1; --j) {
        rr = 1. / ((2. * j + 1.) * xinv - rr);
        if (j % ADJ_K == 0 && j / ADJ_K - 1 < nb) ckr[j / ADJ_K - 1] = rr;
    }
}

// Walks the orders 1..n1 of one radius in ascending order, block by block,
// calling f(j, psi_j, psi_{j-1}, zeta_j, zeta_{j-1}, D_j).
template <class F>
__device__ void ascend(int n1, int n2, double x, cplx z, const cplx *ckD, const double *ckr, F &&f) {
    cplx Dl[ADJ_K];
    double rl[ADJ_K];
    const double xinv = 1. / x;
    const double sx = sin(x), cx = cos(x);
    double psi_p = sx, chi_p = cx, chi = cx * xinv + sx;   // psi_0, chi_0, chi_1
    const int nb = (n1 + ADJ_K - 1) / ADJ_K;
    for (int c = 0; c < nb; ++c) {
        const int lo = c * ADJ_K + 1, hi = min(c * ADJ_K + ADJ_K, n1);
        replay_D(Dl, lo, hi, min(c * ADJ_K + ADJ_K, n2), ckD[c], z);
        replay_r(rl, lo, hi, min(c * ADJ_K + ADJ_K, n1), ckr[c], xinv);
        for (int j = lo; j <= hi; ++j) {
            const double psi = rl[j - lo] * psi_p;
            const cplx zeta = mk(psi, chi), zeta_p = mk(psi_p, chi_p);
            f(j, psi, psi_p, zeta, zeta_p, Dl[j - lo]);
            const double chi_n = (2. * j + 1.) * xinv * chi - chi_p;
            psi_p = psi;
            chi_p = chi;
            chi = chi_n;
        }
    }
}

// ---- forward: coefficients, cross-section sums, checkpoints (thread per (k, r)) ----
__global__ void k_adj_coef(Adj P) {
    const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long) P.L * P.R) return;
    const int k = (int) (t / P.R);
    const int n1 = P.n1[t], n2 = P.n2[t];
    const double x = P.x[t];
    const cplx m = P.m[k], minv = cinv(m), z = m * x;
    cplx *ckD = P.ckD + P.coff[t];
    double *ckr = P.ckr + P.coff[t];
    checkpoints(n1, n2, x, z, ckD, ckr);
    const double xinv = 1. / x;
    cplx *cs = P.cs + P.off[t], *cd = P.cd + P.off[t];
    double e = 0., s = 0., g = 0.;
    cplx ap = mk(0., 0.), bp = mk(0., 0.);
    ascend(n1, n2, x, z, ckD, ckr, [&](int j, double psi, double psi_p, cplx zeta, cplx zeta_p, cplx D) {
        const double tt = j * xinv;
        const cplx ca = D * minv + tt, cb = m * D + tt;
        const cplx a = (ca * psi - psi_p) * cinv(ca * zeta - zeta_p);
        const cplx b = (cb * psi - psi_p) * cinv(cb * zeta - zeta_p);
        const double f1 = 2. * j + 1., f4 = fv4d(j);
        e += f1 * (a.re + b.re);
        s += f1 * (norm2(a) + norm2(b));
        if (j >= 2) g += fv3d(j - 1) * (re_mulc(ap, a) + re_mulc(bp, b)) + fv4d(j - 1) * re_mulc(ap, bp);
        cs[j - 1] = (a + b) * f4;
        cd[j - 1] = (a - b) * f4;
        ap = a;
        bp = b;
    });
    double *o = P.esg + (size_t) t * 4;
    o[0] = e;
    o[1] = s;
    o[2] = g;
}

// sp, sm at half-angle h (and its mirror) of one radius from staged coefficients
__device__ __forceinline__ void angular_sums(const Adj &P, int h, int n1, const cplx *scs, const cplx *scd,
                                             cplx &spA, cplx &smA, cplx &spB, cplx &smB) {
    spA = smA = spB = smB = mk(0., 0.);
    const double *tb = P.tab + 2 * h;
    for (int n = 1; n <= n1; ++n) {
        const double pi = tb[(size_t) (n - 1) * 2 * P.nhu], tau = tb[(size_t) (n - 1) * 2 * P.nhu + 1];
        const double p = pi + tau, q = pi - tau, sg = (n & 1) ? 1. : -1.;
        const cplx c = scs[n - 1], d = scd[n - 1];
        spA = spA + c * p;
        smA = smA + d * q;
        spB = spB + c * (sg * q);
        smB = smB + d * (sg * p);
    }
}

__device__ __forceinline__ double block_sum128(double v, double *sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.;
#pragma unroll
    for (int w = 0; w < ADJ_T / 32; ++w) s += sh[w];
    return s;
}

// ---- forward: phase matrix at the user angles, phi_r (block per (k, radius group)) ----
__global__ void __launch_bounds__(ADJ_T) k_adj_fwd(Adj P) {
    extern __shared__ cplx sco[];                       // [2][n1max]
    __shared__ double sh[ADJ_T / 32];
    const int k = blockIdx.x / P.G, grp = blockIdx.x % P.G;
    const int h = threadIdx.x;
    const int hm = P.na - 1 - h;                        // mirror angle index
    const bool act = h < P.nhu, mir = act && hm != h;
    const double *dw = P.dw + (size_t) k * P.na * 2;
    double p11A = 0., p12A = 0., p11B = 0., p12B = 0.;
    for (int r = grp * ADJ_GR; r < min(P.R, grp * ADJ_GR + ADJ_GR); ++r) {
        const long long t = (long long) k * P.R + r;
        const int n1 = P.n1[t];
        cplx *scs = sco, *scd = sco + n1;
        __syncthreads();
        for (int i = threadIdx.x; i < n1; i += ADJ_T) {
            scs[i] = P.cs[P.off[t] + i];
            scd[i] = P.cd[P.off[t] + i];
        }
        __syncthreads();
        double phi = 0.;
        if (act) {
            cplx spA, smA, spB, smB;
            angular_sums(P, h, n1, scs, scd, spA, smA, spB, smB);
            const double W = P.W[r];
            const double f11 = .25 * (norm2(spA) + norm2(smA)), f12 = -.5 * re_mulc(spA, smA);
            p11A += W * f11;
            p12A += W * f12;
            phi = dw[2 * h] * f11 + dw[2 * h + 1] * f12;
            if (mir) {
                const double g11 = .25 * (norm2(spB) + norm2(smB)), g12 = -.5 * re_mulc(spB, smB);
                p11B += W * g11;
                p12B += W * g12;
                phi += dw[2 * hm] * g11 + dw[2 * hm + 1] * g12;
            }
        }
        phi = block_sum128(phi, sh);
        if (threadIdx.x == 0) P.esg[(size_t) t * 4 + 3] = phi;
    }
    double *o = P.pfp + ((size_t) k * P.G + grp) * P.na * 2;
    if (act) {
        o[2 * h] = p11A;
        o[2 * h + 1] = p12A;
        if (mir) {
            o[2 * hm] = p11B;
            o[2 * hm + 1] = p12B;
        }
    }
}

// ---- per wavelength: loss, phase matrix, adjoints of the sums (block per k) ----
__global__ void __launch_bounds__(ADJ_T) k_adj_lambda(Adj P) {
    __shared__ double sh[ADJ_T / 32];
    const int k = blockIdx.x;
    double N = 0., E = 0., S = 0., Gs = 0., Ph = 0.;
    for (int r = threadIdx.x; r < P.R; r += ADJ_T) {
        const double W = P.W[r];
        const double *v = P.esg + ((size_t) k * P.R + r) * 4;
        N += W;
        E += W * v[0];
        S += W * v[1];
        Gs += W * v[2];
        Ph += W * v[3];
    }
    N = block_sum128(N, sh);
    E = block_sum128(E, sh);
    S = block_sum128(S, sh);
    Gs = block_sum128(Gs, sh);
    Ph = block_sum128(Ph, sh);
    const double lam = P.lam[k], kap = lam * lam / (2. * LMIEB_PI);
    const double *cw = P.cw + (size_t) k * 3;
    double *vals = P.vals + (size_t) k * (3 + 2 * P.na);
    for (int i = threadIdx.x; i < P.na; i += ADJ_T) {
        double a = 0., b = 0.;
        for (int g = 0; g < P.G; ++g) {
            const double *o = P.pfp + ((size_t) k * P.G + g) * P.na * 2;
            a += o[2 * i];
            b += o[2 * i + 1];
        }
        vals[3 + i] = 2. * a / S;
        vals[3 + P.na + i] = 2. * b / S;
    }
    if (threadIdx.x == 0) {
        double *o = P.lw + (size_t) k * 8;
        const double cext = kap * E / N, csca = kap * S / N, g = 2. * Gs / S;
        o[0] = cw[0] * kap / N;                                       // dL/dE
        o[1] = cw[1] * kap / N - 2. * (cw[2] * Gs + Ph) / (S * S);    // dL/dS
        o[2] = 2. * cw[2] / S;                                        // dL/dG
        o[3] = 2. / S;                                                // dL/dPhi
        o[4] = -(cw[0] * kap * E + cw[1] * kap * S) / (N * N);        // dL/dN
        o[5] = cw[0] * cext + cw[1] * csca + 2. * (cw[2] * Gs + Ph) / S;
        o[6] = cext;
        o[7] = csca;
        vals[0] = cext;
        vals[1] = csca;
        vals[2] = g;
    }
}

// ---- reverse: adjoints of the coefficient columns (block per (k, r)) ----
__global__ void __launch_bounds__(ADJ_T) k_adj_back(Adj P) {
    extern __shared__ cplx sco[];                       // [2][n1] coefficients, then [4][nhu] adjoint sums
    const long long t = blockIdx.x;
    const int k = (int) (t / P.R), r = (int) (t % P.R);
    const int n1 = P.n1[t];
    cplx *scs = sco, *scd = sco + n1, *sbar = sco + 2 * n1;
    for (int i = threadIdx.x; i < n1; i += ADJ_T) {
        scs[i] = P.cs[P.off[t] + i];
        scd[i] = P.cd[P.off[t] + i];
    }
    __syncthreads();
    const double aphi = P.W[r] * P.lw[(size_t) k * 8 + 3];
    const double *dw = P.dw + (size_t) k * P.na * 2;
    const int h = threadIdx.x, hm = P.na - 1 - h;
    if (h < P.nhu) {
        cplx spA, smA, spB, smB;
        angular_sums(P, h, n1, scs, scd, spA, smA, spB, smB);
        const double a11 = .5 * aphi * dw[2 * h], a12 = .5 * aphi * dw[2 * h + 1];
        sbar[4 * h] = spA * a11 - smA * a12;            // d phi / d sp (mu_h)
        sbar[4 * h + 1] = smA * a11 - spA * a12;        // d phi / d sm (mu_h)
        if (hm != h) {
            const double b11 = .5 * aphi * dw[2 * hm], b12 = .5 * aphi * dw[2 * hm + 1];
            sbar[4 * h + 2] = spB * b11 - smB * b12;
            sbar[4 * h + 3] = smB * b11 - spB * b12;
        } else {
            sbar[4 * h + 2] = sbar[4 * h + 3] = mk(0., 0.);
        }
    }
    __syncthreads();
    // transposed contraction over the angles, one order per thread
    for (int n = threadIdx.x + 1; n <= n1; n += ADJ_T) {
        const double2 *tb = (const double2 *) P.tabt + (n - 1);   // consecutive threads, consecutive orders
        const double sg = (n & 1) ? 1. : -1.;
        cplx bs = mk(0., 0.), bd = mk(0., 0.);
        for (int hh = 0; hh < P.nhu; ++hh) {
            const double2 pt = tb[(size_t) hh * P.n1max];
            const double pi = pt.x, tau = pt.y;
            const double p = pi + tau, q = pi - tau;
            const cplx *sb = sbar + 4 * hh;
            bs = bs + sb[0] * p + sb[2] * (sg * q);
            bd = bd + sb[1] * q + sb[3] * (sg * p);
        }
        P.cbs[P.off[t] + n - 1] = bs;
        P.cbd[P.off[t] + n - 1] = bd;
    }
}

// ---- reverse: dL/dm of one radius from the checkpoints (thread per (k, r)) ----
__global__ void k_adj_m(Adj P) {
    const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long) P.L * P.R) return;
    const int k = (int) (t / P.R), r = (int) (t % P.R);
    const int n1 = P.n1[t], n2 = P.n2[t];
    const double x = P.x[t];
    const cplx m = P.m[k], minv = cinv(m), z = m * x;
    const double *lw = P.lw + (size_t) k * 8;
    const double W = P.W[r];
    const double aE = W * lw[0], aS = W * lw[1], aG = W * lw[2];
    const double xinv = 1. / x;
    const cplx zinv = cinv(z), z2inv = zinv * zinv, m2inv = minv * minv;
    const cplx *cbs = P.cbs + P.off[t], *cbd = P.cbd + P.off[t];
    cplx Z = mk(0., 0.);
    cplx ap = mk(0., 0.), bp = mk(0., 0.), Ap = mk(0., 0.), Bp = mk(0., 0.);
    ascend(n1, n2, x, z, P.ckD + P.coff[t], P.ckr + P.coff[t],
           [&](int j, double psi, double psi_p, cplx zeta, cplx zeta_p, cplx D) {
               const double tt = j * xinv;
               const cplx ca = D * minv + tt, cb = m * D + tt;
               const cplx ia = cinv(ca * zeta - zeta_p), ib = cinv(cb * zeta - zeta_p);
               const cplx a = (ca * psi - psi_p) * ia, b = (cb * psi - psi_p) * ib;
               // dD/dm = x dD/dz,  dD/dz = j (j + 1) / z^2 - 1 - D^2
               const cplx Dz = z2inv * (j * (j + 1.)) - 1. - D * D;
               const cplx w = zeta * psi_p - zeta_p * psi;     // (zeta_j psi_{j-1} - psi_j zeta_{j-1})
               const cplx A = w * (ia * ia) * (Dz * (x * 1.) * minv - D * m2inv);
               const cplx Bd = w * (ib * ib) * (D + m * Dz * x);
               const double f1 = 2. * j + 1., f4 = fv4d(j);
               // adjoints of a_j, b_j except the a_{j+1}, b_{j+1} terms of g
               cplx abar = mk(aE * f1, 0.) + a * (2. * aS * f1) + (cbs[j - 1] + cbd[j - 1]) * f4;
               cplx bbar = mk(aE * f1, 0.) + b * (2. * aS * f1) + (cbs[j - 1] - cbd[j - 1]) * f4;
               if (j < n1) {
                   abar = abar + b * (aG * f4);
                   bbar = bbar + a * (aG * f4);
               }
               if (j >= 2) {
                   const double f3 = aG * fv3d(j - 1);
                   abar = abar + ap * f3;
                   bbar = bbar + bp * f3;
                   // the a_j, b_j term of the adjoints of a_{j-1}, b_{j-1}
                   Z = Z + conjg(a) * Ap * f3 + conjg(b) * Bp * f3;
               }
               Z = Z + conjg(abar) * A + conjg(bbar) * Bd;
               ap = a;
               bp = b;
               Ap = A;
               Bp = Bd;
           });
    double *o = P.zr + (size_t) t * 3;
    o[0] = Z.re;   // dL/dmr of this radius
    o[1] = Z.im;   // dL/dmi
    const double *v = P.esg + (size_t) t * 4;
    o[2] = lw[0] * v[0] + lw[1] * v[1] + lw[2] * v[2] + lw[3] * v[3] + lw[4];   // dL/dW_r
}

// ---- gradients: dL/dmr, dL/dmi per wavelength, dL/dweight per bin ----
__global__ void __launch_bounds__(ADJ_T) k_adj_final(Adj P) {
    __shared__ double sh[ADJ_T / 32];
    if ((int) blockIdx.x < P.L) {
        const int k = blockIdx.x;
        double a = 0., b = 0.;
        for (int r = threadIdx.x; r < P.R; r += ADJ_T) {
            const double *o = P.zr + ((size_t) k * P.R + r) * 3;
            a += o[0];
            b += o[1];
        }
        a = block_sum128(a, sh);
        b = block_sum128(b, sh);
        if (threadIdx.x == 0) {
            P.gout[k] = a;
            P.gout[P.L + k] = b;
        }
    } else {
        const int bb = blockIdx.x - P.L;
        double s = 0.;
        const int r0 = P.bstart[bb], r1 = P.bstart[bb + 1];
        for (int i = threadIdx.x; i < P.L * (r1 - r0); i += ADJ_T) {
            const int k = i / (r1 - r0), r = r0 + i % (r1 - r0);
            s += P.q[r] * P.zr[((size_t) k * P.R + r) * 3 + 2];
        }
        s = block_sum128(s, sh);
        if (threadIdx.x == 0) P.gout[2 * P.L + bb] = s;
    }
}

// device buffers of the last adjoint solve, kept for the next one
std::mutex g_amu;
char *g_dbuf = nullptr, *g_hbuf = nullptr;
size_t g_dcap = 0, g_hcap = 0;

size_t pad256(size_t b) { return (b + 255) & ~(size_t) 255; }

}  // namespace

extern "C" int lmieb_stream(void **stream);

extern "C" int lmie_solution_adjoint(int n_lambda, const double *lambda, const double *mr, const double *mi,
                                     const lmie_bins *bins, int n_angles, const lmie_loss_weights *weights,
                                     double *loss, double *grad_mr, double *grad_mi, double *grad_weight,
                                     double *values) {
    if (n_lambda < 1 || !lambda || !mr || !mi || !bins || !weights || !loss || n_angles < 2 ||
        n_angles > 2 * ADJ_T - 1 || !bins->edges || !bins->weight || bins->n_bins < 1 || bins->n_quad < 1) {
        fprintf(stderr, "ERROR: lmie_solution_adjoint(): invalid arguments (n_angles must be 2..%d)\n",
                2 * ADJ_T - 1);
        return -1;
    }
    for (int b = 0; b < bins->n_bins; ++b)
        if (!(bins->edges[b] > 0.) || !(bins->edges[b + 1] > bins->edges[b]) || !(bins->weight[b] > 0.)) {
            fprintf(stderr, "ERROR: lmie_solution_adjoint(): bin %d: edges must ascend from > 0, weights > 0\n", b);
            return -1;
        }
    for (int k = 0; k < n_lambda; ++k)
        if (!(lambda[k] > 0.) || !(mr[k] > 0.) || !(mi[k] >= 0.)) {
            fprintf(stderr, "ERROR: lmie_solution_adjoint(): wavelength %d: lambda and mr must be > 0, mi >= 0\n", k);
            return -1;
        }
    void *sp = nullptr;
    if (lmieb_stream(&sp)) return -1;
    cudaStream_t s = (cudaStream_t) sp;
    std::lock_guard<std::mutex> lock(g_amu);

    const int L = n_lambda, nb = bins->n_bins, nq = bins->n_quad, R = nb * nq, na = n_angles;
    const int nhu = (na + 1) / 2, G = (R + ADJ_GR - 1) / ADJ_GR;
    // ---- host tables ----
    std::vector<double> rad(R), q(R), W(R);
    std::vector<int> bin(R), bstart(nb + 1);
    for (int b = 0; b < nb; ++b) {
        bstart[b] = b * nq;
        lmieb_gauss_leg(nq, bins->edges[b], bins->edges[b + 1], &rad[(size_t) b * nq], &q[(size_t) b * nq]);
        for (int i = 0; i < nq; ++i) {
            bin[b * nq + i] = b;
            W[b * nq + i] = bins->weight[b] * q[b * nq + i];
        }
    }
    bstart[nb] = R;
    const size_t LR = (size_t) L * R;
    std::vector<double> x(LR);
    std::vector<int> n1(LR), n2(LR);
    std::vector<long long> off(LR + 1), coff(LR + 1);
    std::vector<cplx> mm(L);
    off[0] = coff[0] = 0;
    int n1max = 1;
    // size parameters and truncations, one wavelength per task on the host's threads
    struct XJob { const double *rad, *lambda, *mr, *mi; double *x; int *n1, *n2; int R; } xj{
        rad.data(), lambda, mr, mi, x.data(), n1.data(), n2.data(), R};
    lmieb_host_parallel(L, 64, [](void *arg, int k) {
        const XJob &j = *(const XJob *) arg;
        for (int r = 0; r < j.R; ++r) {
            const size_t t = (size_t) k * j.R + r;
            j.x[t] = 2. * LMIEB_PI * j.rad[r] / j.lambda[k];
            j.n1[t] = lmieb_calc_n1(j.x[t]);
            j.n2[t] = lmieb_calc_n2(j.n1[t], j.mr[k] * j.x[t], -j.mi[k] * j.x[t]);
        }
    }, &xj);
    for (int k = 0; k < L; ++k) {
        mm[k] = mk(mr[k], -mi[k]);
        for (int r = 0; r < R; ++r) {
            const size_t t = (size_t) k * R + r;
            n1max = std::max(n1max, n1[t]);
            off[t + 1] = off[t] + n1[t];
            coff[t + 1] = coff[t] + (n1[t] + ADJ_K - 1) / ADJ_K;
        }
    }
    const size_t smem_back = (size_t) 2 * n1max * sizeof(cplx) + (size_t) 4 * nhu * sizeof(cplx);
    if (smem_back > 200 * 1024) {
        fprintf(stderr, "ERROR: lmie_solution_adjoint(): size parameters up to %.0f exceed this build's limit\n",
                *std::max_element(x.begin(), x.end()));
        return -1;
    }
    // pi_n, tau_n at the half-angles theta_h = h 180 / (na - 1), h < nhu
    std::vector<double> tab((size_t) n1max * nhu * 2);
    for (int h = 0; h < nhu; ++h) {
        const double mu = cos(h * LMIEB_PI / (na - 1));
        double p0 = 0., p1 = 1.;
        for (int n = 1; n <= n1max; ++n) {
            tab[((size_t) (n - 1) * nhu + h) * 2] = p1;
            tab[((size_t) (n - 1) * nhu + h) * 2 + 1] = n * mu * p1 - (n + 1.) * p0;
            const double p2 = ((2. * n + 1.) * mu * p1 - (n + 1.) * p0) / n;
            p0 = p1;
            p1 = p2;
        }
    }
    std::vector<double> tabt(tab.size());
    for (int n = 1; n <= n1max; ++n)
        for (int h = 0; h < nhu; ++h) {
            tabt[((size_t) h * n1max + n - 1) * 2] = tab[((size_t) (n - 1) * nhu + h) * 2];
            tabt[((size_t) h * n1max + n - 1) * 2 + 1] = tab[((size_t) (n - 1) * nhu + h) * 2 + 1];
        }
    std::vector<double> dw((size_t) L * na * 2, 0.), cw((size_t) L * 3);
    for (int k = 0; k < L; ++k) {
        cw[(size_t) k * 3] = weights[k].c_cext;
        cw[(size_t) k * 3 + 1] = weights[k].c_csca;
        cw[(size_t) k * 3 + 2] = weights[k].c_g;
        for (int i = 0; i < na; ++i) {
            dw[((size_t) k * na + i) * 2] = weights[k].d_p11 ? weights[k].d_p11[i] : 0.;
            dw[((size_t) k * na + i) * 2 + 1] = weights[k].d_p12 ? weights[k].d_p12[i] : 0.;
        }
    }
    const long long tot = off[LR], ctot = coff[LR];

    // ---- staging: inputs in one pinned block, outputs in another ----
    struct Piece { const void *src; size_t bytes; size_t at; };
    std::vector<Piece> in;
    size_t in_bytes = 0;
    auto add = [&](const void *p, size_t b) { in.push_back({p, b, in_bytes}); in_bytes += pad256(b); return in.size() - 1; };
    const size_t i_lam = add(lambda, (size_t) L * 8), i_m = add(mm.data(), (size_t) L * 16);
    const size_t i_W = add(W.data(), (size_t) R * 8), i_q = add(q.data(), (size_t) R * 8);
    const size_t i_bin = add(bin.data(), (size_t) R * 4), i_bs = add(bstart.data(), (size_t) (nb + 1) * 4);
    const size_t i_x = add(x.data(), LR * 8), i_n1 = add(n1.data(), LR * 4), i_n2 = add(n2.data(), LR * 4);
    const size_t i_off = add(off.data(), (LR + 1) * 8), i_coff = add(coff.data(), (LR + 1) * 8);
    const size_t i_tab = add(tab.data(), tab.size() * 8), i_dw = add(dw.data(), dw.size() * 8);
    const size_t i_tabt = add(tabt.data(), tabt.size() * 8);
    const size_t i_cw = add(cw.data(), cw.size() * 8);
    const size_t out_vals = (size_t) L * (3 + 2 * na) * 8, out_lw = (size_t) L * 8 * 8;
    const size_t out_g = (size_t) (2 * L + nb) * 8;
    const size_t out_bytes = pad256(out_vals) + pad256(out_lw) + pad256(out_g);
    size_t dev_bytes = in_bytes + out_bytes;
    const size_t b_cs = pad256((size_t) tot * 16), b_ck = pad256((size_t) ctot * 16), b_ckr = pad256((size_t) ctot * 8);
    const size_t b_esg = pad256(LR * 4 * 8), b_pfp = pad256((size_t) L * G * na * 2 * 8), b_zr = pad256(LR * 3 * 8);
    dev_bytes += 4 * b_cs + b_ck + b_ckr + b_esg + b_pfp + b_zr;
    if (dev_bytes > g_dcap) {
        if (g_dbuf) cudaFree(g_dbuf);
        g_dbuf = nullptr;
        g_dcap = 0;
        LMIEB_CUDA_TRY(cudaMalloc((void **) &g_dbuf, dev_bytes));
        g_dcap = dev_bytes;
    }
    if (in_bytes + out_bytes > g_hcap) {
        if (g_hbuf) cudaFreeHost(g_hbuf);
        g_hbuf = nullptr;
        g_hcap = 0;
        LMIEB_CUDA_TRY(cudaMallocHost((void **) &g_hbuf, in_bytes + out_bytes));
        g_hcap = in_bytes + out_bytes;
    }
    struct CopyJob { const Piece *in; char *dst; } cj{in.data(), g_hbuf};
    lmieb_host_parallel((int) in.size(), 16, [](void *arg, int i) {
        const CopyJob &j = *(const CopyJob *) arg;
        memcpy(j.dst + j.in[i].at, j.in[i].src, j.in[i].bytes);
    }, &cj);
    char *d = g_dbuf;
    auto dp = [&](size_t i) { return (void *) (d + in[i].at); };
    Adj P;
    memset(&P, 0, sizeof(P));
    P.L = L; P.R = R; P.na = na; P.nhu = nhu; P.G = G; P.n_bins = nb;
    P.lam = (const double *) dp(i_lam); P.m = (const cplx *) dp(i_m);
    P.W = (const double *) dp(i_W); P.q = (const double *) dp(i_q); P.bin = (const int *) dp(i_bin);
    P.bstart = (const int *) dp(i_bs);
    P.x = (const double *) dp(i_x); P.n1 = (const int *) dp(i_n1); P.n2 = (const int *) dp(i_n2);
    P.off = (const long long *) dp(i_off); P.coff = (const long long *) dp(i_coff);
    P.tabt = (const double *) dp(i_tabt);
    P.n1max = n1max;
    P.tab = (const double *) dp(i_tab); P.dw = (const double *) dp(i_dw); P.cw = (const double *) dp(i_cw);
    char *o = d + in_bytes;
    P.vals = (double *) o; o += pad256(out_vals);
    P.lw = (double *) o; o += pad256(out_lw);
    P.gout = (double *) o; o += pad256(out_g);
    P.cs = (cplx *) o; o += b_cs;
    P.cd = (cplx *) o; o += b_cs;
    P.cbs = (cplx *) o; o += b_cs;
    P.cbd = (cplx *) o; o += b_cs;
    P.ckD = (cplx *) o; o += b_ck;
    P.ckr = (double *) o; o += b_ckr;
    P.esg = (double *) o; o += b_esg;
    P.pfp = (double *) o; o += b_pfp;
    P.zr = (double *) o; o += b_zr;

    // ---- run ----
    LMIEB_CUDA_TRY(cudaMemcpyAsync(d, g_hbuf, in_bytes, cudaMemcpyHostToDevice, s));
    const size_t smem_fwd = (size_t) 2 * n1max * sizeof(cplx);
    static size_t attr_fwd = 0, attr_back = 0;
    if (smem_fwd > 48 * 1024 && smem_fwd > attr_fwd) {
        LMIEB_CUDA_TRY(cudaFuncSetAttribute(k_adj_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem_fwd));
        attr_fwd = smem_fwd;
    }
    if (smem_back > 48 * 1024 && smem_back > attr_back) {
        LMIEB_CUDA_TRY(cudaFuncSetAttribute(k_adj_back, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem_back));
        attr_back = smem_back;
    }
    const unsigned nthr = 64, nblk = ceil_div(LR, nthr);
    k_adj_coef<<<nblk, nthr, 0, s>>>(P);
    LMIEB_CUDA_TRY(cudaGetLastError());
    k_adj_fwd<<<(unsigned) L * G, ADJ_T, smem_fwd, s>>>(P);
    LMIEB_CUDA_TRY(cudaGetLastError());
    k_adj_lambda<<<L, ADJ_T, 0, s>>>(P);
    LMIEB_CUDA_TRY(cudaGetLastError());
    k_adj_back<<<(unsigned) LR, ADJ_T, smem_back, s>>>(P);
    LMIEB_CUDA_TRY(cudaGetLastError());
    k_adj_m<<<nblk, nthr, 0, s>>>(P);
    LMIEB_CUDA_TRY(cudaGetLastError());
    k_adj_final<<<L + nb, ADJ_T, 0, s>>>(P);
    LMIEB_CUDA_TRY(cudaGetLastError());
    char *ho = g_hbuf + in_bytes;
    LMIEB_CUDA_TRY(cudaMemcpyAsync(ho, d + in_bytes, out_bytes, cudaMemcpyDeviceToHost, s));
    LMIEB_CUDA_TRY(cudaStreamSynchronize(s));
    const double *hv = (const double *) ho;
    const double *hl = (const double *) (ho + pad256(out_vals));
    const double *hg = (const double *) (ho + pad256(out_vals) + pad256(out_lw));
    double sum = 0.;
    for (int k = 0; k < L; ++k) sum += hl[(size_t) k * 8 + 5];
    *loss = sum;
    if (grad_mr) memcpy(grad_mr, hg, (size_t) L * 8);
    if (grad_mi) memcpy(grad_mi, hg + L, (size_t) L * 8);
    if (grad_weight) memcpy(grad_weight, hg + 2 * L, (size_t) nb * 8);
    if (values) memcpy(values, hv, out_vals);
    return 0;
}
