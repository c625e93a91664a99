// k_tc.cu -- K3 in split precision on the fifth-generation tensor cores.
//
// The S1/S2 sums over orders (reference src/lmie_core.c:658-721) of one case
// are the product A+ [S | D'] of tc_layout.cuh: 128 rows (64 half-angles
// mu_h < 0 of the block and their mirrors, interleaved) by 128 operand rows
// of a radius group, over the orders.  A block owns one angle tile of one
// case and a range of radius groups; per group, chunks of TC_KC orders flow
// through shared memory:
//   - warps 0-3 (one thread per row; the two threads of a half-angle both run
//     its recurrence) run the pi/tau recurrence in FP64 (pi_{k+1} =
//     (2k+1)/k mu pi_k - (k+1)/k pi_{k-1}, one dependent FMA per order) and
//     write row 2h = (pi + tau)(mu_h) or 2h+1 = s_k (pi - tau)(mu_h) of A+,
//     split into TF32 hi/lo, in the K-major core-matrix layout;
//   - lane 0 of warp 9 brings the group's B chunks (written by K1) with bulk
//     copies running ahead of the products; lane 0 of warp 8 issues
//     tcgen05.mma kind::tf32
//     (M 128, N 128, K 8): hi*hi into a segment accumulator F, lo*hi + hi*lo
//     into a cross-term accumulator G of the group, both FP32 in tensor
//     memory;
//   - the FP32 accumulation of the tensor cores truncates, so its error grows
//     with the number of products it sums: the hi*hi products (the large
//     ones) of a segment of `seg` chunks go into a fresh F (two buffers
//     alternate), and warps 4-7 add each finished segment into an FP32
//     running sum H while the next segment is computed; the cross terms are
//     2^-11 of those, so their truncation stays below the hi*hi rounding over
//     a whole group.  After a group's last segment warps 4-7 fold G into F,
//     release G to the next group, read the sums of their row (tensor-memory
//     lane = row; sm of a row is in its pair row's lane, one shuffle away),
//     form the phase-matrix quadratic forms and their linearisations per
//     radius in FP64 (reference src/lmie_core.c:723-790) and accumulate them
//     over the block's radii in registers.
// Partials go to the same per-group buffer as the FP64 K3.
//
// Tensor memory (512 columns): F0 [0,128) and F1 [128,256) segment
// accumulators, H [256,384) running sum, G [384,512) cross terms.
//
// Every wait is bounded (about 1 s of clock, or until another block has
// failed); a block that gives up sets the error word, waits (bounded) for
// its tensor-core work and copies in flight, releases its tensor memory and
// returns.
#include <cstdio>

#include "kernels.h"
#include "tc_layout.cuh"
#include "tc_ptx.cuh"

namespace {

constexpr int TC_T = 320;                    // warps 0-3: A operand; 4-7: segment sums and quadratic
                                             // forms; 8: products; 9: B copies
constexpr int TC_MMA_WARP = 8, TC_COPY_WARP = 9;
constexpr int TC_ASTAGES = 3;                // A operand stages
constexpr int TC_BSLOTS = 6;                 // B operand slots (bulk copies)
constexpr int TC_BAHEAD = TC_BSLOTS - 2;     // chunks the B copies run ahead of the products
constexpr int TC_MAX_GN = TC_NHALF / 2;      // radii of a group (tc_rg(0))
constexpr int TC_MAX_NS = 1 + TC_MAX_NC1 + TC_MAX_ND2;
// barriers: afull[TC_ASTAGES], adone[TC_ASTAGES], bfull[TC_BSLOTS], bdone[TC_BSLOTS], segfull[2],
// segfree[2], gfree, fin
constexpr int TC_NBAR = 2 * TC_ASTAGES + 2 * TC_BSLOTS + 4 + 2;
constexpr uint32_t TC_RING = TC_ASTAGES * TC_ASTAGE + TC_BSLOTS * TC_BSTAGE;
constexpr uint32_t TC_WBUF = TC_MAX_GN * TC_MAX_NS * 8;   // a group's radius weights
constexpr uint32_t TC_SMEM = TC_RING + TC_WBUF + TC_NBAR * 8 + 16;
constexpr uint32_t TC_TMEM_COLS = 512;
constexpr uint32_t TC_HCOL = 2 * TC_NP, TC_GCOL = 3 * TC_NP;   // running sum, cross terms

static_assert(TC_ASTAGE % 1024 == 0 && TC_BSTAGE % 1024 == 0, "stages stay 1 KB aligned");
constexpr uint32_t TC_STAGE = TC_ASTAGE + TC_BSTAGE;   // the self-test's single stage
static_assert(TC_NP % 16 == 0 && TC_NP <= 256, "N of an M=128 tf32 MMA");
static_assert(4 * TC_NP <= (int) TC_TMEM_COLS, "segment buffers, running sum, cross terms");
static_assert(TC_WBUF % 16 == 0, "barriers stay 8-byte aligned");
static_assert(TC_SMEM <= 227 * 1024, "shared memory per block");

// instruction descriptor of kind::tf32: D FP32, A and B TF32, both K-major
__host__ __device__ constexpr uint32_t idesc_tf32(int m, int n) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t) (n >> 3) << 17) | ((uint32_t) (m >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

// The 3xTF32 products of one chunk (one thread).  a0/b0: shared addresses of
// the chunk's A and B stages ([hi | lo] each); dF: tensor-memory column of the
// hi*hi accumulator of the segment, dG: of the cross-term (lo*hi + hi*lo)
// accumulator of the group; firstF / firstG: the chunk opens that accumulation.
__device__ __forceinline__ void issue_chunk(uint32_t a0, uint32_t b0, uint32_t dF, uint32_t dG, bool firstF,
                                            bool firstG) {
    constexpr uint32_t idesc = idesc_tf32(TC_M, TC_NP);
    // descriptor of the stage start; the start-address field (bits 0-13, in
    // 16-byte units) of the other operand parts and K steps is an offset
    const uint64_t da = sdesc(a0, TC_LBO_A, 128), db = sdesc(b0, TC_LBO_B, 128);
#pragma unroll
    for (int ks = 0; ks < TC_KC / 8; ++ks) {
        const uint64_t ahi = da + (uint64_t) ((ks * 2 * TC_LBO_A) >> 4), alo = ahi + (TC_APART >> 4);
        const uint64_t bhi = db + (uint64_t) ((ks * 2 * TC_LBO_B) >> 4), blo = bhi + (TC_BPART >> 4);
        mma_tf32(dG, alo, bhi, idesc, (firstG && ks == 0) ? 0u : 1u);
        mma_tf32(dG, ahi, blo, idesc, 1u);
        mma_tf32(dF, ahi, bhi, idesc, (firstF && ks == 0) ? 0u : 1u);
    }
}

template <int NC1>
__global__ void __launch_bounds__(TC_T, 1) k_angular_tc(DevBatch B, const AngItem *__restrict__ items,
                                                        const float *__restrict__ bop, double *__restrict__ part,
                                                        int seg, int *__restrict__ err) {
    constexpr int C1 = 1 + NC1, CPR = 2 * C1;
    extern __shared__ __align__(1024) unsigned char smem[];
    double *wsh = (double *) (smem + TC_RING);              // [TC_MAX_GN][TC_MAX_NS] weights of a group
    uint64_t *bars = (uint64_t *) (smem + TC_RING + TC_WBUF);
    uint32_t *tmem_hold = (uint32_t *) (bars + TC_NBAR);
    const uint32_t sbase = smem_u32(smem), bring = sbase + TC_ASTAGES * TC_ASTAGE;
    const uint32_t afull0 = smem_u32(bars), adone0 = afull0 + 8 * TC_ASTAGES;
    const uint32_t bfull0 = adone0 + 8 * TC_ASTAGES, bdone0 = bfull0 + 8 * TC_BSLOTS;
    const uint32_t segfull0 = bdone0 + 8 * TC_BSLOTS, segfree0 = segfull0 + 16;
    const uint32_t gfree = segfree0 + 16, fin = gfree + 8;

    const int tid = threadIdx.x, warp = tid >> 5;
    const AngItem it = items[blockIdx.x];
    const DevCase &C = B.cs[it.c];
    const int nh = C.nh, n_qang = C.n_qang, R = B.R;
    const int nd2 = B.nd2, NS = 1 + NC1 + nd2;

    // after a failure elsewhere the remaining blocks return at once
    __shared__ int s_skip;
    if (tid == 0) s_skip = *(volatile const int *) err;
    __syncthreads();
    if (s_skip) return;
    if (tid == 0) {
        for (int i = 0; i < TC_ASTAGES; ++i) {
            mbar_init(afull0 + 8 * i, TC_M);
            mbar_init(adone0 + 8 * i, 1);
        }
        for (int i = 0; i < TC_BSLOTS; ++i) {
            mbar_init(bfull0 + 8 * i, 1);
            mbar_init(bdone0 + 8 * i, 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(segfull0 + 8 * i, 1);
            mbar_init(segfree0 + 8 * i, 128);
        }
        mbar_init(gfree, 128);
        mbar_init(fin, 1);
        fence_mbar_init();
    }
    if (warp == 0) tmem_alloc(smem_u32(tmem_hold), TC_TMEM_COLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_hold;
    int bad = 0;

    if (tid < TC_M) {
        // ---------------- warps 0-3: the A operand, one row per thread ----------------
        // row 2h = (pi + tau)(mu_h), row 2h+1 = s_k (pi - tau)(mu_h); both threads
        // of a pair run the recurrence of half-angle h
        const int row = tid, h = row >> 1, mirror = row & 1;
        const int gj = it.xt * TC_HALF + h;
        const bool gact = gj < nh;
        const double mu = gact ? B.mu_pool[C.mu_off + gj] : 0.;
        const double *fv2 = B.fv + (B.n1max + 2);          // (k + 1) / k
        const int fvmax = B.n1max + 1;
        const int ro = (row >> 3) * 32 + (row & 7) * 4;    // float offset of the row in an order group
        int q = 0;
        for (int g = it.rbeg; g < it.rend && !bad; ++g) {
            const int nk = B.tg_nk[g];
            double p0 = 0., p1 = 1., kd = 1.;              // pi_{k-1}, pi_k, k
            for (int kc = 0; kc < nk; ++kc, ++q) {
                const int s = q % TC_ASTAGES;
                // (k + 1) / k of the chunk's orders, loaded while the stage is still in use
                double f2v[TC_KC];
#pragma unroll
                for (int u = 0; u < TC_KC; ++u) f2v[u] = __ldg(fv2 + min(kc * TC_KC + u + 1, fvmax));
                // the stage's previous chunk must have been consumed by its products
                if (q >= TC_ASTAGES && !mbar_wait(adone0 + 8 * s, ((q / TC_ASTAGES) - 1) & 1, err)) {
                    bad = 1;
                    break;
                }
                float *aw = (float *) (smem + s * TC_ASTAGE) + ro;
#pragma unroll
                for (int k4 = 0; k4 < TC_KC / 4; ++k4) {
                    float hv[4], lv[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int k = kc * TC_KC + k4 * 4 + u + 1;
                        const double f2 = f2v[k4 * 4 + u];
                        // tau_k = k mu pi_k - (k + 1) pi_{k-1}
                        const double tau = fma(kd * mu, p1, -(kd + 1.) * p0);
                        const double v = mirror ? ((k & 1) ? p1 - tau : tau - p1) : p1 + tau;
                        tc_split(v, hv[u], lv[u]);
                        const double pn = fma((1. + f2) * mu, p1, -f2 * p0);
                        p0 = p1;
                        p1 = pn;
                        kd += 1.;
                    }
                    if (!gact) {
#pragma unroll
                        for (int u = 0; u < 4; ++u) hv[u] = lv[u] = 0.f;
                    }
                    float *o = aw + k4 * (TC_M / 8) * 32;
                    *(float4 *) o = make_float4(hv[0], hv[1], hv[2], hv[3]);
                    *(float4 *) (o + TC_APART / 4) = make_float4(lv[0], lv[1], lv[2], lv[3]);
                }
                fence_proxy_async();
                mbar_arrive(afull0 + 8 * s);
            }
        }
    } else if (warp == TC_COPY_WARP) {
        // ---------------- warp 9, lane 0: B copies, up to TC_BSLOTS chunks ahead ----------------
        if ((tid & 31) == 0) {
            int pq = 0;
            for (int g = it.rbeg; g < it.rend && !bad; ++g) {
                const int nk = B.tg_nk[g];
                const float *src = bop + B.tg_off[g];
                for (int kc = 0; kc < nk; ++kc, ++pq) {
                    const int ps = pq % TC_BSLOTS;
                    // the slot's previous chunk pq - TC_BSLOTS must have been consumed
                    if (pq >= TC_BSLOTS && !mbar_wait(bdone0 + 8 * ps, ((pq / TC_BSLOTS) - 1) & 1, err)) {
                        bad = 1;
                        break;
                    }
                    mbar_expect_tx(bfull0 + 8 * ps, TC_BSTAGE);
                    const uint32_t dst = bring + ps * TC_BSTAGE;
                    bulk_g2s(dst, src, TC_BPART, bfull0 + 8 * ps);
                    bulk_g2s(dst + TC_BPART, src + TC_BPART / 4, TC_BPART, bfull0 + 8 * ps);
                    src += TC_BSTAGE / 4;
                }
            }
            // the copies in flight land before the block ends
            const int q0 = pq > TC_BSLOTS ? pq - TC_BSLOTS : 0;
            for (int c = q0; c < pq; ++c) mbar_wait(bfull0 + 8 * (c % TC_BSLOTS), (c / TC_BSLOTS) & 1, nullptr);
        }
    } else if (warp == TC_MMA_WARP) {
        // ---------------- warp 8, lane 0: the products ----------------
        if ((tid & 31) == 0) {
            uint32_t ph_free = 0u;   // per F buffer b (bit b): parity of its next segfree phase
            int q = 0, gs = 0, gi = 0;
            int nk_next = it.rbeg < it.rend ? B.tg_nk[it.rbeg] : 0;
            for (int g = it.rbeg; g < it.rend && !bad; ++g, ++gi) {
                const int nk = nk_next;
                if (g + 1 < it.rend) nk_next = B.tg_nk[g + 1];
                int sc = 0;                                  // chunk within the segment
                for (int kc = 0; kc < nk; ++kc, ++q) {
                    const int s = q % TC_ASTAGES, sb = q % TC_BSLOTS;
                    const int b = gs & 1;
                    const bool seg_first = sc == 0;
                    const bool seg_last = sc == seg - 1 || kc == nk - 1;
                    if (!mbar_wait(afull0 + 8 * s, (q / TC_ASTAGES) & 1, err) ||
                        !mbar_wait(bfull0 + 8 * sb, (q / TC_BSLOTS) & 1, err)) {
                        bad = 1;
                        break;
                    }
                    if (seg_first && gs >= 2) {
                        // the segment buffer must have been drained
                        if (!mbar_wait(segfree0 + 8 * b, (ph_free >> b) & 1u, err)) {
                            bad = 1;
                            break;
                        }
                        ph_free ^= 1u << b;
                    }
                    if (kc == 0 && gi >= 1 && !mbar_wait(gfree, (gi - 1) & 1, err)) {
                        // the previous group's cross terms must have been read
                        bad = 1;
                        break;
                    }
                    tc_fence_after();
                    issue_chunk(sbase + s * TC_ASTAGE, bring + sb * TC_BSTAGE, tmem + b * TC_NP, tmem + TC_GCOL,
                                seg_first, kc == 0);
                    mma_commit(adone0 + 8 * s);
                    mma_commit(bdone0 + 8 * sb);
                    if (seg_last) {
                        mma_commit(segfull0 + 8 * b);
                        ++gs;
                        sc = 0;
                    } else {
                        ++sc;
                    }
                }
            }
            // all products of this thread have completed
            mma_commit(fin);
            mbar_wait(fin, 0u, nullptr);
        }
    } else if (warp >= 4) {
        // ---------------- warps 4-7: segment sums, quadratic forms ----------------
        // A warp whose wait fails skips the tensor-memory work from then on but
        // keeps taking the barriers of the four warps, which stop together.
        const int t1 = tid - 128;                            // product row = tensor-memory lane
        const uint32_t trow = tmem + ((uint32_t) ((warp - 4) * 32) << 16);
        const int eh = t1 >> 1, emir = t1 & 1;
        const int ej = it.xt * TC_HALF + eh;
        const bool eact = ej < nh;
        int slot1[NC1 > 0 ? NC1 : 1];
#pragma unroll
        for (int k = 0; k < NC1; ++k) slot1[k] = 1 + B.idx1[k];
        // per column set: f-weighted sums over radii of the four invariants
        double racc[1 + NC1 + TC_MAX_ND2][4];
#pragma unroll
        for (int s = 0; s < 1 + NC1 + TC_MAX_ND2; ++s)
#pragma unroll
            for (int e = 0; e < 4; ++e) racc[s][e] = 0.;
        uint32_t ph_seg = 0u;
        int gs = 0;
        for (int g = it.rbeg; g < it.rend; ++g) {
            const int gr0 = B.tg_r0[g], gn = B.tg_n[g], nk = B.tg_nk[g];
            const int nseg = (nk + seg - 1) / seg;
            // the previous group's weights have been read by all four warps
            if (epi_sync_or(bad || gn > TC_MAX_GN)) {
                bad = 1;
                break;
            }
            for (int i = t1; i < gn * NS; i += 128) {
                const int p = i / NS, s = i - p * NS;
                const int slot = s == 0 ? 0 : (s <= NC1 ? slot1[s - 1] : 1 + B.idx2[s - 1 - NC1]);
                wsh[p * TC_MAX_NS + s] = B.w[(size_t) slot * R + gr0 + p];
            }
            epi_sync_or(0);
            for (int sg = 0; sg < nseg; ++sg, ++gs) {
                const int b = gs & 1;
                if (bad) continue;
                // warp-uniform decision: the tensor-memory accesses below are warp-wide
                const bool arrived = mbar_wait(segfull0 + 8 * b, (ph_seg >> b) & 1u, err);
                if (__any_sync(0xffffffffu, !arrived)) {
                    bad = 1;
                    continue;
                }
                ph_seg ^= 1u << b;
                tc_fence_after();
                const bool first = sg == 0;
                if (sg < nseg - 1) {
                    // running sum H += F_b (FP32, round to nearest)
#pragma unroll 1
                    for (int c0 = 0; c0 < TC_NP; c0 += 16) {
                        const uint32_t base = trow + c0;
                        uint32_t f[16], hh[16];
                        tmem_ld16(base + b * TC_NP, f);
                        if (!first) tmem_ld16(base + TC_HCOL, hh);
                        tmem_wait_ld();
#pragma unroll
                        for (int i = 0; i < 16; ++i) {
                            reg_after_wait(f[i]);
                            if (!first) reg_after_wait(hh[i]);
                        }
#pragma unroll
                        for (int i = 0; i < 16; ++i)
                            hh[i] = first ? f[i]
                                          : __float_as_uint(__fadd_rn(__uint_as_float(hh[i]), __uint_as_float(f[i])));
                        tmem_st16(base + TC_HCOL, hh);
                    }
                    tmem_wait_st();
                } else {
                    // last segment: fold the group's cross terms G into F_b and hand G
                    // back to the products of the next group
#pragma unroll 1
                    for (int c0 = 0; c0 < TC_NP; c0 += 16) {
                        const uint32_t base = trow + c0;
                        uint32_t f[16], gg[16];
                        tmem_ld16(base + b * TC_NP, f);
                        tmem_ld16(base + TC_GCOL, gg);
                        tmem_wait_ld();
#pragma unroll
                        for (int i = 0; i < 16; ++i) {
                            reg_after_wait(f[i]);
                            reg_after_wait(gg[i]);
                            f[i] = __float_as_uint(__fadd_rn(__uint_as_float(f[i]), __uint_as_float(gg[i])));
                        }
                        tmem_st16(base + b * TC_NP, f);
                    }
                    tmem_wait_st();
                    tc_fence_before();
                    mbar_arrive(gfree);
                    // the sums of every radius of the group, then the quadratic forms
                    for (int p = 0; p < gn; ++p) {
                        // columns of S (i < CPR) and D' (i >= CPR) of radius p
                        uint32_t vf[2 * CPR], vh[2 * CPR];
#pragma unroll
                        for (int i = 0; i < 2 * CPR; i += 2) {
                            const uint32_t col = (i < CPR ? 0 : TC_NHALF - CPR) + p * CPR + i;
                            tmem_ld2(trow + b * TC_NP + col, vf[i], vf[i + 1]);
                            if (!first) tmem_ld2(trow + TC_HCOL + col, vh[i], vh[i + 1]);
                        }
                        tmem_wait_ld();
                        double v[2 * CPR];
#pragma unroll
                        for (int i = 0; i < 2 * CPR; ++i) {
                            reg_after_wait(vf[i]);
                            v[i] = (double) __uint_as_float(vf[i]);
                            if (!first) {
                                reg_after_wait(vh[i]);
                                v[i] += (double) __uint_as_float(vh[i]);
                            }
                        }
                        // sm of this row is the D' sum of its pair row (lane ^ 1)
#pragma unroll
                        for (int i = CPR; i < 2 * CPR; ++i) v[i] = __shfl_xor_sync(0xffffffffu, v[i], 1);
                        const double *wp = wsh + p * TC_MAX_NS;
                        const double f = wp[0];
                        // invariants of (sp, sm): |sp|^2, |sm|^2, Re(sp sm*), Im(sm sp*)
                        const double spr = v[0], spi = v[1], smr = v[CPR], smi = v[CPR + 1];
                        const double ia = spr * spr + spi * spi, ib = smr * smr + smi * smi;
                        const double ic = spr * smr + spi * smi, id = smi * spr - smr * spi;
                        racc[0][0] += f * ia;
                        racc[0][1] += f * ib;
                        racc[0][2] += f * ic;
                        racc[0][3] += f * id;
#pragma unroll
                        for (int k = 0; k < NC1; ++k) {
                            const double fl = wp[1 + k];
                            const double plr = v[2 + 2 * k], pli = v[3 + 2 * k];
                            const double mlr = v[CPR + 2 + 2 * k], mli = v[CPR + 3 + 2 * k];
                            const double da = 2. * (plr * spr + pli * spi), db = 2. * (mlr * smr + mli * smi);
                            const double dc = plr * smr + pli * smi + spr * mlr + spi * mli;
                            const double dd = mli * spr - mlr * spi + smi * plr - smr * pli;
                            racc[1 + k][0] += fl * ia + f * da;
                            racc[1 + k][1] += fl * ib + f * db;
                            racc[1 + k][2] += fl * ic + f * dc;
                            racc[1 + k][3] += fl * id + f * dd;
                        }
#pragma unroll
                        for (int k = 0; k < TC_MAX_ND2; ++k) {
                            if (k < nd2) {
                                const double fl = wp[1 + NC1 + k];
                                racc[1 + NC1 + k][0] += fl * ia;
                                racc[1 + NC1 + k][1] += fl * ib;
                                racc[1 + NC1 + k][2] += fl * ic;
                                racc[1 + NC1 + k][3] += fl * id;
                            }
                        }
                    }
                }
                tc_fence_before();
                mbar_arrive(segfree0 + 8 * b);
            }
        }
        if (epi_sync_or(bad)) bad = 1;
        if (!bad && eact) {
            // phase-matrix elements: ((A + B) / 4, (A - B) / 4, -C / 2, D / 2)
            const int jj = emir ? n_qang - 1 - ej : ej;
            const int Q = 4 * (1 + B.nd);
            double *pc = part + C.part_off + (size_t) it.g * Q * n_qang;
#pragma unroll
            for (int s = 0; s < 1 + NC1 + TC_MAX_ND2; ++s) {
                if (s >= NS) break;
                const int slot = s == 0 ? 0 : (s <= NC1 ? slot1[s - 1] : 1 + B.idx2[s - 1 - NC1]);
                double *o = pc + (size_t) slot * 4 * n_qang + jj;
                o[0] = .25 * (racc[s][0] + racc[s][1]);
                o[(size_t) n_qang] = .25 * (racc[s][0] - racc[s][1]);
                o[(size_t) 2 * n_qang] = -.5 * racc[s][2];
                o[(size_t) 3 * n_qang] = .5 * racc[s][3];
            }
        }
    }
    if (bad) atomicExch(err, 1);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, TC_TMEM_COLS);
    }
}

// ---------------------------------------------------------------------------
// Self-test of the contraction machinery: D[128 x TC_NP] = A[128 x K] B^T with
// A, B given in FP64 (row-major, K contiguous), K a multiple of TC_KC, one
// block of 128 threads, the operand split, descriptors, products and
// tensor-memory reads of K3, and one FP32 accumulation over all K (no
// segment sums), so its error shows the accumulation of the tensor cores.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 1) k_tc_selftest(int K, const double *__restrict__ A,
                                                         const double *__restrict__ Bm, double *__restrict__ D,
                                                         int *__restrict__ err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    uint64_t *bars = (uint64_t *) (smem + TC_STAGE);
    uint32_t *tmem_hold = (uint32_t *) (bars + 4);
    const uint32_t a0 = smem_u32(smem), b0 = a0 + TC_ASTAGE, done = smem_u32(bars);
    const int tid = threadIdx.x, warp = tid >> 5;
    if (tid == 0) {
        mbar_init(done, 1);
        fence_mbar_init();
    }
    if (warp == 0) tmem_alloc(smem_u32(tmem_hold), TC_TMEM_COLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_hold;
    float *as = (float *) smem, *bs = (float *) (smem + TC_ASTAGE);
    uint32_t ph = 0;
    int bad = 0;
    for (int kc = 0; kc * TC_KC < K && !bad; ++kc) {
        // A: row tid; B: row tid (< TC_NP)
        for (int kk = 0; kk < TC_KC; ++kk) {
            const int k = kc * TC_KC + kk;
            float h, l;
            tc_split(A[(size_t) tid * K + k], h, l);
            as[tc_idx(tid, kk, TC_M)] = h;
            as[TC_APART / 4 + tc_idx(tid, kk, TC_M)] = l;
            for (int n = tid; n < TC_NP; n += 128) {
                tc_split(Bm[(size_t) n * K + k], h, l);
                bs[tc_idx(n, kk, TC_NP)] = h;
                bs[TC_BPART / 4 + tc_idx(n, kk, TC_NP)] = l;
            }
        }
        fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            issue_chunk(a0, b0, tmem, tmem + TC_GCOL, kc == 0, kc == 0);
            mma_commit(done);
        }
        const int lbad = !mbar_wait(done, ph, err);
        ph ^= 1u;
        bad = __syncthreads_or(lbad);
    }
    if (!bad) {
        tc_fence_after();
        const uint32_t trow = tmem + ((uint32_t) (warp * 32) << 16);
        for (int c = 0; c < TC_NP; c += 2) {
            uint32_t x, y, gx, gy;
            tmem_ld2(trow + c, x, y);
            tmem_ld2(trow + TC_GCOL + c, gx, gy);
            tmem_wait_ld();
            reg_after_wait(x);
            reg_after_wait(y);
            reg_after_wait(gx);
            reg_after_wait(gy);
            D[(size_t) tid * TC_NP + c] = (double) __uint_as_float(x) + (double) __uint_as_float(gx);
            D[(size_t) tid * TC_NP + c + 1] = (double) __uint_as_float(y) + (double) __uint_as_float(gy);
        }
    } else if (tid == 0) {
        atomicExch(err, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, TC_TMEM_COLS);
    }
}

template <int NC1>
int launch_tc(cudaStream_t s, const DevBatch &B, int nitems, const AngItem *items, const float *bop, double *part,
              int seg, int *err) {
    static bool attr = false;
    if (!attr) {
        LMIEB_CUDA_TRY(cudaFuncSetAttribute(k_angular_tc<NC1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int) TC_SMEM));
        attr = true;
    }
    k_angular_tc<NC1><<<nitems, TC_T, TC_SMEM, s>>>(B, items, bop, part, seg, err);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace

int launch_angular_tc(cudaStream_t s, const DevBatch &B, int nitems, const AngItem *items, const float *bop,
                      double *part, int seg, int *err) {
    if (nitems <= 0) return 0;
    if (seg < 1) {
        fprintf(stderr, "ERROR: lmie_b200: tensor-core segment length %d < 1\n", seg);
        return -1;
    }
    switch (B.nd1) {
        case 0: return launch_tc<0>(s, B, nitems, items, bop, part, seg, err);
        case 1: return launch_tc<1>(s, B, nitems, items, bop, part, seg, err);
        case 2: return launch_tc<2>(s, B, nitems, items, bop, part, seg, err);
        case 3: return launch_tc<3>(s, B, nitems, items, bop, part, seg, err);
        case 4: return launch_tc<4>(s, B, nitems, items, bop, part, seg, err);
    }
    fprintf(stderr, "ERROR: lmie_b200: tensor-core angular stage built for at most %d index1 columns\n", TC_MAX_NC1);
    return -1;
}

int launch_tc_selftest(cudaStream_t s, int K, const double *A, const double *Bm, double *D, int *err) {
    static bool attr = false;
    const int smem = (int) (TC_STAGE + 64);
    if (!attr) {
        LMIEB_CUDA_TRY(cudaFuncSetAttribute(k_tc_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        attr = true;
    }
    k_tc_selftest<<<1, 128, smem, s>>>(K, A, Bm, D, err);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}
