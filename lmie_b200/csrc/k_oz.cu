// k_oz.cu -- K3 as an exact fixed-point contraction on the int8 tensor cores
// (LMIEB_PRECISION_INT8; operand format in oz_layout.cuh).
//
// The S1/S2 sums over orders (reference src/lmie_core.c:658-721) of one case
// are the product A+ [S | D'] of 128 rows (64 half-angles of a tile and their
// mirrors, interleaved) by the OZ_NP operand rows of a radius group, over the
// orders.  Four kernels:
//   - k_oz_rowexp: per half-angle, the row exponents g_r of both of its rows
//     for every chunk count a group of its case can have (running maxima of
//     |pi +- tau| 2^-e_k along the same recurrence the product kernel runs);
//   - k_oz_aop: per product row of every angle tile, the pi/tau recurrence
//     over the case's orders and the row's six digit slices of every chunk
//     (the A operand is the same for all radius groups of the case);
//   - k_oz_bop: per radius group, the column exponents f_n and the six digit
//     slices of the B operand, chunk by chunk, from K1's FP64 coefficient
//     columns;
//   - k_angular_oz: a block owns one angle tile of one case and a range of its
//     radius groups; per group, chunks of OZ_KC orders flow through the
//     pipeline:
//       * warps 0-3 (one thread per row, the row's tensor-memory lane) load
//         the chunk's A digit slices of their row -- formed once per (case,
//         angle tile, chunk) by k_oz_aop -- and store them into the A stage
//         in tensor memory (two stages);
//       * lane 0 of warp 9 brings the group's B chunks into shared memory with
//         bulk copies running ahead of the products;
//       * lane 0 of warp 8 issues the 21 digit products of a chunk,
//         tcgen05.mma kind::i8 with A in tensor memory and B in shared memory
//         (M 128, N OZ_NP, K 32, int32 accumulation in tensor memory), one
//         accumulator per digit diagonal;
//       * after a group's last chunk warps 4-7 (S columns) and 0-3 (D'
//         columns) read the six accumulators of their row (tensor-memory
//         lane = row), form C exactly (int64 halves, then FP64) into a
//         shared-memory buffer and hand the accumulators back, so the next
//         group's products start;
//       * warps 10-13 form, from the buffer and while the next group's
//         products run, the phase-matrix quadratic forms and their
//         linearisations per radius (reference src/lmie_core.c:723-790; sm of
//         a row is in its pair row), accumulated over the block's radii in
//         registers.
// The integer sums are exact, so nothing is drained during a group.
// Partials go to the same per-group buffer as the FP64 K3.
//
// Tensor memory: the accumulator of diagonal d at columns [d OZ_NP, (d + 1)
// OZ_NP); A stage s at OZ_ACOL + s OZ_ACOLS, slice i at +8 i.
//
// Every wait is bounded (about 1 s of clock, or until another block has
// failed); a block that gives up sets the error word, waits (bounded) for
// its tensor-core work and copies in flight, releases its tensor memory and
// returns.
#include <climits>
#include <cstdio>

#include "kernels.h"
#include "oz_layout.cuh"
#include "tc_ptx.cuh"

namespace {

constexpr int OZ_T = 448;                     // warps 0-3: A stages, D' sums; 4-7: S sums; 8: products;
                                              // 9: B copies; 10-13: quadratic forms
constexpr int OZ_MMA_WARP = 8, OZ_COPY_WARP = 9, OZ_QUAD_WARP = 10;
constexpr int OZ_ASTAGES = 2;                 // A operand stages (tensor memory)
constexpr int OZ_BSLOTS = 4;                  // B operand slots (bulk copies)
constexpr int OZ_MAX_GN = OZ_NHALF / 2;       // radii of a group (oz_rg(0))
constexpr int OZ_MAX_NS = 1 + OZ_MAX_NC1 + OZ_MAX_ND2;
constexpr uint32_t OZ_ACOLS = OZ_ND * OZ_KC / 4;                 // tensor-memory columns of an A stage
constexpr uint32_t OZ_ACOL = OZ_ND * OZ_NP;                      // first A stage column
// barriers: afull[OZ_ASTAGES], adone[OZ_ASTAGES], bfull[OZ_BSLOTS], bdone[OZ_BSLOTS], accfull, accfree,
// hready[2], hfree[2], fin
constexpr int OZ_NBAR = 2 * OZ_ASTAGES + 2 * OZ_BSLOTS + 7;
constexpr uint32_t OZ_RING = OZ_BSLOTS * OZ_BSTAGE;
constexpr int OZ_HB = OZ_NP * OZ_M;                         // doubles of one sums buffer
constexpr uint32_t OZ_HBUF = 2 * OZ_HB * 8;                 // two groups' sums, unscaled, [column][row]
constexpr uint32_t OZ_WBUF = OZ_MAX_GN * OZ_MAX_NS * 8;     // a group's radius weights
constexpr uint32_t OZ_CBUF = OZ_NP * 8;                     // a group's column scales
// shared-memory offsets
constexpr uint32_t OZ_O_HBUF = OZ_RING, OZ_O_WBUF = OZ_O_HBUF + OZ_HBUF;
constexpr uint32_t OZ_O_CBUF = OZ_O_WBUF + OZ_WBUF;
constexpr uint32_t OZ_O_BARS = OZ_O_CBUF + OZ_CBUF;
constexpr uint32_t OZ_SMEM = OZ_O_BARS + OZ_NBAR * 8 + 16;
constexpr uint32_t OZ_TMEM_COLS = 512;


static_assert(OZ_BSTAGE % 1024 == 0, "stages stay 1 KB aligned");
static_assert(OZ_NP % 16 == 0 && OZ_NP >= 16 && OZ_NP <= 256, "N of an M=128 kind::i8 product");
static_assert(OZ_ACOL + OZ_ASTAGES * OZ_ACOLS <= OZ_TMEM_COLS, "accumulators and A stages in tensor memory");
static_assert(OZ_WBUF % 16 == 0 && OZ_CBUF % 16 == 0, "barriers stay 8-byte aligned");
static_assert(OZ_SMEM <= 227 * 1024, "shared memory per block");
// |V| <= 2^(OZ_FRAC - 1) must stay inside the six balanced digits (-0x808080808080 .. 0x7f7f7f7f7f7f)
static_assert(OZ_FRAC - 1 <= 8 * OZ_ND - 2, "digit weights: the top digit holds |V| / 2^40 <= 64");
static_assert(OZ_ND == 6, "oz_combine splits the six diagonals into two int64 halves");

// instruction descriptor of kind::i8: D int32, A and B signed 8-bit, both K-major
__host__ __device__ constexpr uint32_t idesc_i8(int m, int n) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t) (n >> 3) << 17) | ((uint32_t) (m >> 4) << 24);
}

// true in one lane of a converged warp (the lowest)
__device__ __forceinline__ bool elect_one() {
    uint32_t pred = 0;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "elect.sync _|P, 0xffffffff;\n\t"
        "selp.u32 %0, 1, 0, P;\n\t}"
        : "=r"(pred));
    return pred != 0;
}

// A from tensor memory (column address a), B from shared memory
__device__ __forceinline__ void mma_i8_ts(uint32_t d, uint32_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d),
        "r"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

// warp-wide: four consecutive 32-bit columns of this thread's lane
__device__ __forceinline__ void tmem_st4(uint32_t taddr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr), "r"(a), "r"(b),
                 "r"(c), "r"(d)
                 : "memory");
}

// The OZ_NPROD digit products of one chunk (one thread): a0 the
// tensor-memory column of the chunk's A stage, b0 the shared address of its
// B stage, acc the tensor-memory column of diagonal 0; `first`: the chunk
// opens the group's sums.
__device__ __forceinline__ void issue_chunk_i8(uint32_t a0, uint32_t b0, uint32_t acc, bool first) {
    constexpr uint32_t idesc = idesc_i8(OZ_M, OZ_NP);
    const uint64_t db = sdesc(b0, OZ_LBO_B, 128);
#pragma unroll
    for (int d = 0; d < OZ_ND; ++d)
#pragma unroll
        for (int i = 0; i <= d; ++i) {
            const int j = d - i;
            mma_i8_ts(acc + d * OZ_NP, a0 + i * (OZ_KC / 4), db + (uint64_t) ((j * OZ_BSLICE) >> 4), idesc,
                      (first && i == 0) ? 0u : 1u);
        }
}

// sum_d 2^(-8 d) ACC_d of six int32 accumulators, exactly: U = ACC_0 2^16 +
// ACC_1 2^8 + ACC_2 and L = ACC_3 2^16 + ACC_4 2^8 + ACC_5 are below 2^48 in
// magnitude, become doubles exactly (x + 1.5 2^52 read as an integer), and
// the result is 2^-16 (U + 2^-24 L) with one rounding; times `scale`.
__device__ __forceinline__ longlong2 oz_halves(const uint32_t (&a)[OZ_ND]) {
    const long long U = (long long) (int) a[0] * 65536 + (long long) (int) a[1] * 256 + (long long) (int) a[2];
    const long long L = (long long) (int) a[3] * 65536 + (long long) (int) a[4] * 256 + (long long) (int) a[5];
    return make_longlong2(U, L);
}

// U + 2^-24 L with one rounding (the scale that follows is a power of two)
__device__ __forceinline__ double oz_unscaled(longlong2 h) {
    const double dU = __longlong_as_double(h.x + 0x4338000000000000LL) - 6755399441055744.0;
    const double dL = __longlong_as_double(h.y + 0x4338000000000000LL) - 6755399441055744.0;
    return fma(dL, 5.9604644775390625e-08, dU);   // 2^-24
}

__device__ __forceinline__ double oz_value(longlong2 h, double scale) { return oz_unscaled(h) * scale; }

__device__ __forceinline__ double oz_combine(const uint32_t (&a)[OZ_ND], double scale) {
    return oz_value(oz_halves(a), scale);
}

// The exact sums of `ncol` columns (a multiple of 8) of this thread's lane:
// six accumulators per column from tensor memory (taddr: the lane's first
// column of diagonal 0), eight columns per wait, unscaled values to
// hb[c OZ_M] (warp-wide).
__device__ __forceinline__ void oz_read_sums(uint32_t taddr, int ncol, double *hb) {
#pragma unroll 1
    for (int c = 0; c < ncol; c += 8) {
        uint32_t a[OZ_ND][8];
#pragma unroll
        for (int d = 0; d < OZ_ND; ++d) tmem_ld8(taddr + d * OZ_NP + c, a[d]);
        tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            uint32_t col[OZ_ND];
#pragma unroll
            for (int d = 0; d < OZ_ND; ++d) {
                reg_after_wait(a[d][i]);
                col[d] = a[d][i];
            }
            hb[(c + i) * OZ_M] = oz_unscaled(oz_halves(col));
        }
    }
}

// ---------------------------------------------------------------------------
// Row exponents: thread per (case, half-angle) of the flat index space
// `start`; table entry [C.rx_off + (h C.nkx + c) 2 + mirror] = g of row 2h +
// mirror for the orders 1 .. (c + 1) OZ_KC.
// ---------------------------------------------------------------------------
__global__ void k_oz_rowexp(DevBatch B, long long total, const long long *__restrict__ start,
                            signed char *__restrict__ tab) {
    const long long e = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const int c = find_case(start, B.ncase, e);
    const DevCase &C = B.cs[c];
    const int h = (int) (e - start[c]);
    const double mu = B.mu_pool[C.mu_off + h];
    signed char *o = tab + C.rx_off + (size_t) h * C.nkx * 2;
    double p0 = 0., p1 = 1., kmu = mu, k1 = 2., mp = 0., mm = 0.;
    for (int kc = 0; kc < C.nkx; ++kc) {
        for (int u = 0; u < OZ_KC; ++u) {
            const int k = kc * OZ_KC + u + 1;
            const double s = oz_pow2(-oz_ek(k));
            const double pk = p1;
            double tau;
            oz_step(mu, B.oz_f2[k], kmu, k1, p0, p1, tau);
            mp = fmax(mp, fabs(pk + tau) * s);
            mm = fmax(mm, fabs(pk - tau) * s);
        }
        o[2 * kc] = (signed char) oz_exp_of(mp);
        o[2 * kc + 1] = (signed char) oz_exp_of(mm);
    }
}

// ---------------------------------------------------------------------------
// B operand of the radius groups: block per group, thread per operand row
// n = tid % 64 (S re, S im, ..., then D' re, D' im, ...) and every fourth
// block of 16 orders.  The column exponent f_n (largest ilogb(|v| 2^e_k) + 2
// over the column) comes from the exponents K1 tracked while it wrote the
// coefficients; the kernel writes the digit slices of every chunk; rows and
// orders without a value get zero.
// ---------------------------------------------------------------------------
constexpr int OZ_BOP_T = 256;
constexpr int OZ_BOP_J = OZ_BOP_T / OZ_NP;            // threads per row

__global__ void __launch_bounds__(OZ_BOP_T) k_oz_bop(DevBatch B, const double *__restrict__ coef,
                                                      unsigned char *__restrict__ bop, int *__restrict__ colexp) {
    const int g = blockIdx.x, tid = threadIdx.x;
    const int r0 = B.tg_r0[g], gn = B.tg_n[g], nk = B.tg_nk[g];
    const int C1 = 1 + B.nd1, P = gn * C1;
    const int n = tid % OZ_NP, j0 = tid / OZ_NP;
    const int rp = (n % OZ_NHALF) >> 1;               // operand column pair (radius, Mie column)
    const int comp = (n >= OZ_NHALF ? 2 : 0) + (n & 1);   // re/im of S, then of D'
    const bool real = rp < P, dpart = n >= OZ_NHALF;
    const double *cf = coef + comp;                   // component `comp` of the double4 entries
    const size_t tot = (size_t) B.tot;
    int n1 = 0, f = 0;
    size_t base = 0;
    if (real) {
        const int p = rp / C1, col = rp - p * C1, r = r0 + p;
        n1 = B.n1r[r];
        base = ((size_t) col * tot + B.off[r]) * 4;
        // largest biased exponent + e_k: f = that - 1021 (0: the column is zero)
        const int m = B.oz_radexp[((size_t) col * B.R + r) * 4 + comp];
        f = m ? max(m - 1021, -900) : 0;
    }
    if (j0 == 0) colexp[(size_t) g * OZ_NP + n] = f;
    // digits, 16 orders at a time
    unsigned char *rb = bop + B.tg_off[g] + (n >> 3) * 128 + (n & 7) * 16;
    for (int blk = j0; blk < 2 * nk; blk += OZ_BOP_J) {
        uint32_t w[OZ_ND][4];
#pragma unroll
        for (int qd = 0; qd < 4; ++qd) {
            uint32_t lo[4], hi[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int k = blk * 16 + qd * 4 + u + 1;
                double v = k <= n1 ? __ldg(cf + base + (size_t) (k - 1) * 4) : 0.;
                if (dpart && !(k & 1)) v = -v;        // s_k of D'
                oz_digits(v, oz_pow2(OZ_FRAC + oz_ek(k) - f), lo[u], hi[u]);
            }
            uint32_t s6[OZ_ND];
            oz_slices4(lo, hi, s6);
#pragma unroll
            for (int s = 0; s < OZ_ND; ++s) w[s][qd] = s6[s];
        }
        unsigned char *cb = rb + (size_t) (blk >> 1) * OZ_BSTAGE + (blk & 1) * OZ_LBO_B;
#pragma unroll
        for (int s = 0; s < OZ_ND; ++s)
            *(uint4 *) (cb + s * OZ_BSLICE) = make_uint4(w[s][0], w[s][1], w[s][2], w[s][3]);
    }
}

// The pi/tau recurrence of one product row over 16 orders (recurrence
// thread): the row's values (pi_k + sg tau_k) into v; sg = +1 (row 2h) or -1
// (its mirror).
__device__ __forceinline__ void oz_recur_half(const double *__restrict__ f2, double mu, double sg, double &kmu,
                                              double &k1, double &p0, double &p1, double (&v)[16]) {
    // the (k + 1) / k of eight orders at a time ahead of the dependent steps
#pragma unroll
    for (int u0 = 0; u0 < 16; u0 += 8) {
        double f[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) f[u] = f2[u0 + u];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const double pk = p1;
            double tau;
            oz_step(mu, f[u], kmu, k1, p0, p1, tau);
            v[u0 + u] = fma(sg, tau, pk);
        }
    }
}

// The digits of half hf (orders 16 hf .. 16 hf + 15) of a chunk of one
// product row (recurrence thread): w[2u], w[2u + 1] = the low and high words
// of oz_digits of row value v[u].  sp / sm: the scales of odd / even orders
// (the mirror row carries s_k); FIRST: the case's first chunk, whose orders
// 1..16 have their own exponents (gsc = 2^(OZ_FRAC - g_r), 0 for an inactive
// row).
template <bool FIRST>
__device__ __forceinline__ void oz_digit_words(const double (&v)[16], int hf, double sg, double sp, double sm,
                                               double gsc, uint32_t (&w)[32]) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
        double sc = (u & 1) ? sm : sp;
        if (FIRST && hf == 0) {
            // 2^(OZ_FRAC - e_k - g_r) with e_k = ceil(log2 2k), k = u + 1 (compile-time)
            constexpr double inv[5] = {0.5, 0.25, 0.125, 0.0625, 0.03125};
            const int ek = u == 0 ? 1 : (u == 1 ? 2 : (u < 4 ? 3 : (u < 8 ? 4 : 5)));
            sc = (u & 1) ? sg * gsc * inv[ek - 1] : gsc * inv[ek - 1];
        }
        oz_digits(v[u], sc, w[2 * u], w[2 * u + 1]);
    }
}

// ---------------------------------------------------------------------------
// A operand: thread per product row of every angle tile of every case (flat
// index space `start`, OZ_M rows per tile): the pi/tau recurrence over the
// case's orders; each chunk's row values scaled by 2^(OZ_FRAC - e_k - g_r),
// g_r the row's exponent over all the case's orders (the largest entry of its
// table), their digits and the row's six digit slices, OZ_AROW bytes per
// chunk as OZ_AROW / 16 pieces of 16 bytes, piece i (slice i / 2, orders
// 16 (i % 2) .. + 15) of the row at aop[C.a_off + (tile nkx + chunk)
// OZ_ACHUNK + (i OZ_M + row) 16]: the rows of a piece are consecutive, so the
// product kernel's warps read 512 contiguous bytes per load.  Rows past the
// case's angles get the digits of zero.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_oz_aop(DevBatch B, long long total, const long long *__restrict__ start,
                                                unsigned char *__restrict__ aop) {
    const long long e = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const int c = find_case(start, B.ncase, e);
    const DevCase &C = B.cs[c];
    const long long q = e - start[c];
    const int t = (int) (q / OZ_M), row = (int) (q % OZ_M);
    const int h = t * OZ_HALF + (row >> 1), mirror = row & 1;
    const bool gact = h < C.nh;
    const double mu = gact ? B.mu_pool[C.mu_off + h] : 0.;
    const double sg = mirror ? -1. : 1.;
    const int gr = gact ? (int) B.oz_rowexp[C.rx_off + ((size_t) h * C.nkx + C.nkx - 1) * 2 + mirror] : 0;
    const double gsc = gact ? oz_pow2(OZ_FRAC - gr) : 0.;
    uint4 *dst = (uint4 *) (aop + C.a_off + (size_t) t * C.nkx * OZ_ACHUNK) + row;
    double p0 = 0., p1 = 1., kmu = mu, k1 = 2.;        // pi_{k-1}, pi_k, k mu, k + 1
    for (int kc = 0; kc < C.nkx; ++kc) {
        // the chunk's scale 2^(OZ_FRAC - e_k - g_r); the mirror row carries s_k
        const double sp = gsc * oz_pow2(-oz_ec(kc));
        const double sm = mirror ? -sp : sp;
        uint32_t w[OZ_ND][8];
#pragma unroll
        for (int hf = 0; hf < 2; ++hf) {
            double v[16];
            oz_recur_half(B.oz_f2 + kc * OZ_KC + hf * 16 + 1, mu, sg, kmu, k1, p0, p1, v);
            uint32_t dw[32];
            if (kc == 0 && hf == 0)
                oz_digit_words<true>(v, 0, sg, sp, sm, gsc, dw);
            else
                oz_digit_words<false>(v, hf, sg, sp, sm, gsc, dw);
#pragma unroll
            for (int qd = 0; qd < 4; ++qd) {
                uint32_t s6[OZ_ND];
                const uint32_t l4[4] = {dw[8 * qd], dw[8 * qd + 2], dw[8 * qd + 4], dw[8 * qd + 6]};
                const uint32_t h4[4] = {dw[8 * qd + 1], dw[8 * qd + 3], dw[8 * qd + 5], dw[8 * qd + 7]};
                oz_slices4(l4, h4, s6);
#pragma unroll
                for (int sl = 0; sl < OZ_ND; ++sl) w[sl][hf * 4 + qd] = s6[sl];
            }
        }
        uint4 *dc = dst + (size_t) kc * (OZ_ACHUNK / 16);
#pragma unroll
        for (int sl = 0; sl < OZ_ND; ++sl) {
            dc[(2 * sl) * OZ_M] = make_uint4(w[sl][0], w[sl][1], w[sl][2], w[sl][3]);
            dc[(2 * sl + 1) * OZ_M] = make_uint4(w[sl][4], w[sl][5], w[sl][6], w[sl][7]);
        }
    }
}

// barrier 2 over the 128 threads of warps 4-7, OR-reducing v
__device__ __forceinline__ int oz_epi_sync_or(int v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "bar.red.or.pred p, 2, 128, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(r)
        : "r"(v)
        : "memory");
    return (int) r;
}

// ---------------------------------------------------------------------------
// The product kernel.
// ---------------------------------------------------------------------------
template <int NC1>
__global__ void __launch_bounds__(OZ_T, 1) k_angular_oz(DevBatch B, const AngItem *__restrict__ items,
                                                        const unsigned char *__restrict__ bop,
                                                        double *__restrict__ part, int *__restrict__ err) {
    constexpr int C1 = 1 + NC1, CPR = 2 * C1;
    extern __shared__ __align__(1024) unsigned char smem[];
    double *hbuf = (double *) (smem + OZ_O_HBUF);            // [2][OZ_NP][OZ_M] sums of a group, unscaled
    double *wsh = (double *) (smem + OZ_O_WBUF);             // [OZ_MAX_GN][OZ_MAX_NS] weights
    double *csh = (double *) (smem + OZ_O_CBUF);             // [OZ_NP] column scales
    uint64_t *bars = (uint64_t *) (smem + OZ_O_BARS);
    uint32_t *tmem_hold = (uint32_t *) (bars + OZ_NBAR);
    const uint32_t bring = smem_u32(smem);
    const uint32_t afull0 = smem_u32(bars), adone0 = afull0 + 8 * OZ_ASTAGES;
    const uint32_t bfull0 = adone0 + 8 * OZ_ASTAGES, bdone0 = bfull0 + 8 * OZ_BSLOTS;
    const uint32_t accfull = bdone0 + 8 * OZ_BSLOTS, accfree = accfull + 8;
    const uint32_t hready0 = accfree + 8, hfree0 = hready0 + 16, fin = hfree0 + 16;

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
        for (int i = 0; i < OZ_ASTAGES; ++i) {
            mbar_init(afull0 + 8 * i, OZ_M);
            mbar_init(adone0 + 8 * i, 1);
        }
        for (int i = 0; i < OZ_BSLOTS; ++i) {
            mbar_init(bfull0 + 8 * i, 1);
            mbar_init(bdone0 + 8 * i, 1);
        }
        mbar_init(accfull, 1);
        mbar_init(accfree, 256);
        for (int i = 0; i < 2; ++i) {
            mbar_init(hready0 + 8 * i, 256);
            mbar_init(hfree0 + 8 * i, 128);
        }
        mbar_init(fin, 1);
        fence_mbar_init();
    }
    if (warp == 0) tmem_alloc(smem_u32(tmem_hold), OZ_TMEM_COLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_hold;
    int bad = 0;

    if (tid < OZ_M) {
        // ---------------- warps 0-3: the A digit slices, one row (lane) per thread ----------------
        const int row = tid;
        const uint32_t tlane = tmem + ((uint32_t) (warp * 32) << 16);
        // this row's A digit slices: piece i of chunk kc of the item's angle
        // tile at arow[kc OZ_ACHUNK / 16 + i OZ_M]
        const uint4 *arow = (const uint4 *) (B.oz_aop + C.a_off + (size_t) it.xt * C.nkx * OZ_ACHUNK) + row;
        // The digit warps take the D' columns of a group's finished sums out of
        // tensor memory (warps 4-7 take the S columns): once the quadratic
        // forms are done with the buffer's previous group, after the group's
        // last products.  Returns nonzero when a wait gave up.
        auto take = [&](int gh) -> int {
            const int g = it.rbeg + gh, ncol = B.tg_n[g] * CPR;
            // the buffer's previous group (gh - 2) has been through the quadratic forms
            const int b = gh & 1;
            bool ok = gh < 2 || mbar_wait(hfree0 + 8 * b, ((gh >> 1) - 1) & 1, err);
            ok = ok && mbar_wait(accfull, gh & 1, err);
            double *hb = hbuf + b * OZ_HB;
            if (__any_sync(0xffffffffu, !ok)) return 1;
            tc_fence_after();
            oz_read_sums(tlane + OZ_NHALF, (ncol + 7) & ~7, hb + OZ_NHALF * OZ_M + row);
            tc_fence_before();
            mbar_arrive(accfree);
            mbar_arrive(hready0 + 8 * b);
            return 0;
        };
        int q = 0, gi = 0, hold_next = 0;
        int sgrp[OZ_ASTAGES];                              // group of the chunk last written to each stage
#pragma unroll
        for (int i = 0; i < OZ_ASTAGES; ++i) sgrp[i] = 0;
        for (int g = it.rbeg; g < it.rend && !bad; ++g, ++gi) {
            const int nk = B.tg_nk[g];
            for (int kc = 0; kc < nk; ++kc, ++q) {
                const int s = q % OZ_ASTAGES;
                // the stage's previous chunk must have been consumed by its products,
                // which reach its group once the sums of every earlier group are out;
                // warp-uniform decisions: the tensor-memory accesses are warp-wide
                if (q >= OZ_ASTAGES)
                    while (!bad && hold_next < sgrp[s]) bad = take(hold_next++);
                if (bad) break;
                // the chunk's digit slices of this row, loaded before the wait
                const uint4 *ac = arow + (size_t) kc * (OZ_ACHUNK / 16);
                uint4 a[2 * OZ_ND];
#pragma unroll
                for (int i = 0; i < 2 * OZ_ND; ++i) a[i] = ac[i * OZ_M];
                const bool ok = q < OZ_ASTAGES || mbar_wait(adone0 + 8 * s, ((q / OZ_ASTAGES) - 1) & 1, err);
                if (__any_sync(0xffffffffu, !ok)) {
                    bad = 1;
                    break;
                }
                tc_fence_after();
                const uint32_t acol = tlane + OZ_ACOL + s * OZ_ACOLS;
#pragma unroll
                for (int sl = 0; sl < OZ_ND; ++sl) {
                    tmem_st4(acol + sl * (OZ_KC / 4), a[2 * sl].x, a[2 * sl].y, a[2 * sl].z, a[2 * sl].w);
                    tmem_st4(acol + sl * (OZ_KC / 4) + 4, a[2 * sl + 1].x, a[2 * sl + 1].y, a[2 * sl + 1].z,
                             a[2 * sl + 1].w);
                }
                tmem_wait_st();
                tc_fence_before();
                sgrp[s] = gi;
                mbar_arrive(afull0 + 8 * s);
            }
        }
        while (!bad && hold_next < it.rend - it.rbeg) bad = take(hold_next++);
    } else if (warp >= OZ_QUAD_WARP) {
        // ---------------- warps 10-13: quadratic forms, one row per thread ----------------
        // A warp whose wait fails keeps taking the barriers of the four warps,
        // which stop together.
        const int t1 = tid - OZ_QUAD_WARP * 32;              // product row
        const int eh = t1 >> 1, emir = t1 & 1;
        const int ej = it.xt * OZ_HALF + eh;
        const bool eact = ej < nh;
        const signed char *gtab = B.oz_rowexp + C.rx_off + (size_t) (eact ? ej : 0) * C.nkx * 2 + emir;
        int slot1[NC1 > 0 ? NC1 : 1];
#pragma unroll
        for (int k = 0; k < NC1; ++k) slot1[k] = 1 + B.idx1[k];
        // per column set: f-weighted sums over radii of the four invariants
        double racc[1 + NC1 + OZ_MAX_ND2][4];
#pragma unroll
        for (int s = 0; s < 1 + NC1 + OZ_MAX_ND2; ++s)
#pragma unroll
            for (int e = 0; e < 4; ++e) racc[s][e] = 0.;
        // the scales of this row and of its pair row (which holds this row's sm)
        const double rsc = oz_pow2(eact ? (int) gtab[2 * (C.nkx - 1)] : 0);
        const double rsp = __shfl_xor_sync(0xffffffffu, rsc, 1);
        // A group's radius weights (gn NS <= OZ_MAX_GN OZ_MAX_NS = 128 values:
        // at most one per thread) and column scales (with the row-independent
        // factor of the combination), fetched into registers one group ahead
        // so that their loads overlap the previous group's forms.
        double wnext = 0., cnext = 0.;
        auto fetch = [&](int g) {
            const int gn = B.tg_n[g];
            if (t1 < gn * NS && gn <= OZ_MAX_GN) {
                const int p = t1 / NS, s = t1 - p * NS;
                const int slot = s == 0 ? 0 : (s <= NC1 ? slot1[s - 1] : 1 + B.idx2[s - 1 - NC1]);
                wnext = B.w[(size_t) slot * R + B.tg_r0[g] + p];
            }
            if (t1 < OZ_NP) cnext = oz_pow2(B.oz_colexp[(size_t) g * OZ_NP + t1] + OZ_CSHIFT);
        };
        if (it.rbeg < it.rend) fetch(it.rbeg);
        int gi = 0;
        for (int g = it.rbeg; g < it.rend; ++g, ++gi) {
            const int gn = B.tg_n[g];
            // the previous group's weights and scales have been read by all four warps
            if (oz_epi_sync_or(bad || gn > OZ_MAX_GN)) {
                bad = 1;
                break;
            }
            if (t1 < gn * NS) {
                const int p = t1 / NS;
                wsh[p * OZ_MAX_NS + (t1 - p * NS)] = wnext;
            }
            if (t1 < OZ_NP) csh[t1] = cnext;
            oz_epi_sync_or(0);
            // the next group's loads, in flight during this group's forms (a
            // barrier waits for the loads issued before it)
            if (g + 1 < it.rend) fetch(g + 1);
            // both halves of the group's sums are in its buffer
            const double *hb = hbuf + (gi & 1) * OZ_HB;
            if (__any_sync(0xffffffffu, !mbar_wait(hready0 + 8 * (gi & 1), (gi >> 1) & 1, err))) {
                bad = 1;
                continue;
            }
            // The row scales are left out here: every term of racc[s][0] carries
            // rsc^2, of racc[s][1] rsp^2 and of racc[s][2..3] rsc rsp (powers of
            // two, applied once at the end).
            for (int p = 0; p < gn; ++p) {
                // columns of S (i < CPR, this row) and D' (i >= CPR, the pair row: sm)
                double v[2 * CPR];
#pragma unroll
                for (int i = 0; i < CPR; ++i) {
                    const int cs = p * CPR + i, cd = OZ_NHALF + p * CPR + i;
                    v[i] = hb[cs * OZ_M + t1] * csh[cs];
                    v[CPR + i] = hb[cd * OZ_M + (t1 ^ 1)] * csh[cd];
                }
                const double *wp = wsh + p * OZ_MAX_NS;
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
                for (int k = 0; k < OZ_MAX_ND2; ++k) {
                    if (k < nd2) {
                        const double fl = wp[1 + NC1 + k];
                        racc[1 + NC1 + k][0] += fl * ia;
                        racc[1 + NC1 + k][1] += fl * ib;
                        racc[1 + NC1 + k][2] += fl * ic;
                        racc[1 + NC1 + k][3] += fl * id;
                    }
                }
            }
            // the buffer is free for the group after next
            mbar_arrive(hfree0 + 8 * (gi & 1));
        }
        if (oz_epi_sync_or(bad)) bad = 1;
        if (!bad && eact) {
            // phase-matrix elements: ((A + B) / 4, (A - B) / 4, -C / 2, D / 2),
            // with the row scales
            const int jj = emir ? n_qang - 1 - ej : ej;
            const int Q = 4 * (1 + B.nd);
            double *pc = part + C.part_off + (size_t) it.g * Q * n_qang;
            const double ss = rsc * rsc, mm = rsp * rsp, sm = rsc * rsp;
#pragma unroll
            for (int s = 0; s < 1 + NC1 + OZ_MAX_ND2; ++s) {
                if (s >= NS) break;
                const int slot = s == 0 ? 0 : (s <= NC1 ? slot1[s - 1] : 1 + B.idx2[s - 1 - NC1]);
                double *o = pc + (size_t) slot * 4 * n_qang + jj;
                const double a = racc[s][0] * ss, b = racc[s][1] * mm;
                o[0] = .25 * (a + b);
                o[(size_t) n_qang] = .25 * (a - b);
                o[(size_t) 2 * n_qang] = -.5 * (racc[s][2] * sm);
                o[(size_t) 3 * n_qang] = .5 * (racc[s][3] * sm);
            }
        }
    } else if (warp == OZ_COPY_WARP) {
        // ---------------- warp 9, lane 0: B copies, up to OZ_BSLOTS chunks ahead ----------------
        if ((tid & 31) == 0) {
            int pq = 0;
            for (int g = it.rbeg; g < it.rend && !bad; ++g) {
                const int nk = B.tg_nk[g];
                const unsigned char *src = bop + B.tg_off[g];
                for (int kc = 0; kc < nk; ++kc, ++pq) {
                    const int ps = pq % OZ_BSLOTS;
                    // the slot's previous chunk pq - OZ_BSLOTS must have been consumed
                    if (pq >= OZ_BSLOTS && !mbar_wait(bdone0 + 8 * ps, ((pq / OZ_BSLOTS) - 1) & 1, err)) {
                        bad = 1;
                        break;
                    }
                    mbar_expect_tx(bfull0 + 8 * ps, OZ_BSTAGE);
                    bulk_g2s(bring + ps * OZ_BSTAGE, src, OZ_BSTAGE, bfull0 + 8 * ps);
                    src += OZ_BSTAGE;
                }
            }
            // the copies in flight land before the block ends
            const int q0 = pq > OZ_BSLOTS ? pq - OZ_BSLOTS : 0;
            for (int c = q0; c < pq; ++c) mbar_wait(bfull0 + 8 * (c % OZ_BSLOTS), (c / OZ_BSLOTS) & 1, nullptr);
        }
    } else if (warp == OZ_MMA_WARP) {
        // ---------------- warp 8: the products ----------------
        // The whole warp runs the loop (its values stay warp-uniform) and one
        // elected lane issues; the decisions to stop are warp-uniform.
        int q = 0, gi = 0;
        for (int g = it.rbeg; g < it.rend && !bad; ++g, ++gi) {
            const int nk = B.tg_nk[g];
            for (int kc = 0; kc < nk; ++kc, ++q) {
                const int s = q % OZ_ASTAGES, sb = q % OZ_BSLOTS;
                bool ok = mbar_wait(afull0 + 8 * s, (q / OZ_ASTAGES) & 1, err) &&
                          mbar_wait(bfull0 + 8 * sb, (q / OZ_BSLOTS) & 1, err);
                // the previous group's accumulators must have been read
                if (ok && kc == 0 && gi >= 1) ok = mbar_wait(accfree, (gi - 1) & 1, err);
                if (__any_sync(0xffffffffu, !ok)) {
                    bad = 1;
                    break;
                }
                tc_fence_after();
                if (elect_one()) {
                    issue_chunk_i8(tmem + OZ_ACOL + s * OZ_ACOLS, bring + sb * OZ_BSTAGE, tmem, kc == 0);
                    mma_commit(adone0 + 8 * s);
                    mma_commit(bdone0 + 8 * sb);
                    if (kc == nk - 1) mma_commit(accfull);
                }
                __syncwarp();
            }
        }
        // all products of this warp have completed
        if (elect_one()) mma_commit(fin);
        __syncwarp();
        mbar_wait(fin, 0u, nullptr);
    } else if (warp >= 4) {
        // ---------------- warps 4-7: the S sums of each group ----------------
        const int t1 = tid - 128;                            // product row = tensor-memory lane
        const uint32_t trow = tmem + ((uint32_t) ((warp - 4) * 32) << 16);
        int gi = 0;
        for (int g = it.rbeg; g < it.rend && !bad; ++g, ++gi) {
            const int ncol = B.tg_n[g] * CPR;                 // used columns of each half
            // the buffer's previous group has been through the quadratic
            // forms and this group's products are done (warp-uniform: the
            // tensor-memory accesses below are warp-wide)
            const int b = gi & 1;
            bool ok = gi < 2 || mbar_wait(hfree0 + 8 * b, ((gi >> 1) - 1) & 1, err);
            ok = ok && mbar_wait(accfull, gi & 1, err);
            double *hb = hbuf + b * OZ_HB;
            if (__any_sync(0xffffffffu, !ok)) {
                bad = 1;
                break;
            }
            tc_fence_after();
            // the exact sums of the group's used S columns into the buffer
            // (the digit warps take the D' columns); the accumulators go back
            // right after
            oz_read_sums(trow, (ncol + 7) & ~7, hb + t1);
            tc_fence_before();
            mbar_arrive(accfree);
            mbar_arrive(hready0 + 8 * b);
        }
    }
    if (bad) atomicExch(err, 1);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, OZ_TMEM_COLS);
    }
}

// ---------------------------------------------------------------------------
// Self-test of the fixed-point machinery: D[128 x OZ_NP] = A[128 x K] B^T,
// A, B given in FP64 (row-major, K contiguous), K a multiple of OZ_KC up to
// OZ_MAX_NK chunks; one block of 128 threads, the per-chunk, row and column
// scaling, digit slices (A in tensor memory, B in shared memory),
// descriptors, products, accumulators and exact combination of the product
// kernel.  Its waits for the products give up after `wait_cycles`; with
// `withhold` the first chunk's products are never issued, so that wait runs
// out: the block then releases its tensor memory and sets *err (the failure
// path of the product kernel, without a fault).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 1) k_oz_selftest(int K, const double *__restrict__ A,
                                                         const double *__restrict__ Bm, double *__restrict__ D,
                                                         int *__restrict__ err, long long wait_cycles,
                                                         int withhold) {
    extern __shared__ __align__(1024) unsigned char smem[];
    uint64_t *bars = (uint64_t *) (smem + OZ_BSTAGE);
    uint32_t *tmem_hold = (uint32_t *) (bars + 2);
    __shared__ int fB[OZ_NP];
    const uint32_t b0 = smem_u32(smem), done = smem_u32(bars);
    const int tid = threadIdx.x, warp = tid >> 5;
    if (tid == 0) {
        mbar_init(done, 1);
        fence_mbar_init();
    }
    if (warp == 0) tmem_alloc(smem_u32(tmem_hold), OZ_TMEM_COLS);
    // row exponent of A row tid, column exponents of B rows
    double ma = 0.;
    for (int k = 0; k < K; ++k) ma = fmax(ma, fabs(A[(size_t) tid * K + k]) * oz_pow2(-oz_ek(k + 1)));
    const int gA = oz_exp_of(ma);
    if (tid < OZ_NP) {
        double mb = 0.;
        for (int k = 0; k < K; ++k) mb = fmax(mb, fabs(Bm[(size_t) tid * K + k]) * oz_pow2(oz_ek(k + 1)));
        fB[tid] = oz_exp_of(mb);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_hold;
    const uint32_t tlane = tmem + ((uint32_t) (warp * 32) << 16);
    unsigned char *bs = smem;
    uint32_t ph = 0;
    int bad = 0;
    for (int kc = 0; kc * OZ_KC < K && !bad; ++kc) {
        for (int hf = 0; hf < 2; ++hf) {
            uint32_t wa[OZ_ND][4], wb[OZ_ND][4];
            for (int qd = 0; qd < 4; ++qd) {
                uint32_t lo[4], hi[4], lb[4], hb[4];
                for (int u = 0; u < 4; ++u) {
                    const int k = kc * OZ_KC + hf * 16 + qd * 4 + u;
                    const int ek = oz_ek(k + 1);
                    oz_digits(A[(size_t) tid * K + k], oz_pow2(OZ_FRAC - ek - gA), lo[u], hi[u]);
                    const int n = tid & (OZ_NP - 1);
                    oz_digits(Bm[(size_t) n * K + k], oz_pow2(OZ_FRAC + ek - fB[n]), lb[u], hb[u]);
                }
                uint32_t s6[OZ_ND], t6[OZ_ND];
                oz_slices4(lo, hi, s6);
                oz_slices4(lb, hb, t6);
                for (int s = 0; s < OZ_ND; ++s) {
                    wa[s][qd] = s6[s];
                    wb[s][qd] = t6[s];
                }
            }
            for (int s = 0; s < OZ_ND; ++s)
                tmem_st4(tlane + OZ_ACOL + s * (OZ_KC / 4) + hf * 4, wa[s][0], wa[s][1], wa[s][2], wa[s][3]);
            if (tid < OZ_NP) {
                const uint32_t rb = (tid >> 3) * 128 + (tid & 7) * 16 + hf * OZ_LBO_B;
                for (int s = 0; s < OZ_ND; ++s)
                    *(uint4 *) (bs + s * OZ_BSLICE + rb) = make_uint4(wb[s][0], wb[s][1], wb[s][2], wb[s][3]);
            }
        }
        tmem_wait_st();
        fence_proxy_async();
        tc_fence_before();
        __syncthreads();
        if (tid == 0 && !(withhold && kc == 0)) {
            tc_fence_after();
            issue_chunk_i8(tmem + OZ_ACOL, b0, tmem, kc == 0);
            mma_commit(done);
        }
        const int lbad = !mbar_wait_for(done, ph, err, wait_cycles);
        ph ^= 1u;
        bad = __syncthreads_or(lbad);
        tc_fence_after();
    }
    if (!bad) {
        const uint32_t trow = tmem + ((uint32_t) (warp * 32) << 16);
        for (int c = 0; c < OZ_NP; c += 16) {
            uint32_t a[OZ_ND][16];
            for (int d = 0; d < OZ_ND; ++d) tmem_ld16(trow + d * OZ_NP + c, a[d]);
            tmem_wait_ld();
            for (int i = 0; i < 16; ++i) {
                uint32_t col[OZ_ND];
                for (int d = 0; d < OZ_ND; ++d) {
                    reg_after_wait(a[d][i]);
                    col[d] = a[d][i];
                }
                D[(size_t) tid * OZ_NP + c + i] =
                    oz_combine(col, oz_pow2(gA + fB[c + i] + OZ_CSHIFT));
            }
        }
    } else if (tid == 0) {
        atomicExch(err, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, OZ_TMEM_COLS);
    }
}

template <int NC1>
int launch_oz(cudaStream_t s, const DevBatch &B, int nitems, const AngItem *items, const unsigned char *bop,
              double *part, int *err) {
    static bool attr = false;
    if (!attr) {
        LMIEB_CUDA_TRY(cudaFuncSetAttribute(k_angular_oz<NC1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int) OZ_SMEM));
        attr = true;
    }
    k_angular_oz<NC1><<<nitems, OZ_T, OZ_SMEM, s>>>(B, items, bop, part, err);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace

int launch_oz_operands(cudaStream_t s, const DevBatch &B, long long nrow, const long long *row_start,
                       signed char *rowexp, long long narow, const long long *arow_start, unsigned char *aop,
                       int ngroups, const double *coef, unsigned char *bop, int *colexp) {
    if (nrow > 0) {
        k_oz_rowexp<<<ceil_div(nrow, 128), 128, 0, s>>>(B, nrow, row_start, rowexp);
        LMIEB_CUDA_TRY(cudaGetLastError());
    }
    if (narow > 0) {
        k_oz_aop<<<ceil_div(narow, 128), 128, 0, s>>>(B, narow, arow_start, aop);
        LMIEB_CUDA_TRY(cudaGetLastError());
    }
    if (ngroups > 0) {
        k_oz_bop<<<ngroups, OZ_BOP_T, 0, s>>>(B, coef, bop, colexp);
        LMIEB_CUDA_TRY(cudaGetLastError());
    }
    return 0;
}

int launch_angular_oz(cudaStream_t s, const DevBatch &B, int nitems, const AngItem *items, const unsigned char *bop,
                      double *part, int *err) {
    if (nitems <= 0) return 0;
    switch (B.nd1) {
        case 0: return launch_oz<0>(s, B, nitems, items, bop, part, err);
        case 1: return launch_oz<1>(s, B, nitems, items, bop, part, err);
        case 2: return launch_oz<2>(s, B, nitems, items, bop, part, err);
        case 3: return launch_oz<3>(s, B, nitems, items, bop, part, err);
        case 4: return launch_oz<4>(s, B, nitems, items, bop, part, err);
    }
    fprintf(stderr, "ERROR: lmie_b200: int8 angular stage built for at most %d index1 columns\n", OZ_MAX_NC1);
    return -1;
}

int launch_oz_selftest(cudaStream_t s, int K, const double *A, const double *Bm, double *D, int *err,
                       long long wait_cycles, int withhold) {
    static bool attr = false;
    const int smem = (int) (OZ_BSTAGE + 64);
    if (!attr) {
        LMIEB_CUDA_TRY(cudaFuncSetAttribute(k_oz_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        attr = true;
    }
    k_oz_selftest<<<1, 128, smem, s>>>(K, A, Bm, D, err, wait_cycles, withhold);
    LMIEB_CUDA_TRY(cudaGetLastError());
    return 0;
}
