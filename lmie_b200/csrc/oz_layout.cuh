// oz_layout.cuh -- operands of the fixed-point angular contraction on the
// int8 tensor cores (LMIEB_PRECISION_INT8), shared by its operand kernels and
// its product kernel (k_oz.cu) and the driver.
//
// The S1/S2 sums of a case are the dense products of tc_layout.cuh,
//     C[row, n] = sum_k A+[row, k] Bop[k, n],
// rows 2h / 2h+1 = (pi_k + tau_k)(mu_h) / s_k (pi_k - tau_k)(mu_h), columns
// the real and imaginary parts of S = fv4 (a + b) and D' = s_k fv4 (a - b) of
// the radii of a group.  Here every operand value becomes a signed integer of
// 47 fractional bits and the integer products are summed exactly:
//   - order k gets the power of two 2^e_k, e_k = ceil(log2 2k) (constant over
//     each chunk of 32 orders after the first: 6 + the chunk's bit length):
//     A+ is divided by it and Bop multiplied by it (|pi +- tau| grows like k^2
//     at the poles, fv4 (a +- b) falls like 1/k), and each row r and column n gets its own
//     power of two, g_r and f_n, the smallest that bring every value of the
//     row (all orders of its case) or of the column to at most 1/2 in
//     magnitude;
//   - the scaled value x becomes V = round(x 2^47), |V| <= 2^46, written as
//     six balanced base-256 digits d_0 (most significant) .. d_5 in [-128, 128),
//     V = sum_i d_i 2^(8 (5 - i)): one int8 slice per digit;
//   - the product of A digit i and B digit j has the weight 2^(8 (10 - i - j));
//     the 21 products with i + j < 6 are summed by tcgen05.mma kind::i8 into
//     six int32 accumulators, one per diagonal i + j; the dropped products
//     (i + j >= 6) are below 2^-46 of the largest term each;
//   - A and B digits are signed bytes; every int32 sum is exact (below
//     6 * 128 * 128 * 5120 < 2^31 for groups of up to 5120 orders);
//   - C = 2^(g_r + f_n - 14) sum_d 2^(-8 d) ACC_d, formed exactly in int64
//     halves and FP64.
// Each product then carries ~2^-46 of the largest term of its row and column
// (rounding of the two values and the dropped digit products) instead of
// FP64's 2^-53.
//
// The A operand of a chunk of an angle tile is the same for every radius
// group of its case (the row exponent g_r is taken over all the case's
// orders): it is formed once per (case, tile, chunk) into memory, OZ_AROW
// bytes per product row -- slice s at 32 s, order 4 j + u in byte u of its
// 32-bit word j -- kept as 16-byte pieces with the rows of a piece
// consecutive (piece i of row r at 16 (i OZ_M + r)), and the product kernel
// stores it into tensor memory as it is.
//
// Layout of one chunk (OZ_KC orders) of the B operand in memory: OZ_ND
// slices, slice s holding digit s of every row, each slice in the tensor
// cores' K-major, no-swizzle core-matrix layout for 8-bit elements: 8 rows x
// 16 orders (128 bytes) per core matrix, row groups 128 bytes apart, the two
// order groups rows / 8 * 128 bytes apart.  The A operand of a chunk lives in
// tensor memory: row r in lane r, slice s in 8 columns (4 orders per 32-bit
// column, order 4 j + u in byte u of column j).
#pragma once

#include <stdint.h>

constexpr int OZ_KC = 32;                            // orders per chunk (the K of one kind::i8 product)
constexpr int OZ_ND = 6;                             // base-256 digits per value
constexpr int OZ_NPROD = OZ_ND * (OZ_ND + 1) / 2;    // digit products per chunk (i + j < OZ_ND)
constexpr int OZ_NP = 64;                            // operand rows (product N) per radius group
constexpr int OZ_NHALF = OZ_NP / 2;                  // rows of S (then D')
constexpr int OZ_M = 128;                            // product rows: 64 half-angles and their mirrors
constexpr int OZ_HALF = OZ_M / 2;
constexpr uint32_t OZ_ASLICE = OZ_M * OZ_KC;         // bytes of one A slice of a chunk
constexpr uint32_t OZ_BSLICE = OZ_NP * OZ_KC;        // bytes of one B slice of a chunk
constexpr uint32_t OZ_ASTAGE = OZ_ND * OZ_ASLICE;    // one A chunk (all slices)
constexpr uint32_t OZ_BSTAGE = OZ_ND * OZ_BSLICE;    // one B chunk of a group
constexpr uint32_t OZ_LBO_A = (OZ_M / 8) * 128;      // order-group stride of an A slice
constexpr uint32_t OZ_LBO_B = (OZ_NP / 8) * 128;     // order-group stride of a B slice
constexpr int OZ_MAX_NC1 = 4;                        // index1 columns the kernel is built for
constexpr int OZ_MAX_ND2 = 3;                        // index2 slots the kernel is built for
constexpr int OZ_MAX_NK = 160;                       // chunks per group (5120 orders: int32 sums exact)
constexpr int OZ_MIN_N1 = 16;                        // smaller cases keep the FP64 angular stage
constexpr int OZ_AROW = OZ_ND * OZ_KC;               // bytes of one product row of an A chunk (six slices)
constexpr int OZ_ACHUNK = OZ_M * OZ_AROW;            // bytes of one A chunk of an angle tile
constexpr int OZ_FRAC = 47;                          // fractional bits of the fixed-point values
// exponent of the combination's row- and column-independent factor:
// V_A V_B = 2^80 sum_d 2^(-8 d) ACC_d, and oz_value returns 2^16 of that sum
constexpr int OZ_CSHIFT = 80 - 2 * OZ_FRAC - 16;
// Bound on |beta_l(int8) - beta_l(FP64)| / (2l + 1) of the expansion
// coefficients near the truncation threshold (|beta_l| within 1e-9 .. 1e-5 of
// 2l + 1), for a case whose radii reach n1 orders: measured at most 8e-14 up
// to ~1100 orders (the 4096 seeded uneven cases, x <= 1063) and up to 2.6e-12
// beyond (x from 1500 to 5000, 4 to 8000 radii).  The two forms' own rounding
// differs by this much (the FP64 form and the reference differ by as much).
// A case with some |beta_l| within oz_trunc_band (2l + 1) of `accuracy`
// before its truncation point is solved again in FP64.
__host__ __device__ inline double oz_trunc_band(int n1) { return n1 <= 1152 ? 2.5e-13 : 5e-12; }
// 1.5 * 2^52 + 0x808080808080: see oz_digits
constexpr double OZ_MAGIC = 6896688841130112.0;

// radii per group for nd1 index1 columns
__host__ __device__ inline int oz_rg(int nd1) { return OZ_NHALF / (2 * (1 + nd1)); }

// byte offset of (row n, order kk < OZ_KC) inside one slice of `rows` rows
__host__ __device__ inline int oz_idx(int n, int kk, int rows) {
    return (kk >> 4) * (rows / 8) * 128 + (n >> 3) * 128 + (n & 7) * 16 + (kk & 15);
}

// e_c = 6 + bit length of c: the order exponent of every order of chunk c >= 1
// (orders 32 c + 1 .. 32 c + 32: ceil(log2 2k) is constant there)
__host__ __device__ inline int oz_ec(int c) {
#ifdef __CUDA_ARCH__
    return 6 + (32 - __clz(c));
#else
    return 6 + (c ? 32 - __builtin_clz((unsigned) c) : 0);
#endif
}

// e_k = ceil(log2 2k), k >= 1
__host__ __device__ inline int oz_ek(int k) {
#ifdef __CUDA_ARCH__
    return 32 - __clz(2 * k - 1);
#else
    return 32 - __builtin_clz((unsigned) (2 * k - 1));
#endif
}

#ifdef __CUDACC__
// 2^e as a double, -1022 <= e <= 1023
__device__ __forceinline__ double oz_pow2(int e) { return __hiloint2double((1023 + e) << 20, 0); }

// The digits of V = round(x s) for |x s| <= 2^46: t = x s + 1.5 2^52 + B, with
// B = 0x80 in each of the six low bytes, is an integer in [2^52, 2^53) formed
// with one rounding, so the low 48 bits of its significand are V + B exactly
// (0 < V + B < 2^48), and byte i of V + B is digit 5 - i plus 128 (adding 128
// to each balanced digit makes it a plain byte with no carries).  lo gets
// digits 5, 4, 3, 2 (bytes 0..3), hi digits 1, 0 (bytes 0, 1); a byte xor 0x80
// is the digit as a two's-complement int8.
__device__ __forceinline__ void oz_digits(double x, double s, uint32_t &lo, uint32_t &hi) {
    const double t = fma(x, s, OZ_MAGIC);
    lo = (uint32_t) __double2loint(t);
    hi = (uint32_t) __double2hiint(t);
}

// Byte transpose of four words (consecutive orders): b_i = byte i of w0..w3.
__device__ __forceinline__ void oz_t4(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3, uint32_t &b0,
                                      uint32_t &b1, uint32_t &b2, uint32_t &b3) {
    const uint32_t t0 = __byte_perm(w0, w1, 0x5140), t1 = __byte_perm(w2, w3, 0x5140);
    const uint32_t t2 = __byte_perm(w0, w1, 0x7362), t3 = __byte_perm(w2, w3, 0x7362);
    b0 = __byte_perm(t0, t1, 0x5410);
    b1 = __byte_perm(t0, t1, 0x7632);
    b2 = __byte_perm(t2, t3, 0x5410);
    b3 = __byte_perm(t2, t3, 0x7632);
}

// Digit slices of four consecutive orders of one row: w[s] holds digit s of
// the four orders (byte u = order u) as int8.
__device__ __forceinline__ void oz_slices4(const uint32_t (&lo)[4], const uint32_t (&hi)[4], uint32_t (&w)[OZ_ND]) {
    uint32_t d5, d4, d3, d2, d1, d0, x2, x3;
    oz_t4(lo[0], lo[1], lo[2], lo[3], d5, d4, d3, d2);
    oz_t4(hi[0], hi[1], hi[2], hi[3], d1, d0, x2, x3);
    w[0] = d0 ^ 0x80808080u;
    w[1] = d1 ^ 0x80808080u;
    w[2] = d2 ^ 0x80808080u;
    w[3] = d3 ^ 0x80808080u;
    w[4] = d4 ^ 0x80808080u;
    w[5] = d5 ^ 0x80808080u;
}

// One step of the pi/tau recurrence at order k (reference
// src/lmie_core.c:658-721): with p0 = pi_{k-1}, p1 = pi_k, kmu = k mu, k1 = k + 1
// and f2 = (k + 1) / k, tau = tau_k; then everything advances to k + 1.  The
// product rows are p1 + tau (row 2h) and s_k (p1 - tau) (its mirror).
__device__ __forceinline__ void oz_step(double mu, double f2, double &kmu, double &k1, double &p0, double &p1,
                                        double &tau) {
    tau = fma(kmu, p1, -k1 * p0);
    const double pn = fma((1. + f2) * mu, p1, -f2 * p0);
    p0 = p1;
    p1 = pn;
    kmu += mu;
    k1 += 1.;
}

// smallest g with m <= 2^(g - 1) (m > 0): one bit of headroom; 0 for m = 0
__device__ __forceinline__ int oz_exp_of(double m) { return m > 0. ? ilogb(m) + 2 : 0; }
#endif
