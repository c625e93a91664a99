// tc_layout.cuh -- operand layout of the split-precision (3xTF32) angular
// contraction on the tensor cores, shared by its producer (K1, k_fp64.cu)
// and its consumer (k_tc.cu).
//
// Per case the S1/S2 sums are dense products over the orders k:
//     sp[row, n] = sum_k A+[row, k] S[k, n],   sm[row, n] = sum_k A-[row, k] D[k, n]
// with A+- = pi_k +- tau_k at the Gauss angles and S, D = fv4_k (a_k +- b_k)
// of radius/column n split into real and imaginary parts.  Rows come in pairs
// 2h (half-angle mu_h) and 2h+1 (its mirror -mu_h).  The mirror identities
// (pi +- tau)(-mu) = s_k (pi -+ tau)(mu), s_k = (-1)^(k+1), give
// A-[r, k] = s_k A+[r ^ 1, k], so sm[r, n] = (A+ D')[r ^ 1, n] with
// D'[k, n] = s_k D[k, n]: one product A+ [S | D'] yields both sums.  Each
// operand is split into two TF32 terms (hi + lo), and the product is formed
// as lo*hi + hi*lo + hi*hi with FP32 accumulation in tensor memory.
//
// Radii are cut into groups of TC_RG(nd1) consecutive radii of one case; a
// group owns TC_NP = 128 operand rows: row n = (pos * (1 + nd1) + col) * 2 +
// {re, im} of S, and row TC_NHALF + n of D' (col 0: value, col 1 + k: index1
// derivative k), unused rows zero.  Its orders are cut into chunks of TC_KC;
// chunk kc of a group is one contiguous block of two parts [hi | lo], each
// TC_NP x TC_KC FP32 values in the tensor cores' K-major, no-swizzle
// core-matrix layout: 8 rows x 4 orders (128 bytes) per core matrix, row
// groups 128 bytes apart, order groups TC_NP / 8 * 128 bytes apart.
#pragma once

#include <stdint.h>

constexpr int TC_KC = 16;                           // orders per chunk (pipeline stage)
constexpr int TC_NP = 128;                          // operand rows (product N) per radius group
constexpr int TC_NHALF = TC_NP / 2;                 // rows of S (then D')
constexpr int TC_M = 128;                           // product rows: 64 half-angles and their mirrors
constexpr int TC_HALF = TC_M / 2;
constexpr uint32_t TC_APART = TC_M * TC_KC * 4;     // bytes of one A part per chunk
constexpr uint32_t TC_BPART = TC_NP * TC_KC * 4;    // bytes of one B part per chunk
constexpr uint32_t TC_ASTAGE = 2 * TC_APART;        // [hi | lo]
constexpr uint32_t TC_BSTAGE = 2 * TC_BPART;        // bytes of one chunk of a group
constexpr uint32_t TC_LBO_A = (TC_M / 8) * 128;     // order-group stride of A
constexpr uint32_t TC_LBO_B = (TC_NP / 8) * 128;    // order-group stride of B
constexpr int TC_MAX_NC1 = 4;                       // index1 columns the kernel is built for
constexpr int TC_MAX_ND2 = 3;                       // index2 slots the kernel is built for (accumulators in registers)
// cases of fewer orders keep the FP64 angular stage in split-precision batches
constexpr int TC_MIN_N1 = 16;

// radii per group for nd1 index1 columns
__host__ __device__ inline int tc_rg(int nd1) { return TC_NHALF / (2 * (1 + nd1)); }

// float index of (row n, order kk < TC_KC) inside one part of a chunk
__host__ __device__ inline int tc_idx(int n, int kk, int rows) {
    return (kk >> 2) * (rows / 8) * 32 + (n >> 3) * 32 + (n & 7) * 4 + (kk & 3);
}

#ifdef __CUDACC__
// Round a finite FP32 value to TF32 (nearest, ties away from zero) as an
// FP32 bit pattern: add half a unit of the 13 dropped bits to the magnitude
// and clear them (integer ALU work; a carry moves into the exponent as
// rounding up to the next binade does).
__device__ __forceinline__ float tc_tf32(float x) {
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

// v ~ hi + lo with hi, lo TF32 (about 22 significant bits)
__device__ __forceinline__ void tc_split(double v, float &hi, float &lo) {
    const float f = __double2float_rn(v);
    const float h = tc_tf32(f);
    hi = h;
    lo = tc_tf32(f - h);
}

#endif
