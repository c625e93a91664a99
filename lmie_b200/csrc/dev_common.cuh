// dev_common.cuh -- FP64 complex helpers and launch utilities shared by the
// sm_100a kernels of liblmie_b200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#ifndef LMIEB_PI
#define LMIEB_PI 3.14159265358979323846
#endif

struct cplx {
    double re, im;
};

__host__ __device__ __forceinline__ cplx mk(double r, double i) { cplx c; c.re = r; c.im = i; return c; }
__host__ __device__ __forceinline__ cplx operator+(cplx a, cplx b) { return mk(a.re + b.re, a.im + b.im); }
__host__ __device__ __forceinline__ cplx operator-(cplx a, cplx b) { return mk(a.re - b.re, a.im - b.im); }
__host__ __device__ __forceinline__ cplx operator-(cplx a) { return mk(-a.re, -a.im); }
__host__ __device__ __forceinline__ cplx operator*(cplx a, cplx b) {
    return mk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
__host__ __device__ __forceinline__ cplx operator*(cplx a, double s) { return mk(a.re * s, a.im * s); }
__host__ __device__ __forceinline__ cplx operator*(double s, cplx a) { return mk(a.re * s, a.im * s); }
__host__ __device__ __forceinline__ cplx operator+(cplx a, double s) { return mk(a.re + s, a.im); }
__host__ __device__ __forceinline__ cplx operator-(cplx a, double s) { return mk(a.re - s, a.im); }
__host__ __device__ __forceinline__ cplx conjg(cplx a) { return mk(a.re, -a.im); }
__host__ __device__ __forceinline__ double norm2(cplx a) { return a.re * a.re + a.im * a.im; }
// Re(a * conj(b))
__host__ __device__ __forceinline__ double re_mulc(cplx a, cplx b) { return a.re * b.re + a.im * b.im; }
// Im(a * conj(b))
__host__ __device__ __forceinline__ double im_mulc(cplx a, cplx b) { return a.im * b.re - a.re * b.im; }

// Complex division by Smith's method (Smith 1962), scaled by the larger
// component of the divisor so that |b|^2 is never formed.
__host__ __device__ __forceinline__ cplx operator/(cplx a, cplx b) {
    if (fabs(b.re) >= fabs(b.im)) {
        double r = b.im / b.re, d = b.re + b.im * r;
        return mk((a.re + a.im * r) / d, (a.im - a.re * r) / d);
    } else {
        double r = b.re / b.im, d = b.re * r + b.im;
        return mk((a.re * r + a.im) / d, (a.im * r - a.re) / d);
    }
}
__host__ __device__ __forceinline__ cplx operator/(double s, cplx b) { return mk(s, 0.) / b; }
// 1/c = conj(c) / |c|^2 with one real division; for operands whose squared
// modulus stays inside the double range (all Mie recurrence denominators do).
__host__ __device__ __forceinline__ cplx cinv(cplx c) {
    const double d = 1. / (c.re * c.re + c.im * c.im);
    return mk(c.re * d, -c.im * d);
}
__host__ __device__ __forceinline__ cplx operator/(cplx a, double s) { return mk(a.re / s, a.im / s); }

#define LMIEB_CUDA_TRY(expr)                                                              \
    do {                                                                                  \
        cudaError_t e_ = (expr);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            fprintf(stderr, "ERROR: %s:%d: %s: %s\n", __FILE__, __LINE__, #expr,          \
                    cudaGetErrorString(e_));                                              \
            return -1;                                                                    \
        }                                                                                 \
    } while (0)

static inline unsigned int ceil_div(size_t a, size_t b) { return (unsigned int) ((a + b - 1) / b); }

#ifdef __CUDACC__
// case c with start[c] <= e < start[c + 1] (start: ncase + 1 ascending offsets)
static __device__ __forceinline__ int find_case(const long long *__restrict__ start, int ncase, long long e) {
    int lo = 0, hi = ncase - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= e) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}
#endif
