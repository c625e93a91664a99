// k_noalloc.cu -- per-radius cross sections with no device allocation.
//
// Some callers of this library cannot call cudaMalloc: a radiative-transfer
// model embedded in a host application whose memory pool has already claimed
// the whole GPU, or a retrieval loop that must not pay cudaMalloc's implicit
// device-wide synchronisation on every call.  They own their input and output
// buffers and need the Mie work done without the library touching the
// allocator.  lmie_cross_sections_noalloc serves them: it runs the same
// recurrences as the per-radius kernel of the drop-in solve (value only, no
// derivatives), with its scratch -- the psi ratios and the logarithmic
// derivative D_n, order-major across radii -- in a file-scope static device
// array of fixed size instead of library-allocated memory.
//
// Limits: at most NA_MAX_RADII = 1024 radii per call and size parameters
// 0 < x = 2 pi r / lambda <= NA_MAX_X = 900 (so n1(x) < NA_MAX_ORDER = 1024);
// the scratch is 3 * 1024 * 1024 doubles = 24 MiB plus the truncation orders
// of 1024 radii, and every GPU that loads this library holds it until the
// process exits.
//
// The truncation orders n1, n2 of every radius (reference
// src/lmie_core.c:18-38) are computed on the host with the host's libm, as
// everywhere else in this library, and copied into the static array: the
// device's pow may differ from the host's in the last place and move an
// (int) cast across an integer.
#include <cmath>
#include <cstdio>
#include <mutex>

#include "dev_common.cuh"
#include "../../include/lmie_b200.h"

extern "C" int lmieb_calc_n1(double x);
extern "C" int lmieb_calc_n2(int n1, double zr, double zi);

namespace {

constexpr int NA_MAX_RADII = 1024;
constexpr int NA_MAX_ORDER = 1024;
constexpr double NA_MAX_X = 900.;
constexpr int NA_MAX_DEVICES = 64;

// Scratch shared by every call on a device: psi ratios r_j at
// [j * NA_MAX_RADII + i], then D_j (complex) at
// [NA_MAX_ORDER * NA_MAX_RADII + 2 * (j * NA_MAX_RADII + i)].
static __device__ __align__(256) double g_noalloc_scratch[(size_t) 3 * NA_MAX_ORDER * NA_MAX_RADII];
// (n1, n2) of every radius of the call, written by the host before the kernel.
static __device__ __align__(256) int2 g_noalloc_trunc[NA_MAX_RADII];
// Index + 1 of a radius whose size parameter is out of range (0: none).
static __device__ __align__(256) int g_noalloc_error;

struct DeviceSlot {
    bool ready = false;
    double *scratch = nullptr;   // device address of g_noalloc_scratch on this device
    int2 *trunc = nullptr;       // device address of g_noalloc_trunc on this device
    int *error = nullptr;        // device address of g_noalloc_error on this device
};
DeviceSlot g_slots[NA_MAX_DEVICES];
std::mutex g_slots_mu;

__global__ void __launch_bounds__(128) k_cross_sections_static(int n, const double *__restrict__ radius,
                                                               double lambda, cplx m, cplx minv,
                                                               const int2 *__restrict__ trunc,
                                                               double *__restrict__ scr, int *err,
                                                               double *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = 2. * LMIEB_PI * radius[i] / lambda;
    const int2 nn = trunc[i];
    const int n1 = nn.x, n2 = nn.y;
    if (!(x > 0.) || !(x <= NA_MAX_X) || n1 < 1 || n1 >= NA_MAX_ORDER || n2 < n1) {
        // out of range: record it, write NaN, touch no scratch
        atomicMax(err, i + 1);
        const double nan = __longlong_as_double(0x7ff8000000000000LL);
        for (int q = 0; q < 4; ++q) out[(size_t) q * n + i] = nan;
        return;
    }
    const cplx z = mk(m.re * x, m.im * x);
    const double xinv = 1. / x;
    const cplx zinv = 1. / z;
    double *R = scr;
    double2 *Dv = (double2 *) (scr + (size_t) NA_MAX_ORDER * NA_MAX_RADII);

    // D_n(z) downward from D_{n2} = 0, kept for orders 1..n1
    cplx D = mk(0., 0.);
    for (int j = n2 - 1; j >= 1; --j) {
        const cplx c1 = (j + 1.) * zinv;
        D = c1 - 1. / (D + c1);
        if (j <= n1) Dv[(size_t) j * NA_MAX_RADII + i] = make_double2(D.re, D.im);
    }
    // psi_j / psi_{j-1} downward from r_{n1} = 0 (every slot read below is written here)
    double rn = 0.;
    R[(size_t) n1 * NA_MAX_RADII + i] = 0.;
    for (int j = n1 - 1; j >= 1; --j) {
        rn = 1. / ((2. * j + 1.) * xinv - rn);
        R[(size_t) j * NA_MAX_RADII + i] = rn;
    }
    // upward: psi, chi, a_n, b_n and the extinction, scattering, backscatter
    // and asymmetry sums
    double sinx, cosx;
    sincos(x, &sinx, &cosx);
    double psi_p = sinx, chi_p = cosx, chi_c = xinv * cosx + sinx;
    double se = 0., ss = 0., sg = 0., sgn = -1.;
    cplx sb = mk(0., 0.), a_p = mk(0., 0.), b_p = mk(0., 0.);
    for (int j = 1; j <= n1; ++j) {
        const double psi = R[(size_t) j * NA_MAX_RADII + i] * psi_p;
        const double2 dv = Dv[(size_t) j * NA_MAX_RADII + i];
        const cplx Dj = mk(dv.x, dv.y);
        const cplx zeta = mk(psi, chi_c), zeta_p = mk(psi_p, chi_p);
        const double t = j * xinv;
        const cplx ca = Dj * minv + t;
        const cplx a = (ca * psi - psi_p) / (ca * zeta - zeta_p);
        const cplx cb = m * Dj + t;
        const cplx b = (cb * psi - psi_p) / (cb * zeta - zeta_p);
        const double f1 = 2. * j + 1.;
        se += f1 * (a.re + b.re);
        ss += f1 * (norm2(a) + norm2(b));
        sb = sb + (a - b) * (f1 * sgn);
        if (j >= 2) {
            const double jm = j - 1.;
            const double fv2 = (jm + 1.) / jm;
            const double fv3 = (jm + 2.) / fv2, fv4 = (2. * jm + 1.) / (jm * (jm + 1.));
            sg += fv3 * (re_mulc(a_p, a) + re_mulc(b_p, b)) + fv4 * re_mulc(a_p, b_p);
        }
        if (j < n1) {
            const double chi_n = (2. * j + 1.) * xinv * chi_c - chi_p;
            chi_p = chi_c;
            chi_c = chi_n;
        }
        psi_p = psi;
        a_p = a;
        b_p = b;
        sgn = -sgn;
    }
    const double lam2 = lambda * lambda / (2. * LMIEB_PI);
    out[i] = se * lam2;
    out[(size_t) n + i] = ss * lam2;
    out[(size_t) 2 * n + i] = norm2(sb) * lam2 / (2. * 4. * LMIEB_PI);
    out[(size_t) 3 * n + i] = sg / ss * 2.;
}

// Looks up, once per device and with that device current, the device
// addresses of the static scratch and error word.  In host code the symbol
// names are only host-side stand-ins and must not be passed to a kernel.
int device_slot(DeviceSlot **slot) {
    int dev = 0;
    LMIEB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NA_MAX_DEVICES) {
        fprintf(stderr, "ERROR: lmie_cross_sections_noalloc: device %d out of range\n", dev);
        return -1;
    }
    std::lock_guard<std::mutex> lock(g_slots_mu);
    DeviceSlot &s = g_slots[dev];
    if (!s.ready) {
        LMIEB_CUDA_TRY(cudaGetSymbolAddress((void **) &s.scratch, g_noalloc_scratch));
        LMIEB_CUDA_TRY(cudaGetSymbolAddress((void **) &s.trunc, g_noalloc_trunc));
        LMIEB_CUDA_TRY(cudaGetSymbolAddress((void **) &s.error, g_noalloc_error));
        s.ready = true;
    }
    *slot = &s;
    return 0;
}

}  // namespace

extern "C" int lmie_cross_sections_noalloc(int n_radii, const double *radius, double lambda, double mr,
                                           double mi, double *out, void *stream) {
    if (n_radii < 1 || n_radii > NA_MAX_RADII) {
        fprintf(stderr, "ERROR: lmie_cross_sections_noalloc: n_radii = %d, must be in 1..%d\n", n_radii,
                NA_MAX_RADII);
        return -1;
    }
    if (!radius || !out) {
        fprintf(stderr, "ERROR: lmie_cross_sections_noalloc: radius and out must be device pointers\n");
        return -1;
    }
    if (!(lambda > 0.)) {
        fprintf(stderr, "ERROR: lmie_cross_sections_noalloc: lambda = %g must be positive\n", lambda);
        return -1;
    }
    DeviceSlot *slot = nullptr;
    if (device_slot(&slot)) return -1;
    cudaStream_t s = (cudaStream_t) stream;
    const cplx m = mk(mr, -mi);
    // truncation orders on the host (host libm), through arrays on this
    // thread's stack: the radii come down, n1 and n2 go up into the static array
    double rad[NA_MAX_RADII];
    int2 nn[NA_MAX_RADII];
    LMIEB_CUDA_TRY(cudaMemcpyAsync(rad, radius, sizeof(double) * n_radii, cudaMemcpyDeviceToHost, s));
    LMIEB_CUDA_TRY(cudaStreamSynchronize(s));
    for (int i = 0; i < n_radii; ++i) {
        const double x = 2. * LMIEB_PI * rad[i] / lambda;
        nn[i] = make_int2(0, 0);
        if (x > 0. && x <= NA_MAX_X) {
            const int n1 = lmieb_calc_n1(x);
            nn[i] = make_int2(n1, lmieb_calc_n2(n1, mr * x, -mi * x));
        }
    }
    LMIEB_CUDA_TRY(cudaMemcpyAsync(slot->trunc, nn, sizeof(int2) * n_radii, cudaMemcpyHostToDevice, s));
    LMIEB_CUDA_TRY(cudaMemsetAsync(slot->error, 0, sizeof(int), s));
    k_cross_sections_static<<<ceil_div(n_radii, 128), 128, 0, s>>>(n_radii, radius, lambda, m, 1. / m,
                                                                    slot->trunc, slot->scratch, slot->error,
                                                                    out);
    LMIEB_CUDA_TRY(cudaGetLastError());
    int bad = 0;
    LMIEB_CUDA_TRY(cudaMemcpyAsync(&bad, slot->error, sizeof(int), cudaMemcpyDeviceToHost, s));
    LMIEB_CUDA_TRY(cudaStreamSynchronize(s));
    if (bad) {
        fprintf(stderr, "ERROR: lmie_cross_sections_noalloc: radius %d gives a size parameter outside "
                "(0, %g] (lambda = %g)\n", bad - 1, NA_MAX_X, lambda);
        return -1;
    }
    return 0;
}
