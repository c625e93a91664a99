// driver.cu -- device side of one drop-in solve: owns the CUDA context state
// (stream, device arena, pinned staging), uploads a prepared problem, runs
// the kernel sequence and returns the results.  Replaces the reference's
// lmie_core_shared / lmie_core_sequential / lmie_core_xthreads fan-out
// (src/lmie_schedule.c:154-452) and the driver half of lmie_core_solution
// (src/lmie_schedule.c:942-1268).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "kernels.h"
#include "lmieb.h"
#include "../../include/lmie_b200.h"

namespace {

constexpr int NSTAGE = LMIEB_N_STAGES;
constexpr size_t TABLE_LIMIT = (size_t) 256 << 20;     // expansion basis table per order chunk
constexpr size_t FLUSH_BYTES = (size_t) 256 << 20;     // > 126 MB L2

// Every staged array starts on a 256-byte boundary and takes at least one
// 256-byte block, so empty arrays never alias their neighbours.
inline size_t pad(size_t bytes) { return ((bytes ? bytes : 1) + 255) & ~(size_t) 255; }

struct Ctx {
    bool ready = false;
    int device = -1;
    int sms = 0;
    cudaStream_t stream = nullptr;
    char *dbuf = nullptr;
    size_t dcap = 0;
    char *hbuf = nullptr;
    size_t hcap = 0;
    char *flush = nullptr;
    cudaEvent_t ev[NSTAGE + 1] = {};
    bool timing = false;
    double stage_ms[NSTAGE] = {};
    long long launches = 0;         // kernel launches of the last run_kernels
    double work[4] = {};            // algorithmic flops of the last solve (see lmieb_last_work)
    size_t h2d = 0, d2h = 0;        // bytes copied by the last solve
    // state of the last solve, for re-running the device part in place
    bool have_plan = false;
    struct Plan *plan = nullptr;
    // Gauss-Legendre angles depend only on their number: computed once per n
    // and kept on the device (oldest entry evicted beyond GL_CACHE entries)
    struct GlEntry { int n; double *mu; double *wq; };
    std::vector<GlEntry> gl_cache;
};

constexpr size_t GL_CACHE = 32;

Ctx g_ctx;
std::mutex g_mu;

struct Arena {
    char *base;
    size_t used = 0, cap;
    template <class T>
    T *take(size_t count) {
        size_t bytes = pad(count * sizeof(T));
        if (used + bytes > cap) return nullptr;
        T *p = (T *) (base + used);
        used += bytes;
        return p;
    }
};

// Everything the kernel sequence needs, in device memory.
struct Plan {
    DevProblem P;
    int nd1c = 0;               // number of index1 chunks for K1
    int n_ang_launch = 0;       // launches of K3
    int G = 0;                  // radius groups of K3
    int2 *tiles = nullptr;      // K1b (radius, first order) per block
    int *tstart = nullptr;      // [n+1] first tile of each radius
    int lchunk = 0;
    int want_gc = 0, want_lc = 0, pf_from = 0;
    double accuracy = 0.;
    int save_control = 0;
    int *gstart = nullptr;
    double4 *rec = nullptr;
    double *rsp = nullptr, *coef = nullptr, *rs = nullptr;
    double *sums = nullptr, *part = nullptr, *pfacc = nullptr, *pfn = nullptr;
    double *state = nullptr, *tab = nullptr, *raw = nullptr;
    double *mu_user = nullptr;
    double *save1_in = nullptr, *save2_in = nullptr, *w2 = nullptr;
    // output region (one D2H copy)
    double *o_scal = nullptr, *o_gc = nullptr, *o_lc = nullptr, *o_pf = nullptr;
    int *o_trunc = nullptr;     // [2]: gc, lc
    double *o_save1 = nullptr, *o_save2 = nullptr;
    char *out_begin = nullptr;
    size_t out_bytes = 0;
    long long launches = 0;     // kernel launches one run_kernels issues
};

int g_want_device = -1;

int ensure_ready() {
    Ctx &c = g_ctx;
    if (c.ready) return 0;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        fprintf(stderr, "ERROR: lmie_b200: no CUDA device available (%s); this library has no CPU "
                "fallback\n", e != cudaSuccess ? cudaGetErrorString(e) : "0 devices");
        return -1;
    }
    if (g_want_device >= 0) {
        if (g_want_device >= count) {
            fprintf(stderr, "ERROR: lmie_b200: device %d requested, %d present\n", g_want_device, count);
            return -1;
        }
        LMIEB_CUDA_TRY(cudaSetDevice(g_want_device));
    }
    LMIEB_CUDA_TRY(cudaGetDevice(&c.device));
    cudaDeviceProp prop;
    LMIEB_CUDA_TRY(cudaGetDeviceProperties(&prop, c.device));
    if (prop.major != 10) {
        fprintf(stderr, "ERROR: lmie_b200: device %d (%s, sm_%d%d) is not an sm_100 (B200) GPU\n",
                c.device, prop.name, prop.major, prop.minor);
        return -1;
    }
    c.sms = prop.multiProcessorCount;
    LMIEB_CUDA_TRY(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    for (int i = 0; i <= NSTAGE; ++i) LMIEB_CUDA_TRY(cudaEventCreate(&c.ev[i]));
    c.plan = new Plan();
    c.ready = true;
    return 0;
}

int ensure_device(size_t bytes) {
    Ctx &c = g_ctx;
    if (bytes <= c.dcap) return 0;
    if (c.dbuf) LMIEB_CUDA_TRY(cudaFree(c.dbuf));
    c.dbuf = nullptr;
    c.dcap = 0;
    size_t want = bytes + bytes / 4;
    LMIEB_CUDA_TRY(cudaMalloc((void **) &c.dbuf, want));
    c.dcap = want;
    c.have_plan = false;
    return 0;
}

int ensure_host(size_t bytes) {
    Ctx &c = g_ctx;
    if (bytes <= c.hcap) return 0;
    if (c.hbuf) LMIEB_CUDA_TRY(cudaFreeHost(c.hbuf));
    c.hbuf = nullptr;
    c.hcap = 0;
    size_t want = bytes + bytes / 4;
    LMIEB_CUDA_TRY(cudaMallocHost((void **) &c.hbuf, want));
    c.hcap = want;
    return 0;
}

inline void stage(int i) {
    if (g_ctx.timing) cudaEventRecord(g_ctx.ev[i], g_ctx.stream);
}

// The kernel sequence of one solve on resident inputs (stages 1..8).
int run_kernels(Plan &L) {
    Ctx &c = g_ctx;
    cudaStream_t s = c.stream;
    const DevProblem &P = L.P;
    c.launches = L.launches;
    stage(1);
    if (L.save_control != 2) {
        // K1: recurrences + coefficients, per chunk of up to 4 index1 columns
        for (int ch = 0; ch < (L.nd1c > 0 ? L.nd1c : 1); ++ch) {
            int c0 = ch * 4;
            int nc = P.nd1 - c0 < 4 ? P.nd1 - c0 : 4;
            if (nc < 0) nc = 0;
            if (launch_coef(s, P, nc, c0, ch == 0, L.tiles, L.rec, L.coef, L.rsp)) return -1;
        }
        if (launch_tile_reduce(s, P, L.tstart, L.rsp, L.rs)) return -1;
        stage(2);
        if (launch_reduce_scalars(s, P, L.rs, L.sums, L.save_control == 1 ? L.o_save1 : nullptr)) return -1;
        stage(3);
        if (P.n_qang > 0) {
            for (int t = 0; t < L.n_ang_launch; ++t) {
                int c1 = t * 4, c2 = t * 4;
                int nc1 = P.nd1 - c1 < 4 ? P.nd1 - c1 : 4;
                int nc2 = P.nd2 - c2 < 4 ? P.nd2 - c2 : 4;
                if (nc1 < 0) nc1 = 0;
                if (nc2 < 0) nc2 = 0;
                if (launch_angular(s, P, nc1, c1, nc2, c2, t == 0, L.G, L.gstart, L.coef, L.part,
                                   L.save_control == 1 ? L.o_save2 : nullptr))
                    return -1;
            }
            if (launch_reduce_pf(s, P, L.G, L.part, L.pfacc)) return -1;
        }
    } else {
        stage(2);
        if (launch_save_reweight(s, P, L.save1_in, L.save2_in, L.w2, L.sums, L.pfacc)) return -1;
        stage(3);
    }
    stage(4);
    if (launch_normalize(s, P, L.sums, L.pfacc, L.o_scal, L.pfn)) return -1;
    stage(5);
    if (L.want_gc && launch_expand(s, P, 0, L.lchunk, L.accuracy, L.pfn, L.state, L.tab, L.raw, L.o_gc,
                                   L.o_trunc))
        return -1;
    stage(6);
    if (L.want_lc && launch_expand(s, P, 1, L.lchunk, L.accuracy, L.pfn, L.state, L.tab, L.raw, L.o_lc,
                                   L.o_trunc + 1))
        return -1;
    stage(7);
    if (L.pf_from) {
        const int *tr = L.want_lc ? L.o_trunc + 1 : L.o_trunc;
        const double *cf = L.pf_from == 1 ? L.o_gc : L.o_lc;
        if (launch_phase_user(s, P, L.pf_from == 1 ? 0 : 1, cf, tr, L.mu_user, L.o_pf)) return -1;
    }
    stage(8);
    return 0;
}

template <class T>
T *put(char *&hp, size_t &off, const T *src, size_t count) {
    T *at = (T *) (hp + off);
    if (src && count) memcpy(at, src, count * sizeof(T));
    off += pad(count * sizeof(T));
    return at;
}

}  // namespace

extern "C" int lmieb_device_solve(const lmieb_problem *p, lmieb_result *res) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (ensure_ready()) return -1;
    Ctx &c = g_ctx;
    Plan &L = *c.plan;
    L = Plan();

    const int n = p->n, nd = p->nd, nd1 = p->nd1, nd2 = p->nd2;
    const int ncol = 1 + nd;
    const int n_qang = p->n_qang, nh = n_qang / 2, n_coef = p->n_coef;
    const int na = p->n_angles;

    // ---- host-side plan: offsets, order tables, radius groups ----
    std::vector<long long> off(n + 1);
    off[0] = 0;
    int n1max = 0;
    for (int r = 0; r < n; ++r) {
        off[r + 1] = off[r] + p->n1r[r];
        if (p->n1r[r] > n1max) n1max = p->n1r[r];
    }
    const long long tot = off[n];
    const int n1 = p->n1;
    std::vector<long long> offp(n + 1);
    std::vector<int> tstart(n + 1);
    std::vector<int2> tiles;
    offp[0] = 0;
    for (int r = 0; r < n; ++r) {
        offp[r + 1] = offp[r] + p->n1r[r] + 1;
        tstart[r] = (int) tiles.size();
        for (int j0 = 1; j0 <= p->n1r[r]; j0 += 127) tiles.push_back(make_int2(r, j0));
    }
    tstart[n] = (int) tiles.size();
    const long long totp = offp[n];
    const int ntiles = (int) tiles.size();
    std::vector<double> fv((size_t) 4 * (n1 + 2), 0.);
    for (int i = 1; i <= n1 + 1; ++i) {
        double f1 = 2. * i + 1., f2 = (i + 1.) / i;
        fv[i] = f1;
        fv[(size_t) (n1 + 2) + i] = f2;
        fv[(size_t) 2 * (n1 + 2) + i] = (i + 2.) / f2;
        fv[(size_t) 3 * (n1 + 2) + i] = f1 / (i * (i + 1.));
    }
    fv[0] = 1.;
    // radius groups of roughly equal work for K3
    int G = 1;
    std::vector<int> gstart;
    if (n_qang > 0) {
        const int per = angular_angles_per_block(nd1 < 4 ? nd1 : 4);
        int tiles = (nh + per - 1) / per;
        // one full wave at the kernel's occupancy (4 blocks per SM)
        int target = 4 * c.sms;
        G = (target + tiles - 1) / tiles;
        if (G > n) G = n;
        if (G < 1) G = 1;
        gstart.resize(G + 1);
        gstart[0] = 0;
        int gi = 1;
        for (int r = 0; r < n && gi < G; ++r) {
            if ((double) off[r + 1] * G >= (double) tot * gi) gstart[gi++] = r + 1;
        }
        while (gi < G) gstart[gi++] = n;
        gstart[G] = n;
        // keep the groups strictly increasing
        for (int i = 1; i <= G; ++i)
            if (gstart[i] < gstart[i - 1]) gstart[i] = gstart[i - 1];
    } else {
        gstart.assign(2, 0);
        gstart[1] = n;
    }
    // Newton starting points of the Gauss angles (host libm, as the reference)
    std::vector<double> guess(n_qang > 0 ? (n_qang + 1) / 2 : 1, 0.);
    if (n_qang > 0) {
        const int ia = 4 * n_qang + 2;
        const double da = (n_qang - 1) / (8. * pow((double) n_qang, 3));
        for (int i = 0; i < (n_qang + 1) / 2; ++i) {
            double th = (4. * i + 3.) / ia * LMIEB_PI;
            guess[i] = cos(th + da / tan(th));
        }
    }
    std::vector<double> gl_jr(n_qang > 0 ? n_qang : 1, 0.);
    for (int j = 0; j < n_qang; ++j) gl_jr[j] = j / (j + 1.);
    // GSF / Legendre recurrence coefficients per order l (j = l - 1)
    std::vector<double> rc((size_t) 8 * (n_coef > 0 ? n_coef : 1), 0.);
    for (int l = 3; l < n_coef; ++l) {
        const int j = l - 1;
        const double jj = (double) j * j, jp1 = j + 1., jjp1 = j * jp1, jp1s = jp1 * jp1, tj1 = 2 * j + 1;
        const double a02 = sqrt(jj - 4), b02 = sqrt(jp1s - 4);
        const double a22 = tj1 * 4, b22 = jp1 * (jj - 4), c22 = j * (jp1s - 4);
        double *q = &rc[(size_t) 8 * l];
        q[0] = tj1 / jp1;
        q[1] = j / jp1;
        q[2] = tj1 / b02;
        q[3] = a02 / b02;
        q[4] = tj1 * jjp1 / c22;
        q[5] = a22 / c22;
        q[6] = b22 / c22;
    }
    for (int l = 2; l < 3 && l < n_coef; ++l) rc[(size_t) 8 * l + 1] = 1. / 2.;   // Legendre at l = 2
    std::vector<cplx> ml(nd > 0 ? nd : 1);
    for (int k = 0; k < nd; ++k) ml[k] = mk(p->mr_l[k], -p->mi_l[k]);

    L.nd1c = (nd1 + 3) / 4;
    L.n_ang_launch = (nd1 > nd2 ? (nd1 + 3) / 4 : (nd2 + 3) / 4);
    if (L.n_ang_launch < 1) L.n_ang_launch = 1;
    L.G = G;
    (void) n1max;
    if (nh > 0) {
        size_t lc = TABLE_LIMIT / ((size_t) 4 * nh * 8);
        if (lc < 32) lc = 32;
        L.lchunk = (int) (lc < (size_t) n_coef ? lc : (size_t) n_coef);
    }
    L.want_gc = p->want_gc && n_qang > 0;
    L.want_lc = p->want_lc && n_qang > 0;
    L.pf_from = na > 0 ? p->pf_from : 0;
    L.accuracy = p->accuracy;
    L.save_control = p->save_control;

    // ---- launches per run and algorithmic work (flops) of this solve ----
    {
        long long nl = 0;
        const long long lchunks = nh > 0 ? (n_coef + L.lchunk - 1) / L.lchunk : 0;
        if (p->save_control != 2) {
            nl += (long long) (L.nd1c > 0 ? L.nd1c : 1) * 2 + 1;      // K1a + K1b per chunk, tile sums
            nl += 1;                                                  // K2
            if (n_qang > 0) nl += L.n_ang_launch + 1;                 // K3 + group reduction
        } else {
            nl += 1 + (n_qang > 0);
        }
        nl += 1;                                                      // normalisation
        if (L.want_gc) nl += 2 * lchunks + 1;
        if (L.want_lc) nl += 2 * lchunks + 1;
        if (L.pf_from) nl += 1;
        L.launches = nl;
        // Algorithmic flop counts (fixed per-order constants counted from the
        // FP64 kernels): angular S1/S2 contraction 8 flops per (angle, order,
        // radius, column); recurrences 14 per D_n order + 93 per a_n/b_n order
        // for the value and 16 + 154 for each tangent-linear column;
        // expansion 12 per (order, angle, column); user angles 12 per
        // (order, angle, column).
        double fang = 0., frec = 0.;
        for (int r = 0; r < n; ++r) {
            fang += 8. * n_qang * p->n1r[r] * (1. + nd1);
            frec += (14. * p->n2r[r] + 93. * p->n1r[r]) + nd1 * (16. * p->n2r[r] + 154. * p->n1r[r]);
        }
        if (p->save_control == 2) fang = frec = 0.;
        double fgsf = 12. * n_coef * n_qang * ncol * ((L.want_gc ? 1 : 0) + (L.want_lc ? 1 : 0));
        double fexp = L.pf_from ? 12. * na * n_coef * ncol : 0.;
        c.work[0] = fang;
        c.work[1] = frec;
        c.work[2] = fgsf;
        c.work[3] = fexp;
    }

    // ---- host staging: inputs then outputs ----
    const size_t n_save2 = (size_t) 4 * n * (n_qang > 0 ? n_qang : 1);
    size_t in_bytes = 0;
    {
        auto add = [&](size_t b) { in_bytes += pad(b); };
        add(n * 8); add((size_t) nd1 * n * 8); add((size_t) ncol * n * 8); add(n * 4); add(n * 4);
        add((size_t) (n + 1) * 8); add((size_t) (n + 1) * 8); add((size_t) (n + 1) * 4);
        add(tiles.size() * 8); add(fv.size() * 8); add(ml.size() * 16); add((nd > 0 ? nd : 1) * 8);
        add((nd1 > 0 ? nd1 : 1) * 4); add((nd2 > 0 ? nd2 : 1) * 4); add((na > 0 ? na : 1) * 8);
        add(gstart.size() * 4);
        add(guess.size() * 8);
        add(gl_jr.size() * 8);
        add(rc.size() * 8);
        if (p->save_control == 2) { add((size_t) 4 * n * 8); add(n_save2 * 8); add((size_t) (nd > 0 ? nd : 1) * n * 8); }
    }
    size_t out_bytes = 0;
    {
        auto add = [&](size_t b) { out_bytes += pad(b); };
        add((size_t) ncol * 4 * 8);
        if (L.want_gc) add((size_t) ncol * 6 * n_coef * 8);
        if (L.want_lc) add((size_t) ncol * 6 * n_coef * 8);
        if (L.pf_from) add((size_t) ncol * 6 * na * 8);
        add(2 * 4);
        if (p->save_control == 1) { add((size_t) 4 * n * 8); add(n_save2 * 8); }
    }
    if (ensure_host(in_bytes + out_bytes)) return -1;
    char *hp = c.hbuf;
    size_t ho = 0;
    double *h_x = put(hp, ho, p->x, n);
    double *h_xl = put(hp, ho, p->xl, (size_t) nd1 * n);
    double *h_w = put(hp, ho, p->w, (size_t) ncol * n);
    int *h_n1r = put(hp, ho, p->n1r, n);
    int *h_n2r = put(hp, ho, p->n2r, n);
    long long *h_off = put(hp, ho, off.data(), n + 1);
    long long *h_offp = put(hp, ho, offp.data(), n + 1);
    int *h_tstart = put(hp, ho, tstart.data(), n + 1);
    int2 *h_tiles = put(hp, ho, tiles.data(), tiles.size());
    double *h_fv = put(hp, ho, fv.data(), fv.size());
    cplx *h_ml = put(hp, ho, ml.data(), ml.size());
    double *h_laml = put(hp, ho, p->lambda_l, nd);
    int *h_i1 = put(hp, ho, p->idx1, nd1);
    int *h_i2 = put(hp, ho, p->idx2, nd2);
    double *h_mu = put(hp, ho, p->mu_user, na);
    int *h_gs = put(hp, ho, gstart.data(), gstart.size());
    double *h_guess = put(hp, ho, guess.data(), guess.size());
    double *h_jr = put(hp, ho, gl_jr.data(), gl_jr.size());
    double *h_rc = put(hp, ho, rc.data(), rc.size());
    double *h_s1 = nullptr, *h_s2 = nullptr, *h_w2 = nullptr;
    if (p->save_control == 2) {
        h_s1 = put(hp, ho, p->save1_in, (size_t) 4 * n);
        h_s2 = put(hp, ho, p->save2_in, n_save2);
        h_w2 = put(hp, ho, p->w2, (size_t) (nd > 0 ? nd : 1) * n);
    }
    const size_t h_in_end = ho;
    char *h_out = hp + h_in_end;

    // ---- device arena ----
    const size_t Q = (size_t) 4 * ncol;
    size_t dev_bytes = in_bytes + out_bytes + 64 * 256;
    {
        auto add = [&](size_t b) { dev_bytes += pad(b); };
        if (p->save_control != 2) {
            add((size_t) (1 + nd1) * (size_t) totp * 32);
            add((size_t) (1 + nd1) * 5 * (size_t) ntiles * 8);
            add((size_t) (1 + nd1) * (size_t) tot * 32);
            add((size_t) (1 + nd1) * 5 * n * 8);
            add((size_t) G * Q * (n_qang > 0 ? n_qang : 1) * 8);
        }
        add((size_t) ncol * 4 * 8);
        add(Q * (n_qang > 0 ? n_qang : 1) * 8 * 2);
        if (L.want_gc || L.want_lc) {
            add((size_t) 8 * nh * 8);
            add((size_t) 4 * L.lchunk * nh * 8);
            add((size_t) ncol * 6 * n_coef * 8);
        }
    }
    if (ensure_device(dev_bytes)) return -1;
    Arena A{c.dbuf, 0, c.dcap};
    // inputs mirror the host staging layout exactly: one H2D copy
    char *d_in = A.take<char>(h_in_end);
    auto dptr = [&](void *h) { return d_in + ((char *) h - hp); };
    char *d_out = A.take<char>(out_bytes);
    if (!d_in || !d_out) {
        fprintf(stderr, "ERROR: lmie_b200: device arena too small\n");
        return -1;
    }

    DevProblem &P = L.P;
    P.n = n; P.nd = nd; P.nd1 = nd1; P.nd2 = nd2;
    P.n1 = n1; P.n_qang = n_qang; P.nh = nh; P.n_coef = n_coef;
    P.n_angles = L.pf_from ? na : 0;
    P.save_control = p->save_control;
    P.lambda = p->lambda;
    P.m = mk(p->mr, -p->mi);
    P.minv = 1. / P.m;
    P.m2 = P.m * P.m;
    P.m_l = (const cplx *) dptr(h_ml);
    P.lambda_l = (const double *) dptr(h_laml);
    P.idx1 = (const int *) dptr(h_i1);
    P.idx2 = (const int *) dptr(h_i2);
    P.x = (const double *) dptr(h_x);
    P.xl = (const double *) dptr(h_xl);
    P.w = (const double *) dptr(h_w);
    P.n1r = (const int *) dptr(h_n1r);
    P.n2r = (const int *) dptr(h_n2r);
    P.off = (const long long *) dptr(h_off);
    P.tot = tot;
    P.offp = (const long long *) dptr(h_offp);
    P.totp = totp;
    P.ntiles = ntiles;
    L.tiles = (int2 *) dptr(h_tiles);
    L.tstart = (int *) dptr(h_tstart);
    P.fv = (const double *) dptr(h_fv);
    L.gstart = (int *) dptr(h_gs);
    P.gl_guess = (const double *) dptr(h_guess);
    P.gl_jr = (const double *) dptr(h_jr);
    P.rc = (const double *) dptr(h_rc);
    L.mu_user = (double *) dptr(h_mu);
    if (p->save_control == 2) {
        L.save1_in = (double *) dptr(h_s1);
        L.save2_in = (double *) dptr(h_s2);
        L.w2 = (double *) dptr(h_w2);
    }
    bool gl_new = false;
    P.mu = P.wq = nullptr;
    if (n_qang > 0) {
        for (auto &e : c.gl_cache)
            if (e.n == n_qang) { P.mu = e.mu; P.wq = e.wq; }
        if (!P.mu) {
            if (c.gl_cache.size() >= GL_CACHE) {
                LMIEB_CUDA_TRY(cudaFree(c.gl_cache.front().mu));
                c.gl_cache.erase(c.gl_cache.begin());
            }
            Ctx::GlEntry e{n_qang, nullptr, nullptr};
            LMIEB_CUDA_TRY(cudaMalloc((void **) &e.mu, sizeof(double) * 2 * (size_t) n_qang));
            e.wq = e.mu + n_qang;
            c.gl_cache.push_back(e);
            P.mu = e.mu;
            P.wq = e.wq;
            gl_new = true;
        }
    }
    if (p->save_control != 2) {
        L.rec = A.take<double4>((size_t) (1 + nd1) * (size_t) totp);
        L.rsp = A.take<double>((size_t) (1 + nd1) * 5 * (size_t) ntiles);
        L.coef = A.take<double>((size_t) (1 + nd1) * (size_t) tot * 4);
        L.rs = A.take<double>((size_t) (1 + nd1) * 5 * n);
        L.part = A.take<double>((size_t) G * Q * (n_qang > 0 ? n_qang : 1));
    }
    L.sums = A.take<double>((size_t) ncol * 4);
    L.pfacc = A.take<double>(Q * (n_qang > 0 ? n_qang : 1));
    L.pfn = A.take<double>(Q * (n_qang > 0 ? n_qang : 1));
    if (L.want_gc || L.want_lc) {
        L.state = A.take<double>((size_t) 8 * nh);
        L.tab = A.take<double>((size_t) 4 * L.lchunk * nh);
        L.raw = A.take<double>((size_t) ncol * 6 * n_coef);
    }
    // output region
    {
        char *o = d_out;
        auto take = [&](size_t bytes) { char *r = o; o += pad(bytes); return r; };
        L.o_scal = (double *) take((size_t) ncol * 4 * 8);
        if (L.want_gc) L.o_gc = (double *) take((size_t) ncol * 6 * n_coef * 8);
        if (L.want_lc) L.o_lc = (double *) take((size_t) ncol * 6 * n_coef * 8);
        if (L.pf_from) L.o_pf = (double *) take((size_t) ncol * 6 * na * 8);
        L.o_trunc = (int *) take(2 * 4);
        if (p->save_control == 1) {
            L.o_save1 = (double *) take((size_t) 4 * n * 8);
            L.o_save2 = (double *) take(n_save2 * 8);
        }
        L.out_begin = d_out;
        L.out_bytes = out_bytes;
    }
    if (!L.sums || !L.pfn || (p->save_control != 2 && !L.part) || ((L.want_gc || L.want_lc) && !L.raw)) {
        fprintf(stderr, "ERROR: lmie_b200: device arena too small\n");
        return -1;
    }

    c.h2d = h_in_end;
    c.d2h = out_bytes;

    // ---- run ----
    cudaStream_t s = c.stream;
    stage(0);
    LMIEB_CUDA_TRY(cudaMemcpyAsync(d_in, hp, h_in_end, cudaMemcpyHostToDevice, s));
    LMIEB_CUDA_TRY(cudaMemsetAsync(d_out, 0, out_bytes, s));
    if (gl_new && launch_gauss(s, n_qang, P.gl_guess, P.gl_jr, (double *) P.mu, (double *) P.wq)) return -1;
    if (run_kernels(L)) return -1;
    LMIEB_CUDA_TRY(cudaMemcpyAsync(h_out, d_out, out_bytes, cudaMemcpyDeviceToHost, s));
    stage(9 < NSTAGE ? 9 : NSTAGE);
    LMIEB_CUDA_TRY(cudaStreamSynchronize(s));
    LMIEB_CUDA_TRY(cudaGetLastError());
    if (c.timing) {
        for (int i = 0; i < NSTAGE; ++i) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, c.ev[i], c.ev[i + 1]) != cudaSuccess) ms = 0.f;
            c.stage_ms[i] = ms;
        }
    }
    c.have_plan = true;

    // ---- unpack ----
    auto hostp = [&](void *d) { return h_out + ((char *) d - d_out); };
    memcpy(res->scal, hostp(L.o_scal), (size_t) ncol * 4 * 8);
    if (L.want_gc && res->gc) memcpy(res->gc, hostp(L.o_gc), (size_t) ncol * 6 * n_coef * 8);
    if (L.want_lc && res->lc) memcpy(res->lc, hostp(L.o_lc), (size_t) ncol * 6 * n_coef * 8);
    if (L.pf_from && res->pf) memcpy(res->pf, hostp(L.o_pf), (size_t) ncol * 6 * na * 8);
    {
        const int *tr = (const int *) hostp(L.o_trunc);
        int t = L.want_lc ? tr[1] : (L.want_gc ? tr[0] : 0);
        res->n_coef_out = (L.want_gc || L.want_lc) ? (t > 0 ? n_coef - t + 1 : n_coef) : 0;
    }
    if (p->save_control == 1) {
        if (res->save1) memcpy(res->save1, hostp(L.o_save1), (size_t) 4 * n * 8);
        if (res->save2 && n_qang > 0) memcpy(res->save2, hostp(L.o_save2), n_save2 * 8);
    }
    return 0;
}

// ---------------------------------------------------------------------------
// B200 extensions (include/lmie_b200.h)
// ---------------------------------------------------------------------------
extern "C" int lmieb_set_device(int device) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (g_ctx.ready && device != g_ctx.device) {
        fprintf(stderr, "ERROR: lmieb_set_device: the library already runs on device %d\n", g_ctx.device);
        return -1;
    }
    g_want_device = device;
    return 0;
}

extern "C" int lmieb_set_timing(int on) {
    std::lock_guard<std::mutex> lock(g_mu);
    g_ctx.timing = on != 0;
    return 0;
}

extern "C" int lmieb_last_timing(double *ms, int n) {
    std::lock_guard<std::mutex> lock(g_mu);
    for (int i = 0; i < n && i < NSTAGE; ++i) ms[i] = g_ctx.stage_ms[i];
    return NSTAGE;
}

extern "C" int lmieb_rerun_device(int reps, int flush_l2, double *ms_total, double *ms_stage) {
    std::lock_guard<std::mutex> lock(g_mu);
    Ctx &c = g_ctx;
    if (!c.ready || !c.have_plan) {
        fprintf(stderr, "ERROR: lmieb_rerun_device: no solve has been prepared on this device\n");
        return -1;
    }
    if (flush_l2 && !c.flush) LMIEB_CUDA_TRY(cudaMalloc((void **) &c.flush, FLUSH_BYTES));
    const bool was = c.timing;
    c.timing = true;
    double total = 0., st[NSTAGE] = {};
    cudaEvent_t e0 = c.ev[0], e1 = c.ev[NSTAGE];
    for (int i = 0; i < reps; ++i) {
        if (flush_l2) LMIEB_CUDA_TRY(cudaMemsetAsync(c.flush, i & 0xff, FLUSH_BYTES, c.stream));
        cudaEventRecord(e0, c.stream);
        if (run_kernels(*c.plan)) { c.timing = was; return -1; }
        cudaEventRecord(e1, c.stream);
        LMIEB_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        total += ms;
        for (int k = 1; k < 8; ++k) {
            float sm = 0.f;
            cudaEventElapsedTime(&sm, c.ev[k], c.ev[k + 1]);
            st[k] += sm;
        }
    }
    c.timing = was;
    LMIEB_CUDA_TRY(cudaGetLastError());
    if (ms_total) *ms_total = total;
    if (ms_stage)
        for (int k = 0; k < NSTAGE; ++k) ms_stage[k] = st[k];
    return 0;
}

extern "C" int lmieb_last_work(double *flops, long long *launches, size_t *h2d, size_t *d2h) {
    std::lock_guard<std::mutex> lock(g_mu);
    Ctx &c = g_ctx;
    if (flops)
        for (int i = 0; i < 4; ++i) flops[i] = c.work[i];
    if (launches) *launches = c.plan ? c.plan->launches : 0;
    if (h2d) *h2d = c.h2d;
    if (d2h) *d2h = c.d2h;
    return 0;
}

extern "C" int lmieb_device_info(char *name, int len, int *sms, int *cc_major, int *cc_minor) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (ensure_ready()) return -1;
    cudaDeviceProp prop;
    LMIEB_CUDA_TRY(cudaGetDeviceProperties(&prop, g_ctx.device));
    if (name && len > 0) {
        strncpy(name, prop.name, len - 1);
        name[len - 1] = 0;
    }
    if (sms) *sms = prop.multiProcessorCount;
    if (cc_major) *cc_major = prop.major;
    if (cc_minor) *cc_minor = prop.minor;
    return 0;
}

extern "C" int lmieb_stream(void **stream) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (ensure_ready()) return -1;
    *stream = (void *) g_ctx.stream;
    return 0;
}
