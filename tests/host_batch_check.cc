// CPU check of the C host layer's batch flow (lmie_b200/csrc/host_api.c):
// the device layer is replaced by a stub that records what each problem
// hands to the device (a hash of every per-radius array) and writes
// recognisable results, so that the preparation, the chunking into parts,
// the per-case scratch blocks (carved from one pooled block, re-zeroed when
// reused), the quadrature of every size distribution, the scatter into the
// callers' arrays (the Fortran entry's column-major ones too), save_control,
// the failure path and the radius sharing can be checked without a GPU.  Prints "ok" or the failed
// check; exit status 0 only with "ok".
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "host_pool.h"
#include "lmieb.h"
#include "lmie_interface.h"

extern "C" int lmie_solution_batch2(int n_cases, lmie_in_data *in, lmie_out_data *out, int alloc_out,
                                    int verbose, int n_threads, int precision);
extern "C" int lmieb_set_pipeline(int chunks);

namespace {

struct Seen {
    unsigned long long hash = 0;
    int n_coef = 0, n = 0, n_qang = 0, save_control = 0;
    bool has_w2 = false, has_saved = false;
    std::vector<double> x;
};
std::mutex g_mu;
std::map<double, Seen> g_batch;      // by mr: what the batch path handed over
std::map<double, Seen> g_single;     // by mr: what lmieb_device_solve got
int g_group_rank = 0, g_group_world = 0;
long long g_ticket = 0;

unsigned long long fnv(unsigned long long h, const void *p, size_t bytes) {
    const unsigned char *b = (const unsigned char *) p;
    for (size_t i = 0; i < bytes; ++i) h = (h ^ b[i]) * 1099511628211ull;
    return h;
}

Seen record(const lmieb_problem &p) {
    unsigned long long h = 1469598103934665603ull;
    const int ints[] = {p.n, p.nd, p.nd1, p.nd2, p.n1, p.n_qang, p.n_coef, p.want_gc, p.want_lc,
                        p.pf_from, p.n_angles, p.save_control};
    h = fnv(h, ints, sizeof ints);
    h = fnv(h, p.idx1, sizeof(int) * p.nd1);
    h = fnv(h, p.idx2, sizeof(int) * p.nd2);
    const double d[] = {p.lambda, p.mr, p.mi, p.accuracy};
    h = fnv(h, d, sizeof d);
    h = fnv(h, p.x, sizeof(double) * p.n);
    h = fnv(h, p.xl, sizeof(double) * p.nd1 * p.n);
    h = fnv(h, p.w, sizeof(double) * (1 + p.nd) * p.n);
    h = fnv(h, p.n1r, sizeof(int) * p.n);
    h = fnv(h, p.n2r, sizeof(int) * p.n);
    if (p.n_angles > 0) h = fnv(h, p.mu_user, sizeof(double) * p.n_angles);
    if (p.save_control == 2 && p.w2) h = fnv(h, p.w2, sizeof(double) * (p.nd > 0 ? p.nd : 1) * p.n);
    Seen s;
    s.hash = h;
    s.n_coef = p.n_coef;
    s.n = p.n;
    s.n_qang = p.n_qang;
    s.save_control = p.save_control;
    s.has_w2 = p.w2 != nullptr;
    s.has_saved = p.save1_rows != nullptr && (p.n_qang == 0 || p.save2_rows != nullptr);
    s.x.assign(p.x, p.x + p.n);
    return s;
}

// recognisable results of problem p
double scal_of(double mr, int c, int e) { return mr * 10. + c + 0.125 * e; }
double row_of(double mr, int k, int l) { return mr + k * 1e-3 + l * 1e-7; }

void fill(const lmieb_problem &p, lmieb_result &r) {
    const int ncol = 1 + p.nd;
    for (int c = 0; c < ncol; ++c)
        for (int e = 0; e < 4; ++e) r.scal[c * 4 + e] = scal_of(p.mr, c, e);
    for (int k = 0; k < ncol * 6; ++k) {
        if (r.gc_rows)
            for (int l = 0; l < p.n_coef; ++l) r.gc_rows[k][l] = row_of(p.mr, k, l);
        if (r.pf_rows)
            for (int j = 0; j < p.n_angles; ++j) r.pf_rows[k][j] = row_of(p.mr, k, j) + 0.5;
    }
    r.n_coef_out = p.n_coef - 1;
    if (r.save1)
        for (int i = 0; i < 4 * p.n; ++i) r.save1[i] = p.mr + i * 1e-6;
    if (r.save2)
        for (size_t i = 0; i < (size_t) 4 * p.n * p.n_qang; ++i) r.save2[i] = p.mr - i * 1e-9;
}

}  // namespace

// ---- the device layer, stubbed ----
extern "C" {
void lmieb_host_parallel(int n, int n_threads, void (*fn)(void *, int), void *arg) {
    const int nt = std::max(1, std::min(std::min(n_threads, 64), n));
    std::atomic<int> next(0);
    const std::function<void()> body = [&]() {
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= n) break;
            fn(arg, i);
        }
    };
    if (nt <= 1) body();
    else host_pool().run(nt, body);
}
void lmieb_host_phase(int, double) {}
int lmieb_timing_state(void) { return 0; }
int lmieb_fault_injected(const char *) { return 0; }
int lmieb_device_fit(int n, const lmieb_problem *) { return n; }
long long lmieb_device_submit(int n, const lmieb_problem *p, lmieb_result *r, int) {
    std::lock_guard<std::mutex> lock(g_mu);
    for (int i = 0; i < n; ++i) {
        g_batch[p[i].mr] = record(p[i]);
        fill(p[i], r[i]);
    }
    return g_ticket++;
}
int lmieb_device_collect(long long) { return 0; }
int lmieb_device_solve(const lmieb_problem *p, lmieb_result *r) {
    std::lock_guard<std::mutex> lock(g_mu);
    g_single[p->mr] = record(*p);
    fill(*p, *r);
    return 0;
}
int lmieb_get_radius_group(int *rank, int *world) {
    if (g_group_world < 1) return 0;
    *rank = g_group_rank;
    *world = g_group_world;
    return 1;
}
int lmieb_group_abort(int, int) { return -1; }
int lmieb_get_user_angle_part(void) { return 256; }
double lmieb_get_work_granularity(int) { return 4.; }
int lmieb_set_user_angle_part(int) { return 0; }
int lmieb_set_work_granularity(int, double) { return 0; }
int lmieb_set_timing(int) { return 0; }
int lmieb_last_timing(double *, int) { return 0; }
int lmieb_last_host_timing(double *, int) { return 0; }
}

// ---- the check ----
namespace {

int fails = 0;
#define CHECK(cond, ...)                                  \
    do {                                                  \
        if (!(cond)) {                                    \
            if (fails++ < 10) {                           \
                printf("FAILED %s:%d: ", __FILE__, __LINE__); \
                printf(__VA_ARGS__);                      \
                printf("\n");                             \
            }                                             \
        }                                                 \
    } while (0)

constexpr int ND = 4;
double unit_l[4][ND] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}};
double zero_l[ND] = {0, 0, 0, 0};

// case i: gamma or log-normal, r_eff from 0.05 to ~20 um, 100 .. 1100 radii
lmie_in_data make_case(int i) {
    lmie_in_data in;
    memset(&in, 0, sizeof in);
    const double r_eff = 0.05 * std::exp(0.2 * i), v_eff = 0.02 + 0.01 * (i % 25);
    const double lam = 0.34 + 0.05 * (i % 30);
    in.calc_gc = 1;
    in.calc_lc = 0;
    in.calc_pf = 1;
    in.n_angles = 181;
    in.lambda = lam;
    in.mr = 1.33 + 1e-3 * i;            // the key of the case
    in.mi = 1e-8 * std::pow(10., (i % 7));
    in.r2 = r_eff * (1. + 10. * v_eff);
    in.r1 = 1e-3 * r_eff;
    if (i % 2 == 0) {
        in.dist_type = SIZE_DIST_GAMMA;
        in.a1 = r_eff;
        in.a2 = v_eff;
    } else {
        in.dist_type = SIZE_DIST_LOG_NORMAL;
        in.a2 = std::log(1. + v_eff);
        in.a1 = r_eff / std::pow(1. + v_eff, 2.5);
    }
    const double xmax = 2. * M_PI * in.r2 / lam;
    in.n_int2 = std::min(11, std::max(1, (int) std::ceil((xmax + 20.) / 100.)));
    in.n_quad = 100;
    in.accuracy = 1e-7;
    in.n_derivs = ND;
    in.mr_l = unit_l[0];
    in.mi_l = unit_l[1];
    in.a1_l = unit_l[2];
    in.a2_l = unit_l[3];
    in.lambda_l = in.a3_l = in.a4_l = in.a5_l = in.r1_l = in.r2_l = zero_l;
    return in;
}

// case i of the other distributions (the parameters of the named test cases)
lmie_in_data make_other(int i) {
    lmie_in_data in = make_case(0);
    in.lambda = 0.6 + 0.01 * i;
    in.mr = 1.6 + 1e-3 * i;             // the key of the case (apart from make_case's)
    in.n_int1 = 0;
    in.n_int2 = 3;
    in.n_quad = 40;
    in.a3 = in.a4 = in.a5 = 0.;
    in.r1 = 0.01;
    in.r2 = 4.;
    switch (i % 7) {
    case 0:
        in.dist_type = SIZE_DIST_MODIFIED_GAMMA;
        in.a1 = 2.;
        in.a2 = 0.5;
        in.a3 = 1.;
        in.r2 = 3.;
        in.n_int2 = 2;
        in.n_quad = 50;
        break;
    case 1:
        in.dist_type = SIZE_DIST_POWER_LAW;      // its range follows from a1, a2
        in.a1 = 0.5;
        in.a2 = 0.2;
        break;
    case 2:
        in.dist_type = SIZE_DIST_MODIFIED_POWER_LAW;
        in.a1 = -3.;
        in.r1 = 0.1;
        in.r2 = 2.;
        in.n_int1 = 2;
        in.n_quad = 30;
        break;
    case 3:
        in.dist_type = SIZE_DIST_MODIFIED_BIMODAL_LOG_NORMAL;
        in.a1 = 0.2;
        in.a2 = 0.2;
        in.a3 = 1.;
        in.a4 = 0.3;
        in.a5 = 0.1;
        break;
    case 4:
        in.dist_type = SIZE_DIST_EXPONENTIAL;
        in.a1 = 2.;
        in.r2 = 2.;
        break;
    case 5:
        in.dist_type = SIZE_DIST_MONO;
        in.a1 = in.r1 = in.r2 = 1.3;
        break;
    default:
        in.dist_type = SIZE_DIST_GAMMA;          // an odd number of Gauss points
        in.a1 = 0.5;
        in.a2 = 0.2;
        in.n_quad = 41;
        break;
    }
    return in;
}

// the scatter of case i's stubbed results into out
void check_out(const lmie_in_data &in, const lmie_out_data &o, const Seen &s, int i) {
    const double mr = in.mr;
    CHECK(o.cext == scal_of(mr, 0, 0) && o.csca == scal_of(mr, 0, 1) && o.cbak == scal_of(mr, 0, 2) &&
              o.g == scal_of(mr, 0, 3), "case %d scalars", i);
    for (int k = 0; k < ND; ++k)
        CHECK(o.cext_l[k] == scal_of(mr, 1 + k, 0) && o.g_l[k] == scal_of(mr, 1 + k, 3), "case %d scalar %d", i, k);
    CHECK(o.n_coef == s.n_coef - 1, "case %d n_coef %d vs %d", i, o.n_coef, s.n_coef - 1);
    for (int e = 0; e < 6; ++e) {
        CHECK(o.gc[e][0] == row_of(mr, e, 0) && o.gc[e][s.n_coef - 1] == row_of(mr, e, s.n_coef - 1),
              "case %d gc row %d", i, e);
        CHECK(o.pf[e][180] == row_of(mr, e, 180) + 0.5, "case %d pf row %d", i, e);
        for (int k = 0; k < ND; ++k) {
            CHECK(o.gc_l[k][e][7] == row_of(mr, (1 + k) * 6 + e, 7), "case %d gc_l %d %d", i, k, e);
            CHECK(o.pf_l[k][e][90] == row_of(mr, (1 + k) * 6 + e, 90) + 0.5, "case %d pf_l %d %d", i, k, e);
        }
    }
}

}  // namespace

int main() {
    const int N = 48;
    std::vector<lmie_in_data> in(N);
    std::vector<lmie_out_data> out(N);
    for (int i = 0; i < N; ++i) in[i] = make_case(i);

    // the same cases cut into 1, 3 and 4 parts, and again (recycled blocks):
    // every case hands the device the same arrays, bit for bit
    std::map<double, unsigned long long> first;
    const int parts[] = {1, 3, 4, 4, 1};
    for (int q = 0; q < 5; ++q) {
        lmieb_set_pipeline(parts[q]);
        g_batch.clear();
        const int rc = lmie_solution_batch2(N, in.data(), out.data(), 1, 0, 8, 0);
        CHECK(rc == 0, "batch rc %d with %d parts", rc, parts[q]);
        CHECK((int) g_batch.size() == N, "%d problems seen with %d parts", (int) g_batch.size(), parts[q]);
        for (int i = 0; i < N; ++i) {
            const Seen &s = g_batch[in[i].mr];
            CHECK(s.n >= 100, "case %d has %d radii", i, s.n);
            if (q == 0) first[in[i].mr] = s.hash;
            else CHECK(s.hash == first[in[i].mr], "case %d differs with %d parts (call %d)", i, parts[q], q);
            check_out(in[i], out[i], s, i);
            lmie_out_free(&out[i], 1);
        }
    }

    // one case on its own (lmie_solution): the batch's arrays
    {
        lmie_out_data o;
        memset(&o, 0, sizeof o);
        const int rc = lmie_solution(&in[5], &o, 1, 0, 4, 0);
        CHECK(rc == 0, "single rc %d", rc);
        CHECK(g_single.count(in[5].mr) && g_single[in[5].mr].hash == first[in[5].mr], "single case differs");
        check_out(in[5], o, g_single[in[5].mr], 5);
        lmie_out_free(&o, 1);
    }

    // the Fortran entry (lmie_solution2_l_, all arguments by reference) on
    // flat column-major arrays: gc(max_coef,6), gc_l(max_coef,6,nd),
    // pf(n_angles,6), pf_l(n_angles,6,nd) -- the batch's problem, and the
    // results at their column-major places
    {
        lmie_in_data c = in[3];
        int mc = lmie_calc_max_coef(c.lambda, c.dist_type, c.a1, c.a2, c.a3, c.r1, c.r2);
        int na = c.n_angles, nd = ND, n_coef = 0, one = 1, zero = 0, nt = 4;
        int n_int1 = c.n_int1, n_int2 = c.n_int2, n_quad = c.n_quad;
        enum size_dist_type dt = c.dist_type;
        double lam = c.lambda, mr = c.mr, mi = c.mi, a1 = c.a1, a2 = c.a2, a3 = c.a3, a4 = c.a4, a5 = c.a5;
        double r1 = c.r1, r2 = c.r2, acc = c.accuracy;
        std::vector<double> gc(6 * mc), gcl(6 * mc * nd), pf(6 * na), pfl(6 * na * nd), theta(na);
        double sc[13] = {}, scl[13][ND] = {};
        double **sv1 = nullptr, ***sv2 = nullptr;
        const int rc = lmie_solution2_l_(
            &one, &zero, &one, &dt, &n_int1, &n_int2, &n_quad, &na, &nd, &zero, &lam, &mr, &mi, &a1, &a2, &a3,
            &a4, &a5, &r1, &r2, c.lambda_l, c.mr_l, c.mi_l, c.a1_l, c.a2_l, c.a3_l, c.a4_l, c.a5_l, c.r1_l,
            c.r2_l, &acc, &n_coef, &sc[0], &sc[1], &sc[2], &sc[3], &sc[4], &sc[5], &sc[6], &sc[7], &sc[8],
            &sc[9], &sc[10], &sc[11], &sc[12], gc.data(), nullptr, theta.data(), pf.data(), scl[0], scl[1],
            scl[2], scl[3], scl[4], scl[5], scl[6], scl[7], scl[8], scl[9], scl[10], scl[11], scl[12],
            gcl.data(), nullptr, pfl.data(), &sv1, &sv2, &mc, &zero, &nt, &zero);
        CHECK(rc == 0, "Fortran entry rc %d", rc);
        const Seen &s = g_single[c.mr];
        CHECK(s.hash == first[c.mr], "Fortran entry: the problem differs from the batch's");
        CHECK(n_coef == s.n_coef - 1, "Fortran entry n_coef %d", n_coef);
        CHECK(sc[9] == scal_of(mr, 0, 0) && sc[12] == scal_of(mr, 0, 3), "Fortran entry cext, g");
        CHECK(scl[10][2] == scal_of(mr, 3, 1), "Fortran entry csca_l");
        for (int e = 0; e < 6 && s.n_coef > 5; ++e) {
            CHECK(gc[(size_t) e * mc + 5] == row_of(mr, e, 5), "Fortran gc(6,%d)", e + 1);
            CHECK(pf[(size_t) e * na + 17] == row_of(mr, e, 17) + 0.5, "Fortran pf(18,%d)", e + 1);
            for (int k = 0; k < nd; ++k) {
                CHECK(gcl[((size_t) k * 6 + e) * mc + 5] == row_of(mr, (1 + k) * 6 + e, 5), "Fortran gc_l");
                CHECK(pfl[((size_t) k * 6 + e) * na + 17] == row_of(mr, (1 + k) * 6 + e, 17) + 0.5,
                      "Fortran pf_l");
            }
        }
    }

    // radius sharing: process 1 of 3 gets radii 1, 4, 7, ... of the case
    {
        g_group_rank = 1;
        g_group_world = 3;
        lmie_out_data o;
        memset(&o, 0, sizeof o);
        const int rc = lmie_solution(&in[6], &o, 1, 0, 4, 1);
        g_group_world = 0;
        CHECK(rc == 0, "shared rc %d", rc);
        const Seen &full = g_batch[in[6].mr], &share = g_single[in[6].mr];
        CHECK(share.n == (full.n - 1 + 2) / 3, "share of %d radii: %d", full.n, share.n);
        for (int t = 0; t < share.n && t < (int) share.x.size(); ++t)
            CHECK(share.x[t] == full.x[1 + 3 * t], "share radius %d", t);
        lmie_out_free(&o, 1);
    }

    // save_control 1 (the kernels come back through save1 / save2, which
    // belong to the caller), then 2 (a re-weighting call that reads them and
    // hands over the shape-derivative weights w2)
    {
        lmie_in_data sc = in[2];
        sc.save_control = 1;
        lmie_out_data o;
        memset(&o, 0, sizeof o);
        CHECK(lmie_solution(&sc, &o, 1, 0, 4, 0) == 0, "save_control 1");
        const Seen s1 = g_single[sc.mr];
        CHECK(s1.save_control == 1 && o.save1 && o.save2, "save_control 1 kept no kernels");
        if (o.save1 && o.save2) {
            CHECK(o.save1[3][s1.n - 1] == sc.mr + (3 * s1.n + s1.n - 1) * 1e-6, "save1");
            CHECK(o.save2[0][1][2] == sc.mr - (1.0 * s1.n_qang + 2) * 1e-9, "save2");
        }
        check_out(sc, o, s1, 2);
        sc.save_control = 2;
        sc.a2 *= 1.1;                        // new shape weights, the same radii
        CHECK(lmie_solution(&sc, &o, 0, 0, 4, 0) == 0, "save_control 2");
        const Seen s2 = g_single[sc.mr];
        CHECK(s2.save_control == 2 && s2.has_w2 && s2.has_saved && s2.n == s1.n, "save_control 2 inputs");
        check_out(sc, o, s2, 2);
        sc.save_control = 2;                 // without kept kernels: rejected
        lmie_out_data none;
        memset(&none, 0, sizeof none);
        CHECK(lmie_solution(&sc, &none, 1, 0, 4, 0) == -1, "save_control 2 without kernels accepted");
        lmie_out_free(&none, 1);
        free(o.save1);
        free(o.save2);
        lmie_out_free(&o, 1);
    }

    // a case the host rejects fails the call (-1), and the next call is whole again
    {
        std::vector<lmie_in_data> bad(in.begin(), in.begin() + 8);
        bad[3].calc_gc = 0;                  // calc_pf without calc_gc / calc_lc
        std::vector<lmie_out_data> o(8);
        lmieb_set_pipeline(3);
        CHECK(lmie_solution_batch2(8, bad.data(), o.data(), 1, 0, 4, 0) == -1, "bad case accepted");
        for (auto &x : o) lmie_out_free(&x, 1);
        g_batch.clear();
        std::vector<lmie_out_data> o2(8);
        CHECK(lmie_solution_batch2(8, in.data(), o2.data(), 1, 0, 4, 0) == 0, "call after a failure");
        for (int i = 0; i < 8; ++i) {
            CHECK(g_batch[in[i].mr].hash == first[in[i].mr], "case %d after a failure", i);
            check_out(in[i], o2[i], g_batch[in[i].mr], i);
            lmie_out_free(&o2[i], 1);
        }
    }

    // the other size distributions (their quadratures and weights) the same way
    {
        std::vector<lmie_in_data> oth;
        for (int i = 0; i < 14; ++i) oth.push_back(make_other(i));
        std::map<double, unsigned long long> h1;
        for (int q = 0; q < 3; ++q) {
            lmieb_set_pipeline(q == 1 ? 4 : 1);
            std::vector<lmie_out_data> o(oth.size());
            g_batch.clear();
            const int rc = lmie_solution_batch2((int) oth.size(), oth.data(), o.data(), 1, 0, 4, 0);
            CHECK(rc == 0, "other distributions: rc %d (call %d)", rc, q);
            for (size_t i = 0; i < oth.size(); ++i) {
                const Seen &s = g_batch[oth[i].mr];
                CHECK(s.n > 0 && s.n_coef > 8, "other case %d: %d radii, %d coefficients", (int) i, s.n, s.n_coef);
                if (q == 0) h1[oth[i].mr] = s.hash;
                else CHECK(s.hash == h1[oth[i].mr], "other case %d differs (call %d)", (int) i, q);
                if (s.n_coef > 8) check_out(oth[i], o[i], s, 100 + (int) i);
                lmie_out_free(&o[i], 1);
            }
        }
    }

    if (fails) {
        printf("%d checks failed\n", fails);
        return 1;
    }
    printf("ok\n");
    return 0;
}
