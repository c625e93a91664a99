// driver.cu -- device side of the polydisperse solve: owns the CUDA context
// state (stream, device arena, pinned staging, Gauss-angle pool), lays out a
// batch of prepared cases, uploads it in one copy, runs the kernel sequence
// and returns the results in one copy.  Replaces the reference's
// lmie_core_shared / lmie_core_sequential / lmie_core_xthreads fan-out
// (src/lmie_schedule.c:154-452) and the driver half of lmie_core_solution
// (src/lmie_schedule.c:942-1268); a batch of cases is the unit of work, and a
// single lmie_solution() is a batch of one.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <set>
#include <thread>
#include <unordered_map>
#include <vector>

#include <dlfcn.h>
#include <unistd.h>

#include "host_pool.h"
#include "kernels.h"
#include "oz_layout.cuh"
#include "tc_layout.cuh"
#include "lmieb.h"
#include "../../include/lmie_b200.h"

namespace {

constexpr int NSTAGE = LMIEB_N_STAGES;
constexpr size_t FLUSH_BYTES = (size_t) 256 << 20;     // > 126 MB L2
constexpr size_t BATCH_BYTES = (size_t) 24 << 30;      // device working set of one sub-batch
constexpr int MAX_PIECES = 16;                         // results come back in up to 16 pieces of cases
constexpr int SLOT_GRAPHS = 4;                         // captured kernel sequences kept per slot
constexpr size_t PIECE_BYTES = (size_t) 8 << 20;       // of about 8 MB or more

// Every staged array starts on a 256-byte boundary and takes at least one
// 256-byte block, so empty arrays never alias their neighbours.
inline size_t pad(size_t bytes) { return ((bytes ? bytes : 1) + 255) & ~(size_t) 255; }

struct Plan;

// Results of a submitted sub-batch still to be unpacked.
struct Pending {
    bool active = false;
    long long ticket = -1;
    int ncase = 0, ncol = 0, R = 0;
    std::vector<DevCase> cs;
    lmieb_result *rs = nullptr;
    char *h_out = nullptr, *d_out = nullptr;     // host copy / device origin of the output block
    int want_gc = 0, want_lc = 0, pf_from = 0, save_control = 0, n_qang0 = 0;
    size_t n_save2 = 0;
    double *o_scal = nullptr, *o_gc = nullptr, *o_lc = nullptr, *o_pf = nullptr;
    double *o_save1 = nullptr, *o_save2 = nullptr;
    int *o_trunc = nullptr;
    int acc_mode = 0;
    double *o_acc = nullptr;           // LMIEB_ACC_PARTIAL: the integrals
    size_t acc_n = 0;
    std::vector<int> piece;            // case ranges [piece[p], piece[p+1]) of the result copies
    double t_submit = 0.;
    const lmieb_problem *ps = nullptr; // the problems (alive until the call that submitted them returns)
    int precision = 0;
};

// One of two buffer sets: a sub-batch is packed into one while the device
// still works on the other's.
struct Slot {
    char *dbuf = nullptr;
    size_t dcap = 0;
    char *hbuf = nullptr;
    size_t hcap = 0;
    Plan *plan = nullptr;
    cudaStream_t stream = nullptr;     // the sub-batches of this slot (consecutive ones overlap)
    // The copies of the results run on a stream of their own: a stream whose
    // last operation was a device-to-host copy queues its next commands (the
    // next upload included) behind every download in flight, those of the
    // other slots too.
    cudaStream_t down = nullptr;
    cudaEvent_t kdone = nullptr;       // after the sub-batch's kernels (the downloads wait for it)
    // int8 K3's A operand and row exponents depend on the angles only: they
    // run on this stream beside K1 (fork and join events)
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    cudaEvent_t done = nullptr;
    cudaEvent_t piece[MAX_PIECES] = {};  // after the copy of each piece of the results
    cudaEvent_t t_begin = nullptr, t_end = nullptr;   // device span of the sub-batch
    bool have_plan = false;
    // Kernel sequences of the slot's recent plans, captured for re-runs.  A
    // pipelined call gives each slot several parts in turn, so one graph per
    // slot would be replaced by every part; the cache keeps SLOT_GRAPHS of
    // them (least recently used goes first), each replayed only for the plan
    // whose signature it was captured from.
    struct Graph {
        cudaGraphExec_t exec = nullptr;
        unsigned long long sig = 0, used = 0;
    } graphs[SLOT_GRAPHS];
    unsigned long long seen[2 * SLOT_GRAPHS] = {};   // signatures of the slot's recent plans (a ring)
    int seen_at = 0;
    unsigned long long clock = 0;
    Pending pend;
};

struct Ctx {
    bool ready = false;
    int device = -1;
    int sms = 0;
    cudaStream_t stream = nullptr;
    Slot slot[3];                   // two alternating slots; the third runs the FP64 re-solves
    int last_slot = -1;             // slot of the last submitted sub-batch
    long long next_ticket = 0;
    long long redo_ticket = 1LL << 62;   // tickets of the re-solve slot (their own range)
    int submits = 0;                // sub-batches submitted since the counters were reset
    int call_slot[2] = {-1, -1};    // slots of the first two sub-batches since then
    long long redo = 0;             // INT8 cases solved again in FP64 since then
    // The FP64 re-solve of INT8 cases takes their coefficient columns and
    // per-radius sums from the INT8 sub-batch's arena (K1 computed them there
    // with the same operations) instead of running K1 again.
    struct Gather {
        bool on = false;
        const double *coef = nullptr, *rs = nullptr;   // the source sub-batch's K1 outputs
        long long tot = 0;                             // its orders per coefficient column
        int R = 0;                                     // its radii
        std::vector<DevCase> cs;                       // its cases, in the order of the re-solve
    } gather;
    cudaEvent_t redo_read = nullptr;   // after a re-solve that reads another slot's arena
    int redo_src = -1;                 // that slot: its next upload waits for the event
    std::vector<std::pair<long long, int>> finished;   // (ticket, rc) of recently collected sub-batches
    char *flush = nullptr;
    cudaEvent_t ev[NSTAGE + 1] = {};
    bool timing = false;
    double stage_ms[NSTAGE] = {};
    double work[4] = {};            // algorithmic flops of the last solve (see lmieb_last_work)
    double tensor_ops = 0.;         // tensor-core operations (2 per multiply-add) its int8 products run
    cudaEvent_t k3[2] = {};         // with timing: around the int8 product kernel
    double k3_ms = 0.;
    long long launches = 0;         // kernel launches of one device run of the last solve
    size_t h2d = 0, d2h = 0;        // bytes copied by the last solve
    long long graph_captures = 0, graph_replays = 0;   // kernel sequences captured / replayed (all calls)
    // radius groups: whether this process's solve has entered the group's
    // reduction, and the block a failed solve reduces instead of its own
    bool group_joined = false;
    double *gfail = nullptr;
    size_t gfail_cap = 0;
    // Gauss-Legendre angles depend only on their number: computed once per n
    // into a device pool ([n nodes][n weights] per entry) and kept
    double *gl_pool = nullptr;
    size_t gl_cap = 0, gl_used = 0;
    std::unordered_map<int, long long> gl_map;     // n -> pool offset
    cudaEvent_t t_first = nullptr;                 // upload start of the call's first sub-batch
    // save_control: the last per-radius kernels (save1, save2) seen, kept on
    // the device and recognised by a hash of their contents, so that the
    // re-weighting calls of a retrieval loop upload them once
    struct {
        double *d = nullptr;            // [4 R] save1 then [4 R max(nq, 1)] save2
        size_t cap = 0;                 // doubles
        unsigned long long key = 0;
        int R = 0, nq = 0;
        bool valid = false;
        long long owner = -1;           // sub-batch whose kernels fill it
        cudaEvent_t ready = nullptr;    // after the copy that filled it
        bool pending = false;
        long long hits = 0, misses = 0;
    } save;
    cudaEvent_t gl_ready = nullptr;                // after the last launch that added entries
    bool gl_pending = false;
    // host-side phases of the last batch call (ms): prepare, pack, device and copies, unpack, finish
    double host_ms[LMIEB_N_HOST] = {};
};

Ctx g_ctx;

// Work items per SM the angular stage is cut into ([0] FP64 kernel, [1]
// TF32 tensor-core kernel, [2] int8 tensor-core kernel): finer items balance
// uneven cases, coarser ones cut the per-item overhead; set by
// lmieb_set_work_granularity (the autotuner).
double g_items_per_sm[3] = {64., 2., 2.};

int prec_slot(int precision) {
    return precision == LMIEB_PRECISION_TF32X3 ? 1 : (precision == LMIEB_PRECISION_INT8 ? 2 : 0);
}

// Orders (in chunks of TC_KC) per FP32 segment of the tensor-core stage's
// hi*hi products; set by lmieb_set_split_segment.
int g_tc_seg = 2;
int g_pu_lp = PU_LP;     // orders per K5 block (lmieb_set_user_angle_part)

// Radius sharing: the group lmie_solution(..., use_mpi != 0) shares its radii
// with, and how the integrals are summed over it -- the caller's function, or
// an NCCL all-reduce queued on the solve's stream.
struct NcclUniqueId { char internal[128]; };    // ncclUniqueId
struct Nccl {
    void *lib = nullptr;
    int (*get_unique_id)(NcclUniqueId *) = nullptr;
    int (*comm_init_rank)(void **, int, NcclUniqueId, int) = nullptr;
    int (*all_reduce)(const void *, void *, size_t, int, int, void *, cudaStream_t) = nullptr;
    int (*comm_destroy)(void *) = nullptr;
    const char *(*error_string)(int) = nullptr;
};
constexpr int NCCL_FLOAT64 = 8, NCCL_SUM = 0;   // ncclFloat64, ncclSum
struct RadiusGroup {
    int rank = 0, world = 1;
    lmieb_reduce_fn fn = nullptr;
    void *fn_ctx = nullptr;
    void *comm = nullptr;                       // ncclComm_t of the built-in reduction
    bool on = false;
} g_group;
Nccl g_nccl;

// Physical cores of the host (distinct core ids of the online CPUs; the
// hardware threads if the topology cannot be read): memory-bound copies
// run faster on one thread per core than on both threads of each core.
int host_cores() {
    static const int n = [] {
        const int hw = (int) std::max(1u, std::thread::hardware_concurrency());
        std::set<std::pair<int, int>> ids;
        for (int cpu = 0; cpu < hw; ++cpu) {
            char path[128];
            int pkg = -1, core = -1;
            snprintf(path, sizeof path, "/sys/devices/system/cpu/cpu%d/topology/physical_package_id", cpu);
            if (FILE *f = fopen(path, "r")) {
                if (fscanf(f, "%d", &pkg) != 1) pkg = -1;
                fclose(f);
            }
            snprintf(path, sizeof path, "/sys/devices/system/cpu/cpu%d/topology/core_id", cpu);
            if (FILE *f = fopen(path, "r")) {
                if (fscanf(f, "%d", &core) != 1) core = -1;
                fclose(f);
            }
            if (pkg < 0 || core < 0) return hw;
            ids.insert({pkg, core});
        }
        return ids.empty() ? hw : (int) ids.size();
    }();
    return n;
}

// fn(i) for every i in [0, n) on the host's cores (dynamic chunks of
// `grain`), on at most max_threads threads (0: one per hardware thread)
template <class F>
void parallel_for(int n, int grain, F &&fn, int max_threads = 0) {
    const int hw = max_threads > 0 ? max_threads : (int) std::max(1u, std::thread::hardware_concurrency());
    const int nt = std::min(std::min(hw, 32), (n + grain - 1) / grain);
    if (nt <= 1) {
        for (int i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<int> next(0);
    const std::function<void()> body = [&]() {
        for (;;) {
            const int i0 = next.fetch_add(grain);
            if (i0 >= n) break;
            for (int i = i0; i < std::min(n, i0 + grain); ++i) fn(i);
        }
    };
    host_pool().run(nt, body);
}

// fn(arg, i) for every i in [0, n) on up to n_threads host threads (the
// case preparation and finishing of the C host layer)
extern "C" void lmieb_host_parallel(int n, int n_threads, void (*fn)(void *, int), void *arg) {
    const int nt = std::max(1, std::min(std::min(n_threads, 64), n));
    if (nt <= 1) {
        for (int i = 0; i < n; ++i) fn(arg, i);
        return;
    }
    std::atomic<int> next(0);
    const std::function<void()> body = [&]() {
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= n) break;
            fn(arg, i);
        }
    };
    host_pool().run(nt, body);
}

// memcpy of a large block on one host thread per core
void par_memcpy(void *dst, const void *src, size_t bytes) {
    const size_t chunk = std::max((size_t) 256 << 10, (bytes / 16 + 4095) & ~(size_t) 4095);
    const int n = (int) ((bytes + chunk - 1) / chunk);
    parallel_for(n, 1, [&](int i) {
        const size_t a = (size_t) i * chunk, b = std::min(bytes, a + chunk);
        memcpy((char *) dst + a, (const char *) src + a, b - a);
    }, host_cores());
}

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
std::mutex g_mu;
int g_want_device = -1;

// Content hash of the save_control kernels: save1 as 4 rows of R, then (when
// nq > 0) save2 as 4 R rows of nq, each row hashed on its own (in parallel),
// the row hashes combined in order.  row(i) gives row i.
inline unsigned long long mix64(unsigned long long h, unsigned long long w) {
    h ^= w;
    h *= 0x9E3779B97F4A7C15ull;
    return h ^ (h >> 29);
}

template <class Row>
unsigned long long save_hash(int R, int nq, Row row) {
    const int nrows = 4 + (nq > 0 ? 4 * R : 0);
    std::vector<unsigned long long> rh((size_t) nrows);
    parallel_for(nrows, 64, [&](int i) {
        const size_t len = i < 4 ? (size_t) R : (size_t) nq;
        const unsigned long long *w = (const unsigned long long *) row(i);
        unsigned long long h = 0x243F6A8885A308D3ull ^ len;
        for (size_t k = 0; k < len; ++k) h = mix64(h, w[k]);
        rh[i] = h;
    });
    unsigned long long h = mix64((unsigned long long) R, (unsigned long long) nq);
    for (int i = 0; i < nrows; ++i) h = mix64(h, rh[i]);
    return h;
}

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

// Everything the kernel sequence of one sub-batch needs, in device memory.
struct Plan {
    DevBatch B;
    int ncase = 0;
    int nd1c = 0, n_ang_launch = 0;
    int want_gc = 0, want_lc = 0, pf_from = 0, save_control = 0, n_qang0 = 0;
    double *ck = nullptr, *coef = nullptr, *rs = nullptr, *sums = nullptr, *part = nullptr;
    double *pfacc = nullptr, *pfn = nullptr, *ckpt = nullptr, *exq = nullptr;
    AngItem *ang = nullptr;     // K3 items (tensor-core items when tc)
    int n_ang = 0;
    AngItem *ang64 = nullptr;   // with tc: FP64 K3 items of the cases kept off the tensor cores
    int n_ang64 = 0;
    int tc = 0;                 // K3 in split precision on the tensor cores
    cudaStream_t side = nullptr;       // the slot's side stream and its fork / join events
    cudaEvent_t fork = nullptr, join = nullptr;
    int tc_seg = 2;             // its segment length (chunks)
    float *bop = nullptr;       // its B operand (tc_layout.cuh)
    size_t bop_bytes = 0;
    int oz = 0;                 // K3 as the int8 fixed-point contraction (oz_layout.cuh)
    unsigned char *bop8 = nullptr;   // its B operand digits
    signed char *rowexp = nullptr;   // its row exponents
    int *colexp = nullptr;      // its column exponents
    long long *rx_start = nullptr;   // (case, half-angle) index space of the row exponents
    long long n_rx = 0;
    unsigned char *aop = nullptr;    // its A operand digits, every (case, angle tile, chunk)
    long long *a_start = nullptr;    // (case, tile row) index space of the A operand
    long long n_arow = 0;
    int n_groups = 0;
    ExpItem *ex = nullptr;
    int n_ex = 0;
    ExpItem *gx = nullptr;      // (case, 0, angle tile) of the GSF expansion runs, longest first
    int n_gx = 0;
    GatherSeg *gsegs = nullptr; // K1's outputs copied from an earlier sub-batch instead of computed
    int n_gseg = 0;
    long long *pf_start = nullptr, *ck_gc = nullptr, *ck_lc = nullptr, *fin_start = nullptr, *pu_start = nullptr;
    long long pf_total = 0, nck_gc = 0, nck_lc = 0, nfin = 0, pu_total = 0;
    double *pu_scr = nullptr;   // K5 partial sums of cases of several parts
    long long pu_nred = 0, *pu_red = nullptr;   // their (case, column, element, angle) index space
    double *save1_in = nullptr, *save2_in = nullptr, *w2 = nullptr;
    double *o_scal = nullptr, *o_gc = nullptr, *o_lc = nullptr, *o_pf = nullptr;
    int *o_trunc = nullptr;     // [2][ncase]: gc, lc
    double *o_save1 = nullptr, *o_save2 = nullptr;
    int acc_mode = 0;           // LMIEB_ACC_* (radius sharing)
    bool no_radii = false;      // this share has no radii: its integrals are zero
    size_t acc_n = 0;           // doubles of sums + pfacc, one block
    double *o_acc = nullptr;
    long long launches = 0;
};

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
    // the third slot runs the FP64 re-solves of a few int8 cases next to the
    // following sub-batch: at the highest priority, its blocks are scheduled
    // as soon as SMs free up instead of waiting behind that sub-batch's
    int prio_lo = 0, prio_hi = 0;
    LMIEB_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    for (Slot &S : c.slot) {
        S.plan = new Plan();
        LMIEB_CUDA_TRY(cudaStreamCreateWithPriority(&S.stream, cudaStreamNonBlocking,
                                                    &S == &c.slot[2] ? prio_hi : prio_lo));
        LMIEB_CUDA_TRY(cudaStreamCreateWithFlags(&S.down, cudaStreamNonBlocking));
        LMIEB_CUDA_TRY(cudaStreamCreateWithPriority(&S.side, cudaStreamNonBlocking,
                                                    &S == &c.slot[2] ? prio_hi : prio_lo));
        LMIEB_CUDA_TRY(cudaEventCreateWithFlags(&S.fork, cudaEventDisableTiming));
        LMIEB_CUDA_TRY(cudaEventCreateWithFlags(&S.join, cudaEventDisableTiming));
        LMIEB_CUDA_TRY(cudaEventCreateWithFlags(&S.kdone, cudaEventDisableTiming));
        LMIEB_CUDA_TRY(cudaEventCreateWithFlags(&S.done, cudaEventDisableTiming));
        for (cudaEvent_t &e : S.piece) LMIEB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        LMIEB_CUDA_TRY(cudaEventCreate(&S.t_begin));
        LMIEB_CUDA_TRY(cudaEventCreate(&S.t_end));
    }
    LMIEB_CUDA_TRY(cudaEventCreate(&c.t_first));
    LMIEB_CUDA_TRY(cudaEventCreate(&c.k3[0]));
    LMIEB_CUDA_TRY(cudaEventCreate(&c.k3[1]));
    LMIEB_CUDA_TRY(cudaEventCreateWithFlags(&c.save.ready, cudaEventDisableTiming));
    LMIEB_CUDA_TRY(cudaEventCreateWithFlags(&c.gl_ready, cudaEventDisableTiming));
    LMIEB_CUDA_TRY(cudaEventCreateWithFlags(&c.redo_read, cudaEventDisableTiming));
    c.ready = true;
    return 0;
}

// Host-side fault injection (tests of the failure paths; no GPU fault is
// involved): while the environment variable LMIEB_FAULT holds a site name --
// "alloc" (the device arena), "pinned" (the pinned staging buffer), "h2d" (a
// sub-batch's input upload) or "graph" (instantiating a captured kernel
// sequence), several separated by commas -- that step fails as its CUDA call
// would (the arena and the staging buffer are released first, as when a
// larger one cannot be had), and the error propagates as -1.
bool fault_injected(const char *site);
}  // namespace

// the injector for the host code of host_api.c ("prepare": a case's host
// preparation)
extern "C" int lmieb_fault_injected(const char *site) { return fault_injected(site) ? 1 : 0; }

namespace {
bool fault_injected(const char *site) {
    const char *v = getenv("LMIEB_FAULT");
    if (!v || !*v) return false;
    const size_t n = strlen(site);
    for (const char *p = v; *p;) {
        const char *e = strchr(p, ',');
        const size_t len = e ? (size_t) (e - p) : strlen(p);
        if (len == n && strncmp(p, site, n) == 0) {
            fprintf(stderr, "ERROR: lmie_b200: injected failure at \"%s\" (LMIEB_FAULT)\n", site);
            return true;
        }
        if (!e) break;
        p = e + 1;
    }
    return false;
}

// Forgets every captured sequence of the slot (its arena or a pool they
// point at was replaced).
void drop_graph(Slot &S) {
    for (Slot::Graph &g : S.graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g = Slot::Graph();
    }
    for (unsigned long long &v : S.seen) v = 0;
}

// The slot's captured sequence of plan `sig`, or null.
cudaGraphExec_t find_graph(Slot &S, unsigned long long sig) {
    for (Slot::Graph &g : S.graphs)
        if (g.exec && g.sig == sig) {
            g.used = ++S.clock;
            return g.exec;
        }
    return nullptr;
}

// Whether plan `sig` came to the slot recently; records it.
bool seen_plan(Slot &S, unsigned long long sig) {
    bool hit = false;
    for (unsigned long long v : S.seen) hit = hit || v == sig;
    if (!hit) {
        S.seen[S.seen_at] = sig;
        S.seen_at = (S.seen_at + 1) % (2 * SLOT_GRAPHS);
    }
    return hit;
}

int ensure_device(Slot &S, size_t bytes) {
    const bool fail = fault_injected("alloc");
    if (bytes <= S.dcap && !fail) return 0;
    S.have_plan = false;
    drop_graph(S);
    if (S.dbuf) LMIEB_CUDA_TRY(cudaFree(S.dbuf));
    S.dbuf = nullptr;
    S.dcap = 0;
    size_t want = bytes + bytes / 4;
    LMIEB_CUDA_TRY(fail ? cudaErrorMemoryAllocation : cudaMalloc((void **) &S.dbuf, want));
    S.dcap = want;
    return 0;
}

int ensure_host(Slot &S, size_t bytes) {
    const bool fail = fault_injected("pinned");
    if (bytes <= S.hcap && !fail) return 0;
    if (S.hbuf) LMIEB_CUDA_TRY(cudaFreeHost(S.hbuf));
    S.hbuf = nullptr;
    S.hcap = 0;
    size_t want = bytes + bytes / 4;
    LMIEB_CUDA_TRY(fail ? cudaErrorMemoryAllocation : cudaMallocHost((void **) &S.hbuf, want));
    S.hcap = want;
    return 0;
}

// grow the Gauss pool, keeping its contents
int ensure_gl_pool(size_t doubles) {
    Ctx &c = g_ctx;
    if (doubles <= c.gl_cap) return 0;
    size_t want = std::max(doubles + doubles / 2, (size_t) 1 << 16);
    double *np = nullptr;
    LMIEB_CUDA_TRY(cudaMalloc((void **) &np, want * sizeof(double)));
    if (c.gl_pool) {
        // entries may still be in the making on either slot's stream
        LMIEB_CUDA_TRY(cudaDeviceSynchronize());
        LMIEB_CUDA_TRY(cudaMemcpyAsync(np, c.gl_pool, c.gl_used * sizeof(double), cudaMemcpyDeviceToDevice,
                                       c.stream));
        LMIEB_CUDA_TRY(cudaStreamSynchronize(c.stream));
        LMIEB_CUDA_TRY(cudaFree(c.gl_pool));
    }
    c.gl_pool = np;
    c.gl_cap = want;
    for (Slot &S : c.slot) {   // their plans point at the old pool
        S.have_plan = false;
        drop_graph(S);
    }
    return 0;
}

inline void stage(int i) {
    if (g_ctx.timing) cudaEventRecord(g_ctx.ev[i], g_ctx.stream);
}

// Stages 1..3 of a sub-batch: the radius integrals (sums, pfacc).
int run_accumulate(Plan &L, cudaStream_t s) {
    const DevBatch &B = L.B;
    stage(1);
    if (L.acc_mode == LMIEB_ACC_FINISH || L.no_radii) {
        // summed integrals uploaded with the inputs, or none on this share
        if (L.no_radii) LMIEB_CUDA_TRY(cudaMemsetAsync(L.sums, 0, L.acc_n * sizeof(double), s));
        stage(2);
        stage(3);
        return 0;
    }
    if (L.save_control != 2) {
        // int8 K3's row exponents and A operand (the angles only) on the slot's
        // side stream while K1 runs: K1 keeps 8 warps per SM, so their blocks
        // find room beside it (with per-stage timing: in line, below)
        const bool fork = L.oz && L.n_ang > 0 && L.side && !g_ctx.timing;
        if (fork) {
            LMIEB_CUDA_TRY(cudaEventRecord(L.fork, s));
            LMIEB_CUDA_TRY(cudaStreamWaitEvent(L.side, L.fork, 0));
            if (launch_oz_operands(L.side, B, L.n_rx, L.rx_start, L.rowexp, L.n_arow, L.a_start, L.aop, 0,
                                   nullptr, nullptr, nullptr))
                return -1;
            LMIEB_CUDA_TRY(cudaEventRecord(L.join, L.side));
        }
        if (L.n_gseg > 0) {
            if (launch_gather(s, L.n_gseg, L.gsegs, L.coef, L.rs)) return -1;
        } else {
            for (int ch = 0; ch < (L.nd1c > 0 ? L.nd1c : 1); ++ch) {
                const int c0 = ch * 4;
                const int nc = std::max(0, std::min(4, B.nd1 - c0));
                if (launch_coef(s, B, nc, c0, ch == 0, L.ck, L.coef, L.bop, L.rs)) return -1;
            }
        }
        stage(2);
        if (launch_reduce_scalars(s, B, L.rs, L.sums, L.save_control == 1 ? L.o_save1 : nullptr)) return -1;
        stage(3);
        const bool tcx = L.tc || L.oz;
        const int n64 = tcx ? L.n_ang64 : L.n_ang;
        const AngItem *a64 = tcx ? L.ang64 : L.ang;
        if (L.tc && L.n_ang > 0 &&
            launch_angular_tc(s, B, L.n_ang, L.ang, L.bop, L.part, L.tc_seg, L.o_trunc + 2 * L.ncase))
            return -1;
        if (L.oz && L.n_ang > 0) {
            if (fork) LMIEB_CUDA_TRY(cudaStreamWaitEvent(s, L.join, 0));
            if (launch_oz_operands(s, B, fork ? 0 : L.n_rx, L.rx_start, L.rowexp, fork ? 0 : L.n_arow, L.a_start,
                                   L.aop, L.n_groups, L.coef, L.bop8, L.colexp))
                return -1;
            if (g_ctx.timing) LMIEB_CUDA_TRY(cudaEventRecord(g_ctx.k3[0], s));
            if (launch_angular_oz(s, B, L.n_ang, L.ang, L.bop8, L.part, L.o_trunc + 2 * L.ncase)) return -1;
            if (g_ctx.timing) LMIEB_CUDA_TRY(cudaEventRecord(g_ctx.k3[1], s));
        }
        if (n64 > 0) {
            for (int t = 0; t < L.n_ang_launch; ++t) {
                const int c1 = t * 4, c2 = t * 4;
                const int nc1 = std::max(0, std::min(4, B.nd1 - c1));
                const int nc2 = std::max(0, std::min(4, B.nd2 - c2));
                if (launch_angular(s, B, nc1, c1, nc2, c2, t == 0, n64, a64, L.coef, L.part,
                                   L.save_control == 1 ? L.o_save2 : nullptr))
                    return -1;
            }
        }
        if ((L.n_ang > 0 || n64 > 0) && launch_reduce_pf(s, B, L.pf_total, L.pf_start, L.part, L.pfacc)) return -1;
    } else {
        stage(2);
        if (launch_save_reweight(s, B, L.n_qang0, L.save1_in, L.save2_in, L.w2, L.sums, L.pfacc)) return -1;
        stage(3);
    }
    return 0;
}

// Stages 4..7: normalisation, expansions, phase matrix at the user angles.
int run_finish(Plan &L, cudaStream_t s) {
    const DevBatch &B = L.B;
    stage(4);
    if (launch_normalize(s, B, L.pf_total, L.pf_start, L.sums, L.pfacc, L.o_scal, L.pfn)) return -1;
    LMIEB_CUDA_TRY(cudaMemsetAsync(L.o_trunc, 0, sizeof(int) * 2 * L.ncase, s));
    LMIEB_CUDA_TRY(cudaMemsetAsync(L.o_trunc + 2 * L.ncase + 1, 0, sizeof(int) * 4 * L.ncase, s));
    stage(5);
    if (L.want_gc && launch_expand(s, B, 0, L.nck_gc, L.ck_gc, L.n_ex, L.ex, L.n_gx, L.gx, L.nfin, L.fin_start,
                                   L.pfn, L.ckpt, L.exq, L.o_gc, L.o_trunc, L.o_trunc + 2 * L.ncase + 1))
        return -1;
    stage(6);
    if (L.want_lc && launch_expand(s, B, 1, L.nck_lc, L.ck_lc, L.n_ex, L.ex, 0, nullptr, L.nfin, L.fin_start,
                                   L.pfn, L.ckpt, L.exq, L.o_lc, L.o_trunc + L.ncase, L.o_trunc + 4 * L.ncase + 1))
        return -1;
    stage(7);
    if (L.pf_from) {
        const int *tr = L.want_lc ? L.o_trunc + L.ncase : L.o_trunc;
        const double *cf = L.pf_from == 1 ? L.o_gc : L.o_lc;
        if (launch_phase_user(s, B, L.pf_from == 1 ? 0 : 1, L.pu_total, L.pu_start, cf, tr, L.o_pf, L.pu_scr,
                              L.pu_nred, L.pu_red))
            return -1;
    }
    stage(8);
    return 0;
}

// The kernel sequence of one sub-batch on resident inputs (stages 1..7).
int run_kernels(Plan &L, cudaStream_t s) {
    return run_accumulate(L, s) || run_finish(L, s) ? -1 : 0;
}

// Identity of a kernel sequence: FNV-1a over the plan's bytes -- every
// pointer, count, launch parameter and the batch descriptor the kernels get
// (the plan is plain data, zero-initialised with its padding).
unsigned long long plan_sig(const Plan &L) {
    const unsigned char *b = (const unsigned char *) &L;
    unsigned long long h = 1469598103934665603ull;
    for (size_t i = 0; i < sizeof(Plan); ++i) h = (h ^ b[i]) * 1099511628211ull;
    return h;
}

// Captures the slot's kernel sequence (stages 1..7) on stream s into a graph.
int capture_plan(Slot &S, cudaStream_t s) {
    Ctx &c = g_ctx;
    const bool was = c.timing;
    c.timing = false;
    cudaGraph_t g = nullptr;
    LMIEB_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const int rc = run_kernels(*S.plan, s);
    const cudaError_t ec = cudaStreamEndCapture(s, &g);
    c.timing = was;
    if (rc || ec != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        fprintf(stderr, "ERROR: lmie_b200: graph capture failed (%s)\n", cudaGetErrorString(ec));
        return -1;
    }
    // into a free entry, else in place of the least recently used
    Slot::Graph *slot_g = &S.graphs[0];
    for (Slot::Graph &e : S.graphs)
        if (!e.exec || (slot_g->exec && e.used < slot_g->used)) slot_g = &e;
    if (slot_g->exec) cudaGraphExecDestroy(slot_g->exec);
    *slot_g = Slot::Graph();
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = fault_injected("graph") ? cudaErrorInvalidValue : cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
        fprintf(stderr, "ERROR: lmie_b200: graph instantiation failed (%s)\n", cudaGetErrorString(ei));
        return -1;
    }
    slot_g->exec = exec;
    slot_g->sig = plan_sig(*S.plan);
    slot_g->used = ++S.clock;
    ++c.graph_captures;
    return 0;
}

// In-place sum over the radius group of `count` doubles at device address
// buf, written on stream s: the library's NCCL all-reduce queued on s, or the
// caller's reduction on the synchronised buffer.
int group_reduce(double *buf, size_t count, cudaStream_t s) {
    const RadiusGroup &g = g_group;
    if (g.comm) {
        const int r = g_nccl.all_reduce(buf, buf, count, NCCL_FLOAT64, NCCL_SUM, g.comm, s);
        if (r != 0) {
            fprintf(stderr, "ERROR: lmie_b200: ncclAllReduce: %s\n", g_nccl.error_string(r));
            return -1;
        }
        return 0;
    }
    if (!g.fn) return 0;
    LMIEB_CUDA_TRY(cudaStreamSynchronize(s));
    if (g.fn(buf, (long long) count, (void *) s, g.fn_ctx) != 0) {
        fprintf(stderr, "ERROR: lmie_b200: the radius group's reduction failed\n");
        return -1;
    }
    return 0;
}

// Sums the integrals of a LMIEB_ACC_GROUP sub-batch over the radius group,
// on stream s between run_accumulate and run_finish.  The block carries one
// more double, the number of processes whose solve failed before the
// reduction (zero here, one from each failed process: group_abort); if it
// is not zero after the sum, the error word tells the host to return -1.
int reduce_group(Plan &L, cudaStream_t s) {
    g_ctx.group_joined = true;
    LMIEB_CUDA_TRY(cudaMemsetAsync(L.sums + L.acc_n, 0, sizeof(double), s));
    if (group_reduce(L.sums, L.acc_n + 1, s)) return -1;
    return launch_group_flag(s, L.sums + L.acc_n, L.o_trunc + 2 * L.ncase);
}

// A process of the radius group whose solve failed before the group's
// reduction still takes part in it, with zero integrals and a failure mark in
// the extra slot, so that the other processes are not left waiting in theirs
// and fail as well.  `acc_n`: the integrals of the solve, 4 (1 + n_derivs)
// (1 + n_qang), the same on every process.  Returns -1 (the solve failed).
int group_abort(size_t acc_n) {
    Ctx &c = g_ctx;
    if (!g_group.on || c.group_joined) return -1;
    c.group_joined = true;
    if (ensure_ready()) return -1;
    if (acc_n + 1 > c.gfail_cap) {
        if (c.gfail) cudaFree(c.gfail);
        c.gfail = nullptr;
        c.gfail_cap = 0;
        LMIEB_CUDA_TRY(cudaMalloc((void **) &c.gfail, (acc_n + 1) * sizeof(double)));
        c.gfail_cap = acc_n + 1;
    }
    static const double one = 1.;
    LMIEB_CUDA_TRY(cudaMemsetAsync(c.gfail, 0, acc_n * sizeof(double), c.stream));
    LMIEB_CUDA_TRY(cudaMemcpyAsync(c.gfail + acc_n, &one, sizeof(double), cudaMemcpyHostToDevice, c.stream));
    if (group_reduce(c.gfail, acc_n + 1, c.stream) == 0) cudaStreamSynchronize(c.stream);
    fprintf(stderr, "ERROR: lmie_b200: this process's share of the radius group failed; the group was told\n");
    return -1;
}

template <class T>
T *put(char *hp, size_t &off, const T *src, size_t count) {
    T *at = (T *) (hp + off);
    if (src && count) par_memcpy(at, src, count * sizeof(T));
    off += pad(count * sizeof(T));
    return at;
}

// Makes the save_control cache ready to be overwritten by stream s with a set
// of R radii: waits for the work that may still read the old set, grows it.
int save_fill(int R, size_t n_save2, cudaStream_t s) {
    Ctx &c = g_ctx;
    const size_t need = (size_t) 4 * R + n_save2;
    (void) s;
    LMIEB_CUDA_TRY(cudaDeviceSynchronize());
    c.save.valid = false;
    if (need > c.save.cap) {
        if (c.save.d) LMIEB_CUDA_TRY(cudaFree(c.save.d));
        c.save.d = nullptr;
        c.save.cap = 0;
        LMIEB_CUDA_TRY(cudaMalloc((void **) &c.save.d, need * sizeof(double)));
        c.save.cap = need;
        for (Slot &S : c.slot) drop_graph(S);   // a captured re-run may point at the old set
    }
    return 0;
}

// Device bytes one case needs beyond its inputs (for cutting sub-batches).
size_t case_bytes(const lmieb_problem &p) {
    long long tot = 0;
    for (int r = 0; r < p.n; ++r) tot += p.n1r[r] + 1;
    const size_t ncol = 1 + p.nd;
    size_t b = (size_t) tot * 32 * (1 + p.nd1);                        // coef
    b += (size_t) (tot / K1_B + p.n) * 8 * k1_ck_width(std::min(p.nd1, 4));   // K1 checkpoints
    b += (size_t) p.n * (64 + 8 * ncol + 40 * (1 + p.nd1));           // per-radius arrays, sums
    b += (size_t) 4 * ncol * p.n_qang * 8 * 8;                        // partials (groups), pf, pfn
    b += (size_t) ncol * 6 * p.n_coef * 8 * (3 + (p.n_qang / 2 + 31) / 32);   // expansion partials + outputs
    b += (size_t) 4 * (p.n_qang / 2) * (p.n_coef / EX_LT + 1) * 16;   // checkpoints
    if (p.precision == LMIEB_PRECISION_INT8) {
        // B operand digits (groups padded to whole chunks), row exponents
        b += (size_t) (tot + (size_t) p.n * OZ_KC) * OZ_BSTAGE / (OZ_KC * oz_rg(std::min(p.nd1, OZ_MAX_NC1)));
        b += (size_t) (p.n_qang / 2 + 1) * (tot / std::max(p.n, 1) / OZ_KC + 2) * 2;
        b += (size_t) p.n * (1 + p.nd1) * 16;                          // exponents K1 tracks
        b += (size_t) ((p.n_qang / 2 + OZ_HALF - 1) / OZ_HALF) * ((p.n1 + OZ_KC - 1) / OZ_KC) * OZ_ACHUNK;   // A operand
    }
    return b;
}

// Packs one sub-batch ps[0..n) into slot S and queues its device work and the
// download of its outputs; collect_slot() unpacks them.
int submit_sub(Slot &S, long long ticket, int ncase, const lmieb_problem *ps, lmieb_result *rs_out) {
    Ctx &c = g_ctx;
    const double t_pack = now_ms();
    S.have_plan = false;        // the slot's graph is kept while the plan repeats (below)
    Plan &L = *S.plan;
    L = Plan();
    L.side = S.side;
    L.fork = S.fork;
    L.join = S.join;
    const lmieb_problem &p0 = ps[0];
    const int nd = p0.nd, nd1 = p0.nd1, nd2 = p0.nd2, ncol = 1 + nd;
    const size_t Q = (size_t) 4 * ncol;
    L.ncase = ncase;
    L.want_gc = p0.want_gc && p0.n_qang > 0;
    L.want_lc = p0.want_lc && p0.n_qang > 0;
    L.pf_from = p0.n_angles > 0 ? p0.pf_from : 0;
    L.save_control = p0.save_control;
    L.n_qang0 = p0.n_qang;
    L.nd1c = (nd1 + 3) / 4;
    L.n_ang_launch = std::max(1, std::max((nd1 + 3) / 4, (nd2 + 3) / 4));
    L.acc_mode = p0.acc_mode;
    if (L.acc_mode != LMIEB_ACC_WHOLE && (ncase != 1 || L.save_control != 0)) {
        fprintf(stderr, "ERROR: lmie_b200: radius sharing needs a single case with save_control 0\n");
        return -1;
    }

    // ---- case table and batch-wide per-radius arrays (filled per case in parallel) ----
    std::vector<DevCase> cs(ncase);
    std::vector<int> cr0(ncase + 1, 0), cn1max(ncase, 1);
    std::vector<long long> ct0(ncase + 1, 0);      // K1 checkpoint blocks before each case
    std::vector<long long> cs1(ncase + 1, 0), cs2(ncase, 0);
    parallel_for(ncase, 16, [&](int k) {
        const lmieb_problem &p = ps[k];
        int mx = 1;
        long long a = 0, b = 0, t = 0;
        for (int i = 0; i < p.n; ++i) {
            t += (p.n1r[i] + K1_B - 1) / K1_B;
            a += p.n1r[i];
            b += p.n2r[i];
            mx = std::max(mx, p.n1r[i]);
        }
        ct0[k + 1] = t;
        cs1[k + 1] = a;
        cs2[k] = b;
        cn1max[k] = mx;
    });
    int ncmax = 1, nqmax = 0, n1max = 1;
    for (int k = 0; k < ncase; ++k) {
        cr0[k + 1] = cr0[k] + ps[k].n;
        ct0[k + 1] += ct0[k];
        cs1[k + 1] += cs1[k];
        ncmax = std::max(ncmax, ps[k].n_coef);
        nqmax = std::max(nqmax, ps[k].n_qang);
        n1max = std::max(n1max, cn1max[k]);
    }
    const int R = cr0[ncase];
    L.no_radii = R == 0 && (L.acc_mode == LMIEB_ACC_PARTIAL || L.acc_mode == LMIEB_ACC_GROUP);
    if (R == 0 && L.acc_mode == LMIEB_ACC_WHOLE) {
        fprintf(stderr, "ERROR: lmie_b200: a case without radii\n");
        return -1;
    }
    // per-radius arrays the packing reads: every element is written below;
    // kept between calls (calls are serialised) so that their pages are not
    // faulted in and zeroed again for every sub-batch (the other per-radius
    // inputs go straight into the staging buffer, below)
    static std::vector<int> n1r;
    static std::vector<long long> off, ckoff;
    n1r.resize(R);
    off.resize(R + 1);
    ckoff.resize(R + 1);
    std::vector<cplx> ml((size_t) std::max(1, ncase * nd));
    std::vector<double> laml((size_t) std::max(1, ncase * nd));
    off[0] = ckoff[0] = 0;
    parallel_for(ncase, 16, [&](int k) {
        const lmieb_problem &p = ps[k];
        DevCase &C = cs[k];
        memset(&C, 0, sizeof(C));
        C.lambda = p.lambda;
        C.m = mk(p.mr, -p.mi);
        C.minv = 1. / C.m;
        C.accuracy = p.accuracy;
        C.r0 = cr0[k];
        C.nr = p.n;
        C.o0 = cs1[k];
        C.n1 = p.n1;
        C.n_qang = p.n_qang;
        C.nh = p.n_qang / 2;
        C.n_coef = p.n_coef;
        C.n_angles = L.pf_from ? p.n_angles : 0;
        C.ml_off = k * nd;
        for (int kk = 0; kk < nd; ++kk) {
            ml[(size_t) k * nd + kk] = mk(p.mr_l[kk], -p.mi_l[kk]);
            laml[(size_t) k * nd + kk] = p.lambda_l[kk];
        }
        long long o = cs1[k];
        long long t = ct0[k];
        for (int i = 0, r = cr0[k]; i < p.n; ++i, ++r) {
            n1r[r] = p.n1r[i];
            o += n1r[r];
            off[r + 1] = o;
            t += (n1r[r] + K1_B - 1) / K1_B;
            ckoff[r + 1] = t;
        }
    });
    const long long tot = off[R], ckn = ckoff[R];
    // an FP64 re-solve whose cases' K1 outputs are in an earlier sub-batch's
    // arena: their copy, in pieces of at most GATHER_PIECE doubles (one
    // block each), replaces K1
    std::vector<GatherSeg> gsegs;
    if (c.gather.on && (int) c.gather.cs.size() == ncase && p0.precision == LMIEB_PRECISION_FP64 &&
        L.save_control == 0 && L.acc_mode == LMIEB_ACC_WHOLE) {
        constexpr long long GATHER_PIECE = 1 << 15;
        auto add_seg = [&](const double *src, int which, long long dst_off, long long n) {
            for (long long a = 0; a < n; a += GATHER_PIECE)
                gsegs.push_back(GatherSeg{src + a, dst_off + a, std::min(GATHER_PIECE, n - a), which});
        };
        const int C1 = 1 + nd1;
        for (int k = 0; k < ncase; ++k) {
            const DevCase &F = c.gather.cs[k], &T = cs[k];
            const long long no = cs1[k + 1] - cs1[k];   // the case's orders (the same radii in both)
            for (int col = 0; col < C1; ++col) {
                add_seg(c.gather.coef + ((size_t) col * c.gather.tot + F.o0) * 4, 0, ((long long) col * tot + T.o0) * 4,
                        no * 4);
                for (int q = 0; q < 5; ++q)
                    add_seg(c.gather.rs + (size_t) (col * 5 + q) * c.gather.R + F.r0, 1,
                            (long long) (col * 5 + q) * R + T.r0, T.nr);
            }
        }
    }
    // K1 launch order: cases by their largest n1, largest first, each from its
    // largest radius down, so that the longest recurrences start first
    std::vector<int> k1ord(ncase);
    std::vector<long long> k1pre(ncase + 1, 0);
    for (int k = 0; k < ncase; ++k) k1ord[k] = k;
    std::stable_sort(k1ord.begin(), k1ord.end(), [&](int a, int b) { return cn1max[a] > cn1max[b]; });
    for (int k = 0; k < ncase; ++k) k1pre[k + 1] = k1pre[k] + ps[k1ord[k]].n;

    // ---- order tables ----
    std::vector<double> fv((size_t) 4 * (n1max + 2), 0.);
    for (int i = 1; i <= n1max + 1; ++i) {
        const double f1 = 2. * i + 1., f2 = (i + 1.) / i;
        fv[i] = f1;
        fv[(size_t) (n1max + 2) + i] = f2;
        fv[(size_t) 2 * (n1max + 2) + i] = (i + 2.) / f2;
        fv[(size_t) 3 * (n1max + 2) + i] = f1 / (i * (i + 1.));
    }
    fv[0] = 1.;
    std::vector<double> rc((size_t) 8 * ncmax, 0.);
    for (int l = 3; l < ncmax; ++l) {
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
    if (ncmax > 2) rc[(size_t) 8 * 2 + 1] = 1. / 2.;   // Legendre at l = 2

    // ---- Gauss angles: pool entries, new orders computed on the device ----
    std::vector<int> gl_ns, gl_pt, gl_pi;
    std::vector<long long> gl_mo, gl_go;
    std::vector<double> gl_guess, gl_jr((size_t) std::max(nqmax, 1), 0.);
    for (int j = 0; j < nqmax; ++j) gl_jr[j] = j / (j + 1.);
    {
        size_t need = c.gl_used;
        std::unordered_map<int, long long> fresh;   // entries this batch adds
        for (int k = 0; k < ncase; ++k) {
            const int nq = cs[k].n_qang;
            if (nq <= 0) continue;
            long long at = -1;
            const auto hit = c.gl_map.find(nq);
            if (hit != c.gl_map.end()) at = hit->second;
            const auto hit2 = fresh.find(nq);
            if (hit2 != fresh.end()) at = hit2->second;
            if (at < 0) {
                at = (long long) need;
                fresh[nq] = at;
                need += 2 * (size_t) nq;
                const int ia = 4 * nq + 2, half = (nq + 1) / 2;
                const double da = (nq - 1) / (8. * pow((double) nq, 3));
                gl_ns.push_back(nq);
                gl_mo.push_back(at);
                gl_go.push_back((long long) gl_guess.size());
                for (int i = 0; i < half; ++i) {
                    const double th = (4. * i + 3.) / ia * LMIEB_PI;
                    gl_guess.push_back(cos(th + da / tan(th)));
                    gl_pt.push_back((int) gl_ns.size() - 1);
                    gl_pi.push_back(i);
                }
            }
            cs[k].mu_off = at;
        }
        if (ensure_gl_pool(need)) return -1;
        for (size_t t = 0; t < gl_ns.size(); ++t) c.gl_map[gl_ns[t]] = gl_mo[t];
        c.gl_used = need;
    }

    // ---- angular work items (largest first), partial and pf offsets ----
    bool any_ang = false;
    for (int k = 0; k < ncase; ++k) any_ang |= cs[k].n_qang > 0;
    L.tc = p0.precision == LMIEB_PRECISION_TF32X3 && L.save_control == 0 && any_ang && R > 0 &&
           nd1 <= TC_MAX_NC1 && nd2 <= TC_MAX_ND2;
    L.tc_seg = g_tc_seg;
    L.oz = p0.precision == LMIEB_PRECISION_INT8 && L.save_control == 0 && any_ang && R > 0 &&
           nd1 <= OZ_MAX_NC1 && nd2 <= OZ_MAX_ND2;
    // with split precision, cases below TC_MIN_N1 orders keep the FP64 K3: their
    // linearised phase matrices cancel strongly on normalisation, and they cost little
    std::vector<char> case_tc(ncase, 0), case_oz(ncase, 0);
    for (int k = 0; k < ncase; ++k) case_tc[k] = L.tc && cs[k].n_qang > 0 && cs[k].n1 >= TC_MIN_N1;
    // the int8 stage takes the cases of at least OZ_MIN_N1 orders whose radius
    // groups fit its exact int32 sums (OZ_MAX_NK chunks)
    for (int k = 0; k < ncase; ++k)
        case_oz[k] = L.oz && cs[k].n_qang > 0 && cs[k].n1 >= OZ_MIN_N1 &&
                     (cn1max[k] + OZ_KC - 1) / OZ_KC <= OZ_MAX_NK;
    std::vector<AngItem> ang, ang64;
    std::vector<long long> pf_start(ncase + 1, 0);
    for (int k = 0; k < ncase; ++k) {
        pf_start[k + 1] = pf_start[k] + (long long) Q * cs[k].n_qang;
        cs[k].pf_off = pf_start[k];
        cs[k].G = 0;
    }
    L.pf_total = pf_start[ncase];
    long long part_total = 0;
    // Items go out largest first, so that the long ones do not end the stage
    // alone.  The order only schedules the work (every item writes its own
    // partial-sum slot, reduced in group order), so cost classes of 2^(1/4)
    // are enough: a counting sort, stable within a class.
    auto largest_first = [](const std::vector<std::pair<double, AngItem>> &tmp, std::vector<AngItem> &out) {
        constexpr int NB = 256;
        static std::vector<unsigned char> cls;
        cls.resize(tmp.size());
        size_t cnt[NB] = {};
        for (size_t i = 0; i < tmp.size(); ++i) {
            const double c = tmp[i].first;
            int b = 0;
            if (c > 1.) {
                int ex;
                const double m = frexp(c, &ex);              // c = m 2^ex, m in [0.5, 1)
                b = std::min(NB - 1, 4 * ex + (int) ((m - .5) * 8.));
            }
            cls[i] = (unsigned char) (NB - 1 - b);           // largest class first
            ++cnt[cls[i]];
        }
        size_t at[NB], run = out.size();
        for (int b = 0; b < NB; ++b) { at[b] = run; run += cnt[b]; }
        out.resize(run);
        for (size_t i = 0; i < tmp.size(); ++i) out[at[cls[i]]++] = tmp[i].second;
    };
    // coefficient offsets of the radii whose coefficients K1 writes in FP64
    // (all radii: the order offsets `off`; with split precision those of the
    // FP64 cases)
    static std::vector<long long> coff_tc;
    if (L.tc) {
        coff_tc.resize(R + 1);
        coff_tc[0] = 0;
        for (int k = 0; k < ncase; ++k) {
            const DevCase &C = cs[k];
            for (int r = C.r0; r < C.r0 + C.nr; ++r) coff_tc[r + 1] = coff_tc[r] + (case_tc[k] ? 0 : n1r[r]);
        }
    }
    const std::vector<long long> &coff = L.tc ? coff_tc : off;
    // split precision: radius groups of tc_rg(nd1) radii, each with its B operand block
    static std::vector<int> tc_pos;
    static std::vector<long long> tc_roff;
    std::vector<int> tg_r0, tg_n, tg_nk;
    std::vector<long long> tg_off;
    tc_pos.clear();
    tc_roff.clear();
    long long bop_floats = 0;
    if (L.tc) {
        const int RG = tc_rg(nd1);
        tc_pos.assign(R, -1);
        tc_roff.assign(R, 0);
        std::vector<int> cg0(ncase + 1, 0);
        std::vector<double> wc(ncase, 0.);
        double W = 0.;
        for (int k = 0; k < ncase; ++k) {
            const DevCase &C = cs[k];
            cg0[k] = (int) tg_r0.size();
            if (!case_tc[k]) continue;
            for (int r = C.r0; r < C.r0 + C.nr; r += RG) {
                const int n = std::min(RG, C.r0 + C.nr - r);
                int mx = 1;
                for (int i = 0; i < n; ++i) mx = std::max(mx, n1r[r + i]);
                const int nk = (mx + TC_KC - 1) / TC_KC;
                for (int i = 0; i < n; ++i) {
                    tc_pos[r + i] = i + 256 * nk;
                    tc_roff[r + i] = bop_floats;
                }
                tg_r0.push_back(r);
                tg_n.push_back(n);
                tg_nk.push_back(nk);
                tg_off.push_back(bop_floats);
                bop_floats += (long long) nk * (TC_BSTAGE / 4);
                wc[k] += nk + 1;                       // chunks, plus one for the group's epilogue
            }
            W += wc[k] * ((C.nh + TC_HALF - 1) / TC_HALF);
        }
        cg0[ncase] = (int) tg_r0.size();
        const double wt = std::max(W / (g_items_per_sm[1] * c.sms), 8.);    // chunks per item
        std::vector<std::pair<double, AngItem>> tmp;
        for (int k = 0; k < ncase; ++k) {
            DevCase &C = cs[k];
            if (!case_tc[k]) continue;
            const int ng = cg0[k + 1] - cg0[k];
            const int xt = (C.nh + TC_HALF - 1) / TC_HALF;
            int G = (int) std::lround(wc[k] / wt);
            G = std::max(1, std::min(G, ng));
            std::vector<int> gs(G + 1, cg0[k + 1]);
            gs[0] = cg0[k];
            double run = 0.;
            int gi = 1;
            for (int g = cg0[k]; g < cg0[k + 1] && gi < G; ++g) {
                run += tg_nk[g] + 1;
                if (run * G >= wc[k] * gi) gs[gi++] = g + 1;
            }
            for (int g = 1; g <= G; ++g) gs[g] = std::max(gs[g], gs[g - 1]);
            gs.erase(std::unique(gs.begin(), gs.end()), gs.end());   // every partial slot gets a range
            G = (int) gs.size() - 1;
            C.G = G;
            C.part_off = part_total;
            part_total += (long long) G * Q * C.n_qang;
            for (int g = 0; g < G; ++g) {
                double cost = 0.;
                for (int gg = gs[g]; gg < gs[g + 1]; ++gg) cost += tg_nk[gg] + 1;
                for (int t = 0; t < xt; ++t) tmp.push_back({cost, AngItem{k, t, g, gs[g], gs[g + 1]}});
            }
        }
        largest_first(tmp, ang);
    }
    // int8 fixed point: radius groups of oz_rg(nd1) radii, each with its B
    // operand digits; row-exponent tables per case
    long long bop8_bytes = 0, rx_bytes = 0, aop_bytes = 0;
    int nkx_all = 0;
    std::vector<long long> rx_start(ncase + 1, 0), a_start(ncase + 1, 0);
    if (L.oz) {
        const int RG = oz_rg(nd1);
        std::vector<int> cg0(ncase + 1, 0);
        std::vector<long long> cb0(ncase + 1, 0);     // B operand chunks before each case
        std::vector<double> wc(ncase, 0.);
        // per case, in parallel: its groups of RG radii and their chunks
        parallel_for(ncase, 64, [&](int k) {
            const DevCase &C = cs[k];
            if (!case_oz[k]) return;
            long long ch = 0;
            for (int r = C.r0; r < C.r0 + C.nr; r += RG) {
                const int n = std::min(RG, C.r0 + C.nr - r);
                int mx = 1;
                for (int i = 0; i < n; ++i) mx = std::max(mx, n1r[r + i]);
                ch += (mx + OZ_KC - 1) / OZ_KC;
            }
            cg0[k + 1] = (C.nr + RG - 1) / RG;
            cb0[k + 1] = ch;
            wc[k] = (double) (ch + cg0[k + 1]);       // chunks, plus one per group for its epilogue
        });
        for (int k = 0; k < ncase; ++k) {
            cg0[k + 1] += cg0[k];
            cb0[k + 1] += cb0[k];
        }
        tg_r0.resize(cg0[ncase]);
        tg_n.resize(cg0[ncase]);
        tg_nk.resize(cg0[ncase]);
        tg_off.resize(cg0[ncase]);
        parallel_for(ncase, 64, [&](int k) {
            const DevCase &C = cs[k];
            if (!case_oz[k]) return;
            int g = cg0[k];
            long long o = cb0[k] * OZ_BSTAGE;
            for (int r = C.r0; r < C.r0 + C.nr; r += RG, ++g) {
                const int n = std::min(RG, C.r0 + C.nr - r);
                int mx = 1;
                for (int i = 0; i < n; ++i) mx = std::max(mx, n1r[r + i]);
                const int nk = (mx + OZ_KC - 1) / OZ_KC;
                tg_r0[g] = r;
                tg_n[g] = n;
                tg_nk[g] = nk;
                tg_off[g] = o;
                o += (long long) nk * OZ_BSTAGE;
            }
        });
        bop8_bytes = cb0[ncase] * OZ_BSTAGE;
        double W = 0.;
        for (int k = 0; k < ncase; ++k) {
            DevCase &C = cs[k];
            rx_start[k + 1] = rx_start[k];
            a_start[k + 1] = a_start[k];
            if (!case_oz[k]) continue;
            C.nkx = (cn1max[k] + OZ_KC - 1) / OZ_KC;
            C.rx_off = rx_bytes;
            C.trunc_band = C.accuracy > 0. ? oz_trunc_band(cn1max[k]) : 0.;
            rx_bytes += (long long) C.nh * C.nkx * 2;
            rx_start[k + 1] += C.nh;
            // the A operand of each angle tile and chunk
            const int ntile = (C.nh + OZ_HALF - 1) / OZ_HALF;
            C.a_off = aop_bytes;
            aop_bytes += (long long) ntile * C.nkx * OZ_ACHUNK;
            a_start[k + 1] += (long long) ntile * OZ_M;
            nkx_all = std::max(nkx_all, C.nkx);
            W += wc[k] * ((C.nh + OZ_HALF - 1) / OZ_HALF);
        }
        L.n_groups = (int) tg_r0.size();
        L.n_rx = rx_start[ncase];
        L.n_arow = a_start[ncase];
        const double wt = std::max(W / (g_items_per_sm[2] * c.sms), 8.);    // chunks per item
        std::vector<std::pair<double, AngItem>> tmp;
        for (int k = 0; k < ncase; ++k) {
            DevCase &C = cs[k];
            if (!case_oz[k]) continue;
            const int ng = cg0[k + 1] - cg0[k];
            const int xt = (C.nh + OZ_HALF - 1) / OZ_HALF;
            int G = (int) std::lround(wc[k] / wt);
            G = std::max(1, std::min(G, ng));
            std::vector<int> gs(G + 1, cg0[k + 1]);
            gs[0] = cg0[k];
            double run = 0.;
            int gi = 1;
            for (int g = cg0[k]; g < cg0[k + 1] && gi < G; ++g) {
                run += tg_nk[g] + 1;
                if (run * G >= wc[k] * gi) gs[gi++] = g + 1;
            }
            for (int g = 1; g <= G; ++g) gs[g] = std::max(gs[g], gs[g - 1]);
            gs.erase(std::unique(gs.begin(), gs.end()), gs.end());   // every partial slot gets a range
            G = (int) gs.size() - 1;
            C.G = G;
            C.part_off = part_total;
            part_total += (long long) G * Q * C.n_qang;
            for (int g = 0; g < G; ++g) {
                double cost = 0.;
                for (int gg = gs[g]; gg < gs[g + 1]; ++gg) cost += tg_nk[gg] + 1;
                for (int t = 0; t < xt; ++t) tmp.push_back({cost, AngItem{k, t, g, gs[g], gs[g + 1]}});
            }
        }
        largest_first(tmp, ang);
    }
    std::vector<double> oz_f2;
    if (L.oz) {
        oz_f2.assign((size_t) OZ_KC * nkx_all + 2, 0.);
        for (size_t k = 1; k < oz_f2.size(); ++k) oz_f2[k] = (k + 1.) / (double) k;
    }
    {
        // FP64 K3 over the remaining cases: radius ranges of roughly equal sum of n1
        const int per = angular_angles_per_block(std::min(nd1, 4));
        double W = 0.;
        std::vector<double> wc(ncase, 0.);
        for (int k = 0; k < ncase; ++k) {
            if (cs[k].n_qang <= 0 || case_tc[k] || case_oz[k]) continue;
            wc[k] = (double) (cs1[k + 1] - cs1[k]) * cs[k].nh;
            W += wc[k];
        }
        // work per block; in a tensor-core batch these are the cases under 16
        // orders (a few half-angles, up to ~2000 radii each), whose blocks
        // would otherwise walk all their radii one after the other
        const double wt = std::max(W / (g_items_per_sm[0] * c.sms), (L.tc || L.oz) ? 4096. : 64. * 2 * 64 * 16);
        std::vector<std::pair<double, AngItem>> tmp;
        for (int k = 0; k < ncase; ++k) {
            DevCase &C = cs[k];
            if (C.n_qang <= 0 || case_tc[k] || case_oz[k]) continue;
            const int xt = (C.nh + per - 1) / per;
            int G = (int) std::lround(wc[k] / (xt * wt));
            G = std::max(1, std::min(G, (L.tc || L.oz) ? std::min(C.nr, 64) : C.nr));
            std::vector<int> gs(G + 1, C.r0 + C.nr);
            gs[0] = C.r0;
            const long long o0 = off[C.r0], ot = off[C.r0 + C.nr] - o0;
            int gi = 1;
            for (int r = C.r0; r < C.r0 + C.nr && gi < G; ++r)
                if ((double) (off[r + 1] - o0) * G >= (double) ot * gi) gs[gi++] = r + 1;
            for (int g = 1; g <= G; ++g) gs[g] = std::max(gs[g], gs[g - 1]);
            C.G = G;
            C.part_off = part_total;
            part_total += (long long) G * Q * C.n_qang;
            for (int g = 0; g < G; ++g)
                for (int t = 0; t < xt; ++t) {
                    AngItem it{k, t, g, gs[g], gs[g + 1]};
                    const double cost = (double) (off[gs[g + 1]] - off[gs[g]]) * std::min(per, C.nh - t * per);
                    tmp.push_back({cost, it});
                }
        }
        largest_first(tmp, (L.tc || L.oz) ? ang64 : ang);
    }
    L.n_ang = (int) ang.size();
    L.n_ang64 = (int) ang64.size();
    const long long ctot = coff[R];

    // ---- expansion work items and offsets ----
    static std::vector<ExpItem> ex;          // kept between calls, like the per-radius arrays
    std::vector<long long> ck_gc(ncase + 1, 0), ck_lc(ncase + 1, 0), fin_start(ncase + 1, 0);
    std::vector<long long> exb(ncase + 1, 0);           // first item of each case
    long long ck_total = 0, ex_total = 0;
    auto ex_tiles = [&](const DevCase &C, int &nlt, int &nat) {
        const bool on = (L.want_gc || L.want_lc) && C.n_qang > 0;
        nlt = on ? (C.n_coef + EX_LT - 1) / EX_LT : 0;
        nat = on ? (C.nh + EX_AT - 1) / EX_AT : 0;
        return on;
    };
    for (int k = 0; k < ncase; ++k) {
        DevCase &C = cs[k];
        int nlt, nat;
        const bool on = ex_tiles(C, nlt, nat);
        ck_gc[k + 1] = ck_gc[k] + (on ? 4LL * C.nh : 0);
        ck_lc[k + 1] = ck_lc[k] + (on ? 1LL * C.nh : 0);
        fin_start[k + 1] = fin_start[k] + (on ? (long long) ncol * C.n_coef : 0);
        C.ck_off = ck_total;
        ck_total += (long long) nlt * 4 * C.nh * 2;
        C.ex_off = ex_total;
        ex_total += (long long) nat * ncol * 6 * C.n_coef;
        exb[k + 1] = exb[k] + (long long) nlt * nat;
    }
    ex.resize((size_t) exb[ncase]);
    parallel_for(ncase, 16, [&](int k) {
        int nlt, nat;
        ex_tiles(cs[k], nlt, nat);
        ExpItem *e = ex.data() + exb[k];
        for (int lt = 0; lt < nlt; ++lt)
            for (int at = 0; at < nat; ++at) *e++ = ExpItem{k, lt, at};
    });
    // the GSF expansion runs one block per (case, angle tile) over all the
    // case's orders: cases with the most orders first
    static std::vector<ExpItem> gx;
    gx.clear();
    if (L.want_gc) {
        std::vector<int> byn(ncase);
        for (int k = 0; k < ncase; ++k) byn[k] = k;
        std::stable_sort(byn.begin(), byn.end(), [&](int a, int b) { return cs[a].n_coef > cs[b].n_coef; });
        for (int k : byn) {
            int nlt, nat;
            if (!ex_tiles(cs[k], nlt, nat) || nlt == 0) continue;
            for (int at = 0; at < nat; ++at) gx.push_back(ExpItem{k, 0, at});
        }
    }
    L.nck_gc = ck_gc[ncase];
    L.nck_lc = ck_lc[ncase];
    L.nfin = fin_start[ncase];
    L.n_ex = (int) ex.size();
    L.n_gx = (int) gx.size();

    // ---- user angles and output offsets ----
    // the user angles depend only on their number: one copy per distinct count
    std::vector<long long> pu_start(ncase + 1, 0), pu_red(ncase + 1, 0);
    long long pu_scr_total = 0;
    std::vector<double> mu_user;
    std::unordered_map<int, long long> mu_at;
    size_t o_scal = 0, o_gc = 0, o_lc = 0, o_pf = 0;
    for (int k = 0; k < ncase; ++k) {
        DevCase &C = cs[k];
        if (C.n_angles > 0) {
            const auto hit = mu_at.find(C.n_angles);
            if (hit != mu_at.end()) {
                C.mu_user_off = hit->second;
            } else {
                C.mu_user_off = (long long) mu_user.size();
                mu_at[C.n_angles] = C.mu_user_off;
                mu_user.insert(mu_user.end(), ps[k].mu_user, ps[k].mu_user + C.n_angles);
            }
        }
        // K5: parts of PU_LP orders; the partial sums of a case of several
        C.pu_parts = (L.pf_from && C.n_angles > 0) ? std::max(1, (C.n_coef + g_pu_lp - 1) / g_pu_lp) : 0;
        C.pu_scr_off = pu_scr_total;
        const long long pu_n = (long long) ncol * 6 * C.n_angles;
        if (C.pu_parts > 1) pu_scr_total += C.pu_parts * pu_n;
        pu_red[k + 1] = pu_red[k] + (C.pu_parts > 1 ? pu_n : 0);
        C.scal_off = (int) o_scal;
        o_scal += (size_t) ncol * 4;
        C.gc_off = (long long) o_gc;
        if (L.want_gc) o_gc += (size_t) ncol * 6 * C.n_coef;
        C.lc_off = (long long) o_lc;
        if (L.want_lc) o_lc += (size_t) ncol * 6 * C.n_coef;
        C.pf_out_off = (long long) o_pf;
        o_pf += (size_t) ncol * 6 * C.n_angles;
    }
    // K5 blocks (all columns per block), cases in K1's launch order: the most
    // orders first
    for (int kr = 0; kr < ncase; ++kr) {
        const DevCase &C = cs[k1ord[kr]];
        pu_start[kr + 1] = pu_start[kr] + (long long) ((C.n_angles + PU_T - 1) / PU_T) * C.pu_parts;
    }
    L.pu_total = pu_start[ncase];
    L.pu_nred = pu_red[ncase];

    // ---- launches per device run and algorithmic work ----
    {
        long long nl = 0;
        const bool solve = L.acc_mode != LMIEB_ACC_FINISH && !L.no_radii;
        const bool finish = L.acc_mode != LMIEB_ACC_PARTIAL;
        if (!solve) {
            // integrals uploaded (or zero on an empty share)
        } else if (L.save_control != 2) {
            nl += (gsegs.empty() ? (long long) std::max(L.nd1c, 1) : 1) + 1;   // K1 per chunk (or its copy), K2
            if (L.tc) nl += (L.n_ang > 0) + (L.n_ang64 > 0 ? L.n_ang_launch : 0);   // K3
            else if (L.oz) nl += (L.n_ang > 0 ? 4 : 0) + (L.n_ang64 > 0 ? L.n_ang_launch : 0);   // row exponents, A, B, K3
            else nl += L.n_ang > 0 ? L.n_ang_launch : 0;
            if (L.n_ang > 0 || L.n_ang64 > 0) nl += 1;                          // group reduction
        } else {
            nl += 1 + (L.n_qang0 > 0);
        }
        if (finish) {
            nl += 1 + (L.pf_total > 0);                                          // normalisation
            if (L.want_gc && L.n_ex > 0) nl += 1 + expand_gsf_launches(ncol);
            if (L.want_lc && L.n_ex > 0) nl += 3;
            if (L.pf_from && L.pu_total > 0) nl += 1 + (L.pu_nred > 0);
        }
        L.launches = nl;
        double fang = 0., frec = 0., fgsf = 0., fexp = 0.;
        for (int k = 0; k < ncase; ++k) {
            const DevCase &C = cs[k];
            const double s1 = (double) (cs1[k + 1] - cs1[k]), s2 = (double) cs2[k];
            fang += 8. * C.n_qang * s1 * (1. + nd1);
            frec += (14. * s2 + 93. * s1) + nd1 * (16. * s2 + 154. * s1);
            fgsf += 12. * C.n_coef * C.n_qang * ncol * ((L.want_gc ? 1 : 0) + (L.want_lc ? 1 : 0));
            fexp += 12. * C.n_angles * C.n_coef * ncol;
        }
        if (L.save_control == 2 || !solve) fang = frec = 0.;
        if (!finish) fgsf = fexp = 0.;
        c.work[0] += fang;
        if (L.oz) {
            // OZ_NPROD products of M x N x K per chunk of every (angle tile, group) pair
            double chunks = 0.;
            for (const AngItem &a : ang)
                for (int gg = a.rbeg; gg < a.rend; ++gg) chunks += tg_nk[gg];
            c.tensor_ops += 2. * OZ_NPROD * (double) OZ_M * OZ_NP * OZ_KC * chunks;
        }
        c.work[1] += frec;
        c.work[2] += fgsf;
        c.work[3] += fexp;
        c.launches += nl + (gl_pt.empty() ? 0 : 1);
    }

    // ---- host staging: inputs then outputs ----
    L.acc_n = (size_t) ncase * ncol * 4 + (size_t) L.pf_total;   // sums, then pfacc
    const size_t n_save2 = (size_t) 4 * R * std::max(L.n_qang0, 1);
    // save_control 2: the caller's kernels, unless the device still holds them
    const int save_nq = p0.save2_rows ? L.n_qang0 : 0;
    auto save_row = [&](int i) -> const double * {
        return i < 4 ? p0.save1_rows[i] : p0.save2_rows[(i - 4) / R][(i - 4) % R];
    };
    bool save_hit = false;
    unsigned long long save_key = 0;
    if (L.save_control == 2) {
        save_key = save_hash(R, save_nq, save_row);
        save_hit = c.save.valid && c.save.key == save_key && c.save.R == R && c.save.nq == save_nq &&
                   c.save.cap >= (size_t) 4 * R + n_save2;
        ++(save_hit ? c.save.hits : c.save.misses);
    }
    size_t in_bytes = 0;
    {
        auto add = [&](size_t b) { in_bytes += pad(b); };
        add(cs.size() * sizeof(DevCase)); add((size_t) R * 8); add((size_t) std::max(nd1, 1) * R * 8);
        add((size_t) ncol * R * 8);
        add((size_t) R * 4); add((size_t) R * 4); add((size_t) R * 4);
        add((size_t) (R + 1) * 8); add((size_t) (R + 1) * 8);
        add(fv.size() * 8); add(rc.size() * 8); add(ml.size() * 16); add(laml.size() * 8);
        add((size_t) nd1 * 4); add((size_t) nd2 * 4); add(mu_user.size() * 8);
        add(ang.size() * sizeof(AngItem)); add(ang64.size() * sizeof(AngItem)); add(ex.size() * sizeof(ExpItem));
        add(gx.size() * sizeof(ExpItem));
        add(gsegs.size() * sizeof(GatherSeg));
        add(tc_pos.size() * 4); add(tc_roff.size() * 8); add(tg_r0.size() * 4); add(tg_n.size() * 4);
        add(tg_nk.size() * 4); add(tg_off.size() * 8); add(oz_f2.size() * 8); add(rx_start.size() * 8);
        add(a_start.size() * 8);
        for (int q = 0; q < 6; ++q) add((size_t) (ncase + 1) * 8);   // prefix arrays over the cases
        add((size_t) ncase * 4); add((size_t) (ncase + 1) * 8);             // K1 launch order
        add(gl_ns.size() * 4); add(gl_mo.size() * 8); add(gl_go.size() * 8); add(gl_pt.size() * 4);
        add(gl_pi.size() * 4); add(gl_guess.size() * 8); add(gl_jr.size() * 8);
        if (L.save_control == 2) {
            if (!save_hit) { add((size_t) 4 * R * 8); add(n_save2 * 8); }
            add((size_t) std::max(nd, 1) * R * 8);
        }
        if (L.acc_mode == LMIEB_ACC_FINISH) add((size_t) L.acc_n * 8);
    }
    size_t out_bytes = 0;
    {
        auto add = [&](size_t b) { out_bytes += pad(b); };
        add(o_scal * 8); add(o_gc * 8); add(o_lc * 8); add(o_pf * 8); add((size_t) (6 * ncase + 1) * 4);
        if (L.save_control == 1) { add((size_t) 4 * R * 8); add(n_save2 * 8); }
        if (L.acc_mode == LMIEB_ACC_PARTIAL) add(L.acc_n * 8);
    }
    if (ensure_host(S, in_bytes + out_bytes)) return -1;
    char *hp = S.hbuf;
    size_t ho = 0;
    DevCase *h_cs = put(hp, ho, cs.data(), cs.size());
    // the per-radius inputs go straight from the cases into the staging
    // buffer (one pass over them, on one thread per core)
    double *h_x = put(hp, ho, (const double *) nullptr, (size_t) R);
    double *h_xl = put(hp, ho, (const double *) nullptr, (size_t) std::max(nd1, 1) * R);
    double *h_w = put(hp, ho, (const double *) nullptr, (size_t) ncol * R);
    int *h_n1r = put(hp, ho, n1r.data(), (size_t) R);
    int *h_n2r = put(hp, ho, (const int *) nullptr, (size_t) R);
    int *h_rcase = put(hp, ho, (const int *) nullptr, (size_t) R);
    parallel_for(ncase, 16, [&](int k) {
        const lmieb_problem &p = ps[k];
        const int r0 = cr0[k];
        memcpy(h_x + r0, p.x, (size_t) p.n * 8);
        for (int q = 0; q < nd1; ++q) memcpy(h_xl + (size_t) q * R + r0, p.xl + (size_t) q * p.n, (size_t) p.n * 8);
        for (int q = 0; q < ncol; ++q) memcpy(h_w + (size_t) q * R + r0, p.w + (size_t) q * p.n, (size_t) p.n * 8);
        memcpy(h_n2r + r0, p.n2r, (size_t) p.n * 4);
        for (int i = 0; i < p.n; ++i) h_rcase[r0 + i] = k;
    }, host_cores());
    int *h_k1ord = put(hp, ho, k1ord.data(), (size_t) ncase);
    long long *h_k1pre = put(hp, ho, k1pre.data(), (size_t) ncase + 1);
    long long *h_off = put(hp, ho, coff.data(), (size_t) R + 1);
    long long *h_ckoff = put(hp, ho, ckoff.data(), (size_t) R + 1);
    double *h_fv = put(hp, ho, fv.data(), fv.size());
    double *h_rc = put(hp, ho, rc.data(), rc.size());
    cplx *h_ml = put(hp, ho, ml.data(), ml.size());
    double *h_laml = put(hp, ho, laml.data(), laml.size());
    int *h_i1 = put(hp, ho, p0.idx1, (size_t) nd1);
    int *h_i2 = put(hp, ho, p0.idx2, (size_t) nd2);
    double *h_mu = put(hp, ho, mu_user.data(), mu_user.size());
    AngItem *h_ang = put(hp, ho, ang.data(), ang.size());
    AngItem *h_ang64 = put(hp, ho, ang64.data(), ang64.size());
    ExpItem *h_ex = put(hp, ho, ex.data(), ex.size());
    ExpItem *h_gx = put(hp, ho, gx.data(), gx.size());
    GatherSeg *h_gs = put(hp, ho, gsegs.data(), gsegs.size());
    int *h_tcpos = put(hp, ho, tc_pos.data(), tc_pos.size());
    long long *h_tcroff = put(hp, ho, tc_roff.data(), tc_roff.size());
    int *h_tgr0 = put(hp, ho, tg_r0.data(), tg_r0.size());
    int *h_tgn = put(hp, ho, tg_n.data(), tg_n.size());
    int *h_tgnk = put(hp, ho, tg_nk.data(), tg_nk.size());
    long long *h_tgoff = put(hp, ho, tg_off.data(), tg_off.size());
    double *h_ozf2 = put(hp, ho, oz_f2.data(), oz_f2.size());
    long long *h_rxs = put(hp, ho, rx_start.data(), rx_start.size());
    long long *h_axs = put(hp, ho, a_start.data(), a_start.size());
    long long *h_pfs = put(hp, ho, pf_start.data(), pf_start.size());
    long long *h_ckg = put(hp, ho, ck_gc.data(), ck_gc.size());
    long long *h_ckl = put(hp, ho, ck_lc.data(), ck_lc.size());
    long long *h_fin = put(hp, ho, fin_start.data(), fin_start.size());
    long long *h_pus = put(hp, ho, pu_start.data(), pu_start.size());
    long long *h_pur = put(hp, ho, pu_red.data(), pu_red.size());
    int *h_gns = put(hp, ho, gl_ns.data(), gl_ns.size());
    long long *h_gmo = put(hp, ho, gl_mo.data(), gl_mo.size());
    long long *h_ggo = put(hp, ho, gl_go.data(), gl_go.size());
    int *h_gpt = put(hp, ho, gl_pt.data(), gl_pt.size());
    int *h_gpi = put(hp, ho, gl_pi.data(), gl_pi.size());
    double *h_gguess = put(hp, ho, gl_guess.data(), gl_guess.size());
    double *h_gjr = put(hp, ho, gl_jr.data(), gl_jr.size());
    double *h_s1 = nullptr, *h_s2 = nullptr, *h_w2 = nullptr;
    if (L.save_control == 2) {
        if (!save_hit) {
            // gathered through the caller's row pointers
            h_s1 = put(hp, ho, (const double *) nullptr, (size_t) 4 * R);
            h_s2 = put(hp, ho, (const double *) nullptr, n_save2);
            const int nrows = 4 + (save_nq > 0 ? 4 * R : 0);
            parallel_for(nrows, 64, [&](int i) {
                if (i < 4) memcpy(h_s1 + (size_t) i * R, save_row(i), (size_t) R * 8);
                else memcpy(h_s2 + (size_t) (i - 4) * save_nq, save_row(i), (size_t) save_nq * 8);
            });
            if (save_nq == 0) memset(h_s2, 0, n_save2 * 8);
        }
        h_w2 = put(hp, ho, p0.w2, (size_t) std::max(nd, 1) * R);
    }
    double *h_acc = nullptr;
    if (L.acc_mode == LMIEB_ACC_FINISH) h_acc = put(hp, ho, p0.acc_in, L.acc_n);
    const size_t h_in_end = ho;
    if (h_in_end > in_bytes) {
        fprintf(stderr, "ERROR: lmie_b200: staging layout mismatch\n");
        return -1;
    }
    char *h_out = hp + h_in_end;

    // ---- device arena ----
    size_t dev_bytes = in_bytes + out_bytes + 64 * 256;
    {
        auto add = [&](size_t b) { dev_bytes += pad(b); };
        if (L.save_control != 2 && L.acc_mode != LMIEB_ACC_FINISH) {
            add((size_t) ckn * 8 * k1_ck_width(std::min(nd1, 4)));
            if (L.tc) add((size_t) bop_floats * 4);
            if (L.oz) {
                add((size_t) bop8_bytes);
                add((size_t) rx_bytes);
                add((size_t) L.n_groups * OZ_NP * 4);
                add((size_t) (1 + nd1) * R * 16);
                add((size_t) aop_bytes);
            }
            add((size_t) (1 + nd1) * (size_t) ctot * 32);
            add((size_t) (1 + nd1) * 5 * (size_t) R * 8);
            add((size_t) part_total * 8);
        }
        add((L.acc_n + 1) * 8);                                  // sums + pfacc + the group's failure count
        add((size_t) L.pf_total * 8);
        add((size_t) ck_total * 8);
        add((size_t) ex_total * 8);
        add((size_t) pu_scr_total * 8);
    }
    if (ensure_device(S, dev_bytes)) return -1;
    Arena A{S.dbuf, 0, S.dcap};
    char *d_in = A.take<char>(h_in_end);
    char *d_out = A.take<char>(out_bytes);
    if (!d_in || !d_out) {
        fprintf(stderr, "ERROR: lmie_b200: device arena too small\n");
        return -1;
    }
    auto dptr = [&](void *h) { return d_in + ((char *) h - hp); };

    DevBatch &B = L.B;
    memset(&B, 0, sizeof(B));
    B.ncase = ncase;
    B.R = R;
    B.nd = nd; B.nd1 = nd1; B.nd2 = nd2;
    B.n1max = n1max; B.ncmax = ncmax;
    B.pu_lp = g_pu_lp;
    B.cs = (const DevCase *) dptr(h_cs);
    B.idx1 = (const int *) dptr(h_i1);
    B.idx2 = (const int *) dptr(h_i2);
    B.m_l = (const cplx *) dptr(h_ml);
    B.lambda_l = (const double *) dptr(h_laml);
    B.rcase = (const int *) dptr(h_rcase);
    B.k1ord = (const int *) dptr(h_k1ord);
    B.k1pre = (const long long *) dptr(h_k1pre);
    B.x = (const double *) dptr(h_x);
    B.xl = (const double *) dptr(h_xl);
    B.w = (const double *) dptr(h_w);
    B.n1r = (const int *) dptr(h_n1r);
    B.n2r = (const int *) dptr(h_n2r);
    B.off = (const long long *) dptr(h_off);
    B.ckoff = (const long long *) dptr(h_ckoff);
    B.tot = ctot;
    B.ckn = ckn;
    B.fv = (const double *) dptr(h_fv);
    B.rc = (const double *) dptr(h_rc);
    B.mu_pool = c.gl_pool;
    B.mu_user = (const double *) dptr(h_mu);
    if (L.tc || L.oz) {
        B.tc_pos = L.tc ? (const int *) dptr(h_tcpos) : nullptr;
        B.tc_roff = L.tc ? (const long long *) dptr(h_tcroff) : nullptr;
        B.tg_r0 = (const int *) dptr(h_tgr0);
        B.tg_n = (const int *) dptr(h_tgn);
        B.tg_nk = (const int *) dptr(h_tgnk);
        B.tg_off = (const long long *) dptr(h_tgoff);
    }
    L.ang = (AngItem *) dptr(h_ang);
    L.ang64 = (AngItem *) dptr(h_ang64);
    L.ex = (ExpItem *) dptr(h_ex);
    L.gx = (ExpItem *) dptr(h_gx);
    L.gsegs = (GatherSeg *) dptr(h_gs);
    L.n_gseg = (int) gsegs.size();
    L.pf_start = (long long *) dptr(h_pfs);
    L.ck_gc = (long long *) dptr(h_ckg);
    L.ck_lc = (long long *) dptr(h_ckl);
    L.fin_start = (long long *) dptr(h_fin);
    L.pu_start = (long long *) dptr(h_pus);
    L.pu_red = (long long *) dptr(h_pur);
    if (L.save_control == 2) {
        L.save1_in = save_hit ? c.save.d : (double *) dptr(h_s1);
        L.save2_in = save_hit ? c.save.d + (size_t) 4 * R : (double *) dptr(h_s2);
        L.w2 = (double *) dptr(h_w2);
    }
    const bool solve = L.save_control != 2 && L.acc_mode != LMIEB_ACC_FINISH;
    if (solve) {
        L.ck = A.take<double>((size_t) ckn * k1_ck_width(std::min(nd1, 4)));
        if (L.tc) {
            L.bop_bytes = (size_t) bop_floats * 4;
            L.bop = A.take<float>((size_t) bop_floats);
        }
        if (L.oz) {
            L.bop8 = A.take<unsigned char>((size_t) bop8_bytes);
            L.rowexp = A.take<signed char>((size_t) rx_bytes);
            L.colexp = A.take<int>((size_t) L.n_groups * OZ_NP);
            B.oz_radexp = A.take<int>((size_t) (1 + nd1) * R * 4);
            L.rx_start = (long long *) dptr(h_rxs);
            L.aop = A.take<unsigned char>((size_t) aop_bytes);
            L.a_start = (long long *) dptr(h_axs);
            B.oz_aop = L.aop;
            B.oz_f2 = (const double *) dptr(h_ozf2);
            B.oz_rowexp = L.rowexp;
            B.oz_colexp = L.colexp;
        }
        L.coef = A.take<double>((size_t) (1 + nd1) * (size_t) ctot * 4);
        L.rs = A.take<double>((size_t) (1 + nd1) * 5 * (size_t) R);
        L.part = A.take<double>((size_t) part_total);
    }
    // the integrals in one block, so that a radius group sums them in one call
    L.sums = L.acc_mode == LMIEB_ACC_FINISH ? (double *) dptr(h_acc) : A.take<double>(L.acc_n + 1);
    L.pfacc = L.sums ? L.sums + (size_t) ncase * ncol * 4 : nullptr;
    L.pfn = A.take<double>((size_t) L.pf_total);
    L.ckpt = A.take<double>((size_t) ck_total);
    L.exq = A.take<double>((size_t) ex_total);
    L.pu_scr = A.take<double>((size_t) pu_scr_total);
    {
        char *o = d_out;
        auto take = [&](size_t bytes) { char *r = o; o += pad(bytes); return r; };
        L.o_scal = (double *) take(o_scal * 8);
        L.o_gc = (double *) take(o_gc * 8);
        L.o_lc = (double *) take(o_lc * 8);
        L.o_pf = (double *) take(o_pf * 8);
        // gc, lc truncations; error word; gc, lc truncation bands
        L.o_trunc = (int *) take((size_t) (6 * ncase + 1) * 4);
        if (L.save_control == 1) {
            L.o_save1 = (double *) take((size_t) 4 * R * 8);
            L.o_save2 = (double *) take(n_save2 * 8);
        }
        if (L.acc_mode == LMIEB_ACC_PARTIAL) L.o_acc = (double *) take(L.acc_n * 8);
    }
    if (!L.sums || !L.pfn || !L.exq || (solve && !L.part) || (L.tc && !L.bop) ||
        (L.oz && solve && (!L.bop8 || !L.rowexp || !L.colexp || (aop_bytes && !L.aop)))) {
        fprintf(stderr, "ERROR: lmie_b200: device arena too small\n");
        return -1;
    }

    // ---- queue: upload, kernels, download ----
    const double t_dev = now_ms();
    c.host_ms[1] += t_dev - t_pack;
    c.h2d += h_in_end;
    c.d2h += out_bytes;
    // Each slot has its own stream, so a sub-batch's copies and kernels overlap
    // those of the previous one; with per-stage timing both use the context's
    // stream (the stage events are shared) and run one after the other.
    cudaStream_t s = c.timing ? c.stream : S.stream;
    if (c.redo_src == (int) (&S - c.slot)) {
        LMIEB_CUDA_TRY(cudaStreamWaitEvent(s, c.redo_read, 0));
        c.redo_src = -1;
    }
    stage(0);
    LMIEB_CUDA_TRY(cudaEventRecord(S.t_begin, s));
    if (c.submits == 1) LMIEB_CUDA_TRY(cudaEventRecord(c.t_first, s));
    LMIEB_CUDA_TRY(fault_injected("h2d") ? cudaErrorInvalidValue
                                         : cudaMemcpyAsync(d_in, hp, h_in_end, cudaMemcpyHostToDevice, s));
    // the slot's previous results must have left the output block
    if (!c.timing) LMIEB_CUDA_TRY(cudaStreamWaitEvent(s, S.done, 0));
    LMIEB_CUDA_TRY(cudaMemsetAsync(d_out, 0, out_bytes, s));
    // Gauss-angle pool entries another sub-batch is still computing
    if (c.gl_pending) LMIEB_CUDA_TRY(cudaStreamWaitEvent(s, c.gl_ready, 0));
    if (L.save_control == 2 && save_hit && c.save.pending) LMIEB_CUDA_TRY(cudaStreamWaitEvent(s, c.save.ready, 0));
    if (L.save_control == 2 && !save_hit) {
        // keep this set of kernels on the device for the next re-weighting
        // calls (replacing the previous set once nothing reads it any more)
        if (save_fill(R, n_save2, s)) return -1;
        LMIEB_CUDA_TRY(cudaMemcpyAsync(c.save.d, L.save1_in, (size_t) 4 * R * 8, cudaMemcpyDeviceToDevice, s));
        LMIEB_CUDA_TRY(cudaMemcpyAsync(c.save.d + (size_t) 4 * R, L.save2_in, n_save2 * 8,
                                       cudaMemcpyDeviceToDevice, s));
        LMIEB_CUDA_TRY(cudaEventRecord(c.save.ready, s));
        c.save.pending = true;
        c.save.key = save_key;
        c.save.R = R;
        c.save.nq = save_nq;
        c.save.valid = true;
        c.save.owner = ticket;
    }
    if (!gl_pt.empty()) {
        if (launch_gauss(s, (int) gl_pt.size(), (int *) dptr(h_gpt), (int *) dptr(h_gpi), (int *) dptr(h_gns),
                         (long long *) dptr(h_gmo), (long long *) dptr(h_ggo), (double *) dptr(h_gguess),
                         (double *) dptr(h_gjr), c.gl_pool))
            return -1;
        LMIEB_CUDA_TRY(cudaEventRecord(c.gl_ready, s));
        c.gl_pending = true;
    }
    // A sub-batch whose kernel sequence the slot ran recently (the same
    // structure of radii, orders and angles in the same arena: retrieval loops
    // that change the refractive index or the weights, the parts of repeated
    // pipelined calls) replays it as a CUDA graph, captured the second time it
    // comes.
    const unsigned long long sig = plan_sig(L);
    const bool replayable = !c.timing && L.acc_mode == LMIEB_ACC_WHOLE && L.save_control == 0;
    cudaGraphExec_t graph = replayable ? find_graph(S, sig) : nullptr;
    const bool again = seen_plan(S, sig);
    if (replayable && !graph && again) {
        if (capture_plan(S, s)) return -1;
        graph = find_graph(S, sig);
    }
    if (graph) {
        LMIEB_CUDA_TRY(cudaGraphLaunch(graph, s));
        ++c.graph_replays;
    } else if (run_accumulate(L, s)) {
        return -1;
    } else if (L.acc_mode == LMIEB_ACC_PARTIAL) {
        // this share's integrals are the result
        LMIEB_CUDA_TRY(cudaMemcpyAsync(L.o_acc, L.sums, L.acc_n * 8, cudaMemcpyDeviceToDevice, s));
        for (int i = 4; i < NSTAGE; ++i) stage(i);
    } else {
        if (L.acc_mode == LMIEB_ACC_GROUP && reduce_group(L, s)) return -1;
        if (run_finish(L, s)) return -1;
    }
    if (L.save_control == 1) {
        // the kernels this solve saves: kept on the device as well, recognised
        // once their hash is known (when the sub-batch is collected)
        if (save_fill(R, n_save2, s)) return -1;
        LMIEB_CUDA_TRY(cudaMemcpyAsync(c.save.d, L.o_save1, (size_t) 4 * R * 8, cudaMemcpyDeviceToDevice, s));
        LMIEB_CUDA_TRY(cudaMemcpyAsync(c.save.d + (size_t) 4 * R, L.o_save2, n_save2 * 8,
                                       cudaMemcpyDeviceToDevice, s));
        LMIEB_CUDA_TRY(cudaEventRecord(c.save.ready, s));
        c.save.pending = true;
        c.save.valid = false;
        c.save.R = R;
        c.save.nq = L.n_qang0;
        c.save.owner = ticket;
    }
    // The results come back in pieces of consecutive cases, each followed by
    // an event, so that the host unpacks one piece while the next is copied.
    // First the small tail of the block (truncations and error word,
    // save_control kernels, integrals), then per piece its slices of the
    // cross sections, expansions and phase matrices.
    std::vector<int> piece(1, 0);
    cudaStream_t ds = s;
    if (!c.timing) {
        ds = S.down;
        LMIEB_CUDA_TRY(cudaEventRecord(S.kdone, s));
        LMIEB_CUDA_TRY(cudaStreamWaitEvent(ds, S.kdone, 0));
    }
    {
        const char *misc = (const char *) L.o_trunc;
        const size_t moff = (size_t) (misc - d_out);
        LMIEB_CUDA_TRY(cudaMemcpyAsync(h_out + moff, misc, out_bytes - moff, cudaMemcpyDeviceToHost, ds));
        const int np = (int) std::max<size_t>(1, std::min<size_t>(MAX_PIECES, out_bytes / PIECE_BYTES));
        const double per = (double) (o_scal + o_gc + o_lc + o_pf) / np;
        double run = 0.;
        for (int k = 0; k < ncase; ++k) {
            const DevCase &C = cs[k];
            run += ncol * (4. + 6. * (C.n_angles + (L.want_gc ? C.n_coef : 0) + (L.want_lc ? C.n_coef : 0)));
            if ((k + 1 == ncase || run >= per * (double) piece.size()) && (int) piece.size() <= np)
                piece.push_back(k + 1);
        }
        if (piece.back() != ncase) piece.back() = ncase;
        auto ends = [&](int k, size_t &sc, size_t &g, size_t &l, size_t &f) {
            if (k == ncase) { sc = o_scal; g = o_gc; l = o_lc; f = o_pf; return; }
            sc = (size_t) cs[k].scal_off; g = (size_t) cs[k].gc_off; l = (size_t) cs[k].lc_off;
            f = (size_t) cs[k].pf_out_off;
        };
        auto down = [&](double *base, size_t a, size_t b) -> cudaError_t {
            if (b <= a) return cudaSuccess;
            const size_t off = (size_t) ((char *) (base + a) - d_out);
            return cudaMemcpyAsync(h_out + off, base + a, (b - a) * 8, cudaMemcpyDeviceToHost, ds);
        };
        for (size_t p = 0; p + 1 < piece.size(); ++p) {
            size_t s0, g0, l0, f0, s1, g1, l1, f1;
            ends(piece[p], s0, g0, l0, f0);
            ends(piece[p + 1], s1, g1, l1, f1);
            LMIEB_CUDA_TRY(down(L.o_scal, s0, s1));
            LMIEB_CUDA_TRY(down(L.o_gc, g0, g1));
            LMIEB_CUDA_TRY(down(L.o_lc, l0, l1));
            LMIEB_CUDA_TRY(down(L.o_pf, f0, f1));
            LMIEB_CUDA_TRY(cudaEventRecord(S.piece[p], ds));
        }
    }
    stage(NSTAGE);
    LMIEB_CUDA_TRY(cudaEventRecord(S.t_end, ds));
    LMIEB_CUDA_TRY(cudaEventRecord(S.done, ds));
    S.have_plan = true;
    c.last_slot = (int) (&S - c.slot);

    Pending &P = S.pend;
    P.active = true;
    P.ticket = ticket;
    P.ncase = ncase;
    P.ncol = ncol;
    P.R = R;
    P.cs.swap(cs);
    P.rs = rs_out;
    P.h_out = h_out;
    P.d_out = d_out;
    P.want_gc = L.want_gc;
    P.want_lc = L.want_lc;
    P.pf_from = L.pf_from;
    P.save_control = L.save_control;
    P.n_qang0 = L.n_qang0;
    P.n_save2 = n_save2;
    P.o_scal = L.o_scal;
    P.o_gc = L.o_gc;
    P.o_lc = L.o_lc;
    P.o_pf = L.o_pf;
    P.o_save1 = L.o_save1;
    P.o_save2 = L.o_save2;
    P.o_trunc = L.o_trunc;
    P.acc_mode = L.acc_mode;
    P.o_acc = L.o_acc;
    P.acc_n = L.acc_n;
    P.piece.swap(piece);
    P.t_submit = now_ms();
    P.ps = ps;
    P.precision = p0.precision;
    return 0;
}

long long submit_locked(int n, const lmieb_problem *p, lmieb_result *r);
int collect_ticket(long long ticket);
int fit_sub(int n, const lmieb_problem *p);

// INT8 cases whose truncation n_coef is not certain at the contraction's
// error: some |beta_l| (l up to the truncation) lies within the band of
// `accuracy` (k_exp_final's band outputs).  They are solved again in FP64 by
// the caller of collect_slot.
void uncertain_truncations(const Pending &P, const int *htr, std::vector<int> &out) {
    if (P.precision != LMIEB_PRECISION_INT8 || !(P.want_gc || P.want_lc)) return;
    const int ncase = P.ncase;
    const int *tr = P.want_lc ? htr + ncase : htr;
    const int *band = htr + 2 * ncase + 1 + (P.want_lc ? 2 * ncase : 0);
    for (int k = 0; k < ncase; ++k) {
        const DevCase &C = P.cs[k];
        if (!(C.trunc_band > 0.)) continue;
        auto idx = [&](int v) { return v > 0 ? C.n_coef - v : C.n_coef; };
        const int ti = idx(tr[k]), ui = idx(band[2 * k]), wi = idx(band[2 * k + 1]);
        if (ui < ti || wi > ti) out.push_back(k);
    }
}

// Waits for the slot's sub-batch and unpacks its outputs into the callers'
// result arrays.
int collect_slot(Slot &S) {
    Ctx &c = g_ctx;
    Pending &P = S.pend;
    if (!P.active) return 0;
    P.active = false;
    // the first piece of the results (and the truncations, error word, kept kernels)
    LMIEB_CUDA_TRY(cudaEventSynchronize(S.piece[0]));
    LMIEB_CUDA_TRY(cudaGetLastError());
    const double t_unpack = now_ms();
    double waited = 0.;                 // unpacking waits for later pieces
    const int ncase = P.ncase, ncol = P.ncol;
    auto hostp = [&](void *d) { return P.h_out + ((char *) d - P.d_out); };
    const double *hs = (const double *) hostp(P.o_scal);
    const double *hg = (const double *) hostp(P.o_gc);
    const double *hl = (const double *) hostp(P.o_lc);
    const double *hpf = (const double *) hostp(P.o_pf);
    const int *htr = (const int *) hostp(P.o_trunc);
    if (htr[2 * ncase]) {
        LMIEB_CUDA_TRY(cudaEventSynchronize(S.done));   // no copy may still write the staging
        if (htr[2 * ncase] == 2)
            fprintf(stderr, "ERROR: lmie_b200: a process of the radius group failed before the group's sum\n");
        else
            fprintf(stderr, "ERROR: lmie_b200: a tensor-core angular stage timed out waiting for its pipeline\n");
        return -1;
    }
    // Cases whose truncation the int8 contraction's error could have moved
    // are solved again in FP64.  They go to the re-solve slot now, so that
    // the device runs them while the host unpacks this sub-batch; their
    // results replace these cases' when they are collected below.
    std::vector<int> redo;
    std::vector<lmieb_problem> rq;
    std::vector<lmieb_result> rr;
    lmieb_result *const rs_keep = P.rs;
    int redo_early = 0;
    uncertain_truncations(P, htr, redo);
    if (!redo.empty()) {
        for (int k : redo) {
            rq.push_back(P.ps[k]);
            rq.back().precision = LMIEB_PRECISION_FP64;
            rr.push_back(rs_keep[k]);
        }
        c.redo += (long long) redo.size();
        Slot &R3 = c.slot[2];
        if (!c.timing && !R3.pend.active) {
            redo_early = fit_sub((int) rq.size(), rq.data());
            if (c.submits < 2) c.call_slot[c.submits] = 2;
            ++c.submits;
            // their coefficient columns and per-radius sums from this
            // sub-batch's arena, which this slot's next upload waits for
            const Plan &SL = *S.plan;
            // (offsets: without the split form, coefficient offsets are the n1 prefix sums)
            c.gather.on = SL.coef && SL.rs && !SL.tc && P.save_control == 0 && P.acc_mode == LMIEB_ACC_WHOLE;
            c.gather.coef = SL.coef;
            c.gather.rs = SL.rs;
            c.gather.tot = SL.B.tot;
            c.gather.R = SL.B.R;
            c.gather.cs.clear();
            for (int i = 0; i < redo_early; ++i) c.gather.cs.push_back(P.cs[redo[i]]);
            const int rc3 = submit_sub(R3, c.redo_ticket++, redo_early, rq.data(), rr.data());
            c.gather.on = false;
            if (rc3) {
                R3.pend.active = false;
                return -1;
            }
            LMIEB_CUDA_TRY(cudaEventRecord(c.redo_read, R3.stream));
            c.redo_src = (int) (&S - c.slot);
        }
    }
    for (size_t p = 0; p + 1 < P.piece.size(); ++p) {
        if (p > 0) {
            const double tw = now_ms();
            LMIEB_CUDA_TRY(cudaEventSynchronize(S.piece[p]));
            waited += now_ms() - tw;
        }
        const int k0 = P.piece[p];
        parallel_for(P.piece[p + 1] - k0, 8, [&](int i) {
            const int k = k0 + i;
            const DevCase &C = P.cs[k];
            lmieb_result &r = P.rs[k];
            memcpy(r.scal, hs + C.scal_off, (size_t) ncol * 4 * 8);
            // rows laid out one after the other (the blocks of lmie_out_alloc)
            // take one copy per run
            auto put = [&](double **rows, double *flat, const double *src, size_t len) {
                if (rows) {
                    for (int j = 0; j < ncol * 6;) {
                        int e = j + 1;
                        while (e < ncol * 6 && rows[e] == rows[j] + (size_t) (e - j) * len) ++e;
                        memcpy(rows[j], src + (size_t) j * len, (size_t) (e - j) * len * 8);
                        j = e;
                    }
                } else if (flat) {
                    memcpy(flat, src, (size_t) ncol * 6 * len * 8);
                }
            };
            if (P.want_gc) put(r.gc_rows, r.gc, hg + C.gc_off, (size_t) C.n_coef);
            if (P.want_lc) put(r.lc_rows, r.lc, hl + C.lc_off, (size_t) C.n_coef);
            if (P.pf_from) put(r.pf_rows, r.pf, hpf + C.pf_out_off, (size_t) C.n_angles);
            const int t = P.want_lc ? htr[ncase + k] : (P.want_gc ? htr[k] : 0);
            r.n_coef_out = (P.want_gc || P.want_lc) ? (t > 0 ? C.n_coef - t + 1 : C.n_coef) : 0;
        }, host_cores());
    }
    LMIEB_CUDA_TRY(cudaEventSynchronize(S.done));
    c.host_ms[2] += t_unpack - P.t_submit + waited;
    {
        float a = 0.f, b = 0.f;
        if (cudaEventElapsedTime(&a, S.t_begin, S.t_end) == cudaSuccess) c.host_ms[6] += a;
        if (cudaEventElapsedTime(&b, c.t_first, S.t_end) == cudaSuccess) c.host_ms[5] = std::max(c.host_ms[5], (double) b);
    }
    if (c.timing) {
        for (int i = 0; i < NSTAGE; ++i) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, c.ev[i], c.ev[i + 1]) != cudaSuccess) ms = 0.f;
            c.stage_ms[i] += ms;
        }
    }
    if (P.save_control == 1 && c.save.owner == P.ticket) {
        // the set just saved: its hash, over the same rows a later
        // save_control 2 call hashes through its row pointers
        const double *h1 = (const double *) hostp(P.o_save1), *h2 = (const double *) hostp(P.o_save2);
        const int R = P.R, nq = P.n_qang0;
        c.save.key = save_hash(R, nq, [&](int i) -> const double * {
            return i < 4 ? h1 + (size_t) i * R : h2 + (size_t) (i - 4) * nq;
        });
        c.save.nq = nq;
        c.save.valid = true;
    }
    if (P.acc_mode == LMIEB_ACC_PARTIAL && P.rs[0].acc)
        memcpy(P.rs[0].acc, hostp(P.o_acc), P.acc_n * 8);
    if (P.save_control == 1) {
        lmieb_result &r = P.rs[0];
        if (r.save1) memcpy(r.save1, hostp(P.o_save1), (size_t) 4 * P.R * 8);
        if (r.save2 && P.n_qang0 > 0) memcpy(r.save2, hostp(P.o_save2), P.n_save2 * 8);
    }
    c.host_ms[3] += now_ms() - t_unpack - waited;
    if (!redo.empty()) {
        // the re-solve submitted above, then any cases left over (more than
        // one sub-batch, or timing mode) one sub-batch at a time; the slot's
        // staging is no longer read, so these may reuse it (P too: what is
        // needed was kept)
        if (redo_early > 0 && collect_slot(c.slot[2])) return -1;
        for (int k0 = redo_early; k0 < (int) rq.size();) {
            const int m = fit_sub((int) rq.size() - k0, rq.data() + k0);
            const long long t = submit_locked(m, rq.data() + k0, rr.data() + k0);
            if (t < 0 || collect_ticket(t)) return -1;
            k0 += m;
        }
        // the arrays went straight to the callers' storage; the counts come back here
        for (size_t i = 0; i < redo.size(); ++i) rs_keep[redo[i]].n_coef_out = rr[i].n_coef_out;
    }
    return 0;
}

// Collects `ticket` if it is still pending, and remembers its status.
int collect_ticket(long long ticket) {
    Ctx &c = g_ctx;
    for (Slot &S : c.slot)
        if (S.pend.active && S.pend.ticket == ticket) {
            const int rc = collect_slot(S);
            c.finished.push_back({ticket, rc});
            if (c.finished.size() > 64) c.finished.erase(c.finished.begin());
            return rc;
        }
    for (auto &f : c.finished)
        if (f.first == ticket) return f.second;
    return 0;
}

// A free slot for the next sub-batch (the older pending one is collected).
Slot &free_slot() {
    Ctx &c = g_ctx;
    Slot &S = c.slot[c.next_ticket & 1];
    if (S.pend.active) collect_ticket(S.pend.ticket);
    return S;
}

// Cases of p[0..n) that fit one sub-batch (at least one).
int fit_sub(int n, const lmieb_problem *p) {
    size_t bytes = 0;
    int k = 0;
    while (k < n) {
        const size_t b = case_bytes(p[k]);
        if (k > 0 && bytes + b > BATCH_BYTES) break;
        bytes += b;
        ++k;
    }
    return k;
}

int check_uniform(int n, const lmieb_problem *p) {
    for (int k = 1; k < n; ++k) {
        bool same = p[k].nd == p[0].nd && p[k].nd1 == p[0].nd1 && p[k].nd2 == p[0].nd2 &&
                    p[k].want_gc == p[0].want_gc && p[k].want_lc == p[0].want_lc &&
                    p[k].pf_from == p[0].pf_from && p[k].save_control == 0 && p[0].save_control == 0 &&
                    p[k].precision == p[0].precision;
        for (int q = 0; same && q < p[0].nd1; ++q) same = p[k].idx1[q] == p[0].idx1[q];
        for (int q = 0; same && q < p[0].nd2; ++q) same = p[k].idx2[q] == p[0].idx2[q];
        if (!same) {
            fprintf(stderr, "ERROR: lmie_b200: case %d of a batch differs from case 0 in its derivative "
                    "layout, requested outputs or save_control\n", k);
            return -1;
        }
    }
    return 0;
}

void reset_counters() {
    Ctx &c = g_ctx;
    for (int i = 0; i < NSTAGE; ++i) c.stage_ms[i] = 0.;
    for (int i = 1; i < 4; ++i) c.host_ms[i] = 0.;
    c.host_ms[5] = c.host_ms[6] = 0.;
    for (int i = 0; i < 4; ++i) c.work[i] = 0.;
    c.launches = 0;
    c.h2d = c.d2h = 0;
    c.submits = 0;
    c.call_slot[0] = c.call_slot[1] = -1;
    c.redo = 0;
    c.tensor_ops = 0.;
}

// submits p[0..n) (one sub-batch); returns its ticket or -1
long long submit_locked(int n, const lmieb_problem *p, lmieb_result *r) {
    Ctx &c = g_ctx;
    Slot &S = free_slot();
    const long long t = c.next_ticket++;
    if (c.submits < 2) c.call_slot[c.submits] = (int) (&S - c.slot);
    ++c.submits;
    if (submit_sub(S, t, n, p, r)) {
        S.pend.active = false;
        return -1;
    }
    if (c.timing && collect_ticket(t)) return -1;   // stage events are shared: one sub-batch at a time
    return t;
}

}  // namespace

extern "C" int lmieb_device_solve_batch(int n, const lmieb_problem *p, lmieb_result *r) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (n < 1) return 0;
    if (ensure_ready()) return -1;
    if (check_uniform(n, p)) return -1;
    reset_counters();
    // sub-batches by device working set, each packed while the previous one runs
    std::vector<long long> tickets;
    int rc = 0;
    for (int k0 = 0; k0 < n && rc == 0;) {
        const int m = fit_sub(n - k0, p + k0);
        const long long t = submit_locked(m, p + k0, r + k0);
        if (t < 0) rc = -1;
        else tickets.push_back(t);
        k0 += m;
    }
    for (long long t : tickets)
        if (collect_ticket(t)) rc = -1;
    return rc;
}

extern "C" long long lmieb_device_submit(int n, const lmieb_problem *p, lmieb_result *r, int first) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (n < 1) return -1;
    if (ensure_ready()) return -1;
    if (check_uniform(n, p)) return -1;
    if (first) reset_counters();
    return submit_locked(n, p, r);
}

extern "C" int lmieb_device_collect(long long ticket) {
    std::lock_guard<std::mutex> lock(g_mu);
    return collect_ticket(ticket);
}

extern "C" int lmieb_device_fit(int n, const lmieb_problem *p) {
    return n < 1 ? 0 : fit_sub(n, p);
}

extern "C" int lmieb_device_solve(const lmieb_problem *p, lmieb_result *r) {
    if (p->acc_mode == LMIEB_ACC_GROUP) {
        std::lock_guard<std::mutex> lock(g_mu);
        g_ctx.group_joined = false;
    }
    const int rc = lmieb_device_solve_batch(1, p, r);
    if (rc && p->acc_mode == LMIEB_ACC_GROUP) {
        // failed before the group's reduction: join it with a failure mark
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_ctx.group_joined) group_abort((size_t) 4 * (1 + p->nd) * (1 + p->n_qang));
    }
    return rc;
}

extern "C" int lmieb_group_abort(int n_derivs, int n_qang) {
    std::lock_guard<std::mutex> lock(g_mu);
    g_ctx.group_joined = false;
    return group_abort((size_t) 4 * (1 + n_derivs) * (1 + n_qang));
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

extern "C" int lmieb_save_cache_stats(long long *hits, long long *misses) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (hits) *hits = g_ctx.save.hits;
    if (misses) *misses = g_ctx.save.misses;
    return 0;
}

namespace {

// Loads NCCL (the libnccl.so.2 already in the process, or the system's) and
// resolves the entry points of the built-in group reduction.
int nccl_load() {
    Nccl &n = g_nccl;
    if (n.lib) return 0;
    void *lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
    if (!lib) {
        fprintf(stderr, "ERROR: lmie_b200: cannot load NCCL (%s)\n", dlerror());
        return -1;
    }
    Nccl t;
    t.get_unique_id = (decltype(t.get_unique_id)) dlsym(lib, "ncclGetUniqueId");
    t.comm_init_rank = (decltype(t.comm_init_rank)) dlsym(lib, "ncclCommInitRank");
    t.all_reduce = (decltype(t.all_reduce)) dlsym(lib, "ncclAllReduce");
    t.comm_destroy = (decltype(t.comm_destroy)) dlsym(lib, "ncclCommDestroy");
    t.error_string = (decltype(t.error_string)) dlsym(lib, "ncclGetErrorString");
    if (!t.get_unique_id || !t.comm_init_rank || !t.all_reduce || !t.comm_destroy || !t.error_string) {
        fprintf(stderr, "ERROR: lmie_b200: libnccl.so.2 lacks an entry point\n");
        dlclose(lib);
        return -1;
    }
    t.lib = lib;
    n = t;
    return 0;
}

// Ends the current radius group (and its NCCL communicator).
void group_release() {
    if (g_group.comm) {
        cudaDeviceSynchronize();                 // no solve may still use it
        g_nccl.comm_destroy(g_group.comm);
    }
    g_group = RadiusGroup();
}

}  // namespace

extern "C" int lmieb_set_radius_group(int rank, int world, lmieb_reduce_fn reduce, void *ctx) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (world < 1 || rank < 0 || rank >= world || (world > 1 && !reduce)) {
        fprintf(stderr, "ERROR: lmieb_set_radius_group: rank %d of %d%s\n", rank, world,
                world > 1 && !reduce ? " without a reduction" : "");
        return -1;
    }
    group_release();
    g_group.rank = rank;
    g_group.world = world;
    g_group.fn = reduce;
    g_group.fn_ctx = ctx;
    g_group.on = reduce != nullptr;
    return 0;
}

extern "C" int lmieb_nccl_unique_id(void *id) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!id || nccl_load()) return -1;
    NcclUniqueId u;
    const int r = g_nccl.get_unique_id(&u);
    if (r != 0) {
        fprintf(stderr, "ERROR: lmie_b200: ncclGetUniqueId: %s\n", g_nccl.error_string(r));
        return -1;
    }
    memcpy(id, &u, sizeof(u));
    return 0;
}

extern "C" int lmieb_set_radius_group_nccl(const void *id, int rank, int world) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!id || world < 1 || rank < 0 || rank >= world) {
        fprintf(stderr, "ERROR: lmieb_set_radius_group_nccl: rank %d of %d\n", rank, world);
        return -1;
    }
    if (ensure_ready() || nccl_load()) return -1;
    group_release();
    NcclUniqueId u;
    memcpy(&u, id, sizeof(u));
    int prev = -1;
    LMIEB_CUDA_TRY(cudaGetDevice(&prev));
    LMIEB_CUDA_TRY(cudaSetDevice(g_ctx.device));     // the communicator lives on the library's GPU
    void *comm = nullptr;
    const int r = g_nccl.comm_init_rank(&comm, world, u, rank);
    LMIEB_CUDA_TRY(cudaSetDevice(prev));
    if (r != 0) {
        fprintf(stderr, "ERROR: lmie_b200: ncclCommInitRank: %s\n", g_nccl.error_string(r));
        return -1;
    }
    g_group.rank = rank;
    g_group.world = world;
    g_group.comm = comm;
    g_group.on = true;
    return 0;
}

extern "C" int lmieb_get_radius_group(int *rank, int *world) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (rank) *rank = g_group.rank;
    if (world) *world = g_group.world;
    return g_group.on ? 1 : 0;
}

extern "C" int lmieb_timing_state(void) {
    std::lock_guard<std::mutex> lock(g_mu);
    return g_ctx.timing ? 1 : 0;
}

extern "C" int lmieb_last_timing(double *ms, int n) {
    std::lock_guard<std::mutex> lock(g_mu);
    for (int i = 0; i < n && i < NSTAGE; ++i) ms[i] = g_ctx.stage_ms[i];
    return NSTAGE;
}

extern "C" int lmieb_rerun_device(int reps, int flush_l2, double *ms_total, double *ms_stage) {
    std::lock_guard<std::mutex> lock(g_mu);
    Ctx &c = g_ctx;
    // a re-run repeats the resident sub-batches of the last call: exactly one,
    // or an INT8 sub-batch and the FP64 re-solve of its uncertain cases
    const int ns = c.submits;
    bool ok = c.ready && (ns == 1 || (ns == 2 && c.redo > 0 && c.call_slot[0] != c.call_slot[1]));
    for (int i = 0; ok && i < ns; ++i) {
        const int si = c.call_slot[i];
        ok = si >= 0 && c.slot[si].have_plan && c.slot[si].plan->acc_mode == LMIEB_ACC_WHOLE;
    }
    if (!ok) {
        fprintf(stderr, "ERROR: lmieb_rerun_device: no single-sub-batch solve is resident on the device\n");
        return -1;
    }
    if (flush_l2 && !c.flush) LMIEB_CUDA_TRY(cudaMalloc((void **) &c.flush, FLUSH_BYTES));
    const bool was = c.timing;
    // each plan's kernel sequence as one CUDA graph (captured once per plan)
    cudaGraphExec_t gx[2] = {nullptr, nullptr};
    for (int i = 0; i < ns; ++i) {
        Slot &S = c.slot[c.call_slot[i]];
        const unsigned long long sig = plan_sig(*S.plan);
        if (!find_graph(S, sig) && capture_plan(S, c.stream)) return -1;
        gx[i] = find_graph(S, sig);
    }
    double total = 0., st[NSTAGE] = {}, k3 = 0.;
    cudaEvent_t e0 = c.ev[0], e1 = c.ev[NSTAGE];
    for (int i = 0; i < reps; ++i) {
        if (flush_l2) LMIEB_CUDA_TRY(cudaMemsetAsync(c.flush, i & 0xff, FLUSH_BYTES, c.stream));
        LMIEB_CUDA_TRY(cudaEventRecord(e0, c.stream));
        for (int j = 0; j < ns; ++j) LMIEB_CUDA_TRY(cudaGraphLaunch(gx[j], c.stream));
        LMIEB_CUDA_TRY(cudaEventRecord(e1, c.stream));
        LMIEB_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        total += ms;
    }
    // stage times: the same kernel sequences launched one by one between events
    c.timing = true;
    for (int i = 0; i < reps; ++i) {
        if (flush_l2) LMIEB_CUDA_TRY(cudaMemsetAsync(c.flush, i & 0xff, FLUSH_BYTES, c.stream));
        for (int j = 0; j < ns; ++j) {
            const Plan &PL = *c.slot[c.call_slot[j]].plan;
            if (run_kernels(*c.slot[c.call_slot[j]].plan, c.stream)) { c.timing = was; return -1; }
            LMIEB_CUDA_TRY(cudaEventSynchronize(c.ev[8]));
            for (int k = 1; k < 8; ++k) {
                float sm = 0.f;
                cudaEventElapsedTime(&sm, c.ev[k], c.ev[k + 1]);
                st[k] += sm;
            }
            if (PL.oz && PL.n_ang > 0) {
                float km = 0.f;
                if (cudaEventElapsedTime(&km, c.k3[0], c.k3[1]) == cudaSuccess) k3 += km;
            }
        }
    }
    c.timing = was;
    LMIEB_CUDA_TRY(cudaGetLastError());
    if (ms_total) *ms_total = total;
    if (ms_stage)
        for (int k = 0; k < NSTAGE; ++k) ms_stage[k] = st[k];
    c.k3_ms = k3;
    return 0;
}

extern "C" int lmieb_last_redo(long long *cases) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (cases) *cases = g_ctx.redo;
    return 0;
}

extern "C" int lmieb_last_int8_kernel(double *tensor_ops, double *ms) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (tensor_ops) *tensor_ops = g_ctx.tensor_ops;
    if (ms) *ms = g_ctx.k3_ms;
    return 0;
}

extern "C" int lmieb_last_work(double *flops, long long *launches, size_t *h2d, size_t *d2h) {
    std::lock_guard<std::mutex> lock(g_mu);
    Ctx &c = g_ctx;
    if (flops)
        for (int i = 0; i < 4; ++i) flops[i] = c.work[i];
    if (launches) *launches = c.launches;
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

extern "C" int lmieb_tc_selftest(int K, double *max_rel_err) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (K <= 0 || K % TC_KC || K > 4096 || !max_rel_err) {
        fprintf(stderr, "ERROR: lmieb_tc_selftest: K must be a positive multiple of %d, at most 4096\n", TC_KC);
        return -1;
    }
    if (ensure_ready()) return -1;
    const int M = TC_M, N = TC_NP;   // one product tile
    std::vector<double> a((size_t) M * K), b((size_t) N * K), d((size_t) M * N), ref((size_t) M * N, 0.);
    // seeded operands with the spread of magnitudes of the angular products
    unsigned long long st = 0x9E3779B97F4A7C15ull;
    auto rnd = [&]() {
        st ^= st << 13; st ^= st >> 7; st ^= st << 17;
        return (double) (st >> 11) * (1. / 9007199254740992.) * 2. - 1.;
    };
    for (int i = 0; i < M; ++i)
        for (int k = 0; k < K; ++k) a[(size_t) i * K + k] = rnd() * (k + 1.);
    for (int n = 0; n < N; ++n)
        for (int k = 0; k < K; ++k) b[(size_t) n * K + k] = rnd() / (k + 1.) * exp(-4. * k / K);
    double mx = 0.;
    for (int i = 0; i < M; ++i)
        for (int n = 0; n < N; ++n) {
            double s = 0.;
            for (int k = 0; k < K; ++k) s += a[(size_t) i * K + k] * b[(size_t) n * K + k];
            ref[(size_t) i * N + n] = s;
            mx = std::max(mx, fabs(s));
        }
    double *da = nullptr, *db = nullptr, *dd = nullptr;
    int *derr = nullptr, herr = 0;
    cudaStream_t s = g_ctx.stream;
    int rc = -1;
    if (cudaMalloc((void **) &da, a.size() * 8) == cudaSuccess && cudaMalloc((void **) &db, b.size() * 8) == cudaSuccess &&
        cudaMalloc((void **) &dd, d.size() * 8) == cudaSuccess && cudaMalloc((void **) &derr, 4) == cudaSuccess &&
        cudaMemcpyAsync(da, a.data(), a.size() * 8, cudaMemcpyHostToDevice, s) == cudaSuccess &&
        cudaMemcpyAsync(db, b.data(), b.size() * 8, cudaMemcpyHostToDevice, s) == cudaSuccess &&
        cudaMemsetAsync(derr, 0, 4, s) == cudaSuccess && launch_tc_selftest(s, K, da, db, dd, derr) == 0 &&
        cudaMemcpyAsync(d.data(), dd, d.size() * 8, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
        cudaMemcpyAsync(&herr, derr, 4, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
        cudaStreamSynchronize(s) == cudaSuccess)
        rc = 0;
    cudaFree(da); cudaFree(db); cudaFree(dd); cudaFree(derr);
    if (rc) {
        fprintf(stderr, "ERROR: lmieb_tc_selftest: %s\n", cudaGetErrorString(cudaGetLastError()));
        return -1;
    }
    if (herr) {
        fprintf(stderr, "ERROR: lmieb_tc_selftest: the tensor-core pipeline timed out\n");
        return -1;
    }
    double e = 0.;
    for (size_t i = 0; i < d.size(); ++i) e = std::max(e, fabs(d[i] - ref[i]));
    *max_rel_err = mx > 0. ? e / mx : e;
    return 0;
}

extern "C" int lmieb_graph_stats(long long *captures, long long *replays) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (captures) *captures = g_ctx.graph_captures;
    if (replays) *replays = g_ctx.graph_replays;
    return 0;
}

extern "C" int lmieb_memory(long long out[4]) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!out || ensure_ready()) return -1;
    size_t fr = 0, tot = 0;
    LMIEB_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
    const Ctx &c = g_ctx;
    long long dev = (long long) (c.gl_cap * sizeof(double) + c.save.cap * sizeof(double));
    if (c.flush) dev += (long long) FLUSH_BYTES;
    long long pin = 0;
    for (const Slot &S : c.slot) {
        dev += (long long) S.dcap;
        pin += (long long) S.hcap;
    }
    out[0] = (long long) fr;
    out[1] = (long long) tot;
    out[2] = dev;
    out[3] = pin;
    return 0;
}

extern "C" int lmieb_oz_selftest(int K, double *max_rel_err) {
    return lmieb_oz_selftest_wait(K, LMIEB_WAIT_CYCLES, 0, max_rel_err);
}

extern "C" int lmieb_oz_selftest_wait(int K, long long wait_cycles, int withhold, double *max_rel_err) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (K <= 0 || K % OZ_KC || K > OZ_KC * OZ_MAX_NK || !max_rel_err || wait_cycles < 1 ||
        wait_cycles > LMIEB_WAIT_CYCLES) {
        fprintf(stderr, "ERROR: lmieb_oz_selftest: K must be a positive multiple of %d, at most %d; "
                "the wait limit 1 .. %lld cycles\n", OZ_KC, OZ_KC * OZ_MAX_NK, (long long) LMIEB_WAIT_CYCLES);
        return -1;
    }
    if (ensure_ready()) return -1;
    const int M = OZ_M, N = OZ_NP;   // one product tile
    std::vector<double> a((size_t) M * K), b((size_t) N * K), d((size_t) M * N), ref((size_t) M * N, 0.);
    // seeded operands with the growth of the angular products in k: A ~ k^2,
    // B ~ 1/k with a decaying tail, both spanning orders of magnitude over rows
    unsigned long long st = 0x9E3779B97F4A7C15ull;
    auto rnd = [&]() {
        st ^= st << 13; st ^= st >> 7; st ^= st << 17;
        return (double) (st >> 11) * (1. / 9007199254740992.) * 2. - 1.;
    };
    for (int i = 0; i < M; ++i)
        for (int k = 0; k < K; ++k) a[(size_t) i * K + k] = rnd() * (k + 1.) * (k + 2.) * exp2(-(i % 17));
    for (int n = 0; n < N; ++n)
        for (int k = 0; k < K; ++k) b[(size_t) n * K + k] = rnd() / (k + 1.) * exp(-4. * k / K) * exp2(n % 23 - 11);
    // reference sums in long double; the error of each element against the
    // largest |a_ik b_nk| of its row and column pair
    double worst = 0.;
    for (int i = 0; i < M; ++i)
        for (int n = 0; n < N; ++n) {
            long double sum = 0.L;
            for (int k = 0; k < K; ++k) sum += (long double) a[(size_t) i * K + k] * b[(size_t) n * K + k];
            ref[(size_t) i * N + n] = (double) sum;
        }
    double *da = nullptr, *db = nullptr, *dd = nullptr;
    int *derr = nullptr, herr = 0;
    cudaStream_t s = g_ctx.stream;
    int rc = -1;
    if (cudaMalloc((void **) &da, a.size() * 8) == cudaSuccess && cudaMalloc((void **) &db, b.size() * 8) == cudaSuccess &&
        cudaMalloc((void **) &dd, d.size() * 8) == cudaSuccess && cudaMalloc((void **) &derr, 4) == cudaSuccess &&
        cudaMemcpyAsync(da, a.data(), a.size() * 8, cudaMemcpyHostToDevice, s) == cudaSuccess &&
        cudaMemcpyAsync(db, b.data(), b.size() * 8, cudaMemcpyHostToDevice, s) == cudaSuccess &&
        cudaMemsetAsync(derr, 0, 4, s) == cudaSuccess &&
        launch_oz_selftest(s, K, da, db, dd, derr, wait_cycles, withhold) == 0 &&
        cudaMemcpyAsync(d.data(), dd, d.size() * 8, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
        cudaMemcpyAsync(&herr, derr, 4, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
        cudaStreamSynchronize(s) == cudaSuccess)
        rc = 0;
    cudaFree(da); cudaFree(db); cudaFree(dd); cudaFree(derr);
    if (rc) {
        fprintf(stderr, "ERROR: lmieb_oz_selftest: %s\n", cudaGetErrorString(cudaGetLastError()));
        return -1;
    }
    if (herr) {
        fprintf(stderr, "ERROR: lmieb_oz_selftest: the tensor-core pipeline timed out\n");
        return -1;
    }
    for (int i = 0; i < M; ++i)
        for (int n = 0; n < N; ++n) {
            double ma = 0., mb = 0.;
            for (int k = 0; k < K; ++k) {
                ma = std::max(ma, fabs(a[(size_t) i * K + k]));
                mb = std::max(mb, fabs(b[(size_t) n * K + k]));
            }
            const double scale = ma * mb;
            const double e = fabs(d[(size_t) i * N + n] - ref[(size_t) i * N + n]);
            worst = std::max(worst, scale > 0. ? e / scale : e);
        }
    *max_rel_err = worst;
    return 0;
}

extern "C" void lmieb_host_phase(int phase, double ms) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (phase >= 0 && phase < LMIEB_N_HOST) g_ctx.host_ms[phase] = ms;
}

extern "C" int lmieb_last_host_timing(double *ms, int n) {
    std::lock_guard<std::mutex> lock(g_mu);
    for (int i = 0; i < n && i < LMIEB_N_HOST; ++i) ms[i] = g_ctx.host_ms[i];
    return LMIEB_N_HOST;
}

extern "C" int lmieb_set_work_granularity(int precision, double items_per_sm) {
    std::lock_guard<std::mutex> lock(g_mu);
    if ((precision != LMIEB_PRECISION_FP64 && precision != LMIEB_PRECISION_TF32X3 &&
         precision != LMIEB_PRECISION_INT8) || !(items_per_sm >= 0.25) || items_per_sm > 256.) {
        fprintf(stderr, "ERROR: lmieb_set_work_granularity: precision %d, items per SM %g\n", precision, items_per_sm);
        return -1;
    }
    g_items_per_sm[prec_slot(precision)] = items_per_sm;
    return 0;
}

extern "C" int lmieb_set_split_segment(int chunks) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (chunks < 1 || chunks > 64) {
        fprintf(stderr, "ERROR: lmieb_set_split_segment: %d chunks (1..64)\n", chunks);
        return -1;
    }
    g_tc_seg = chunks;
    return 0;
}

extern "C" int lmieb_set_user_angle_part(int orders) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (orders < PU_T || orders > 4096 || orders % PU_T) {
        fprintf(stderr, "ERROR: lmieb_set_user_angle_part: %d orders (a multiple of %d, %d..4096)\n", orders, PU_T,
                PU_T);
        return -1;
    }
    g_pu_lp = orders;
    return 0;
}

extern "C" int lmieb_get_user_angle_part(void) {
    std::lock_guard<std::mutex> lock(g_mu);
    return g_pu_lp;
}

extern "C" int lmieb_get_split_segment(void) {
    std::lock_guard<std::mutex> lock(g_mu);
    return g_tc_seg;
}

extern "C" double lmieb_get_work_granularity(int precision) {
    std::lock_guard<std::mutex> lock(g_mu);
    return g_items_per_sm[prec_slot(precision)];
}
