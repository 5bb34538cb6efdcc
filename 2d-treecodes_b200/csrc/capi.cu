// capi.cu -- the C ABI: contexts, host and device entry points, statistics, inspection.
//
// treecode_potential / treecode_force_mrag keep the reference's prototypes
// (drivers/treecode-potential.h:21-29, drivers/treecode-force.h:21-31).  Each calling thread
// gets its own context (stream + grow-only device buffers), so the functions are reentrant,
// unlike the reference whose Tree:: globals are shared (drivers/upward.cpp:51-59).
#include <algorithm>
#include <chrono>
#include <climits>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "treecodes_b200.h"
#include <initializer_list>

#include "tc_internal.h"

namespace tc {

int direct_potential(Context &c, const double *xs, const double *ys, const double *vs, int n,
                     const double *xt, const double *yt, int m, double *out);
int log_probe(Context &c, const double *x, int n, double *out);
int direct_force(Context &c, const double *xs, const double *ys, const double *vs, int n,
                 const double *xt, const double *yt, int m, double *xo, double *yo);
int measure_fma_peak(int fp64, double *tflops);

static thread_local int tls_status = TC_OK;
static thread_local char tls_msg[512] = "";
thread_local long long g_launches = 0;

void set_error(int status, const char *fmt, ...) {
    tls_status = status;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(tls_msg, sizeof(tls_msg), fmt, ap);
    va_end(ap);
}

static void clear_error() {
    tls_status = TC_OK;
    tls_msg[0] = 0;
}

void phase_mark(Context &c, int idx) {
    if (c.timing) cudaEventRecord(c.ev[idx], c.stream);
}

long long scratch_layout(const Context &c, int nkinds, int nwarps, int nitems,
                         long long max_entries, ScratchLayout &s) {
    const long long per_warp = nwarps > 0 ? ((long long)nitems + nwarps - 1) / nwarps : 0;
    max_entries = std::min<long long>(max_entries, INT_MAX / 2);   // offsets stay ints
    long long total = 0;
    for (int k = 0; k < 3; ++k) {
        long long cap = k < nkinds ? c.list_per_item[k] * per_warp + 16 : 0;
        if (k < nkinds && cap * nwarps * nkinds > max_entries) cap = max_entries / (nwarps * nkinds);
        s.cap[k] = (int)cap;
        s.koff[k] = (int)total;
        total += cap * nwarps;
    }
    return total;
}

ListScratch::~ListScratch() {
    if (owned && p) cudaFreeAsync(p, stream);
}

int list_scratch(Context &c, int nkinds, int nwarps, int nitems, size_t entry_bytes,
                 ScratchLayout &sl, ListScratch &out) {
    const long long per_warp = nwarps > 0 ? ((long long)nitems + nwarps - 1) / nwarps : 0;
    long long need = 0;
    for (int k = 0; k < nkinds; ++k) need += (c.list_per_item[k] * per_warp + 16) * nwarps;
    const long long have = (long long)(c.buf[S_REC].bytes / entry_bytes);
    if (need <= std::min<long long>(have, INT_MAX / 2)) {
        scratch_layout(c, nkinds, nwarps, nitems, have, sl);
        out.p = c.buf[S_REC].p;
        return TC_OK;
    }
    const long long n = scratch_layout(c, nkinds, nwarps, nitems,
                                       (2048ll << 20) / (long long)entry_bytes, sl);
    const cudaError_t e = cudaMallocAsync(&out.p, (size_t)n * entry_bytes + 16, c.stream);
    if (e != cudaSuccess) {
        out.p = nullptr;
        set_error(TC_ERR_ALLOC, "cudaMallocAsync(%lld bytes) for the list scratch failed: %s",
                  n * (long long)entry_bytes, cudaGetErrorString(e));
        return TC_ERR_ALLOC;
    }
    out.owned = true;
    out.stream = c.stream;
    return TC_OK;
}

void scratch_learn(Context &c, int nkinds, int nwarps, int nitems, const unsigned *longest) {
    const long long per_warp = nwarps > 0 ? ((long long)nitems + nwarps - 1) / nwarps : 1;
    for (int k = 0; k < nkinds; ++k) {
        const long long need = ((long long)longest[k] * 5 / 4 + per_warp - 1) / per_warp;
        if (need > c.list_per_item[k]) c.list_per_item[k] = (int)std::min<long long>(need, 1 << 20);
    }
}

// Host waits of a solve.  By default the thread spins in the CUDA call, the lowest latency.  A
// context with sleeping_waits polls: back to back for the first 32 queries (a few microseconds,
// which ends the short waits at once), then every 20 us with the thread asleep in between.  The
// request server's slot threads wait that way, so that four waiting slots do not take four
// host cores from the threads that stage inputs and submit requests.
template <class Query>
static cudaError_t poll_and_sleep(Query query) {
    for (int i = 0;; ++i) {
        const cudaError_t e = query();
        if (e != cudaErrorNotReady) return e;
        if (i >= 32) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

cudaError_t wait_stream(Context &c, cudaStream_t s) {
    if (!c.sleeping_waits) return cudaStreamSynchronize(s);
    return poll_and_sleep([s] { return cudaStreamQuery(s); });
}

cudaError_t wait_event(Context &c, cudaEvent_t e) {
    if (!c.sleeping_waits) return cudaEventSynchronize(e);
    return poll_and_sleep([e] { return cudaEventQuery(e); });
}

// Reads back the device error word and the work counters (one sync).  The counters land in
// h_pinned[16 ...] as unsigned long long.
int check_device_errors(Context &c, const char *where) {
    unsigned *err = slot_ptr<unsigned>(c, S_ERR);
    TC_CUDA_TRY(cudaMemcpyAsync(c.h_pinned + 8, err, sizeof(unsigned), cudaMemcpyDeviceToHost,
                                c.stream));
    TC_CUDA_TRY(cudaMemcpyAsync(c.h_pinned + 16, c.buf[S_STATS].p,
                                sizeof(unsigned long long) * STAT_SLOTS, cudaMemcpyDeviceToHost,
                                c.stream));
    TC_CUDA_TRY(wait_stream(c, c.stream));
    c.counts.launches = g_launches;
    const unsigned e = c.h_pinned[8];
    if (e & DEVERR_SPIN_LIMIT) {
        set_error(TC_ERR_TIMEOUT, "%s: a bounded device wait gave up (flags 0x%x)", where, e);
        return TC_ERR_TIMEOUT;
    }
    if (e & DEVERR_STACK) {
        set_error(TC_ERR_CAPACITY, "%s: traversal stack capacity exceeded (flags 0x%x)", where, e);
        return TC_ERR_CAPACITY;
    }
    if (e) {
        set_error(TC_ERR_CUDA, "%s: inconsistent tree bookkeeping or index out of bounds (flags 0x%x)",
                  where, e);
        return TC_ERR_CUDA;
    }
    return TC_OK;
}

static unsigned long long stat_counter(Context &c, int slot) {
    return reinterpret_cast<unsigned long long *>(c.h_pinned + 16)[slot];
}

int device_sm_count() {
    static const int sms = [] {
        int dev = 0, n = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        return n > 0 ? n : 148;
    }();
    return sms;
}

// The contexts' small page-locked read-back areas (4 KB each) come from slabs allocated once
// per process and recycled: cudaMallocHost per context cost a synchronising call on every
// context creation, which stalled the other contexts' work whenever a serving client arrived.
// A slab serves 256 contexts (a request server keeps hundreds of resident clients).
constexpr size_t PINNED_AREA = 4096, PINNED_SLAB = 256 * PINNED_AREA;
static std::mutex g_pinned_mu;
static std::vector<unsigned *> g_pinned_free;

static unsigned *pinned_area() {
    std::lock_guard<std::mutex> lock(g_pinned_mu);
    if (g_pinned_free.empty()) {
        void *slab = nullptr;
        if (cudaMallocHost(&slab, PINNED_SLAB) != cudaSuccess) return nullptr;
        for (size_t o = 0; o < PINNED_SLAB; o += PINNED_AREA)
            g_pinned_free.push_back(reinterpret_cast<unsigned *>(static_cast<char *>(slab) + o));
    }
    unsigned *a = g_pinned_free.back();
    g_pinned_free.pop_back();
    return a;
}

static void pinned_release(unsigned *a) {
    if (!a) return;
    std::lock_guard<std::mutex> lock(g_pinned_mu);
    g_pinned_free.push_back(a);
}

// Hands the pool blocks that no context holds back to the driver.
static cudaError_t release_pool_cache(int device) {
    cudaMemPool_t pool;
    cudaError_t e = cudaDeviceGetDefaultMemPool(&pool, device);
    return e == cudaSuccess ? cudaMemPoolTrimTo(pool, 0) : e;
}

// Freed pool blocks stay cached in the process for the next allocation (the default release
// threshold of 0 would hand them back to the driver at every synchronisation); set once per
// device.
static cudaError_t keep_pool_cache(int device) {
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lock(mu);
    if (std::find(done.begin(), done.end(), device) != done.end()) return cudaSuccess;
    cudaMemPool_t pool;
    cudaError_t e = cudaDeviceGetDefaultMemPool(&pool, device);
    if (e != cudaSuccess) return e;
    uint64_t keep = UINT64_MAX;
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e == cudaSuccess) done.push_back(device);
    return e;
}

// Live contexts per device.  Freed buffers stay cached in the device's pool while any context
// lives, for the next allocation of any of them: a trim at every context's end (a request
// server evicting idle clients) handed the memory back only for the next solve to map it anew.
// The last context of a device hands the cache back (tc_release_cached_memory does it at once).
static std::mutex g_live_mu;
static std::vector<int> g_live;

static void context_counted(int device, int delta) {
    std::lock_guard<std::mutex> lock(g_live_mu);
    if ((int)g_live.size() <= device) g_live.resize(device + 1, 0);
    g_live[device] += delta;
    if (g_live[device] == 0) release_pool_cache(device);
}

// Loads every kernel of the library on `device`, once per process.  Under lazy module loading
// (the CUDA default) a kernel is loaded at its first launch, and loading may synchronise the
// whole device: in the request server, the first solve of a form, order or list-walk mode not
// seen before stalled every concurrent solve.  Querying each kernel's attributes loads it, so
// the first context pays that cost at start-up instead.
static int preload_kernels(int device) {
    static std::mutex mu;
    static std::vector<int> loaded;
    std::lock_guard<std::mutex> lock(mu);
    if (std::find(loaded.begin(), loaded.end(), device) != loaded.end()) return TC_OK;
    KernelList v;
    kernels_sort(v);
    kernels_tree(v);
    kernels_upward(v);
    kernels_force(v);
    kernels_potential(v);
    kernels_direct(v);
    for (const void *k : v) {
        cudaFuncAttributes a;
        TC_CUDA_TRY(cudaFuncGetAttributes(&a, k));
    }
    loaded.push_back(device);
    return TC_OK;
}

static int context_init(Context &c, int device, cudaStream_t stream) {
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        set_error(TC_ERR_NO_DEVICE, "no CUDA device available (%s)",
                  e == cudaSuccess ? "device count 0" : cudaGetErrorString(e));
        return TC_ERR_NO_DEVICE;
    }
    if (device < 0) TC_CUDA_TRY(cudaGetDevice(&device));
    TC_CUDA_TRY(cudaSetDevice(device));
    c.device = device;
    if (int rc = preload_kernels(device)) return rc;
    if (stream) {
        c.stream = stream;
        c.own_stream = false;
    } else {
        // default priority: the main stream at the highest priority (the critical path) made a
        // single solve of the 16M sheet 2.6% faster in FP64 and no faster in the mixed form, but
        // with several contexts solving at once (the request server) every context's
        // auxiliary-stream work waited behind the others' main streams: the 2000-request
        // stream's p99 went from 0.2 to 1.6 s
        TC_CUDA_TRY(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
        c.own_stream = true;
    }
    TC_CUDA_TRY(keep_pool_cache(device));
    TC_CUDA_TRY(cudaStreamCreateWithFlags(&c.aux, cudaStreamNonBlocking));
    TC_CUDA_TRY(cudaEventCreateWithFlags(&c.ev_fork, cudaEventDisableTiming));
    TC_CUDA_TRY(cudaEventCreateWithFlags(&c.ev_totals, cudaEventDisableTiming));
    TC_CUDA_TRY(cudaEventCreateWithFlags(&c.ev_join, cudaEventDisableTiming));
    TC_CUDA_TRY(cudaEventCreateWithFlags(&c.ev_inputs, cudaEventDisableTiming));
    for (auto &ev : c.ev_chunk) TC_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    TC_CUDA_TRY(cudaEventCreateWithFlags(&c.ev_leafset, cudaEventDisableTiming));
    TC_CUDA_TRY(cudaEventCreateWithFlags(&c.ev_moments, cudaEventDisableTiming));
    TC_CUDA_TRY(cudaEventCreateWithFlags(&c.ev_near, cudaEventDisableTiming));
    TC_CUDA_TRY(cudaEventCreateWithFlags(&c.ev_serial, cudaEventDisableTiming));
    c.h_pinned = pinned_area();
    if (!c.h_pinned) {
        set_error(TC_ERR_ALLOC, "page-locked host allocation failed");
        return TC_ERR_ALLOC;
    }
    for (auto &ev : c.ev) TC_CUDA_TRY(cudaEventCreate(&ev));
    unsigned *err;
    unsigned long long *stats;
    int rc;
    if ((rc = ensure(c, S_ERR, 64, &err))) return rc;
    if ((rc = ensure(c, S_STATS, STAT_SLOTS, &stats))) return rc;
    TC_CUDA_TRY(cudaMemsetAsync(err, 0, 64 * sizeof(unsigned), c.stream));
    TC_CUDA_TRY(cudaMemsetAsync(stats, 0, STAT_SLOTS * sizeof(unsigned long long), c.stream));
    context_counted(device, +1);
    c.live = true;
    return TC_OK;
}

static void context_free(Context &c) {
    cudaSetDevice(c.device);
    if (c.stream) cudaStreamSynchronize(c.stream);
    if (c.aux) cudaStreamSynchronize(c.aux);
    // stream-ordered frees (cudaFree would synchronise the whole device)
    cudaStream_t fs = c.stream ? c.stream : c.aux;
    for (auto &b : c.buf)
        if (b.p) cudaFreeAsync(b.p, fs);
    if (fs) cudaStreamSynchronize(fs);
    if (c.live) context_counted(c.device, -1);
    c.live = false;
    for (auto &ev : c.ev)
        if (ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : {c.ev_fork, c.ev_totals, c.ev_join, c.ev_inputs, c.ev_leafset, c.ev_moments,
                           c.ev_near, c.ev_serial})
        if (ev) cudaEventDestroy(ev);
    for (auto &ev : c.ev_chunk)
        if (ev) cudaEventDestroy(ev);
    if (c.aux) cudaStreamDestroy(c.aux);
    pinned_release(c.h_pinned);
    c.h_pinned = nullptr;
    if (c.own_stream && c.stream) cudaStreamDestroy(c.stream);
}

static void finish_timing(Context &c) {
    if (!c.timing) return;
    wait_event(c, c.ev[5]);
    float t[6] = {};
    for (int i = 1; i <= 5; ++i) cudaEventElapsedTime(&t[i], c.ev[i - 1], c.ev[i]);
    c.times.sort_ms = t[1];
    c.times.tree_ms = t[2];
    c.times.upward_ms = t[3];
    c.times.lists_ms = t[4];
    c.times.eval_ms = t[5];
    float tot = 0;
    cudaEventElapsedTime(&tot, c.ev[0], c.ev[5]);
    c.times.total_ms = tot;
    // the evaluation kernel (potential), or the far-field kernel plus the near-field one
    // (force; the near field runs on the auxiliary stream, beside the upward pass)
    float k = 0, nk = 0;
    cudaEventElapsedTime(&k, c.ev[6], c.ev[7]);
    if (c.near_marked) cudaEventElapsedTime(&nk, c.ev[9], c.ev[10]);
    c.times.far_kernel_ms = c.near_marked ? k : 0.f;
    c.times.eval_kernel_ms = k + nk;
}

// Sort, topology and upward pass for `kind` (0 potential, 1 force).
// Sort, topology and the moments of every node for `kind` (0 potential, 1 force): all that the
// traversals read.  The expansions follow separately (upward_expansions), so that they can be
// formed while the interaction lists are built.
static int build_tree_moments(Context &c, int kind, const double *x, const double *y,
                              const double *v, int n, cudaEvent_t values_ready = nullptr) {
    int rc;
    g_launches = 0;
    c.near_marked = false;
    TC_CUDA_TRY(cudaMemsetAsync(slot_ptr<unsigned>(c, S_ERR), 0, sizeof(unsigned), c.stream));
    TC_CUDA_TRY(cudaMemsetAsync(c.buf[S_STATS].p, 0, STAT_SLOTS * sizeof(unsigned long long),
                                c.stream));
    if ((rc = sort_sources(c, x, y, v, n, values_ready))) return rc;
    phase_mark(c, 1);
    if ((rc = build_topology(c, kind ? LEAF_FORCE : LEAF_POTENTIAL))) return rc;
    if ((rc = finish_sources(c))) return rc;
    phase_mark(c, 2);
    if ((rc = upward_prepare(c, kind ? c.order_force : c.order_potential)) ||
        (rc = upward_moments(c)))
        return rc;
    return TC_OK;
}

// The whole tree with its expansions (tree inspection).
static int build_tree(Context &c, int kind, const double *x, const double *y, const double *v,
                      int n) {
    int rc;
    if ((rc = build_tree_moments(c, kind, x, y, v, n)) || (rc = upward_expansions(c))) return rc;
    phase_mark(c, 3);
    return TC_OK;
}

// Run on the main stream while the lists are built: the expansions, then the phase mark.
static int expansions_then_mark(Context &c) {
    const int rc = upward_expansions(c);
    phase_mark(c, 3);
    return rc;
}

static int potential_device(Context &c, double theta, const double *xs, const double *ys,
                            const double *vs, int n, const double *xt, const double *yt, int m,
                            double *out, cudaEvent_t values_ready = nullptr) {
    if (n < 0 || m < 0) {
        set_error(TC_ERR_INVALID, "negative size (nsources %d, ntargets %d)", n, m);
        return TC_ERR_INVALID;
    }
    if (m == 0) return TC_OK;
    if (n == 0) {
        TC_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(double) * m, c.stream));
        TC_CUDA_TRY(cudaStreamSynchronize(c.stream));
        return TC_OK;
    }
    int rc;
    phase_mark(c, 0);
    if ((rc = build_tree_moments(c, 0, xs, ys, vs, n, values_ready))) return rc;
    if ((rc = potential(c, theta, xt, yt, m, out, expansions_then_mark))) return rc;
    phase_mark(c, 5);
    if ((rc = check_device_errors(c, "treecode_potential"))) return rc;
    c.counts.e2p_pairs = (long long)stat_counter(c, STAT_E2P_PAIRS);
    c.counts.p2p_pairs = (long long)stat_counter(c, STAT_P2P_PAIRS);
    finish_timing(c);
    return TC_OK;
}

static int force_device(Context &c, double theta, const double *xs, const double *ys,
                        const double *vs, int n, const double *x0s, const double *y0s,
                        const double *hs, int nb, double *xo, double *yo,
                        cudaEvent_t values_ready = nullptr, double *host_x = nullptr,
                        double *host_y = nullptr) {
    c.host_copied = false;
    if (n < 0 || nb < 0) {
        set_error(TC_ERR_INVALID, "negative size (nsources %d, nblocks %d)", n, nb);
        return TC_ERR_INVALID;
    }
    if (nb == 0) return TC_OK;
    if (nb > (1 << 30) / (c.blocksize * c.blocksize)) {
        set_error(TC_ERR_INVALID, "too many blocks (%d)", nb);
        return TC_ERR_INVALID;
    }
    const size_t nt = (size_t)nb * c.blocksize * c.blocksize;
    if (n == 0) {
        TC_CUDA_TRY(cudaMemsetAsync(xo, 0, sizeof(double) * nt, c.stream));
        TC_CUDA_TRY(cudaMemsetAsync(yo, 0, sizeof(double) * nt, c.stream));
        TC_CUDA_TRY(cudaStreamSynchronize(c.stream));
        return TC_OK;
    }
    int rc;
    phase_mark(c, 0);
    if ((rc = build_tree_moments(c, 1, xs, ys, vs, n, values_ready))) return rc;
    if ((rc = force_mrag(c, theta, x0s, y0s, hs, nb, xo, yo, expansions_then_mark, host_x,
                         host_y)))
        return rc;
    phase_mark(c, 5);
    if ((rc = check_device_errors(c, "treecode_force_mrag"))) return rc;
    c.counts.p2p_pairs = (long long)stat_counter(c, STAT_P2P_SOURCES) * TILE * TILE;
    finish_timing(c);
    return TC_OK;
}

template <class T>
static int stage(Context &c, Slot s, const T *host, size_t n, T **dev) {
    int rc;
    if ((rc = ensure(c, s, n, dev))) return rc;
    if (n) TC_CUDA_TRY(cudaMemcpyAsync(*dev, host, sizeof(T) * n, cudaMemcpyHostToDevice, c.stream));
    return TC_OK;
}

// Host inputs in two parts: what the key sort needs first (x, y and anything `first` names)
// on the main stream, then the source values and `later` arrays on the auxiliary stream once
// the first part has been copied (one link, so the copies do not share it).  The solve's key
// sort and tree build run while the later part is still in flight; c.ev_inputs marks the
// values' arrival.  The buffers are allocated on the main stream before either copy.
struct StagedArray {
    Slot slot;
    const double *host;
    size_t n;
    double **dev;
};

static int stage_split(Context &c, std::initializer_list<StagedArray> first,
                       std::initializer_list<StagedArray> later) {
    int rc;
    for (const StagedArray &a : first)
        if ((rc = stage(c, a.slot, a.host, a.n, a.dev))) return rc;
    for (const StagedArray &a : later)
        if ((rc = ensure(c, a.slot, a.n, a.dev))) return rc;
    TC_CUDA_TRY(cudaEventRecord(c.ev_fork, c.stream));
    TC_CUDA_TRY(cudaStreamWaitEvent(c.aux, c.ev_fork, 0));
    bool values = true;
    for (const StagedArray &a : later) {
        if (a.n)
            TC_CUDA_TRY(cudaMemcpyAsync(*a.dev, a.host, sizeof(double) * a.n,
                                        cudaMemcpyHostToDevice, c.aux));
        if (values) TC_CUDA_TRY(cudaEventRecord(c.ev_inputs, c.aux));   // after the values
        values = false;
    }
    return TC_OK;
}

// Error return of a host entry point after staging began: copies already queued on either
// stream may still read the caller's memory, so both streams are waited for before returning.
static int drain_and_fail(Context &c, int rc) {
    wait_stream(c, c.aux);
    wait_stream(c, c.stream);
    return rc;
}

static int potential_host(Context &c, double theta, const double *xs, const double *ys,
                          const double *vs, int n, const double *xt, const double *yt, int m,
                          double *out) {
    if (n < 0 || m < 0 || (m > 0 && (!xt || !yt || !out)) || (n > 0 && (!xs || !ys || !vs))) {
        set_error(TC_ERR_INVALID, "invalid arguments (nsources %d, ntargets %d)", n, m);
        return TC_ERR_INVALID;
    }
    if (m == 0) return TC_OK;
    int rc;
    double *dx, *dy, *dv, *dxt, *dyt, *dout;
    // the targets follow the values on the auxiliary stream, where the target sort runs
    if ((rc = stage_split(c, {{S_XIN, xs, (size_t)n, &dx}, {S_YIN, ys, (size_t)n, &dy}},
                          {{S_VIN, vs, (size_t)n, &dv}, {S_XT, xt, (size_t)m, &dxt},
                           {S_YT, yt, (size_t)m, &dyt}})) ||
        (rc = ensure(c, S_OUTX, m, &dout)))
        return drain_and_fail(c, rc);
    rc = potential_device(c, theta, dx, dy, dv, n, dxt, dyt, m, dout, c.ev_inputs);
    // the copies on the auxiliary stream read the caller's memory: done before returning
    const cudaError_t e = wait_stream(c, c.aux);
    if (rc) return rc;
    TC_CUDA_TRY(e);
    TC_CUDA_TRY(cudaMemcpyAsync(out, dout, sizeof(double) * m, cudaMemcpyDeviceToHost, c.stream));
    TC_CUDA_TRY(wait_stream(c, c.stream));
    return TC_OK;
}

static int force_host(Context &c, double theta, const double *xs, const double *ys,
                      const double *vs, int n, const double *x0s, const double *y0s,
                      const double *hs, int nb, double *xo, double *yo) {
    if (n < 0 || nb < 0 || (nb > 0 && (!x0s || !y0s || !hs || !xo || !yo)) ||
        (n > 0 && (!xs || !ys || !vs))) {
        set_error(TC_ERR_INVALID, "invalid arguments (nsources %d, nblocks %d)", n, nb);
        return TC_ERR_INVALID;
    }
    if (nb == 0) return TC_OK;
    int rc;
    const size_t nt = (size_t)nb * c.blocksize * c.blocksize;
    double *dx, *dy, *dv, *d0x, *d0y, *dh, *dox, *doy;
    if ((rc = stage_split(c, {{S_XIN, xs, (size_t)n, &dx}, {S_YIN, ys, (size_t)n, &dy},
                              {S_X0, x0s, (size_t)nb, &d0x}, {S_Y0, y0s, (size_t)nb, &d0y},
                              {S_H, hs, (size_t)nb, &dh}},
                          {{S_VIN, vs, (size_t)n, &dv}})) ||
        (rc = ensure(c, S_OUTX, nt, &dox)) || (rc = ensure(c, S_OUTY, nt, &doy)))
        return drain_and_fail(c, rc);
    // the outputs come back run by run while later runs are evaluated (force_mrag)
    rc = force_device(c, theta, dx, dy, dv, n, d0x, d0y, dh, nb, dox, doy, c.ev_inputs, xo, yo);
    const cudaError_t e = wait_stream(c, c.aux);
    if (rc) return rc;
    TC_CUDA_TRY(e);
    if (!c.host_copied) {
        TC_CUDA_TRY(cudaMemcpyAsync(xo, dox, sizeof(double) * nt, cudaMemcpyDeviceToHost, c.stream));
        TC_CUDA_TRY(cudaMemcpyAsync(yo, doy, sizeof(double) * nt, cudaMemcpyDeviceToHost, c.stream));
    }
    TC_CUDA_TRY(wait_stream(c, c.stream));
    return TC_OK;
}

// Per-thread default context of the reference-compatible entry points.
struct TlsContext {
    Context *c = nullptr;
    ~TlsContext() {
        if (c) {
            context_free(*c);
            delete c;
        }
    }
};
static thread_local TlsContext tls_ctx;

static Context *default_context() {
    if (!tls_ctx.c) {
        Context *c = new Context();
        if (context_init(*c, -1, nullptr) != TC_OK) {
            delete c;
            return nullptr;
        }
        tls_ctx.c = c;
    }
    return tls_ctx.c;
}

static void report_failure(const char *fn) {
    // The reference signatures return void; a failed solve is reported on stderr as well as
    // through treecode_last_status(), so it cannot pass unnoticed.
    fprintf(stderr, "%s failed (status %d): %s\n", fn, tls_status, tls_msg);
}

}  // namespace tc

struct tc_context {
    tc::Context c;
};

using namespace tc;

extern "C" {

TC_API void treecode_potential(const double theta, const double *const xsources,
                               const double *const ysources, const double *const sourcevalues,
                               const int nsources, const double *const xtargets,
                               const double *const ytargets, const int ntargets,
                               double *const targetvalues) {
    clear_error();
    Context *c = default_context();
    if (!c || potential_host(*c, theta, xsources, ysources, sourcevalues, nsources, xtargets,
                             ytargets, ntargets, targetvalues) != TC_OK)
        report_failure("treecode_potential");
}

TC_API void treecode_force_mrag(const double theta, const double *const xsources,
                                const double *const ysources, const double *const sourcevalues,
                                const int nsources, const double *const x0s,
                                const double *const y0s, const double *const hs,
                                const int nblocks, double *const xresults,
                                double *const yresults) {
    clear_error();
    Context *c = default_context();
    if (!c || force_host(*c, theta, xsources, ysources, sourcevalues, nsources, x0s, y0s, hs,
                         nblocks, xresults, yresults) != TC_OK)
        report_failure("treecode_force_mrag");
}

TC_API int treecode_last_status(void) { return tls_status; }
TC_API const char *treecode_last_error(void) { return tls_msg; }

TC_API int tc_context_create(tc_context **ctx, int device, void *cuda_stream) {
    clear_error();
    if (!ctx) {
        set_error(TC_ERR_INVALID, "ctx is NULL");
        return TC_ERR_INVALID;
    }
    tc_context *t = new tc_context();
    int rc = context_init(t->c, device, (cudaStream_t)cuda_stream);
    if (rc) {
        context_free(t->c);
        delete t;
        *ctx = nullptr;
        return rc;
    }
    *ctx = t;
    return TC_OK;
}

TC_API void tc_context_destroy(tc_context *ctx) {
    if (!ctx) return;
    context_free(ctx->c);
    delete ctx;
}

TC_API int tc_set_precision(tc_context *ctx, int precision) {
    clear_error();
    if (!ctx || precision < 0 || precision > 1) {
        set_error(TC_ERR_INVALID, "invalid precision mode %d", precision);
        return TC_ERR_INVALID;
    }
    ctx->c.precision = precision;
    return TC_OK;
}

TC_API int tc_set_host_waits(tc_context *ctx, int sleeping) {
    clear_error();
    if (!ctx || sleeping < 0 || sleeping > 1) {
        set_error(TC_ERR_INVALID, "invalid host wait mode %d", sleeping);
        return TC_ERR_INVALID;
    }
    ctx->c.sleeping_waits = sleeping != 0;
    return TC_OK;
}

TC_API int tc_set_launch_overlap(tc_context *ctx, int on) {
    clear_error();
    if (!ctx || on < 0 || on > 1) {
        set_error(TC_ERR_INVALID, "invalid launch overlap setting %d", on);
        return TC_ERR_INVALID;
    }
    ctx->c.launch_overlap = on != 0;
    return TC_OK;
}

TC_API int tc_set_wait_test(tc_context *ctx, int stall, int spin_limit, int stack_limit) {
    clear_error();
    if (!ctx || stall < TC_STALL_NONE || stall > TC_STALL_TREE) {
        set_error(TC_ERR_INVALID, "invalid wait test setting (stall %d)", stall);
        return TC_ERR_INVALID;
    }
    ctx->c.test_stall = stall;
    ctx->c.spin_limit = spin_limit > 0 ? spin_limit : DEFAULT_SPIN_LIMIT;
    ctx->c.stack_limit = stack_limit > 0 ? stack_limit : 0;
    return TC_OK;
}

TC_API int tc_set_orders(tc_context *ctx, int potential_order, int force_order) {
    clear_error();
    if (!ctx) {
        set_error(TC_ERR_INVALID, "no context");
        return TC_ERR_INVALID;
    }
    int rc;
    if ((rc = dispatch_order(potential_order, [](auto) -> int { return TC_OK; })) ||
        (rc = dispatch_order(force_order, [](auto) -> int { return TC_OK; })))
        return rc;
    ctx->c.order_potential = potential_order;
    ctx->c.order_force = force_order;
    return TC_OK;
}

TC_API int tc_set_blocksize(tc_context *ctx, int blocksize) {
    clear_error();
    if (!ctx || (blocksize != 8 && blocksize != 16 && blocksize != 32 && blocksize != 64)) {
        set_error(TC_ERR_INVALID, "unsupported MRAG block size %d (8, 16, 32 or 64)", blocksize);
        return TC_ERR_INVALID;
    }
    ctx->c.blocksize = blocksize;
    return TC_OK;
}

TC_API int tc_supported_orders(int *orders, int capacity) {
    static const int list[] = {
#define TC_ORDER_ITEM(P) P,
        TC_FOR_EACH_ORDER(TC_ORDER_ITEM)
#undef TC_ORDER_ITEM
    };
    const int n = (int)(sizeof(list) / sizeof(list[0]));
    for (int i = 0; i < n && i < capacity; ++i)
        if (orders) orders[i] = list[i];
    return n;
}

TC_API int tc_set_timing(tc_context *ctx, int enabled) {
    if (!ctx || enabled < 0 || enabled > 2) return TC_ERR_INVALID;
    ctx->c.timing = enabled != 0;
    ctx->c.serial_eval = enabled == 2;
    return TC_OK;
}

TC_API void *tc_get_stream(tc_context *ctx) { return ctx ? (void *)ctx->c.stream : nullptr; }

TC_API size_t tc_context_device_bytes(tc_context *ctx) {
    if (!ctx) return 0;
    size_t b = 0;
    for (const auto &d : ctx->c.buf) b += d.bytes;
    return b;
}

TC_API int tc_context_trim(tc_context *ctx) {
    if (!ctx) return TC_ERR_INVALID;
    Context &c = ctx->c;
    cudaSetDevice(c.device);
    TC_CUDA_TRY(cudaStreamSynchronize(c.stream));
    TC_CUDA_TRY(cudaStreamSynchronize(c.aux));
    for (int s = 0; s < S_NUM_SLOTS; ++s) {
        if (s == S_ERR || s == S_STATS) continue;   // created with the context, tiny
        DevBuf &b = c.buf[s];
        if (b.p) cudaFreeAsync(b.p, c.stream);   // no device-wide synchronisation
        b.p = nullptr;
        b.bytes = 0;
    }
    TC_CUDA_TRY(cudaStreamSynchronize(c.stream));
    c.nnodes = c.nsrc = 0;
    return TC_OK;
}

TC_API int tc_reserve_cached_memory(int device, size_t bytes) {
    clear_error();
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) return TC_ERR_NO_DEVICE;
    TC_CUDA_TRY(cudaSetDevice(device));
    TC_CUDA_TRY(keep_pool_cache(device));
    size_t free_b = 0, total_b = 0;
    TC_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    const size_t margin = (size_t)2 << 30;   // left to the driver and to other allocators
    bytes = std::min(bytes, free_b > margin ? free_b - margin : 0);
    if (bytes == 0) return TC_OK;
    cudaStream_t s;
    TC_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    void *p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, bytes, s);
    if (e == cudaSuccess) e = cudaFreeAsync(p, s);
    const cudaError_t es = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (e != cudaSuccess || es != cudaSuccess) {
        cudaGetLastError();
        set_error(TC_ERR_ALLOC, "reserving %zu bytes in the device pool failed: %s", bytes,
                  cudaGetErrorString(e != cudaSuccess ? e : es));
        return TC_ERR_ALLOC;
    }
    return TC_OK;
}

TC_API int tc_release_cached_memory(int device) {
    clear_error();
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) return TC_ERR_NO_DEVICE;
    TC_CUDA_TRY(cudaSetDevice(device));
    TC_CUDA_TRY(release_pool_cache(device));
    return TC_OK;
}

TC_API int tc_get_stats(tc_context *ctx, tc_stats *out) {
    if (!ctx || !out) return TC_ERR_INVALID;
    const Context &c = ctx->c;
    out->sort_ms = c.times.sort_ms;
    out->tree_ms = c.times.tree_ms;
    out->upward_ms = c.times.upward_ms;
    out->lists_ms = c.times.lists_ms;
    out->eval_ms = c.times.eval_ms;
    out->total_ms = c.times.total_ms;
    out->nnodes = c.counts.nnodes;
    out->nleaves = c.counts.nleaves;
    out->ninner = c.counts.ninner;
    out->nlevels = c.counts.nlevels;
    out->n_e2l = c.counts.n_e2l;
    out->n_e2p = c.counts.n_e2p;
    out->n_p2p = c.counts.n_p2p;
    out->p2p_pairs = c.counts.p2p_pairs;
    out->e2p_pairs = c.counts.e2p_pairs;
    out->e2l_pairs = c.counts.e2l_pairs;
    out->l2p_targets = c.counts.l2p_targets;
    out->launches = c.counts.launches;
    out->eval_kernel_ms = c.times.eval_kernel_ms;
    out->list_walks = c.list_walks;
    out->far_kernel_ms = c.times.far_kernel_ms;
    return TC_OK;
}

#define CTX_GUARD()                                             \
    clear_error();                                              \
    if (!ctx) {                                                 \
        set_error(TC_ERR_INVALID, "context is NULL");           \
        return TC_ERR_INVALID;                                  \
    }                                                           \
    cudaSetDevice(ctx->c.device)

TC_API int tc_potential_host(tc_context *ctx, double theta, const double *xs, const double *ys,
                             const double *vs, int n, const double *xt, const double *yt, int m,
                             double *out) {
    CTX_GUARD();
    return potential_host(ctx->c, theta, xs, ys, vs, n, xt, yt, m, out);
}

TC_API int tc_force_mrag_host(tc_context *ctx, double theta, const double *xs, const double *ys,
                              const double *vs, int n, const double *x0s, const double *y0s,
                              const double *hs, int nb, double *xo, double *yo) {
    CTX_GUARD();
    return force_host(ctx->c, theta, xs, ys, vs, n, x0s, y0s, hs, nb, xo, yo);
}

TC_API int tc_potential_device(tc_context *ctx, double theta, const double *xs, const double *ys,
                               const double *vs, int n, const double *xt, const double *yt,
                               int m, double *out) {
    CTX_GUARD();
    return potential_device(ctx->c, theta, xs, ys, vs, n, xt, yt, m, out);
}

TC_API int tc_force_mrag_device(tc_context *ctx, double theta, const double *xs,
                                const double *ys, const double *vs, int n, const double *x0s,
                                const double *y0s, const double *hs, int nb, double *xo,
                                double *yo) {
    CTX_GUARD();
    return force_device(ctx->c, theta, xs, ys, vs, n, x0s, y0s, hs, nb, xo, yo);
}

TC_API int tc_tree_build_device(tc_context *ctx, int kind, const double *xs, const double *ys,
                                const double *vs, int n) {
    CTX_GUARD();
    if (n <= 0 || (kind != 0 && kind != 1)) {
        set_error(TC_ERR_INVALID, "invalid tree request (kind %d, n %d)", kind, n);
        return TC_ERR_INVALID;
    }
    int rc = build_tree(ctx->c, kind, xs, ys, vs, n);
    if (rc) return rc;
    return check_device_errors(ctx->c, "tc_tree_build_device");
}

TC_API int tc_tree_size(tc_context *ctx, int *nnodes, int *order, int *nsources) {
    CTX_GUARD();
    if (nnodes) *nnodes = ctx->c.nnodes;
    if (order) *order = ctx->c.order;
    if (nsources) *nsources = ctx->c.nsrc;
    return TC_OK;
}

TC_API int tc_tree_copy(tc_context *ctx, int *keys, int *perm, double *xs, double *ys,
                        double *vs, double *frame, int *s, int *e, int *child, int *count,
                        int *level, int *cx, int *cy, int *parent, double *mass, double *xcom,
                        double *ycom, double *r, double *exps) {
    CTX_GUARD();
    Context &c = ctx->c;
    const int n = c.nsrc, nn = c.nnodes;
    auto d2h = [&](void *dst, const void *src, size_t bytes) {
        return cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost);
    };
    TC_CUDA_TRY(cudaStreamSynchronize(c.stream));
    if (keys) TC_CUDA_TRY(d2h(keys, c.buf[S_KEYS].p, sizeof(int) * n));
    if (perm) TC_CUDA_TRY(d2h(perm, c.buf[S_PERM].p, sizeof(int) * n));
    if (xs) TC_CUDA_TRY(d2h(xs, c.buf[S_XS].p, sizeof(double) * n));
    if (ys) TC_CUDA_TRY(d2h(ys, c.buf[S_YS].p, sizeof(double) * n));
    if (vs) TC_CUDA_TRY(d2h(vs, c.buf[S_VS].p, sizeof(double) * n));
    if (frame) {
        Frame f;
        TC_CUDA_TRY(d2h(&f, c.buf[S_FRAME].p, sizeof(Frame)));
        frame[0] = f.xmin;
        frame[1] = f.ymin;
        frame[2] = f.ext;
    }
    if (s || e || child || count || level || cx || cy || parent || xcom || ycom || r) {
        TNode *tn = new TNode[nn];
        int2 *rg = new int2[nn];
        int4 *cl = new int4[nn];
        cudaError_t err = d2h(tn, c.buf[S_TNODE].p, sizeof(TNode) * nn);
        if (err == cudaSuccess) err = d2h(rg, c.buf[S_RANGE].p, sizeof(int2) * nn);
        if (err == cudaSuccess) err = d2h(cl, c.buf[S_CELL].p, sizeof(int4) * nn);
        if (err == cudaSuccess)
            for (int i = 0; i < nn; ++i) {
                // a leaf emptied by the all-negligible rule keeps its range for the upward
                // pass; report it as the reference does, s = e = 0 (upward.cpp:179)
                const bool emptied = tn[i].child < 0 && tn[i].count == 0 && rg[i].y > rg[i].x;
                if (s) s[i] = emptied ? 0 : rg[i].x;
                if (e) e[i] = emptied ? 0 : rg[i].y;
                if (child) child[i] = tn[i].child;
                if (count) count[i] = tn[i].count;
                if (level) level[i] = cl[i].x;
                if (cx) cx[i] = cl[i].y;
                if (cy) cy[i] = cl[i].z;
                if (parent) parent[i] = cl[i].w;
                if (xcom) xcom[i] = tn[i].xcom;
                if (ycom) ycom[i] = tn[i].ycom;
                if (r) r[i] = tn[i].r;
            }
        delete[] tn;
        delete[] rg;
        delete[] cl;
        TC_CUDA_TRY(err);
    }
    if (mass) TC_CUDA_TRY(d2h(mass, c.buf[S_MASS].p, sizeof(double) * nn));
    if (exps) TC_CUDA_TRY(d2h(exps, c.buf[S_EXPS].p, sizeof(double) * nn * 2 * c.order));
    return TC_OK;
}

TC_API int tc_direct_potential_device(tc_context *ctx, const double *xs, const double *ys,
                                      const double *vs, int n, const double *xt,
                                      const double *yt, int m, double *out) {
    CTX_GUARD();
    int rc = direct_potential(ctx->c, xs, ys, vs, n, xt, yt, m, out);
    if (rc) return rc;
    TC_CUDA_TRY(cudaStreamSynchronize(ctx->c.stream));
    return TC_OK;
}

TC_API int tc_log_probe_device(tc_context *ctx, const double *x, int n, double *out) {
    CTX_GUARD();
    int rc = log_probe(ctx->c, x, n, out);
    if (rc) return rc;
    TC_CUDA_TRY(cudaStreamSynchronize(ctx->c.stream));
    return TC_OK;
}

TC_API int tc_direct_force_device(tc_context *ctx, const double *xs, const double *ys,
                                  const double *vs, int n, const double *xt, const double *yt,
                                  int m, double *xo, double *yo) {
    CTX_GUARD();
    int rc = direct_force(ctx->c, xs, ys, vs, n, xt, yt, m, xo, yo);
    if (rc) return rc;
    TC_CUDA_TRY(cudaStreamSynchronize(ctx->c.stream));
    return TC_OK;
}

TC_API int tc_measure_fma_peak(int fp64, double *tflops) {
    clear_error();
    if (!tflops) return TC_ERR_INVALID;
    return measure_fma_peak(fp64, tflops);
}

TC_API const char *tc_version(void) { return "2d-treecodes-b200 0.1 (sm_100a)"; }

}  // extern "C"
