// tc_internal.h -- host-side state of one treecode context and the entry points shared
// between the translation units of the library.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "tc_common.cuh"

namespace tc {

// Grow-only device allocation.  A context keeps its buffers between calls, so repeated
// solves of similar size allocate nothing.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

enum Slot {
    // inputs staged from host memory
    S_XIN, S_YIN, S_VIN, S_XT, S_YT, S_X0, S_Y0, S_H, S_OUTX, S_OUTY,
    // sorted sources
    S_XS, S_YS, S_VS, S_KEYS, S_PERM, S_FRAME, S_ITEMS_A, S_ITEMS_B, S_REC,
    // radix sort scratch
    S_RS_STATUS, S_RS_HIST, S_RS_COUNTER,
    // scan scratch
    S_SCAN_BLOCKS,
    // tree build
    S_TMASK, S_TFLAG, S_TOFF, S_LPOS, S_LMASK, S_LRANK, S_LINV, S_LBLK, S_LEVEL_TOTALS,
    // nodes
    S_TNODE, S_RANGE, S_CELL, S_MASS, S_W, S_WX, S_WY, S_EXPS, S_UPCNT,
    // force traversal / lists
    S_FCOUNT, S_FOFF, S_E2L, S_E2P, S_P2P, S_BRICK_CTR, S_FPART, S_SEXP, S_SSCALE, S_TASKMAP,
    S_LSTART, S_LMETA, S_FARX, S_FARY, S_FAR_CTR,
    // potential targets / lists
    S_TKEYS, S_TPERM, S_TKEYS2, S_TPERM2, S_PCOUNT, S_POFF, S_PE2P, S_PP2P,
    // misc
    S_ERR, S_STATS,
    S_NUM_SLOTS
};

// First node id of each level (breadth-first numbering): level l occupies [off[l], off[l+1]),
// off[LMAX + 1] = number of nodes.  Passed to kernels by value.
struct LevelOffsets {
    int off[LMAX + 3];
};

struct PhaseTimes {
    float sort_ms, tree_ms, upward_ms, lists_ms, eval_ms, total_ms, eval_kernel_ms, far_kernel_ms;
};

struct Counts {
    long long nnodes, nleaves, ninner, nlevels;
    long long n_e2l, n_e2p, n_p2p;        // interaction-list entries
    long long p2p_pairs;                  // source-target pairs evaluated directly
    long long e2p_pairs;                  // (target, cell) pairs of far-field evaluation
    long long e2l_pairs;                  // (brick, cell) pairs of local-expansion builds
    long long l2p_targets;                // targets evaluated from a local expansion
    long long launches;                   // kernels launched by the last solve
};

// Device-side work counters (unsigned long long each) in the S_STATS slot.
enum { STAT_P2P_SOURCES = 0, STAT_E2P_PAIRS = 1, STAT_P2P_PAIRS = 2, STAT_SLOTS = 8 };

// Expansion orders a context can be set to (tc_set_orders).  The reference fixes its orders at
// build time (Makefile:13-14 of the reference: 12 for the potential, 24 for the force); here
// every order-dependent kernel is instantiated for each order of this list.  28 is the
// largest order whose E2L binomials C(2p - 1, p - 1) are exact in FP64.
#define TC_FOR_EACH_ORDER(X) X(4) X(8) X(12) X(16) X(20) X(24) X(28)

// f(std::integral_constant<int, p>) for a supported order p; TC_ERR_INVALID otherwise.
template <class F>
int dispatch_order(int p, F &&f) {
    switch (p) {
#define TC_ORDER_CASE(P) \
    case P:              \
        return f(std::integral_constant<int, P>{});
        TC_FOR_EACH_ORDER(TC_ORDER_CASE)
#undef TC_ORDER_CASE
    default:
        set_error(TC_ERR_INVALID, "unsupported expansion order %d", p);
        return TC_ERR_INVALID;
    }
}

// Per-warp scratch regions of a one-walk list build: kind k of warp w holds cap[k] entries from
// koff[k] + w cap[k] on.
struct ScratchLayout {
    int cap[3];
    int koff[3];
};

struct Context;
// Regions for `nkinds` kinds, `nwarps` warps and `nitems` bricks / groups, from the context's
// learned sizes, at most `max_entries` entries in all (smaller regions when they do not fit);
// returns the entries used.
long long scratch_layout(const Context &c, int nkinds, int nwarps, int nitems,
                         long long max_entries, ScratchLayout &s);
// Scratch of a one-walk list build: the sort's record buffer (32 B per source, dead once the
// sources are gathered) when the regions fit in it, else a transient block from the device's
// pool (at most 2 GB), allocated on the context's current stream and released on it, in
// stream order, when the guard goes out of scope after the last use has been enqueued.
struct ListScratch {
    void *p = nullptr;
    bool owned = false;
    cudaStream_t stream = nullptr;
    ~ListScratch();
};
int list_scratch(Context &c, int nkinds, int nwarps, int nitems, size_t entry_bytes,
                 ScratchLayout &sl, ListScratch &out);
// Raises the learned sizes from a build's per-kind longest runs (meta[1..nkinds]).
void scratch_learn(Context &c, int nkinds, int nwarps, int nitems, const unsigned *longest);

struct Context {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // kernel chains launched with programmatic dependent launch (launch_pdl); the request
    // server turns it off for its contexts (tc_set_launch_overlap)
    bool launch_overlap = true;
    // auxiliary stream: interaction lists are built on it while the expansions are formed on
    // `stream`; ordered against `stream` with the events below
    cudaStream_t aux = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_totals = nullptr, ev_join = nullptr;
    // host entry points: x/y are copied on `stream`, v (and targets) on `aux` after them;
    // ev_inputs marks v's arrival
    cudaEvent_t ev_inputs = nullptr;
    cudaEvent_t ev_chunk[4] = {};        // force output runs ready for their host copy
    cudaEvent_t ev_leafset = nullptr;     // leaf moments written (main stream)
    cudaEvent_t ev_moments = nullptr;     // parent moments written (auxiliary stream)
    cudaEvent_t ev_near = nullptr;        // force near field written (auxiliary stream)
    cudaEvent_t ev_serial = nullptr;      // main stream's work so far (serial_eval)
    bool host_copied = false;
    // a source sort whose values arrive late (sort_sources / finish_sources)
    const double *late_x = nullptr, *late_y = nullptr, *late_v = nullptr;
    cudaEvent_t late_ready = nullptr;
    DevBuf buf[S_NUM_SLOTS];
    unsigned *h_pinned = nullptr;         // small pinned staging area for readbacks
    int precision = 0;                    // 0 = plain FP64, 1 = mixed
    int order_potential = ORDER_POTENTIAL;  // expansion orders of the next solves
    int order_force = ORDER_FORCE;
    int blocksize = BLOCKSIZE;            // MRAG block side of the force entry points
    // one-walk list builds: entries per brick / target group and list kind that a warp's
    // scratch region is sized for, raised after every solve to what it needed
    int list_per_item[3] = {32, 32, 32};
    int list_walks = 0;                   // walks the last list build took (1 or 2)
    // host waits of a solve: spin in the CUDA call (false) or poll and sleep (wait_stream)
    bool sleeping_waits = false;
    bool live = false;                    // counted among the device's live contexts
    // test settings (tc_set_wait_test): a look-back tile that never publishes (TC_STALL_*),
    // the bound of the device waits, and the force traversal's stack capacity (0: full)
    int test_stall = TC_STALL_NONE;
    int spin_limit = DEFAULT_SPIN_LIMIT;
    int stack_limit = 0;
    bool timing = false;
    // a measurement mode: the force's near- and far-field kernels run one after the other,
    // after the upward pass, each alone on the GPU, so their events time each kernel by itself
    bool serial_eval = false;
    // phase events: 0-5 the phases, 6/7 the evaluation kernel (the far field of a force
    // solve), 9/10 the force's near field on the auxiliary stream
    cudaEvent_t ev[11] = {};
    bool near_marked = false;             // ev[9], ev[10] recorded in this solve
    PhaseTimes times = {};
    Counts counts = {};

    // current tree
    int nsrc = 0, order = 0, leafcap = 0;
    int nnodes = 0, ninner = 0;
    int level_off[LMAX + 3] = {};         // node id of the first node of each level
    Frame frame_h = {};
};

// Buffers come from the device's stream-ordered pool (cudaMallocAsync on the context's current
// stream): growing one frees the old block in stream order instead of synchronising the device,
// and a context created or grown while other contexts compute does not stall them.  Work on the
// auxiliary stream is ordered against the main stream by events, so a block freed on either
// stream is no longer in use on the other.
template <class T>
int ensure(Context &c, Slot s, size_t count, T **out) {
    size_t need = count * sizeof(T);
    if (need == 0) need = sizeof(T);
    DevBuf &b = c.buf[s];
    if (b.bytes < need) {
        if (b.p) {
            cudaFreeAsync(b.p, c.stream);
            b.p = nullptr;
            b.bytes = 0;
        }
        size_t alloc = need + need / 8;   // headroom for the next call
        cudaError_t e = cudaMallocAsync(&b.p, alloc, c.stream);
        if (e != cudaSuccess) {
            b.p = nullptr;
            set_error(TC_ERR_ALLOC, "cudaMallocAsync(%zu bytes) failed: %s", alloc,
                      cudaGetErrorString(e));
            return TC_ERR_ALLOC;
        }
        b.bytes = alloc;
    }
    *out = static_cast<T *>(b.p);
    return TC_OK;
}

template <class T>
T *slot_ptr(Context &c, Slot s) { return static_cast<T *>(c.buf[s].p); }

// Streaming multiprocessors of the current device (queried once; thread-safe).
int device_sm_count();

// Launches `kernel` on `s` with programmatic stream serialization when `overlap` is set (the
// context's launch_overlap): its blocks may be scheduled while the previous kernel of `s`
// drains, and wait in pdl_begin() (the kernel's first statement) until that kernel has
// completed.  Otherwise an ordinary launch.  Follow with TC_KERNEL_CHECK().
template <class... P, class... A>
cudaError_t launch_pdl(bool overlap, void (*kernel)(P...), dim3 grid, dim3 block, size_t smem,
                       cudaStream_t s, A &&...args) {
    if (!overlap) {
        kernel<<<grid, block, smem, s>>>(std::forward<A>(args)...);
        return cudaSuccess;   // (TC_KERNEL_CHECK reads the launch error)
    }
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr.val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

// Resident blocks per SM of a kernel at a block size and dynamic shared memory size, computed
// once per kernel instance (thread-safe initialisation of a function-local static).
template <auto Kernel>
int blocks_per_sm(int threads, size_t smem) {
    static const int occ = [&] {
        int o = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, Kernel, threads, smem);
        return o > 0 ? o : 1;
    }();
    return occ;
}

// ---- sort.cu
int exclusive_scan(Context &c, const int *d_in, int *d_out, int n);   // d_out has n+1 entries
int radix_sort_pairs(Context &c, const int *keys_in, const int *vals_in, int n, int nbits,
                     int *keys_a, int *vals_a, int *keys_b, int *vals_b, int **keys_out,
                     int **vals_out);
// Sorts the sources.  With `values_ready`, an event that completes once v is in device memory,
// v is read only by finish_sources() after a wait on that event, so that the key sort and the
// tree build run while v is still being copied in; without it x/y/v are all sorted here and
// finish_sources() does nothing.
int sort_sources(Context &c, const double *x, const double *y, const double *v, int n,
                 cudaEvent_t values_ready = nullptr);
int finish_sources(Context &c);
int target_keys(Context &c, const double *xt, const double *yt, int m, int *keys, int *idx);

// ---- tree.cu
int build_topology(Context &c, int leafcap);

// ---- upward.cu
int upward_prepare(Context &c, int order);   // buffers of the upward pass, c.order
int upward_moments(Context &c);              // leaf setup + parent moments (what traversals read)
int upward_expansions(Context &c);           // P2E + E2E
int upward_pass(Context &c, int order);      // all three

// Swaps the context's main and auxiliary streams for the lifetime of the object, so that the
// helpers (which all launch on c.stream) run on the auxiliary stream.
struct AuxScope {
    Context &c;
    explicit AuxScope(Context &ctx) : c(ctx) { std::swap(c.stream, c.aux); }
    ~AuxScope() { std::swap(c.stream, c.aux); }
};

// Work launched on the main stream while the interaction lists are built on the auxiliary one.
typedef int (*OverlapFn)(Context &c);

// ---- force.cu
// With host_x / host_y, the outputs are also copied there, run by run while later runs are
// evaluated (c.host_copied tells whether that happened; the copies are on the auxiliary
// stream).
int force_mrag(Context &c, double theta, const double *x0s, const double *y0s, const double *hs,
               int nblocks, double *xout, double *yout, OverlapFn between,
               double *host_x = nullptr, double *host_y = nullptr);

// ---- potential.cu
int potential(Context &c, double theta, const double *xt, const double *yt, int m, double *out,
              OverlapFn between);

// ---- kernel lists: each source file's kernels, every instance the library launches (for
// preload_kernels in capi.cu)
using KernelList = std::vector<const void *>;
void kernels_sort(KernelList &v);
void kernels_tree(KernelList &v);
void kernels_upward(KernelList &v);
void kernels_force(KernelList &v);
void kernels_potential(KernelList &v);
void kernels_direct(KernelList &v);

// ---- capi.cu
int check_device_errors(Context &c, const char *where);
// A solve's host waits for a stream / an event (see Context::sleeping_waits).
cudaError_t wait_stream(Context &c, cudaStream_t s);
cudaError_t wait_event(Context &c, cudaEvent_t e);
void phase_mark(Context &c, int idx);

}  // namespace tc
