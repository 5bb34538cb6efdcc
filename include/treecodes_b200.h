/*
 * treecodes_b200.h -- C ABI of the B200 (sm_100a) 2-D treecode library
 * (lib2d-treecodes-b200.so).
 *
 * The first two functions are drop-in replacements for the reference's public entry points,
 * with identical prototypes (realtype = double) and semantics:
 *   treecode_potential   replaces drivers/treecode-potential.h:21-29
 *                        (definition drivers/treecode-potential.cpp:91-106)
 *   treecode_force_mrag  replaces drivers/treecode-force.h:21-31
 *                        (definition drivers/treecode-force.cpp:201-236)
 * Both take host pointers, copy them to the GPU, solve there and copy the results back.
 * Expansion orders (12 potential, 24 force), leaf capacities (512, 192), the MRAG block size
 * (32 x 32) and LMAX = 15 are those of the reference build (Makefile:13-15).
 * The force output of block ib, target (ix, iy), is at ix + 32 * (iy + 32 * ib).
 *
 * Differences from the reference, all additive: the functions are reentrant (state lives in
 * a per-thread context), print nothing, and report failures through treecode_last_status() /
 * treecode_last_error() instead of undefined behaviour.  nsources == 0 yields zero outputs.
 *
 * The tc_* functions are an extended API (no counterpart in the reference): explicit contexts
 * on a CUDA stream, device-pointer entry points, statistics, tree inspection for tests, GPU
 * direct sums for accuracy checks.  They return a tc_status code.
 */
#ifndef TREECODES_B200_H
#define TREECODES_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define TC_API __attribute__((visibility("default")))

/* ---- reference-compatible entry points ---------------------------------------------- */

/* drivers/treecode-potential.h:21-29 */
TC_API void treecode_potential(const double theta,
                               const double * const xsources,
                               const double * const ysources,
                               const double * const sourcevalues,
                               const int nsources,
                               const double * const xtargets,
                               const double * const ytargets,
                               const int ntargets,
                               double * const targetvalues);

/* drivers/treecode-force.h:21-31 */
TC_API void treecode_force_mrag(const double theta,
                                const double * const xsources,
                                const double * const ysources,
                                const double * const sourcevalues,
                                const int nsources,
                                const double * const x0s,
                                const double * const y0s,
                                const double * const hs,
                                const int nblocks,
                                double * const xresults,
                                double * const yresults);

/* ---- status ----------------------------------------------------------------------- */

typedef enum {
    TC_OK = 0,
    TC_ERR_INVALID = 1,    /* bad argument (negative size, NULL pointer, unsupported mode) */
    TC_ERR_CUDA = 2,       /* a CUDA call failed */
    TC_ERR_CAPACITY = 3,   /* a device-side capacity (traversal stack) was exceeded */
    TC_ERR_TIMEOUT = 4,    /* a bounded device-side wait gave up */
    TC_ERR_NO_DEVICE = 5,  /* no CUDA device is visible */
    TC_ERR_ALLOC = 6       /* device memory could not be allocated */
} tc_status;

/* Status and message of the last call made by this thread (any entry point). */
TC_API int treecode_last_status(void);
TC_API const char *treecode_last_error(void);

/* ---- extended API ------------------------------------------------------------------ */

typedef struct tc_context tc_context;

typedef enum { TC_PRECISION_FP64 = 0, TC_PRECISION_MIXED = 1 } tc_precision;

/* Stages whose first look-back tile can be told never to publish (tc_set_wait_test). */
typedef enum { TC_STALL_NONE = 0, TC_STALL_SORT = 1, TC_STALL_TREE = 2 } tc_stall;

typedef struct {
    /* phase times in ms (filled when timing is enabled) */
    float sort_ms, tree_ms, upward_ms, lists_ms, eval_ms, total_ms;
    /* sizes of the last solve */
    long long nnodes, nleaves, ninner, nlevels;
    long long n_e2l, n_e2p, n_p2p;   /* interaction-list entries */
    long long p2p_pairs;             /* source-target pairs evaluated directly */
    long long e2p_pairs;             /* (target, cell) pairs evaluated from multipoles */
    long long e2l_pairs;             /* (brick, cell) multipole-to-local translations */
    long long l2p_targets;           /* targets evaluated from local expansions */
    long long launches;              /* kernels launched by the last solve */
    float eval_kernel_ms;            /* the evaluation kernel alone (timing enabled) */
    int list_walks;                  /* tree walks that built the lists: 1, or 2 when the
                                        one-walk build outgrew its scratch (which then grows) */
    float far_kernel_ms;             /* force: the far-field kernel alone; eval_kernel_ms is
                                        it plus the near-field kernel, which runs beside the
                                        upward pass (timing enabled; 0 otherwise) */
} tc_stats;

/* device < 0 selects the current device; stream may be NULL (the context creates one). */
TC_API int tc_context_create(tc_context **ctx, int device, void *cuda_stream);
TC_API void tc_context_destroy(tc_context *ctx);
TC_API int tc_set_precision(tc_context *ctx, int precision);
/* How the calling thread waits for the device inside a solve: 0 (the default) spins in the CUDA
 * call, the lowest latency; 1 polls every 20 us and sleeps in between, which leaves the host core
 * to other threads (the request server's slots wait this way). */
TC_API int tc_set_host_waits(tc_context *ctx, int sleeping);
/* Programmatic dependent launch of the solve's kernel chains (the source and target sorts, the
 * tree build, the upward pass): 1 (the default) lets each kernel of a chain be scheduled while
 * the one before it drains, and it waits on the device until that one has completed; 0 launches
 * them one after another.  It saves about 2.5 us per launch on a lone solve.  The request
 * server turns it off on its contexts: with four solving at once it caused occasional stalls of
 * tens of milliseconds. */
TC_API int tc_set_launch_overlap(tc_context *ctx, int on);
/* Test settings that make the library's bounded device waits and capacities run out on
 * purpose, so that their error paths can be exercised without faulting or hanging a GPU (no
 * counterpart in the reference, whose overflows are silent, drivers/upward.cpp:253).
 *   stall:       TC_STALL_SORT / TC_STALL_TREE: in the source sort's first radix pass, or in
 *                the tree build's list pass, tile 0 publishes nothing, so the tile after it
 *                waits on it until the spin limit, raises the device error flag and moves on;
 *                the solve then stops after that stage with TC_ERR_TIMEOUT.  Needs more
 *                sources than one tile (3072 for the sort, 4096 for the tree).
 *   spin_limit:  reads without progress after which a device wait gives up (<= 0: the default,
 *                4,194,304).
 *   stack_limit: traversal stack entries per warp of the force lists (<= 0: all 2048); a walk
 *                that would exceed it stops with the lists so far and the solve returns
 *                TC_ERR_CAPACITY.
 * tc_set_wait_test(ctx, TC_STALL_NONE, 0, 0) restores the defaults; the context stays usable
 * after every such failure. */
TC_API int tc_set_wait_test(tc_context *ctx, int stall, int spin_limit, int stack_limit);
/* Expansion orders of the context's next solves: the reference fixes them when it is built
 * (Makefile:13-14 of the reference, potential-order = 12 and force-order = 24, which stay the
 * defaults here).  Any order that tc_supported_orders lists may be chosen, independently for
 * the two entry points; others are refused with TC_ERR_INVALID. */
TC_API int tc_set_orders(tc_context *ctx, int potential_order, int force_order);
/* Writes up to `capacity` supported orders (ascending) to `orders`; returns how many exist. */
TC_API int tc_supported_orders(int *orders, int capacity);
/* MRAG block side of the context's force solves (tc_force_mrag_host / _device): 8, 16, 32 or
 * 64 targets, the reference's build-time mrag-blocksize (Makefile:15 of the reference, 32 by
 * default and for treecode_force_mrag).  Outputs hold nblocks * blocksize^2 values, target
 * (ix, iy) of block ib at ix + blocksize * (iy + blocksize * ib). */
TC_API int tc_set_blocksize(tc_context *ctx, int blocksize);
/* 1: record phase times (tc_get_stats); 2: also run the force evaluation's near- and far-field
 * kernels one after the other, after the upward pass, each alone on the GPU, so that their
 * times measure each kernel by itself (a measurement mode: the solve is slower, results are
 * the same); 0: off. */
TC_API int tc_set_timing(tc_context *ctx, int enabled);
TC_API int tc_get_stats(tc_context *ctx, tc_stats *out);
TC_API void *tc_get_stream(tc_context *ctx);

/* Same as the reference entry points, host pointers, explicit context and status. */
TC_API int tc_potential_host(tc_context *ctx, double theta, const double *xsources,
                             const double *ysources, const double *sourcevalues, int nsources,
                             const double *xtargets, const double *ytargets, int ntargets,
                             double *targetvalues);
TC_API int tc_force_mrag_host(tc_context *ctx, double theta, const double *xsources,
                              const double *ysources, const double *sourcevalues, int nsources,
                              const double *x0s, const double *y0s, const double *hs,
                              int nblocks, double *xresults, double *yresults);

/* Device pointers (all arrays resident in GPU memory); work is ordered on the context's
 * stream and complete when the call returns. */
TC_API int tc_potential_device(tc_context *ctx, double theta, const double *xsources,
                               const double *ysources, const double *sourcevalues, int nsources,
                               const double *xtargets, const double *ytargets, int ntargets,
                               double *targetvalues);
TC_API int tc_force_mrag_device(tc_context *ctx, double theta, const double *xsources,
                                const double *ysources, const double *sourcevalues,
                                int nsources, const double *x0s, const double *y0s,
                                const double *hs, int nblocks, double *xresults,
                                double *yresults);

/* Tree inspection (tests).  kind: 0 = potential tree (order 12, leaf 512),
 * 1 = force tree (order 24, leaf 192).  Sources are device pointers. */
TC_API int tc_tree_build_device(tc_context *ctx, int kind, const double *xsources,
                                const double *ysources, const double *sourcevalues,
                                int nsources);
TC_API int tc_tree_size(tc_context *ctx, int *nnodes, int *order, int *nsources);
/* Host arrays: keys/perm/xs/ys/vs (nsources each), frame (xmin, ymin, ext), per node
 * s, e, child (-1 = leaf), count, level, cx, cy, parent, mass, xcom, ycom, r,
 * exps (nnodes * 2 * order: real parts then imaginary parts).  Any pointer may be NULL. */
TC_API int tc_tree_copy(tc_context *ctx, int *keys, int *perm, double *xs, double *ys,
                        double *vs, double *frame, int *s, int *e, int *child, int *count,
                        int *level, int *cx, int *cy, int *parent, double *mass, double *xcom,
                        double *ycom, double *r, double *exps);

/* FP64 direct sums (main.cpp:201-245 of the reference) on device pointers. */
TC_API int tc_direct_potential_device(tc_context *ctx, const double *xsources,
                                      const double *ysources, const double *sourcevalues,
                                      int nsources, const double *xtargets,
                                      const double *ytargets, int ntargets, double *out);
TC_API int tc_direct_force_device(tc_context *ctx, const double *xsources,
                                  const double *ysources, const double *sourcevalues,
                                  int nsources, const double *xtargets, const double *ytargets,
                                  int ntargets, double *xout, double *yout);
/* Diagnostic: out[2i] = the logarithm the potential kernels use (a positive normal x only),
 * out[2i + 1] = the CUDA library's log, both on the device (device pointers, n values). */
TC_API int tc_log_probe_device(tc_context *ctx, const double *x, int n, double *out);

/* Allocation-free source sort.  No counterpart in the reference.
 *
 * Some callers cannot call cudaMalloc at the moment they need the tree: code that owns all of
 * device memory through its own pool (a flow solver or a framework allocator that hands out
 * every byte and must not be bypassed), code on a latency-critical path where an allocation's
 * implicit device synchronisation and unbounded cost are not acceptable, and long-running
 * services that must not grow or fragment device memory after start-up.  For them this entry
 * point runs the first stage
 * of the solve -- padded bounding square, 30-bit Morton keys, stable radix sort, gather of
 * x/y/value into Morton order, as drivers/sort-sources.cpp:23-132 of the reference defines it
 * -- with all of its scratch memory in one fixed, statically allocated device array.  It runs the
 * same kernels as the library's host entry points.
 *
 *   nsources <= TC_NOALLOC_MAX_SOURCES (1,048,576); larger inputs are rejected with
 *   TC_ERR_INVALID and a message naming the limit.  The scratch array is about 1.5 MB, held by
 *   every GPU that loads the library until the process exits.  During the call xsorted and
 *   ysorted also serve as the radix passes' working buffers (they hold the final results when
 *   the call returns).
 *   All arrays are device pointers supplied by the caller: inputs xsources/ysources/
 *   sourcevalues; outputs keys and perm (nsources ints: sorted keys and, for each sorted
 *   position, the input index), xsorted/ysorted/vsorted (nsources doubles) and frame
 *   (4 doubles: xmin, ymin, ext of the padded square, and the key scale 2^15 / ext).
 *   The work is ordered on cuda_stream (NULL: the legacy default stream) and complete when the
 *   call returns.  The results equal those of the allocating solve path bit for bit.
 *   The first call on each device looks up the array's device address (cudaGetSymbolAddress);
 *   make that first call before any stream capture begins.
 *   All calls share the one array: calls whose GPU work could overlap (other streams, other
 *   threads) race on it and must be serialised by the caller.  The call allocates nothing:
 *   no cudaMalloc, no cudaFree, no allocating library routine. */
#define TC_NOALLOC_MAX_SOURCES (1 << 20)
TC_API int tc_sort_sources_noalloc(const double *xsources, const double *ysources,
                                   const double *sourcevalues, int nsources, int *keys,
                                   int *perm, double *xsorted, double *ysorted, double *vsorted,
                                   double *frame, void *cuda_stream);

/* Device memory held by a context's grow-only buffers, in bytes. */
TC_API size_t tc_context_device_bytes(tc_context *ctx);
/* Frees a context's device buffers; the next solve on it allocates them again.  Freed memory
 * (here and in tc_context_destroy) stays cached in the device's stream-ordered pool for the
 * process's next allocations while any context of the device lives; the last context's
 * destruction, or tc_release_cached_memory, hands it back to the driver. */
TC_API int tc_context_trim(tc_context *ctx);
/* Hands the device's cached, unused pool memory back to the driver (device < 0: current). */
TC_API int tc_release_cached_memory(int device);
/* Maps up to `bytes` of device memory into the device's stream-ordered pool and leaves it there
 * unused (at most the free memory less 2 GB), so that later context allocations are carved from
 * it instead of growing the pool while solves run; growing it mapped new memory in the middle of
 * other contexts' work.  The memory returns to the driver as described for tc_context_trim. */
TC_API int tc_reserve_cached_memory(int device, size_t bytes);

/* ---- serving loop ---------------------------------------------------------------------
 * A request server on one GPU: solves submitted from any thread are queued, admitted in
 * arrival order as execution slots and device memory free up, and run concurrently, one
 * context (and CUDA stream) per slot or per resident client, so the work of admitted requests
 * overlaps on the device.  Admission charges each request's device-memory footprint (estimated
 * from its sizes, corrected by the context's actual size once known) against a budget; idle
 * resident clients are released, least recently used first, when a request does not fit.
 * A request with client > 0 runs on that client's own context, whose device buffers (sorted
 * sources, tree, expansions, interaction lists, staged inputs) stay resident between its
 * requests; requests of one client run one at a time in submission order.  Results are the
 * same as those of a solve on its own context (the kernels are deterministic). */
typedef struct tc_server tc_server;

typedef enum { TC_REQUEST_POTENTIAL = 0, TC_REQUEST_FORCE_MRAG = 1 } tc_request_kind;

typedef struct {
    int kind;                       /* tc_request_kind */
    int precision;                  /* tc_precision */
    double theta;
    long long client;               /* > 0: resident client id; 0: one-off request */
    int nsources;
    const double *xsources, *ysources, *sourcevalues;   /* host arrays */
    int ntargets;                   /* potential */
    const double *xtargets, *ytargets;
    int nblocks;                    /* force_mrag */
    const double *x0s, *y0s, *hs;
    double *out0;                   /* potential: values; force_mrag: x components */
    double *out1;                   /* force_mrag: y components */
} tc_request;                       /* all arrays must stay valid until the request completes */

typedef struct {
    int status;                     /* tc_status of the solve */
    int slot;                       /* execution slot that ran it */
    double queue_ms;                /* submission to admission */
    double service_ms;              /* admission to completion */
    double latency_ms;              /* submission to completion */
    size_t footprint_bytes;         /* device memory charged at admission */
    double finished_s;              /* completion instant, seconds on CLOCK_MONOTONIC (the
                                       clock of Python's time.perf_counter() on Linux), so
                                       that a caller can time a request from its own
                                       arrival stamp whatever order it collects results in */
} tc_request_result;

typedef struct {
    long long submitted, completed, failed, evictions;
    size_t hbm_budget, hbm_charged, hbm_peak;
    int slots, max_in_service, resident_clients;
} tc_server_stats;

/* slots: concurrent solves (>= 1); with 3 or more, the last slot serves only requests of at
 * most 2^17 sources, so that small requests do not queue behind a burst of large ones.
 * hbm_budget_bytes: device memory the server may hold, which it maps into the device's pool at
 * creation (tc_reserve_cached_memory). */
TC_API int tc_server_create(tc_server **srv, int device, int slots, size_t hbm_budget_bytes);
/* Waits for all submitted requests, then frees every context. */
TC_API void tc_server_destroy(tc_server *srv);
TC_API int tc_server_submit(tc_server *srv, const tc_request *req, long long *ticket);
/* Blocks until the request has completed; each ticket is waited for once. */
TC_API int tc_server_wait(tc_server *srv, long long ticket, tc_request_result *result);
/* Blocks until any submitted, not yet collected request has completed and collects it: *ticket
   receives its ticket, the return value its status (the earliest completion first).  Returns
   TC_ERR_INVALID with *ticket = 0 when no request is outstanding.  A caller that collects in
   completion order releases each result's buffers as soon as it is done, instead of holding
   them behind a longer solve submitted earlier. */
TC_API int tc_server_wait_any(tc_server *srv, long long *ticket, tc_request_result *result);
/* Releases a resident client's device memory once its queued requests are done. */
TC_API int tc_server_release_client(tc_server *srv, long long client);
TC_API int tc_server_get_stats(tc_server *srv, tc_server_stats *out);
/* Device-memory estimate used for admission (bytes) of a request of the given sizes. */
TC_API size_t tc_request_footprint(int kind, int nsources, int ntargets, int nblocks,
                                   int precision);

/* Measured FMA throughput of the current device in TFLOP/s (fp64 != 0: FP64, else FP32). */
TC_API int tc_measure_fma_peak(int fp64, double *tflops);

/* Library version string. */
TC_API const char *tc_version(void);

#ifdef __cplusplus
}
#endif

#endif /* TREECODES_B200_H */
