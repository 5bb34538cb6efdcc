// Stand-in for the library's context API, linked with server.cu to exercise the request
// server's scheduling on the CPU: a "solve" sleeps, writes its request's marker into the
// outputs, records the order in which each client's requests ran, and grows the context's
// device-memory figure to a chosen multiple of the admission estimate.
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <random>
#include <thread>
#include <vector>

#include "treecodes_b200.h"

struct tc_context {
    size_t bytes = 0;
    int precision = 0;
};

std::atomic<int> g_live{0};
std::atomic<int> g_order_errors{0};
double g_actual_lo = 0.9, g_actual_hi = 0.9;   // actual bytes / estimate after a solve
static std::mutex g_mu;
static long long g_last_seq[1024];             // per client: last sequence number seen

extern "C" {
int tc_context_create(tc_context **c, int, void *) {
    *c = new tc_context();
    g_live++;
    return 0;
}
void tc_context_destroy(tc_context *c) {
    if (!c) return;
    delete c;
    g_live--;
}
int tc_set_host_waits(tc_context *, int) { return 0; }
int tc_set_launch_overlap(tc_context *, int) { return 0; }
int tc_set_precision(tc_context *c, int p) {
    c->precision = p;
    return 0;
}
size_t tc_context_device_bytes(tc_context *c) { return c ? c->bytes : 0; }
int tc_reserve_cached_memory(int, size_t) { return 0; }
int tc_context_trim(tc_context *c) {
    c->bytes = 0;
    return 0;
}
}

// xs[0] = client id, xs[1] = the request's sequence number within its client
static void work(tc_context *c, int kind, const double *xs, int n, int nt, int nb) {
    const long long client = (long long)xs[0], seq = (long long)xs[1];
    if (client > 0 && client < 1024) {
        std::lock_guard<std::mutex> lock(g_mu);
        if (seq != g_last_seq[client] + 1) g_order_errors++;
        g_last_seq[client] = seq;
    }
    thread_local std::mt19937 g(std::hash<std::thread::id>()(std::this_thread::get_id()));
    std::this_thread::sleep_for(std::chrono::microseconds(20 + g() % 400));
    const double f = g_actual_lo + (g_actual_hi - g_actual_lo) * (g() % 1001) / 1000.0;
    const size_t need = (size_t)(f * tc_request_footprint(kind, n, nt, nb, c->precision));
    if (need > c->bytes) c->bytes = need;
}

extern "C" {
int tc_potential_host(tc_context *c, double, const double *xs, const double *, const double *,
                      int n, const double *, const double *, int m, double *out) {
    work(c, 0, xs, n, m, 0);
    for (int i = 0; i < m; ++i) out[i] = xs[0] * 1e6 + xs[1];
    return 0;
}
int tc_force_mrag_host(tc_context *c, double, const double *xs, const double *, const double *,
                       int n, const double *, const double *, const double *, int nb, double *xo,
                       double *yo) {
    work(c, 1, xs, n, 0, nb);
    for (int i = 0; i < nb * 1024; ++i) xo[i] = yo[i] = xs[0] * 1e6 + xs[1];
    return 0;
}
}
