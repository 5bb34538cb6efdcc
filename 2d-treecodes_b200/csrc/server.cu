// server.cu -- the serving loop: a device-resident request server on one GPU.
//
// No counterpart in the reference, whose entry points are blocking, not reentrant and allocate
// per call (drivers/upward.cpp:289-324).  Here a request is a potential or force_mrag solve with
// host inputs.  Submissions go into one FIFO queue.  `slots` worker threads each take the
// oldest admissible request, run it on a context of their own (or on the request's resident
// client context) through the public host entry points, and signal its ticket; since every
// context owns a CUDA stream, the solves of different slots overlap on the device -- requests
// that arrive while others are on the GPU start as soon as a slot and memory are free
// (continuous batching of independent solves).
//
// Slots: with three or more, the last one is an express slot for requests of at most 2^17
// sources; the others take any request.
//
// Admission (under the server lock):
//   * a request of client k is admissible only when no earlier request of k is queued or in
//     service, so one client's steps run in submission order on its resident buffers;
//   * its footprint is max(estimate from its sizes, bytes its context already holds); the
//     increase over what that context holds must fit into budget - charged, where charged sums
//     the bytes held by every live context plus the reserved increase of requests in service;
//   * when it does not fit, the admitting slot frees the pooled contexts of idle slots and then
//     evicts idle resident clients, least recently used first (those with no queued request
//     before those whose next step is queued: every request carries its inputs, so an evicted
//     client's next step starts on a fresh context); if it still does not fit, it waits for a
//     completion (later requests do not overtake it for memory).  With nothing in service all
//     held memory can be freed, so a request that fits the budget is always admitted.  A request whose footprint alone exceeds the
//     budget fails with TC_ERR_CAPACITY without touching the device.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <ctime>
#include <deque>
#include <list>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "treecodes_b200.h"
#include "tc_common.cuh"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// Seconds on CLOCK_MONOTONIC (the clock of Python's time.perf_counter() on Linux).
double monotonic_s() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

struct Job {
    long long ticket = 0;
    tc_request req{};
    size_t estimate = 0;
    Clock::time_point submitted, admitted, finished;
    bool done = false;
    tc_request_result result{};
};

struct Client {
    tc_context *ctx = nullptr;
    size_t bytes = 0;             // device memory the context holds (as last measured)
    bool busy = false;            // a request of this client is in service
    int queued = 0;               // requests of this client waiting in the queue
    bool release_pending = false;
    std::list<long long>::iterator lru;
};

}  // namespace

struct tc_server {
    int device = 0;
    int nslots = 1;
    size_t budget = 0;

    std::mutex mu;
    std::condition_variable cv_work;   // queue changed or memory freed
    std::condition_variable cv_done;   // a job finished
    std::deque<Job *> queue;
    std::unordered_map<long long, Job *> jobs;
    std::deque<long long> done_order;  // finished tickets in completion order (for wait_any)
    std::unordered_map<long long, Client> clients;
    std::list<long long> lru;          // idle clients, least recently used first
    std::vector<tc_context *> pool;    // one pooled context per slot (one-off requests)
    // evicted client contexts, destroyed by whoever evicted them once the lock is released:
    // destroying a context synchronises its streams and frees its buffers, which must not hold
    // up admission and submission (one release under the lock stalled both for 86 ms)
    std::vector<tc_context *> graveyard;
    std::vector<size_t> pool_bytes;
    std::vector<char> slot_busy;
    std::vector<std::thread> workers;
    size_t charged = 0;                // bytes held by contexts + reservations in service
    double ratio[2] = {1.0, 1.0};      // observed actual / estimated bytes, per request kind
    size_t peak = 0;
    long long next_ticket = 1;
    long long submitted = 0, completed = 0, failed = 0, evictions = 0;
    int in_service = 0, max_in_service = 0;
    bool stop = false;

    void worker(int slot);
    Job *pick(int slot, size_t *reserve, tc_context **ctx);
    bool make_room(int slot, size_t need, long long keep_client);
    void evict_client_locked(long long id);
    std::vector<tc_context *> take_graveyard_locked() {
        std::vector<tc_context *> dead;
        dead.swap(graveyard);
        return dead;
    }
};

namespace {

// With three slots or more, the last slot takes only requests of at most this many sources, so
// that small requests do not queue behind a burst of large ones that holds every slot.
constexpr int EXPRESS_MAX_SOURCES = 1 << 17;

size_t footprint_estimate(int kind, long long n, long long ntargets, long long nblocks,
                          int precision) {
    const bool force = kind == TC_REQUEST_FORCE_MRAG;
    const long long leaf = force ? tc::LEAF_FORCE : tc::LEAF_POTENTIAL;
    const long long p = force ? tc::ORDER_FORCE : tc::ORDER_POTENTIAL;
    // per source: staged x/y/v, sorted x/y/v, keys and permutation, the sort's two item arrays
    // and packed records, tree-build flags; per-level ranks of the split list
    const long long nodes = 4 * (n / leaf + 1) + 64;
    size_t b = (size_t)n * 128 + (size_t)std::min(n, nodes) * 8 * tc::LMAX;
    // per node: traversal record, range, cell, moments, expansion (+ scaled FP32 copy)
    b += (size_t)nodes * (88 + 16 * p + (precision ? 8 * p + 4 : 0));
    if (force) {
        const long long m = nblocks * tc::BLOCKSIZE * tc::BLOCKSIZE;
        b += (size_t)m * 16 + (size_t)m * 64;   // outputs + per-brick lists and partial sums
    } else {
        // staged targets, output, target sort, partials and the per-group lists, whose far
        // part grows as 1/theta^2 (about 14 entries per target at theta = 0.3); the list
        // build's scratch, held only while the lists are built, is not charged
        b += (size_t)ntargets * 210;
    }
    return b + (4u << 20);
}

int validate(const tc_request &r) {
    if (r.kind != TC_REQUEST_POTENTIAL && r.kind != TC_REQUEST_FORCE_MRAG) return TC_ERR_INVALID;
    if (r.precision < 0 || r.precision > 1 || r.nsources < 0 || r.client < 0) return TC_ERR_INVALID;
    if (r.nsources > 0 && (!r.xsources || !r.ysources || !r.sourcevalues)) return TC_ERR_INVALID;
    if (r.kind == TC_REQUEST_POTENTIAL) {
        if (r.ntargets < 0 || (r.ntargets > 0 && (!r.xtargets || !r.ytargets || !r.out0)))
            return TC_ERR_INVALID;
    } else {
        if (r.nblocks < 0 ||
            (r.nblocks > 0 && (!r.x0s || !r.y0s || !r.hs || !r.out0 || !r.out1)))
            return TC_ERR_INVALID;
    }
    return TC_OK;
}

int run_request(tc_context *ctx, const tc_request &r) {
    // slot threads sleep while their solve runs instead of spinning on a host core
    int rc = tc_set_host_waits(ctx, 1);
    if (rc) return rc;
    // plain launches: programmatic dependent launch in four contexts solving at once gave
    // occasional stalls of tens of milliseconds
    rc = tc_set_launch_overlap(ctx, 0);
    if (rc) return rc;
    rc = tc_set_precision(ctx, r.precision);
    if (rc) return rc;
    if (r.kind == TC_REQUEST_POTENTIAL)
        return tc_potential_host(ctx, r.theta, r.xsources, r.ysources, r.sourcevalues, r.nsources,
                                 r.xtargets, r.ytargets, r.ntargets, r.out0);
    return tc_force_mrag_host(ctx, r.theta, r.xsources, r.ysources, r.sourcevalues, r.nsources,
                              r.x0s, r.y0s, r.hs, r.nblocks, r.out0, r.out1);
}

}  // namespace

// Frees an idle client's context.  The entry stays while requests of the client are queued
// (their inputs come with them, so the next one simply starts on a fresh context).
void tc_server::evict_client_locked(long long id) {
    auto it = clients.find(id);
    if (it == clients.end()) return;
    Client &cl = it->second;
    if (cl.ctx) {
        lru.erase(cl.lru);
        charged -= cl.bytes;
        graveyard.push_back(cl.ctx);   // destroyed outside the lock (take_graveyard_locked)
        cl.ctx = nullptr;
        cl.bytes = 0;
    }
    if (cl.queued == 0 && !cl.busy) clients.erase(it);
}

// Frees memory for a request that needs `need` more bytes: the pooled contexts of idle slots
// (this slot's own only when the request runs on a client context), then idle clients in LRU
// order.  Returns whether the request fits.
bool tc_server::make_room(int slot, size_t need, long long keep_client) {
    if (charged + need <= budget) return true;
    for (int i = 0; i < nslots && charged + need > budget; ++i) {
        if (pool_bytes[i] == 0 || (i == slot ? keep_client == 0 : slot_busy[i] != 0)) continue;
        tc_context_trim(pool[i]);
        charged -= pool_bytes[i];
        pool_bytes[i] = 0;
    }
    // idle clients with nothing queued first, then idle clients whose next steps are queued
    for (int pass = 0; pass < 2; ++pass)
        for (auto it = lru.begin(); it != lru.end() && charged + need > budget;) {
            const long long id = *it++;
            if (id == keep_client) continue;
            const Client &cl = clients[id];
            if (cl.busy || (pass == 0 && cl.queued > 0)) continue;
            evict_client_locked(id);
            ++evictions;
        }
    return charged + need <= budget;
}

// Oldest admissible job; sets the reservation and the context it runs on.  Called locked.
Job *tc_server::pick(int slot, size_t *reserve, tc_context **ctx) {
    std::vector<long long> blocked;   // clients with an earlier request still queued
    for (auto it = queue.begin(); it != queue.end(); ++it) {
        Job *j = *it;
        const long long k = j->req.client;
        if (k > 0) {
            bool earlier = false;
            for (long long b : blocked) earlier |= (b == k);
            if (earlier) continue;
            blocked.push_back(k);
            auto ci = clients.find(k);
            if (ci != clients.end() && ci->second.busy) continue;
        }
        // the express slot leaves large requests to the others (after the client bookkeeping
        // above, so that a later step of the same client cannot overtake a skipped one)
        if (nslots >= 3 && slot == nslots - 1 && j->req.nsources > EXPRESS_MAX_SOURCES) continue;
        const size_t held = k > 0 ? (clients.count(k) ? clients[k].bytes : 0) : pool_bytes[slot];
        // the charge: the estimate scaled by the learned actual/estimate ratio, at most the
        // whole budget, so that admitting it never charges more than the budget
        const size_t est =
            std::min(budget, (size_t)((double)j->estimate * ratio[j->req.kind]));
        const size_t need = est > held ? est - held : 0;
        if (j->estimate > budget) {
            // can never fit: fail it without running
            queue.erase(it);
            if (k > 0 && clients.count(k)) clients[k].queued--;
            j->result.status = TC_ERR_CAPACITY;
            j->result.slot = slot;
            j->admitted = j->finished = Clock::now();
            j->result.finished_s = monotonic_s();
            j->done = true;
            done_order.push_back(j->ticket);
            ++failed;
            ++completed;
            cv_done.notify_all();
            return pick(slot, reserve, ctx);
        }
        if (!make_room(slot, need, k) && in_service > 0) {
            // keep arrival order for memory: a large request is not overtaken indefinitely.
            // With nothing in service everything evictable is gone and waiting cannot help
            // (the memory still held is the request's own context), so it is admitted.
            return nullptr;
        }
        queue.erase(it);
        if (k > 0) {
            Client &cl = clients[k];
            cl.queued--;
            if (!cl.ctx) {
                if (tc_context_create(&cl.ctx, device, nullptr) != TC_OK) {
                    cl.ctx = nullptr;
                    j->result.status = TC_ERR_CUDA;
                    j->result.slot = slot;
                    j->admitted = j->finished = Clock::now();
                    j->result.finished_s = monotonic_s();
                    j->done = true;
                    done_order.push_back(j->ticket);
                    ++failed;
                    ++completed;
                    cv_done.notify_all();
                    return pick(slot, reserve, ctx);
                }
                lru.push_back(k);
                cl.lru = std::prev(lru.end());
            }
            cl.busy = true;
            *ctx = cl.ctx;
        } else {
            *ctx = pool[slot];
        }
        *reserve = need;
        charged += need;
        peak = std::max(peak, charged);
        j->result.footprint_bytes = held + need;
        return j;
    }
    return nullptr;
}

void tc_server::worker(int slot) {
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lock(mu);
    for (;;) {
        size_t reserve = 0;
        tc_context *ctx = nullptr;
        Job *j = nullptr;
        cv_work.wait(lock, [&] {
            if (stop && queue.empty()) return true;
            j = pick(slot, &reserve, &ctx);
            return j != nullptr;
        });
        if (!j) return;   // stopping and nothing left
        j->admitted = Clock::now();
        slot_busy[slot] = 1;
        ++in_service;
        max_in_service = std::max(max_in_service, in_service);
        std::vector<tc_context *> dead = take_graveyard_locked();   // evicted while admitting
        lock.unlock();
        for (tc_context *d : dead) tc_context_destroy(d);

        const int rc = run_request(ctx, j->req);
        const size_t bytes = tc_context_device_bytes(ctx);

        lock.lock();
        slot_busy[slot] = 0;
        const size_t held_before = j->result.footprint_bytes - reserve;
        --in_service;
        charged -= reserve;
        const long long k = j->req.client;
        if (k > 0) {
            Client &cl = clients[k];
            charged = charged - cl.bytes + bytes;
            cl.bytes = bytes;
            cl.busy = false;
            lru.erase(cl.lru);   // most recently used goes last
            lru.push_back(k);
            cl.lru = std::prev(lru.end());
            if (cl.release_pending && cl.queued == 0) evict_client_locked(k);
        } else {
            charged = charged - pool_bytes[slot] + bytes;
            pool_bytes[slot] = bytes;
        }
        if (bytes > held_before && j->estimate > 0) {
            // this request set the context's size: learn how far the estimate was off
            const double r = (double)bytes / (double)j->estimate;
            ratio[j->req.kind] = std::min(8.0, std::max(ratio[j->req.kind], r));
        }
        peak = std::max(peak, charged);
        j->finished = Clock::now();
        j->result.finished_s = monotonic_s();
        j->result.status = rc;
        j->result.slot = slot;
        j->done = true;
        done_order.push_back(j->ticket);
        ++completed;
        if (rc) ++failed;
        cv_done.notify_all();
        cv_work.notify_all();
        dead = take_graveyard_locked();   // a client released after its last step
        if (!dead.empty()) {
            lock.unlock();
            for (tc_context *d : dead) tc_context_destroy(d);
            lock.lock();
        }
    }
}

extern "C" {

TC_API size_t tc_request_footprint(int kind, int nsources, int ntargets, int nblocks,
                                   int precision) {
    return footprint_estimate(kind, nsources, ntargets, nblocks, precision);
}

TC_API int tc_server_create(tc_server **srv, int device, int slots, size_t hbm_budget_bytes) {
    if (!srv || slots < 1 || slots > 64 || hbm_budget_bytes == 0) return TC_ERR_INVALID;
    *srv = nullptr;
    tc_server *s = new tc_server();
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) {
        delete s;
        return TC_ERR_NO_DEVICE;
    }
    s->device = device;
    s->nslots = slots;
    s->budget = hbm_budget_bytes;
    s->pool.assign(slots, nullptr);
    s->pool_bytes.assign(slots, 0);
    s->slot_busy.assign(slots, 0);
    for (int i = 0; i < slots; ++i) {
        const int rc = tc_context_create(&s->pool[i], device, nullptr);
        if (rc) {
            for (auto *c : s->pool) tc_context_destroy(c);
            delete s;
            return rc;
        }
    }
    // the budget mapped into the device pool now, not while other requests' solves run (best
    // effort: a server whose budget exceeds the free memory still works, with a smaller pool)
    tc_reserve_cached_memory(device, hbm_budget_bytes);
    for (int i = 0; i < slots; ++i) s->workers.emplace_back(&tc_server::worker, s, i);
    *srv = s;
    return TC_OK;
}

TC_API void tc_server_destroy(tc_server *srv) {
    if (!srv) return;
    {
        std::lock_guard<std::mutex> lock(srv->mu);
        srv->stop = true;
    }
    srv->cv_work.notify_all();
    for (auto &t : srv->workers) t.join();
    for (auto *c : srv->pool) tc_context_destroy(c);
    for (auto &kv : srv->clients) tc_context_destroy(kv.second.ctx);
    for (auto *c : srv->graveyard) tc_context_destroy(c);
    for (auto &kv : srv->jobs) delete kv.second;
    delete srv;
}

TC_API int tc_server_submit(tc_server *srv, const tc_request *req, long long *ticket) {
    if (!srv || !req || !ticket) return TC_ERR_INVALID;
    const int v = validate(*req);
    if (v) return v;
    Job *j = new Job();
    j->req = *req;
    j->estimate = footprint_estimate(req->kind, req->nsources, req->ntargets, req->nblocks,
                                     req->precision);
    j->submitted = Clock::now();
    {
        std::lock_guard<std::mutex> lock(srv->mu);
        if (srv->stop) {
            delete j;
            return TC_ERR_INVALID;
        }
        j->ticket = srv->next_ticket++;
        srv->jobs[j->ticket] = j;
        srv->queue.push_back(j);
        if (req->client > 0) {
            Client &cl = srv->clients[req->client];
            if (!cl.ctx && cl.queued == 0 && !cl.busy) {
                // first sighting: an entry without a context yet (created at admission)
                cl.lru = srv->lru.end();
            }
            cl.queued++;
            cl.release_pending = false;
        }
        ++srv->submitted;
        *ticket = j->ticket;
    }
    srv->cv_work.notify_all();
    return TC_OK;
}

namespace {

// Hands a finished job's result to the caller and forgets the job (under the server lock).
int collect_locked(tc_server *srv, Job *j, tc_request_result *result) {
    j->result.queue_ms = ms_between(j->submitted, j->admitted);
    j->result.service_ms = ms_between(j->admitted, j->finished);
    j->result.latency_ms = ms_between(j->submitted, j->finished);
    if (result) *result = j->result;
    const int status = j->result.status;
    srv->jobs.erase(j->ticket);
    delete j;
    // a wait_any blocked on the last outstanding ticket, which this call took, must return
    srv->cv_done.notify_all();
    return status;
}

}  // namespace

TC_API int tc_server_wait(tc_server *srv, long long ticket, tc_request_result *result) {
    if (!srv) return TC_ERR_INVALID;
    std::unique_lock<std::mutex> lock(srv->mu);
    auto it = srv->jobs.find(ticket);
    if (it == srv->jobs.end()) return TC_ERR_INVALID;
    Job *j = it->second;
    srv->cv_done.wait(lock, [&] { return j->done; });
    return collect_locked(srv, j, result);
}

TC_API int tc_server_wait_any(tc_server *srv, long long *ticket, tc_request_result *result) {
    if (!srv || !ticket) return TC_ERR_INVALID;
    std::unique_lock<std::mutex> lock(srv->mu);
    for (;;) {
        // the oldest completion not yet collected (tickets that tc_server_wait took are skipped)
        while (!srv->done_order.empty()) {
            const long long t = srv->done_order.front();
            srv->done_order.pop_front();
            auto it = srv->jobs.find(t);
            if (it == srv->jobs.end()) continue;
            *ticket = t;
            return collect_locked(srv, it->second, result);
        }
        if (srv->jobs.empty()) {   // nothing submitted and uncollected: nothing to wait for
            *ticket = 0;
            return TC_ERR_INVALID;
        }
        srv->cv_done.wait(lock);
    }
}

TC_API int tc_server_release_client(tc_server *srv, long long client) {
    if (!srv || client <= 0) return TC_ERR_INVALID;
    std::vector<tc_context *> dead;
    {
        std::lock_guard<std::mutex> lock(srv->mu);
        auto it = srv->clients.find(client);
        if (it == srv->clients.end()) return TC_OK;
        Client &cl = it->second;
        if (cl.busy || cl.queued > 0)
            cl.release_pending = true;
        else
            srv->evict_client_locked(client);
        dead = srv->take_graveyard_locked();
        srv->cv_work.notify_all();
    }
    for (tc_context *d : dead) tc_context_destroy(d);
    return TC_OK;
}

TC_API int tc_server_get_stats(tc_server *srv, tc_server_stats *out) {
    if (!srv || !out) return TC_ERR_INVALID;
    std::lock_guard<std::mutex> lock(srv->mu);
    out->submitted = srv->submitted;
    out->completed = srv->completed;
    out->failed = srv->failed;
    out->evictions = srv->evictions;
    out->hbm_budget = srv->budget;
    out->hbm_charged = srv->charged;
    out->hbm_peak = srv->peak;
    out->slots = srv->nslots;
    out->max_in_service = srv->max_in_service;
    int resident = 0;
    for (auto &kv : srv->clients) resident += kv.second.ctx != nullptr;
    out->resident_clients = resident;
    return TC_OK;
}

}  // extern "C"
