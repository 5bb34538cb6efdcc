// Random request streams against the request server (with the stand-in context API).
// Checks: every request completes, each output carries its own request's marker, one
// client's requests run in submission order, no context outlives the server, and -- when
// contexts never exceed their estimate -- the charged device memory stays within the budget.
// Exit status 0 on success; a hang is caught by the caller's timeout.
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <map>
#include <thread>
#include <vector>

#include "treecodes_b200.h"

extern std::atomic<int> g_live, g_order_errors;
extern double g_actual_lo, g_actual_hi;

int main(int argc, char **argv) {
    const int trials = argc > 1 ? atoi(argv[1]) : 50;
    g_actual_lo = argc > 2 ? atof(argv[2]) : 0.9;
    g_actual_hi = argc > 3 ? atof(argv[3]) : 0.9;
    std::mt19937 rng(argc > 4 ? atoi(argv[4]) : 1);
    int failures = 0;
    std::map<long long, long long> seq;   // client id -> last sequence number handed out
    for (int trial = 0; trial < trials; ++trial) {
        const size_t budget = (size_t)(24 + rng() % 400) << 20;
        tc_server *s;
        const int nslots = 1 + rng() % 4;
        if (tc_server_create(&s, 0, nslots, budget)) return 10;
        // with 3 slots or more the last one (the express slot) runs only requests of at most
        // 2^17 sources
        auto check_slot = [&](const tc_request_result &res, int nsrc) {
            if (nslots >= 3 && nsrc > (1 << 17) && res.slot == nslots - 1) {
                fprintf(stderr, "trial %d: a request of %d sources ran on the express slot\n",
                        trial, nsrc);
                ++failures;
            }
        };
        std::vector<int> nsrc_of;
        const int nreq = 40 + rng() % 40;
        std::vector<std::vector<double>> in(nreq), out(nreq);
        std::vector<long long> tickets;
        std::vector<double> marker(nreq);
        for (int i = 0; i < nreq; ++i) {
            tc_request r{};
            r.kind = rng() % 2;
            r.precision = rng() % 2;
            r.theta = 0.5;
            // client ids are unique to the trial (at most 8 per trial, below 1024 overall)
            r.client = (rng() % 3 == 0) ? 1 + (trial % 120) * 8 + rng() % 5 : 0;
            r.nsources = 1000 + rng() % 150000;
            nsrc_of.push_back(r.nsources);
            in[i] = {(double)r.client, (double)(r.client > 0 ? ++seq[r.client] : 0)};
            r.xsources = r.ysources = r.sourcevalues = in[i].data();
            marker[i] = in[i][0] * 1e6 + in[i][1];
            if (r.kind == 0) {
                r.ntargets = 8;
                r.xtargets = r.ytargets = in[i].data();
                out[i].assign(8, -1);
                r.out0 = out[i].data();
            } else {
                r.nblocks = 1;
                r.x0s = r.y0s = r.hs = in[i].data();
                out[i].assign(2048, -1);
                r.out0 = out[i].data();
                r.out1 = r.out0 + 1024;
            }
            long long t;
            if (tc_server_submit(s, &r, &t)) return 11;
            tickets.push_back(t);
            if (rng() % 4 == 0) std::this_thread::sleep_for(std::chrono::microseconds(rng() % 300));
        }
        if (trial % 2 == 0) {
            for (int i = 0; i < nreq; ++i) {
                tc_request_result res;
                if (tc_server_wait(s, tickets[i], &res) != 0) ++failures;
                check_slot(res, nsrc_of[i]);
                for (double v : out[i])
                    if (v != marker[i]) ++failures;
            }
        } else {
            // one ticket by tc_server_wait, the rest in completion order by tc_server_wait_any:
            // every ticket exactly once, completion stamps non-decreasing, then nothing left
            std::map<long long, int> index;
            for (int i = 0; i < nreq; ++i) index[tickets[i]] = i;
            const int mid = nreq / 2;
            tc_request_result res;
            if (tc_server_wait(s, tickets[mid], &res) != 0) ++failures;
            index.erase(tickets[mid]);
            for (double v : out[mid])
                if (v != marker[mid]) ++failures;
            double last = -1.0;
            for (int k = 0; k + 1 < nreq; ++k) {
                long long t = 0;
                const int rc = tc_server_wait_any(s, &t, &res);
                auto it = index.find(t);
                if (rc != 0 || it == index.end()) {
                    fprintf(stderr, "trial %d: wait_any gave ticket %lld (status %d)\n", trial, t, rc);
                    ++failures;
                    continue;
                }
                const int i = it->second;
                index.erase(it);
                check_slot(res, nsrc_of[i]);
                if (res.finished_s < last) ++failures;
                last = res.finished_s;
                for (double v : out[i])
                    if (v != marker[i]) ++failures;
            }
            long long t = -1;
            if (tc_server_wait_any(s, &t, nullptr) != TC_ERR_INVALID || t != 0) ++failures;
            if (!index.empty()) ++failures;
        }
        tc_server_stats st;
        tc_server_get_stats(s, &st);
        if (st.completed != nreq) ++failures;
        if (g_actual_hi <= 1.0 && st.hbm_peak > budget) {
            fprintf(stderr, "trial %d: peak %zu > budget %zu\n", trial, st.hbm_peak, budget);
            ++failures;
        }
        tc_server_destroy(s);
        if (g_live != 0) {
            fprintf(stderr, "trial %d: %d contexts alive after destroy\n", trial, g_live.load());
            ++failures;
        }
        seq.clear();
    }
    if (g_order_errors) fprintf(stderr, "%d out-of-order client steps\n", g_order_errors.load());
    printf("trials %d failures %d order_errors %d\n", trials, failures, g_order_errors.load());
    return failures || g_order_errors ? 1 : 0;
}
