// Served form: a request loop with continuous batching on top of OpoBatch.
//
// Requests (sweep points: one OPO instance each) arrive on the wall clock.  Between
// round trips the loop admits every arrived request that fits a free slot and the HBM
// budget (fields initialised on the device), runs one batched round trip of all
// resident instances, tallies their powers in FP64, and retires each instance whose
// signal power changed by less than its tolerance over the last round trip, that
// reached its round-trip limit, or whose fields stopped being finite.  Requests that
// are malformed or larger than the whole budget are answered at once with an error.
// The reference has no serving layer: its sweep is a bash loop that re-runs the binary
// per point (cuOPO3D.sh:65-86).

#include <algorithm>
#include <chrono>
#include <cmath>
#include <deque>
#include <thread>
#include <vector>

#include "../../include/cuopo3d.h"
#include "solver_internal.h"

namespace {

double now_s(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

double percentile(std::vector<double> v, double q)
{
    if (v.empty()) return 0;
    std::sort(v.begin(), v.end());
    const double pos = q * (v.size() - 1);
    const size_t lo = (size_t)pos;
    const size_t hi = std::min(lo + 1, v.size() - 1);
    return v[lo] + (pos - lo) * (v[hi] - v[lo]);
}

struct Live {
    int req;
    int slot;
    double prev_ps;
};

}  // namespace

extern "C" int opo_serve(const OpoServeRequest *reqs, int n, const OpoServeOptions *opt, OpoServeResult *out,
                         double stats[8])
{
    if (!reqs || n < 0 || !opt || !out || !stats) return OPO_ERR_INVALID;
    OpoBatch *b = nullptr;
    int rc = opo_batch_create(opt->precision, opt->capacity, opt->hbm_budget, opt->tuning_set ? opt->tuning : nullptr, &b);
    if (rc) return rc;
    const auto t0 = std::chrono::steady_clock::now();
    std::deque<int> waiting;  // arrived, not yet admitted (FIFO)
    std::vector<Live> live;
    int next = 0, done = 0, max_live = 0;
    long long total_vs = 0;
    std::vector<double> sums(3 * (size_t)opt->capacity);
    for (int k = 0; k < n; k++) {
        out[k] = OpoServeResult{};
        out[k].status = -1;
    }
    auto finish = [&](int r, int status, int rts, const double *p) {
        OpoServeResult &o = out[r];
        o.status = status;
        o.round_trips = rts;
        o.done_s = now_s(t0);
        o.latency_s = o.done_s - reqs[r].arrival_s;
        if (p)
            for (int k = 0; k < 3; k++) o.power[k] = p[k];
        done++;
    };
    while (done < n) {
        const double t = now_s(t0);
        while (next < n && (!opt->realtime || reqs[next].arrival_s <= t)) waiting.push_back(next++);
        // admission, FIFO; a request that does not fit waits for slots or memory to free up
        while (!waiting.empty()) {
            const int r = waiting.front();
            const OpoServeRequest &q = reqs[r];
            OpoParams p;
            if (q.cfg.precision != opt->precision || opo_params_from_config(&q.cfg, &p, nullptr) != OPO_OK) {
                waiting.pop_front();
                finish(r, OPO_ERR_INVALID, 0, nullptr);
                continue;
            }
            if (opo::batch_instance_bytes(opt->precision, (size_t)p.nx * p.ny * p.nt) > opt->hbm_budget) {
                waiting.pop_front();
                finish(r, OPO_ERR_CAPACITY, 0, nullptr);
                continue;
            }
            std::vector<double> w(p.nt);
            opo_time_freq(p.nt, p.t_window, nullptr, w.data());
            int slot = -1;
            rc = opo_batch_add(b, &p, w.data(), &slot);
            if (rc == OPO_ERR_CAPACITY) {
                // no slot, no memory, or another z-step count than the resident instances:
                // wait for a retirement -- unless nothing is resident, when no retirement
                // can ever make room
                if (!live.empty()) break;
                waiting.pop_front();
                finish(r, OPO_ERR_CAPACITY, 0, nullptr);
                continue;
            }
            if (rc == OPO_ERR_INVALID) {
                waiting.pop_front();
                finish(r, OPO_ERR_INVALID, 0, nullptr);
                continue;
            }
            if (rc) goto fail;
            rc = opo_batch_init_fields(b, slot, &q.cfg, q.seed, q.noise_sigma, 0);
            if (rc) goto fail;
            waiting.pop_front();
            out[r].admit_s = now_s(t0);
            live.push_back(Live{r, slot, -1.0});
        }
        max_live = std::max(max_live, (int)live.size());
        if (live.empty()) {
            if (next < n && opt->realtime) {
                const double dt = reqs[next].arrival_s - now_s(t0);
                if (dt > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(dt, 0.05)));
            }
            continue;
        }
        if ((rc = opo_batch_run_round_trips(b, 1))) goto fail;
        if ((rc = opo_batch_sums(b, sums.data()))) goto fail;
        for (size_t k = 0; k < live.size();) {
            Live &L = live[k];
            long long info[4];
            opo_batch_info(b, L.slot, info);
            const double *ps = &sums[3 * (size_t)L.slot];
            const bool finite = std::isfinite(ps[0]) && std::isfinite(ps[1]) && std::isfinite(ps[2]);
            const double tol = reqs[L.req].tol;
            const bool steady = L.prev_ps > 0 && tol > 0 && std::fabs(ps[1] - L.prev_ps) <= tol * std::fabs(L.prev_ps);
            const bool limit = info[0] >= info[1];
            L.prev_ps = ps[1];
            if (!finite || steady || limit) {
                OpoParams p;
                opo_params_from_config(&reqs[L.req].cfg, &p, nullptr);
                for (int f = 0; f < 3; f++)
                    if (reqs[L.req].out_fields[f] &&
                        (rc = opo_batch_get_field(b, L.slot, OPO_FIELD_PUMP + f, reqs[L.req].out_fields[f],
                                                  OPO_MEM_HOST, OPO_FP64)))
                        goto fail;
                out[L.req].voxel_steps = info[0] * (long long)p.n_steps * info[2];
                total_vs += out[L.req].voxel_steps;
                finish(L.req, finite ? OPO_OK : OPO_ERR_NONFINITE, (int)info[0], ps);
                opo_batch_remove(b, L.slot);
                live.erase(live.begin() + k);
            } else {
                k++;
            }
        }
    }
    {
        const double wall = now_s(t0);
        std::vector<double> lat;
        for (int k = 0; k < n; k++)
            if (out[k].status == OPO_OK) lat.push_back(out[k].latency_s);
        stats[0] = percentile(lat, 0.5);
        stats[1] = percentile(lat, 0.99);
        stats[2] = wall;
        stats[3] = wall > 0 ? total_vs / wall : 0;
        stats[4] = max_live;
        long long st[4];
        opo_batch_stats(b, st);
        stats[5] = (double)st[3];
        stats[6] = (double)total_vs;
        stats[7] = (double)lat.size();
    }
    opo_batch_destroy(b);
    return OPO_OK;
fail:
    opo_batch_destroy(b);
    return rc;
}
