// Serving loop over the C ABI: continuous batching of DVM simulations with
// HBM-budget admission (declared in include/dvm_cuda.h, dvm_server_*).
//
// Each tick: admit every arrived request that fits (FIFO, no overtaking), step
// all admitted simulations once with dvm_step_batch (one batched launch
// sequence; a CUDA graph while the batch is unchanged), then retire the
// finished ones.  Simulation state never leaves the device until retirement.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "../../include/dvm_cuda.h"
#include "dvm_internal.h"

namespace {

struct Request {
    uint64_t id = 0;
    dvm_sim_params p{};
    std::vector<double> bx, bz;
    uint32_t steps = 0;
    double arrival = 0.0;
    // run state
    dvm_sim* sim = nullptr;
    uint64_t bytes = 0;
    uint32_t done = 0;
    double admitted = -1.0, finished = -1.0;
    int status = DVM_OK;
    uint64_t blobs = 0;
    double fx = 0, fz = 0, cd = 0, cl = 0;
    std::vector<double> x, z, circ;  // final state (keep_state)
};

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t lo = (size_t)std::floor(pos), hi = std::min(v.size() - 1, lo + 1);
    return v[lo] + (pos - (double)lo) * (v[hi] - v[lo]);
}

}  // namespace

struct dvm_server {
    dvm_ctx* ctx = nullptr;
    uint64_t budget = 0;
    int max_active = 64;
    bool keep = false;
    std::vector<Request> reqs;
    dvm_server_summary stats{};
    bool ran = false;
    bool graph = true;       // DVM_SERVE_GRAPH
    bool sync_tick = true;   // DVM_SERVE_SYNC
    bool autotune = false;   // DVM_SERVE_AUTOTUNE
    std::set<int> tuned;     // shape classes already tuned
    uint32_t tunings = 0;
};

extern "C" {

int dvm_server_create(dvm_ctx* ctx, uint64_t budget, int max_active, int keep_state,
                      dvm_server** out) {
    if (!ctx || !out || max_active < 1 || max_active > 1024)
        return dvmk::report_error(DVM_ERR_ARG, "dvm_server_create: bad argument");
    auto* s = new dvm_server();
    s->ctx = ctx;
    s->max_active = max_active;
    s->keep = keep_state != 0;
    if (budget == 0) {
        uint64_t used = 0, total = 0;
        dvm_ctx_memory(ctx, &used, &total);
        budget = total > used ? total - used : 0;
    }
    s->budget = budget;
    *out = s;
    return DVM_OK;
}

int dvm_server_destroy(dvm_server* s) {
    if (!s) return DVM_OK;
    for (auto& r : s->reqs)
        if (r.sim) dvm_sim_destroy(r.sim);
    delete s;
    return DVM_OK;
}

int dvm_server_set_option(dvm_server* s, int option, int value) {
    if (!s) return dvmk::report_error(DVM_ERR_ARG, "server is null");
    switch (option) {
        case DVM_SERVE_GRAPH: s->graph = value != 0; return DVM_OK;
        case DVM_SERVE_SYNC: s->sync_tick = value != 0; return DVM_OK;
        case DVM_SERVE_AUTOTUNE: s->autotune = value != 0; return DVM_OK;
        default: return dvmk::report_error(DVM_ERR_ARG, "dvm_server_set_option: unknown option");
    }
}

int dvm_server_submit(dvm_server* s, const dvm_sim_params* p, const double* bx, const double* bz,
                      int npts, uint32_t steps, double arrival, uint64_t* id) {
    if (!s || !p || !bx || !bz || npts < 3 || steps == 0)
        return dvmk::report_error(DVM_ERR_ARG, "dvm_server_submit: bad argument");
    if (s->ran) return dvmk::report_error(DVM_ERR_STATE, "dvm_server_submit: server already ran");
    Request r;
    r.id = s->reqs.size();
    r.p = *p;
    r.bx.assign(bx, bx + npts);
    r.bz.assign(bz, bz + npts);
    r.steps = steps;
    r.arrival = arrival;
    const int rc = dvm_sim_bytes(p, npts - 1, &r.bytes);
    if (rc) return rc;
    if (r.bytes > s->budget)
        return dvmk::report_error(DVM_ERR_OOM, "dvm_server_submit: request larger than the budget");
    if (id) *id = r.id;
    s->reqs.push_back(std::move(r));
    return DVM_OK;
}

int dvm_server_run(dvm_server* s, int serial, int realtime) {
    if (!s) return dvmk::report_error(DVM_ERR_ARG, "server is null");
    if (s->ran) return dvmk::report_error(DVM_ERR_STATE, "dvm_server_run: already ran");
    s->ran = true;
    const int cap_active = serial ? 1 : s->max_active;
    // Size the shared workspace once for the largest batch this run can form
    // (the cap_active largest capacities), so admissions never reallocate it.
    {
        std::vector<uint64_t> caps;
        int max_np = 2;
        bool del = false;
        for (auto& r : s->reqs) {
            caps.push_back(r.p.capacity);
            max_np = std::max(max_np, (int)r.bx.size() - 1);
            del = del || r.p.surface_cross == DVM_DELETE;
        }
        std::sort(caps.rbegin(), caps.rend());
        uint64_t T = 0;
        for (size_t i = 0; i < caps.size() && (int)i < cap_active; ++i) T += caps[i];
        const int rc = dvm_ctx_reserve(s->ctx, T, std::max(1, std::min(cap_active, (int)caps.size())),
                                       max_np, del ? 1 : 0);
        if (rc) return rc;
        uint64_t used = 0, total = 0;
        dvm_ctx_memory(s->ctx, &used, &total);
        s->budget = std::min<uint64_t>(s->budget, total > used ? total - used : 0);
        // Map the pool once for the cap_active largest slabs (and the largest
        // set-up scratch), within the budget, so admissions do not grow it.
        std::vector<uint64_t> slabs;
        uint64_t scratch = 0;
        for (auto& r : s->reqs) {
            slabs.push_back(r.bytes);
            const uint64_t np = r.bx.size() - 1;  // influence + factorisation scratch
            scratch = std::max<uint64_t>(
                scratch, 8 * (2 * np * np + dvmk::pseudo_inverse_work_doubles((int)np)));
        }
        std::sort(slabs.rbegin(), slabs.rend());
        uint64_t want = scratch;
        for (size_t i = 0; i < slabs.size() && (int)i < cap_active; ++i) want += slabs[i];
        // (an unreserved pool still works, only slower to admit)
        (void)dvm_ctx_pool_reserve(s->ctx, std::min<uint64_t>(want, s->budget));
    }
    std::vector<size_t> order(s->reqs.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t a, size_t b) { return s->reqs[a].arrival < s->reqs[b].arrival; });
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    auto now = [&]() { return std::chrono::duration<double>(clk::now() - t0).count(); };
    size_t next = 0, finished = 0;
    std::deque<size_t> waiting;
    std::vector<size_t> active;
    uint64_t in_use = 0, peak = 0, ticks = 0, sim_steps = 0;
    uint32_t peak_active = 0;
    std::vector<dvm_sim*> batch;
    std::vector<int32_t> tick_status;
    double t_admit = 0.0, t_step = 0.0, t_retire = 0.0;
    while (finished < s->reqs.size()) {
        const double t = now();
        while (next < order.size() && (!realtime || s->reqs[order[next]].arrival <= t))
            waiting.push_back(order[next++]);
        // admission: FIFO while a slot is free and the slab fits the budget
        const double ta = now();
        while (!waiting.empty() && (int)active.size() < cap_active) {
            Request& r = s->reqs[waiting.front()];
            if (in_use + r.bytes > s->budget) break;
            const int rc = dvm_sim_create(s->ctx, &r.p, r.bx.data(), r.bz.data(),
                                          (int)r.bx.size(), &r.sim);
            if (rc == DVM_ERR_OOM && !active.empty()) break;  // wait for memory to free up
            waiting.pop_front();
            r.admitted = now();
            if (rc) {
                r.status = rc;
                r.finished = r.admitted;
                ++finished;
                continue;
            }
            in_use += r.bytes;
            active.push_back((size_t)r.id);
        }
        t_admit += now() - ta;
        peak = std::max(peak, in_use);
        peak_active = std::max<uint32_t>(peak_active, (uint32_t)active.size());
        if (active.empty()) {
            if (next < order.size() && realtime) {
                const double wait = s->reqs[order[next]].arrival - now();
                if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait));
            }
            continue;
        }
        batch.clear();
        for (size_t i : active) batch.push_back(s->reqs[i].sim);
        // With DVM_SERVE_SYNC each tick is waited for (device status read per
        // simulation); without it the host runs ahead and the status of a
        // simulation is read only when it retires (step counts are host-known).
        const double tsx = now();
        if (s->autotune) {  // once per new shape class (tuning never changes results)
            int cls = -1;
            int rc = dvm_batch_shape_class(s->ctx, batch.data(), (int)batch.size(), &cls);
            if (rc) return rc;
            if (cls >= 0 && s->tuned.insert(cls).second) {
                dvm_tune_result tr;
                rc = dvm_ctx_autotune(s->ctx, batch.data(), (int)batch.size(), 1, &tr);
                if (rc) return rc;
                ++s->tunings;
            }
        }
        int rc = dvm_step_batch(s->ctx, batch.data(), (int)batch.size(), 1, s->graph ? 1 : 0);
        if (rc) return rc;
        ++ticks;
        sim_steps += active.size();
        if (s->sync_tick) {  // one status copy (and wait) for the whole tick
            tick_status.resize(batch.size());
            rc = dvm_batch_status(s->ctx, batch.data(), (int)batch.size(), tick_status.data());
            if (rc) return rc;
        }
        const double tr = now();
        t_step += tr - tsx;
        // retire: finished (or failed) simulations leave the batch at once
        std::vector<size_t> keep_active;
        for (size_t a = 0; a < active.size(); ++a) {
            const size_t i = active[a];
            Request& r = s->reqs[i];
            r.done += 1;
            int st = DVM_OK;
            if (s->sync_tick) st = tick_status[a];
            if (st == DVM_OK && r.done < r.steps) {
                keep_active.push_back(i);
                continue;
            }
            r.status = s->sync_tick ? st : dvm_sim_status(r.sim);
            if (r.status != DVM_OK) dvm_sim_status(r.sim);  // sets the thread's error message
            dvm_sim_get_loads(r.sim, &r.fx, &r.fz, &r.cd, &r.cl);
            dvm_sim_num_blobs(r.sim, &r.blobs);
            if (s->keep) {
                r.x.resize(r.blobs);
                r.z.resize(r.blobs);
                r.circ.resize(r.blobs);
                uint64_t n = 0;
                dvm_sim_get_blobs(r.sim, r.blobs, &n, r.x.data(), r.z.data(), r.circ.data(),
                                  nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
            }
            dvm_sim_destroy(r.sim);
            r.sim = nullptr;
            in_use -= r.bytes;
            r.finished = now();
            ++finished;
        }
        active.swap(keep_active);
        t_retire += now() - tr;
    }
    const double wall = now();
    std::vector<double> lat, queue;
    uint64_t failed = 0;
    for (auto& r : s->reqs) {
        if (r.status != DVM_OK) ++failed;
        lat.push_back(r.finished - (realtime ? r.arrival : 0.0));
        queue.push_back(r.admitted - (realtime ? r.arrival : 0.0));
    }
    dvm_server_summary& S = s->stats;
    std::memset(&S, 0, sizeof(S));
    S.requests = s->reqs.size();
    S.completed = S.requests - failed;
    S.failed = failed;
    S.sim_steps = sim_steps;
    S.ticks = ticks;
    S.wall_s = wall;
    S.sim_steps_per_s = wall > 0 ? (double)sim_steps / wall : 0.0;
    S.admit_s = t_admit;
    S.step_s = t_step;
    S.retire_s = t_retire;
    S.tunings = s->tunings;
    S.latency_p50_s = percentile(lat, 0.50);
    S.latency_p95_s = percentile(lat, 0.95);
    S.latency_p99_s = percentile(lat, 0.99);
    double m = 0;
    for (double v : lat) m += v;
    S.latency_mean_s = lat.empty() ? 0 : m / (double)lat.size();
    S.queue_p50_s = percentile(queue, 0.50);
    S.queue_p99_s = percentile(queue, 0.99);
    S.peak_active = peak_active;
    S.peak_bytes = peak;
    return DVM_OK;
}

int dvm_server_result(dvm_server* s, uint64_t id, dvm_request_result* out) {
    if (!s || !out || id >= s->reqs.size())
        return dvmk::report_error(DVM_ERR_ARG, "dvm_server_result: bad request id");
    const Request& r = s->reqs[id];
    out->id = r.id;
    out->arrival_s = r.arrival;
    out->admitted_s = r.admitted;
    out->finished_s = r.finished;
    out->latency_s = r.finished - r.arrival;
    out->steps_done = r.done;
    out->status = r.status;
    out->blobs = r.blobs;
    out->fx = r.fx;
    out->fz = r.fz;
    out->cd = r.cd;
    out->cl = r.cl;
    return DVM_OK;
}

int dvm_server_final_blobs(dvm_server* s, uint64_t id, uint64_t cap, uint64_t* n, double* x,
                           double* z, double* circ) {
    if (!s || id >= s->reqs.size())
        return dvmk::report_error(DVM_ERR_ARG, "dvm_server_final_blobs: bad request id");
    const Request& r = s->reqs[id];
    if (!s->keep) return dvmk::report_error(DVM_ERR_STATE, "server created without keep_state");
    if (n) *n = r.x.size();
    if (r.x.size() > cap && (x || z || circ))
        return dvmk::report_error(DVM_ERR_ARG, "output capacity smaller than the blob count");
    if (x) std::memcpy(x, r.x.data(), 8 * r.x.size());
    if (z) std::memcpy(z, r.z.data(), 8 * r.z.size());
    if (circ) std::memcpy(circ, r.circ.data(), 8 * r.circ.size());
    return DVM_OK;
}

int dvm_server_stats(dvm_server* s, dvm_server_summary* out) {
    if (!s || !out) return dvmk::report_error(DVM_ERR_ARG, "null argument");
    *out = s->stats;
    return DVM_OK;
}

}  // extern "C"
