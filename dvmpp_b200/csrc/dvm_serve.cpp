// Serving loop over the C ABI: continuous batching of DVM simulations with
// HBM-budget admission (declared in include/dvm_cuda.h, dvm_server_*).
//
// Each tick: take in the requests submitted since the last one (other host
// threads may submit while the loop runs), admit every arrived request that
// fits (FIFO, no overtaking), step all admitted simulations once with
// dvm_step_batch (one batched launch sequence; a CUDA graph while the batch is
// unchanged), then retire the finished ones.  Simulation state never leaves
// the device until retirement.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
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
    double submitted = 0.0;  // run-clock time of submission (0 before the run)
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
    // Requests by id (stable addresses).  `mu` guards reqs, the intake and the
    // run flags: dvm_server_submit / _result / _close_intake may be called from
    // other host threads while dvm_server_run works.
    std::mutex mu;
    std::condition_variable cv;             // signalled on submit and on close
    std::vector<std::unique_ptr<Request>> reqs;
    std::vector<size_t> intake;             // ids submitted while running, not yet seen
    dvm_server_summary stats{};
    bool running = false, ran = false;
    bool intake_closed = false;
    std::chrono::steady_clock::time_point t0;
    bool graph = true;       // DVM_SERVE_GRAPH
    bool sync_tick = true;   // DVM_SERVE_SYNC
    bool autotune = false;   // DVM_SERVE_AUTOTUNE
    bool live = false;       // DVM_SERVE_LIVE
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
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->running)
            return dvmk::report_error(DVM_ERR_STATE, "dvm_server_destroy: the server is running");
    }
    for (auto& r : s->reqs)
        if (r->sim) dvm_sim_destroy(r->sim);
    delete s;
    return DVM_OK;
}

int dvm_server_set_option(dvm_server* s, int option, int value) {
    if (!s) return dvmk::report_error(DVM_ERR_ARG, "server is null");
    switch (option) {
        case DVM_SERVE_GRAPH: s->graph = value != 0; return DVM_OK;
        case DVM_SERVE_SYNC: s->sync_tick = value != 0; return DVM_OK;
        case DVM_SERVE_AUTOTUNE: s->autotune = value != 0; return DVM_OK;
        case DVM_SERVE_LIVE: s->live = value != 0; return DVM_OK;
        default: return dvmk::report_error(DVM_ERR_ARG, "dvm_server_set_option: unknown option");
    }
}

int dvm_server_submit(dvm_server* s, const dvm_sim_params* p, const double* bx, const double* bz,
                      int npts, uint32_t steps, double arrival, uint64_t* id) {
    if (!s || !p || !bx || !bz || npts < 3 || steps == 0)
        return dvmk::report_error(DVM_ERR_ARG, "dvm_server_submit: bad argument");
    auto r = std::make_unique<Request>();
    r->p = *p;
    r->bx.assign(bx, bx + npts);
    r->bz.assign(bz, bz + npts);
    r->steps = steps;
    int rc = dvm_sim_bytes(p, npts - 1, &r->bytes);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->ran) return dvmk::report_error(DVM_ERR_STATE, "dvm_server_submit: the run has ended");
    if (s->running && s->intake_closed)
        return dvmk::report_error(DVM_ERR_STATE, "dvm_server_submit: intake closed");
    if (r->bytes > s->budget)
        return dvmk::report_error(DVM_ERR_OOM, "dvm_server_submit: request larger than the budget");
    r->id = s->reqs.size();
    if (s->running) {
        // a live request: it arrives now on the run's clock (or at the given
        // later time); its latency counts from its submission in every mode
        const double now =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - s->t0).count();
        r->submitted = now;
        r->arrival = arrival < 0 ? now : std::max(arrival, now);
        s->intake.push_back(r->id);
    } else {
        r->arrival = arrival < 0 ? 0.0 : arrival;
    }
    if (id) *id = r->id;
    s->reqs.push_back(std::move(r));
    s->cv.notify_all();
    return DVM_OK;
}

int dvm_server_close_intake(dvm_server* s) {
    if (!s) return dvmk::report_error(DVM_ERR_ARG, "server is null");
    std::lock_guard<std::mutex> lk(s->mu);
    s->intake_closed = true;
    s->cv.notify_all();
    return DVM_OK;
}

int dvm_server_run(dvm_server* s, int serial, int realtime) {
    if (!s) return dvmk::report_error(DVM_ERR_ARG, "server is null");
    using clk = std::chrono::steady_clock;
    std::vector<Request*> pre;  // submitted before the run
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->ran || s->running) return dvmk::report_error(DVM_ERR_STATE, "dvm_server_run: already ran");
        s->running = true;
        for (auto& r : s->reqs) pre.push_back(r.get());
    }
    const int cap_active = serial ? 1 : s->max_active;
    // Size the shared workspace once for the largest batch the pre-submitted
    // requests can form (the cap_active largest capacities), so admissions do
    // not reallocate it; live requests beyond that grow it when they join.
    if (!pre.empty()) {
        std::vector<uint64_t> caps;
        int max_np = 2;
        bool del = false;
        for (Request* r : pre) {
            caps.push_back(r->p.capacity);
            max_np = std::max(max_np, (int)r->bx.size() - 1);
            del = del || r->p.surface_cross == DVM_DELETE;
        }
        std::sort(caps.rbegin(), caps.rend());
        uint64_t T = 0;
        for (size_t i = 0; i < caps.size() && (int)i < cap_active; ++i) T += caps[i];
        const int rc = dvm_ctx_reserve(s->ctx, T, std::max(1, std::min(cap_active, (int)caps.size())),
                                       max_np, del ? 1 : 0);
        if (rc) {
            std::lock_guard<std::mutex> lk(s->mu);
            s->running = false;
            return rc;
        }
        uint64_t used = 0, total = 0;
        dvm_ctx_memory(s->ctx, &used, &total);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->budget = std::min<uint64_t>(s->budget, total > used ? total - used : 0);
        }
        // Map the pool once for the cap_active largest slabs (and the largest
        // set-up scratch), within the budget, so admissions do not grow it.
        std::vector<uint64_t> slabs;
        uint64_t scratch = 0;
        for (Request* r : pre) {
            slabs.push_back(r->bytes);
            const uint64_t np = r->bx.size() - 1;  // influence + factorisation scratch
            scratch = std::max<uint64_t>(
                scratch, 8 * (2 * np * np + dvmk::pseudo_inverse_work_doubles((int)np)));
        }
        std::sort(slabs.rbegin(), slabs.rend());
        uint64_t want = scratch;
        for (size_t i = 0; i < slabs.size() && (int)i < cap_active; ++i) want += slabs[i];
        // (an unreserved pool still works, only slower to admit)
        (void)dvm_ctx_pool_reserve(s->ctx, std::min<uint64_t>(want, s->budget));
    }
    std::vector<Request*> order = pre;  // not yet arrived, by arrival time
    std::stable_sort(order.begin(), order.end(),
                     [](const Request* a, const Request* b) { return a->arrival < b->arrival; });
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->t0 = clk::now();  // the run's clock: live submissions are stamped on it
    }
    const auto t0 = s->t0;
    auto now = [&]() { return std::chrono::duration<double>(clk::now() - t0).count(); };
    size_t next = 0;
    std::deque<Request*> waiting;
    std::vector<Request*> active;
    uint64_t in_use = 0, peak = 0, ticks = 0, sim_steps = 0;
    uint32_t peak_active = 0;
    std::vector<dvm_sim*> batch;
    std::vector<int32_t> tick_status;
    double t_admit = 0.0, t_step = 0.0, t_retire = 0.0;
    int run_rc = DVM_OK;
    for (;;) {
        // live requests submitted since the last tick join the arrival order
        bool closed = false;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            std::vector<Request*> fresh;
            for (size_t id : s->intake) fresh.push_back(s->reqs[id].get());
            s->intake.clear();
            closed = s->intake_closed;
            if (!fresh.empty()) {
                std::vector<Request*> rest(order.begin() + (long)next, order.end());
                rest.insert(rest.end(), fresh.begin(), fresh.end());
                std::stable_sort(rest.begin(), rest.end(), [](const Request* a, const Request* b) {
                    return a->arrival < b->arrival;
                });
                order.assign(rest.begin(), rest.end());
                next = 0;
            }
        }
        const double t = now();
        while (next < order.size() && (!realtime || order[next]->arrival <= t))
            waiting.push_back(order[next++]);
        const bool idle = waiting.empty() && active.empty();
        if (idle && next >= order.size()) {
            if (!s->live || closed) break;  // every submitted request is done
            // live intake: wait for a submission or the close
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv.wait_for(lk, std::chrono::milliseconds(50),
                           [&] { return !s->intake.empty() || s->intake_closed; });
            continue;
        }
        // admission: FIFO while a slot is free and the slab fits the budget.  The
        // requests that fit now are created together (their bodies' factorisations
        // share launches); if that fails, the loop below takes them one at a time,
        // so a request that cannot be created fails alone.
        const double ta = now();
        {
            std::vector<Request*> group;
            uint64_t group_bytes = 0;
            for (Request* r : waiting) {
                if ((int)(active.size() + group.size()) >= cap_active) break;
                if (in_use + group_bytes + r->bytes > s->budget) break;
                group.push_back(r);
                group_bytes += r->bytes;
            }
            if (group.size() > 1) {
                const size_t g = group.size();
                std::vector<const dvm_sim_params*> ps(g);
                std::vector<const double*> xs(g), zs(g);
                std::vector<int> npts(g);
                std::vector<dvm_sim*> sims(g, nullptr);
                for (size_t k = 0; k < g; ++k) {
                    ps[k] = &group[k]->p;
                    xs[k] = group[k]->bx.data();
                    zs[k] = group[k]->bz.data();
                    npts[k] = (int)group[k]->bx.size();
                }
                if (dvm_sims_create(s->ctx, (int)g, ps.data(), xs.data(), zs.data(), npts.data(),
                                    sims.data()) == DVM_OK) {
                    const double t_adm = now();
                    std::lock_guard<std::mutex> lk(s->mu);
                    for (size_t k = 0; k < g; ++k) {
                        waiting.pop_front();
                        group[k]->sim = sims[k];
                        group[k]->admitted = t_adm;
                        in_use += group[k]->bytes;
                        active.push_back(group[k]);
                    }
                }
            }
        }
        while (!waiting.empty() && (int)active.size() < cap_active) {
            Request& r = *waiting.front();
            if (in_use + r.bytes > s->budget) break;
            dvm_sim* sim = nullptr;
            const int rc = dvm_sim_create(s->ctx, &r.p, r.bx.data(), r.bz.data(),
                                          (int)r.bx.size(), &sim);
            if (rc == DVM_ERR_OOM && !active.empty()) break;  // wait for memory to free up
            waiting.pop_front();
            std::lock_guard<std::mutex> lk(s->mu);
            r.sim = sim;
            r.admitted = now();
            if (rc) {
                r.status = rc;
                r.finished = r.admitted;
                continue;
            }
            in_use += r.bytes;
            active.push_back(&r);
        }
        t_admit += now() - ta;
        peak = std::max(peak, in_use);
        peak_active = std::max<uint32_t>(peak_active, (uint32_t)active.size());
        if (active.empty()) {
            if (realtime && next < order.size()) {  // sleep until the next arrival (or a submission)
                const double wait = order[next]->arrival - now();
                if (wait > 0) {
                    std::unique_lock<std::mutex> lk(s->mu);
                    s->cv.wait_for(lk, std::chrono::duration<double>(wait),
                                   [&] { return !s->intake.empty(); });
                }
            }
            continue;
        }
        batch.clear();
        for (Request* r : active) batch.push_back(r->sim);
        // With DVM_SERVE_SYNC each tick is waited for (device status read per
        // simulation); without it the host runs ahead and the status of a
        // simulation is read only when it retires (step counts are host-known).
        const double tsx = now();
        if (s->autotune) {  // once per new shape class (tuning never changes results)
            int cls = -1;
            int rc = dvm_batch_shape_class(s->ctx, batch.data(), (int)batch.size(), &cls);
            if (rc) { run_rc = rc; break; }
            if (cls >= 0 && s->tuned.insert(cls).second) {
                dvm_tune_result tr;
                rc = dvm_ctx_autotune(s->ctx, batch.data(), (int)batch.size(), 1, &tr);
                if (rc) { run_rc = rc; break; }
                ++s->tunings;
            }
        }
        int rc = dvm_step_batch(s->ctx, batch.data(), (int)batch.size(), 1, s->graph ? 1 : 0);
        if (rc) { run_rc = rc; break; }
        ++ticks;
        sim_steps += active.size();
        if (s->sync_tick) {  // one status copy (and wait) for the whole tick
            tick_status.resize(batch.size());
            rc = dvm_batch_status(s->ctx, batch.data(), (int)batch.size(), tick_status.data());
            if (rc) { run_rc = rc; break; }
        }
        const double tr = now();
        t_step += tr - tsx;
        // retire: finished (or failed) simulations leave the batch at once
        std::vector<Request*> keep_active;
        for (size_t a = 0; a < active.size(); ++a) {
            Request& r = *active[a];
            int st = DVM_OK;
            if (s->sync_tick) st = tick_status[a];
            if (st == DVM_OK && r.done + 1 < r.steps) {
                std::lock_guard<std::mutex> lk(s->mu);
                r.done += 1;
                keep_active.push_back(&r);
                continue;
            }
            int status = s->sync_tick ? st : dvm_sim_status(r.sim);
            if (status != DVM_OK) dvm_sim_status(r.sim);  // sets the thread's error message
            double fx = 0, fz = 0, cd = 0, cl = 0;
            uint64_t blobs = 0;
            dvm_sim_get_loads(r.sim, &fx, &fz, &cd, &cl);
            dvm_sim_num_blobs(r.sim, &blobs);
            std::vector<double> x, z, circ;
            if (s->keep) {
                x.resize(blobs);
                z.resize(blobs);
                circ.resize(blobs);
                uint64_t n = 0;
                dvm_sim_get_blobs(r.sim, blobs, &n, x.data(), z.data(), circ.data(), nullptr,
                                  nullptr, nullptr, nullptr, nullptr, nullptr);
            }
            dvm_sim_destroy(r.sim);
            in_use -= r.bytes;
            std::lock_guard<std::mutex> lk(s->mu);
            r.done += 1;
            r.status = status;
            r.fx = fx;
            r.fz = fz;
            r.cd = cd;
            r.cl = cl;
            r.blobs = blobs;
            r.x.swap(x);
            r.z.swap(z);
            r.circ.swap(circ);
            r.sim = nullptr;
            r.finished = now();
        }
        active.swap(keep_active);
        t_retire += now() - tr;
    }
    const double wall = now();
    std::lock_guard<std::mutex> lk(s->mu);
    if (run_rc != DVM_OK) {  // a failed launch: what is still active is released
        for (Request* r : active) {
            if (r->sim) dvm_sim_destroy(r->sim);
            r->sim = nullptr;
            r->status = run_rc;
        }
    }
    std::vector<double> lat, queue;
    uint64_t failed = 0, completed = 0;
    for (auto& rp : s->reqs) {
        const Request& r = *rp;
        if (r.finished < 0) continue;  // never reached (intake closed by an error)
        if (r.status != DVM_OK) ++failed;
        else ++completed;
        // latency from the request's arrival: its trace time when arrivals are
        // honoured, its submission otherwise (t = 0 for a pre-submitted trace)
        const double from = realtime ? r.arrival : r.submitted;
        lat.push_back(r.finished - from);
        queue.push_back(r.admitted - from);
    }
    dvm_server_summary& S = s->stats;
    std::memset(&S, 0, sizeof(S));
    S.requests = s->reqs.size();
    S.completed = completed;
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
    s->running = false;
    s->ran = true;
    s->cv.notify_all();
    return run_rc;
}

int dvm_server_result(dvm_server* s, uint64_t id, dvm_request_result* out) {
    if (!s || !out) return dvmk::report_error(DVM_ERR_ARG, "dvm_server_result: null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    if (id >= s->reqs.size()) return dvmk::report_error(DVM_ERR_ARG, "dvm_server_result: bad request id");
    const Request& r = *s->reqs[id];
    out->id = r.id;
    out->arrival_s = r.arrival;
    out->admitted_s = r.admitted;
    out->finished_s = r.finished;
    out->latency_s = r.finished >= 0 ? r.finished - r.arrival : -1.0;
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
    if (!s) return dvmk::report_error(DVM_ERR_ARG, "server is null");
    std::lock_guard<std::mutex> lk(s->mu);
    if (id >= s->reqs.size())
        return dvmk::report_error(DVM_ERR_ARG, "dvm_server_final_blobs: bad request id");
    const Request& r = *s->reqs[id];
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
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->stats;
    return DVM_OK;
}

}  // extern "C"
