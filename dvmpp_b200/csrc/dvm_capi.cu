// Host runtime and C ABI of libdvm_cuda.so (declared in include/dvm_cuda.h).
//
// A dvm_ctx owns one stream on one device, a table of simulation descriptors
// in device memory, an HBM budget, and a grow-only workspace shared by all
// batched launches.  A dvm_sim is one slab (one cudaMalloc) holding its blob
// arrays, body data and solver matrices.  Steps of any set of simulations are
// issued as one sequence of batched kernels (dvm_step_batch), optionally
// captured once in a CUDA graph and replayed.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_profiler_api.h>
#include <nvtx3/nvToolsExt.h>

#include "../../include/dvm_cuda.h"
#include "dvm_internal.h"

using namespace dvmk;

namespace {

thread_local std::string g_err;
std::atomic<uint64_t> g_launches{0};

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

}  // namespace

// Lets entry points defined in other translation units set dvm_last_error().
int dvmk::report_error(int code, const char* msg) { return fail(code, msg); }

namespace {

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(DVM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

constexpr size_t kMaxPlans = 32;       // cached batch plans per context (LRU)
constexpr size_t kPoolPerPlan = 6144;  // list entries per plan: 4 partitions + 1 reordered
                                       // pair-kernel list, x 1024 sims

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Source chunks of a simulation's pair kernel.  Fixed by the capacity alone, so
// a simulation's sums are associated the same way alone and inside any batch:
// at least one chunk per 32 k sources (up to 32), and for small simulations
// enough chunks (~2^23 / cap per 256-target tile, ~32 k work items) to occupy
// the GPU when stepped alone, but never chunks shorter than 512 sources.  In
// FP32 a chunk costs two 64-bit atomic adds per target (FP64: a partial sum).
int nbody_chunks(uint32_t cap) {
    const int by_size = (int)std::min<uint32_t>(32, (cap + 32767) / 32768);
    const int by_fill = (int)((8u << 20) / std::max<uint32_t>(cap, 1));
    const int most = (int)std::max<uint32_t>(1, std::min<uint32_t>(64, cap / 512));
    return std::max(1, std::min(most, std::max(by_size, by_fill)));
}

}  // namespace

struct SubList {
    std::vector<int> slots;
    ListEntry* d_list = nullptr;
    int n = 0;
    int max_np = 0;
    uint64_t total = 0;  // sum of capacities
    std::vector<ListEntry> host;  // the entries as uploaded
    // FP32 pair-kernel launch shape (from the context's tuning table) and, for
    // order 1, the same entries costliest-first (the pair kernel's list only)
    PairConfig cfg;
    int cls = -1;
    ListEntry* d_pair_list = nullptr;
};

// Batch-shape class of a tuning-table entry: log2 of the summed capacity of the
// FP32 simulations (capacity, not the device-resident blob count, so a plan's
// class is known on the host and stable) and a bucket of their number.
int shape_class(uint64_t total_cap, int count) {
    int lb = 0;
    while (lb < 40 && (1ull << lb) < total_cap) ++lb;
    const int cb = count <= 1 ? 0 : count <= 8 ? 1 : count <= 64 ? 2 : 3;
    return lb * 4 + cb;
}

// Order 1: entries whose work items cost most (item cost ~ capacity / chunks
// source pairs per target) first, ties in list order.
std::vector<ListEntry> costliest_first(const std::vector<ListEntry>& h) {
    std::vector<ListEntry> o(h);
    std::stable_sort(o.begin(), o.end(), [](const ListEntry& a, const ListEntry& b) {
        return (uint64_t)a.cap * (uint64_t)b.chunks > (uint64_t)b.cap * (uint64_t)a.chunks;
    });
    return o;
}

bool valid_pair_config(const dvm_pair_config& p) {
    if (p.tile != 256) return false;
    if (p.ctas_per_sm < 1 || p.ctas_per_sm > 4) return false;
    return p.order == 0 || p.order == 1;
}

struct Plan {
    std::vector<int> slots;            // the batch, in launch order
    SubList all, euler, rk3, rk3_f32, rk3_f64, eul_f32, eul_f64, refl, del;
    uint64_t ws_need_cap = 0;          // sizing inputs
    uint64_t part_elems = 0, rhs_elems = 0, circ_elems = 0;
    bool need_delete = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t ws_generation = 0;
    uint64_t launches_per_step = 0;
    bool warmed = false;  // one eager step issued (kernel attributes set, buffers touched)
    uint64_t last_use = 0;
    int pool_slot = -1;   // slot of the context's list pool holding the sublists
    int pool_used = 0;
};

struct dvm_ctx {
    int device = 0;
    int sms = 148;
    int cc_major = 0, cc_minor = 0;
    cudaStream_t stream = nullptr;
    uint64_t budget = 0, in_use = 0;
    InstDesc* d_table = nullptr;
    InstState* d_state = nullptr;
    std::vector<dvm_sim*> slots;  // index = table slot
    uint32_t next_uid = 1;
    // shared workspace
    Workspace ws;
    uint64_t ws_cap = 0, ws_part = 0, ws_rhs = 0, ws_circ = 0, ws_lists = 0;
    bool ws_delete = false;
    void* ws_block = nullptr;
    uint64_t ws_generation = 0;
    uint64_t ws_bytes = 0;
    // raw plugin-call scratch
    void* raw_block = nullptr;
    size_t raw_bytes = 0;
    std::map<std::vector<int>, Plan*> plans;
    // pair-kernel launch shapes chosen by dvm_ctx_autotune / set by the caller
    std::map<int, PairConfig> tuning;
    bool tuning_default_set = false;
    PairConfig tuning_default;
    ListEntry* d_tune_list = nullptr;  // scratch list for the tuner (1024 entries)
    InstState* h_state = nullptr;      // pinned copy of the state table (batched status)
    // Simulation slabs and set-up scratch come from this stream-ordered pool:
    // retiring a simulation returns its slab without a device-wide cudaFree
    // (which, measured, took 0.4 ms to over a second per call), and the next
    // admission reuses the memory.
    cudaMemPool_t mempool = nullptr;
    int h_state_slots = 0;
    uint64_t plan_clock = 0;
    ListEntry* list_pool = nullptr;  // kMaxPlans slots of kPoolPerPlan entries
    std::vector<int> pool_free;
    std::mutex mu;
    // CUDA-event profiling of kernel families on the ctx stream (eager steps only)
    bool profiling = false;
    // true while a step is being captured into a graph (no NVTX ranges then:
    // they would time the capture, not the work)
    bool capturing = false;
    struct Rec {
        int fam;
        cudaEvent_t a, b;
    };
    std::vector<Rec> pending;
    std::vector<cudaEvent_t> pool;
    double prof_ms[DVM_PROF_FAMILIES] = {};
    uint64_t prof_n[DVM_PROF_FAMILIES] = {};
    cudaEvent_t marks[16] = {};
    // pipelined host loops: a copy stream for uniforms pushed and snapshots
    // read back while the compute stream runs the neighbouring step
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t push_ev = nullptr, snap_ev = nullptr;
    double* snap_buf = nullptr;  // pool memory: x, z, circ of every snapshotted simulation
    uint64_t snap_doubles = 0;
    InstState* h_state_snap = nullptr;  // pinned copy of the state table at the snapshot
    uint64_t* h_ucount = nullptr;  // pinned staging of the uniform counts pushed asynchronously
    cudaEvent_t ucount_ev = nullptr;  // the last upload from h_ucount
    std::vector<int> snap_slots;
    std::vector<uint64_t> snap_off, snap_cap;
    bool snap_pending = false;
};

struct dvm_sim {
    dvm_ctx* ctx = nullptr;
    int slot = -1;
    dvm_sim_params p{};
    InstDesc h{};        // host copy of the descriptor in the table
    void* slab = nullptr;
    uint64_t bytes = 0;
    double* uniforms = nullptr;  // inject buffer (inside the slab)
    uint64_t ucap = 0;
    uint64_t consumed_base = 0;  // uniforms discarded by compaction
    // host-side panel data (reference geometry, src/VortexSheet.cpp:78-102)
    std::vector<double> xc, zc, ds, theta, enx, enz;
};

namespace {

// ---- plans ------------------------------------------------------------------------
void free_plan(dvm_ctx* c, Plan* pl) {
    if (!pl) return;
    if (pl->exec) cudaGraphExecDestroy(pl->exec);
    if (pl->graph) cudaGraphDestroy(pl->graph);
    if (pl->pool_slot >= 0) c->pool_free.push_back(pl->pool_slot);  // list memory is pooled
    delete pl;
}

// Drop the plans (and graphs) whose FP32 pair lists belong to shape class cls.
void drop_plans_of_class(dvm_ctx* c, int cls) {
    for (auto it = c->plans.begin(); it != c->plans.end();) {
        if (it->second->eul_f32.cls == cls || it->second->rk3_f32.cls == cls) {
            free_plan(c, it->second);
            it = c->plans.erase(it);
        } else {
            ++it;
        }
    }
}

void drop_plans_with(dvm_ctx* c, int slot) {
    for (auto it = c->plans.begin(); it != c->plans.end();) {
        if (slot < 0 || std::find(it->first.begin(), it->first.end(), slot) != it->first.end()) {
            free_plan(c, it->second);
            it = c->plans.erase(it);
        } else {
            ++it;
        }
    }
}

PairConfig tuned_config(const dvm_ctx* c, int cls) {
    auto it = c->tuning.find(cls);
    if (it != c->tuning.end()) return it->second;
    return c->tuning_default_set ? c->tuning_default : PairConfig();
}

// Stream-ordered allocation from the context's pool; on exhaustion the pool's
// cached memory is released to the device and the allocation retried once.
cudaError_t pool_alloc(dvm_ctx* c, void** p, size_t bytes) {
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes, c->mempool, c->stream);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        cudaStreamSynchronize(c->stream);
        cudaMemPoolTrimTo(c->mempool, 0);
        e = cudaMallocFromPoolAsync(p, bytes, c->mempool, c->stream);
    }
    return e;
}

void pool_free(dvm_ctx* c, void* p) {
    if (p) cudaFreeAsync(p, c->stream);
}

int build_sublist(dvm_ctx* c, SubList& sl, Plan& pl, bool f32_pairs = false) {
    sl.n = (int)sl.slots.size();
    if (sl.n == 0) return DVM_OK;
    if (pl.pool_used + (size_t)sl.n * (f32_pairs ? 2 : 1) > kPoolPerPlan)
        return fail(DVM_ERR_STATE, "plan list pool exhausted");
    std::vector<ListEntry> h(sl.n);
    uint64_t coff = 0, poff = 0, roff = 0, cofs = 0;
    for (int k = 0; k < sl.n; ++k) {
        const dvm_sim* s = c->slots[sl.slots[k]];
        ListEntry& e = h[k];
        std::memset(&e, 0, sizeof(e));
        e.inst = s->slot;
        e.cap = s->h.cap;
        e.chunks = nbody_chunks(e.cap);
        e.rhs_chunk = rhs_chunk_for(e.cap, s->h.np);
        e.rhs_chunks = (int)std::max<uint64_t>(1, (e.cap + e.rhs_chunk - 1) / e.rhs_chunk);
        e.npad = (int)align_up((size_t)s->h.np, 256);
        e.coff = coff;
        e.poff = poff;
        e.roff = roff;
        e.cofs = cofs;
        coff += e.cap;  // caps are multiples of kCapAlign
        if (s->h.precision != kF32)  // the FP32 path sums in fixed point, without partials
            poff += (uint64_t)e.chunks * e.cap;
        roff += (uint64_t)e.rhs_chunks * e.npad;
        cofs += (uint64_t)e.rhs_chunks;
        sl.max_np = std::max(sl.max_np, s->h.np);
    }
    sl.total = coff;
    pl.ws_need_cap = std::max(pl.ws_need_cap, coff);
    pl.part_elems = std::max(pl.part_elems, poff);
    pl.rhs_elems = std::max(pl.rhs_elems, roff);
    pl.circ_elems = std::max(pl.circ_elems, cofs);
    // The plan's lists live in its slot of the context's list pool; the copy is
    // ordered on the stream after every kernel that read the slot before.
    sl.d_list = c->list_pool + (size_t)pl.pool_slot * kPoolPerPlan + pl.pool_used;
    pl.pool_used += sl.n;
    CK(cudaMemcpyAsync(sl.d_list, h.data(), sizeof(ListEntry) * sl.n, cudaMemcpyHostToDevice,
                       c->stream));
    sl.host = h;
    if (f32_pairs) {
        sl.cls = shape_class(sl.total, sl.n);
        sl.cfg = tuned_config(c, sl.cls);
        sl.d_pair_list = sl.d_list;
        if (sl.cfg.order == 1 && sl.n > 1) {
            const std::vector<ListEntry> o = costliest_first(h);
            sl.d_pair_list = c->list_pool + (size_t)pl.pool_slot * kPoolPerPlan + pl.pool_used;
            pl.pool_used += sl.n;
            CK(cudaMemcpyAsync(sl.d_pair_list, o.data(), sizeof(ListEntry) * sl.n,
                               cudaMemcpyHostToDevice, c->stream));
        }
    }
    return DVM_OK;
}

int ensure_workspace(dvm_ctx* c, uint64_t cap, uint64_t part, uint64_t rhs, uint64_t circ,
                     int nlist, bool need_delete) {
    if (cap <= c->ws_cap && part <= c->ws_part && rhs <= c->ws_rhs && circ <= c->ws_circ &&
        (uint64_t)nlist <= c->ws_lists && (!need_delete || c->ws_delete))
        return DVM_OK;
    cap = std::max<uint64_t>({cap, c->ws_cap, kCapAlign});
    part = std::max(part, c->ws_part);
    rhs = std::max(rhs, c->ws_rhs);
    circ = std::max(circ, c->ws_circ);
    const uint64_t lists = std::max<uint64_t>({(uint64_t)nlist, c->ws_lists, 64});
    need_delete = need_delete || c->ws_delete;
    CK(cudaStreamSynchronize(c->stream));
    if (c->ws_block) {
        cudaFree(c->ws_block);
        c->in_use -= c->ws_bytes;
        c->ws_block = nullptr;
    }
    const size_t cub = cub_sort_bytes(cap);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = align_up(off + bytes, 256);
        return o;
    };
    const size_t o_keys_in = take(8 * cap), o_keys_out = take(8 * cap), o_vals = take(4 * cap),
                 o_perm = take(4 * cap), o_packed = take(32 * cap),
                 o_meta = take(sizeof(TileMeta) * (cap / kBsST + 1)), o_part = take(16 * part),
                 o_macc = take(16 * cap), o_mexp = take(sizeof(int) * 4 * kTableCap),
                 o_rhs = take(16 * rhs), o_circ = take(8 * circ + 8), o_cub = take(cub + 256),
                 o_work = take(64 * sizeof(unsigned)), o_flags = take(cap),
                 o_tiles = take(4 * (cap / 1024 + 1)),
                 o_tbase = take(4 * (cap / 1024 + 1)), o_kept = take(4 * 1024),
                 o_ready = take(4 * (cap / 1024 + 1)),
                 o_jobs = take(256 * lists);
    const uint64_t bytes = off;
    if (c->in_use + bytes > c->budget)
        return fail(DVM_ERR_OOM, "workspace of " + std::to_string(bytes) +
                                     " B exceeds the HBM budget");
    void* blk = nullptr;
    CK(cudaMalloc(&blk, bytes));
    c->ws_block = blk;
    c->ws_bytes = bytes;
    c->in_use += bytes;
    char* b = static_cast<char*>(blk);
    Workspace& w = c->ws;
    w.total_cap = cap;
    w.keys_in = reinterpret_cast<uint64_t*>(b + o_keys_in);
    w.keys_out = reinterpret_cast<uint64_t*>(b + o_keys_out);
    w.vals_in = reinterpret_cast<uint32_t*>(b + o_vals);
    w.perm = reinterpret_cast<uint32_t*>(b + o_perm);
    w.packed = reinterpret_cast<double4*>(b + o_packed);
    w.packed_cap = cap;
    w.meta = reinterpret_cast<TileMeta*>(b + o_meta);
    w.part = reinterpret_cast<double2*>(b + o_part);
    w.macc = reinterpret_cast<unsigned long long*>(b + o_macc);
    w.mexp = reinterpret_cast<int*>(b + o_mexp);
    w.rhs_part = reinterpret_cast<double2*>(b + o_rhs);
    w.circ_part = reinterpret_cast<double*>(b + o_circ);
    w.cub_tmp = b + o_cub;
    w.cub_bytes = cub;
    w.work = reinterpret_cast<unsigned*>(b + o_work);
    w.flags = reinterpret_cast<uint8_t*>(b + o_flags);
    w.tile_counts = reinterpret_cast<uint32_t*>(b + o_tiles);
    w.tile_base = reinterpret_cast<uint32_t*>(b + o_tbase);
    w.del_kept = reinterpret_cast<uint32_t*>(b + o_kept);
    w.del_ready = reinterpret_cast<uint32_t*>(b + o_ready);
    w.jobs = b + o_jobs;
    c->ws_cap = cap;
    c->ws_part = part;
    c->ws_rhs = rhs;
    c->ws_circ = circ;
    c->ws_lists = lists;
    c->ws_delete = need_delete;
    c->ws_generation++;
    return DVM_OK;
}

int key_bits_for(int nlist) {
    int b = 1;
    while ((1 << b) < nlist) ++b;
    return 32 + b;
}

// Profiling helpers: an event pair around a kernel family on the ctx stream.
// NVTX range names of the kernel families (DVM_PROF_*), one range per phase
// of every eagerly issued step, for an external timeline profiler.
const char* const kNvtxNames[DVM_PROF_FAMILIES] = {
    "dvm.biot_savart", "dvm.rhs", "dvm.sheet_solve", "dvm.sheet_velocity_convect",
    "dvm.diffuse_release", "dvm.surface_cross", "dvm.loads", "dvm.sort_pack_combine", "dvm.step"};

int prof_begin(dvm_ctx* c, int fam) {
    if (!c->capturing) nvtxRangePushA(kNvtxNames[fam]);
    if (!c->profiling) return -1;
    cudaEvent_t a, b;
    if (c->pool.size() >= 2) {
        a = c->pool.back();
        c->pool.pop_back();
        b = c->pool.back();
        c->pool.pop_back();
    } else {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    cudaEventRecord(a, c->stream);
    c->pending.push_back({fam, a, b});
    return (int)c->pending.size() - 1;
}

void prof_end(dvm_ctx* c, int idx) {
    if (!c->capturing) nvtxRangePop();
    if (idx < 0) return;
    cudaEventRecord(c->pending[idx].b, c->stream);
}

void prof_fold(dvm_ctx* c) {
    if (c->pending.empty()) return;
    cudaStreamSynchronize(c->stream);
    for (auto& r : c->pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
            c->prof_ms[r.fam] += ms;
            c->prof_n[r.fam] += 1;
        }
        c->pool.push_back(r.a);
        c->pool.push_back(r.b);
    }
    c->pending.clear();
}

// Issue one step of every simulation in the plan (no synchronisation).
void issue_step(dvm_ctx* c, Plan& pl) {
    cudaStream_t s = c->stream;
    InstDesc* T = c->d_table;
    InstState* S = c->d_state;
    Workspace ws = c->ws;
    const int sms = c->sms;
    uint64_t L = 0;
    auto on = [&](const SubList& sl) {
        ws.total_cap = sl.total;
        ws.key_bits = key_bits_for(sl.n);
        return ws;
    };
    auto nbody = [&](SubList& sl, int prec) {
        if (!sl.n) return;
        on(sl);
        int p = prof_begin(c, DVM_PROF_SORT);
        biot_savart_prepare(T, S, sl.d_list, sl.n, prec, ws, sms, s);
        prof_end(c, p);
        p = prof_begin(c, DVM_PROF_NBODY);
        if (prec == kF32)
            biot_savart_compute(T, S, sl.d_pair_list, sl.n, prec, ws, sms, s, sl.cfg);
        else
            biot_savart_compute(T, S, sl.d_list, sl.n, prec, ws, sms, s);
        prof_end(c, p);
        p = prof_begin(c, DVM_PROF_SORT);
        biot_savart_finish(T, S, sl.d_list, sl.n, prec, ws, sms, s);
        prof_end(c, p);
        L += 4;  // keys, pack, pair kernel, combine
        p = prof_begin(c, DVM_PROF_RHS);
        sheet_rhs(T, S, sl.d_list, sl.n, sl.max_np, prec, ws, sms, s);
        prof_end(c, p);
        L += 3;
    };
    auto stage = [&](SubList& g, int mode) {
        on(g);
        int p = prof_begin(c, DVM_PROF_SOLVE);
        sheet_solve(T, S, g.d_list, g.n, g.max_np, s);
        prof_end(c, p);
        p = prof_begin(c, DVM_PROF_SHEETVEL);
        sheet_velocity(T, S, g.d_list, g.n, mode, g.max_np, ws, sms, s);
        prof_end(c, p);
        L += 4;
    };
    const int pstep = prof_begin(c, DVM_PROF_STEP);
    int p = prof_begin(c, DVM_PROF_LOADS);
    step_counter(S, pl.all.d_list, pl.all.n, s);
    prof_end(c, p);
    L += 1;
    if (pl.euler.n) {
        nbody(pl.eul_f32, kF32);
        nbody(pl.eul_f64, kF64);
        stage(pl.euler, 1);
    }
    if (pl.rk3.n) {
        for (int st = 0; st < 3; ++st) {
            nbody(pl.rk3_f32, kF32);
            nbody(pl.rk3_f64, kF64);
            stage(pl.rk3, 2 + st);
        }
    }
    on(pl.all);
    p = prof_begin(c, DVM_PROF_DIFFREL);
    diffuse(T, S, pl.all.d_list, pl.all.n, ws, sms, s);
    release(T, S, pl.all.d_list, pl.all.n, pl.all.max_np, s);
    prof_end(c, p);
    L += 2;
    if (pl.refl.n) {
        on(pl.refl);
        p = prof_begin(c, DVM_PROF_CROSS);
        reflect(T, S, pl.refl.d_list, pl.refl.n, pl.refl.max_np, ws, sms, s);
        prof_end(c, p);
        L += 1;
    }
    if (pl.del.n) {
        on(pl.del);
        p = prof_begin(c, DVM_PROF_CROSS);
        delete_inside(T, S, pl.del.d_list, pl.del.n, pl.del.max_np, ws, sms, s);
        prof_end(c, p);
        L += 5;
    }
    p = prof_begin(c, DVM_PROF_LOADS);
    loads(T, S, pl.all.d_list, pl.all.n, pl.all.max_np, s);
    prof_end(c, p);
    prof_end(c, pstep);
    L += 1;
    pl.launches_per_step = L;
}

int get_plan(dvm_ctx* c, const std::vector<int>& slots, Plan** out) {
    auto it = c->plans.find(slots);
    if (it != c->plans.end()) {
        it->second->last_use = ++c->plan_clock;
        *out = it->second;
        return DVM_OK;
    }
    if (c->plans.size() >= kMaxPlans) {  // a serving loop changes its batch often
        auto victim = c->plans.begin();
        for (auto jt = c->plans.begin(); jt != c->plans.end(); ++jt)
            if (jt->second->last_use < victim->second->last_use) victim = jt;
        free_plan(c, victim->second);
        c->plans.erase(victim);
    }
    if (c->pool_free.empty()) return fail(DVM_ERR_STATE, "no free plan slot");
    Plan* pl = new Plan();
    pl->pool_slot = c->pool_free.back();
    c->pool_free.pop_back();
    pl->last_use = ++c->plan_clock;
    pl->slots = slots;
    for (int sl : slots) {
        const dvm_sim* s = c->slots[sl];
        pl->all.slots.push_back(sl);
        const bool rk3 = s->h.scheme == kRK3, f32 = s->h.precision == kF32;
        (rk3 ? pl->rk3 : pl->euler).slots.push_back(sl);
        if (rk3) (f32 ? pl->rk3_f32 : pl->rk3_f64).slots.push_back(sl);
        else (f32 ? pl->eul_f32 : pl->eul_f64).slots.push_back(sl);
        if (s->h.cross == kDelete) {
            pl->del.slots.push_back(sl);
            pl->need_delete = true;
        } else {
            pl->refl.slots.push_back(sl);
        }
    }
    SubList* subs[] = {&pl->all, &pl->euler, &pl->rk3, &pl->rk3_f32, &pl->rk3_f64,
                       &pl->eul_f32, &pl->eul_f64, &pl->refl, &pl->del};
    for (SubList* s : subs) {
        const int rc = build_sublist(c, *s, *pl, s == &pl->rk3_f32 || s == &pl->eul_f32);
        if (rc) {
            free_plan(c, pl);
            return rc;
        }
    }
    c->plans[slots] = pl;
    *out = pl;
    return DVM_OK;
}

int upload_desc(dvm_sim* s) {
    CK(cudaMemcpyAsync(s->ctx->d_table + s->slot, &s->h, sizeof(InstDesc), cudaMemcpyHostToDevice,
                       s->ctx->stream));
    return DVM_OK;
}

int check_device_status(dvm_sim* s) {
    int st = 0;
    CK(cudaMemcpyAsync(&st, &s->ctx->d_state[s->slot].status, sizeof(int), cudaMemcpyDeviceToHost,
                       s->ctx->stream));
    CK(cudaStreamSynchronize(s->ctx->stream));
    return st;
}

int run_steps(dvm_ctx* c, const std::vector<int>& slots, int nsteps, bool use_graph) {
    Plan* pl = nullptr;
    int rc = get_plan(c, slots, &pl);
    if (rc) return rc;
    rc = ensure_workspace(c, pl->ws_need_cap, pl->part_elems, pl->rhs_elems, pl->circ_elems,
                          (int)slots.size(), pl->need_delete);
    if (rc) return rc;
    if (pl->exec && pl->ws_generation != c->ws_generation) {
        cudaGraphExecDestroy(pl->exec);
        cudaGraphDestroy(pl->graph);
        pl->exec = nullptr;
        pl->graph = nullptr;
    }
    if (c->profiling) use_graph = false;  // events are recorded around eager launches
    for (int k = 0; k < nsteps; ++k) {
        if (use_graph && pl->exec) {
            CK(cudaGraphLaunch(pl->exec, c->stream));
            g_launches += pl->launches_per_step;
            continue;
        }
        if (use_graph && pl->warmed) {  // capture only after one eager step of this plan
            CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            c->capturing = true;
            issue_step(c, *pl);
            c->capturing = false;
            cudaGraph_t g = nullptr;
            CK(cudaStreamEndCapture(c->stream, &g));
            cudaGraphExec_t ex = nullptr;
            CK(cudaGraphInstantiate(&ex, g, 0));
            pl->graph = g;
            pl->exec = ex;
            pl->ws_generation = c->ws_generation;
            CK(cudaGraphLaunch(pl->exec, c->stream));
            g_launches += pl->launches_per_step;
            continue;
        }
        issue_step(c, *pl);
        CK(cudaGetLastError());
        pl->warmed = true;
        g_launches += pl->launches_per_step;
    }
    CK(cudaGetLastError());
    return DVM_OK;
}

// Reference panel geometry on the host, in FP64 with the C library's functions
// (src/VortexSheet.cpp:74, 78-102); O(np) once per body.
void host_geometry(dvm_sim* s, const double* xp, const double* zp, int npts) {
    const int np = npts - 1;
    s->xc.resize(np);
    s->zc.resize(np);
    s->ds.resize(np);
    s->theta.resize(np);
    s->enx.resize(np);
    s->enz.resize(np);
    for (int i = 0; i < np; ++i) {
        s->xc[i] = 0.5 * (xp[i] + xp[i + 1]);
        s->zc[i] = 0.5 * (zp[i] + zp[i + 1]);
        const double dx = xp[i + 1] - xp[i];
        const double dz = zp[i + 1] - zp[i];
        s->ds[i] = std::sqrt(std::pow(dx, 2.0) + std::pow(dz, 2.0));
        s->theta[i] = std::atan2(dz, dx);
        s->enx[i] = dz / s->ds[i];
        s->enz[i] = -dx / s->ds[i];
    }
}

// A body contour the panel method can use: finite coordinates, closed (the
// last point repeats the first, the reference's domain_file format,
// src/VortexSheet.cpp:56-76), at least 3 panels, and no panel of zero length
// (ds divides the normals, src/VortexSheet.cpp:93-96, and the influence
// coefficients).  The reference does not check these; an open contour or a
// repeated point silently gives a singular or meaningless system there.
// Returns an empty string when the contour is valid, else the reason.
std::string body_problem(const double* xp, const double* zp, int npts) {
    if (npts < 4) return "a closed body needs at least 3 panels (4 points, the first repeated last)";
    double xmn = xp[0], xmx = xp[0], zmn = zp[0], zmx = zp[0];
    for (int i = 0; i < npts; ++i) {
        if (!std::isfinite(xp[i]) || !std::isfinite(zp[i]))
            return "body point " + std::to_string(i) + " is not finite";
        xmn = std::min(xmn, xp[i]);
        xmx = std::max(xmx, xp[i]);
        zmn = std::min(zmn, zp[i]);
        zmx = std::max(zmx, zp[i]);
    }
    const double L = std::max(xmx - xmn, zmx - zmn);
    if (!(L > 0)) return "body points are all the same";
    const double tol = 1e-12 * L;
    if (std::fabs(xp[npts - 1] - xp[0]) > tol || std::fabs(zp[npts - 1] - zp[0]) > tol)
        return "body contour is not closed: its last point must repeat the first";
    for (int i = 0; i + 1 < npts; ++i)
        if (std::hypot(xp[i + 1] - xp[i], zp[i + 1] - zp[i]) <= tol)
            return "body panel " + std::to_string(i) + " has zero length (repeated point)";
    return std::string();
}

// Serialises calls on one simulation's context (its host-side descriptor and
// stream) and makes its device current, for the per-simulation entry points.
struct SimLock {
    std::lock_guard<std::mutex> lk;
    cudaError_t dev;
    explicit SimLock(dvm_sim* s) : lk(s->ctx->mu), dev(cudaSetDevice(s->ctx->device)) {}
};
#define SIM_LOCK(s)                                                         \
    SimLock sim_lock_(s);                                                   \
    if (sim_lock_.dev != cudaSuccess)                                       \
        return fail(DVM_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(sim_lock_.dev))

// Rejects a list that names one simulation twice (the batched pushes and
// reads would otherwise reuse one offset or one stale cursor for both).
int check_distinct(dvm_ctx* c, dvm_sim* const* sims, int nsims) {
    std::vector<char> seen(kTableCap, 0);
    for (int i = 0; i < nsims; ++i) {
        if (!sims[i] || sims[i]->ctx != c) return fail(DVM_ERR_ARG, "simulation of another ctx");
        if (seen[sims[i]->slot]++) return fail(DVM_ERR_ARG, "a simulation is listed twice");
    }
    return DVM_OK;
}

}  // namespace

// =====================================================================================
extern "C" {

int dvm_abi_version(void) { return DVM_ABI_VERSION; }

const char* dvm_status_string(int status) {
    switch (status) {
        case DVM_OK: return "ok";
        case DVM_ERR_ARG: return "bad argument";
        case DVM_ERR_OOM: return "out of device memory / HBM budget";
        case DVM_ERR_CUDA: return "CUDA error";
        case DVM_ERR_TIMEOUT: return "device wait timed out";
        case DVM_ERR_CAPACITY: return "blob capacity exceeded";
        case DVM_ERR_RELEASE: return "negative PanelNewVort in release";
        case DVM_ERR_STATE: return "invalid state";
        case DVM_ERR_RNG: return "injected random stream exhausted";
        case DVM_ERR_NO_DEVICE: return "no usable CUDA device";
        default: return "unknown status";
    }
}

const char* dvm_last_error(void) { return g_err.c_str(); }

int dvm_ctx_create(int device, uint64_t budget, dvm_ctx** out) {
    if (!out) return fail(DVM_ERR_ARG, "out is null");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(DVM_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(DVM_ERR_ARG, "bad device index");
    CK(cudaSetDevice(device));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return fail(DVM_ERR_NO_DEVICE, "library is built for sm_100a only");
    auto* c = new dvm_ctx();
    c->device = device;
    c->sms = prop.multiProcessorCount;
    c->cc_major = prop.major;
    c->cc_minor = prop.minor;
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    c->budget = budget ? budget : (uint64_t)(0.9 * (double)fr);
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        e = cudaMemPoolCreate(&c->mempool, &props);
        uint64_t keep = UINT64_MAX;  // never release on synchronisation
        if (e == cudaSuccess)
            e = cudaMemPoolSetAttribute(c->mempool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (e == cudaSuccess) e = cudaMalloc(&c->d_table, sizeof(InstDesc) * kTableCap);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_state, sizeof(InstState) * kTableCap);
    if (e == cudaSuccess) e = cudaMemset(c->d_state, 0, sizeof(InstState) * kTableCap);
    if (e == cudaSuccess) e = cudaMalloc(&c->list_pool, sizeof(ListEntry) * kMaxPlans * kPoolPerPlan);
    for (int i = (int)kMaxPlans - 1; i >= 0; --i) c->pool_free.push_back(i);
    if (e != cudaSuccess) {
        dvm_ctx_destroy(c);
        return fail(DVM_ERR_CUDA, std::string("ctx create: ") + cudaGetErrorString(e));
    }
    c->slots.assign(kTableCap, nullptr);
    c->in_use = 2 * sizeof(InstDesc) * kTableCap;
    *out = c;
    return DVM_OK;
}

int dvm_ctx_destroy(dvm_ctx* c) {
    if (!c) return DVM_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (dvm_sim* s : c->slots)
        if (s) {
            pool_free(c, s->slab);
            delete s;
        }
    if (c->stream) cudaStreamSynchronize(c->stream);
    drop_plans_with(c, -1);
    for (auto& r : c->pending) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (cudaEvent_t e : c->pool) cudaEventDestroy(e);
    for (cudaEvent_t e : c->marks)
        if (e) cudaEventDestroy(e);
    if (c->ws_block) cudaFree(c->ws_block);
    if (c->raw_block) cudaFree(c->raw_block);
    if (c->list_pool) cudaFree(c->list_pool);
    if (c->d_tune_list) cudaFree(c->d_tune_list);
    if (c->h_state) cudaFreeHost(c->h_state);
    if (c->copy_stream) {
        cudaStreamSynchronize(c->copy_stream);
        cudaStreamDestroy(c->copy_stream);
    }
    if (c->snap_buf) {
        pool_free(c, c->snap_buf);
        cudaStreamSynchronize(c->stream);
    }
    if (c->push_ev) cudaEventDestroy(c->push_ev);
    if (c->snap_ev) cudaEventDestroy(c->snap_ev);
    if (c->h_state_snap) cudaFreeHost(c->h_state_snap);
    if (c->h_ucount) cudaFreeHost(c->h_ucount);
    if (c->ucount_ev) cudaEventDestroy(c->ucount_ev);
    if (c->d_table) cudaFree(c->d_table);
    if (c->d_state) cudaFree(c->d_state);
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->mempool) cudaMemPoolDestroy(c->mempool);
    delete c;
    return DVM_OK;
}

int dvm_ctx_synchronize(dvm_ctx* c) {
    if (!c) return fail(DVM_ERR_ARG, "ctx is null");
    CK(cudaStreamSynchronize(c->stream));
    return DVM_OK;
}

int dvm_ctx_memory(dvm_ctx* c, uint64_t* in_use, uint64_t* budget) {
    if (!c) return fail(DVM_ERR_ARG, "ctx is null");
    if (in_use) *in_use = c->in_use;
    if (budget) *budget = c->budget;
    return DVM_OK;
}

int dvm_ctx_device_info(dvm_ctx* c, int* sms, int* ma, int* mi) {
    if (!c) return fail(DVM_ERR_ARG, "ctx is null");
    if (sms) *sms = c->sms;
    if (ma) *ma = c->cc_major;
    if (mi) *mi = c->cc_minor;
    return DVM_OK;
}

int dvm_ctx_reserve(dvm_ctx* c, uint64_t total_capacity, int max_sims, int max_panels,
                    int with_delete) {
    if (!c || max_sims < 1 || max_panels < 2) return fail(DVM_ERR_ARG, "bad argument");
    std::lock_guard<std::mutex> lk(c->mu);
    CK(cudaSetDevice(c->device));
    const uint64_t S = (uint64_t)max_sims;
    const uint64_t T = align_up(total_capacity, kCapAlign) + S * kCapAlign;
    // bounds of the per-list sums: chunks*cap <= 16 cap + 2^21; rhs chunks per
    // simulation <= 601 or cap / kAtChunk + 1 (rhs_chunk_for)
    const uint64_t part = 16 * T + S * (2u << 20);
    const uint64_t rchunks = T / kAtChunk + S * 602;
    return ensure_workspace(c, T, part, rchunks * align_up((size_t)max_panels, 256), rchunks,
                            max_sims, with_delete != 0);
}

int dvm_ctx_pool_reserve(dvm_ctx* c, uint64_t bytes) {
    if (!c) return fail(DVM_ERR_ARG, "null context");
    if (bytes == 0) return DVM_OK;
    std::lock_guard<std::mutex> lk(c->mu);
    CK(cudaSetDevice(c->device));
    uint64_t held = 0;
    CK(cudaMemPoolGetAttribute(c->mempool, cudaMemPoolAttrReservedMemCurrent, &held));
    if (held >= bytes) return DVM_OK;
    void* p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, c->mempool, c->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(DVM_ERR_OOM, std::string("pool reserve: ") + cudaGetErrorString(e));
    }
    e = cudaFreeAsync(p, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return fail(DVM_ERR_CUDA, std::string("pool reserve: ") + cudaGetErrorString(e));
    return DVM_OK;
}

int dvm_ctx_workspace_bytes(dvm_ctx* c, uint64_t* bytes) {
    if (!c || !bytes) return fail(DVM_ERR_ARG, "null argument");
    *bytes = c->ws_bytes;
    return DVM_OK;
}

int dvm_ctx_mark(dvm_ctx* c, int slot) {
    if (!c || slot < 0 || slot >= 16) return fail(DVM_ERR_ARG, "bad marker slot");
    if (!c->marks[slot]) CK(cudaEventCreate(&c->marks[slot]));
    CK(cudaEventRecord(c->marks[slot], c->stream));
    return DVM_OK;
}

int dvm_ctx_elapsed(dvm_ctx* c, int a, int b, double* ms) {
    if (!c || !ms || a < 0 || a >= 16 || b < 0 || b >= 16 || !c->marks[a] || !c->marks[b])
        return fail(DVM_ERR_ARG, "bad marker slot");
    CK(cudaEventSynchronize(c->marks[b]));
    float f = 0.f;
    CK(cudaEventElapsedTime(&f, c->marks[a], c->marks[b]));
    *ms = f;
    return DVM_OK;
}

int dvm_ctx_profiler_range(dvm_ctx* c, int on) {
    if (!c) return fail(DVM_ERR_ARG, "ctx is null");
    CK(cudaSetDevice(c->device));
    CK(on ? cudaProfilerStart() : cudaProfilerStop());
    return DVM_OK;
}

int dvm_ctx_set_profiling(dvm_ctx* c, int on) {
    if (!c) return fail(DVM_ERR_ARG, "ctx is null");
    std::lock_guard<std::mutex> lk(c->mu);
    c->profiling = on != 0;
    return DVM_OK;
}

int dvm_ctx_profile(dvm_ctx* c, int fam, double* ms, uint64_t* n) {
    if (!c || fam < 0 || fam >= DVM_PROF_FAMILIES) return fail(DVM_ERR_ARG, "bad argument");
    std::lock_guard<std::mutex> lk(c->mu);
    prof_fold(c);
    if (ms) *ms = c->prof_ms[fam];
    if (n) *n = c->prof_n[fam];
    return DVM_OK;
}

int dvm_ctx_profile_reset(dvm_ctx* c) {
    if (!c) return fail(DVM_ERR_ARG, "ctx is null");
    std::lock_guard<std::mutex> lk(c->mu);
    prof_fold(c);
    for (int f = 0; f < DVM_PROF_FAMILIES; ++f) {
        c->prof_ms[f] = 0.0;
        c->prof_n[f] = 0;
    }
    return DVM_OK;
}

int dvm_ctx_launch_count(dvm_ctx* c, uint64_t* n) {
    if (!c || !n) return fail(DVM_ERR_ARG, "null argument");
    *n = g_launches.load();
    return DVM_OK;
}

// Slab layout of one simulation (doubles unless noted; each array 256-B aligned).
static uint64_t sim_layout(const dvm_sim_params* p, int np, uint64_t cap,
                           std::vector<size_t>* offs) {
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = align_up(off + bytes, 256);
        if (offs) offs->push_back(o);
        return o;
    };
    for (int a = 0; a < 10; ++a) take(8 * cap);  // x z circ sigma u w uvs wvs q1 q2
    take(4 * cap);                               // id
    take(8 * (np + 1));                          // xp
    take(8 * (np + 1));                          // zp
    for (int a = 0; a < 14; ++a) take(8 * np);   // xc zc ds theta enx enz etx etz cth sth c2th s2th psigma gamma
    take(8 * (size_t)(np + 1) * np);             // A
    take(8 * (size_t)(np + 1) * np);             // P
    take(8 * (np + 1));                          // b
    take(8 * (np + 1));                          // res
    take(p->rng == DVM_RNG_INJECT ? 8 * std::max<uint64_t>(p->rng_capacity, 1) : 8);
    return off;
}

int dvm_sim_bytes(const dvm_sim_params* p, int np, uint64_t* bytes) {
    if (!p || !bytes || np < 2) return fail(DVM_ERR_ARG, "bad argument");
    const uint64_t cap = align_up(std::max<uint64_t>(p->capacity, 1), kCapAlign);
    *bytes = sim_layout(p, np, cap, nullptr);
    return DVM_OK;
}

}  // extern "C"

namespace {

// The checks of a simulation's parameters and body, made before anything
// touches a device, so a caller (or a test without a GPU) learns about a bad
// contour from its message.
int check_sim_args(const dvm_sim_params* p, const double* bx, const double* bz, int npts) {
    if (!p || !bx || !bz) return fail(DVM_ERR_ARG, "null argument");
    if (npts < 0) return fail(DVM_ERR_ARG, "negative point count");
    const std::string why = body_problem(bx, bz, npts);
    if (!why.empty()) return fail(DVM_ERR_ARG, why);
    if (!std::isfinite(p->ux) || !std::isfinite(p->uz) || !std::isfinite(p->cutoff_exp) ||
        !std::isfinite(p->dt) || !std::isfinite(p->nu) || !std::isfinite(p->rho))
        return fail(DVM_ERR_ARG, "non-finite parameter");
    if (p->scheme != DVM_EULER && p->scheme != DVM_RK3) return fail(DVM_ERR_ARG, "bad scheme");
    if (p->surface_cross < 0 || p->surface_cross > 2) return fail(DVM_ERR_ARG, "bad surface_cross");
    if (p->precision != DVM_F64 && p->precision != DVM_F32) return fail(DVM_ERR_ARG, "bad precision");
    if (p->rng != DVM_RNG_INJECT && p->rng != DVM_RNG_PHILOX) return fail(DVM_ERR_ARG, "bad rng");
    if (!(p->dt > 0) || !(p->nu > 0) || !(p->rho > 0)) return fail(DVM_ERR_ARG, "dt, nu, density must be > 0");
    if (p->capacity == 0 || p->capacity > 0xF0000000ull) return fail(DVM_ERR_ARG, "bad capacity");
    if (npts - 1 > 2048) return fail(DVM_ERR_ARG, "too many panels (max 2048)");
    return DVM_OK;
}

uint64_t setup_scratch_bytes(int np) {
    return 8 * (2 * (uint64_t)np * np + pseudo_inverse_work_doubles(np));
}

// One simulation's set-up, enqueued on the context's stream up to its
// factorisation: slab, descriptor, host geometry and panel tables, uploads and
// the influence matrix; *scratch receives the factorisation's workspace.
int begin_sim(dvm_ctx* c, int slot, const dvm_sim_params* p, const double* bx, const double* bz,
              int npts, dvm_sim** out, double** scratch) {
    const int np = npts - 1;
    const uint64_t cap = align_up(p->capacity, kCapAlign);
    std::vector<size_t> offs;
    const uint64_t bytes = sim_layout(p, np, cap, &offs);
    const uint64_t qr_bytes = setup_scratch_bytes(np);
    auto* s = new dvm_sim();
    s->ctx = c;
    s->slot = slot;
    s->p = *p;
    s->bytes = bytes;
    cudaError_t e = pool_alloc(c, &s->slab, bytes);
    if (e != cudaSuccess) {
        delete s;
        return fail(DVM_ERR_OOM, std::string("slab allocation: ") + cudaGetErrorString(e));
    }
    char* b = static_cast<char*>(s->slab);
    int a = 0;
    auto nxt = [&]() { return reinterpret_cast<double*>(b + offs[a++]); };
    InstDesc& h = s->h;
    std::memset(&h, 0, sizeof(h));
    h.x = nxt(); h.z = nxt(); h.circ = nxt(); h.sigma = nxt(); h.u = nxt(); h.w = nxt();
    h.uvs = nxt(); h.wvs = nxt(); h.q1 = nxt(); h.q2 = nxt();
    h.id = reinterpret_cast<uint32_t*>(nxt());
    double* xp = nxt();
    double* zp = nxt();
    double* xc = nxt(); double* zc = nxt(); double* ds = nxt(); double* th = nxt();
    double* enx = nxt(); double* enz = nxt(); double* etx = nxt(); double* etz = nxt();
    double* cth = nxt(); double* sth = nxt(); double* c2 = nxt(); double* s2 = nxt();
    double* psig = nxt();
    h.gamma = nxt();
    double* A = nxt();
    double* P = nxt();
    h.b = nxt();
    h.res = nxt();
    s->uniforms = nxt();
    s->ucap = p->rng == DVM_RNG_INJECT ? std::max<uint64_t>(p->rng_capacity, 1) : 0;
    h.xp = xp; h.zp = zp; h.xc = xc; h.zc = zc; h.ds = ds; h.enx = enx; h.enz = enz;
    h.etx = etx; h.etz = etz; h.cth = cth; h.sth = sth; h.c2th = c2; h.s2th = s2; h.psigma = psig;
    h.A = A; h.P = P; h.uniforms = s->uniforms; h.ucount = 0;
    h.rho = p->rho; h.nu = p->nu; h.dt = p->dt; h.ux = p->ux; h.uz = p->uz;
    h.cutoff_exp = p->cutoff_exp;
    h.Ur = std::sqrt(p->ux * p->ux + p->uz * p->uz);  // src/DVMBase.cpp:29
    h.M = p->max_numpanelvort;
    h.np = np;
    h.scheme = p->scheme;
    h.cross = p->surface_cross;
    h.rng = p->rng;
    h.precision = p->precision;
    h.refine = 1;
    h.cap = (uint32_t)cap;
    h.seed = (uint64_t)p->seed;
    h.uid = 0;  // random streams depend on the seed only, never on the table slot
    // host geometry (reference arithmetic) and derived per-panel tables
    host_geometry(s, bx, bz, npts);
    std::vector<double> vetx(np), vetz(np), vcth(np), vsth(np), vc2(np), vs2(np), vps(np);
    for (int i = 0; i < np; ++i) {
        vetx[i] = -s->enz[i];
        vetz[i] = s->enx[i];
        vcth[i] = std::cos(s->theta[i]);
        vsth[i] = std::sin(s->theta[i]);
        vc2[i] = std::cos(-2.0 * s->theta[i]);
        vs2[i] = std::sin(-2.0 * s->theta[i]);
        vps[i] = std::pow(s->ds[i], p->cutoff_exp);  // src/VortexSheet.cpp:325
    }
    double xmx = bx[0], xmn = bx[0], zmx = bz[0], zmn = bz[0];
    for (int i = 1; i < npts; ++i) {
        xmx = std::max(xmx, bx[i]);
        xmn = std::min(xmn, bx[i]);
        zmx = std::max(zmx, bz[i]);
        zmn = std::min(zmn, bz[i]);
    }
    h.area = xmx - xmn;  // src/VortexSheet.cpp:74
    h.bxmax = xmx + 1e-9 * (1.0 + std::fabs(xmx));
    h.bxmin = xmn - 1e-9 * (1.0 + std::fabs(xmn));
    h.bzmin = zmn;
    h.bzmax = zmx;
    const double L = std::max(xmx - xmn, zmx - zmn);
    const double cx = 0.5 * (xmx + xmn), cz = 0.5 * (zmx + zmn);
    h.kx0 = cx - 32.0 * L;
    h.kz0 = cz - 64.0 * L;
    h.kinv = 65536.0 / (128.0 * L);
    auto up = [&](double* d, const double* src, size_t n) {
        return cudaMemcpyAsync(d, src, 8 * n, cudaMemcpyHostToDevice, c->stream);
    };
    e = cudaSuccess;
    if (e == cudaSuccess) e = up(xp, bx, npts);
    if (e == cudaSuccess) e = up(zp, bz, npts);
    if (e == cudaSuccess) e = up(xc, s->xc.data(), np);
    if (e == cudaSuccess) e = up(zc, s->zc.data(), np);
    if (e == cudaSuccess) e = up(ds, s->ds.data(), np);
    if (e == cudaSuccess) e = up(th, s->theta.data(), np);
    if (e == cudaSuccess) e = up(enx, s->enx.data(), np);
    if (e == cudaSuccess) e = up(enz, s->enz.data(), np);
    if (e == cudaSuccess) e = up(etx, vetx.data(), np);
    if (e == cudaSuccess) e = up(etz, vetz.data(), np);
    if (e == cudaSuccess) e = up(cth, vcth.data(), np);
    if (e == cudaSuccess) e = up(sth, vsth.data(), np);
    if (e == cudaSuccess) e = up(c2, vc2.data(), np);
    if (e == cudaSuccess) e = up(s2, vs2.data(), np);
    if (e == cudaSuccess) e = up(psig, vps.data(), np);
    if (e == cudaSuccess) e = cudaMemsetAsync(h.gamma, 0, 8 * np, c->stream);
    if (e == cudaSuccess) e = pool_alloc(c, reinterpret_cast<void**>(scratch), qr_bytes);
    if (e == cudaSuccess) influence_matrix(xp, zp, xc, zc, ds, th, np, *scratch, A, c->stream);
    if (e != cudaSuccess) {
        pool_free(c, *scratch);
        *scratch = nullptr;
        pool_free(c, s->slab);
        delete s;
        return fail(DVM_ERR_CUDA, std::string("sim create: ") + cudaGetErrorString(e));
    }
    *out = s;
    return DVM_OK;
}

// Creates n simulations (all or none).  Their set-up is enqueued body after
// body; the factorisations of the bodies then run together (pseudo_inverse_many:
// up to 8 bodies per cooperative launch, the same arithmetic as alone), and one
// wait covers them all.
int create_sims(dvm_ctx* c, int n, const dvm_sim_params* const* p, const double* const* bx,
                const double* const* bz, const int* npts, dvm_sim** out) {
    for (int i = 0; i < n; ++i) out[i] = nullptr;
    for (int i = 0; i < n; ++i) {
        const int rc = check_sim_args(p[i], bx[i], bz[i], npts[i]);
        if (rc && n > 1) return fail(rc, "simulation " + std::to_string(i) + ": " + g_err);
        if (rc) return rc;
    }
    if (!c) return fail(DVM_ERR_ARG, "ctx is null");
    std::lock_guard<std::mutex> lk(c->mu);
    std::vector<int> slots;
    for (int i = 1; i < kTableCap && (int)slots.size() < n; ++i)  // slot 0: plugin-call scratch
        if (!c->slots[i]) slots.push_back(i);
    if ((int)slots.size() < n) return fail(DVM_ERR_OOM, "simulation table full");
    CK(cudaSetDevice(c->device));
    uint64_t need = 0, bytes0 = 0;
    for (int i = 0; i < n; ++i) {
        const int np = npts[i] - 1;
        const uint64_t cap = align_up(p[i]->capacity, kCapAlign);
        const uint64_t bytes = sim_layout(p[i], np, cap, nullptr);
        if (i == 0) bytes0 = bytes;
        need += bytes + setup_scratch_bytes(np);  // the scratch is freed once set up
    }
    if (c->in_use + need > c->budget)
        return fail(DVM_ERR_OOM, n == 1 ? "simulation of " + std::to_string(bytes0) +
                                              " B does not fit the HBM budget"
                                        : std::to_string(n) + " simulations with their set-up (" +
                                              std::to_string(need) +
                                              " B) do not fit the HBM budget");
    std::vector<dvm_sim*> sims(n, nullptr);
    std::vector<double*> scratch(n, nullptr);
    auto abandon = [&](int rc) {  // nothing of the group is registered
        for (int i = 0; i < n; ++i) {
            pool_free(c, scratch[i]);
            if (sims[i]) {
                pool_free(c, sims[i]->slab);
                delete sims[i];
            }
        }
        return rc;
    };
    for (int i = 0; i < n; ++i) {
        const int rc = begin_sim(c, slots[i], p[i], bx[i], bz[i], npts[i], &sims[i], &scratch[i]);
        if (rc) return abandon(rc);
    }
    // influence matrices are enqueued; the factorisations, once per body
    std::vector<const double*> A(n);
    std::vector<double*> P(n);
    std::vector<int> np(n);
    for (int i = 0; i < n; ++i) {
        A[i] = sims[i]->h.A;
        P[i] = const_cast<double*>(sims[i]->h.P);  // the slab is ours; kernels read it const
        np[i] = sims[i]->h.np;
    }
    int launches = 0;
    cudaError_t e = pseudo_inverse_many(n, A.data(), np.data(), P.data(), scratch.data(),
                                        c->stream, &launches);
    g_launches += 3 * (uint64_t)n + (uint64_t)launches;  // influence matrix 2, load 1 per body
    const cudaError_t e2 = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess) e = e2;
    for (int i = 0; i < n; ++i) {
        pool_free(c, scratch[i]);
        scratch[i] = nullptr;
    }
    InstState st0;
    std::memset(&st0, 0, sizeof(st0));
    for (int i = 0; i < n && e == cudaSuccess; ++i) {
        const int slot = sims[i]->slot;
        e = cudaMemcpyAsync(c->d_state + slot, &st0, sizeof(st0), cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(c->d_table + slot, &sims[i]->h, sizeof(InstDesc),
                                cudaMemcpyHostToDevice, c->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess)
        return abandon(fail(DVM_ERR_CUDA, std::string("sim create: ") + cudaGetErrorString(e)));
    for (int i = 0; i < n; ++i) {
        c->slots[sims[i]->slot] = sims[i];
        c->in_use += sims[i]->bytes;
        out[i] = sims[i];
    }
    return DVM_OK;
}

}  // namespace

extern "C" {

int dvm_sim_create(dvm_ctx* c, const dvm_sim_params* p, const double* bx, const double* bz,
                   int npts, dvm_sim** out) {
    if (!p || !bx || !bz || !out) return fail(DVM_ERR_ARG, "null argument");
    return create_sims(c, 1, &p, &bx, &bz, &npts, out);
}

int dvm_sims_create(dvm_ctx* c, int n, const dvm_sim_params* const* p, const double* const* bx,
                    const double* const* bz, const int* npts, dvm_sim** out) {
    if (n < 0 || (n > 0 && (!p || !bx || !bz || !npts || !out)))
        return fail(DVM_ERR_ARG, "bad argument");
    if (n == 0) return DVM_OK;
    return create_sims(c, n, p, bx, bz, npts, out);
}

int dvm_sim_destroy(dvm_sim* s) {
    if (!s) return DVM_OK;
    dvm_ctx* c = s->ctx;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);  // no graph of this simulation may still run
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);  // nor a copy into it
    drop_plans_with(c, s->slot);
    c->slots[s->slot] = nullptr;
    c->in_use -= s->bytes;
    pool_free(c, s->slab);  // stream-ordered: later work on the stream may reuse it
    delete s;
    return DVM_OK;
}

int dvm_sim_set_blobs(dvm_sim* s, uint64_t n, const double* x, const double* z, const double* circ,
                      const double* sigma) {
    if (!s) return fail(DVM_ERR_ARG, "sim is null");
    if (n > s->h.cap) return fail(DVM_ERR_CAPACITY, "more blobs than the simulation's capacity");
    if (n && (!x || !z || !circ || !sigma)) return fail(DVM_ERR_ARG, "null blob array");
    for (uint64_t i = 0; i < n; ++i)
        if (!std::isfinite(x[i]) || !std::isfinite(z[i]) || !std::isfinite(circ[i]) ||
            !std::isfinite(sigma[i]))
            return fail(DVM_ERR_ARG, "blob " + std::to_string(i) + " has a non-finite value");
    SIM_LOCK(s);
    cudaStream_t st = s->ctx->stream;
    CK(cudaStreamSynchronize(st));
    if (n) {
        CK(cudaMemcpyAsync(s->h.x, x, 8 * n, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(s->h.z, z, 8 * n, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(s->h.circ, circ, 8 * n, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(s->h.sigma, sigma, 8 * n, cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(s->h.u, 0, 8 * n, st));
        CK(cudaMemsetAsync(s->h.w, 0, 8 * n, st));
        CK(cudaMemsetAsync(s->h.uvs, 0, 8 * n, st));
        CK(cudaMemsetAsync(s->h.wvs, 0, 8 * n, st));
        std::vector<uint32_t> ids(n);
        for (uint64_t i = 0; i < n; ++i) ids[i] = (uint32_t)i;
        CK(cudaMemcpyAsync(s->h.id, ids.data(), 4 * n, cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
    }
    const uint32_t n32 = (uint32_t)n;
    CK(cudaMemcpyAsync(&s->ctx->d_state[s->slot].n, &n32, 4, cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    return DVM_OK;
}

}  // extern "C"

namespace {
// Blob count of a simulation (device value); caller holds the sim's lock.
int num_blobs_locked(dvm_sim* s, uint64_t* n) {
    uint32_t v = 0;
    CK(cudaMemcpyAsync(&v, &s->ctx->d_state[s->slot].n, 4, cudaMemcpyDeviceToHost, s->ctx->stream));
    CK(cudaStreamSynchronize(s->ctx->stream));
    *n = v;
    return DVM_OK;
}
}  // namespace

extern "C" {

int dvm_sim_num_blobs(dvm_sim* s, uint64_t* n) {
    if (!s || !n) return fail(DVM_ERR_ARG, "null argument");
    SIM_LOCK(s);
    uint32_t v = 0;
    CK(cudaMemcpyAsync(&v, &s->ctx->d_state[s->slot].n, 4, cudaMemcpyDeviceToHost, s->ctx->stream));
    CK(cudaStreamSynchronize(s->ctx->stream));
    *n = v;
    return DVM_OK;
}

int dvm_sim_num_panels(dvm_sim* s, int* np) {
    if (!s || !np) return fail(DVM_ERR_ARG, "null argument");
    *np = s->h.np;
    return DVM_OK;
}

int dvm_sim_get_blobs(dvm_sim* s, uint64_t cap, uint64_t* n_out, double* x, double* z, double* circ,
                      double* sigma, double* u, double* w, double* uvs, double* wvs, uint32_t* id) {
    if (!s) return fail(DVM_ERR_ARG, "sim is null");
    SIM_LOCK(s);
    uint64_t n = 0;
    int rc = num_blobs_locked(s, &n);
    if (rc) return rc;
    if (n_out) *n_out = n;
    if (n > cap && (x || z || circ || sigma || u || w || uvs || wvs || id))
        return fail(DVM_ERR_ARG, "output capacity smaller than the blob count");
    cudaStream_t st = s->ctx->stream;
    const double* src[] = {s->h.x, s->h.z, s->h.circ, s->h.sigma, s->h.u, s->h.w, s->h.uvs, s->h.wvs};
    double* dst[] = {x, z, circ, sigma, u, w, uvs, wvs};
    for (int a = 0; a < 8; ++a)
        if (dst[a] && n) CK(cudaMemcpyAsync(dst[a], src[a], 8 * n, cudaMemcpyDeviceToHost, st));
    if (id && n) CK(cudaMemcpyAsync(id, s->h.id, 4 * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return DVM_OK;
}

int dvm_sim_get_gamma(dvm_sim* s, double* g) {
    if (!s || !g) return fail(DVM_ERR_ARG, "null argument");
    SIM_LOCK(s);
    CK(cudaMemcpyAsync(g, s->h.gamma, 8 * s->h.np, cudaMemcpyDeviceToHost, s->ctx->stream));
    CK(cudaStreamSynchronize(s->ctx->stream));
    return DVM_OK;
}

int dvm_sim_set_gamma(dvm_sim* s, const double* g) {
    if (!s || !g) return fail(DVM_ERR_ARG, "null argument");
    SIM_LOCK(s);
    CK(cudaMemcpyAsync(s->h.gamma, g, 8 * s->h.np, cudaMemcpyHostToDevice, s->ctx->stream));
    CK(cudaStreamSynchronize(s->ctx->stream));
    return DVM_OK;
}

int dvm_sim_get_rhs(dvm_sim* s, double* b) {
    if (!s || !b) return fail(DVM_ERR_ARG, "null argument");
    SIM_LOCK(s);
    CK(cudaMemcpyAsync(b, s->h.b, 8 * (s->h.np + 1), cudaMemcpyDeviceToHost, s->ctx->stream));
    CK(cudaStreamSynchronize(s->ctx->stream));
    return DVM_OK;
}

int dvm_sim_get_influence(dvm_sim* s, double* A) {
    if (!s || !A) return fail(DVM_ERR_ARG, "null argument");
    SIM_LOCK(s);
    CK(cudaMemcpyAsync(A, s->h.A, 8 * (size_t)(s->h.np + 1) * s->h.np, cudaMemcpyDeviceToHost,
                       s->ctx->stream));
    CK(cudaStreamSynchronize(s->ctx->stream));
    return DVM_OK;
}

int dvm_sim_get_panels(dvm_sim* s, double* xc, double* zc, double* ds, double* theta, double* enx,
                       double* enz) {
    if (!s) return fail(DVM_ERR_ARG, "sim is null");
    const size_t b = 8 * (size_t)s->h.np;
    if (xc) std::memcpy(xc, s->xc.data(), b);
    if (zc) std::memcpy(zc, s->zc.data(), b);
    if (ds) std::memcpy(ds, s->ds.data(), b);
    if (theta) std::memcpy(theta, s->theta.data(), b);
    if (enx) std::memcpy(enx, s->enx.data(), b);
    if (enz) std::memcpy(enz, s->enz.data(), b);
    return DVM_OK;
}

int dvm_sim_get_loads(dvm_sim* s, double* fx, double* fz, double* cd, double* cl) {
    if (!s) return fail(DVM_ERR_ARG, "sim is null");
    SIM_LOCK(s);
    InstState st;
    CK(cudaMemcpyAsync(&st, &s->ctx->d_state[s->slot], sizeof(st), cudaMemcpyDeviceToHost, s->ctx->stream));
    CK(cudaStreamSynchronize(s->ctx->stream));
    if (fx) *fx = st.fx;
    if (fz) *fz = st.fz;
    if (cd) *cd = st.cd;
    if (cl) *cl = st.cl;
    return DVM_OK;
}

int dvm_sim_get_step(dvm_sim* s, uint32_t* step) {
    if (!s || !step) return fail(DVM_ERR_ARG, "null argument");
    SIM_LOCK(s);
    CK(cudaMemcpyAsync(step, &s->ctx->d_state[s->slot].step, 4, cudaMemcpyDeviceToHost, s->ctx->stream));
    CK(cudaStreamSynchronize(s->ctx->stream));
    return DVM_OK;
}

int dvm_sim_clear_uniforms(dvm_sim* s) {
    if (!s) return fail(DVM_ERR_ARG, "sim is null");
    SIM_LOCK(s);
    uint64_t cursor = 0;
    CK(cudaMemcpyAsync(&cursor, &s->ctx->d_state[s->slot].cursor, 8, cudaMemcpyDeviceToHost, s->ctx->stream));
    CK(cudaStreamSynchronize(s->ctx->stream));
    s->consumed_base += cursor;  // what was consumed stays counted
    const uint64_t zero = 0;
    CK(cudaMemcpyAsync(&s->ctx->d_state[s->slot].cursor, &zero, 8, cudaMemcpyHostToDevice, s->ctx->stream));
    s->h.ucount = 0;
    int rc = upload_desc(s);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s->ctx->stream));
    return DVM_OK;
}

int dvm_sim_pending_uniforms(dvm_sim* s, double* out, uint64_t cap, uint64_t* n) {
    if (!s || !n) return fail(DVM_ERR_ARG, "null argument");
    SIM_LOCK(s);
    uint64_t cursor = 0;
    CK(cudaMemcpyAsync(&cursor, &s->ctx->d_state[s->slot].cursor, 8, cudaMemcpyDeviceToHost, s->ctx->stream));
    CK(cudaStreamSynchronize(s->ctx->stream));
    const uint64_t avail = s->h.ucount > cursor ? s->h.ucount - cursor : 0;
    *n = avail;
    if (!out) return DVM_OK;
    if (cap < avail) return fail(DVM_ERR_ARG, "output capacity smaller than the pending count");
    if (avail)
        CK(cudaMemcpyAsync(out, s->uniforms + cursor, 8 * avail, cudaMemcpyDeviceToHost, s->ctx->stream));
    CK(cudaStreamSynchronize(s->ctx->stream));
    return DVM_OK;
}

int dvm_sim_set_step(dvm_sim* s, uint32_t step) {
    if (!s) return fail(DVM_ERR_ARG, "sim is null");
    SIM_LOCK(s);
    CK(cudaMemcpyAsync(&s->ctx->d_state[s->slot].step, &step, 4, cudaMemcpyHostToDevice, s->ctx->stream));
    CK(cudaStreamSynchronize(s->ctx->stream));
    return DVM_OK;
}

int dvm_sim_push_uniforms(dvm_sim* s, const double* u, uint64_t n) {
    if (!s || (n && !u)) return fail(DVM_ERR_ARG, "null argument");
    SIM_LOCK(s);
    if (s->h.rng != kInject) return fail(DVM_ERR_STATE, "simulation is not in inject mode");
    cudaStream_t st = s->ctx->stream;
    if (s->ctx->copy_stream) CK(cudaStreamSynchronize(s->ctx->copy_stream));
    uint64_t cursor = 0;
    CK(cudaMemcpyAsync(&cursor, &s->ctx->d_state[s->slot].cursor, 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    uint64_t count = s->h.ucount;
    if (count + n > s->ucap) {  // drop the consumed prefix
        const uint64_t keep = count - cursor;
        if (keep + n > s->ucap) return fail(DVM_ERR_CAPACITY, "uniform buffer too small");
        if (keep && cursor)
            CK(cudaMemcpyAsync(s->uniforms, s->uniforms + cursor, 8 * keep, cudaMemcpyDeviceToDevice, st));
        s->consumed_base += cursor;
        count = keep;
        const uint64_t zero = 0;
        CK(cudaMemcpyAsync(&s->ctx->d_state[s->slot].cursor, &zero, 8, cudaMemcpyHostToDevice, st));
    }
    if (n) CK(cudaMemcpyAsync(s->uniforms + count, u, 8 * n, cudaMemcpyHostToDevice, st));
    s->h.ucount = count + n;
    int rc = upload_desc(s);
    if (rc) return rc;
    CK(cudaStreamSynchronize(st));
    return DVM_OK;
}

int dvm_sim_rng_position(dvm_sim* s, uint64_t* consumed, uint64_t* avail) {
    if (!s) return fail(DVM_ERR_ARG, "sim is null");
    SIM_LOCK(s);
    uint64_t cursor = 0;
    CK(cudaMemcpyAsync(&cursor, &s->ctx->d_state[s->slot].cursor, 8, cudaMemcpyDeviceToHost, s->ctx->stream));
    CK(cudaStreamSynchronize(s->ctx->stream));
    if (consumed) *consumed = s->consumed_base + cursor;
    if (avail) *avail = s->h.ucount - cursor;
    return DVM_OK;
}

// ---- state save / restore ---------------------------------------------------------
}  // extern "C"

namespace {

// Layout of a saved simulation state (native byte order): the header, then
// the contour (xp, zp: np+1 each), the eight blob arrays (n each), the IDs (n
// uint32, padded to 8 bytes), gamma (np), A ((np+1) x np), P (np x (np+1)) and
// the injected uniforms not yet consumed.
constexpr char kStateMagic[8] = {'D', 'V', 'M', 'S', 'T', 'A', 'T', 'E'};
constexpr uint32_t kStateVersion = 1;
struct StateHeader {
    char magic[8];
    uint32_t version;
    uint32_t header_bytes;
    dvm_sim_params p;
    int32_t np;
    uint32_t n;
    uint32_t step;
    int32_t status;
    uint64_t consumed_total;  // uniforms consumed since creation (inject mode)
    uint64_t pending;         // uniforms pushed and not yet consumed
    double fx, fz, cd, cl, totalcirc;
    uint64_t reserved[4];
};

uint64_t state_bytes(int np, uint64_t n, uint64_t pending) {
    const uint64_t m = (uint64_t)np;
    return sizeof(StateHeader) + 8 * (2 * (m + 1)) + 8 * 8 * n + 8 * ((n + 1) / 2) + 8 * m +
           16 * (m + 1) * m + 8 * pending;
}

}  // namespace

extern "C" {

int dvm_sim_state_size(dvm_sim* s, uint64_t* bytes) {
    if (!s || !bytes) return fail(DVM_ERR_ARG, "null argument");
    SIM_LOCK(s);
    InstState st;
    CK(cudaMemcpyAsync(&st, &s->ctx->d_state[s->slot], sizeof(st), cudaMemcpyDeviceToHost, s->ctx->stream));
    CK(cudaStreamSynchronize(s->ctx->stream));
    const uint64_t pending = s->h.ucount > st.cursor ? s->h.ucount - st.cursor : 0;
    *bytes = state_bytes(s->h.np, st.n, pending);
    return DVM_OK;
}

int dvm_sim_save(dvm_sim* s, void* buf, uint64_t cap, uint64_t* written) {
    if (!s || !buf) return fail(DVM_ERR_ARG, "null argument");
    SIM_LOCK(s);
    cudaStream_t str = s->ctx->stream;
    if (s->ctx->copy_stream) CK(cudaStreamSynchronize(s->ctx->copy_stream));
    InstState st;
    CK(cudaMemcpyAsync(&st, &s->ctx->d_state[s->slot], sizeof(st), cudaMemcpyDeviceToHost, str));
    CK(cudaStreamSynchronize(str));
    const int np = s->h.np;
    const uint64_t n = st.n;
    const uint64_t pending = s->h.ucount > st.cursor ? s->h.ucount - st.cursor : 0;
    const uint64_t need = state_bytes(np, n, pending);
    if (written) *written = need;
    if (cap < need) return fail(DVM_ERR_ARG, "buffer smaller than dvm_sim_state_size");
    StateHeader H;
    std::memset(&H, 0, sizeof(H));
    std::memcpy(H.magic, kStateMagic, 8);
    H.version = kStateVersion;
    H.header_bytes = sizeof(StateHeader);
    H.p = s->p;
    H.np = np;
    H.n = st.n;
    H.step = st.step;
    H.status = st.status;
    H.consumed_total = s->consumed_base + st.cursor;
    H.pending = pending;
    H.fx = st.fx;
    H.fz = st.fz;
    H.cd = st.cd;
    H.cl = st.cl;
    H.totalcirc = st.totalcirc;
    char* o = static_cast<char*>(buf);
    std::memcpy(o, &H, sizeof(H));
    o += sizeof(H);
    auto down = [&](const void* src, uint64_t nbytes) -> cudaError_t {
        const cudaError_t e = nbytes ? cudaMemcpyAsync(o, src, nbytes, cudaMemcpyDeviceToHost, str)
                                     : cudaSuccess;
        o += nbytes;
        return e;
    };
    const InstDesc& h = s->h;
    CK(down(h.xp, 8 * (np + 1)));
    CK(down(h.zp, 8 * (np + 1)));
    const double* arrs[8] = {h.x, h.z, h.circ, h.sigma, h.u, h.w, h.uvs, h.wvs};
    for (const double* a : arrs) CK(down(a, 8 * n));
    CK(down(h.id, 4 * n));
    if (n & 1) {
        std::memset(o, 0, 4);
        o += 4;
    }
    CK(down(h.gamma, 8 * np));
    CK(down(h.A, 8 * (uint64_t)(np + 1) * np));
    CK(down(h.P, 8 * (uint64_t)(np + 1) * np));
    CK(down(s->uniforms + st.cursor, 8 * pending));
    CK(cudaStreamSynchronize(str));
    return DVM_OK;
}

int dvm_sim_restore(dvm_ctx* c, const void* buf, uint64_t size, dvm_sim** out) {
    if (!c || !buf || !out) return fail(DVM_ERR_ARG, "null argument");
    *out = nullptr;
    if (size < sizeof(StateHeader)) return fail(DVM_ERR_ARG, "not a saved simulation state (too short)");
    StateHeader H;
    std::memcpy(&H, buf, sizeof(H));
    if (std::memcmp(H.magic, kStateMagic, 8) != 0 || H.header_bytes != sizeof(StateHeader))
        return fail(DVM_ERR_ARG, "not a saved simulation state");
    if (H.version != kStateVersion) return fail(DVM_ERR_ARG, "unsupported saved-state version");
    if (H.np < 3 || H.np > 2048 || H.n > H.p.capacity)
        return fail(DVM_ERR_ARG, "corrupt saved state (sizes)");
    if (size != state_bytes(H.np, H.n, H.pending))
        return fail(DVM_ERR_ARG, "saved state has the wrong size");
    if (H.p.rng == DVM_RNG_INJECT && H.pending > std::max<uint64_t>(H.p.rng_capacity, 1))
        return fail(DVM_ERR_ARG, "corrupt saved state (uniforms)");
    const int np = H.np;
    const uint64_t n = H.n;
    const char* q = static_cast<const char*>(buf) + sizeof(H);
    const double* xp = reinterpret_cast<const double*>(q);
    const double* zp = xp + (np + 1);
    dvm_sim* s = nullptr;
    int rc = dvm_sim_create(c, &H.p, xp, zp, np + 1, &s);
    if (rc) return rc;
    q += 16 * (uint64_t)(np + 1);
    {
        SimLock lk(s);
        cudaStream_t str = c->stream;
        cudaError_t e = lk.dev;
        auto up = [&](void* dst, uint64_t nbytes) {
            if (e == cudaSuccess && nbytes)
                e = cudaMemcpyAsync(dst, q, nbytes, cudaMemcpyHostToDevice, str);
            q += nbytes;
        };
        InstDesc& h = s->h;
        double* arrs[8] = {h.x, h.z, h.circ, h.sigma, h.u, h.w, h.uvs, h.wvs};
        for (double* a : arrs) up(a, 8 * n);
        up(h.id, 4 * n);
        if (n & 1) q += 4;
        up(h.gamma, 8 * np);
        up(const_cast<double*>(h.A), 8 * (uint64_t)(np + 1) * np);
        up(const_cast<double*>(h.P), 8 * (uint64_t)(np + 1) * np);
        up(s->uniforms, 8 * H.pending);
        InstState st;
        std::memset(&st, 0, sizeof(st));
        st.n = H.n;
        st.step = H.step;
        st.cursor = 0;
        st.status = H.status;
        st.fx = H.fx;
        st.fz = H.fz;
        st.cd = H.cd;
        st.cl = H.cl;
        st.totalcirc = H.totalcirc;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&c->d_state[s->slot], &st, sizeof(st), cudaMemcpyHostToDevice, str);
        h.ucount = H.p.rng == DVM_RNG_INJECT ? H.pending : 0;
        s->consumed_base = H.consumed_total;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(c->d_table + s->slot, &h, sizeof(h), cudaMemcpyHostToDevice, str);
        if (e == cudaSuccess) e = cudaStreamSynchronize(str);
        if (e != cudaSuccess) rc = fail(DVM_ERR_CUDA, std::string("restore: ") + cudaGetErrorString(e));
    }
    if (rc) {
        dvm_sim_destroy(s);
        return rc;
    }
    *out = s;
    return DVM_OK;
}

// The listed simulations' InstState rows into c->h_state: one copy, one wait.
// Call with c->mu held.
static int read_states(dvm_ctx* c, dvm_sim* const* sims, int nsims) {
    int hi = 0;
    for (int i = 0; i < nsims; ++i) {
        if (!sims[i] || sims[i]->ctx != c) return fail(DVM_ERR_ARG, "simulation of another ctx");
        hi = std::max(hi, sims[i]->slot + 1);
    }
    if (c->h_state_slots < hi) {
        if (c->h_state) cudaFreeHost(c->h_state);
        c->h_state = nullptr;
        c->h_state_slots = 0;
        CK(cudaMallocHost(&c->h_state, sizeof(InstState) * (size_t)kTableCap));
        c->h_state_slots = kTableCap;
    }
    CK(cudaMemcpyAsync(c->h_state, c->d_state, sizeof(InstState) * (size_t)hi,
                       cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DVM_OK;
}

int dvm_batch_status(dvm_ctx* c, dvm_sim* const* sims, int nsims, int32_t* status) {
    if (!c || nsims < 0 || (nsims && (!sims || !status))) return fail(DVM_ERR_ARG, "bad argument");
    if (nsims == 0) return DVM_OK;
    std::lock_guard<std::mutex> lk(c->mu);
    CK(cudaSetDevice(c->device));
    const int rc = read_states(c, sims, nsims);
    if (rc) return rc;
    for (int i = 0; i < nsims; ++i) {
        const int st = c->h_state[sims[i]->slot].status;
        status[i] = st == 0 ? DVM_OK
                  : st == kErrCapacity ? DVM_ERR_CAPACITY
                  : st == kErrRelease ? DVM_ERR_RELEASE
                  : st == kErrRngExhausted ? DVM_ERR_RNG : st;
    }
    return DVM_OK;
}

int dvm_batch_get_state(dvm_ctx* c, dvm_sim* const* sims, int nsims, double* const* x,
                        double* const* z, double* const* circ, const uint64_t* caps,
                        uint64_t* counts, double* loads) {
    if (!c || nsims < 0 || (nsims && (!sims || !counts))) return fail(DVM_ERR_ARG, "bad argument");
    if (nsims == 0) return DVM_OK;
    std::lock_guard<std::mutex> lk(c->mu);
    CK(cudaSetDevice(c->device));
    int rc = read_states(c, sims, nsims);
    if (rc) return rc;
    for (int i = 0; i < nsims; ++i) {
        const InstState& S = c->h_state[sims[i]->slot];
        const uint64_t n = S.n;
        counts[i] = n;
        if (loads) {
            loads[4 * i] = S.fx;
            loads[4 * i + 1] = S.fz;
            loads[4 * i + 2] = S.cd;
            loads[4 * i + 3] = S.cl;
        }
        const bool any = (x && x[i]) || (z && z[i]) || (circ && circ[i]);
        if (!any || n == 0) continue;
        if (!caps || n > caps[i])
            return fail(DVM_ERR_ARG, "output capacity smaller than the blob count");
        const InstDesc& h = sims[i]->h;
        if (x && x[i]) CK(cudaMemcpyAsync(x[i], h.x, 8 * n, cudaMemcpyDeviceToHost, c->stream));
        if (z && z[i]) CK(cudaMemcpyAsync(z[i], h.z, 8 * n, cudaMemcpyDeviceToHost, c->stream));
        if (circ && circ[i])
            CK(cudaMemcpyAsync(circ[i], h.circ, 8 * n, cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    return DVM_OK;
}

int dvm_batch_push_uniforms(dvm_ctx* c, dvm_sim* const* sims, int nsims, const double* const* u,
                            const uint64_t* counts) {
    if (!c || nsims < 0 || (nsims && (!sims || !u || !counts)))
        return fail(DVM_ERR_ARG, "bad argument");
    if (nsims == 0) return DVM_OK;
    std::lock_guard<std::mutex> lk(c->mu);
    CK(cudaSetDevice(c->device));
    int rc = check_distinct(c, sims, nsims);
    if (rc) return rc;
    if (c->copy_stream) CK(cudaStreamSynchronize(c->copy_stream));  // compaction moves data
    rc = read_states(c, sims, nsims);
    if (rc) return rc;
    const uint64_t zero = 0;
    for (int i = 0; i < nsims; ++i) {
        dvm_sim* s = sims[i];
        const uint64_t n = counts[i];
        if (s->h.rng != kInject) return fail(DVM_ERR_STATE, "simulation is not in inject mode");
        if (n && !u[i]) return fail(DVM_ERR_ARG, "null uniform array");
        const uint64_t cursor = c->h_state[s->slot].cursor;
        uint64_t count = s->h.ucount;
        if (count + n > s->ucap) {  // drop the consumed prefix (as dvm_sim_push_uniforms)
            const uint64_t keep = count - cursor;
            if (keep + n > s->ucap) return fail(DVM_ERR_CAPACITY, "uniform buffer too small");
            if (keep && cursor)
                CK(cudaMemcpyAsync(s->uniforms, s->uniforms + cursor, 8 * keep,
                                   cudaMemcpyDeviceToDevice, c->stream));
            s->consumed_base += cursor;
            count = keep;
            CK(cudaMemcpyAsync(&c->d_state[s->slot].cursor, &zero, 8, cudaMemcpyHostToDevice,
                               c->stream));
        }
        if (n)
            CK(cudaMemcpyAsync(s->uniforms + count, u[i], 8 * n, cudaMemcpyHostToDevice,
                               c->stream));
        s->h.ucount = count + n;
        rc = upload_desc(s);
        if (rc) return rc;
    }
    CK(cudaStreamSynchronize(c->stream));
    return DVM_OK;
}

namespace {
int ensure_async(dvm_ctx* c) {
    if (c->copy_stream) return DVM_OK;
    CK(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->push_ev, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->snap_ev, cudaEventDisableTiming));
    CK(cudaMallocHost(&c->h_state_snap, sizeof(InstState) * (size_t)kTableCap));
    CK(cudaMallocHost(&c->h_ucount, sizeof(uint64_t) * (size_t)kTableCap));
    CK(cudaEventCreateWithFlags(&c->ucount_ev, cudaEventDisableTiming));
    CK(cudaEventRecord(c->ucount_ev, c->stream));
    return DVM_OK;
}
}  // namespace

int dvm_batch_push_uniforms_async(dvm_ctx* c, dvm_sim* const* sims, int nsims,
                                  const double* const* u, const uint64_t* counts) {
    if (!c || nsims < 0 || (nsims && (!sims || !u || !counts)))
        return fail(DVM_ERR_ARG, "bad argument");
    if (nsims == 0) return DVM_OK;
    std::lock_guard<std::mutex> lk(c->mu);
    CK(cudaSetDevice(c->device));
    int rc = check_distinct(c, sims, nsims);
    if (rc) return rc;
    for (int i = 0; i < nsims; ++i) {  // check everything before copying anything
        dvm_sim* s = sims[i];
        if (!s || s->ctx != c) return fail(DVM_ERR_ARG, "simulation of another ctx");
        if (s->h.rng != kInject) return fail(DVM_ERR_STATE, "simulation is not in inject mode");
        if (counts[i] && !u[i]) return fail(DVM_ERR_ARG, "null uniform array");
        if (s->h.ucount + counts[i] > s->ucap)
            return fail(DVM_ERR_CAPACITY,
                        "uniform buffer too small for an asynchronous push (it does not compact)");
    }
    rc = ensure_async(c);
    if (rc) return rc;
    // The copies land beyond every uniform the device may read until the
    // descriptors below raise the count, so they can overlap a running step.
    for (int i = 0; i < nsims; ++i) {
        dvm_sim* s = sims[i];
        if (counts[i])
            CK(cudaMemcpyAsync(s->uniforms + s->h.ucount, u[i], 8 * counts[i],
                               cudaMemcpyHostToDevice, c->copy_stream));
    }
    CK(cudaEventRecord(c->push_ev, c->copy_stream));
    CK(cudaStreamWaitEvent(c->stream, c->push_ev, 0));
    // Only the descriptors' uniform counts change; they go up from pinned
    // staging, so nothing here waits for the running step (a copy from pageable
    // memory could).  The staging is rewritten only after its previous upload.
    CK(cudaEventSynchronize(c->ucount_ev));
    for (int i = 0; i < nsims; ++i) {
        dvm_sim* s = sims[i];
        s->h.ucount += counts[i];
        c->h_ucount[s->slot] = s->h.ucount;
        CK(cudaMemcpyAsync(&c->d_table[s->slot].ucount, &c->h_ucount[s->slot], sizeof(uint64_t),
                           cudaMemcpyHostToDevice, c->stream));
    }
    CK(cudaEventRecord(c->ucount_ev, c->stream));
    return DVM_OK;
}

int dvm_batch_get_state_async(dvm_ctx* c, dvm_sim* const* sims, int nsims) {
    if (!c || nsims < 0 || (nsims && !sims)) return fail(DVM_ERR_ARG, "bad argument");
    std::lock_guard<std::mutex> lk(c->mu);
    CK(cudaSetDevice(c->device));
    if (c->snap_pending)
        return fail(DVM_ERR_STATE, "a snapshot is pending: call dvm_batch_wait_state first");
    int hi = 0;
    uint64_t need = 0;
    for (int i = 0; i < nsims; ++i) {
        if (!sims[i] || sims[i]->ctx != c) return fail(DVM_ERR_ARG, "simulation of another ctx");
        hi = std::max(hi, sims[i]->slot + 1);
        need += 3 * (uint64_t)sims[i]->h.cap;
    }
    int rc = ensure_async(c);
    if (rc) return rc;
    if (need > c->snap_doubles) {  // grow (stream-ordered on the compute stream)
        CK(cudaStreamSynchronize(c->copy_stream));  // no copy-out may still read the old one
        if (c->snap_buf) pool_free(c, c->snap_buf);
        c->snap_buf = nullptr;
        c->snap_doubles = 0;
        void* p = nullptr;
        const cudaError_t e = pool_alloc(c, &p, 8 * need);
        if (e != cudaSuccess) return fail(DVM_ERR_OOM, std::string("snapshot: ") + cudaGetErrorString(e));
        c->snap_buf = static_cast<double*>(p);
        c->snap_doubles = need;
    }
    c->snap_slots.assign(nsims, 0);
    c->snap_off.assign(nsims, 0);
    c->snap_cap.assign(nsims, 0);
    uint64_t off = 0;
    for (int i = 0; i < nsims; ++i) {
        const InstDesc& h = sims[i]->h;
        const uint64_t cap = h.cap;
        c->snap_slots[i] = sims[i]->slot;
        c->snap_off[i] = off;
        c->snap_cap[i] = cap;
        CK(cudaMemcpyAsync(c->snap_buf + off, h.x, 8 * cap, cudaMemcpyDeviceToDevice, c->stream));
        CK(cudaMemcpyAsync(c->snap_buf + off + cap, h.z, 8 * cap, cudaMemcpyDeviceToDevice,
                           c->stream));
        CK(cudaMemcpyAsync(c->snap_buf + off + 2 * cap, h.circ, 8 * cap,
                           cudaMemcpyDeviceToDevice, c->stream));
        off += 3 * cap;
    }
    if (hi)
        CK(cudaMemcpyAsync(c->h_state_snap, c->d_state, sizeof(InstState) * (size_t)hi,
                           cudaMemcpyDeviceToHost, c->stream));
    CK(cudaEventRecord(c->snap_ev, c->stream));
    c->snap_pending = true;
    return DVM_OK;
}

int dvm_batch_wait_state(dvm_ctx* c, int nsims, double* const* x, double* const* z,
                         double* const* circ, const uint64_t* caps, uint64_t* counts,
                         double* loads) {
    if (!c || nsims < 0 || (nsims && !counts)) return fail(DVM_ERR_ARG, "bad argument");
    std::lock_guard<std::mutex> lk(c->mu);
    CK(cudaSetDevice(c->device));
    if (!c->snap_pending) return fail(DVM_ERR_STATE, "no snapshot is pending");
    if ((size_t)nsims != c->snap_slots.size())
        return fail(DVM_ERR_ARG, "nsims differs from the pending snapshot's");
    c->snap_pending = false;
    CK(cudaEventSynchronize(c->snap_ev));
    for (int i = 0; i < nsims; ++i) {  // counts and loads; sizes checked before any copy
        const InstState& S = c->h_state_snap[c->snap_slots[i]];
        counts[i] = S.n;
        if (loads) {
            loads[4 * i] = S.fx;
            loads[4 * i + 1] = S.fz;
            loads[4 * i + 2] = S.cd;
            loads[4 * i + 3] = S.cl;
        }
        const bool any = (x && x[i]) || (z && z[i]) || (circ && circ[i]);
        if (any && S.n && (!caps || S.n > caps[i] || S.n > c->snap_cap[i]))
            return fail(DVM_ERR_ARG, "output capacity smaller than the blob count");
    }
    for (int i = 0; i < nsims; ++i) {
        const uint64_t n = counts[i];
        if (n == 0) continue;
        const double* b = c->snap_buf + c->snap_off[i];
        const uint64_t cap = c->snap_cap[i];
        if (x && x[i]) CK(cudaMemcpyAsync(x[i], b, 8 * n, cudaMemcpyDeviceToHost, c->copy_stream));
        if (z && z[i])
            CK(cudaMemcpyAsync(z[i], b + cap, 8 * n, cudaMemcpyDeviceToHost, c->copy_stream));
        if (circ && circ[i])
            CK(cudaMemcpyAsync(circ[i], b + 2 * cap, 8 * n, cudaMemcpyDeviceToHost,
                               c->copy_stream));
    }
    CK(cudaStreamSynchronize(c->copy_stream));
    return DVM_OK;
}

int dvm_sim_status(dvm_sim* s) {
    if (!s) return fail(DVM_ERR_ARG, "sim is null");
    SIM_LOCK(s);
    const int st = check_device_status(s);
    if (st < 0) return st;
    switch (st) {
        case 0: return DVM_OK;
        case kErrCapacity: return fail(DVM_ERR_CAPACITY, "release exceeded the blob capacity");
        case kErrRelease:
            return fail(DVM_ERR_RELEASE,
                        "VortexSheet::release_nascent_vortices_rw: negative PanelNewVort");
        case kErrRngExhausted: return fail(DVM_ERR_RNG, "injected uniform stream exhausted");
        case kErrTimeout:
            return fail(DVM_ERR_TIMEOUT,
                        "a bounded device wait ran out; the simulation's blobs are not consistent");
        default: return fail(st, "device status " + std::to_string(st));
    }
}

int dvm_sim_clear_status(dvm_sim* s) {
    if (!s) return fail(DVM_ERR_ARG, "sim is null");
    SIM_LOCK(s);
    const int z = 0;
    CK(cudaMemcpyAsync(&s->ctx->d_state[s->slot].status, &z, 4, cudaMemcpyHostToDevice, s->ctx->stream));
    CK(cudaStreamSynchronize(s->ctx->stream));
    return DVM_OK;
}

int dvm_sim_phase(dvm_sim* s, int phase) {
    if (!s) return fail(DVM_ERR_ARG, "sim is null");
    dvm_ctx* c = s->ctx;
    std::lock_guard<std::mutex> lk(c->mu);
    CK(cudaSetDevice(c->device));
    std::vector<int> one{s->slot};
    Plan* pl = nullptr;
    int rc = get_plan(c, one, &pl);
    if (rc) return rc;
    rc = ensure_workspace(c, pl->ws_need_cap, pl->part_elems, pl->rhs_elems, pl->circ_elems, 1,
                          pl->need_delete || phase == DVM_PHASE_DELETE);
    if (rc) return rc;
    InstDesc* T = c->d_table;
    InstState* S = c->d_state;
    Workspace ws = c->ws;
    ws.key_bits = key_bits_for(1);
    ws.total_cap = pl->all.total;
    cudaStream_t st = c->stream;
    const ListEntry* L = pl->all.d_list;
    const int np = s->h.np, prec = s->h.precision;
    switch (phase) {
        case DVM_PHASE_BIOTSAVART: {
            int pr = prof_begin(c, DVM_PROF_SORT);
            biot_savart_prepare(T, S, L, 1, prec, ws, c->sms, st);
            prof_end(c, pr);
            pr = prof_begin(c, DVM_PROF_NBODY);
            biot_savart_compute(T, S, L, 1, prec, ws, c->sms, st,
                                tuned_config(c, shape_class(s->h.cap, 1)));
            prof_end(c, pr);
            pr = prof_begin(c, DVM_PROF_SORT);
            biot_savart_finish(T, S, L, 1, prec, ws, c->sms, st);
            prof_end(c, pr);
            break;
        }
        case DVM_PHASE_SOLVE:
            sheet_rhs(T, S, L, 1, np, prec, ws, c->sms, st);
            sheet_solve(T, S, L, 1, np, st);
            break;
        case DVM_PHASE_SHEETBC: sheet_velocity(T, S, L, 1, 0, np, ws, c->sms, st); break;
        case DVM_PHASE_CONVECT:
            for (int k = 0; k < (s->h.scheme == kRK3 ? 3 : 1); ++k) {
                biot_savart_self(T, S, L, 1, prec, ws, c->sms, st,
                                 tuned_config(c, shape_class(s->h.cap, 1)));
                sheet_rhs(T, S, L, 1, np, prec, ws, c->sms, st);
                sheet_solve(T, S, L, 1, np, st);
                sheet_velocity(T, S, L, 1, s->h.scheme == kRK3 ? 2 + k : 1, np, ws, c->sms, st);
            }
            break;
        case DVM_PHASE_DIFFUSE: diffuse(T, S, L, 1, ws, c->sms, st); break;
        case DVM_PHASE_RELEASE: release(T, S, L, 1, np, st); break;
        case DVM_PHASE_CROSS:
            if (s->h.cross == kDelete) delete_inside(T, S, L, 1, np, ws, c->sms, st);
            else reflect(T, S, L, 1, np, ws, c->sms, st);
            break;
        case DVM_PHASE_LOADS: loads(T, S, L, 1, np, st); break;
        case DVM_PHASE_INCREMENT: step_counter(S, L, 1, st); break;
        case DVM_PHASE_REFLECT: reflect(T, S, L, 1, np, ws, c->sms, st); break;
        case DVM_PHASE_DELETE: delete_inside(T, S, L, 1, np, ws, c->sms, st); break;
        default: return fail(DVM_ERR_ARG, "bad phase");
    }
    g_launches += 1;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    return DVM_OK;
}

int dvm_sim_step(dvm_sim* s, int nsteps) {
    if (!s) return fail(DVM_ERR_ARG, "sim is null");
    dvm_sim* one[1] = {s};
    return dvm_step_batch(s->ctx, one, 1, nsteps, 0);
}

int dvm_step_batch(dvm_ctx* c, dvm_sim* const* sims, int nsims, int nsteps, int use_graph) {
    if (!c || (nsims && !sims) || nsims < 0 || nsteps < 0) return fail(DVM_ERR_ARG, "bad argument");
    if (nsims == 0 || nsteps == 0) return DVM_OK;
    if (nsims > dvmk::kMaxBatch) return fail(DVM_ERR_ARG, "at most 1024 simulations per batch");
    std::lock_guard<std::mutex> lk(c->mu);
    CK(cudaSetDevice(c->device));
    std::vector<int> slots(nsims);
    for (int i = 0; i < nsims; ++i) {
        if (!sims[i] || sims[i]->ctx != c) return fail(DVM_ERR_ARG, "simulation of another ctx");
        slots[i] = sims[i]->slot;
    }
    return run_steps(c, slots, nsteps, use_graph != 0);
}

// ---- pair-kernel autotuning ------------------------------------------------------------
namespace {
const dvm_pair_config kCandidates[] = {
    {256, 4, 0, 0}, {256, 3, 0, 0}, {256, 2, 0, 0}, {256, 4, 1, 0}, {256, 3, 1, 0},
    {256, 2, 1, 0}};
constexpr int kNumCandidates = (int)(sizeof(kCandidates) / sizeof(kCandidates[0]));
static_assert(kNumCandidates <= DVM_TUNE_MAX_CANDIDATES, "candidate table too long");

PairConfig to_internal(const dvm_pair_config& p) {
    PairConfig c;
    c.tile = p.tile;
    c.ctas = p.ctas_per_sm;
    c.order = p.order;
    return c;
}
dvm_pair_config to_abi(const PairConfig& c) { return dvm_pair_config{c.tile, c.ctas, c.order, 0}; }

int f32_members(dvm_ctx* c, dvm_sim* const* sims, int nsims, std::vector<int>& slots,
                uint64_t& total_cap) {
    slots.clear();
    total_cap = 0;
    for (int i = 0; i < nsims; ++i) {
        if (!sims[i] || sims[i]->ctx != c) return fail(DVM_ERR_ARG, "simulation of another ctx");
        if (sims[i]->h.precision != kF32) continue;
        if (std::find(slots.begin(), slots.end(), sims[i]->slot) != slots.end())
            return fail(DVM_ERR_ARG, "simulation listed twice");
        slots.push_back(sims[i]->slot);
        total_cap += sims[i]->h.cap;
    }
    return DVM_OK;
}
}  // namespace

int dvm_tune_candidate(int index, dvm_pair_config* out) {
    if (!out || index < 0 || index >= kNumCandidates) return fail(DVM_ERR_ARG, "no such candidate");
    *out = kCandidates[index];
    return DVM_OK;
}

int dvm_batch_shape_class(dvm_ctx* c, dvm_sim* const* sims, int nsims, int* cls) {
    if (!c || !cls || nsims < 0 || (nsims && !sims)) return fail(DVM_ERR_ARG, "bad argument");
    std::vector<int> slots;
    uint64_t total = 0;
    const int rc = f32_members(c, sims, nsims, slots, total);
    if (rc) return rc;
    *cls = slots.empty() ? -1 : shape_class(total, (int)slots.size());
    return DVM_OK;
}

int dvm_ctx_set_pair_config(dvm_ctx* c, int cls, const dvm_pair_config* cfg) {
    if (!c || !cfg || cls < -1) return fail(DVM_ERR_ARG, "bad argument");
    if (!valid_pair_config(*cfg)) return fail(DVM_ERR_ARG, "invalid pair-kernel configuration");
    std::lock_guard<std::mutex> lk(c->mu);
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));  // graphs of the old shapes are about to go
    if (cls == -1) {
        c->tuning.clear();
        c->tuning_default = to_internal(*cfg);
        c->tuning_default_set = true;
        drop_plans_with(c, -1);
    } else {
        c->tuning[cls] = to_internal(*cfg);
        drop_plans_of_class(c, cls);
    }
    return DVM_OK;
}

int dvm_ctx_tuning_table(dvm_ctx* c, int max_entries, int* classes, dvm_pair_config* cfgs,
                         int* count) {
    if (!c || !count || max_entries < 0 || (max_entries && (!classes || !cfgs)))
        return fail(DVM_ERR_ARG, "bad argument");
    std::lock_guard<std::mutex> lk(c->mu);
    int k = 0;
    for (const auto& kv : c->tuning) {
        if (k < max_entries) {
            classes[k] = kv.first;
            cfgs[k] = to_abi(kv.second);
        }
        ++k;
    }
    *count = k;
    return DVM_OK;
}

int dvm_ctx_get_pair_config(dvm_ctx* c, int cls, dvm_pair_config* out) {
    if (!c || !out) return fail(DVM_ERR_ARG, "bad argument");
    std::lock_guard<std::mutex> lk(c->mu);
    *out = to_abi(tuned_config(c, cls));
    return DVM_OK;
}

int dvm_ctx_autotune(dvm_ctx* c, dvm_sim* const* sims, int nsims, int reps, dvm_tune_result* out) {
    if (!c || !out || nsims <= 0 || nsims > 1024 || !sims) return fail(DVM_ERR_ARG, "bad argument");
    reps = std::max(1, std::min(reps, 100));
    std::lock_guard<std::mutex> lk(c->mu);
    CK(cudaSetDevice(c->device));
    std::vector<int> slots;
    uint64_t total = 0;
    int rc = f32_members(c, sims, nsims, slots, total);
    if (rc) return rc;
    if (slots.empty()) return fail(DVM_ERR_ARG, "no FP32 simulation in the batch");
    std::sort(slots.begin(), slots.end());
    Plan* pl = nullptr;
    rc = get_plan(c, slots, &pl);  // its `all` list is exactly the FP32 members
    if (rc) return rc;
    rc = ensure_workspace(c, pl->ws_need_cap, pl->part_elems, pl->rhs_elems, pl->circ_elems,
                          (int)slots.size(), pl->need_delete);
    if (rc) return rc;
    if (!c->d_tune_list) CK(cudaMalloc(&c->d_tune_list, sizeof(ListEntry) * 1024));
    const SubList& sl = pl->all;
    const std::vector<ListEntry> ordered = costliest_first(sl.host);
    CK(cudaMemcpyAsync(c->d_tune_list, ordered.data(), sizeof(ListEntry) * sl.n,
                       cudaMemcpyHostToDevice, c->stream));
    Workspace ws = c->ws;
    ws.total_cap = sl.total;
    ws.key_bits = key_bits_for(sl.n);
    InstDesc* T = c->d_table;
    InstState* S = c->d_state;
    biot_savart_prepare(T, S, sl.d_list, sl.n, kF32, ws, c->sms, c->stream);
    cudaEvent_t a = nullptr, b = nullptr;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    auto launch = [&](const dvm_pair_config& p) {
        cudaMemsetAsync(ws.work, 0, sizeof(unsigned), c->stream);
        biot_savart_compute(T, S, p.order == 1 ? c->d_tune_list : sl.d_list, sl.n, kF32, ws,
                            c->sms, c->stream, to_internal(p));
    };
    int err = DVM_OK;
    // one untimed launch (module load, caches)
    launch(kCandidates[0]);
    std::memset(out, 0, sizeof(*out));
    out->shape_class = shape_class(total, (int)slots.size());
    out->candidates = kNumCandidates;
    int best = 0;
    for (int k = 0; k < kNumCandidates && !err; ++k) {
        double ms = 0.0;
        for (int r = 0; r < reps; ++r) {
            cudaMemsetAsync(ws.work, 0, sizeof(unsigned), c->stream);
            cudaEventRecord(a, c->stream);
            biot_savart_compute(T, S, kCandidates[k].order == 1 ? c->d_tune_list : sl.d_list,
                                sl.n, kF32, ws, c->sms, c->stream, to_internal(kCandidates[k]));
            cudaEventRecord(b, c->stream);
            float t = 0.f;
            if (cudaEventSynchronize(b) != cudaSuccess || cudaEventElapsedTime(&t, a, b) != cudaSuccess) {
                err = fail(DVM_ERR_CUDA, std::string("autotune: ") +
                                             cudaGetErrorString(cudaGetLastError()));
                break;
            }
            ms += t;
        }
        out->ms[k] = ms / reps;
        if (out->ms[k] < out->ms[best]) best = k;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (err) return err;
    CK(cudaGetLastError());
    g_launches += 3 + (uint64_t)kNumCandidates * reps;  // keys + pack, the warm-up, the timed ones
    out->best = kCandidates[best];
    out->best_ms = out->ms[best];
    out->default_ms = out->ms[0];
    c->tuning[out->shape_class] = to_internal(out->best);
    CK(cudaStreamSynchronize(c->stream));
    drop_plans_of_class(c, out->shape_class);  // they rebuild with the tuned shape
    return DVM_OK;
}

// ---- plugin seam ---------------------------------------------------------------------
static int raw_reserve(dvm_ctx* c, size_t bytes) {
    if (bytes <= c->raw_bytes) return DVM_OK;
    CK(cudaStreamSynchronize(c->stream));
    if (c->raw_block) {
        cudaFree(c->raw_block);
        c->in_use -= c->raw_bytes;
        c->raw_block = nullptr;
        c->raw_bytes = 0;
    }
    bytes = align_up(bytes + bytes / 4, 1 << 20);
    if (c->in_use + bytes > c->budget) return fail(DVM_ERR_OOM, "plugin scratch exceeds the HBM budget");
    CK(cudaMalloc(&c->raw_block, bytes));
    c->raw_bytes = bytes;
    c->in_use += bytes;
    return DVM_OK;
}

// Runs the batched self-induced kernel on caller buffers through table slot 0.
static int raw_self(dvm_ctx* c, const double* x, const double* z, const double* circ,
                    const double* sigma, uint64_t n, double* u, double* w, int precision,
                    double kx0, double kz0, double kinv) {
    if (n == 0) return DVM_OK;
    if (n > 0xF0000000ull) return fail(DVM_ERR_ARG, "too many particles");
    const uint64_t cap = align_up(n, kCapAlign);
    InstDesc h;
    std::memset(&h, 0, sizeof(h));
    h.x = const_cast<double*>(x);
    h.z = const_cast<double*>(z);
    h.circ = const_cast<double*>(circ);
    h.sigma = const_cast<double*>(sigma);
    h.u = u;
    h.w = w;
    h.cap = (uint32_t)cap;
    h.precision = precision;
    h.kx0 = kx0;
    h.kz0 = kz0;
    h.kinv = kinv;
    h.np = 1;
    ListEntry e;
    std::memset(&e, 0, sizeof(e));
    e.inst = 0;
    e.cap = (uint32_t)cap;
    e.chunks = nbody_chunks(e.cap);
    e.rhs_chunks = 1;
    e.rhs_chunk = kAtChunk;
    e.npad = 256;
    const uint64_t part = precision == kF32 ? 1 : (uint64_t)e.chunks * cap;  // FP64 partials
    int rc = ensure_workspace(c, cap, part, 256, 1, 1, false);
    if (rc) return rc;
    ListEntry* d_list = reinterpret_cast<ListEntry*>(c->ws.jobs);
    InstState st0;
    std::memset(&st0, 0, sizeof(st0));
    st0.n = (uint32_t)n;
    CK(cudaMemcpyAsync(c->d_table, &h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_state, &st0, sizeof(st0), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d_list, &e, sizeof(e), cudaMemcpyHostToDevice, c->stream));
    Workspace ws = c->ws;
    ws.key_bits = key_bits_for(1);
    ws.total_cap = cap;
    biot_savart_self(c->d_table, c->d_state, d_list, 1, precision, ws, c->sms, c->stream,
                     tuned_config(c, shape_class(cap, 1)));
    g_launches += 4;  // keys, pack, pair kernel, combine
    CK(cudaGetLastError());
    return DVM_OK;
}

int dvm_biot_savart_self_device(dvm_ctx* c, const double* x, const double* z, const double* circ,
                                const double* sigma, uint64_t n, double* u, double* w,
                                int precision) {
    if (!c || (n && (!x || !z || !circ || !sigma || !u || !w))) return fail(DVM_ERR_ARG, "null argument");
    if (precision != DVM_F64 && precision != DVM_F32) return fail(DVM_ERR_ARG, "bad precision");
    std::lock_guard<std::mutex> lk(c->mu);
    CK(cudaSetDevice(c->device));
    return raw_self(c, x, z, circ, sigma, n, u, w, precision, -64.0, -64.0, 65536.0 / 128.0);
}

int dvm_biot_savart_self(dvm_ctx* c, const dvm_particle* p, uint64_t n, dvm_velocity* out,
                         int precision) {
    if (!c || (n && (!p || !out))) return fail(DVM_ERR_ARG, "null argument");
    if (precision != DVM_F64 && precision != DVM_F32) return fail(DVM_ERR_ARG, "bad precision");
    if (n == 0) return DVM_OK;
    std::lock_guard<std::mutex> lk(c->mu);
    CK(cudaSetDevice(c->device));
    // AoS -> SoA on the host while computing the Morton domain.
    std::vector<double> h(6 * n);
    double xmn = p[0].x, xmx = p[0].x, zmn = p[0].z, zmx = p[0].z;
    for (uint64_t i = 0; i < n; ++i) {
        h[i] = p[i].x;
        h[n + i] = p[i].z;
        h[2 * n + i] = p[i].circ;
        h[3 * n + i] = p[i].sigma;
        xmn = std::min(xmn, p[i].x);
        xmx = std::max(xmx, p[i].x);
        zmn = std::min(zmn, p[i].z);
        zmx = std::max(zmx, p[i].z);
    }
    int rc = raw_reserve(c, 8 * 6 * n);
    if (rc) return rc;
    double* d = static_cast<double*>(c->raw_block);
    CK(cudaMemcpyAsync(d, h.data(), 8 * 4 * n, cudaMemcpyHostToDevice, c->stream));
    double L = std::max(xmx - xmn, zmx - zmn);
    if (!(L > 0)) L = 1.0;
    rc = raw_self(c, d, d + n, d + 2 * n, d + 3 * n, n, d + 4 * n, d + 5 * n, precision, xmn, zmn,
                  65535.0 / L);
    if (rc) return rc;
    CK(cudaMemcpyAsync(h.data() + 4 * n, d + 4 * n, 8 * 2 * n, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (uint64_t i = 0; i < n; ++i) {
        out[i].u = h[4 * n + i];
        out[i].w = h[5 * n + i];
    }
    return DVM_OK;
}

int dvm_random_walk(dvm_ctx* c, double* x, double* z, uint64_t n, const double* R, double nu,
                    double dt) {
    if (!c || (n && (!x || !z || !R))) return fail(DVM_ERR_ARG, "null argument");
    if (n == 0) return DVM_OK;
    if (n > 0xF0000000ull) return fail(DVM_ERR_ARG, "too many blobs");
    std::lock_guard<std::mutex> lk(c->mu);
    CK(cudaSetDevice(c->device));
    int rc = raw_reserve(c, 8 * 4 * n);
    if (rc) return rc;
    double* d = static_cast<double*>(c->raw_block);
    CK(cudaMemcpyAsync(d, x, 8 * n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d + n, z, 8 * n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d + 2 * n, R, 16 * n, cudaMemcpyHostToDevice, c->stream));
    diffuse_raw(d, d + n, (uint32_t)n, d + 2 * n, nu, dt, c->sms, c->stream);
    g_launches += 1;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(x, d, 8 * n, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(z, d + n, 8 * n, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DVM_OK;
}

int dvm_biot_savart_at_device(dvm_ctx* c, const double* x, const double* z, const double* circ,
                              const double* sigma, uint64_t ns, const double* tx, const double* tz,
                              uint64_t nt, double* u, double* w, int precision, int skip_close) {
    if (!c) return fail(DVM_ERR_ARG, "ctx is null");
    if (nt && (!tx || !tz || !u || !w)) return fail(DVM_ERR_ARG, "null target array");
    if (ns && (!x || !z || !circ || !sigma)) return fail(DVM_ERR_ARG, "null source array");
    if (precision != DVM_F64 && precision != DVM_F32) return fail(DVM_ERR_ARG, "bad precision");
    if (nt == 0) return DVM_OK;
    if (ns > 0xF0000000ull || nt > 0xF0000000ull) return fail(DVM_ERR_ARG, "too many points");
    std::lock_guard<std::mutex> lk(c->mu);
    CK(cudaSetDevice(c->device));
    const size_t elems = direct_at_part_elems((uint32_t)ns, (uint32_t)nt);
    int rc = raw_reserve(c, 16 * elems);
    if (rc) return rc;
    direct_at_raw(x, z, circ, sigma, (uint32_t)ns, tx, tz, (uint32_t)nt, u, w, precision, skip_close,
                  static_cast<double2*>(c->raw_block), c->sms, c->stream);
    g_launches += 2;
    CK(cudaGetLastError());
    return DVM_OK;
}

// ---- vortex merging ----------------------------------------------------------------------
int dvm_sim_merge(dvm_sim* s, double threshold, uint64_t* merged) {
    if (!s) return fail(DVM_ERR_ARG, "sim is null");
    dvm_ctx* c = s->ctx;
    uint32_t cnt = 0;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        CK(cudaSetDevice(c->device));
        uint32_t n = 0;
        CK(cudaMemcpyAsync(&n, &c->d_state[s->slot].n, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                           c->stream));
        CK(cudaStreamSynchronize(c->stream));
        void* scratch = nullptr;
        const cudaError_t e = pool_alloc(c, &scratch, merge_scratch_bytes(n));
        if (e != cudaSuccess)
            return fail(DVM_ERR_OOM, std::string("merge scratch: ") + cudaGetErrorString(e));
        const InstDesc& h = s->h;
        uint32_t* cdev =
            reinterpret_cast<uint32_t*>(static_cast<char*>(scratch) + merge_count_offset(n));
        merge_run(MergeArrays{h.x, h.z, h.circ, h.sigma, h.u, h.w, h.uvs, h.wvs}, h.id, n,
                  threshold, &c->d_state[s->slot].n, cdev, scratch, c->sms, c->stream);
        CK(cudaMemcpyAsync(&cnt, cdev, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
        pool_free(c, scratch);
        g_launches += 4;
        CK(cudaStreamSynchronize(c->stream));
    }
    if (merged) *merged = cnt;
    return DVM_OK;
}

int dvm_merge_blobs(dvm_ctx* c, double* x, double* z, double* circ, double* sigma, double* u,
                    double* w, double* uvs, double* wvs, uint32_t* id, uint64_t n,
                    double threshold, uint64_t* n_out, uint64_t* merged) {
    if (!c || !n_out || (n && (!x || !z || !circ || !sigma || !u || !w || !uvs || !wvs)))
        return fail(DVM_ERR_ARG, "null argument");
    if (n > 0xF0000000ull) return fail(DVM_ERR_ARG, "too many blobs");
    *n_out = n;
    if (merged) *merged = 0;
    if (n < 2) return DVM_OK;
    std::lock_guard<std::mutex> lk(c->mu);
    CK(cudaSetDevice(c->device));
    int rc = raw_reserve(c, 8 * 8 * (size_t)n);
    if (rc) return rc;
    double* d = static_cast<double*>(c->raw_block);
    double* const host[8] = {x, z, circ, sigma, u, w, uvs, wvs};
    for (int k = 0; k < 8; ++k)
        CK(cudaMemcpyAsync(d + k * n, host[k], 8 * n, cudaMemcpyHostToDevice, c->stream));
    void* scratch = nullptr;
    const uint32_t nn = (uint32_t)n;
    const cudaError_t e = pool_alloc(c, &scratch, merge_scratch_bytes(nn));
    if (e != cudaSuccess) return fail(DVM_ERR_OOM, std::string("merge scratch: ") + cudaGetErrorString(e));
    uint32_t* cdev = reinterpret_cast<uint32_t*>(static_cast<char*>(scratch) + merge_count_offset(nn));
    merge_run(MergeArrays{d, d + n, d + 2 * n, d + 3 * n, d + 4 * n, d + 5 * n, d + 6 * n, d + 7 * n},
              nullptr, nn, threshold, nullptr, cdev, scratch, c->sms, c->stream);
    uint32_t cnt = 0;
    CK(cudaMemcpyAsync(&cnt, cdev, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    pool_free(c, scratch);
    g_launches += 4;
    CK(cudaStreamSynchronize(c->stream));
    const uint64_t m = n - cnt;
    for (int k = 0; k < 8; ++k)
        CK(cudaMemcpyAsync(host[k], d + k * n, 8 * m, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (cnt && id)
        for (uint64_t q = 0; q < m; ++q) id[q] = (uint32_t)q;
    *n_out = m;
    if (merged) *merged = cnt;
    return DVM_OK;
}

// ---- remeshing -------------------------------------------------------------------------
static int remesh_grid_of(const dvm_remesh_params* p, RemeshGrid* g) {
    if (!p) return fail(DVM_ERR_ARG, "remesh parameters are null");
    if (!(p->dx > 0) || !(p->dz > 0)) return fail(DVM_ERR_ARG, "remesh dx, dz must be > 0");
    if (!(p->xmax >= p->xmin) || !(p->zmax >= p->zmin))
        return fail(DVM_ERR_ARG, "remesh bounds: need xmax >= xmin and zmax >= zmin");
    if (p->kernel < DVM_REMESH_M4PRIME || p->kernel > DVM_REMESH_GAUSSIAN)
        return fail(DVM_ERR_ARG, "unknown remesh kernel");
    const double fx = std::floor((p->xmax - p->xmin) / p->dx + 1e-9);
    const double fz = std::floor((p->zmax - p->zmin) / p->dz + 1e-9);
    if (!(fx < 65535.0) || !(fz < 65535.0) || (fx + 1.0) * (fz + 1.0) > (double)(1u << 28))
        return fail(DVM_ERR_ARG, "remesh mesh too large (at most 2^28 nodes)");
    g->x0 = p->xmin;
    g->z0 = p->zmin;
    g->dx = p->dx;
    g->dz = p->dz;
    g->sigma = p->sigma;
    g->threshold = p->circ_threshold;
    g->nx = (int)fx + 1;
    g->nz = (int)fz + 1;
    g->kernel = p->kernel;
    return DVM_OK;
}

int dvm_remesh_grid(const dvm_remesh_params* p, uint32_t* nx, uint32_t* nz) {
    RemeshGrid g;
    const int rc = remesh_grid_of(p, &g);
    if (rc) return rc;
    if (nx) *nx = (uint32_t)g.nx;
    if (nz) *nz = (uint32_t)g.nz;
    return DVM_OK;
}

int dvm_sim_remesh(dvm_sim* s, const dvm_remesh_params* p, uint64_t* n_out) {
    if (!s) return fail(DVM_ERR_ARG, "sim is null");
    RemeshGrid g;
    int rc = remesh_grid_of(p, &g);
    if (rc) return rc;
    dvm_ctx* c = s->ctx;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        CK(cudaSetDevice(c->device));
        uint32_t n = 0;
        CK(cudaMemcpyAsync(&n, &c->d_state[s->slot].n, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                           c->stream));
        CK(cudaStreamSynchronize(c->stream));
        void* scratch = nullptr;
        const cudaError_t e =
            pool_alloc(c, &scratch, remesh_scratch_bytes(g, n, s->h.cap));
        if (e != cudaSuccess)
            return fail(DVM_ERR_OOM, std::string("remesh scratch: ") + cudaGetErrorString(e));
        const InstDesc& h = s->h;
        RemeshDest d{h.x, h.z, h.circ, h.sigma, h.u, h.w, h.uvs, h.wvs, h.id,
                     &c->d_state[s->slot].n, nullptr};
        remesh_run(g, h.x, h.z, h.circ, h.sigma, n, h.cap, d, &c->d_state[s->slot].status,
                   scratch, c->sms, c->stream);
        pool_free(c, scratch);
        g_launches += 7;
        CK(cudaGetLastError());
    }
    rc = dvm_sim_status(s);
    if (rc) return rc;
    if (n_out) return dvm_sim_num_blobs(s, n_out);
    return DVM_OK;
}

int dvm_remesh(dvm_ctx* c, const dvm_particle* in, uint64_t n, const dvm_remesh_params* p,
               dvm_particle* out, uint64_t out_cap, uint64_t* n_out) {
    if (!c || (n && !in) || (out_cap && !out) || !n_out) return fail(DVM_ERR_ARG, "null argument");
    if (n > 0xF0000000ull || out_cap > 0xF0000000ull) return fail(DVM_ERR_ARG, "too many blobs");
    RemeshGrid g;
    int rc = remesh_grid_of(p, &g);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    CK(cudaSetDevice(c->device));
    const size_t data = align_up(8 * 4 * (size_t)n, 256) + align_up(8 * 4 * (size_t)out_cap, 256) + 256;
    rc = raw_reserve(c, data);
    if (rc) return rc;
    char* base = static_cast<char*>(c->raw_block);
    double* din = reinterpret_cast<double*>(base);
    double* dout = reinterpret_cast<double*>(base + align_up(8 * 4 * (size_t)n, 256));
    uint32_t* dneed = reinterpret_cast<uint32_t*>(base + data - 256);
    std::vector<double> h(4 * n);
    for (uint64_t i = 0; i < n; ++i) {
        h[i] = in[i].x;
        h[n + i] = in[i].z;
        h[2 * n + i] = in[i].circ;
        h[3 * n + i] = in[i].sigma;
    }
    if (n) CK(cudaMemcpyAsync(din, h.data(), 8 * 4 * n, cudaMemcpyHostToDevice, c->stream));
    void* scratch = nullptr;
    const cudaError_t e = pool_alloc(c, &scratch, remesh_scratch_bytes(g, (uint32_t)n, (uint32_t)out_cap));
    if (e != cudaSuccess) return fail(DVM_ERR_OOM, std::string("remesh scratch: ") + cudaGetErrorString(e));
    RemeshDest d{dout, dout + out_cap, dout + 2 * out_cap, dout + 3 * out_cap, nullptr, nullptr,
                 nullptr, nullptr, nullptr, nullptr, dneed};
    remesh_run(g, din, din + n, din + 2 * n, din + 3 * n, (uint32_t)n, (uint32_t)out_cap, d,
               nullptr, scratch, c->sms, c->stream);
    pool_free(c, scratch);
    g_launches += 7;
    uint32_t need = 0;
    CK(cudaMemcpyAsync(&need, dneed, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *n_out = need;
    if (need > out_cap)
        return fail(DVM_ERR_CAPACITY, "remesh: " + std::to_string(need) + " blobs do not fit out_cap");
    std::vector<double> r(4 * (size_t)out_cap);
    if (need) CK(cudaMemcpy(r.data(), dout, 8 * 4 * (size_t)out_cap, cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < need; ++i)
        out[i] = dvm_particle{r[i], r[out_cap + i], r[2 * out_cap + i], r[3 * out_cap + i]};
    return DVM_OK;
}

int dvm_sim_probe(dvm_sim* s, const double* px, const double* pz, uint64_t n, double* u,
                  double* w, double* uvs, double* wvs) {
    if (!s) return fail(DVM_ERR_ARG, "sim is null");
    if (n && (!px || !pz || !u || !w)) return fail(DVM_ERR_ARG, "null probe array");
    if (n == 0) return DVM_OK;
    if (n > (1u << 24)) return fail(DVM_ERR_ARG, "too many probe points (max 2^24)");
    dvm_ctx* c = s->ctx;
    std::lock_guard<std::mutex> lk(c->mu);
    CK(cudaSetDevice(c->device));
    uint32_t ns = 0;
    CK(cudaMemcpyAsync(&ns, &c->d_state[s->slot].n, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const uint32_t nt = (uint32_t)n;
    const size_t part_bytes = align_up(16 * direct_at_part_elems(ns, nt), 256);
    int rc = raw_reserve(c, part_bytes + 8 * 6 * (size_t)n);
    if (rc) return rc;
    double* d = reinterpret_cast<double*>(static_cast<char*>(c->raw_block) + part_bytes);
    double *dx = d, *dz = d + n, *dres = d + 2 * n;  // dres: u, w, uvs, wvs
    CK(cudaMemcpyAsync(dx, px, 8 * n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(dz, pz, 8 * n, cudaMemcpyHostToDevice, c->stream));
    // blobs: the at-target sum (pairs closer than r^2 = 1e-15 skipped, as in
    // src/VelocityKernel.cpp:89), in the simulation's precision
    direct_at_raw(s->h.x, s->h.z, s->h.circ, s->h.sigma, ns, dx, dz, nt, dres, dres + n,
                  s->h.precision, 1, static_cast<double2*>(c->raw_block), c->sms, c->stream);
    sheet_at(s->h, dx, dz, nt, dres + 2 * n, dres + 3 * n, c->stream);
    g_launches += ns ? 3 : 1;
    std::vector<double> h(4 * n);
    CK(cudaMemcpyAsync(h.data(), dres, 8 * 4 * n, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (uint64_t i = 0; i < n; ++i) {
        u[i] = (h[i] + h[2 * n + i]) + s->h.ux;
        w[i] = (h[n + i] + h[3 * n + i]) + s->h.uz;
        if (uvs) uvs[i] = h[2 * n + i];
        if (wvs) wvs[i] = h[3 * n + i];
    }
    return DVM_OK;
}

int dvm_biot_savart_at(dvm_ctx* c, const dvm_particle* p, uint64_t ns, const double* tx,
                       const double* tz, uint64_t nt, dvm_velocity* out, int precision) {
    if (!c || (ns && !p) || (nt && (!tx || !tz || !out))) return fail(DVM_ERR_ARG, "null argument");
    if (precision != DVM_F64 && precision != DVM_F32) return fail(DVM_ERR_ARG, "bad precision");
    if (nt == 0) return DVM_OK;
    std::lock_guard<std::mutex> lk(c->mu);
    CK(cudaSetDevice(c->device));
    const size_t elems = direct_at_part_elems((uint32_t)ns, (uint32_t)nt);
    const size_t part_bytes = align_up(16 * elems, 256);
    const size_t data_bytes = 8 * (4 * ns + 4 * nt);
    int rc = raw_reserve(c, part_bytes + data_bytes);
    if (rc) return rc;
    char* base = static_cast<char*>(c->raw_block);
    double* d = reinterpret_cast<double*>(base + part_bytes);
    std::vector<double> h(4 * ns + 2 * nt);
    for (uint64_t i = 0; i < ns; ++i) {
        h[i] = p[i].x;
        h[ns + i] = p[i].z;
        h[2 * ns + i] = p[i].circ;
        h[3 * ns + i] = p[i].sigma;
    }
    std::memcpy(h.data() + 4 * ns, tx, 8 * nt);
    std::memcpy(h.data() + 4 * ns + nt, tz, 8 * nt);
    CK(cudaMemcpyAsync(d, h.data(), 8 * h.size(), cudaMemcpyHostToDevice, c->stream));
    double* du = d + 4 * ns + 2 * nt;
    double* dw = du + nt;
    direct_at_raw(d, d + ns, d + 2 * ns, d + 3 * ns, (uint32_t)ns, d + 4 * ns, d + 4 * ns + nt,
                  (uint32_t)nt, du, dw, precision, 1, reinterpret_cast<double2*>(base), c->sms,
                  c->stream);
    g_launches += 2;
    std::vector<double> r(2 * nt);
    CK(cudaMemcpyAsync(r.data(), du, 8 * 2 * nt, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (uint64_t i = 0; i < nt; ++i) {
        out[i].u = r[i];
        out[i].w = r[nt + i];
    }
    return DVM_OK;
}

}  // extern "C"
