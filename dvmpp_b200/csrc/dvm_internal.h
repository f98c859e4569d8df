// Internal definitions shared by the CUDA translation units of libdvm_cuda.so.
//
// Data model (one GPU, everything resident in HBM):
//   * A simulation instance ("sim") owns SoA FP64 blob arrays with a fixed
//     capacity, its body (contour, panels, influence matrix A and its
//     least-squares pseudo-inverse P = R^-1 Q^T), its sheet strengths gamma and
//     its counters.  All of it is described by one InstDesc in a device-side
//     table, so every kernel can serve any subset of sims in one launch
//     ("batched"), addressed through a list of ListEntry records.
//   * The blob count n of a sim lives on the device (InstState) and is updated
//     by the release / delete kernels; no kernel needs the host to know it,
//     which is what lets a whole step be captured in one CUDA graph.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace dvmk {

constexpr double kPi = 3.14159265358979323846;                 // src/BaseTypes.hpp:18
constexpr double kRpi2 = 1.0 / (2.0 * 3.14159265358979323846);  // src/BaseTypes.hpp:21

enum Status : int {
    kOk = 0,
    kErrArg = 1,
    kErrOom = 2,
    kErrCuda = 3,
    kErrTimeout = 4,
    kErrCapacity = 5,
    kErrRelease = 6,
    kErrState = 7,
    kErrRngExhausted = 8,
};

enum Precision : int { kF64 = 0, kF32 = 1 };
enum Scheme : int { kEuler = 0, kRK3 = 1 };
enum Cross : int { kDelete = 0, kAbsorb = 1, kReflect = 2 };
enum Rng : int { kInject = 0, kPhilox = 1 };

// N-body tiling (targets per work item, sources per shared-memory stage).
constexpr int kBsThreads = 256;
constexpr int kBsR = 4;                        // consecutive targets per thread
constexpr int kBsTT = kBsThreads * kBsR;       // 1024 targets per item
constexpr int kBsST = 256;                     // sources per stage (= sort tile)
constexpr int kAtChunk = 4096;                 // sources per item of the at-target kernels
constexpr int kCapAlign = 1024;                // capacities are multiples of this
constexpr int kMaxBatch = 1024;                // simulations per batched step
constexpr int kTableCap = 4096;                // simulation slots per context

// Sources per work item of a simulation's blob-on-collocation right-hand side:
// a power of two in [512, kAtChunk], the smallest that still leaves about 600
// items (four per SM) when the simulation is evaluated alone, so a single
// simulation fills the GPU.  It depends only on the capacity and the panel
// count, so the sum is grouped the same way alone and in any batch; a
// simulation then has at most ~600 chunks, or cap / kAtChunk + 1 when large.
inline uint32_t rhs_chunk_for(uint32_t cap, int np) {
    const uint64_t tiles = ((uint64_t)np + 511) / 512;
    const uint64_t want = ((uint64_t)cap * tiles + 599) / 600;
    uint32_t c = 512;
    while (c < (uint32_t)kAtChunk && c < want) c <<= 1;
    return c;
}

// Device-side description of one simulation instance.
struct InstDesc {
    // blob state, SoA, capacity `cap`
    double* x;
    double* z;
    double* circ;
    double* sigma;
    double* u;
    double* w;
    double* uvs;
    double* wvs;
    double* q1;  // RK3 low-storage registers
    double* q2;
    uint32_t* id;
    // body: contour points (np+1) and per-panel data (np)
    const double* xp;
    const double* zp;
    const double* xc;
    const double* zc;
    const double* ds;
    const double* enx;
    const double* enz;
    const double* etx;
    const double* etz;
    const double* cth;     // cos(theta)
    const double* sth;     // sin(theta)
    const double* c2th;    // cos(-2 theta)
    const double* s2th;    // sin(-2 theta)
    const double* psigma;  // pow(ds, cutoff_exp): core size of blobs released by the panel
    const double* A;       // (np+1) x np influence matrix, row-major
    const double* P;       // np x (np+1) pseudo-inverse, row-major
    double* gamma;         // np
    double* b;             // np+1 right-hand side
    double* res;           // np+1 refinement residual
    // random stream (inject mode): uniforms[0 .. ucount), read at state.cursor
    const double* uniforms;
    uint64_t ucount;
    // scalars
    double rho, nu, dt, ux, uz, cutoff_exp, Ur, area;
    double bxmax, bzmin, bzmax;     // contour bounding box (x padded) for the crossing early-out
    double bxmin;
    double kx0, kz0, kinv;          // Morton-key domain: cell = (x - kx0) * kinv
    uint32_t M;                     // max_NumPanelVort
    int np;
    int scheme, cross, rng, precision, refine;
    uint32_t cap;
    uint64_t seed;
    uint32_t uid;  // reserved (0): Philox counters depend on (index, step, stream) only
};

// Mutable per-instance counters, kept apart from the (read-mostly) descriptor.
struct InstState {
    uint32_t n;        // current blob count
    uint32_t step;     // DVMBase::m_step
    uint64_t cursor;   // next uniform to consume (inject mode)
    int status;        // first error raised on the device for this instance
    int pad;
    double fx, fz, cd, cl;  // last loads
    double totalcirc;       // last Kelvin sum (sum of circ)
};

// One simulation inside a batched launch.  Offsets are host-known (derived
// from capacities), so work buffers can be sized before a graph is captured.
struct ListEntry {
    int inst;          // table index
    int chunks;        // N-body source chunks (fixed by capacity)
    int rhs_chunks;    // at-target source chunks = ceil(cap / rhs_chunk)
    int npad;          // np rounded up to kBsThreads
    uint32_t cap;
    uint32_t rhs_chunk;  // sources per at-target work item (rhs_chunk_for)
    uint64_t coff;     // offset in the concatenated capacity space (multiple of kCapAlign)
    uint64_t poff;     // N-body partials offset (double2): sum chunks * cap
    uint64_t roff;     // at-target partials offset (double2): sum rhs_chunks * npad
    uint64_t cofs;     // circulation partials offset (double): sum rhs_chunks
};

// Per-tile bounds of a 256-blob tile of the spatially sorted sources.
struct TileMeta {
    double xmin, xmax, zmin, zmax, thr, pad0, pad1, pad2;
};

// Device work buffers of a batched step, sized by the host for one list.
struct Workspace {
    uint64_t total_cap = 0;  // sum of capacities in the list
    uint64_t* keys_in = nullptr;
    uint64_t* keys_out = nullptr;
    uint32_t* vals_in = nullptr;
    uint32_t* perm = nullptr;      // sorted slot -> original blob index
    double4* packed = nullptr;     // sorted (x, z, circ, sigma); the FP32 path reuses it as
                                   // double2 (x, z) | float4 (circ, 10 sigma^2, 1/sigma^2, -)
    uint64_t packed_cap = 0;       // slots of `packed`
    TileMeta* meta = nullptr;      // total_cap / kBsST
    double2* part = nullptr;       // N-body partials
    // FP32 N-body, mutual far tiles: per sorted blob two 64-bit fixed-point sums
    // (Gamma_i K dz, Gamma_i K dx over the targets i whose tile evaluated this blob as a
    // source), 2 * total_cap; and per simulation slot the exponent bounds of
    // their scale (max |Gamma|, 1 / min core radius, max |coordinate|, one unused:
    // 4 * kTableCap)
    unsigned long long* macc = nullptr;
    int* mexp = nullptr;
    double2* rhs_part = nullptr;   // at-target partials
    double* circ_part = nullptr;
    void* cub_tmp = nullptr;
    size_t cub_bytes = 0;
    unsigned* work = nullptr;      // 16 dynamic work counters
    uint8_t* flags = nullptr;      // delete: keep flags, total_cap
    uint32_t* tile_counts = nullptr;  // delete: kept per 1024-tile, total_cap / 1024
    uint32_t* tile_base = nullptr;    // delete: exclusive prefix of tile_counts, per simulation
    uint32_t* del_kept = nullptr;     // delete: kept blobs per list entry
    uint32_t* del_ready = nullptr;  // delete: per 1024-tile "sources read" flags
    void* jobs = nullptr;          // per-entry job records (256 B each)
    int key_bits = 40;
};

// Sets the calling thread's dvm_last_error() message; returns `code`.
int report_error(int code, const char* msg);

// ---- launchers (all asynchronous on `s`) ------------------------------------
size_t cub_sort_bytes(uint64_t total);

// Launch shape of the FP32 pair kernel.  None of it changes a result: the
// source chunking (which does) is fixed by each simulation's capacity.
struct PairConfig {
    int tile = 256;  // targets per work item (one sort tile)
    int ctas = 4;    // persistent CTAs per SM
    int order = 0;   // 0: list order; 1: costliest simulations' items first (the caller
                     // passes the list in that order)
};

// Self-induced Biot-Savart (src/VelocityKernel.cpp:30-67) for every listed sim:
// FP32 + compensated sums over spatially sorted blobs, or FP64 in blob order.
void biot_savart_self(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
                      int precision, const Workspace& ws, int sms, cudaStream_t s,
                      const PairConfig& cfg = PairConfig());
// The same in three parts (sort + pack / pair kernel / combine + scatter), so
// the pair kernel can be timed on its own.
void biot_savart_prepare(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
                         int precision, const Workspace& ws, int sms, cudaStream_t s);
void biot_savart_compute(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
                         int precision, const Workspace& ws, int sms, cudaStream_t s,
                         const PairConfig& cfg = PairConfig());
void biot_savart_finish(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
                        int precision, const Workspace& ws, int sms, cudaStream_t s);
// Blob-on-collocation right-hand side b (src/VortexSheet.cpp:171-210).
void sheet_rhs(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
               int max_np, int precision, const Workspace& ws, int sms, cudaStream_t s);
// Velocity at arbitrary targets from one blob set (src/VelocityKernel.cpp:69-109).
void direct_at_raw(const double* x, const double* z, const double* circ, const double* sigma,
                   uint32_t ns, const double* tx, const double* tz, uint32_t nt, double* u,
                   double* w, int precision, int skip_close, double2* part, int sms,
                   cudaStream_t s);
size_t direct_at_part_elems(uint32_t ns, uint32_t nt);
// Remeshing onto a background mesh (k_remesh.cu).  Nodes are x0 + i dx,
// z0 + j dz for i < nx, j < nz.
enum RemeshKernel : int { kRemeshM4p = 0, kRemeshM6 = 1, kRemeshGauss = 2 };
struct RemeshGrid {
    double x0, z0, dx, dz, sigma, threshold;
    int nx, nz, kernel;
};
struct RemeshDest {  // where the new blob set goes (u..id may be null)
    double *x, *z, *circ, *sigma, *u, *w, *uvs, *wvs;
    uint32_t* id;
    uint32_t* n;     // new count, written only when it fits the capacity
    uint32_t* need;  // new count, always (may be null)
};
size_t remesh_scratch_bytes(const RemeshGrid& g, uint32_t n, uint32_t cap);
void remesh_run(const RemeshGrid& g, const double* x, const double* z, const double* circ,
                const double* sigma, uint32_t n, uint32_t cap, const RemeshDest& dest,
                int* status, void* scratch, int sms, cudaStream_t s);

// Vortex merging (k_merge.cu), in place on 8 SoA arrays of n blobs; the merge
// count goes to scratch + merge_count_offset(n), the new length to n_dev.
struct MergeArrays {
    double *x, *z, *circ, *sigma, *u, *w, *uvs, *wvs;
};
size_t merge_scratch_bytes(uint32_t n);
size_t merge_count_offset(uint32_t n);
void merge_run(const MergeArrays& a, uint32_t* id, uint32_t n, double threshold,
               uint32_t* n_dev, uint32_t* count_dev, void* scratch, int sms, cudaStream_t s);

// Sheet velocity at arbitrary points from one simulation's panels and gamma
// (the sheet-on-blob sum of src/VortexSheet.cpp:217-273, FP64), for probes.
void sheet_at(const InstDesc& d, const double* px, const double* pz, uint32_t n, double* uvs,
              double* wvs, cudaStream_t s);

// gamma = P b (+ refinement), replacing src/VortexSheet.cpp:214.
void sheet_solve(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
                 int max_np, cudaStream_t s);
// Sheet-on-blob velocity (src/VortexSheet.cpp:217-273), optionally fused with
// the convection update of the Euler / RK3 stage (src/DVMBase.cpp:167-209).
//   mode 0: uvs/wvs only; 1: Euler update; 2+k: RK3 stage k (k = 0,1,2)
void sheet_velocity(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
                    int mode, int max_np, const Workspace& ws, int sms, cudaStream_t s);
// x += (u + uvs + Ux) dt without recomputing uvs (used by the phase API).
void convect_update(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
                    int mode, const Workspace& ws, int sms, cudaStream_t s);
void diffuse(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
             const Workspace& ws, int sms, cudaStream_t s);
// src/VortexBlobs.cpp:251-265 on caller device buffers, uniforms R[2i], R[2i+1].
void diffuse_raw(double* x, double* z, uint32_t n, const double* R, double nu, double dt,
                 int sms, cudaStream_t s);
void release(const InstDesc* table, InstState* st, const ListEntry* list, int nlist, int max_np,
             cudaStream_t s);
void reflect(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
             int max_np, const Workspace& ws, int sms, cudaStream_t s);
void delete_inside(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
                   int max_np, const Workspace& ws, int sms, cudaStream_t s);
void loads(const InstDesc* table, InstState* st, const ListEntry* list, int nlist, int max_np,
           cudaStream_t s);
void step_counter(InstState* st, const ListEntry* list, int nlist, cudaStream_t s);

// Body set-up, once per body (FP64).
void influence_matrix(const double* xp, const double* zp, const double* xc, const double* zc,
                      const double* ds, const double* theta, int np, double* pq_scratch,
                      double* A, cudaStream_t s);
// Householder QR of A ((np+1) x np, row-major) and P = R^-1 Q^T (np x (np+1))
// for n bodies, each with its own A, P and workspace
// (pseudo_inverse_work_doubles(np)): bodies that take the register-resident
// path are factorised together, up to 8 per cooperative launch, with the same
// arithmetic per body as alone.  *launches (if not null) receives the number of
// factorisation kernels launched.
cudaError_t pseudo_inverse_many(int n, const double* const* A, const int* np, double* const* P,
                                double* const* work, cudaStream_t s, int* launches);
size_t pseudo_inverse_work_doubles(int np);

}  // namespace dvmk
