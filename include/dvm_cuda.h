/* dvm_cuda.h -- C ABI of libdvm_cuda.so, the B200 (sm_100a) implementation of
 * the DVMpp per-step hot path.
 *
 * Plain C types only (pointers, sizes, doubles); no CUDA or C++ types cross
 * this boundary.  Every entry point returns a status code (DVM_OK == 0) and
 * never throws; dvm_last_error() gives the message of the calling thread's
 * last failure.  The C++ drop-in classes (dvmpp_b200/host) map statuses to the
 * reference's dvm:: exceptions (src/Exceptions.hpp:13-81).
 *
 * Reference interfaces replaced (gdeskos/DVMpp, file:line):
 *   dvm_biot_savart_self      DirectKernel::computeSelfInduced  src/VelocityKernel.cpp:30-67
 *   dvm_biot_savart_at        DirectKernel::computeInducedAt    src/VelocityKernel.cpp:69-109
 *   dvm_sim_create /
 *   dvm_sims_create           VortexSheet(xml, stamp) set-up    src/VortexSheet.cpp:12-54,78-165
 *   dvm_sim_set_blobs /
 *   dvm_sim_get_blobs         VortexBlobs public SoA members    src/VortexBlobs.hpp:24-32
 *   dvm_sim_phase(BIOTSAVART) VortexBlobs::biotsavart           src/VortexBlobs.cpp:229-249
 *   dvm_sim_phase(SOLVE)      VortexSheet::solvevortexsheet     src/VortexSheet.cpp:167-215
 *   dvm_sim_phase(SHEETBC)    VortexSheet::vortexsheetbc        src/VortexSheet.cpp:217-273
 *   dvm_sim_phase(CONVECT)    DVMBase::convect                  src/DVMBase.cpp:167-209
 *   dvm_sim_phase(DIFFUSE)    VortexBlobs::diffusion_random_walk src/VortexBlobs.cpp:251-265
 *   dvm_sim_phase(RELEASE)    release_nascent_vortices_rw + append_vortices
 *                                                               src/VortexSheet.cpp:275-333,
 *                                                               src/VortexBlobs.cpp:211-227
 *   dvm_sim_phase(CROSS)      surface-crossing dispatch         src/DVMBase.cpp:107-118
 *   dvm_sim_phase(REFLECT)    VortexSheet::reflect              src/VortexSheet.cpp:345-405
 *   dvm_sim_phase(DELETE)     VortexSheet::delete_inside        src/VortexSheet.cpp:407-445
 *   dvm_sim_phase(LOADS)      VortexSheet::compute_loads        src/VortexSheet.cpp:487-514
 *   dvm_sim_step              DVMBase::compute_step (+increment_step)
 *                                                               src/DVMBase.cpp:86-133,145-149
 *   dvm_sim_push_uniforms     Random::rand stream feed          src/Random.cpp:8-18
 *   dvm_step_batch            (no counterpart: many simulations per launch)
 *   dvm_ctx_autotune          (no counterpart: pair-kernel launch shapes)
 *   dvm_server_*              (no counterpart: continuous-batching request loop)
 */
#ifndef DVM_CUDA_H
#define DVM_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DVM_ABI_VERSION 1

/* status codes */
#define DVM_OK 0
#define DVM_ERR_ARG 1        /* bad argument (null pointer, size mismatch, bad enum) */
#define DVM_ERR_OOM 2        /* device allocation failed or HBM budget exceeded */
#define DVM_ERR_CUDA 3       /* CUDA runtime error (message in dvm_last_error) */
#define DVM_ERR_TIMEOUT 4    /* bounded device wait ran out (reserved) */
#define DVM_ERR_CAPACITY 5   /* a release would exceed the simulation's blob capacity */
#define DVM_ERR_RELEASE 6    /* release count not > 1e-15 (reference throws VortexException) */
#define DVM_ERR_STATE 7      /* call not valid in the current state */
#define DVM_ERR_RNG 8        /* injected uniform stream exhausted */
#define DVM_ERR_NO_DEVICE 9  /* no CUDA device / library built for another GPU */

/* arithmetic of the pair interactions */
#define DVM_F64 0 /* FP64, reference operation order */
#define DVM_F32 1 /* FP32 pair terms with compensated / FP64 sums; FP64 state, QR,
                     refinement residual and Kelvin row */

#define DVM_EULER 0 /* Scheme::Euler, src/DVMBase.hpp:27-30 */
#define DVM_RK3 1   /* Scheme::RK3 */

#define DVM_DELETE 0  /* SurfaceCross, src/DVMBase.hpp:33-41 */
#define DVM_ABSORB 1  /* falls back to REFLECT as in src/DVMBase.cpp:111-114 */
#define DVM_REFLECT 2

#define DVM_RNG_INJECT 0 /* uniforms supplied by the host (reference mt19937 stream) */
#define DVM_RNG_PHILOX 1 /* counter-based Philox4x32-10 on the device */

/* phases of DVMBase::compute_step, for dvm_sim_phase */
#define DVM_PHASE_BIOTSAVART 0
#define DVM_PHASE_SOLVE 1
#define DVM_PHASE_SHEETBC 2
#define DVM_PHASE_CONVECT 3
#define DVM_PHASE_DIFFUSE 4
#define DVM_PHASE_RELEASE 5
#define DVM_PHASE_CROSS 6
#define DVM_PHASE_LOADS 7
#define DVM_PHASE_INCREMENT 8
#define DVM_PHASE_REFLECT 9
#define DVM_PHASE_DELETE 10

typedef struct dvm_ctx dvm_ctx; /* one device, one stream, a workspace, a table of sims */
typedef struct dvm_sim dvm_sim; /* one simulation resident in the ctx's HBM budget */

/* Same layout as dvm::VortexParticle / dvm::VelocityResult (src/VelocityKernel.hpp:15-26). */
typedef struct {
    double x, z, circ, sigma;
} dvm_particle;
typedef struct {
    double u, w;
} dvm_velocity;

/* XML parameters the hot path reads (src/XmlHandler.cpp:162-202) plus device options. */
typedef struct {
    double rho;            /* constants/density */
    double nu;             /* constants/nu */
    double dt;             /* time/dt */
    double ux, uz;         /* flow/ux, flow/uz */
    double cutoff_exp;     /* constants/cutoff_exp */
    uint32_t max_numpanelvort; /* constants/max_NumPanelVort */
    int32_t scheme;        /* DVM_EULER | DVM_RK3 */
    int32_t surface_cross; /* DVM_DELETE | DVM_ABSORB | DVM_REFLECT */
    int32_t rng;           /* DVM_RNG_INJECT | DVM_RNG_PHILOX */
    int32_t precision;     /* DVM_F64 | DVM_F32 */
    int32_t reserved;
    int64_t seed;          /* constants/seed (Philox key) */
    uint64_t capacity;     /* maximum number of blobs held on the device */
    uint64_t rng_capacity; /* inject mode: uniforms held on the device at once */
} dvm_sim_params;

int dvm_abi_version(void);
const char* dvm_status_string(int status);
const char* dvm_last_error(void);

/* ---- context ---------------------------------------------------------------- */
/* hbm_budget_bytes == 0: 90 % of the device's free memory. */
int dvm_ctx_create(int device, uint64_t hbm_budget_bytes, dvm_ctx** out);
int dvm_ctx_destroy(dvm_ctx* ctx);
int dvm_ctx_synchronize(dvm_ctx* ctx);
int dvm_ctx_memory(dvm_ctx* ctx, uint64_t* in_use, uint64_t* budget);
int dvm_ctx_device_info(dvm_ctx* ctx, int* sms, int* cc_major, int* cc_minor);
/* Kernel launches issued so far by this context (graph replays count every
 * kernel node of the graph). */
int dvm_ctx_launch_count(dvm_ctx* ctx, uint64_t* launches);
/* Per-kernel-family device time, measured with CUDA events recorded on the
 * ctx stream around each launch while profiling is on (steps then run without
 * graph capture).  dvm_ctx_profile synchronises and returns the total
 * milliseconds and the number of timed launches of one family. */
#define DVM_PROF_NBODY 0      /* self-induced pair kernel only */
#define DVM_PROF_RHS 1        /* blob-on-collocation right-hand side */
#define DVM_PROF_SOLVE 2      /* gamma = P b + refinement */
#define DVM_PROF_SHEETVEL 3   /* sheet-on-blob velocity + convection update */
#define DVM_PROF_DIFFREL 4    /* diffusion + release/append */
#define DVM_PROF_CROSS 5      /* reflect / delete */
#define DVM_PROF_LOADS 6      /* loads + step counter */
#define DVM_PROF_SORT 7       /* Morton sort, pack, partial combine */
#define DVM_PROF_STEP 8       /* whole step */
#define DVM_PROF_FAMILIES 9
/* Pre-size the shared workspace for batches of up to max_sims simulations whose
 * capacities sum to total_capacity blobs (avoids allocations, and re-captured
 * graphs, while a serving loop admits and retires simulations). */
int dvm_ctx_reserve(dvm_ctx* ctx, uint64_t total_capacity, int max_sims, int max_panels,
                    int with_delete);
int dvm_ctx_workspace_bytes(dvm_ctx* ctx, uint64_t* bytes);
/* Grow the context's stream-ordered memory pool (simulation slabs and set-up
 * scratch come from it) to hold at least `bytes`, once, so that admissions
 * carve their slabs from memory already mapped instead of growing the pool
 * one simulation at a time.  The memory stays with the pool until the ctx is
 * destroyed; it does not count against the simulations' HBM budget. */
int dvm_ctx_pool_reserve(dvm_ctx* ctx, uint64_t bytes);
/* Timing markers: dvm_ctx_mark records CUDA event `slot` (0..15) on the ctx
 * stream; dvm_ctx_elapsed synchronises and returns the device time between
 * two recorded markers. */
int dvm_ctx_mark(dvm_ctx* ctx, int slot);
int dvm_ctx_elapsed(dvm_ctx* ctx, int slot_a, int slot_b, double* ms);
int dvm_ctx_set_profiling(dvm_ctx* ctx, int on);
/* Bracket a region for an external profiler started with collection off
 * (cudaProfilerStart / cudaProfilerStop); harmless without one. */
int dvm_ctx_profiler_range(dvm_ctx* ctx, int on);
int dvm_ctx_profile(dvm_ctx* ctx, int family, double* ms_total, uint64_t* launches);
int dvm_ctx_profile_reset(dvm_ctx* ctx);
/* Bytes a simulation with these parameters and np panels occupies. */
int dvm_sim_bytes(const dvm_sim_params* p, int npanels, uint64_t* bytes);

/* ---- VelocityKernel plugin seam (host AoS in, host AoS out) ------------------------ */
int dvm_biot_savart_self(dvm_ctx* ctx, const dvm_particle* p, uint64_t n, dvm_velocity* out,
                         int precision);
int dvm_biot_savart_at(dvm_ctx* ctx, const dvm_particle* src, uint64_t ns, const double* tx,
                       const double* tz, uint64_t nt, dvm_velocity* out, int precision);
/* Device-resident SoA variants (pointers from cudaMalloc); asynchronous on the
 * ctx stream.  skip_close: 1 skips pairs with r^2 <= 1e-15 like computeInducedAt. */
int dvm_biot_savart_self_device(dvm_ctx* ctx, const double* x, const double* z,
                                const double* circ, const double* sigma, uint64_t n, double* u,
                                double* w, int precision);
int dvm_biot_savart_at_device(dvm_ctx* ctx, const double* x, const double* z, const double* circ,
                              const double* sigma, uint64_t ns, const double* tx,
                              const double* tz, uint64_t nt, double* u, double* w,
                              int precision, int skip_close);

/* Random walk of a host blob set with host uniforms R (2n values, R1 R2 per
 * blob in blob order): VortexBlobs::diffusion_random_walk,
 * src/VortexBlobs.cpp:251-265.  x and z are updated in place. */
int dvm_random_walk(dvm_ctx* ctx, double* x, double* z, uint64_t n, const double* R, double nu,
                    double dt);

/* The device's Philox4x32-10 generator (Salmon, Moraes, Dror, Shaw, SC'11), the
 * one the DVM_RNG_PHILOX walk draws from, applied to n caller blocks: counter
 * ctr[4i..4i+3] and key key[2i..2i+1] give out[4i..4i+3].  No counterpart in
 * the reference (whose walk draws from std::mt19937, src/Random.cpp:8-18); it
 * lets a caller check the generator against published known-answer vectors.
 * Host arrays; synchronous on the current device; n <= 2^26. */
int dvm_philox4x32_10(const uint32_t* ctr, const uint32_t* key, uint64_t n, uint32_t* out);

/* Velocity at targets without any device allocation.  This entry point has no
 * counterpart in the reference.  It is for callers that cannot call
 * cudaMalloc: code whose device memory is owned by a host framework's
 * allocator or memory pool (a stray allocation would fail or fragment it),
 * plug-in hosts that forbid allocation outside their own allocator, and
 * latency-critical loops that cannot afford an allocation's implicit
 * synchronisation.  It needs no dvm_ctx.  The caller passes device buffers
 * for inputs and outputs; the chunk partials live in a fixed 4 MiB array
 * inside the library, which every GPU that loads the library keeps until the
 * process exits.  Limit: ceil(ns/4096) * ceil(nt/256) * 256 <= 262080 (for
 * example ns up to 1,048,576 sources with nt up to 256 targets); larger sizes
 * are rejected with DVM_ERR_ARG.  Each call looks up that array's device
 * address on the calling thread's current device (so a device reset, which
 * may move the array, needs nothing special); the first call on a device also
 * loads the library's device code, so make it before any stream capture.
 * All calls share the one array: calls that overlap on the
 * GPU (different streams, or different host threads) race and corrupt each
 * other's results; serialise them on one stream.  Nothing needs clearing
 * between calls: every partial is written before it is read.  Asynchronous on
 * `stream` (a cudaStream_t, or NULL for the default stream).  Arguments and
 * results are those of dvm_biot_savart_at_device. */
int dvm_biot_savart_at_noalloc(const double* x, const double* z, const double* circ,
                               const double* sigma, uint64_t ns, const double* tx,
                               const double* tz, uint64_t nt, double* u, double* w,
                               int precision, int skip_close, void* stream);

/* ---- simulations ---------------------------------------------------------------- */
/* body_x/body_z: closed CCW contour of npoints (first point repeated last),
 * the reference's domain_file format (src/VortexSheet.cpp:56-76). */
int dvm_sim_create(dvm_ctx* ctx, const dvm_sim_params* p, const double* body_x,
                   const double* body_z, int npoints, dvm_sim** out);
/* n simulations created together, as n calls of dvm_sim_create would create
 * them (same set-up arithmetic, bit for bit), but the once-per-body QR
 * factorisations of their influence matrices share cooperative launches (up to
 * 8 bodies per launch) and one wait covers them all: a serving loop admitting
 * several requests at once pays for about one factorisation chain instead of n.
 * All or none: on any error no simulation is created and out[] stays NULL; an
 * argument error names the offending index.  The set-up scratch of all n
 * bodies (about 32 np^2 bytes each) is held at once and counts against the
 * budget (DVM_ERR_OOM if it does not fit); it returns to the pool before the
 * call returns.  The reference builds one body per
 * VortexSheet(xml, stamp) (src/VortexSheet.cpp:12-54,78-165). */
int dvm_sims_create(dvm_ctx* ctx, int n, const dvm_sim_params* const* p,
                    const double* const* body_x, const double* const* body_z,
                    const int* npoints, dvm_sim** out);
int dvm_sim_destroy(dvm_sim* sim);
int dvm_sim_set_blobs(dvm_sim* sim, uint64_t n, const double* x, const double* z,
                      const double* circ, const double* sigma);
/* Any output pointer may be NULL.  Fails with DVM_ERR_ARG if cap < n. */
int dvm_sim_get_blobs(dvm_sim* sim, uint64_t cap, uint64_t* n, double* x, double* z,
                      double* circ, double* sigma, double* u, double* w, double* uvs,
                      double* wvs, uint32_t* id);
int dvm_sim_num_blobs(dvm_sim* sim, uint64_t* n);
int dvm_sim_num_panels(dvm_sim* sim, int* np);
int dvm_sim_get_gamma(dvm_sim* sim, double* gamma);
int dvm_sim_set_gamma(dvm_sim* sim, const double* gamma);
int dvm_sim_get_rhs(dvm_sim* sim, double* b);             /* np+1 */
int dvm_sim_get_influence(dvm_sim* sim, double* A);       /* (np+1) x np, row-major */
int dvm_sim_get_panels(dvm_sim* sim, double* xc, double* zc, double* ds, double* theta,
                       double* enx, double* enz);
int dvm_sim_get_loads(dvm_sim* sim, double* fx, double* fz, double* cd, double* cl);
int dvm_sim_get_step(dvm_sim* sim, uint32_t* step);
int dvm_sim_set_step(dvm_sim* sim, uint32_t step);
/* Inject mode: append uniforms in (0,1) to the device stream (in draw order). */
int dvm_sim_push_uniforms(dvm_sim* sim, const double* u, uint64_t n);
int dvm_sim_rng_position(dvm_sim* sim, uint64_t* consumed_total, uint64_t* available);
/* Inject mode: drop the uniforms still held on the device. */
int dvm_sim_clear_uniforms(dvm_sim* sim);
/* Inject mode: copy out the uniforms pushed but not yet consumed (in order). */
int dvm_sim_pending_uniforms(dvm_sim* sim, double* out, uint64_t cap, uint64_t* n);
/* First error raised on the device for this simulation (synchronises). */
int dvm_sim_status(dvm_sim* sim);
int dvm_sim_clear_status(dvm_sim* sim);
int dvm_sim_phase(dvm_sim* sim, int phase);
int dvm_sim_step(dvm_sim* sim, int nsteps);
/* State dump and resume (no counterpart in the reference, whose de-facto dump is
 * the per-step text file of every blob, src/VortexBlobs.cpp:322-325, which
 * nothing reads back).  dvm_sim_save writes everything a later step depends
 * on into a host buffer of dvm_sim_state_size bytes: the parameters, the
 * contour, the blob arrays (x z circ sigma u w uvs wvs, IDs), gamma, the
 * influence matrix and its pseudo-inverse, the step counter, the status, the
 * last loads, and the random stream's position (inject mode: the uniforms
 * pushed but not consumed; Philox: the step counter is the position).
 * dvm_sim_restore rebuilds the simulation in any context from such a buffer;
 * stepping it gives the same bits as stepping the original.  Synchronous;
 * the buffer layout is this library's (native byte order, versioned). */
int dvm_sim_state_size(dvm_sim* sim, uint64_t* bytes);
int dvm_sim_save(dvm_sim* sim, void* buf, uint64_t cap, uint64_t* written);
int dvm_sim_restore(dvm_ctx* ctx, const void* buf, uint64_t size, dvm_sim** out);
/* Vortex merging, VortexBlobs::merge_blobs (src/VortexBlobs.cpp:110-209): the
 * reference's greedy merge in index order (each surviving blob absorbs every
 * later unmerged blob with |gi gj / (gi + gj)| |xi - xj| < threshold, its state
 * updated after each absorption), then merged blobs removed and IDs renumbered
 * (unchanged when nothing merged).  Bit-identical to the reference.  In place on
 * the device (dvm_sim_merge) or on host arrays of n blobs (dvm_merge_blobs; id
 * may be null); *merged = the merge count. */
int dvm_sim_merge(dvm_sim* sim, double threshold, uint64_t* merged);
int dvm_merge_blobs(dvm_ctx* ctx, double* x, double* z, double* circ, double* sigma, double* u,
                    double* w, double* uvs, double* wvs, uint32_t* id, uint64_t n,
                    double threshold, uint64_t* n_out, uint64_t* merged);
/* Remeshing (BackgroundMesh; src/DVMBase.cpp:91-92, 160-164, options
 * src/XmlHandler.cpp:191-201 -- its source is not part of the reference, the
 * behaviour follows tests/unit/test_BackgroundMesh.cpp).  Nodes x = xmin + i dx
 * (i <= (xmax - xmin) / dx), z likewise.  Every blob whose kernel support lies
 * inside the mesh spreads its circulation to the nodes with the tensor-product
 * weight W(xi - i) W(zeta - j) (node units; M4' support 2, M6 support 3,
 * Gaussian truncated at 3 and normalised per blob); nodes with |circulation| >
 * circ_threshold become the new blobs (core size sigma, row-major), followed by
 * the blobs whose support leaves the mesh, unchanged.  IDs are renumbered and
 * velocities zeroed.  Deterministic (no atomics). */
#define DVM_REMESH_M4PRIME 0
#define DVM_REMESH_M6 1
#define DVM_REMESH_GAUSSIAN 2
typedef struct {
    double xmin, xmax, zmin, zmax; /* remesh/xmin ... remesh/zmax */
    double dx, dz;                 /* remesh/dx, remesh/dz */
    double sigma;                  /* remesh/sigma: core size of the new blobs */
    double circ_threshold;         /* remesh/circ_threshold */
    int32_t kernel;                /* DVM_REMESH_* (remesh/kernel) */
    int32_t reserved;
} dvm_remesh_params;
/* Node counts of the mesh the parameters describe (at most 2^28 nodes). */
int dvm_remesh_grid(const dvm_remesh_params* p, uint32_t* nx, uint32_t* nz);
/* Remesh a simulation in place on the device; DVM_ERR_CAPACITY (state left
 * unchanged) when the new blob set exceeds its capacity.  n_out may be null. */
int dvm_sim_remesh(dvm_sim* sim, const dvm_remesh_params* p, uint64_t* n_out);
/* The same on host arrays (BackgroundMesh::remesh(VortexBlobs)): *n_out = the
 * new count; DVM_ERR_CAPACITY when it exceeds out_cap (out untouched). */
int dvm_remesh(dvm_ctx* ctx, const dvm_particle* in, uint64_t n, const dvm_remesh_params* p,
               dvm_particle* out, uint64_t out_cap, uint64_t* n_out);
/* Velocity at probe points (host arrays, n of them) from the simulation's
 * current blobs, sheet and free stream: the intended formula of
 * VortexSheet::probe_velocities (src/VortexSheet.cpp:559-646), i.e. what a
 * blob at the point would be convected with -- (1/2pi) sum over all blobs
 * (pairs with r^2 <= 1e-15 skipped, as computeInducedAt) + the sheet's
 * velocity summed over all panels + (ux, uz).  The reference's loop skips
 * blob 0 and panel 0, keeps only the last panel's term and flips a sign; those
 * slips are not reproduced.  uvs / wvs (may be null) receive the sheet part. */
int dvm_sim_probe(dvm_sim* sim, const double* px, const double* pz, uint64_t n, double* u,
                  double* w, double* uvs, double* wvs);

/* ---- batches ---------------------------------------------------------------------- */
/* Advance every listed simulation by nsteps; each kernel of the step serves all
 * of them in one launch.  use_graph != 0 captures the step in a CUDA graph
 * (re-used while the list is unchanged).  Asynchronous: check dvm_sim_status. */
int dvm_step_batch(dvm_ctx* ctx, dvm_sim* const* sims, int nsims, int nsteps, int use_graph);
/* Device status of every listed simulation with one copy and one wait (what
 * dvm_sim_status returns, per simulation, into status[i]). */
int dvm_batch_status(dvm_ctx* ctx, dvm_sim* const* sims, int nsims, int32_t* status);
/* Read back many simulations with one wait: counts[i] = blob count; x[i], z[i],
 * circ[i] (any of the three arrays, or entries, may be null) receive the first
 * counts[i] values (DVM_ERR_ARG if counts[i] > caps[i]); loads (may be null)
 * gets fx, fz, Cd, Cl per simulation.  What DVMBase::write_outputs consumes. */
int dvm_batch_get_state(dvm_ctx* ctx, dvm_sim* const* sims, int nsims, double* const* x,
                        double* const* z, double* const* circ, const uint64_t* caps,
                        uint64_t* counts, double* loads);
/* dvm_sim_push_uniforms for many simulations with one wait (u[i]: counts[i]
 * values for simulation i). */
int dvm_batch_push_uniforms(dvm_ctx* ctx, dvm_sim* const* sims, int nsims, const double* const* u,
                            const uint64_t* counts);
/* Pipelined host loops (no counterpart in the reference, whose state lives on
 * the host): these three calls let the copies of one step's inputs and results
 * cross PCIe on a second stream while the GPU computes the neighbouring step.
 * None of them waits for the GPU's compute.
 *
 * dvm_batch_push_uniforms_async: appends counts[i] uniforms from u[i] (pinned
 * host memory, left unchanged until dvm_batch_wait_state or a synchronising
 * call returns) to each simulation's injected stream; the next step enqueued
 * after the call waits for these copies.  It never compacts the stream, so
 * every simulation needs room in its rng_capacity for all uniforms pushed
 * since the last synchronous push (DVM_ERR_CAPACITY otherwise, nothing copied).
 *
 * dvm_batch_get_state_async: snapshots x, z, circ, the blob counts and the
 * loads of the listed simulations on the GPU after the work enqueued so far
 * (a device-side copy), without waiting.  One snapshot per context may be
 * pending (DVM_ERR_STATE otherwise).
 *
 * dvm_batch_wait_state: waits for the pending snapshot, copies the first
 * counts[i] values of x, z, circ of the i-th listed simulation into x[i], z[i],
 * circ[i] (pinned host memory of caps[i] values; arrays or entries may be
 * null) on the second stream -- while later enqueued steps run -- and fills
 * counts[i] and, if non-null, loads[4 i ..] (fx, fz, Cd, Cl).  nsims must
 * equal the snapshot's count. */
int dvm_batch_push_uniforms_async(dvm_ctx* ctx, dvm_sim* const* sims, int nsims,
                                  const double* const* u, const uint64_t* counts);
int dvm_batch_get_state_async(dvm_ctx* ctx, dvm_sim* const* sims, int nsims);
int dvm_batch_wait_state(dvm_ctx* ctx, int nsims, double* const* x, double* const* z,
                         double* const* circ, const uint64_t* caps, uint64_t* counts,
                         double* loads);

/* ---- pair-kernel autotuning (no counterpart in the reference) ---------------------
 * The FP32 blob-on-blob kernel's launch shape: persistent CTAs per SM and the
 * order in which simulations' work items are handed out (a work item is one
 * 256-blob sort tile of targets against one source chunk).  Neither changes a
 * result (source chunking, which would, is fixed by each simulation's capacity),
 * so tuning never changes velocities.  Shapes are kept
 * per batch-shape class (log2 of the summed capacity of the batch's FP32
 * simulations x a bucket of their count: 1, 2-8, 9-64, more); plans and graphs
 * built afterwards use them. */
typedef struct dvm_pair_config {
    int32_t tile;        /* targets per work item: 256 */
    int32_t ctas_per_sm; /* 1..4 */
    int32_t order;       /* 0: list order; 1: costliest simulations' items first */
    int32_t reserved;
} dvm_pair_config;

#define DVM_TUNE_MAX_CANDIDATES 16
typedef struct dvm_tune_result {
    dvm_pair_config best;
    int32_t shape_class;
    int32_t candidates;          /* configurations timed (dvm_tune_candidate order) */
    double best_ms;              /* mean pair-kernel time of the best */
    double default_ms;           /* mean time of the built-in shape (256, 4, 0) */
    double ms[DVM_TUNE_MAX_CANDIDATES];
} dvm_tune_result;

/* The search space, enumerated: index 0 .. count-1; DVM_ERR_ARG past the end. */
int dvm_tune_candidate(int index, dvm_pair_config* out);
/* Time every candidate on this batch's FP32 simulations (reps launches each,
 * after one untimed launch) and store the fastest for the
 * batch's class.  Simulation state is not modified (the pair kernel writes only
 * workspace partials; the next step recomputes velocities).  Synchronous: meant
 * for set-up (or once per class in a long-running server), not per step. */
int dvm_ctx_autotune(dvm_ctx* ctx, dvm_sim* const* sims, int nsims, int reps,
                     dvm_tune_result* out);
/* Class of a batch (-1: no FP32 simulation in it). */
int dvm_batch_shape_class(dvm_ctx* ctx, dvm_sim* const* sims, int nsims, int* shape_class);
/* Set / read the shape for one class; shape_class -1 sets the default for every
 * class and clears the table.  Setting drops cached plans and graphs. */
int dvm_ctx_set_pair_config(dvm_ctx* ctx, int shape_class, const dvm_pair_config* cfg);
int dvm_ctx_get_pair_config(dvm_ctx* ctx, int shape_class, dvm_pair_config* out);
/* The tuned classes (up to max_entries of them; *count = how many there are), so
 * a host can persist a table and restore it with dvm_ctx_set_pair_config. */
int dvm_ctx_tuning_table(dvm_ctx* ctx, int max_entries, int* shape_classes,
                         dvm_pair_config* cfgs, int* count);

/* ---- serving (no counterpart in the reference) ----------------------------------------
 * A request loop over one context: requests (a body, parameters and a step
 * count) arrive at given times; each is admitted as soon as it has arrived,
 * a batch slot is free and its slab fits the HBM budget (FIFO, no overtaking);
 * every tick advances ALL admitted simulations by one step in one batched
 * launch sequence (continuous batching: new requests join while others run);
 * finished ones are retired immediately and free their memory.  `serial`
 * runs the same requests one at a time (the plain GPU path) for comparison.
 * `realtime` != 0 honours arrival times on the wall clock; 0 treats every
 * request as arrived when it was submitted (t = 0 for requests submitted
 * before the run).
 *
 * Requests may be submitted from other host threads while dvm_server_run
 * works: the loop takes them in at its next tick.  Such a live request
 * arrives at its submission time on the run's clock (or at arrival_s, if that
 * is later); its latency counts from then.  The run returns once every
 * submitted request has finished -- or, with DVM_SERVE_LIVE set, only after
 * dvm_server_close_intake has been called and everything submitted before it
 * has finished (an idle live server waits for submissions).  Submissions after
 * the close, or after the run returned, fail with DVM_ERR_STATE.
 * dvm_server_result may be read at any time (finished_s < 0 until the request
 * finishes). */
typedef struct dvm_server dvm_server;
typedef struct {
    uint64_t id;
    double arrival_s, admitted_s, finished_s; /* seconds since the run started */
    double latency_s;                         /* finished - arrival */
    uint32_t steps_done;
    int32_t status;                           /* DVM_OK or the simulation's error */
    uint64_t blobs;                           /* blob count at the end */
    double fx, fz, cd, cl;                    /* last loads */
} dvm_request_result;
typedef struct {
    uint64_t requests, completed, failed, sim_steps, ticks;
    double wall_s, sim_steps_per_s;
    double latency_p50_s, latency_p95_s, latency_p99_s, latency_mean_s;
    double queue_p50_s, queue_p99_s;
    uint32_t peak_active;
    uint64_t peak_bytes;
    /* host wall time spent admitting (simulation set-up, incl. the QR), issuing
     * and waiting for ticks, and retiring (results read back); tunings run */
    double admit_s, step_s, retire_s;
    uint32_t tunings;
} dvm_server_summary;

/* hbm_budget_bytes: device memory the server's simulations may hold (0: the
 * context budget minus its workspace).  max_active: batch size limit.
 * keep_state != 0 keeps every request's final x, z, circ on the host. */
int dvm_server_create(dvm_ctx* ctx, uint64_t hbm_budget_bytes, int max_active, int keep_state,
                      dvm_server** out);
int dvm_server_destroy(dvm_server* srv);
/* Options (before dvm_server_run): DVM_SERVE_GRAPH 1 captures the step in a CUDA
 * graph, re-used while the batch is unchanged (default 1); DVM_SERVE_SYNC 1
 * waits for each tick before the next admission (default 1; 0 lets the host
 * run ahead and reads device status only at retirement); DVM_SERVE_AUTOTUNE 1
 * runs dvm_ctx_autotune (one launch per candidate) the first time a batch of a
 * new shape class is stepped (default 0). */
#define DVM_SERVE_GRAPH 0
#define DVM_SERVE_SYNC 1
#define DVM_SERVE_AUTOTUNE 2
#define DVM_SERVE_LIVE 3 /* 1: keep running for live submissions until the intake closes */
int dvm_server_set_option(dvm_server* srv, int option, int value);
/* arrival_s < 0: arrives at submission (t = 0 before the run). */
int dvm_server_submit(dvm_server* srv, const dvm_sim_params* p, const double* body_x,
                      const double* body_z, int npoints, uint32_t steps, double arrival_s,
                      uint64_t* id);
int dvm_server_run(dvm_server* srv, int serial, int realtime);
/* No more submissions: a live run returns once what was submitted is done. */
int dvm_server_close_intake(dvm_server* srv);
int dvm_server_result(dvm_server* srv, uint64_t id, dvm_request_result* out);
int dvm_server_final_blobs(dvm_server* srv, uint64_t id, uint64_t cap, uint64_t* n, double* x,
                           double* z, double* circ);
int dvm_server_stats(dvm_server* srv, dvm_server_summary* out);

#ifdef __cplusplus
}
#endif
#endif /* DVM_CUDA_H */
