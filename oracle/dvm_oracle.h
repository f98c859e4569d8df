/* CPU restatement of the DVMpp per-step hot path (FP64, OpenMP).
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA path is checked
 * against; it is loaded only by tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py.  The product library
 * (dvmpp_b200/) never links or calls it.
 *
 * Each function cites the reference line range (gdeskos/DVMpp) it restates and
 * keeps that code's operation order, so that with FP contraction disabled the
 * results are bit-identical to the reference sources compiled the same way
 * (oracle/_ref/libdvmref.so).  Arrays are plain SoA doubles.
 */
#ifndef DVM_ORACLE_H
#define DVM_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* src/VelocityKernel.cpp:30-67 — self-induced velocity, self skipped by index. */
void or_direct_self(const double* x, const double* z, const double* circ, const double* sigma,
                    size_t n, double* u, double* w);
/* src/VelocityKernel.cpp:69-109 — velocity at targets, pairs with r^2 <= 1e-15 skipped. */
void or_direct_at(const double* x, const double* z, const double* circ, const double* sigma,
                  size_t ns, const double* tx, const double* tz, size_t nt, double* u, double* w);

/* src/VortexSheet.cpp:78-102 — panels from a closed contour of np+1 points. */
void or_sheet_geometry(const double* xp, const double* zp, int np, double* xc, double* zc,
                       double* ds, double* theta, double* enx, double* enz, double* etx,
                       double* etz);
/* src/VortexSheet.cpp:104-165 — (np+1) x np influence matrix, column-major. */
void or_influence_matrix(const double* xp, const double* zp, const double* xc, const double* zc,
                         const double* ds, const double* theta, int np, double* A);
/* src/VortexSheet.cpp:167-211 — right-hand side b (np+1 entries). */
void or_sheet_rhs(const double* xc, const double* zc, const double* enx, const double* enz, int np,
                  double Ux, double Uz, const double* x, const double* z, const double* circ,
                  const double* sigma, size_t n, double* b);
/* src/VortexSheet.cpp:214 — gamma = solve(A^T A, A^T b) by LU with partial pivoting. */
int or_sheet_solve(const double* A, const double* b, int np, double* gamma);
/* src/VortexSheet.cpp:217-273 — sheet-induced velocity at the blobs. */
void or_sheet_on_blobs(const double* xc, const double* zc, const double* theta, const double* ds,
                       const double* gamma, int np, const double* x, const double* z, size_t n,
                       double* uvs, double* wvs);
/* src/VortexBlobs.cpp:251-265 — random walk with uniforms R[2i], R[2i+1]. */
void or_diffuse(double* x, double* z, size_t n, const double* R, double nu, double dt);
/* src/VortexSheet.cpp:282-297 — per-panel release counts; returns Nrv, or -1 when
 * the reference throws (a count not > 1e-15). */
long or_release_counts(const double* gamma, const double* ds, int np, unsigned M, double* counts,
                       double* circ_new);
/* src/VortexSheet.cpp:299-333 — positions of the nascent blobs (R: Nrv uniforms). */
void or_release_place(const double* xp, const double* zp, const double* ds, const double* etx,
                      const double* etz, const double* enx, const double* enz, int np,
                      const double* counts, const double* circ_new, double nu, double dt,
                      double cutoff_exp, const double* R, double* x, double* z, double* circ,
                      double* sigma);
/* src/VortexSheet.cpp:447-464 — crossing number == 1. */
int or_inside(const double* xp, const double* zp, int np, double x, double z);
/* src/VortexBlobs.cpp:110-209 — greedy pairwise merge in index order (each
 * surviving i absorbs, one after another, every later unmerged j with
 * |gi gj / (gi + gj)| |xi - xj| < threshold, using i's updated state), then a
 * stable compaction with IDs renumbered.  In place on the 8 SoA arrays + ids;
 * returns the merge count, the new length in *n_out. */
unsigned or_merge_blobs(double* x, double* z, double* circ, double* sigma, double* u, double* w,
                        double* uvs, double* wvs, unsigned* id, size_t n, double threshold,
                        size_t* n_out);
/* Remeshing (BackgroundMesh: source absent from the reference; behaviour from
 * tests/unit/test_BackgroundMesh.cpp and options src/XmlHandler.cpp:191-201).
 * kernel 0 M4', 1 M6, 2 Gaussian truncated at 3 (normalised per blob).  Nodes
 * x0 + i dx, i < nx; z likewise.  Each node sums, in a fixed order (cells
 * around it row-major, blobs in index order within a cell), W(xi-i) W(ze-j)
 * circ of the blobs whose support lies inside the mesh; nodes with |sum| >
 * threshold become blobs (row-major), then the other blobs follow unchanged.
 * Writes at most cap blobs; returns the total count. */
size_t or_remesh(const double* x, const double* z, const double* circ, const double* sigma,
                 size_t n, double x0, double z0, double dx, double dz, int nx, int nz, int kernel,
                 double new_sigma, double threshold, double* ox, double* oz, double* oc,
                 double* os, size_t cap);
/* src/VortexSheet.cpp:345-405 — reflect inside blobs; returns how many moved. */
size_t or_reflect(const double* xp, const double* zp, const double* enx, const double* enz, int np,
                  double* x, double* z, size_t n);
/* src/VortexSheet.cpp:407-445 — keep flags (1 = outside = kept); returns kept count. */
size_t or_keep_flags(const double* xp, const double* zp, int np, const double* x, const double* z,
                     size_t n, uint8_t* keep);
/* src/VortexSheet.cpp:487-514 — pressure loads. */
void or_loads(const double* gamma, const double* ds, const double* enx, const double* enz, int np,
              double rho, double dt, double Ur, double* fx, double* fz);

/* src/Random.cpp: std::mt19937 + uniform_real_distribution<double> in [0,1)
 * (MT19937 of Matsumoto & Nishimura 1998; generate_canonical per the C++
 * standard [rand.util.canonical] with 2 draws of 32 bits). */
typedef struct { uint32_t mt[624]; int idx; } or_mt19937;
void or_mt_seed(or_mt19937* g, uint32_t seed);
double or_mt_uniform(or_mt19937* g);
void or_mt_stream(uint32_t seed, size_t n, double* out);

/* A whole simulation (src/DVMBase.cpp), state in growable arrays. */
typedef struct or_sim or_sim;
typedef struct {
    double rho, nu, dt, ux, uz, cutoff_exp;
    unsigned max_numpanelvort;
    int scheme;        /* 0 euler, 1 RK3 */
    int surface_cross; /* 0 DELETE, 1 ABSORB, 2 REFLECT */
    int seed;
} or_params;
or_sim* or_sim_create(const or_params* p, const double* xp, const double* zp, int npts);
void or_sim_destroy(or_sim* s);
/* Replace the blob set (IDs 0..n-1, velocities zero). */
void or_sim_set_blobs(or_sim* s, size_t n, const double* x, const double* z, const double* circ,
                      const double* sigma);
/* src/DVMBase.cpp:86-133 (+ increment_step :145-149).  Returns 0, or 1 when
 * the release throws. */
int or_sim_step(or_sim* s);
/* Phases, same numbering as oracle/ref_driver.cpp ref_sim_phase. */
int or_sim_phase(or_sim* s, int phase);
size_t or_sim_nblobs(const or_sim* s);
int or_sim_npanels(const or_sim* s);
void or_sim_get_blobs(const or_sim* s, double* x, double* z, double* circ, double* sigma,
                      double* u, double* w, double* uvs, double* wvs, unsigned* id);
void or_sim_get_sheet(const or_sim* s, double* gamma);
void or_sim_get_forces(const or_sim* s, double* fx, double* fz, double* area);
const double* or_sim_infm(const or_sim* s);

#ifdef __cplusplus
}
#endif
#endif
