// Bookkeeping kernels of the step: random-walk diffusion
// (src/VortexBlobs.cpp:251-265), nascent-vortex release + append
// (src/VortexSheet.cpp:275-333, src/VortexBlobs.cpp:211-227) and surface
// crossing (src/VortexSheet.cpp:345-464, dispatch src/DVMBase.cpp:107-118).
//
// These are HBM-bound integer/byte work around FP64 positions.  Counts are
// exact: release counts come from the same FP64 arithmetic as the reference,
// the inside test is the reference's crossing-number test with one rounding
// per operation, and DELETE is a stable (order-preserving) compaction.
#include <cfloat>

#include <cub/cub.cuh>

#include "dvm_device.cuh"
#include "dvm_internal.h"

namespace dvmk {
namespace {

__device__ __forceinline__ void raise_status(InstState& s, int code) {
    atomicCAS(&s.status, 0, code);
}

// ---- diffusion -------------------------------------------------------------------
// One flat index space over the blobs of every simulation in the list, so the
// grid's threads get equal shares whatever the sizes (a simulation of 4e5 blobs
// beside ones of 1e4).  A failed simulation, or one whose injected stream cannot
// cover this step, contributes no blobs; block 0 flags the exhausted stream.
__device__ __forceinline__ int locate64(const uint64_t* pre, int nlist, uint64_t g) {
    int lo = 0, hi = nlist - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void k_diffuse(const InstDesc* __restrict__ table, InstState* __restrict__ st,
                          const ListEntry* __restrict__ list, int nlist) {
    __shared__ uint64_t s_pre[kMaxBatch + 1];
    const int tid = threadIdx.x;
    for (int k = tid; k < nlist; k += blockDim.x) {
        const int inst = list[k].inst;
        InstState& S = st[inst];
        uint32_t n = S.status ? 0u : S.n;
        if (n && table[inst].rng == kInject && S.cursor + 2ull * n > table[inst].ucount) {
            if (blockIdx.x == 0) raise_status(S, kErrRngExhausted);
            n = 0;
        }
        s_pre[k + 1] = n;
    }
    __syncthreads();
    if (tid < 32) {  // inclusive scan of the counts, 32 simulations per pass
        uint64_t carry = 0;
        for (int b = 0; b < nlist; b += 32) {
            const int k = b + tid;
            uint64_t v = k < nlist ? s_pre[k + 1] : 0ull;
            for (int o = 1; o < 32; o <<= 1) {
                const uint64_t t = __shfl_up_sync(0xffffffffu, v, o);
                if (tid >= o) v += t;
            }
            if (k < nlist) s_pre[k + 1] = v + carry;
            carry += __shfl_sync(0xffffffffu, v, 31);
        }
        if (tid == 0) s_pre[0] = 0;
    }
    __syncthreads();
    const uint64_t total = s_pre[nlist];
    const double twopi = dmul(2.0, kPi);
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + tid; g < total;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const int k = locate64(s_pre, nlist, g);
        const uint32_t i = (uint32_t)(g - s_pre[k]);
        const int inst = list[k].inst;
        const InstDesc& d = table[inst];
        const InstState& S = st[inst];
        const double c4 = dmul(dmul(4.0, d.nu), d.dt);
        double R1, R2;
        if (d.rng == kInject) {
            const uint64_t cur = S.cursor;
            R1 = d.uniforms[cur + 2ull * i];
            R2 = d.uniforms[cur + 2ull * i + 1];
        } else {
            philox_uniform2(d.seed, i, S.step, d.uid, 0u, R1, R2);
        }
        const double rrw = sqrt(dmul(c4, log(ddiv(1.0, R1))));
        const double th = dmul(twopi, R2);
        d.x[i] = dadd(d.x[i], dmul(rrw, cos(th)));
        d.z[i] = dadd(d.z[i], dmul(rrw, sin(th)));
    }
}

// The same walk on caller buffers with caller uniforms R[2i], R[2i+1].
__global__ void k_diffuse_raw(double* __restrict__ x, double* __restrict__ z, uint32_t n,
                              const double* __restrict__ R, double nu, double dt) {
    const double c4 = dmul(dmul(4.0, nu), dt);
    const double twopi = dmul(2.0, kPi);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double rrw = sqrt(dmul(c4, log(ddiv(1.0, R[2ull * i]))));
        const double th = dmul(twopi, R[2ull * i + 1]);
        x[i] = dadd(x[i], dmul(rrw, cos(th)));
        z[i] = dadd(z[i], dmul(rrw, sin(th)));
    }
}

// ---- release + append: one block per simulation -------------------------------------
constexpr int kRelThreads = 256;

__global__ void __launch_bounds__(kRelThreads) k_release(const InstDesc* __restrict__ table,
                                                         InstState* __restrict__ st,
                                                         const ListEntry* __restrict__ list) {
    extern __shared__ double s_dyn[];  // counts[np] | circ_new[np]
    __shared__ double s_red[kRelThreads / 32];
    __shared__ uint32_t s_part[kRelThreads + 1];
    __shared__ int s_bad;
    const ListEntry e = list[blockIdx.x];
    const InstDesc& d = table[e.inst];
    InstState& S = st[e.inst];
    if (S.status) return;
    const int np = d.np;
    double* cnt = s_dyn;
    double* cnew = s_dyn + np;
    const int tid = threadIdx.x;
    if (tid == 0) s_bad = 0;
    // Signed maximum of the panel circulations (src/VortexSheet.cpp:282-285).
    double mx = -DBL_MAX;
    for (int j = tid; j < np; j += kRelThreads) mx = fmax(mx, dmul(d.gamma[j], d.ds[j]));
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((tid & 31) == 0) s_red[tid >> 5] = mx;
    __syncthreads();
    mx = s_red[0];
    for (int q = 1; q < kRelThreads / 32; ++q) mx = fmax(mx, s_red[q]);
    // Arma's max: NaN elements never replace the running maximum; fmax skips
    // NaN the same way, and a NaN in any count is caught below as in :289.
    const double Md = (double)d.M;
    // Contiguous panel ranges per thread so the scan below is in panel order.
    const int per = (np + kRelThreads - 1) / kRelThreads;
    const int jb = tid * per, je = min(np, jb + per);
    uint32_t mine = 0;
    for (int j = jb; j < je; ++j) {
        const double pc = dmul(d.gamma[j], d.ds[j]);
        const double c = dadd(floor(fabs(dmul(ddiv(pc, mx), Md))), 1.0);
        cnt[j] = c;
        cnew[j] = ddiv(pc, c);
        if (!(c > 1.0e-15)) s_bad = 1;
        else mine += (uint32_t)c;
    }
    s_part[tid] = mine;
    __syncthreads();
    if (tid == 0) {
        uint32_t acc = 0;
        for (int t = 0; t < kRelThreads; ++t) {
            const uint32_t v = s_part[t];
            s_part[t] = acc;
            acc += v;
        }
        s_part[kRelThreads] = acc;
    }
    __syncthreads();
    if (s_bad) {  // the reference throws VortexException (src/VortexSheet.cpp:289-291)
        if (tid == 0) raise_status(S, kErrRelease);
        return;
    }
    const uint32_t n0 = S.n;
    const uint32_t nrv = s_part[kRelThreads];
    const uint64_t cur = S.cursor;
    if ((uint64_t)n0 + nrv > d.cap) {
        if (tid == 0) raise_status(S, kErrCapacity);
        return;
    }
    if (d.rng == kInject && cur + 2ull * n0 + nrv > d.ucount) {
        if (tid == 0) raise_status(S, kErrRngExhausted);
        return;
    }
    const double c4 = dmul(dmul(4.0, d.nu), d.dt);
    uint32_t o = n0 + s_part[tid];
    for (int j = jb; j < je; ++j) {
        const uint32_t c = (uint32_t)cnt[j];
        const double xm = dadd(d.xp[j], ddiv(dmul(d.ds[j], d.etx[j]), dadd(cnt[j], 1.0)));
        const double zm = dadd(d.zp[j], ddiv(dmul(d.ds[j], d.etz[j]), dadd(cnt[j], 1.0)));
        for (uint32_t q = 0; q < c; ++q, ++o) {
            const uint32_t r = o - n0;  // release index, panel order
            double R;
            if (d.rng == kInject) {
                R = d.uniforms[cur + 2ull * n0 + r];
            } else {
                double R2;
                philox_uniform2(d.seed, r, S.step, d.uid, 1u, R, R2);
            }
            const double rrw = fabs(sqrt(dmul(c4, log(ddiv(1.0, R)))));
            d.x[o] = dadd(xm, dmul(rrw, d.enx[j]));
            d.z[o] = dadd(zm, dmul(rrw, d.enz[j]));
            d.circ[o] = cnew[j];
            d.sigma[o] = d.psigma[j];
            d.u[o] = 0.0;
            d.w[o] = 0.0;
            d.uvs[o] = 0.0;
            d.wvs[o] = 0.0;
            d.id[o] = n0;  // nascent IDs are 0, shifted by Nold (src/VortexBlobs.cpp:215-217)
        }
    }
    __syncthreads();
    if (tid == 0) {
        S.n = n0 + nrv;
        if (d.rng == kInject) S.cursor = cur + 2ull * n0 + nrv;
    }
}

// ---- crossing test ----------------------------------------------------------------
struct Body {
    const double* xp;
    const double* zp;
    int np;
};

// Crossing-number test, cn == 1 (src/VortexSheet.cpp:447-464), with the 32
// lanes of a warp sharing one point's edges (every lane passes the same point;
// the crossing count is an integer sum, so the result is the sequential
// loop's).  Points outside the contour's z-range or x-range cross no edge or an
// even number of them, so the bounding box settles them.
__device__ __forceinline__ bool in_bbox(const InstDesc& d, double xc, double zc) {
    return !(zc < d.bzmin || zc >= d.bzmax || xc > d.bxmax || xc < d.bxmin);
}

__device__ __forceinline__ bool inside_body_warp(const double* __restrict__ xp,
                                                 const double* __restrict__ zp, int np,
                                                 double xc, double zc) {
    int cn = 0;
    for (int i = threadIdx.x & 31; i < np; i += 32) {
        const double z0 = zp[i], z1 = zp[i + 1];
        if (((z0 <= zc) && (z1 > zc)) || ((z0 > zc) && (z1 <= zc))) {
            const double vt = ddiv(dsub(zc, z0), dsub(z1, z0));
            if (xc < dadd(xp[i], dmul(vt, dsub(xp[i + 1], xp[i])))) ++cn;
        }
    }
    return __reduce_add_sync(0xffffffffu, (unsigned)cn) == 1u;
}

__device__ __forceinline__ void load_contour(const InstDesc& d, double* sx, double* sz,
                                             double* snx, double* snz) {
    for (int j = threadIdx.x; j <= d.np; j += blockDim.x) {
        sx[j] = d.xp[j];
        sz[j] = d.zp[j];
        if (j < d.np) {
            snx[j] = d.enx[j];
            snz[j] = d.enz[j];
        }
    }
}

// REFLECT / ABSORB (src/VortexSheet.cpp:345-405): each blob moves independently.
__global__ void __launch_bounds__(256) k_reflect(const InstDesc* __restrict__ table,
                                                 const InstState* __restrict__ st,
                                                 const ListEntry* __restrict__ list, int nlist,
                                                 unsigned* __restrict__ work) {
    extern __shared__ double s_c[];
    __shared__ unsigned s_pre[1025];
    __shared__ unsigned s_item;
    __shared__ int s_loaded;
    if (threadIdx.x == 0) {
        unsigned acc = 0;
        for (int k = 0; k < nlist; ++k) {
            s_pre[k] = acc;
            acc += st[list[k].inst].status ? 0u : (st[list[k].inst].n + 255) / 256;
        }
        s_pre[nlist] = acc;
        s_loaded = -1;
    }
    __syncthreads();
    const unsigned total = s_pre[nlist];
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(work, 1u);
        __syncthreads();
        const unsigned item = s_item;
        if (item >= total) break;
        const int k = locate(s_pre, nlist, item);
        const ListEntry e = list[k];
        const InstDesc& d = table[e.inst];
        const int np = d.np;
        double* sx = s_c;
        double* sz = sx + (np + 1);
        double* snx = sz + (np + 1);
        double* snz = snx + np;
        if (s_loaded != k) load_contour(d, sx, sz, snx, snz);
        __syncthreads();
        if (threadIdx.x == 0) s_loaded = k;
        const uint32_t n = st[e.inst].n;
        const uint32_t i = (item - s_pre[k]) * 256 + threadIdx.x;
        const bool valid = i < n;
        const double px = valid ? d.x[i] : 0.0, pz = valid ? d.z[i] : 0.0;
        // blobs in the contour's bounding box, handled one at a time by the
        // whole warp (edges and panels split over the lanes)
        unsigned cand = __ballot_sync(0xffffffffu, valid && in_bbox(d, px, pz));
        const int lane = threadIdx.x & 31;
        while (cand) {
            const int src = __ffs(cand) - 1;
            cand &= cand - 1;
            const double qx = __shfl_sync(0xffffffffu, px, src);
            const double qz = __shfl_sync(0xffffffffu, pz, src);
            if (!inside_body_warp(sx, sz, np, qx, qz)) continue;
            // nearest panel: the first minimum of the clamped point-segment
            // distance (src/VortexSheet.cpp:378-390), per lane over its
            // panels in order, then the least (distance, panel) over the warp
            int cp = 0;
            double md = 1e10;
            for (int j = lane; j < np; j += 32) {
                const double x0 = sx[j], z0 = sz[j], x1 = sx[j + 1], z1 = sz[j + 1];
                const double vx = dsub(qx, x0), vz = dsub(qz, z0);
                const double dx = dsub(x1, x0), dz = dsub(z1, z0);
                const double len = dadd(dmul(dx, dx), dmul(dz, dz));
                double t = ddiv(dadd(dmul(vx, dx), dmul(vz, dz)), len);
                t = (t < 1.0) ? t : 1.0;  // std::min(1.0, t)
                t = (0.0 < t) ? t : 0.0;  // std::max(0.0, .)
                const double cx = dadd(x0, dmul(t, dx)), cz = dadd(z0, dmul(t, dz));
                const double ex = dsub(qx, cx), ez = dsub(qz, cz);
                const double dist = sqrt(dadd(dmul(ex, ex), dmul(ez, ez)));
                if (dist < md) {
                    md = dist;
                    cp = j;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double m2 = __shfl_xor_sync(0xffffffffu, md, o);
                const int c2 = __shfl_xor_sync(0xffffffffu, cp, o);
                if (m2 < md || (m2 == md && c2 < cp)) {
                    md = m2;
                    cp = c2;
                }
            }
            const double off = dadd(dmul(2.0, md), 1e-6);
            double nx = dadd(qx, dmul(off, snx[cp]));
            double nz = dadd(qz, dmul(off, snz[cp]));
            if (inside_body_warp(sx, sz, np, nx, nz)) {
                nx = dadd(qx, dmul(dmul(3.0, off), snx[cp]));
                nz = dadd(qz, dmul(dmul(3.0, off), snz[cp]));
            }
            if (lane == src) {
                d.x[i] = nx;
                d.z[i] = nz;
            }
        }
        __syncthreads();
    }
}

// DELETE (src/VortexSheet.cpp:407-445): keep flags and kept count per 1024-tile.
constexpr int kDelTile = 1024;

__global__ void __launch_bounds__(256) k_del_flags(const InstDesc* __restrict__ table,
                                                   const InstState* __restrict__ st,
                                                   const ListEntry* __restrict__ list,
                                                   uint8_t* __restrict__ flags,
                                                   uint32_t* __restrict__ tile_counts) {
    extern __shared__ double s_c[];
    __shared__ uint32_t s_cnt;
    const ListEntry e = list[blockIdx.y];
    const InstDesc& d = table[e.inst];
    const InstState& S = st[e.inst];
    const uint32_t n = S.n;
    const uint32_t ntiles = (n + kDelTile - 1) / kDelTile;
    if (S.status) return;
    double* sx = s_c;
    double* sz = sx + (d.np + 1);
    double* snx = sz + (d.np + 1);
    double* snz = snx + d.np;
    load_contour(d, sx, sz, snx, snz);
    __syncthreads();
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        if (threadIdx.x == 0) s_cnt = 0;
        __syncthreads();
        uint32_t mine = 0;
        for (uint32_t q = threadIdx.x; q < kDelTile; q += blockDim.x) {  // uniform trip count
            const uint32_t i = t * kDelTile + q;
            const bool valid = i < n;
            const double px = valid ? d.x[i] : 0.0, pz = valid ? d.z[i] : 0.0;
            // bounding-box candidates, tested by the whole warp one at a time
            unsigned cand = __ballot_sync(0xffffffffu, valid && in_bbox(d, px, pz));
            bool inside = false;
            while (cand) {
                const int src = __ffs(cand) - 1;
                cand &= cand - 1;
                const bool in = inside_body_warp(sx, sz, d.np, __shfl_sync(0xffffffffu, px, src),
                                                 __shfl_sync(0xffffffffu, pz, src));
                if ((threadIdx.x & 31) == src) inside = in;
            }
            if (valid) {
                const uint8_t keep = inside ? 0 : 1;
                flags[e.coff + i] = keep;
                mine += keep;
            }
        }
        for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&s_cnt, mine);
        __syncthreads();
        if (threadIdx.x == 0) tile_counts[e.coff / kDelTile + t] = s_cnt;
        __syncthreads();
    }
}

// Per simulation (one block each): exclusive prefix of the kept counts of its
// 1024-tiles, and the total kept.
__global__ void __launch_bounds__(1024) k_del_scan(const InstState* __restrict__ st,
                                                   const ListEntry* __restrict__ list,
                                                   const uint32_t* __restrict__ tile_counts,
                                                   uint32_t* __restrict__ tile_base,
                                                   uint32_t* __restrict__ del_kept) {
    using Scan = cub::BlockScan<uint32_t, 1024>;
    __shared__ typename Scan::TempStorage tmp;
    const ListEntry e = list[blockIdx.x];
    const InstState& S = st[e.inst];
    if (S.status) {  // a failed simulation deletes nothing (k_del_move skips it)
        if (threadIdx.x == 0) del_kept[blockIdx.x] = S.n;
        return;
    }
    const uint32_t ntiles = (S.n + kDelTile - 1) / kDelTile;
    const uint32_t* tc = tile_counts + e.coff / kDelTile;
    uint32_t* tb = tile_base + e.coff / kDelTile;
    uint32_t carry = 0;
    for (uint32_t c0 = 0; c0 < ntiles; c0 += 1024) {
        const uint32_t t = c0 + threadIdx.x;
        uint32_t v = t < ntiles ? tc[t] : 0u, ex = 0, agg = 0;
        Scan(tmp).ExclusiveSum(v, ex, agg);
        if (t < ntiles) tb[t] = carry + ex;
        carry += agg;
        __syncthreads();
    }
    if (threadIdx.x == 0) del_kept[blockIdx.x] = carry;
}

// Stable in-place compaction of the kept blobs (all eight FP64 arrays; IDs
// renumbered 0..k-1, src/VortexSheet.cpp:424-437).  A kept blob moves down by
// the number of deleted blobs before it, so tile t (kDelTile blobs) writes its
// kept blobs to [base_t, base_t + kept_t), a range that starts inside tile
// floor(base_t / kDelTile) <= t.  Each block takes tiles in ticket order (one
// counter over the whole list, tiles of a simulation in increasing order),
// loads its kept blobs into registers, publishes that its tile has been read,
// and writes only after every lower tile its destination range overlaps has
// published the same -- so no blob is overwritten before it has been read,
// with no staging copy.  A tile waits only for tiles of lower tickets, which
// blocks that are already running hold, so the waits always end; they are
// bounded all the same, and a wait that runs out stops the simulation with
// kErrTimeout instead of writing.  Tiles that do not move (no deletion at or
// before them) only renumber their IDs.
constexpr uint32_t kDelSpinLimit = 1u << 22;  // x ~100 ns: well under a second

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__global__ void __launch_bounds__(kDelTile) k_del_move(const InstDesc* __restrict__ table,
                                                       InstState* __restrict__ st,
                                                       const ListEntry* __restrict__ list,
                                                       int nlist,
                                                       const uint8_t* __restrict__ flags,
                                                       const uint32_t* __restrict__ tile_base,
                                                       const uint32_t* __restrict__ del_kept,
                                                       uint32_t* __restrict__ ready,
                                                       unsigned* __restrict__ ticket) {
    __shared__ unsigned s_pre[1025];
    __shared__ uint32_t s_warp[kDelTile / 32];
    __shared__ unsigned s_item;
    __shared__ int s_ok;
    if (threadIdx.x == 0) {  // tiles of each listed simulation that deletes something
        // (from values no block of this launch changes, so every block agrees
        // on which tile a ticket names)
        unsigned acc = 0;
        for (int k = 0; k < nlist; ++k) {
            s_pre[k] = acc;
            const uint32_t n = st[list[k].inst].n;
            if (del_kept[k] != n) acc += (n + kDelTile - 1) / kDelTile;
        }
        s_pre[nlist] = acc;
    }
    __syncthreads();
    const unsigned total = s_pre[nlist];
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(ticket, 1u);
        __syncthreads();
        const unsigned item = s_item;
        if (item >= total) break;
        const int k = locate(s_pre, nlist, item);
        const ListEntry e = list[k];
        const InstDesc& d = table[e.inst];
        const uint32_t n = st[e.inst].n;
        const uint32_t t = item - s_pre[k];
        const uint32_t tile0 = (uint32_t)(e.coff / kDelTile);
        const uint32_t base = tile_base[tile0 + t];
        const uint32_t i = t * kDelTile + threadIdx.x;
        const bool keep = i < n && flags[e.coff + i] != 0;
        const uint32_t ball = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) s_warp[wid] = __popc(ball);
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t acc = 0;
            for (int q = 0; q < kDelTile / 32; ++q) {
                const uint32_t v = s_warp[q];
                s_warp[q] = acc;
                acc += v;
            }
        }
        __syncthreads();
        const uint32_t o = base + s_warp[wid] + __popc(ball & ((1u << lane) - 1u));
        // unmoved: nothing deleted before this tile nor inside it
        const bool moves = __syncthreads_or(keep && o != i);
        double v[8];
        if (moves && keep) {
            v[0] = d.x[i];
            v[1] = d.z[i];
            v[2] = d.circ[i];
            v[3] = d.sigma[i];
            v[4] = d.u[i];
            v[5] = d.w[i];
            v[6] = d.uvs[i];
            v[7] = d.wvs[i];
        }
        __syncthreads();  // every source of this tile is in registers
        if (threadIdx.x == 0) {
            __threadfence();
            st_release(&ready[tile0 + t], 1u);
            int ok = 1;
            if (moves)  // lower tiles the destination range overlaps must be read first
                for (uint32_t u = base / kDelTile; u < t && ok; ++u) {
                    uint32_t it = 0;
                    while (!ld_acquire(&ready[tile0 + u])) {
                        if (++it >= kDelSpinLimit) {
                            ok = 0;
                            raise_status(st[e.inst], kErrTimeout);
                            break;
                        }
                        __nanosleep(100);
                    }
                }
            s_ok = ok;
        }
        __syncthreads();
        if (s_ok && keep) {
            if (moves) {
                d.x[o] = v[0];
                d.z[o] = v[1];
                d.circ[o] = v[2];
                d.sigma[o] = v[3];
                d.u[o] = v[4];
                d.w[o] = v[5];
                d.uvs[o] = v[6];
                d.wvs[o] = v[7];
            }
            d.id[o] = o;  // IDs renumbered 0..k-1 (src/VortexSheet.cpp:429)
        }
        __syncthreads();
    }
}

__global__ void k_del_finish(InstState* __restrict__ st, const ListEntry* __restrict__ list,
                             int nlist, const uint32_t* __restrict__ del_kept) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nlist) return;
    InstState& S = st[list[k].inst];
    if (S.status) return;
    S.n = del_kept[k];
}

size_t contour_smem(int max_np) { return sizeof(double) * (4 * (size_t)max_np + 2); }

}  // namespace

void diffuse(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
             const Workspace& ws, int sms, cudaStream_t s) {
    (void)ws;
    // many resident warps: each blob is a chain of FP64 log / sqrt / sincos
    k_diffuse<<<sms * 16, 256, 0, s>>>(table, st, list, nlist);
}

void diffuse_raw(double* x, double* z, uint32_t n, const double* R, double nu, double dt,
                 int sms, cudaStream_t s) {
    if (n == 0) return;
    const unsigned g = (unsigned)std::min<uint64_t>((n + 255) / 256, (uint64_t)sms * 8);
    k_diffuse_raw<<<g, 256, 0, s>>>(x, z, n, R, nu, dt);
}

void release(const InstDesc* table, InstState* st, const ListEntry* list, int nlist, int max_np,
             cudaStream_t s) {
    k_release<<<nlist, kRelThreads, sizeof(double) * 2 * max_np, s>>>(table, st, list);
}

void reflect(const InstDesc* table, InstState* st, const ListEntry* list, int nlist, int max_np,
             const Workspace& ws, int sms, cudaStream_t s) {
    const size_t smem = contour_smem(max_np);
    static bool attr = false;  // set once, before any graph capture (first call is eager)
    if (!attr) {
        cudaFuncSetAttribute(k_reflect, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        attr = true;
    }
    cudaMemsetAsync(ws.work + 2, 0, sizeof(unsigned), s);
    k_reflect<<<sms * 4, 256, smem, s>>>(table, st, list, nlist, ws.work + 2);
}

void delete_inside(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
                   int max_np, const Workspace& ws, int sms, cudaStream_t s) {
    const size_t smem = contour_smem(max_np);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_del_flags, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        attr = true;
    }
    const int gx = std::max(1, sms * 4 / std::max(1, nlist));
    k_del_flags<<<dim3(gx, nlist), 256, smem, s>>>(table, st, list, ws.flags, ws.tile_counts);
    k_del_scan<<<nlist, 1024, 0, s>>>(st, list, ws.tile_counts, ws.tile_base, ws.del_kept);
    cudaMemsetAsync(ws.del_ready, 0, sizeof(uint32_t) * (ws.total_cap / kDelTile + 1), s);
    cudaMemsetAsync(ws.work + 3, 0, sizeof(unsigned), s);
    k_del_move<<<sms * 2, kDelTile, 0, s>>>(table, st, list, nlist, ws.flags, ws.tile_base,
                                            ws.del_kept, ws.del_ready, ws.work + 3);
    k_del_finish<<<(nlist + 127) / 128, 128, 0, s>>>(st, list, nlist, ws.del_kept);
}

}  // namespace dvmk

// ---- the device Philox4x32-10 on caller blocks (known-answer checks) -------------
namespace dvmk {
namespace {
__global__ void k_philox_blocks(const uint32_t* __restrict__ ctr, const uint32_t* __restrict__ key,
                                uint32_t n, uint32_t* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const U4 o = philox4x32_10(U4{ctr[4 * i], ctr[4 * i + 1], ctr[4 * i + 2], ctr[4 * i + 3]},
                                   key[2 * i], key[2 * i + 1]);
        out[4 * i] = o.a;
        out[4 * i + 1] = o.b;
        out[4 * i + 2] = o.c;
        out[4 * i + 3] = o.d;
    }
}
}  // namespace
}  // namespace dvmk

extern "C" int dvm_philox4x32_10(const uint32_t* ctr, const uint32_t* key, uint64_t n,
                                 uint32_t* out) {
    using namespace dvmk;
    if (n == 0) return 0;
    if (!ctr || !key || !out) return report_error(1, "null argument");
    if (n > (1ull << 26)) return report_error(1, "at most 2^26 blocks per call");
    uint32_t* d = nullptr;
    const size_t words = 10 * (size_t)n;  // ctr 4n | key 2n | out 4n
    cudaError_t e = cudaMalloc(&d, 4 * words);
    if (e != cudaSuccess) return report_error(e == cudaErrorMemoryAllocation ? 2 : 3, cudaGetErrorString(e));
    if (e == cudaSuccess) e = cudaMemcpy(d, ctr, 16 * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + 4 * n, key, 8 * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const unsigned blocks = (unsigned)std::min<uint64_t>((n + 255) / 256, 4096);
        k_philox_blocks<<<blocks, 256>>>(d, d + 4 * n, (uint32_t)n, d + 6 * n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d + 6 * n, 16 * n, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? 0 : report_error(3, cudaGetErrorString(e));
}
