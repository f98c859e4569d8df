// Regularised 2-D Biot-Savart kernels (reference: src/VelocityKernel.cpp:30-109,
// src/VortexSheet.cpp:171-210).
//
// Pair kernel:  K(r2) = (1 - exp(-r2/sigma_j^2)) / r2   if r2 < 10 sigma_j^2
//                     = 1 / r2                          otherwise
//               u_i = -(1/2pi) sum_j K dz Gamma_j,  w_i = (1/2pi) sum_j K dx Gamma_j
//
// FP32 path (the throughput path): blobs of every listed simulation are sorted
// along a Morton curve, packed as FP64 (x, z) + FP32 (Gamma, 10 sigma^2,
// 1/sigma^2) and split into 256-blob tiles with bounding boxes.  A work item is
// (simulation, 256 or 128 sorted targets, one source chunk); every warp pulls
// items from an atomic counter on its own and stages 256 sources at a time in
// its slice of shared memory.  Per staged tile the warp checks once, from the
// boxes of its 256-target block and of the tile, whether any pair can fall
// inside the 10 sigma^2 core: far tiles (almost all) run packed FP32x2
// arithmetic with one MUFU reciprocal per pair and no test; near tiles run the
// same packed arithmetic plus the exact per-pair test, the core kernel
// evaluated as (1/sigma^2) phi(r^2/sigma^2) with the r -> 0 limit built in
// (core_kernel).  Coordinates
// are FP32 offsets from the first target of the enclosing 256-target block,
// sums are FP32 within a stage and Kahan-compensated across stages, and chunk
// partials are combined in FP64 in chunk order: deterministic, and independent
// of the batch a simulation runs in and of the launch shape.
//
// FP64 path (the parity path): same work decomposition in original blob order
// and the reference's exact operation sequence (no FMA contraction).
#include <cfloat>
#include <mutex>
#include <string>

#include <cub/cub.cuh>

#include "dvm_device.cuh"
#include "dvm_internal.h"

namespace dvmk {
namespace {

constexpr int kMaxList = kMaxBatch;  // simulations per batched launch

__device__ __forceinline__ uint32_t spread16(uint32_t v) {
    v &= 0xFFFFu;
    v = (v | (v << 8)) & 0x00FF00FFu;
    v = (v | (v << 4)) & 0x0F0F0F0Fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

__device__ __forceinline__ uint32_t morton_key(double x, double z, double x0, double z0,
                                               double inv) {
    double fx = (x - x0) * inv, fz = (z - z0) * inv;
    fx = fmin(fmax(fx, 0.0), 65535.0);
    fz = fmin(fmax(fz, 0.0), 65535.0);
    const uint32_t key = spread16((uint32_t)fx) | (spread16((uint32_t)fz) << 1);
    return key == 0xFFFFFFFFu ? 0xFFFFFFFEu : key;
}

__device__ __forceinline__ int entry_of_slot(const ListEntry* list, int nlist, uint64_t g) {
    int lo = 0, hi = nlist - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (list[mid].coff <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Sort keys over the concatenated capacity space: (entry << 32 | morton);
// unused slots sort to the end of their simulation's range.
__global__ void k_keys(const InstDesc* __restrict__ table, const InstState* __restrict__ st,
                       const ListEntry* __restrict__ list, int nlist, uint64_t total,
                       uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < total;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const int k = entry_of_slot(list, nlist, g);
        const ListEntry e = list[k];
        const uint32_t i = (uint32_t)(g - e.coff);
        const InstDesc& d = table[e.inst];
        uint32_t mk = 0xFFFFFFFFu;
        if (i < st[e.inst].n) mk = morton_key(d.x[i], d.z[i], d.kx0, d.kz0, d.kinv);
        keys[g] = ((uint64_t)k << 32) | mk;
        vals[g] = i;
    }
}

// Gather (x, z, Gamma, sigma) into sorted order and record per-tile bounds.
__global__ void __launch_bounds__(kBsST) k_pack(const InstDesc* __restrict__ table,
                                                const InstState* __restrict__ st,
                                                const ListEntry* __restrict__ list, int nlist,
                                                const uint32_t* __restrict__ perm,
                                                double4* __restrict__ packed,
                                                double2* __restrict__ pxz,
                                                float4* __restrict__ pf,
                                                TileMeta* __restrict__ meta,
                                                int* __restrict__ mexp) {
    __shared__ unsigned s_pre[kMaxList + 1];
    __shared__ double s_red[7][kBsST / 32];
    if (threadIdx.x == 0) {
        unsigned acc = 0;
        for (int k = 0; k < nlist; ++k) {
            s_pre[k] = acc;
            acc += (st[list[k].inst].n + kBsST - 1) / kBsST;
        }
        s_pre[nlist] = acc;
    }
    __syncthreads();
    const unsigned total = s_pre[nlist];
    for (unsigned item = blockIdx.x; item < total; item += gridDim.x) {
        const int k = locate(s_pre, nlist, item);
        const ListEntry e = list[k];
        const InstDesc& d = table[e.inst];
        const uint32_t n = st[e.inst].n;
        const uint32_t i = (item - s_pre[k]) * kBsST + threadIdx.x;
        double xmin = DBL_MAX, xmax = -DBL_MAX, zmin = DBL_MAX, zmax = -DBL_MAX, thr = 0.0;
        double gmax = 0.0, tmin = DBL_MAX;  // max |Gamma| (as the FP32 path rounds it), min 10 sigma^2
        if (i < n) {
            const uint32_t p = perm ? perm[e.coff + i] : i;
            const double4 v = make_double4(d.x[p], d.z[p], d.circ[p], d.sigma[p]);
            if (pxz) {  // FP32 path: positions in FP64, per-source constants in FP32
                const double s2 = v.w * v.w;
                pxz[e.coff + i] = make_double2(v.x, v.y);
                pf[e.coff + i] = make_float4((float)v.z, (float)(10.0 * s2), (float)(1.0 / s2), 0.f);
            } else {
                packed[e.coff + i] = v;
            }
            xmin = xmax = v.x;
            zmin = zmax = v.y;
            thr = tmin = 10.0 * (v.w * v.w);
            gmax = fabs((double)(float)v.z);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            xmin = fmin(xmin, __shfl_xor_sync(0xffffffffu, xmin, o));
            xmax = fmax(xmax, __shfl_xor_sync(0xffffffffu, xmax, o));
            zmin = fmin(zmin, __shfl_xor_sync(0xffffffffu, zmin, o));
            zmax = fmax(zmax, __shfl_xor_sync(0xffffffffu, zmax, o));
            thr = fmax(thr, __shfl_xor_sync(0xffffffffu, thr, o));
            gmax = fmax(gmax, __shfl_xor_sync(0xffffffffu, gmax, o));
            tmin = fmin(tmin, __shfl_xor_sync(0xffffffffu, tmin, o));
        }
        const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if (lane == 0) {
            s_red[0][wid] = xmin;
            s_red[1][wid] = xmax;
            s_red[2][wid] = zmin;
            s_red[3][wid] = zmax;
            s_red[4][wid] = thr;
            s_red[5][wid] = gmax;
            s_red[6][wid] = tmin;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            TileMeta m;
            m.xmin = s_red[0][0];
            m.xmax = s_red[1][0];
            m.zmin = s_red[2][0];
            m.zmax = s_red[3][0];
            m.thr = s_red[4][0];
            for (int q = 1; q < kBsST / 32; ++q) {
                m.xmin = fmin(m.xmin, s_red[0][q]);
                m.xmax = fmax(m.xmax, s_red[1][q]);
                m.zmin = fmin(m.zmin, s_red[2][q]);
                m.zmax = fmax(m.zmax, s_red[3][q]);
                m.thr = fmax(m.thr, s_red[4][q]);
            }
            m.pad0 = m.pad1 = m.pad2 = 0.0;
            meta[(e.coff + (uint64_t)(item - s_pre[k]) * kBsST) / kBsST] = m;
            if (mexp) {  // exponent bounds of the simulation's mutual sums (order-free max)
                double gm = s_red[5][0], tm = s_red[6][0];
                for (int q = 1; q < kBsST / 32; ++q) {
                    gm = fmax(gm, s_red[5][q]);
                    tm = fmin(tm, s_red[6][q]);
                }
                const int eg = gm > 0.0 ? ilogb(gm) + 1 : -1100;  // max |Gamma| < 2^eg
                const int es = (1 - ilogb(fmax(tm, 1e-30))) >> 1;  // 1 / sqrt(min) <= 2^es
                const double cm = fmax(fmax(fabs(m.xmin), fabs(m.xmax)),
                                       fmax(fabs(m.zmin), fabs(m.zmax)));
                const int ec = cm > 0.0 ? ilogb(cm) + 1 : -1100;  // |coordinates| < 2^ec
                atomicMax(&mexp[4 * e.inst], eg);
                atomicMax(&mexp[4 * e.inst + 1], es);
                atomicMax(&mexp[4 * e.inst + 2], ec);
            }
        }
        __syncthreads();
    }
}

__device__ __forceinline__ void item_prefix_f64(unsigned* s_pre, const InstState* st,
                                                 const ListEntry* list, int nlist) {
    if (threadIdx.x == 0) {
        unsigned acc = 0;
        for (int k = 0; k < nlist; ++k) {
            s_pre[k] = acc;
            acc += ((st[list[k].inst].n + kBsTT - 1) / kBsTT) * (unsigned)list[k].chunks;
        }
        s_pre[nlist] = acc;
    }
    __syncthreads();
}

__device__ __forceinline__ uint32_t chunk_size(uint32_t n, int chunks) {
    uint32_t cs = (n + chunks - 1) / chunks;
    return (cs + kBsST - 1) / kBsST * kBsST;
}

// ---- FP32 pair loops --------------------------------------------------------
// A work item belongs to ONE warp: one 256-blob sort tile of targets (8
// consecutive ones per lane, 4 packed FP32x2 target pairs) against one source
// chunk.  The warp stages its own source tiles in shared memory and never waits
// for other warps, so far-path and near-path warps of a block do not hold each
// other up at barriers.
//
// Tile pairs.  A (target tile a, source tile b) stage is
//   mutual far  when the two tiles' boxes are farther apart than both tiles'
//               core radii (every pair, either way round, has K = 1/r2): the
//               item of the lower tile evaluates it once for both directions
//               and the item of the upper tile skips it;
//   far         when only the source cores are out of reach (no core test);
//   near        otherwise (the exact core test per pair; a == b is near).
constexpr int kWWarps = 4;            // independent warps per block
constexpr int kSelfMinBlocks = 4;     // blocks per SM the registers allow (128 each)
constexpr int kWR = 8;                // targets per lane
constexpr int kWP = kWR / 2;          // packed target pairs per lane

// A warp's staged source tile: pos2[i] = (x, z) of sources 2i and 2i+1 (FP32
// offsets), gam2[i] = (Gamma, Gamma) of both, core[j] = (10 sigma^2,
// 1/sigma^2).  The loops read two sources with two 16-byte loads and duplicate
// x and z into packed register pairs themselves (half the shared-memory loads
// of one 32-byte record per source: 0.6 % faster, same results).
struct StagedTile {
    float4 pos2[kBsST / 2];
    float4 gam2[kBsST / 2];
    float2 core[kBsST];
};

// One staged source against the warp's targets (far: no core test).
template <int WP>
__device__ __forceinline__ void far_pair(uint64_t sx, uint64_t sz, uint64_t sg,
                                         const uint64_t (&tx2)[WP], const uint64_t (&tz2)[WP],
                                         uint64_t (&nu2)[WP], uint64_t (&w2)[WP]) {
#pragma unroll
    for (int q = 0; q < WP; ++q) {
        const uint64_t dx = f2sub(tx2[q], sx);
        const uint64_t dz = f2sub(tz2[q], sz);
        const uint64_t r2 = f2fma(dx, dx, f2mul(dz, dz));
        // one MUFU reciprocal per pair (padded sources: rcp of ~2e36, Gamma 0)
        const uint64_t inv = f2pack(rcp_approx(f2lo(r2)), rcp_approx(f2hi(r2)));
        const uint64_t g = f2mul(inv, sg);
        nu2[q] = f2fma(g, dz, nu2[q]);
        w2[q] = f2fma(g, dx, w2[q]);
    }
}

// Far pairs: no core test.  Accumulates -u (so every update is one FMA) and w.
// (Sharing one reciprocal between the two targets of a packed pair, 1/a = b/(ab),
// trades one MUFU operation for three FP32 multiplications; it measured 1-4 %
// slower for 1/8 to 1/2 of the sources, the FMA pipe being nearly as loaded as
// the MUFU pipe.  So did a Newton reciprocal on the FMA pipe for one source in
// sixteen: 3.5 % slower at N = 2^20.)
template <int WP>
__device__ __forceinline__ void stage_far(const StagedTile& __restrict__ src,
                                          const uint64_t (&tx2)[WP], const uint64_t (&tz2)[WP],
                                          uint64_t (&nu2)[WP], uint64_t (&w2)[WP]) {
#pragma unroll 4  // 8 sources per unrolled body
    for (int i = 0; i < kBsST / 2; ++i) {
        const float4 P = src.pos2[i];
        const float4 G = src.gam2[i];
        far_pair(f2pack(P.x, P.x), f2pack(P.y, P.y), f2pack(G.x, G.y), tx2, tz2, nu2, w2);
        far_pair(f2pack(P.z, P.z), f2pack(P.w, P.w), f2pack(G.z, G.w), tx2, tz2, nu2, w2);
    }
}

// Mutual far pairs: one reciprocal per pair serves both directions.  Besides
// the targets' sums (as far_pair), the lane adds Gamma_i K (dz_ij, dx_ij) of its
// targets i to source j's packed sums snu, sw; the source's own velocity takes
// them with the opposite sign (dx_ji = -dx_ij).  Padding targets carry Gamma 0.
__device__ __forceinline__ void mutual_pair(uint64_t sx, uint64_t sz, uint64_t sg,
                                            const uint64_t (&tx2)[kWP],
                                            const uint64_t (&tz2)[kWP],
                                            const uint64_t (&tg2)[kWP], uint64_t (&nu2)[kWP],
                                            uint64_t (&w2)[kWP], uint64_t& snu, uint64_t& sw) {
#pragma unroll
    for (int q = 0; q < kWP; ++q) {
        const uint64_t dx = f2sub(tx2[q], sx);
        const uint64_t dz = f2sub(tz2[q], sz);
        const uint64_t r2 = f2fma(dx, dx, f2mul(dz, dz));
        const uint64_t inv = f2pack(rcp_approx(f2lo(r2)), rcp_approx(f2hi(r2)));
        const uint64_t g = f2mul(inv, sg);
        nu2[q] = f2fma(g, dz, nu2[q]);
        w2[q] = f2fma(g, dx, w2[q]);
        const uint64_t h = f2mul(inv, tg2[q]);
        snu = f2fma(h, dz, snu);
        sw = f2fma(h, dx, sw);
    }
}

// v 2^shift rounded to a 64-bit integer (two's complement in the unsigned
// accumulator; the conversion saturates outside the 64-bit range).
__device__ __forceinline__ unsigned long long to_fixed(double v, double scale) {
    return (unsigned long long)__double2ll_rn(v * scale);
}

// A mutual far stage.  The staged sources form 64 groups of four, taken in
// two rounds of 32.  In step s of a round lane l evaluates group (l + s) mod 32
// against its 8 targets, adding to the group's packed sums (Gamma_i K dz,
// Gamma_i K dx per source; low and high halves from the even and odd targets),
// then hands the sums to lane l - 1, which takes that group in step s + 1.
// After 32 steps lane l holds the sums of group l over all 256 targets, in a
// fixed order, and adds them to the sources' 64-bit fixed-point accumulators
// acc[2 j], acc[2 j + 1] (value x 2^shift, rounded; integer addition is exact
// and order-free, so the sums do not depend on which warp adds first).  The
// hand-over costs 16 shuffles per 32 pairs and no arithmetic (a shuffle-tree
// reduction per batch of sources was 3.5 % slower).  Sources j >= n are padding.
__device__ __forceinline__ void stage_mutual(const StagedTile& __restrict__ src,
                                             const uint64_t (&tx2)[kWP],
                                             const uint64_t (&tz2)[kWP],
                                             const uint64_t (&tg2)[kWP], uint64_t (&nu2)[kWP],
                                             uint64_t (&w2)[kWP],
                                             unsigned long long* __restrict__ acc,
                                             uint32_t nsrc, double scale, int lane) {
    const unsigned all = 0xffffffffu;
    const int next = (lane + 1) & 31;
#pragma unroll 1
    for (int rnd = 0; rnd < kBsST / 128; ++rnd) {
        uint64_t au[4], aw[4];  // packed sums of the group this lane holds
#pragma unroll
        for (int b = 0; b < 4; ++b) au[b] = aw[b] = 0ull;
#pragma unroll 1
        for (int s = 0; s < 32; ++s) {
            const int gi = rnd * 32 + ((lane + s) & 31);  // group of 4 sources
            const float4 P0 = src.pos2[2 * gi], P1 = src.pos2[2 * gi + 1];
            const float4 G0 = src.gam2[2 * gi], G1 = src.gam2[2 * gi + 1];
            mutual_pair(f2pack(P0.x, P0.x), f2pack(P0.y, P0.y), f2pack(G0.x, G0.y), tx2, tz2,
                        tg2, nu2, w2, au[0], aw[0]);
            mutual_pair(f2pack(P0.z, P0.z), f2pack(P0.w, P0.w), f2pack(G0.z, G0.w), tx2, tz2,
                        tg2, nu2, w2, au[1], aw[1]);
            mutual_pair(f2pack(P1.x, P1.x), f2pack(P1.y, P1.y), f2pack(G1.x, G1.y), tx2, tz2,
                        tg2, nu2, w2, au[2], aw[2]);
            mutual_pair(f2pack(P1.z, P1.z), f2pack(P1.w, P1.w), f2pack(G1.z, G1.w), tx2, tz2,
                        tg2, nu2, w2, au[3], aw[3]);
            // the group moves on to the lane that takes it next (lane - 1)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                au[b] = __shfl_sync(all, au[b], next);
                aw[b] = __shfl_sync(all, aw[b], next);
            }
        }
        // after 32 steps every lane's targets have passed over the group this lane holds
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const uint32_t j = 4 * (rnd * 32 + lane) + b;
            if (j < nsrc) {  // u_j += sum Gamma_i K dz_ij, w_j -= sum Gamma_i K dx_ij
                atomicAdd(&acc[2 * j], to_fixed((double)(f2lo(au[b]) + f2hi(au[b])), scale));
                atomicAdd(&acc[2 * j + 1], to_fixed(-(double)(f2lo(aw[b]) + f2hi(aw[b])), scale));
            }
        }
    }
}

// Core kernel (1 - exp(-r2/sigma^2)) / r2 in FP32, written as rs phi(t) with
// t = r2 rs, rs = 1/sigma^2 and phi(t) = (1 - e^-t) / t.  For t < 1/2 phi is
// a degree-5 polynomial, minimax in relative error on [0, 1/2] (Lawson's
// algorithm, csrc/fit_polys.py: 6.1e-8 relative in FP32 Horner form, the
// degree-8 Taylor series it replaced gave 6.5e-8 with three more FMAs per
// half).  Its constant term 1 = phi(0) gives the r -> 0 limit 1/sigma^2: the
// self pair then contributes exactly zero, as the reference's i != j skip
// gives, and distinct blobs closer than FP32 resolves stay finite, as the
// FP64 reference is.  For t >= 1/2 it is (1 - e) / r2 with e = 2^(-t log2 e)
// from one MUFU ex2; 1 - e >= 0.39 there, so the ex2 error stays below 4e-7
// relative.
__device__ __forceinline__ float core_kernel(float r2, float rs, float rcp_r2) {
    const float t = r2 * rs;
    float p = -1.121634850e-03f;
    p = fmaf(p, t, 8.187386207e-03f);
    p = fmaf(p, t, -4.162909091e-02f);
    p = fmaf(p, t, 1.666622460e-01f);
    p = fmaf(p, t, -4.999998212e-01f);
    p = fmaf(p, t, 1.0f);
    const float e = ex2_approx(-t * 1.44269504088896341f);
    return t < 0.5f ? rs * p : (1.0f - e) * rcp_r2;
}

// The same core kernel through expm1f (about 1 ulp): the blob-on-collocation
// right-hand side keeps it, since that sum is a small residual of nearly
// cancelling terms.  Below FLT_MIN the r -> 0 limit 1/sigma^2 is used.
__device__ __forceinline__ float core_kernel_expm1(float r2, float rs, float rcp_r2) {
    const float e = expm1f(-r2 * rs);
    return r2 > 1e-30f ? -e * rcp_r2 : rs;
}

// One staged source against the warp's targets with the exact core test.  SELF
// (the target tile's own sources): a pair at r2 == 0 adds nothing, which is the
// reference's i != j skip for the self pair whatever the core size (sigma = 0
// would otherwise give 1/0 times dz = 0).
template <int WP, bool SELF>
__device__ __forceinline__ void near_pair(uint64_t sx, uint64_t sz, uint64_t sg, float2 C,
                                          const uint64_t (&tx2)[WP], const uint64_t (&tz2)[WP],
                                          uint64_t (&nu2)[WP], uint64_t (&w2)[WP]) {
#pragma unroll
    for (int q = 0; q < WP; ++q) {
        const uint64_t dx = f2sub(tx2[q], sx);
        const uint64_t dz = f2sub(tz2[q], sz);
        const uint64_t r2 = f2fma(dx, dx, f2mul(dz, dz));
        const float ra = f2lo(r2), rb = f2hi(r2);
        float ka = rcp_approx(ra), kb = rcp_approx(rb);
        const bool ca = ra < C.x, cb = rb < C.x;
        if (__any_sync(0xffffffffu, ca || cb)) {
            const float qa = core_kernel(ra, C.y, ka), qb = core_kernel(rb, C.y, kb);
            ka = ca ? qa : ka;
            kb = cb ? qb : kb;
        }
        if (SELF) {
            ka = ra > 0.0f ? ka : 0.0f;
            kb = rb > 0.0f ? kb : 0.0f;
        }
        const uint64_t g = f2mul(f2pack(ka, kb), sg);
        nu2[q] = f2fma(g, dz, nu2[q]);
        w2[q] = f2fma(g, dx, w2[q]);
    }
}

// Near pairs: the reference's exact test per pair.  The shared arithmetic is
// packed like the far path (each half rounds like the scalar instruction, so a
// pair outside the core gets the same bits on either path); the core kernel
// runs for both halves of a packed pair, branch-free, whenever any lane of the
// warp has a pair inside the core, and a select keeps it only for those pairs,
// so a pair's value does not depend on its neighbours in the warp.
template <int WP, bool SELF>
__device__ __forceinline__ void stage_near(const StagedTile& __restrict__ src,
                                           const uint64_t (&tx2)[WP], const uint64_t (&tz2)[WP],
                                           uint64_t (&nu2)[WP], uint64_t (&w2)[WP]) {
#pragma unroll 1
    for (int i = 0; i < kBsST / 2; ++i) {
        const float4 P = src.pos2[i];
        const float4 G = src.gam2[i];
        const float2 C0 = src.core[2 * i], C1 = src.core[2 * i + 1];
        near_pair<WP, SELF>(f2pack(P.x, P.x), f2pack(P.y, P.y), f2pack(G.x, G.y), C0, tx2, tz2,
                            nu2, w2);
        near_pair<WP, SELF>(f2pack(P.z, P.z), f2pack(P.w, P.w), f2pack(G.z, G.w), C1, tx2, tz2,
                            nu2, w2);
    }
}

__device__ __forceinline__ void kahan(float& s, float& c, float x) {
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

// Scale exponent of a simulation's fixed-point velocity sums.  One pair adds at
// most |Gamma_j| K r: 1/r <= 1/sqrt(10 sigma_j^2) outside the core and at most
// 0.64/sigma_j = 2.02/sqrt(10 sigma_j^2) inside it, so every sum is below
// 2.02 n max|Gamma| / r_min with r_min = sqrt(min 10 sigma^2); k_pack bounds
// max|Gamma| < 2^mexp[0] and 1/sqrt(min) <= 2^mexp[1].  Cores far smaller than
// the blobs' spacing (sigma = 0 above all: 1/r^2 for every pair) would make that
// bound meaningless and round every sum to zero, so r_min is floored at 2^-20 of
// the coordinates' magnitude (|x|, |z| < 2^mexp[2]).  With the shift below
// |sum| 2^shift < 2^58, well inside 64 bits, and one unit is 2^-56 of the bound
// (below 2e-17 of it; the FP32 terms carry 6e-8).  Under the floor a sum can
// leave the 64-bit range (32 times the bound) only through a pair closer than
// 2^-26 / n of 2^mexp[2] with a core smaller still: point vortices closer than
// the FP32 offsets (relative to a 256-blob tile) resolve in most layouts.
__device__ __forceinline__ int mutual_shift(const int* __restrict__ mexp, int inst, uint32_t n) {
    const int lgn = n > 1 ? 32 - __clz(n - 1) : 0;
    const long long es = min((long long)mexp[4 * inst + 1], 20ll - mexp[4 * inst + 2]);
    const long long e = (long long)lgn + mexp[4 * inst] + es;
    return (int)max(-1000ll, min(1000ll, 56 - e));
}

template <int MINB>
__global__ void __launch_bounds__(32 * kWWarps, MINB)
    k_self_f32(const InstState* __restrict__ st, const ListEntry* __restrict__ list, int nlist,
               const double2* __restrict__ pxz, const float4* __restrict__ pf,
               const TileMeta* __restrict__ meta, unsigned long long* __restrict__ macc,
               const int* __restrict__ mexp, unsigned* __restrict__ work) {
    __shared__ unsigned s_pre[kMaxList + 1];
    __shared__ StagedTile s_src[kWWarps];
    // Kahan sums of -u and w per lane, in shared memory rather than registers
    // (touched once per stage; the registers go to the pair arithmetic: 4 CTAs per
    // SM at 128 registers, 6 % faster than 3 CTAs with the sums in registers)
    __shared__ float s_kahan[kWWarps][4][kWR][32];
    constexpr int kWTT = 32 * kWR;
    static_assert(kWTT == kBsST, "a work item's targets are one sort tile");
    if (threadIdx.x == 0) {
        unsigned acc = 0;
        for (int k = 0; k < nlist; ++k) {
            s_pre[k] = acc;
            acc += ((st[list[k].inst].n + kWTT - 1) / kWTT) * (unsigned)list[k].chunks;
        }
        s_pre[nlist] = acc;
    }
    __syncthreads();
    const unsigned total = s_pre[nlist];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    StagedTile& wsrc = s_src[wid];
    float2* __restrict__ wpos = reinterpret_cast<float2*>(wsrc.pos2);
    float2* __restrict__ wgam = reinterpret_cast<float2*>(wsrc.gam2);
    for (;;) {
        unsigned item = 0;
        if (lane == 0) item = atomicAdd(work, 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= total) break;
        const int k = locate(s_pre, nlist, item);
        const ListEntry e = list[k];
        const uint32_t n = st[e.inst].n;
        const unsigned local = item - s_pre[k];
        const uint32_t tile = local / e.chunks, c = local % e.chunks;
        const uint32_t t0 = tile * kWTT;
        const uint32_t cs = chunk_size(n, e.chunks);
        const uint32_t j0 = c * cs, j1 = min(n, j0 + cs);
        const double2* __restrict__ X = pxz + e.coff;
        const float4* __restrict__ F = pf + e.coff;
        // FP32 offsets from the tile's first target
        const double2 o = X[t0];
        const double scale = ldexp(1.0, mutual_shift(mexp, e.inst, n));

        uint64_t tx2[kWP], tz2[kWP], tg2[kWP];
        const uint32_t tb = t0 + lane * kWR;
#pragma unroll
        for (int q = 0; q < kWP; ++q) {
            float xs[2], zs[2], gs[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                xs[h] = 0.0f;  // padding targets sit on the origin (a real target), Gamma 0
                zs[h] = 0.0f;
                gs[h] = 0.0f;
                const uint32_t t = tb + 2 * q + h;
                if (t < n) {
                    const double2 p = X[t];
                    xs[h] = (float)(p.x - o.x);
                    zs[h] = (float)(p.y - o.y);
                    gs[h] = F[t].x;
                }
            }
            tx2[q] = f2pack(xs[0], xs[1]);
            tz2[q] = f2pack(zs[0], zs[1]);
            tg2[q] = f2pack(gs[0], gs[1]);
        }
        const TileMeta& tm = meta[(e.coff + t0) / kBsST];
        float (*kh)[kWR][32] = s_kahan[wid];  // [0] -u, [1] its compensation, [2] w, [3]
#pragma unroll
        for (int r = 0; r < kWR; ++r)
            kh[0][r][lane] = kh[1][r][lane] = kh[2][r][lane] = kh[3][r][lane] = 0.0f;

        for (uint32_t s0 = j0; s0 < j1; s0 += kBsST) {
            const TileMeta m = meta[(e.coff + s0) / kBsST];
            const double gx = fmax(0.0, fmax(m.xmin - tm.xmax, tm.xmin - m.xmax));
            const double gz = fmax(0.0, fmax(m.zmin - tm.zmax, tm.zmin - m.zmax));
            const double g2 = gx * gx + gz * gz;
            // the same test in both tiles' items (symmetric in the two tiles)
            const bool mutual = g2 > fmax(m.thr, tm.thr) * 1.001 + 1e-30;
            if (mutual && s0 < t0) continue;  // the source tile's item adds this stage
            __syncwarp();
#pragma unroll
            for (int q = 0; q < kBsST / 32; ++q) {
                const uint32_t jj = q * 32 + lane, j = s0 + jj;
                if (j < j1) {
                    const double2 p = X[j];
                    const float4 f = F[j];  // (circ, 10 sigma^2, 1/sigma^2, -)
                    wpos[jj] = make_float2((float)(p.x - o.x), (float)(p.y - o.y));
                    wgam[jj] = make_float2(f.x, f.x);
                    wsrc.core[jj] = make_float2(f.y, f.z);
                } else {  // padding: far away, no circulation, never in a core
                    wpos[jj] = make_float2(1e18f, 1e18f);
                    wgam[jj] = make_float2(0.0f, 0.0f);
                    wsrc.core[jj] = make_float2(-1.0f, 0.0f);
                }
            }
            __syncwarp();
            uint64_t nu2[kWP], w2[kWP];
#pragma unroll
            for (int q = 0; q < kWP; ++q) nu2[q] = w2[q] = 0ull;  // +0.0f in both halves
            if (mutual) {
                stage_mutual(wsrc, tx2, tz2, tg2, nu2, w2, macc + 2 * (e.coff + s0),
                             min((uint32_t)kBsST, j1 - s0), scale, lane);
            } else if (g2 > m.thr * 1.001 + 1e-30) {
                stage_far(wsrc, tx2, tz2, nu2, w2);
            } else if (s0 == t0) {
                stage_near<kWP, true>(wsrc, tx2, tz2, nu2, w2);
            } else {
                stage_near<kWP, false>(wsrc, tx2, tz2, nu2, w2);
            }
#pragma unroll
            for (int q = 0; q < kWP; ++q) {  // Kahan fold of the stage partials
                kahan(kh[0][2 * q][lane], kh[1][2 * q][lane], f2lo(nu2[q]));
                kahan(kh[0][2 * q + 1][lane], kh[1][2 * q + 1][lane], f2hi(nu2[q]));
                kahan(kh[2][2 * q][lane], kh[3][2 * q][lane], f2lo(w2[q]));
                kahan(kh[2][2 * q + 1][lane], kh[3][2 * q + 1][lane], f2hi(w2[q]));
            }
        }
        // the item's sums join the targets' fixed-point sums (exact, order-free)
        unsigned long long* __restrict__ ta = macc + 2 * (e.coff + tb);
#pragma unroll
        for (int r = 0; r < kWR; ++r)
            if (tb + r < n) {
                atomicAdd(&ta[2 * r],
                          to_fixed(-((double)kh[0][r][lane] - (double)kh[1][r][lane]), scale));
                atomicAdd(&ta[2 * r + 1],
                          to_fixed((double)kh[2][r][lane] - (double)kh[3][r][lane], scale));
            }
    }
}

// ---- FP64, the reference's per-pair arithmetic -------------------------------
// Every pair is evaluated with the reference's operations (src/VelocityKernel.cpp:
// 44-60: IEEE division and exp inside the core, 1/r2 outside), over the same
// Morton-sorted tiles as the FP32 path.  A source stage whose tile box is beyond
// 10 sigma^2 of the item's target box (the union of its sort tiles) holds no core
// pair and no self pair, and runs the 1/r2 branch without the per-pair test; in
// blob order nearly every warp met a core pair somewhere and ran both branches.
// 3 CTAs of 8 warps per SM (80 registers): the FP64 division / exp chains need
// the warps (1 CTA per SM ran 2.2x slower)
constexpr int kF64Ctas = 3;
__global__ void __launch_bounds__(kBsThreads, kF64Ctas)
    k_self_f64(const InstState* __restrict__ st, const ListEntry* __restrict__ list, int nlist,
               const double4* __restrict__ packed, const TileMeta* __restrict__ meta,
               double2* __restrict__ part, unsigned* __restrict__ work) {
    __shared__ unsigned s_pre[kMaxList + 1];
    __shared__ double4 s_src[kBsST];  // x, z, circ, threshold
    __shared__ double s_rs[kBsST];
    __shared__ double s_box[4];  // the item's target box: xmin, xmax, zmin, zmax
    __shared__ unsigned s_item;
    item_prefix_f64(s_pre, st, list, nlist);
    const unsigned total = s_pre[nlist];
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) s_item = atomicAdd(work, 1u);
        __syncthreads();
        const unsigned item = s_item;
        __syncthreads();
        if (item >= total) break;
        const int k = locate(s_pre, nlist, item);
        const ListEntry e = list[k];
        const uint32_t n = st[e.inst].n;
        const unsigned local = item - s_pre[k];
        const uint32_t tile = local / e.chunks, c = local % e.chunks;
        const uint32_t cs = chunk_size(n, e.chunks);
        const uint32_t j0 = c * cs, j1 = min(n, j0 + cs);
        const double4* __restrict__ P = packed + e.coff;
        const uint32_t tb = tile * kBsTT + tid * kBsR;
        double tx[kBsR], tz[kBsR], uu[kBsR], ww[kBsR];
#pragma unroll
        for (int r = 0; r < kBsR; ++r) {
            const double4 p = (tb + r < n) ? P[tb + r] : make_double4(0, 0, 0, 1);
            tx[r] = p.x;
            tz[r] = p.y;
            uu[r] = ww[r] = 0.0;
        }
        if (tid == 0) {  // the item's target box (read after the next barrier)
            double b0 = DBL_MAX, b1 = -DBL_MAX, b2 = DBL_MAX, b3 = -DBL_MAX;
            for (int q = 0; q < kBsTT / kBsST; ++q) {
                const uint32_t t = tile * kBsTT + q * kBsST;
                if (t < n) {
                    const TileMeta& m = meta[(e.coff + t) / kBsST];
                    b0 = fmin(b0, m.xmin);
                    b1 = fmax(b1, m.xmax);
                    b2 = fmin(b2, m.zmin);
                    b3 = fmax(b3, m.zmax);
                }
            }
            s_box[0] = b0;
            s_box[1] = b1;
            s_box[2] = b2;
            s_box[3] = b3;
        }
        for (uint32_t s0 = j0; s0 < j1; s0 += kBsST) {
            __syncthreads();
            const TileMeta& m = meta[(e.coff + s0) / kBsST];
            const double gx = fmax(0.0, fmax(m.xmin - s_box[1], s_box[0] - m.xmax));
            const double gz = fmax(0.0, fmax(m.zmin - s_box[3], s_box[2] - m.zmax));
            const bool far = gx * gx + gz * gz > m.thr * 1.001 + 1e-30;
            const uint32_t j = s0 + tid;
            if (j < j1) {
                const double4 p = P[j];
                const double s2 = dmul(p.w, p.w);
                s_src[tid] = make_double4(p.x, p.y, p.z, dmul(10.0, s2));
                if (!far) s_rs[tid] = ddiv(1.0, s2);
            }
            __syncthreads();
            const int cnt = (int)min((uint32_t)kBsST, j1 - s0);
            if (far) {
                for (int jj = 0; jj < cnt; ++jj) {
                    const double4 sj = s_src[jj];
#pragma unroll
                    for (int r = 0; r < kBsR; ++r) {
                        const double dx = dsub(tx[r], sj.x);
                        const double dz = dsub(tz[r], sj.y);
                        const double K = __drcp_rn(dadd(dmul(dx, dx), dmul(dz, dz)));
                        uu[r] = dsub(uu[r], dmul(dmul(K, dz), sj.z));
                        ww[r] = dadd(ww[r], dmul(dmul(K, dx), sj.z));
                    }
                }
                continue;
            }
            for (int jj = 0; jj < cnt; ++jj) {
                const double4 s = s_src[jj];
#pragma unroll
                for (int r = 0; r < kBsR; ++r) {
                    if (tb + r == s0 + jj) continue;  // i != j (src/VelocityKernel.cpp:43)
                    const double dx = dsub(tx[r], s.x);
                    const double dz = dsub(tz[r], s.y);
                    const double r2 = dadd(dmul(dx, dx), dmul(dz, dz));
                    double K;
                    if (r2 < s.w) K = ddiv(dsub(1.0, exp(dmul(-r2, s_rs[jj]))), r2);
                    else K = __drcp_rn(r2);  // correctly rounded: the same value as 1.0 / r2
                    uu[r] = dsub(uu[r], dmul(dmul(K, dz), s.z));
                    ww[r] = dadd(ww[r], dmul(dmul(K, dx), s.z));
                }
            }
        }
        double2* __restrict__ out = part + e.poff + (uint64_t)c * e.cap;
#pragma unroll
        for (int r = 0; r < kBsR; ++r)
            if (tb + r < n) out[tb + r] = make_double2(uu[r], ww[r]);
    }
}

// Per blob: the FP32 path's fixed-point sums, or the FP64 path's chunk partials
// in chunk order; scale by 1/(2 pi), scatter to blob order.
__global__ void k_self_combine(const InstDesc* __restrict__ table,
                               const InstState* __restrict__ st,
                               const ListEntry* __restrict__ list, int nlist,
                               const uint32_t* __restrict__ perm,
                               const double2* __restrict__ part,
                               const unsigned long long* __restrict__ macc,
                               const int* __restrict__ mexp) {
    __shared__ unsigned s_pre[kMaxList + 1];
    if (threadIdx.x == 0) {
        unsigned acc = 0;
        for (int k = 0; k < nlist; ++k) {
            s_pre[k] = acc;
            acc += (st[list[k].inst].n + blockDim.x - 1) / blockDim.x;
        }
        s_pre[nlist] = acc;
    }
    __syncthreads();
    const unsigned total = s_pre[nlist];
    for (unsigned item = blockIdx.x; item < total; item += gridDim.x) {
        const int k = locate(s_pre, nlist, item);
        const ListEntry e = list[k];
        const uint32_t n = st[e.inst].n;
        const uint32_t t = (item - s_pre[k]) * blockDim.x + threadIdx.x;
        if (t >= n) continue;
        double su = 0.0, sw = 0.0;
        if (macc) {  // FP32: the blob's fixed-point sums
            const double inv = ldexp(1.0, -mutual_shift(mexp, e.inst, n));
            const uint64_t g = 2 * (e.coff + t);
            su = (double)(long long)macc[g] * inv;
            sw = (double)(long long)macc[g + 1] * inv;
        } else {  // FP64: the chunk partials in chunk order
            for (int c = 0; c < e.chunks; ++c) {
                const double2 v = part[e.poff + (uint64_t)c * e.cap + t];
                su += v.x;
                sw += v.y;
            }
        }
        const InstDesc& d = table[e.inst];
        const uint32_t p = perm ? perm[e.coff + t] : t;
        d.u[p] = su * kRpi2;
        d.w[p] = sw * kRpi2;
    }
}

// ---- arbitrary targets --------------------------------------------------------
// One item = (job, a tile of targets, a chunk of `chunk` sources: kAtChunk for
// at-target calls, rhs_chunk_for(...) for a simulation's right-hand side).
// Sources are staged with FP64 positions; each pair forms dx, dz in FP64
// (exact for close pairs) and, in FP32 mode, evaluates the kernel in FP32 with
// Kahan-compensated sums.
struct AtJob {
    const double* tx;
    const double* tz;
    uint32_t nt;
    int skip_close;  // 1: pairs with r2 <= 1e-15 skipped (computeInducedAt)
    const double* sx;
    const double* sz;
    const double* sc;
    const double* ss;
    const uint32_t* pns;  // source count on the device, or null -> ns
    uint32_t ns;
    int npad;             // partial row length
    uint32_t chunk;       // sources per work item (a multiple of 256)
    double2* part;        // [chunk][npad]
    double* circ_part;    // [chunk], or null
};

// Kahan sum of packed pairs with the compensation kept negated (e = -c):
// y = x + e, t = s + y, e = y - (t - s), s = t -- each half the scalar
// algorithm; x = a b enters through one fused multiply-add.
__device__ __forceinline__ void kahan2_fma(uint64_t& s, uint64_t& e, uint64_t a, uint64_t b) {
    const uint64_t y = f2fma(a, b, e);
    const uint64_t t = f2add(s, y);
    e = f2sub(y, f2sub(t, s));
    s = t;
}

// Velocity at targets from a chunk of J.chunk sources per work item, 256
// targets per item, one per thread.
//
// FP32 jobs without the close-pair skip (the blob-on-collocation right-hand
// side) pack two SOURCES per FP32x2 instruction, so no lane idles however few
// targets a body has.  Offsets are formed without per-pair conversions: every
// position is taken relative to the job's first target in FP64 and split
// exactly into an FP32 pair (hi, lo = the FP64 remainder); dx = (t_hi - s_hi)
// + (t_lo - s_lo), exact before its final rounding for close pairs (Sterbenz)
// and within an ulp otherwise.  Each pair keeps its compensated update (the
// right-hand side is the small residual normal velocity, so its rounding must
// stay relative to the few large near-blob terms, not compound): one Kahan
// sum per half, the halves added at the end.  The core kernel runs for both
// halves when any lane of the warp has a pair inside a core.  Sources are
// staged as packed pairs (two 16-byte loads bring positions, two more the
// circulations and core constants).  Skip jobs (at-target plugin calls,
// probes) and FP64 jobs run the scalar loops.
struct AtStage {
    float4 pos_hi[128];  // (x_hi a, x_hi b, z_hi a, z_hi b) of sources 2i, 2i+1
    float4 pos_lo[128];  // (x_lo a, x_lo b, z_lo a, z_lo b)
    float4 cst[128];     // (circ a, circ b, 10 sigma^2 a, 10 sigma^2 b)
    float2 rs[128];      // (1/sigma^2 a, 1/sigma^2 b)
};

__device__ __forceinline__ void split_hi_lo(double v, float& hi, float& lo) {
    hi = (float)v;
    lo = (float)(v - (double)hi);
}

template <bool F32>
__global__ void __launch_bounds__(256) k_at(const AtJob* __restrict__ jobs, int njobs) {
    __shared__ unsigned s_pre[kMaxList + 1];
    __shared__ double s_x[256], s_z[256], s_c[256], s_thr[256], s_rs[256];
    __shared__ float s_cf[256], s_thrf[256], s_rsf[256];  // FP32 copies (scalar FP32 path)
    __shared__ AtStage s_pk;                               // packed pairs (fast FP32 path)
    __shared__ double s_red[8];
    if (threadIdx.x == 0) {
        unsigned acc = 0;
        for (int k = 0; k < njobs; ++k) {
            s_pre[k] = acc;
            const uint32_t ns = jobs[k].pns ? *jobs[k].pns : jobs[k].ns;
            acc += ((jobs[k].nt + 255) / 256) * ((ns + jobs[k].chunk - 1) / jobs[k].chunk);
        }
        s_pre[njobs] = acc;
    }
    __syncthreads();
    const unsigned total = s_pre[njobs];
    for (unsigned item = blockIdx.x; item < total; item += gridDim.x) {
        const int k = locate(s_pre, njobs, item);
        const AtJob J = jobs[k];
        const bool packed = F32 && !J.skip_close;
        const uint32_t ns = J.pns ? *J.pns : J.ns;
        const uint32_t nchunk = (ns + J.chunk - 1) / J.chunk;
        const unsigned local = item - s_pre[k];
        const uint32_t ttile = local / nchunk, c = local % nchunk;
        const uint32_t t = ttile * 256 + threadIdx.x;
        const double tx = t < J.nt ? J.tx[t] : 0.0, tz = t < J.nt ? J.tz[t] : 0.0;
        const double ox = J.tx[0], oz = J.tz[0];  // the job's origin: its first target
        float txh, txl, tzh, tzl;
        split_hi_lo(tx - ox, txh, txl);
        split_hi_lo(tz - oz, tzh, tzl);
        const uint64_t TXH = f2pack(txh, txh), TXL = f2pack(txl, txl);
        const uint64_t TZH = f2pack(tzh, tzh), TZL = f2pack(tzl, tzl);
        const uint32_t j0 = c * J.chunk, j1 = min(ns, j0 + J.chunk);
        double uu = 0.0, ww = 0.0, csum = 0.0;
        const uint64_t zero2 = f2pack(0.0f, 0.0f);
        uint64_t snu = zero2, enu = zero2, sw = zero2, ew = zero2;  // -u and w, packed Kahan
        float su = 0.f, cu = 0.f, sws = 0.f, cws = 0.f;
        for (uint32_t s0 = j0; s0 < j1; s0 += 256) {
            __syncthreads();
            const uint32_t j = s0 + threadIdx.x;
            if (packed) {
                // slot (pair i = tid / 2, half h = tid % 2); a slot past the
                // chunk holds a far, circulation-free source (it adds 0)
                float xh = 1.0e18f, xl = 0.f, zh = 0.f, zl = 0.f, cf = 0.f, thr = 0.f, rsf = 0.f;
                if (j < j1) {
                    const double sg = J.ss[j];
                    const double s2 = dmul(sg, sg);
                    split_hi_lo(J.sx[j] - ox, xh, xl);
                    split_hi_lo(J.sz[j] - oz, zh, zl);
                    cf = (float)J.sc[j];
                    thr = (float)dmul(10.0, s2);
                    rsf = (float)ddiv(1.0, s2);
                    if (ttile == 0) csum += J.sc[j];
                }
                const int i = threadIdx.x >> 1, h = threadIdx.x & 1;
                float* ph = reinterpret_cast<float*>(&s_pk.pos_hi[i]);
                float* pl = reinterpret_cast<float*>(&s_pk.pos_lo[i]);
                float* pc = reinterpret_cast<float*>(&s_pk.cst[i]);
                float* pr = reinterpret_cast<float*>(&s_pk.rs[i]);
                ph[h] = xh;
                ph[2 + h] = zh;
                pl[h] = xl;
                pl[2 + h] = zl;
                pc[h] = cf;
                pc[2 + h] = thr;
                pr[h] = rsf;
            } else if (j < j1) {
                const double sg = J.ss[j];
                const double s2 = dmul(sg, sg);
                s_x[threadIdx.x] = J.sx[j];
                s_z[threadIdx.x] = J.sz[j];
                s_c[threadIdx.x] = J.sc[j];
                s_thr[threadIdx.x] = dmul(10.0, s2);
                s_rs[threadIdx.x] = ddiv(1.0, s2);
                if (F32) {  // converted once per source instead of once per pair
                    s_cf[threadIdx.x] = (float)s_c[threadIdx.x];
                    s_thrf[threadIdx.x] = (float)s_thr[threadIdx.x];
                    s_rsf[threadIdx.x] = (float)s_rs[threadIdx.x];
                }
                if (ttile == 0) csum += J.sc[j];
            }
            __syncthreads();
            const int cnt = (int)min(256u, j1 - s0);
            if (packed) {
                for (int i = 0; i < (cnt + 1) / 2; ++i) {
                    const float4 H = s_pk.pos_hi[i], L = s_pk.pos_lo[i], Cs = s_pk.cst[i];
                    const uint64_t DX = f2add(f2sub(TXH, f2pack(H.x, H.y)),
                                              f2sub(TXL, f2pack(L.x, L.y)));
                    const uint64_t DZ = f2add(f2sub(TZH, f2pack(H.z, H.w)),
                                              f2sub(TZL, f2pack(L.z, L.w)));
                    const uint64_t R2 = f2fma(DX, DX, f2mul(DZ, DZ));
                    const float ra = f2lo(R2), rb = f2hi(R2);
                    float ka = rcp_approx(ra), kb = rcp_approx(rb);
                    const bool ca = ra < Cs.z, cb = rb < Cs.w;
                    if (__any_sync(0xffffffffu, ca || cb)) {
                        const float2 R = s_pk.rs[i];
                        const float qa = core_kernel_expm1(ra, R.x, ka);
                        const float qb = core_kernel_expm1(rb, R.y, kb);
                        ka = ca ? qa : ka;
                        kb = cb ? qb : kb;
                    }
                    const uint64_t G = f2mul(f2pack(ka, kb), f2pack(Cs.x, Cs.y));
                    kahan2_fma(snu, enu, G, DZ);
                    kahan2_fma(sw, ew, G, DX);
                }
            } else if (F32) {
                for (int jj = 0; jj < cnt; ++jj) {
                    const float dx = (float)(tx - s_x[jj]);
                    const float dz = (float)(tz - s_z[jj]);
                    const float r2 = fmaf(dx, dx, dz * dz);
                    if (!(r2 > 1e-15f)) continue;  // skip_close (computeInducedAt :89)
                    float K = rcp_approx(r2);
                    if (r2 < s_thrf[jj]) K = core_kernel_expm1(r2, s_rsf[jj], K);
                    const float g = K * s_cf[jj];
                    kahan(su, cu, -g * dz);
                    kahan(sws, cws, g * dx);
                }
            } else {
                for (int jj = 0; jj < cnt; ++jj) {
                    const double dx = dsub(tx, s_x[jj]);
                    const double dz = dsub(tz, s_z[jj]);
                    const double r2 = dadd(dmul(dx, dx), dmul(dz, dz));
                    if (J.skip_close && !(r2 > 1e-15)) continue;
                    double K;
                    if (r2 < s_thr[jj]) K = ddiv(dsub(1.0, exp(dmul(-r2, s_rs[jj]))), r2);
                    else K = __drcp_rn(r2);  // correctly rounded: the same value as 1.0 / r2
                    uu = dsub(uu, dmul(dmul(K, dz), s_c[jj]));
                    ww = dadd(ww, dmul(dmul(K, dx), s_c[jj]));
                }
            }
        }
        if (packed) {
            uu = -(((double)f2lo(snu) + (double)f2lo(enu)) + ((double)f2hi(snu) + (double)f2hi(enu)));
            ww = ((double)f2lo(sw) + (double)f2lo(ew)) + ((double)f2hi(sw) + (double)f2hi(ew));
        } else if (F32) {
            uu = (double)su - (double)cu;
            ww = (double)sws - (double)cws;
        }
        if (t < J.nt) J.part[(uint64_t)c * J.npad + t] = make_double2(uu, ww);
        if (ttile == 0 && J.circ_part) {
            for (int o = 16; o > 0; o >>= 1) csum += __shfl_xor_sync(0xffffffffu, csum, o);
            if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = csum;
            __syncthreads();
            if (threadIdx.x == 0) {
                double a = 0.0;
                for (int q = 0; q < 8; ++q) a += s_red[q];
                J.circ_part[c] = a;
            }
        }
    }
}

__global__ void k_at_combine(const AtJob* __restrict__ jobs, double* __restrict__ u,
                             double* __restrict__ w) {
    const AtJob J = jobs[0];
    const uint32_t ns = J.pns ? *J.pns : J.ns;
    const uint32_t nchunk = (ns + J.chunk - 1) / J.chunk;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < J.nt; t += gridDim.x * blockDim.x) {
        double su = 0.0, sw = 0.0;
        for (uint32_t c = 0; c < nchunk; ++c) {
            const double2 v = J.part[(uint64_t)c * J.npad + t];
            su += v.x;
            sw += v.y;
        }
        u[t] = su * kRpi2;
        w[t] = sw * kRpi2;
    }
}

// b_i = (Ux + u_i) enx_i + (Uz + w_i) enz_i, b_np = -sum(circ)
// (src/VortexSheet.cpp:206-210).  Block (x, k) finishes targets 32x .. 32x+31
// of simulation k: warp w sums chunks w, w + 8, ... for its lane's target and
// the eight warp sums are added in warp order; block x = 0 also sums the
// Kelvin row's circulation partials (thread t takes chunks t, t + 256, ...,
// then a fixed shuffle tree and the warp sums in order).  The order depends
// only on the simulation's chunk count, never on the batch.
__global__ void __launch_bounds__(256) k_rhs_combine(const InstDesc* __restrict__ table,
                                                     InstState* __restrict__ st,
                                                     const ListEntry* __restrict__ list,
                                                     const AtJob* __restrict__ jobs) {
    __shared__ double s_u[8][32], s_w[8][32], s_c[8];
    const int k = blockIdx.y;
    const ListEntry e = list[k];
    const InstDesc& d = table[e.inst];
    const AtJob J = jobs[k];
    const uint32_t ns = st[e.inst].n;
    const uint32_t nchunk = (ns + J.chunk - 1) / J.chunk;
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * 32 + lane;
    const bool targets = (int)(blockIdx.x * 32) < d.np;  // block-uniform
    if (targets) {
        double su = 0.0, sw = 0.0;
        if (i < d.np)
            for (uint32_t c = wid; c < nchunk; c += 8) {
                const double2 v = J.part[(uint64_t)c * J.npad + i];
                su += v.x;
                sw += v.y;
            }
        s_u[wid][lane] = su;
        s_w[wid][lane] = sw;
    }
    __syncthreads();
    if (targets && threadIdx.x < 32 && i < d.np) {
        double su = 0.0, sw = 0.0;
        for (int q = 0; q < 8; ++q) {
            su += s_u[q][lane];
            sw += s_w[q][lane];
        }
        const double ui = dmul(su, kRpi2), wi = dmul(sw, kRpi2);
        d.b[i] = dadd(dmul(dadd(d.ux, ui), d.enx[i]), dmul(dadd(d.uz, wi), d.enz[i]));
    }
    if (blockIdx.x == 0) {  // block-uniform
        double tc = 0.0;
        for (uint32_t c = threadIdx.x; c < nchunk; c += 256) tc += J.circ_part[c];
        for (int o = 16; o > 0; o >>= 1) tc += __shfl_xor_sync(0xffffffffu, tc, o);
        if (lane == 0) s_c[wid] = tc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double a = 0.0;
            for (int q = 0; q < 8; ++q) a += s_c[q];
            d.b[d.np] = -a;
            st[e.inst].totalcirc = a;
        }
    }
}

__global__ void k_build_rhs_jobs(const InstDesc* __restrict__ table, InstState* __restrict__ st,
                                 const ListEntry* __restrict__ list, int nlist,
                                 double2* rhs_part, double* circ_part, AtJob* jobs) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nlist) return;
    const ListEntry e = list[k];
    const InstDesc& d = table[e.inst];
    AtJob J;
    J.tx = d.xc;
    J.tz = d.zc;
    J.nt = (uint32_t)d.np;
    J.skip_close = 0;  // solvevortexsheet has no close-pair skip (src/VortexSheet.cpp:186-203)
    J.sx = d.x;
    J.sz = d.z;
    J.sc = d.circ;
    J.ss = d.sigma;
    J.pns = &st[e.inst].n;
    J.ns = 0;
    J.npad = e.npad;
    J.chunk = e.rhs_chunk;
    J.part = rhs_part + e.roff;
    J.circ_part = circ_part + e.cofs;
    jobs[k] = J;
}

}  // namespace

size_t cub_sort_bytes(uint64_t total) {
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                    (const uint32_t*)nullptr, (uint32_t*)nullptr, (int64_t)total,
                                    0, 48);
    return bytes;
}

void biot_savart_prepare(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
                         int precision, const Workspace& ws, int sms, cudaStream_t s) {
    {  // both precisions evaluate over Morton-sorted tiles
        const int g = (int)std::min<uint64_t>((ws.total_cap + 255) / 256, (uint64_t)sms * 16);
        k_keys<<<g, 256, 0, s>>>(table, st, list, nlist, ws.total_cap, ws.keys_in, ws.vals_in);
        size_t bytes = ws.cub_bytes;
        cub::DeviceRadixSort::SortPairs(ws.cub_tmp, bytes, ws.keys_in, ws.keys_out, ws.vals_in,
                                        ws.perm, (int64_t)ws.total_cap, 0, ws.key_bits, s);
    }
    const uint32_t* perm = ws.perm;
    double2* pxz = precision == kF32 ? reinterpret_cast<double2*>(ws.packed) : nullptr;
    float4* pf = precision == kF32 ? reinterpret_cast<float4*>(ws.packed + ws.packed_cap / 2)
                                   : nullptr;
    if (precision == kF32)  // 0x80808080 per exponent: below any bound k_pack writes
        cudaMemsetAsync(ws.mexp, 0x80, sizeof(int) * 4 * kTableCap, s);
    k_pack<<<sms * 8, kBsST, 0, s>>>(table, st, list, nlist, perm, ws.packed, pxz, pf, ws.meta,
                                     precision == kF32 ? ws.mexp : nullptr);
    cudaMemsetAsync(ws.work, 0, sizeof(unsigned), s);
}

void biot_savart_compute(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
                         int precision, const Workspace& ws, int sms, cudaStream_t s,
                         const PairConfig& cfg) {
    (void)table;
    if (precision == kF32) {
        const double2* pxz = reinterpret_cast<const double2*>(ws.packed);
        const float4* pf = reinterpret_cast<const float4*>(ws.packed + ws.packed_cap / 2);
        const int g = sms * std::max(1, std::min(cfg.ctas, kSelfMinBlocks));
        cudaMemsetAsync(ws.macc, 0, 16 * ws.total_cap, s);
        k_self_f32<kSelfMinBlocks><<<g, 32 * kWWarps, 0, s>>>(st, list, nlist, pxz, pf, ws.meta,
                                                             ws.macc, ws.mexp, ws.work);
    } else {
        k_self_f64<<<sms * kF64Ctas, kBsThreads, 0, s>>>(st, list, nlist, ws.packed, ws.meta,
                                                             ws.part, ws.work);
    }
}

void biot_savart_finish(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
                        int precision, const Workspace& ws, int sms, cudaStream_t s) {
    const bool f32 = precision == kF32;
    k_self_combine<<<sms * 8, 256, 0, s>>>(table, st, list, nlist, ws.perm, ws.part,
                                           f32 ? ws.macc : nullptr, ws.mexp);
}

void biot_savart_self(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
                      int precision, const Workspace& ws, int sms, cudaStream_t s,
                      const PairConfig& cfg) {
    biot_savart_prepare(table, st, list, nlist, precision, ws, sms, s);
    biot_savart_compute(table, st, list, nlist, precision, ws, sms, s, cfg);
    biot_savart_finish(table, st, list, nlist, precision, ws, sms, s);
}

void sheet_rhs(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
               int max_np, int precision, const Workspace& ws, int sms, cudaStream_t s) {
    static_assert(sizeof(AtJob) <= 256, "job record size");
    AtJob* jobs = reinterpret_cast<AtJob*>(ws.jobs);
    k_build_rhs_jobs<<<(nlist + 127) / 128, 128, 0, s>>>(table, st, list, nlist, ws.rhs_part,
                                                         ws.circ_part, jobs);
    if (precision == kF32) k_at<true><<<sms * 4, 256, 0, s>>>(jobs, nlist);
    else k_at<false><<<sms * 4, 256, 0, s>>>(jobs, nlist);
    k_rhs_combine<<<dim3((max_np + 31) / 32, nlist), 256, 0, s>>>(table, st, list, jobs);
}

size_t direct_at_part_elems(uint32_t ns, uint32_t nt) {
    const size_t nchunk = (ns + kAtChunk - 1) / kAtChunk;
    const size_t npad = (nt + 255) / 256 * 256;
    return std::max<size_t>(1, nchunk) * std::max<size_t>(npad, 256) + 64;
}

void direct_at_raw(const double* x, const double* z, const double* circ, const double* sigma,
                   uint32_t ns, const double* tx, const double* tz, uint32_t nt, double* u,
                   double* w, int precision, int skip_close, double2* part, int sms,
                   cudaStream_t s) {
    // The job record sits in the last 64 entries of the partials buffer.
    const size_t elems = direct_at_part_elems(ns, nt);
    AtJob* job = reinterpret_cast<AtJob*>(part + elems - 64);
    AtJob J;
    J.tx = tx;
    J.tz = tz;
    J.nt = nt;
    J.skip_close = skip_close;
    J.sx = x;
    J.sz = z;
    J.sc = circ;
    J.ss = sigma;
    J.pns = nullptr;
    J.ns = ns;
    J.npad = (int)std::max<size_t>((nt + 255) / 256 * 256, 256);
    J.chunk = kAtChunk;
    J.part = part;
    J.circ_part = nullptr;
    cudaMemcpyAsync(job, &J, sizeof(AtJob), cudaMemcpyHostToDevice, s);
    if (ns > 0) {
        if (precision == kF32) k_at<true><<<sms * 4, 256, 0, s>>>(job, 1);
        else k_at<false><<<sms * 4, 256, 0, s>>>(job, 1);
        k_at_combine<<<std::max<uint32_t>(1, std::min<uint32_t>((nt + 255) / 256, sms * 8)), 256, 0,
                       s>>>(job, u, w);
    } else {
        cudaMemsetAsync(u, 0, sizeof(double) * nt, s);
        cudaMemsetAsync(w, 0, sizeof(double) * nt, s);
    }
}

// ---- at-target velocity with fixed, library-owned scratch -------------------
// For callers that must not allocate device memory (see
// dvm_biot_savart_at_noalloc in include/dvm_cuda.h).  The chunk partials of
// k_at live in this file-scope array instead of a caller- or context-owned
// buffer; every GPU that loads the library holds it until the process exits.
namespace {

constexpr size_t kNoAllocElems = 262144;  // double2 entries: 4 MiB per device
constexpr size_t kNoAllocJobElems = 64;   // tail entries that hold the job record
static __device__ __align__(256) double2 g_noalloc_scratch[kNoAllocElems];

__global__ void k_write_job(AtJob* dst, AtJob job) { *dst = job; }

}  // namespace

}  // namespace dvmk

extern "C" int dvm_biot_savart_at_noalloc(const double* x, const double* z, const double* circ,
                                          const double* sigma, uint64_t ns, const double* tx,
                                          const double* tz, uint64_t nt, double* u, double* w,
                                          int precision, int skip_close, void* stream) {
    using namespace dvmk;
    if (nt && (!tx || !tz || !u || !w)) return report_error(1, "null target or output array");
    if (ns && (!x || !z || !circ || !sigma)) return report_error(1, "null source array");
    if (precision != kF64 && precision != kF32) return report_error(1, "bad precision");
    if (nt == 0) return 0;
    const size_t nchunk = (ns + kAtChunk - 1) / kAtChunk;
    const size_t npad = std::max<size_t>((nt + 255) / 256 * 256, 256);
    if (ns > 0xF0000000ull || nt > 0xF0000000ull ||
        nchunk * npad > kNoAllocElems - kNoAllocJobElems) {
        return report_error(
            1, "dvm_biot_savart_at_noalloc: ceil(ns/4096) * ceil(nt/256) * 256 must not exceed "
               "262080 (fixed 4 MiB scratch); use dvm_biot_savart_at_device for larger sizes");
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0)
        return report_error(3, "dvm_biot_savart_at_noalloc: no current CUDA device");
    // The array's device address, looked up with the device current on every
    // call (host code cannot use the symbol itself).  Not cached: a device
    // reset reloads the library's device code, and the array may then move.
    // The first call on a device also loads that code, which is why it should
    // come before any stream capture.
    void* scratch_p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&scratch_p, g_noalloc_scratch);
    if (e != cudaSuccess)
        return report_error(3, (std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e)).c_str());
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess)
        return report_error(3, (std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(e)).c_str());
    double2* const scratch = static_cast<double2*>(scratch_p);
    if (ns == 0) {  // no sources: zero velocity, as the reference's empty loop gives
        if (cudaMemsetAsync(u, 0, sizeof(double) * nt, s) != cudaSuccess ||
            cudaMemsetAsync(w, 0, sizeof(double) * nt, s) != cudaSuccess)
            return report_error(3, "cudaMemsetAsync failed");
        return 0;
    }
    AtJob J;
    J.tx = tx;
    J.tz = tz;
    J.nt = (uint32_t)nt;
    J.skip_close = skip_close ? 1 : 0;
    J.sx = x;
    J.sz = z;
    J.sc = circ;
    J.ss = sigma;
    J.pns = nullptr;
    J.ns = (uint32_t)ns;
    J.npad = (int)npad;
    J.chunk = kAtChunk;
    J.part = scratch;  // every entry read by k_at_combine is written by k_at first
    J.circ_part = nullptr;
    AtJob* job = reinterpret_cast<AtJob*>(scratch + (kNoAllocElems - kNoAllocJobElems));
    k_write_job<<<1, 1, 0, s>>>(job, J);
    if (precision == kF32) k_at<true><<<sms * 4, 256, 0, s>>>(job, 1);
    else k_at<false><<<sms * 4, 256, 0, s>>>(job, 1);
    const unsigned cb = (unsigned)std::min<uint64_t>((nt + 255) / 256, (uint64_t)sms * 8);
    k_at_combine<<<std::max(1u, cb), 256, 0, s>>>(job, u, w);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return report_error(3, (std::string("dvm_biot_savart_at_noalloc launch: ") +
                                cudaGetErrorString(e)).c_str());
    return 0;
}
