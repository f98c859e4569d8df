// Vortex merging, VortexBlobs::merge_blobs (src/VortexBlobs.cpp:110-209),
// hooked at src/DVMBase.cpp:124-132.
//
// The reference merges greedily in index order: each surviving blob i absorbs,
// one after another, every later unmerged j with |gi gj / (gi + gj)| |xi - xj|
// < threshold, where i's position, circulation and core size are updated after
// every absorption; then merged blobs are removed (stable) and IDs renumbered.
// The result depends on that order, so it is reproduced exactly: one block
// walks the absorbers i in order, and for each it scans all later blobs in
// parallel, taking the FIRST qualifying j (a block-wide minimum), merging it
// and rescanning from j + 1 with i's new state.  Every arithmetic step is the
// reference's, in FP64 with one rounding per operation, so the merged state is
// bit-identical.  A division-free pre-test rejects pairs that cannot pass:
// crit < thr implies (|gi gj| d)^2 < (thr |gi + gj|)^2, and the test keeps a
// 1e-12 relative margin so rounding can never reject a pair the exact formula
// would accept.
//
// Candidates are found through a cell grid when that is safe: a later blob j
// keeps its original position until it is scanned, and since |gi + gj| <=
// |gi| + |gj| a pair can pass only if |xi - xj| < thr (1/|gj| + 1/|gi|).  Blobs
// with the smallest |g| (at most kSmallList of them, plus any non-finite one)
// sit in a short list scanned at every pass; the others are bucketed by cell,
// and a pass searches the cells within thr (1/g_cut + 1/|gi|) of the absorber
// (g_cut: the smallest |g| in the grid), falling back to the full scan when that
// radius is large or undefined.  The minimum over the candidates is the same
// first qualifying j as the full scan's, so the result is unchanged.
//
// Most blobs absorb nothing.  A blob's state is still its original one when its
// turn comes, and its later candidates then are a subset of the original later
// blobs with their original states, so a blob with no qualifying partner among
// those can be skipped: all SMs find, in parallel, the blobs that have one, and
// the sequential walk visits only them.
#include <cfloat>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include <cub/cub.cuh>

#include "dvm_device.cuh"
#include "dvm_internal.h"

namespace dvmk {
namespace {

constexpr int kMergeThreads = 1024;
constexpr uint32_t kSmallList = 2048;  // blobs kept out of the grid, at most
constexpr int kGridMax = 1024;         // cells per axis, at most
constexpr int kCellReach = 8;          // a pass searches at most this many cells of radius

struct MergeGrid {
    double x0, z0, inv_h, h, g_cut;
    int nxc, nzc, enabled;
    const uint32_t* svals;   // blob indices, cell-sorted (index order within a cell)
    const uint32_t* cstart;  // per cell
    const uint32_t* cend;
    const uint32_t* n_grid;  // svals[n_grid .. n): the short list, in index order
};

// The reference's test for the pair (i's current state, j): crit < thr.
__device__ __forceinline__ bool merge_test(double xi, double zi, double gi, double xj, double zj,
                                           double gj, double thr) {
    const double gs = dadd(gi, gj);
    if (fabs(gs) < 1e-15) return false;
    const double dx = dsub(xi, xj), dz = dsub(zi, zj);
    const double d2 = dadd(dmul(dx, dx), dmul(dz, dz));
    const double a = fabs(dmul(gi, gj)), b = dmul(thr, fabs(gs));
    if (a < 1e100 && b < 1e100 && a > 1e-140 && b > 1e-140 &&
        dmul(dmul(a, a), d2) > dmul(dmul(b, b), 1.000000000001))
        return false;  // cannot pass the exact test below
    const double crit = dmul(fabs(ddiv(dmul(gi, gj), gs)), __dsqrt_rn(d2));
    return crit < thr;
}

// Cell range to search for absorber state (xi, zi, gi); false: scan everything.
__device__ __forceinline__ bool cell_range(const MergeGrid& G, double xi, double zi, double gi,
                                           double thr, long long& cx0, long long& cx1,
                                           long long& cz0, long long& cz1) {
    if (!G.enabled) return false;
    const double R = thr * (1.0 / G.g_cut + 1.0 / fabs(gi)) * (1.0 + 1e-9);
    if (!(R < kCellReach * G.h) || !(fabs(xi) < 1e300) || !(fabs(zi) < 1e300)) return false;
    // cell coordinates clamped as doubles before the integer conversion
    auto cell = [&](double v, int nc) {
        return (long long)floor(fmin(fmax(v, -2.0), (double)nc + 1.0));
    };
    cx0 = max(0LL, cell((xi - R - G.x0) * G.inv_h, G.nxc) - 1);
    cx1 = min((long long)G.nxc - 1, cell((xi + R - G.x0) * G.inv_h, G.nxc) + 1);
    cz0 = max(0LL, cell((zi - R - G.z0) * G.inv_h, G.nzc) - 1);
    cz1 = min((long long)G.nzc - 1, cell((zi + R - G.z0) * G.inv_h, G.nzc) + 1);
    return true;
}

// Whether blob i, in its original state, has a qualifying later partner.
__global__ void k_mg_absorbers(const double* __restrict__ x, const double* __restrict__ z,
                               const double* __restrict__ circ, uint32_t n, double thr,
                               MergeGrid G, uint32_t* __restrict__ flag) {
    const uint32_t n_grid = G.enabled ? G.n_grid[0] : 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double xi = x[i], zi = z[i], gi = circ[i];
        bool found = false;
        long long cx0, cx1, cz0, cz1;
        if (cell_range(G, xi, zi, gi, thr, cx0, cx1, cz0, cz1)) {
            for (long long cz = cz0; cz <= cz1 && !found; ++cz)
                for (long long cx = cx0; cx <= cx1 && !found; ++cx) {
                    const uint64_t c = (uint64_t)cz * G.nxc + cx;
                    for (uint32_t q = G.cstart[c]; q < G.cend[c]; ++q) {
                        const uint32_t j = G.svals[q];
                        if (j > i && merge_test(xi, zi, gi, x[j], z[j], circ[j], thr)) {
                            found = true;
                            break;
                        }
                    }
                }
            for (uint32_t q = n_grid; q < n && !found; ++q) {
                const uint32_t j = G.svals[q];
                found = j > i && merge_test(xi, zi, gi, x[j], z[j], circ[j], thr);
            }
        } else {
            for (uint32_t j = i + 1; j < n && !found; ++j)
                found = merge_test(xi, zi, gi, x[j], z[j], circ[j], thr);
        }
        flag[i] = found ? 1u : 0u;
    }
}

__global__ void __launch_bounds__(kMergeThreads, 1)
    k_merge_greedy(double* __restrict__ x, double* __restrict__ z, double* __restrict__ circ,
                   double* __restrict__ sigma, double* __restrict__ u, double* __restrict__ w,
                   double* __restrict__ uvs, double* __restrict__ wvs, uint32_t n, double thr,
                   MergeGrid G, const uint32_t* __restrict__ absorbers,
                   const uint32_t* __restrict__ n_abs, uint32_t* __restrict__ keep,
                   uint32_t* __restrict__ count) {
    using Reduce = cub::BlockReduce<uint32_t, kMergeThreads>;
    __shared__ typename Reduce::TempStorage red;
    __shared__ double si[4];  // x, z, circ, sigma of the current absorber
    __shared__ uint32_t s_best;
    const uint32_t tid = threadIdx.x;
    for (uint32_t p = tid; p < n; p += kMergeThreads) keep[p] = 1u;
    const uint32_t n_grid = G.enabled ? G.n_grid[0] : 0;
    __syncthreads();
    uint32_t merges = 0;
    const uint32_t na = n_abs[0];
    for (uint32_t t = 0; t < na; ++t) {
        const uint32_t i = absorbers[t];  // ascending: the reference's order
        if (!keep[i]) continue;           // every thread reads the same value
        if (tid == 0) {
            si[0] = x[i];
            si[1] = z[i];
            si[2] = circ[i];
            si[3] = sigma[i];
        }
        __syncthreads();
        uint32_t j0 = i + 1;
        while (j0 < n) {
            const double xi = si[0], zi = si[1], gi = si[2];
            uint32_t best = UINT32_MAX;
            // cell range of this pass (the same decision in every thread)
            long long cx0 = 0, cx1 = -1, cz0 = 0, cz1 = -1;
            const bool full = !cell_range(G, xi, zi, gi, thr, cx0, cx1, cz0, cz1);
            if (full) {
                for (uint32_t j = j0 + tid; j < n; j += kMergeThreads) {
                    if (!keep[j]) continue;
                    if (merge_test(xi, zi, gi, x[j], z[j], circ[j], thr)) {
                        best = j;  // this thread's candidates ascend: its first is its least
                        break;
                    }
                }
            } else {
                // one warp per cell, so the cells' bounds are loaded concurrently
                const long long ncx = cx1 - cx0 + 1, ncell = ncx * (cz1 - cz0 + 1);
                const uint32_t warp = tid >> 5, lane = tid & 31;
                for (long long k = warp; k < ncell; k += kMergeThreads / 32) {
                    const uint64_t c = (uint64_t)(cz0 + k / ncx) * G.nxc + (cx0 + k % ncx);
                    for (uint32_t q = G.cstart[c] + lane; q < G.cend[c]; q += 32) {
                        const uint32_t j = G.svals[q];
                        if (j < j0 || j >= best || !keep[j]) continue;
                        if (merge_test(xi, zi, gi, x[j], z[j], circ[j], thr)) best = j;
                    }
                }
                for (uint32_t q = n_grid + tid; q < n; q += kMergeThreads) {
                    const uint32_t j = G.svals[q];
                    if (j < j0 || j >= best || !keep[j]) continue;
                    if (merge_test(xi, zi, gi, x[j], z[j], circ[j], thr)) best = j;
                }
            }
            best = Reduce(red).Reduce(best, cub::Min());
            if (tid == 0) s_best = best;
            __syncthreads();
            best = s_best;
            if (best == UINT32_MAX) break;
            if (tid == 0) {
                const double gj = circ[best], gs = dadd(gi, gj);
                const double nx = ddiv(dadd(dmul(gi, xi), dmul(gj, x[best])), gs);
                const double nz = ddiv(dadd(dmul(gi, zi), dmul(gj, z[best])), gs);
                const double ns = ddiv(dadd(dmul(fabs(gi), si[3]), dmul(fabs(gj), sigma[best])),
                                       dadd(fabs(gi), fabs(gj)));
                si[0] = x[i] = nx;
                si[1] = z[i] = nz;
                si[2] = circ[i] = gs;
                si[3] = sigma[i] = ns;
                u[i] = w[i] = uvs[i] = wvs[i] = 0.0;
                keep[best] = 0u;
                ++merges;
            }
            __syncthreads();
            j0 = best + 1;
        }
        __syncthreads();
    }
    if (tid == 0) count[0] = merges;
}

// |g| as sortable bits (non-finite last) and the bounding box of the finite
// positions, per block.
__global__ void k_mg_stats(const double* __restrict__ x, const double* __restrict__ z,
                           const double* __restrict__ circ, uint32_t n,
                           uint64_t* __restrict__ gbits, double4* __restrict__ part) {
    double xmn = DBL_MAX, xmx = -DBL_MAX, zmn = DBL_MAX, zmx = -DBL_MAX;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const double g = fabs(circ[p]);
        gbits[p] = (g <= DBL_MAX) ? (uint64_t)__double_as_longlong(g) : 0x7FF0000000000000ull;
        if (fabs(x[p]) < 1e300 && fabs(z[p]) < 1e300) {
            xmn = fmin(xmn, x[p]);
            xmx = fmax(xmx, x[p]);
            zmn = fmin(zmn, z[p]);
            zmx = fmax(zmx, z[p]);
        }
    }
    using R = cub::BlockReduce<double, 256>;
    __shared__ typename R::TempStorage t;
    xmn = R(t).Reduce(xmn, cub::Min());
    __syncthreads();
    xmx = R(t).Reduce(xmx, cub::Max());
    __syncthreads();
    zmn = R(t).Reduce(zmn, cub::Min());
    __syncthreads();
    zmx = R(t).Reduce(zmx, cub::Max());
    if (threadIdx.x == 0) part[blockIdx.x] = make_double4(xmn, xmx, zmn, zmx);
}

__global__ void k_mg_classify(const double* __restrict__ x, const double* __restrict__ z,
                              const double* __restrict__ circ, uint32_t n, double x0, double z0,
                              double inv_h, int nxc, int nzc, double g_cut,
                              uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const uint64_t sentinel = (uint64_t)nxc * nzc;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const double g = fabs(circ[p]);
        uint64_t k = sentinel;
        if (g >= g_cut && g <= DBL_MAX && fabs(x[p]) < 1e300 && fabs(z[p]) < 1e300) {
            const long long cx = (long long)floor((x[p] - x0) * inv_h);
            const long long cz = (long long)floor((z[p] - z0) * inv_h);
            if (cx >= 0 && cx < nxc && cz >= 0 && cz < nzc) k = (uint64_t)cz * nxc + cx;
        }
        keys[p] = k;
        vals[p] = p;
    }
}

__global__ void k_mg_bounds(const uint64_t* __restrict__ skeys, uint32_t n, uint64_t ncells,
                            uint32_t* __restrict__ cstart, uint32_t* __restrict__ cend,
                            uint32_t* __restrict__ n_grid) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const uint64_t k = skeys[q];
        if (k >= ncells) {
            if (q == 0 || skeys[q - 1] < ncells) n_grid[0] = q;
            continue;
        }
        if (q == 0 || skeys[q - 1] != k) cstart[k] = q;
        if (q == n - 1 || skeys[q + 1] != k) cend[k] = q + 1;
    }
}

__global__ void k_merge_scatter(const uint32_t* __restrict__ count, uint32_t n,
                                const uint32_t* __restrict__ keep, const uint32_t* __restrict__ pos,
                                MergeArrays a, MergeArrays t) {
    if (count[0] == 0) return;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        if (!keep[p]) continue;
        const uint32_t o = pos[p];
        t.x[o] = a.x[p];
        t.z[o] = a.z[p];
        t.circ[o] = a.circ[p];
        t.sigma[o] = a.sigma[p];
        t.u[o] = a.u[p];
        t.w[o] = a.w[p];
        t.uvs[o] = a.uvs[p];
        t.wvs[o] = a.wvs[p];
    }
}

__global__ void k_merge_copyback(const uint32_t* __restrict__ count, uint32_t n, MergeArrays t,
                                 MergeArrays a, uint32_t* __restrict__ id,
                                 uint32_t* __restrict__ n_dev) {
    const uint32_t c = count[0];
    if (c == 0) return;  // nothing merged: IDs unchanged (src/VortexBlobs.cpp:171-173)
    const uint32_t m = n - c;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x) {
        a.x[q] = t.x[q];
        a.z[q] = t.z[q];
        a.circ[q] = t.circ[q];
        a.sigma[q] = t.sigma[q];
        a.u[q] = t.u[q];
        a.w[q] = t.w[q];
        a.uvs[q] = t.uvs[q];
        a.wvs[q] = t.wvs[q];
        if (id) id[q] = q;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && n_dev) n_dev[0] = m;
}

struct MLayout {
    size_t keep, pos, tmp, tmp_bytes, t, count, gbits, gsorted, keys, skeys, vals, svals, cstart,
        cend, part, scal, aflag, alist, bytes;
};

constexpr int kStatBlocks = 256;

int sort_bits(uint64_t v) {
    int b = 1;
    while (b < 64 && (1ull << b) <= v) ++b;
    return b;
}

MLayout mlayout(uint32_t n) {
    const uint64_t ncells = (uint64_t)kGridMax * kGridMax;
    size_t scan_b = 0, sk_b = 0, sp_b = 0, sel_b = 0;
    const int64_t nn = (int64_t)std::max<uint32_t>(n, 1);
    cub::DeviceScan::ExclusiveSum(nullptr, scan_b, (const uint32_t*)nullptr, (uint32_t*)nullptr, nn);
    cub::DeviceRadixSort::SortKeys(nullptr, sk_b, (const uint64_t*)nullptr, (uint64_t*)nullptr, nn);
    cub::DeviceRadixSort::SortPairs(nullptr, sp_b, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                    (const uint32_t*)nullptr, (uint32_t*)nullptr, nn, 0,
                                    sort_bits(ncells));
    cub::DeviceSelect::Flagged(nullptr, sel_b, cub::CountingInputIterator<uint32_t>(0),
                               (const uint32_t*)nullptr, (uint32_t*)nullptr, (uint32_t*)nullptr,
                               nn);
    MLayout L{};
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += (bytes + 255) / 256 * 256;
        return o;
    };
    L.keep = take(4ull * n + 4);
    L.pos = take(4ull * n + 4);
    L.tmp_bytes = std::max({scan_b, sk_b, sp_b, sel_b}) + 256;
    L.tmp = take(L.tmp_bytes);
    L.t = take(8 * 8ull * n + 8);
    L.count = take(64);
    L.gbits = take(8ull * n + 8);
    L.gsorted = take(8ull * n + 8);
    L.keys = take(8ull * n + 8);
    L.skeys = take(8ull * n + 8);
    L.vals = take(4ull * n + 4);
    L.svals = take(4ull * n + 4);
    L.cstart = take(4 * ncells);
    L.cend = take(4 * ncells);
    L.part = take(sizeof(double4) * kStatBlocks);
    L.scal = take(64);
    L.aflag = take(4ull * n + 4);
    L.alist = take(4ull * n + 4);
    L.bytes = off;
    return L;
}

// Builds the candidate grid (synchronises the stream once to size it); leaves
// G.enabled = 0 when a grid would not narrow the search.
MergeGrid build_grid(const MergeArrays& a, uint32_t n, double thr, const MLayout& L, char* b,
                     cudaStream_t s) {
    MergeGrid G{};
    G.enabled = 0;
    if (n < 4096) return G;  // the full scan is cheap
    uint64_t* gbits = reinterpret_cast<uint64_t*>(b + L.gbits);
    uint64_t* gsorted = reinterpret_cast<uint64_t*>(b + L.gsorted);
    double4* part = reinterpret_cast<double4*>(b + L.part);
    k_mg_stats<<<kStatBlocks, 256, 0, s>>>(a.x, a.z, a.circ, n, gbits, part);
    size_t tb = L.tmp_bytes;
    cub::DeviceRadixSort::SortKeys(b + L.tmp, tb, gbits, gsorted, (int64_t)n, 0, 64, s);
    const uint32_t k = std::min<uint32_t>(kSmallList, n);
    uint64_t h_cut = 0, h_med = 0;
    std::vector<double4> h_part(kStatBlocks);
    cudaMemcpyAsync(&h_cut, gsorted + (k - 1), 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&h_med, gsorted + n / 2, 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h_part.data(), part, sizeof(double4) * kStatBlocks, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return G;
    double g_cut, g_med;
    std::memcpy(&g_cut, &h_cut, 8);
    std::memcpy(&g_med, &h_med, 8);
    double xmn = DBL_MAX, xmx = -DBL_MAX, zmn = DBL_MAX, zmx = -DBL_MAX;
    for (const double4& v : h_part) {
        xmn = std::min(xmn, v.x);
        xmx = std::max(xmx, v.y);
        zmn = std::min(zmn, v.z);
        zmx = std::max(zmx, v.w);
    }
    if (!(g_cut > 0) || !(g_cut <= DBL_MAX) || !(xmx >= xmn) || !(zmx >= zmn)) return G;
    const double span = std::max({xmx - xmn, zmx - zmn, 1e-300});
    const double r_typ = thr * (1.0 / g_cut + 1.0 / g_med);
    if (!(r_typ > 0) || !(r_typ < span / 4)) return G;  // a grid would not narrow the search
    const double h = std::max(r_typ, span / (kGridMax - 1));
    G.h = h;
    G.inv_h = 1.0 / h;
    G.x0 = xmn;
    G.z0 = zmn;
    G.nxc = std::min(kGridMax, (int)std::floor((xmx - xmn) * G.inv_h) + 1);
    G.nzc = std::min(kGridMax, (int)std::floor((zmx - zmn) * G.inv_h) + 1);
    G.g_cut = g_cut;
    const uint64_t ncells = (uint64_t)G.nxc * G.nzc;
    uint64_t* keys = reinterpret_cast<uint64_t*>(b + L.keys);
    uint64_t* skeys = reinterpret_cast<uint64_t*>(b + L.skeys);
    uint32_t* vals = reinterpret_cast<uint32_t*>(b + L.vals);
    uint32_t* svals = reinterpret_cast<uint32_t*>(b + L.svals);
    uint32_t* cstart = reinterpret_cast<uint32_t*>(b + L.cstart);
    uint32_t* cend = reinterpret_cast<uint32_t*>(b + L.cend);
    uint32_t* n_grid = reinterpret_cast<uint32_t*>(b + L.scal);
    k_mg_classify<<<256, 256, 0, s>>>(a.x, a.z, a.circ, n, G.x0, G.z0, G.inv_h, G.nxc, G.nzc,
                                      g_cut, keys, vals);
    tb = L.tmp_bytes;
    cub::DeviceRadixSort::SortPairs(b + L.tmp, tb, keys, skeys, vals, svals, (int64_t)n, 0,
                                    sort_bits(ncells), s);
    cudaMemsetAsync(cstart, 0, 4 * ncells, s);
    cudaMemsetAsync(cend, 0, 4 * ncells, s);
    cudaMemcpyAsync(n_grid, &n, sizeof(uint32_t), cudaMemcpyHostToDevice, s);
    k_mg_bounds<<<256, 256, 0, s>>>(skeys, n, ncells, cstart, cend, n_grid);
    cudaStreamSynchronize(s);  // the host value of n above must be copied before it goes
    G.svals = svals;
    G.cstart = cstart;
    G.cend = cend;
    G.n_grid = n_grid;
    G.enabled = 1;
    return G;
}

}  // namespace

size_t merge_scratch_bytes(uint32_t n) { return mlayout(n).bytes; }
size_t merge_count_offset(uint32_t n) { return mlayout(n).count; }

void merge_run(const MergeArrays& a, uint32_t* id, uint32_t n, double threshold,
               uint32_t* n_dev, uint32_t* count_dev, void* scratch, int sms, cudaStream_t s) {
    const MLayout L = mlayout(n);
    char* b = static_cast<char*>(scratch);
    uint32_t* keep = reinterpret_cast<uint32_t*>(b + L.keep);
    uint32_t* pos = reinterpret_cast<uint32_t*>(b + L.pos);
    double* t0 = reinterpret_cast<double*>(b + L.t);
    MergeArrays t{t0, t0 + n, t0 + 2ull * n, t0 + 3ull * n, t0 + 4ull * n, t0 + 5ull * n,
                  t0 + 6ull * n, t0 + 7ull * n};
    uint32_t* count = count_dev ? count_dev : reinterpret_cast<uint32_t*>(b + L.count);
    if (n < 2 || !(threshold > 0)) {  // crit >= 0 never passes a threshold <= 0
        cudaMemsetAsync(count, 0, sizeof(uint32_t), s);
        return;
    }
    const MergeGrid G = build_grid(a, n, threshold, L, b, s);
    uint32_t* aflag = reinterpret_cast<uint32_t*>(b + L.aflag);
    uint32_t* alist = reinterpret_cast<uint32_t*>(b + L.alist);
    uint32_t* n_abs = reinterpret_cast<uint32_t*>(b + L.scal) + 4;
    k_mg_absorbers<<<sms * 4, 256, 0, s>>>(a.x, a.z, a.circ, n, threshold, G, aflag);
    size_t sb = L.tmp_bytes;
    cub::DeviceSelect::Flagged(b + L.tmp, sb, cub::CountingInputIterator<uint32_t>(0), aflag,
                               alist, n_abs, (int64_t)n, s);
    k_merge_greedy<<<1, kMergeThreads, 0, s>>>(a.x, a.z, a.circ, a.sigma, a.u, a.w, a.uvs, a.wvs,
                                               n, threshold, G, alist, n_abs, keep, count);
    size_t tb = L.tmp_bytes;
    cub::DeviceScan::ExclusiveSum(b + L.tmp, tb, keep, pos, (int64_t)n, s);
    const int grid = sms * 4;
    k_merge_scatter<<<grid, 256, 0, s>>>(count, n, keep, pos, a, t);
    k_merge_copyback<<<grid, 256, 0, s>>>(count, n, t, a, id, n_dev);
}

}  // namespace dvmk
