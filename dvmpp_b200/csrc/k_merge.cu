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
#include <cfloat>
#include <cmath>

#include <cub/cub.cuh>

#include "dvm_device.cuh"
#include "dvm_internal.h"

namespace dvmk {
namespace {

constexpr int kMergeThreads = 1024;

__global__ void __launch_bounds__(kMergeThreads, 1)
    k_merge_greedy(double* __restrict__ x, double* __restrict__ z, double* __restrict__ circ,
                   double* __restrict__ sigma, double* __restrict__ u, double* __restrict__ w,
                   double* __restrict__ uvs, double* __restrict__ wvs, uint32_t n, double thr,
                   uint32_t* __restrict__ keep, uint32_t* __restrict__ count) {
    using Reduce = cub::BlockReduce<uint32_t, kMergeThreads>;
    __shared__ typename Reduce::TempStorage red;
    __shared__ double si[4];  // x, z, circ, sigma of the current absorber
    __shared__ uint32_t s_best;
    const uint32_t tid = threadIdx.x;
    for (uint32_t p = tid; p < n; p += kMergeThreads) keep[p] = 1u;
    __syncthreads();
    uint32_t merges = 0;
    for (uint32_t i = 0; i + 1 < n; ++i) {
        if (!keep[i]) continue;  // every thread reads the same value
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
            for (uint32_t j = j0 + tid; j < n; j += kMergeThreads) {
                if (!keep[j]) continue;
                const double gj = circ[j];
                const double gs = dadd(gi, gj);
                if (fabs(gs) < 1e-15) continue;
                const double dx = dsub(xi, x[j]), dz = dsub(zi, z[j]);
                const double d2 = dadd(dmul(dx, dx), dmul(dz, dz));
                const double a = fabs(dmul(gi, gj)), b = dmul(thr, fabs(gs));
                if (a < 1e100 && b < 1e100 && a > 1e-140 && b > 1e-140 &&
                    dmul(dmul(a, a), d2) > dmul(dmul(b, b), 1.000000000001))
                    continue;  // cannot pass the exact test below
                const double crit = dmul(fabs(ddiv(dmul(gi, gj), gs)), __dsqrt_rn(d2));
                if (crit < thr) {
                    best = j;  // this thread's candidates ascend: its first is its least
                    break;
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
    size_t keep, pos, tmp, tmp_bytes, t, count, bytes;
};

MLayout mlayout(uint32_t n) {
    size_t scan_b = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_b, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                  (int64_t)std::max<uint32_t>(n, 1));
    MLayout L{};
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += (bytes + 255) / 256 * 256;
        return o;
    };
    L.keep = take(4ull * n + 4);
    L.pos = take(4ull * n + 4);
    L.tmp_bytes = scan_b + 256;
    L.tmp = take(L.tmp_bytes);
    L.t = take(8 * 8ull * n + 8);
    L.count = take(64);
    L.bytes = off;
    return L;
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
    if (n < 2) {
        cudaMemsetAsync(count, 0, sizeof(uint32_t), s);
        return;
    }
    k_merge_greedy<<<1, kMergeThreads, 0, s>>>(a.x, a.z, a.circ, a.sigma, a.u, a.w, a.uvs, a.wvs,
                                               n, threshold, keep, count);
    size_t tb = L.tmp_bytes;
    cub::DeviceScan::ExclusiveSum(b + L.tmp, tb, keep, pos, (int64_t)n, s);
    const int grid = sms * 4;
    k_merge_scatter<<<grid, 256, 0, s>>>(count, n, keep, pos, a, t);
    k_merge_copyback<<<grid, 256, 0, s>>>(count, n, t, a, id, n_dev);
}

}  // namespace dvmk
