// Remeshing onto a background mesh: the reference's BackgroundMesh
// (src/DVMBase.hpp:51, called at src/DVMBase.cpp:91-92, 160-164; options
// src/XmlHandler.cpp:191-201) whose source is not part of the reference.  Its
// behaviour is taken from the reference's tests (tests/unit/test_BackgroundMesh.cpp):
// tensor-product interpolation kernels M4' (support 2), M6 (support 3) and a
// Gaussian truncated at 3, partition of unity, conservation of circulation.
//
// Each blob whose kernel support lies inside the mesh gives its circulation to
// the mesh nodes with weight W(xi - i) W(zeta - j) (xi, zeta: the blob's
// position in node units); nodes whose circulation exceeds the threshold in
// magnitude become the new blobs (core size `sigma`, row-major node order),
// and blobs whose support leaves the mesh are kept unchanged after them (so
// no circulation leaks at the mesh edge).  The Gaussian weights are
// normalised per blob by their sum (the truncated Gaussian alone sums to
// 1 - 0.27 %).
//
// GPU layout: blobs are bucketed by cell with a stable radix sort, and every
// node gathers from the 2S x 2S cells around it in a fixed order (cells
// row-major, blobs in index order within a cell), so the sums are
// deterministic -- no atomics.
#include <cfloat>
#include <cmath>

#include <cub/cub.cuh>

#include "dvm_device.cuh"
#include "dvm_internal.h"

namespace dvmk {
namespace {

__device__ __forceinline__ double w_m4p(double r) {
    r = fabs(r);
    if (r < 1.0) return dadd(dsub(1.0, dmul(2.5, dmul(r, r))), dmul(1.5, dmul(dmul(r, r), r)));
    if (r < 2.0) {
        const double t = dsub(2.0, r);
        return dmul(dmul(dmul(0.5, t), t), dsub(1.0, r));
    }
    return 0.0;
}

__device__ __forceinline__ double pow5p(double x) {
    if (!(x > 0.0)) return 0.0;
    const double x2 = dmul(x, x);
    return dmul(dmul(x2, x2), x);
}

__device__ __forceinline__ double w_m6(double r) {
    r = fabs(r);
    if (!(r < 3.0)) return 0.0;
    const double s = dadd(dsub(pow5p(dsub(3.0, r)), dmul(6.0, pow5p(dsub(2.0, r)))),
                          dmul(15.0, pow5p(dsub(1.0, r))));
    return ddiv(s, 120.0);
}

__device__ __forceinline__ double w_gauss(double r) {
    r = fabs(r);
    if (!(r < 3.0)) return 0.0;
    return dmul(exp(dmul(-0.5, dmul(r, r))), 0.398942280401432677939946);  // 1/sqrt(2 pi)
}

__device__ __forceinline__ double weight(int kernel, double r) {
    return kernel == kRemeshM4p ? w_m4p(r) : kernel == kRemeshM6 ? w_m6(r) : w_gauss(r);
}

__device__ __forceinline__ int support(int kernel) { return kernel == kRemeshM4p ? 2 : 3; }

// Position in node units; false when not finite or far outside any mesh.
__device__ __forceinline__ bool node_coords(const RemeshGrid& g, double x, double z, double& xi,
                                            double& ze, long long& fx, long long& fz) {
    xi = ddiv(dsub(x, g.x0), g.dx);
    ze = ddiv(dsub(z, g.z0), g.dz);
    if (!(fabs(xi) < 1e9) || !(fabs(ze) < 1e9)) return false;
    fx = (long long)floor(xi);
    fz = (long long)floor(ze);
    return true;
}

__global__ void k_rm_classify(RemeshGrid g, const double* __restrict__ x,
                              const double* __restrict__ z, const double* __restrict__ circ,
                              uint32_t n, uint64_t* __restrict__ keys, uint32_t* __restrict__ vals,
                              double* __restrict__ gcirc, uint32_t* __restrict__ flags_out) {
    const uint64_t ncells = (uint64_t)g.nx * g.nz;
    const int S = support(g.kernel);
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        double xi, ze;
        long long fx, fz;
        bool in = node_coords(g, x[p], z[p], xi, ze, fx, fz);
        in = in && fx - (S - 1) >= 0 && fx + S <= g.nx - 1 && fz - (S - 1) >= 0 &&
             fz + S <= g.nz - 1;
        keys[p] = in ? (uint64_t)fz * g.nx + (uint64_t)fx : ncells;
        vals[p] = p;
        flags_out[p] = in ? 0u : 1u;  // kept unchanged
        double gc = circ[p];
        if (in && g.kernel == kRemeshGauss) {  // normalise the truncated weights
            double sx = 0.0, sz = 0.0;
            for (long long i = fx - (S - 1); i <= fx + S; ++i) sx = dadd(sx, w_gauss(dsub(xi, (double)i)));
            for (long long j = fz - (S - 1); j <= fz + S; ++j) sz = dadd(sz, w_gauss(dsub(ze, (double)j)));
            gc = ddiv(gc, dmul(sx, sz));
        }
        gcirc[p] = gc;
    }
}

__global__ void k_rm_bounds(const uint64_t* __restrict__ skeys, uint32_t n, uint64_t ncells,
                            uint32_t* __restrict__ cstart, uint32_t* __restrict__ cend) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const uint64_t k = skeys[q];
        if (k >= ncells) continue;
        if (q == 0 || skeys[q - 1] != k) cstart[k] = q;
        if (q == n - 1 || skeys[q + 1] != k) cend[k] = q + 1;
    }
}

__global__ void k_rm_gather(RemeshGrid g, const double* __restrict__ x, const double* __restrict__ z,
                            const double* __restrict__ gcirc, const uint32_t* __restrict__ svals,
                            const uint32_t* __restrict__ cstart, const uint32_t* __restrict__ cend,
                            double* __restrict__ node, uint32_t* __restrict__ flags) {
    const uint64_t nn = (uint64_t)g.nx * g.nz;
    const int S = support(g.kernel);
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nn;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const int i = (int)(k % g.nx), j = (int)(k / g.nx);
        double acc = 0.0;
        for (int b = max(0, j - S); b <= min(g.nz - 1, j + S - 1); ++b)
            for (int a = max(0, i - S); a <= min(g.nx - 1, i + S - 1); ++a) {
                const uint64_t c = (uint64_t)b * g.nx + a;
                for (uint32_t q = cstart[c]; q < cend[c]; ++q) {
                    const uint32_t p = svals[q];
                    const double xi = ddiv(dsub(x[p], g.x0), g.dx);
                    const double ze = ddiv(dsub(z[p], g.z0), g.dz);
                    const double wx = weight(g.kernel, dsub(xi, (double)i));
                    const double wz = weight(g.kernel, dsub(ze, (double)j));
                    acc = dadd(acc, dmul(dmul(wx, wz), gcirc[p]));
                }
            }
        node[k] = acc;
        flags[k] = fabs(acc) > g.threshold ? 1u : 0u;
    }
}

__global__ void k_rm_total(const uint32_t* __restrict__ flags, const uint32_t* __restrict__ pos,
                           uint64_t m, uint32_t cap, uint32_t* __restrict__ total,
                           int* __restrict__ ok, int* __restrict__ status,
                           uint32_t* __restrict__ need) {
    const uint64_t t = m ? (uint64_t)pos[m - 1] + flags[m - 1] : 0;
    total[0] = (uint32_t)t;
    if (need) need[0] = (uint32_t)t;
    ok[0] = t <= cap;
    if (t > cap && status) atomicCAS(status, 0, kErrCapacity);
}

__global__ void k_rm_scatter(RemeshGrid g, const double* __restrict__ x,
                             const double* __restrict__ z, const double* __restrict__ circ,
                             const double* __restrict__ sigma, uint32_t n,
                             const double* __restrict__ node, const uint32_t* __restrict__ flags,
                             const uint32_t* __restrict__ pos, uint32_t cap,
                             double* __restrict__ tx, double* __restrict__ tz,
                             double* __restrict__ tc, double* __restrict__ ts) {
    const uint64_t nn = (uint64_t)g.nx * g.nz, m = nn + n;
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < m;
         k += (uint64_t)gridDim.x * blockDim.x) {
        if (!flags[k]) continue;
        const uint32_t o = pos[k];
        if (o >= cap) continue;
        if (k < nn) {
            const int i = (int)(k % g.nx), j = (int)(k / g.nx);
            tx[o] = dadd(g.x0, dmul((double)i, g.dx));
            tz[o] = dadd(g.z0, dmul((double)j, g.dz));
            tc[o] = node[k];
            ts[o] = g.sigma;
        } else {
            const uint32_t p = (uint32_t)(k - nn);
            tx[o] = x[p];
            tz[o] = z[p];
            tc[o] = circ[p];
            ts[o] = sigma[p];
        }
    }
}

__global__ void k_rm_copyback(const uint32_t* __restrict__ total, const int* __restrict__ ok,
                              const double* __restrict__ tx, const double* __restrict__ tz,
                              const double* __restrict__ tc, const double* __restrict__ ts,
                              RemeshDest d) {
    if (!ok[0]) return;
    const uint32_t t = total[0];
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < t; q += gridDim.x * blockDim.x) {
        d.x[q] = tx[q];
        d.z[q] = tz[q];
        d.circ[q] = tc[q];
        d.sigma[q] = ts[q];
        if (d.u) d.u[q] = 0.0;
        if (d.w) d.w[q] = 0.0;
        if (d.uvs) d.uvs[q] = 0.0;
        if (d.wvs) d.wvs[q] = 0.0;
        if (d.id) d.id[q] = q;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && d.n) d.n[0] = t;
}

int key_bits(uint64_t ncells) {
    int b = 1;
    while (b < 63 && (1ull << b) <= ncells) ++b;
    return b;
}

struct Layout {
    size_t keys_in, keys_out, vals_in, vals_out, gcirc, cstart, cend, node, flags, pos, tmp, tx,
        tz, tc, ts, scal, bytes, tmp_bytes;
};

Layout layout(const RemeshGrid& g, uint32_t n, uint32_t cap) {
    const uint64_t nn = (uint64_t)g.nx * g.nz, m = nn + n;
    size_t sort_b = 0, scan_b = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_b, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                    (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (int64_t)std::max<uint32_t>(n, 1), 0, key_bits(nn));
    cub::DeviceScan::ExclusiveSum(nullptr, scan_b, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                  (int64_t)m);
    Layout L{};
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += (bytes + 255) / 256 * 256;
        return o;
    };
    L.keys_in = take(8ull * n);
    L.keys_out = take(8ull * n);
    L.vals_in = take(4ull * n);
    L.vals_out = take(4ull * n);
    L.gcirc = take(8ull * n);
    L.cstart = take(4 * nn);
    L.cend = take(4 * nn);
    L.node = take(8 * nn);
    L.flags = take(4 * m);
    L.pos = take(4 * m);
    L.tmp_bytes = std::max(sort_b, scan_b) + 256;
    L.tmp = take(L.tmp_bytes);
    L.tx = take(8ull * cap);
    L.tz = take(8ull * cap);
    L.tc = take(8ull * cap);
    L.ts = take(8ull * cap);
    L.scal = take(64);
    L.bytes = off;
    return L;
}

}  // namespace

size_t remesh_scratch_bytes(const RemeshGrid& g, uint32_t n, uint32_t cap) {
    return layout(g, n, cap).bytes;
}

void remesh_run(const RemeshGrid& g, const double* x, const double* z, const double* circ,
                const double* sigma, uint32_t n, uint32_t cap, const RemeshDest& dest,
                int* status, void* scratch, int sms, cudaStream_t s) {
    const Layout L = layout(g, n, cap);
    char* b = static_cast<char*>(scratch);
    auto at = [&](size_t o) { return static_cast<void*>(b + o); };
    uint64_t* keys_in = static_cast<uint64_t*>(at(L.keys_in));
    uint64_t* keys_out = static_cast<uint64_t*>(at(L.keys_out));
    uint32_t* vals_in = static_cast<uint32_t*>(at(L.vals_in));
    uint32_t* vals_out = static_cast<uint32_t*>(at(L.vals_out));
    double* gcirc = static_cast<double*>(at(L.gcirc));
    uint32_t* cstart = static_cast<uint32_t*>(at(L.cstart));
    uint32_t* cend = static_cast<uint32_t*>(at(L.cend));
    double* node = static_cast<double*>(at(L.node));
    uint32_t* flags = static_cast<uint32_t*>(at(L.flags));
    uint32_t* pos = static_cast<uint32_t*>(at(L.pos));
    double* tx = static_cast<double*>(at(L.tx));
    double* tz = static_cast<double*>(at(L.tz));
    double* tc = static_cast<double*>(at(L.tc));
    double* ts = static_cast<double*>(at(L.ts));
    uint32_t* total = static_cast<uint32_t*>(at(L.scal));
    int* ok = reinterpret_cast<int*>(total + 4);
    const uint64_t nn = (uint64_t)g.nx * g.nz, m = nn + n;
    const int grid = sms * 8;
    if (n) {
        k_rm_classify<<<grid, 256, 0, s>>>(g, x, z, circ, n, keys_in, vals_in, gcirc, flags + nn);
        size_t tb = L.tmp_bytes;
        cub::DeviceRadixSort::SortPairs(at(L.tmp), tb, keys_in, keys_out, vals_in, vals_out,
                                        (int64_t)n, 0, key_bits(nn), s);
    }
    cudaMemsetAsync(cstart, 0, 4 * nn, s);
    cudaMemsetAsync(cend, 0, 4 * nn, s);
    if (n) k_rm_bounds<<<grid, 256, 0, s>>>(keys_out, n, nn, cstart, cend);
    k_rm_gather<<<grid, 256, 0, s>>>(g, x, z, gcirc, vals_out, cstart, cend, node, flags);
    size_t tb = L.tmp_bytes;
    cub::DeviceScan::ExclusiveSum(at(L.tmp), tb, flags, pos, (int64_t)m, s);
    k_rm_total<<<1, 1, 0, s>>>(flags, pos, m, cap, total, ok, status, dest.need);
    k_rm_scatter<<<grid, 256, 0, s>>>(g, x, z, circ, sigma, n, node, flags, pos, cap, tx, tz, tc,
                                      ts);
    k_rm_copyback<<<grid, 256, 0, s>>>(total, ok, tx, tz, tc, ts, dest);
}

}  // namespace dvmk
