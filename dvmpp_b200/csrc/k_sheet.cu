// Vortex-sheet kernels: influence matrix (src/VortexSheet.cpp:104-165), the
// least-squares panel-strength solve (src/VortexSheet.cpp:214), sheet-on-blob
// velocity fused with the convection update (src/VortexSheet.cpp:217-273,
// src/DVMBase.cpp:167-209) and the pressure loads (src/VortexSheet.cpp:487-514).
//
// FP64 instances: pair formulas keep the reference's operation order with one
// rounding per operation (dadd/dmul/...), so they round like the reference
// compiled without FP contraction.  FP32 instances evaluate the sheet-on-blob
// panel terms in single precision (accumulated in FP64); the influence matrix,
// QR, solve, refinement and loads are FP64 for both.
//
// The solve: the reference forms A^T A and A^T b and solves with LAPACK every
// call.  Here A ((np+1) x np) is factorised ONCE per body by Householder QR on
// the GPU and the pseudo-inverse P = R^-1 Q^T is kept in HBM; each step is then
// gamma = P b (a batched GEMV) plus one iterative-refinement step with the FP64
// residual r = b - A gamma (gamma += P r).  Same least-squares solution, no
// O(np^3) work per step.
#include <cfloat>

#include <cooperative_groups.h>

#include "dvm_device.cuh"
#include "dvm_internal.h"

namespace dvmk {
namespace {
namespace cg = cooperative_groups;

// ---- influence matrix -------------------------------------------------------
__global__ void k_pq(const double* __restrict__ xp, const double* __restrict__ zp,
                     const double* __restrict__ xc, const double* __restrict__ zc,
                     const double* __restrict__ ds, const double* __restrict__ theta, int np,
                     double* __restrict__ p, double* __restrict__ q) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= np) return;
    double pij, qij;
    if (i == j) {
        pij = -1.0;
        qij = 1.0;
    } else {
        const double xci = xc[i], zci = zc[i], thi = theta[i];
        const double xj = xp[j], zj = zp[j], thj = theta[j], dsj = ds[j];
        const double dx = dsub(xci, xj), dz = dsub(zci, zj);
        const double cj = cos(thj), sj = sin(thj);
        const double c1 = dsub(dmul(-dx, cj), dmul(dz, sj));
        const double c2 = dadd(dmul(dx, dx), dmul(dz, dz));
        const double c3 = sin(dsub(thi, thj));
        const double c4 = cos(dsub(thi, thj));
        const double c5 = dsub(dmul(dx, sj), dmul(dz, cj));
        const double c6 = log(dadd(1.0, dmul(dsj, ddiv(dadd(dsj, dmul(2.0, c1)), c2))));
        const double c7 = atan2(dmul(c5, dsj), dadd(c2, dmul(c1, dsj)));
        const double a2 = dsub(thi, dmul(2.0, thj));
        const double c9 = dsub(dmul(dx, cos(a2)), dmul(dz, sin(a2)));
        qij = dsub(dadd(c4, ddiv(dmul(dmul(0.5, c9), c6), dsj)),
                   ddiv(dmul(dadd(dmul(c1, c3), dmul(c4, c5)), c7), dsj));
        pij = dsub(dadd(dmul(dmul(0.5, c4), c6), dmul(c3, c7)), qij);
    }
    p[(size_t)i * np + j] = pij;
    q[(size_t)i * np + j] = qij;
}

__global__ void k_assemble_A(const double* __restrict__ p, const double* __restrict__ q,
                             const double* __restrict__ ds, int np, double* __restrict__ A) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= np) return;
    if (i == np) {
        A[(size_t)np * np + j] = ds[j];  // Kelvin row (src/VortexSheet.cpp:159-161)
        return;
    }
    const int jm = (j == 0) ? np - 1 : j - 1;
    A[(size_t)i * np + j] = dmul(-kRpi2, dadd(p[(size_t)i * np + j], q[(size_t)i * np + jm]));
}

// ---- Householder QR of A (column-major, m = np+1 rows) ------------------------
// M holds [A | Q^T]: columns 0..np-1 are A (overwritten by R on and above the
// diagonal), columns np..np+m-1 receive Q^T.  Both paths are one cooperative
// launch with one grid barrier per Householder step (a chain of np dependent
// steps; separate launches per step cost ~2.5 us each).  For m <= 1056 each
// warp keeps one column of [A | I] in registers and the identity columns turn
// into Q^T in place (k_qr_reg); above that the columns of A stay in memory,
// their reflectors' tails are kept below the diagonal, and Q^T is formed
// afterwards by applying the stored reflectors to the identity (k_qr_coop,
// k_form_qt).
__global__ void k_load_aug(const double* __restrict__ A, int np, double* __restrict__ M) {
    const int m = np + 1;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)m * np;
         t += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(t / m), r = (int)(t % m);
        M[t] = A[(size_t)r * np + c];
    }
}

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Householder reflector of column k (one warp): H = I - tau v v^T maps
// col[k..m) to (alpha, 0, ...), alpha = -sign(x0) |col[k..m)|, v = (x0 - alpha,
// col[k+1..m)).  Writes v to vout (zeros above row k), v0 and tau to v0s[k],
// taus[k], and alpha to col[k]; rows below k keep v's tail.
__device__ __forceinline__ void house_col(double* __restrict__ M, int m, int k,
                                          double* __restrict__ vout, double* __restrict__ v0s,
                                          double* __restrict__ taus, int lane) {
    double* col = M + (size_t)k * m;
    double acc = 0.0;
    for (int i = k + lane; i < m; i += 32) acc = fma(col[i], col[i], acc);
    const double nrm2 = warp_sum(acc);
    const double x0 = col[k];
    const double alpha = (x0 >= 0.0) ? -sqrt(nrm2) : sqrt(nrm2);
    const double v0 = x0 - alpha;
    const double vn2 = nrm2 - x0 * x0 + v0 * v0;
    for (int i = lane; i < m; i += 32) vout[i] = (i < k) ? 0.0 : (i == k ? v0 : col[i]);
    __syncwarp();
    if (lane == 0) {
        col[k] = alpha;
        v0s[k] = v0;
        taus[k] = (vn2 > 0.0) ? 2.0 / vn2 : 0.0;
    }
}

// Cooperative launch (all blocks resident; grid.sync is the only wait).  Step
// k: every warp applies H_k to its columns c > k; the warp holding column k+1
// then forms reflector k+1 from it (double-buffered v), so each column costs
// one grid barrier.
__global__ void __launch_bounds__(256) k_qr_coop(double* __restrict__ M, int np,
                                                 double* __restrict__ vbuf,
                                                 double* __restrict__ v0s,
                                                 double* __restrict__ taus) {
    cg::grid_group grid = cg::this_grid();
    const int m = np + 1;
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nw = (int)((gridDim.x * blockDim.x) >> 5);
    if (gw == 0) house_col(M, m, 0, vbuf, v0s, taus, lane);
    grid.sync();
    for (int k = 0; k + 1 < np; ++k) {
        const double* v = vbuf + (size_t)(k & 1) * m;
        const double tau = taus[k];
        for (int c = k + 1 + gw; c < np; c += nw) {
            double* col = M + (size_t)c * m;
            double acc = 0.0;
            for (int i = k + lane; i < m; i += 32) acc = fma(v[i], col[i], acc);
            const double f = warp_sum(acc) * tau;
            for (int i = k + lane; i < m; i += 32) col[i] = fma(-f, v[i], col[i]);
            if (c == k + 1) {
                __syncwarp();
                house_col(M, m, k + 1, vbuf + (size_t)((k + 1) & 1) * m, v0s, taus, lane);
            }
        }
        grid.sync();
    }
}

// Column c of Q^T = H_{np-1} ... H_0 e_c, one warp per column, the vector in
// registers (CH = ceil(m / 32) values per lane); written to column np + c of M.
template <int CH>
__global__ void __launch_bounds__(128) k_form_qt(double* __restrict__ M, int np,
                                                 const double* __restrict__ v0s,
                                                 const double* __restrict__ taus) {
    const int m = np + 1;
    const int lane = threadIdx.x & 31;
    const int c = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (c >= m) return;
    double x[CH];
#pragma unroll
    for (int t = 0; t < CH; ++t) x[t] = (lane + 32 * t == c) ? 1.0 : 0.0;
    for (int k = 0; k < np; ++k) {
        const double* vk = M + (size_t)k * m;  // tail below row k; v0s[k] at row k
        const double v0 = v0s[k];
        double acc = 0.0;
#pragma unroll
        for (int t = 0; t < CH; ++t) {
            const int i = lane + 32 * t;
            if (i >= k && i < m) acc = fma(i == k ? v0 : vk[i], x[t], acc);
        }
        const double f = warp_sum(acc) * taus[k];
#pragma unroll
        for (int t = 0; t < CH; ++t) {
            const int i = lane + 32 * t;
            if (i >= k && i < m) x[t] = fma(-f, i == k ? v0 : vk[i], x[t]);
        }
    }
    double* out = M + (size_t)(np + c) * m;
#pragma unroll
    for (int t = 0; t < CH; ++t) {
        const int i = lane + 32 * t;
        if (i < m) out[i] = x[t];
    }
}

// Reflector k of a column held in registers (CH values per lane, rows >= k
// used): writes v to vout, v0 and tau to v0s[k], taus[k], and alpha into the
// column.  Selects rather than branches keep x in registers.
template <int CH>
__device__ __forceinline__ void house_reg(double (&x)[CH], int m, int k,
                                          double* __restrict__ vout, double* __restrict__ v0s,
                                          double* __restrict__ taus, int lane) {
    double acc = 0.0, xk = 0.0;
    const int tk = k >> 5;
#pragma unroll
    for (int t = 0; t < CH; ++t) {
        const int i = lane + 32 * t;
        acc = (i >= k && i < m) ? fma(x[t], x[t], acc) : acc;
        xk = (t == tk) ? x[t] : xk;
    }
    const double nrm2 = warp_sum(acc);
    const double x0 = __shfl_sync(0xffffffffu, xk, k & 31);
    const double alpha = (x0 >= 0.0) ? -sqrt(nrm2) : sqrt(nrm2);
    const double v0 = x0 - alpha;
    const double vn2 = nrm2 - x0 * x0 + v0 * v0;
#pragma unroll
    for (int t = 0; t < CH; ++t) {
        const int i = lane + 32 * t;
        if (i < m) vout[i] = (i < k) ? 0.0 : (i == k ? v0 : x[t]);
        x[t] = (i == k) ? alpha : x[t];
    }
    if (lane == 0) {
        v0s[k] = v0;
        taus[k] = (vn2 > 0.0) ? 2.0 / vn2 : 0.0;
    }
}

// Register-resident variant for m <= 32 CH: one warp owns one column of the
// augmented [A | I] for the whole factorisation (CH values per lane), so a step
// reads only the reflector from memory.  Step k: every warp with a column
// c > k applies H_k; the warp owning column k+1 then forms reflector k+1 from
// its registers (double-buffered v).  The identity columns become Q^T in
// place.  At the end each warp stores its column of M.
template <int CH>
__global__ void __launch_bounds__(256, 2) k_qr_reg(double* __restrict__ M, int np,
                                                double* __restrict__ vbuf,
                                                double* __restrict__ v0s,
                                                double* __restrict__ taus) {
    cg::grid_group grid = cg::this_grid();
    const int m = np + 1, cols = np + m;
    const int lane = threadIdx.x & 31;
    const int c = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const bool own = c < cols;
    double x[CH];
#pragma unroll
    for (int t = 0; t < CH; ++t) {
        const int i = lane + 32 * t;
        const bool in = own && i < m;
        x[t] = (in && c < np) ? M[(size_t)c * m + i] : ((in && i == c - np) ? 1.0 : 0.0);
    }
    if (c == 0) house_reg<CH>(x, m, 0, vbuf, v0s, taus, lane);
    grid.sync();
    for (int k = 0; k < np; ++k) {
        if (own && c > k) {
            const double* v = vbuf + (size_t)(k & 1) * m;  // zero above row k
            double acc = 0.0;
#pragma unroll
            for (int t = 0; t < CH; ++t) {
                const int i = lane + 32 * t;
                acc = (i < m) ? fma(v[i], x[t], acc) : acc;
            }
            const double f = warp_sum(acc) * taus[k];
#pragma unroll
            for (int t = 0; t < CH; ++t) {  // second read of v hits L1
                const int i = lane + 32 * t;
                x[t] = (i < m) ? fma(-f, v[i], x[t]) : x[t];
            }
            if (c == k + 1 && k + 1 < np)
                house_reg<CH>(x, m, k + 1, vbuf + (size_t)((k + 1) & 1) * m, v0s, taus, lane);
        }
        if (k + 1 < np) grid.sync();
    }
    if (own) {
#pragma unroll
        for (int t = 0; t < CH; ++t) {
            const int i = lane + 32 * t;
            if (i < m) M[(size_t)c * m + i] = x[t];
        }
    }
}

// P[:, c] = R^-1 (Q^T)[0:np, c] with the right-hand side in registers (one warp
// per column c, CH values per lane) and R's next column prefetched while the
// current one is applied.
template <int CH>
__global__ void __launch_bounds__(256) k_backsub_reg(const double* __restrict__ M, int np,
                                                     double* __restrict__ P) {
    const int m = np + 1;
    const int lane = threadIdx.x & 31;
    const int c = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (c >= m) return;
    const double* qt = M + (size_t)(np + c) * m;
    double y[CH], rc[CH];
#pragma unroll
    for (int t = 0; t < CH; ++t) {
        const int j = lane + 32 * t;
        y[t] = j < np ? qt[j] : 0.0;
        rc[t] = j < np ? M[(size_t)(np - 1) * m + j] : 0.0;  // column np-1 of R
    }
    for (int i = np - 1; i >= 0; --i) {
        double rn[CH];
#pragma unroll
        for (int t = 0; t < CH; ++t) {  // prefetch column i-1
            const int j = lane + 32 * t;
            rn[t] = (i > 0 && j < i) ? M[(size_t)(i - 1) * m + j] : 0.0;
        }
        // (selects rather than branches keep the arrays in registers)
        double yi = 0.0, rii = 0.0;
        const int ti = i >> 5;
#pragma unroll
        for (int t = 0; t < CH; ++t) {
            yi = (t == ti) ? y[t] : yi;
            rii = (t == ti) ? rc[t] : rii;
        }
        yi = __shfl_sync(0xffffffffu, yi, i & 31);
        rii = __shfl_sync(0xffffffffu, rii, i & 31);
        const double xi = yi / rii;
#pragma unroll
        for (int t = 0; t < CH; ++t) {
            const int j = lane + 32 * t;
            y[t] = (j < i) ? fma(-rc[t], xi, y[t]) : (j == i ? xi : y[t]);
            rc[t] = rn[t];
        }
    }
#pragma unroll
    for (int t = 0; t < CH; ++t) {
        const int j = lane + 32 * t;
        if (j < np) P[(size_t)j * m + c] = y[t];
    }
}

// P[:, c] = R^-1 (Q^T)[0:np, c] for every column c of Q^T; one warp per column,
// column-oriented back substitution (coalesced reads of R's columns).
__global__ void k_backsub(const double* __restrict__ M, int np, double* __restrict__ P) {
    extern __shared__ double s_y[];
    const int m = np + 1;
    const int wl = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + wl;
    if (c >= m) return;
    double* y = s_y + (size_t)wl * np;
    const double* qt = M + (size_t)(np + c) * m;
    for (int i = lane; i < np; i += 32) y[i] = qt[i];
    __syncwarp();
    for (int i = np - 1; i >= 0; --i) {
        const double* Rcol = M + (size_t)i * m;  // column i of R
        const double xi = y[i] / Rcol[i];
        __syncwarp();
        for (int j = lane; j < i; j += 32) y[j] = fma(-Rcol[j], xi, y[j]);
        if (lane == 0) y[i] = xi;
        __syncwarp();
    }
    for (int i = lane; i < np; i += 32) P[(size_t)i * m + c] = y[i];
}

// ---- per-step solve -------------------------------------------------------------
// mode 0: gamma = P b; mode 1: gamma += P res
__global__ void k_gemv_P(const InstDesc* __restrict__ table, const ListEntry* __restrict__ list,
                         int mode) {
    const ListEntry e = list[blockIdx.y];
    const InstDesc& d = table[e.inst];
    const int m = d.np + 1;
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (row >= d.np) return;
    const double* pr = d.P + (size_t)row * m;
    const double* rhs = mode == 0 ? d.b : d.res;
    double acc = 0.0;
    for (int c = lane; c < m; c += 32) acc = fma(pr[c], rhs[c], acc);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) d.gamma[row] = (mode == 0) ? acc : d.gamma[row] + acc;
}

__global__ void k_residual(const InstDesc* __restrict__ table, const ListEntry* __restrict__ list) {
    const ListEntry e = list[blockIdx.y];
    const InstDesc& d = table[e.inst];
    const int np = d.np;
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (row > np) return;
    const double* ar = d.A + (size_t)row * np;
    double acc = 0.0;
    for (int c = lane; c < np; c += 32) acc = fma(ar[c], d.gamma[c], acc);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) d.res[row] = d.b[row] - acc;
}

// ---- sheet-on-blob velocity (+ convection) -------------------------------------
// One panel term of src/VortexSheet.cpp:235-249 in FP32 for the FP32-precision
// instances.  The blob's offsets from the panel's start (the collocation
// point) and end are formed in FP64 and rounded once.  c6 = log(|p-e|^2 /
// |p-s|^2) is taken as log1p(x), x = ds (ds + 2 c1) / c2, while |x| < 1/2,
// and as the log of the two squared distances' ratio otherwise, so a blob
// next to the panel's end (nascent blobs sit there) keeps full relative
// accuracy.  The contribution px g0 + qx g1 is evaluated as
// (px + qx) g0 + qx (g1 - g0): px + qx = -c6/2 sin - c7 cos has no
// cancellation, whereas px and qx separately are O(1) terms that cancel to
// O(ds / r) for distant blobs, so this grouping keeps FP32 rounding relative
// to the result (the FP64 instances keep the reference's grouping).
struct PanelF32 {
    float ct, st, ds, ids, c2, s2;
};

__device__ __forceinline__ void sheet_pair_f32(float dx, float dz, float dxe, float dze,
                                               const PanelF32& P, float g0, float dg, double& us,
                                               double& ws) {
    const float c1 = -dx * P.ct - dz * P.st;
    const float c2 = fmaf(dx, dx, dz * dz);
    const float c5 = dx * P.st - dz * P.ct;
    const float x = __fdividef(P.ds * fmaf(2.0f, c1, P.ds), c2);
    const float c6 = fabsf(x) < 0.5f ? log1pf(x)
                                     : logf(__fdividef(fmaf(dxe, dxe, dze * dze), c2));
    const float c7 = atan2f(c5 * P.ds, fmaf(c1, P.ds, c2));
    const float c8 = dx * P.s2 + dz * P.c2;
    const float c9 = dx * P.c2 - dz * P.s2;
    const float h6 = 0.5f * c6 * P.ids, c7i = c7 * P.ids;
    const float qx = -P.st + c8 * h6 + (c1 * P.ct + c5 * P.st) * c7i;
    const float qy = P.ct + c9 * h6 + (c1 * P.st - c5 * P.ct) * c7i;
    const float ax = -0.5f * c6 * P.st - c7 * P.ct;  // px + qx
    const float ay = 0.5f * c6 * P.ct - c7 * P.st;   // py + qy
    us += (double)fmaf(ax, g0, qx * dg);
    ws += (double)fmaf(ay, g0, qy * dg);
}

// One panel term of src/VortexSheet.cpp:235-249, 261-268 in FP64 with the
// reference's operation order (one rounding per operation); dx, dz are the
// point's offsets from the panel's collocation point.
__device__ __forceinline__ void sheet_pair_f64(double dx, double dz, double dsj, double ct,
                                               double stt, double c2t, double s2t, double g0,
                                               double g1, double& us, double& ws) {
    const double c1 = dsub(dmul(-dx, ct), dmul(dz, stt));
    const double c2 = dadd(dmul(dx, dx), dmul(dz, dz));
    const double c5 = dsub(dmul(dx, stt), dmul(dz, ct));
    const double c6 = log(dadd(1.0, dmul(dsj, ddiv(dadd(dsj, dmul(2.0, c1)), c2))));
    const double c7 = atan2(dmul(c5, dsj), dadd(c2, dmul(c1, dsj)));
    const double c8 = dadd(dmul(dx, s2t), dmul(dz, c2t));
    const double c9 = dsub(dmul(dx, c2t), dmul(dz, s2t));
    const double qx = dadd(dadd(-stt, ddiv(dmul(dmul(0.5, c8), c6), dsj)),
                           ddiv(dmul(dadd(dmul(c1, ct), dmul(c5, stt)), c7), dsj));
    const double px = dsub(dsub(dmul(dmul(-0.5, c6), stt), dmul(c7, ct)), qx);
    const double qy = dadd(dadd(ct, ddiv(dmul(dmul(0.5, c9), c6), dsj)),
                           ddiv(dmul(dsub(dmul(c1, stt), dmul(c5, ct)), c7), dsj));
    const double py = dsub(dsub(dmul(dmul(0.5, c6), ct), dmul(c7, stt)), qy);
    us = dadd(us, dadd(dmul(px, g0), dmul(qx, g1)));
    ws = dadd(ws, dadd(dmul(py, g0), dmul(qy, g1)));
}

// Sheet velocity at arbitrary points (probes): the same panel sum as the
// sheet-on-blob velocity, over every panel, in FP64; one thread per point.
__global__ void __launch_bounds__(128) k_sheet_at(const double* __restrict__ xc,
                                                  const double* __restrict__ zc,
                                                  const double* __restrict__ ds,
                                                  const double* __restrict__ cth,
                                                  const double* __restrict__ sth,
                                                  const double* __restrict__ c2th,
                                                  const double* __restrict__ s2th,
                                                  const double* __restrict__ gamma, int np,
                                                  const double* __restrict__ px,
                                                  const double* __restrict__ pz, uint32_t n,
                                                  double* __restrict__ uvs,
                                                  double* __restrict__ wvs) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double xi = px[i], zi = pz[i];
    double us = 0.0, ws = 0.0;
    for (int j = 0; j < np; ++j)
        sheet_pair_f64(dsub(xi, xc[j]), dsub(zi, zc[j]), ds[j], cth[j], sth[j], c2th[j], s2th[j],
                       gamma[j], gamma[j == np - 1 ? 0 : j + 1], us, ws);
    uvs[i] = dmul(us, kRpi2);
    wvs[i] = dmul(ws, kRpi2);
}

__global__ void __launch_bounds__(256) k_sheet_velocity(const InstDesc* __restrict__ table,
                                                        const InstState* __restrict__ st,
                                                        const ListEntry* __restrict__ list,
                                                        int nlist, int mode,
                                                        unsigned* __restrict__ work) {
    extern __shared__ double s_pan[];  // FP64: 8 arrays of max_np; FP32: see below
    __shared__ unsigned s_pre[1025];
    __shared__ unsigned s_item;
    __shared__ int s_loaded;
    if (threadIdx.x == 0) {
        unsigned acc = 0;
        for (int k = 0; k < nlist; ++k) {
            s_pre[k] = acc;
            acc += (st[list[k].inst].n + 255) / 256;
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
        const bool f32 = d.precision == kF32;
        double* sxc = s_pan;
        double* szc = sxc + np;
        double* sds = szc + np;
        double* sct = sds + np;
        double* sst = sct + np;
        double* sc2 = sst + np;
        double* ss2 = sc2 + np;
        double* sg = ss2 + np;
        // FP32 layout after xc, zc: the panel ends (FP64), np PanelF32
        // records, then np gamma_j and np (gamma_{j+1} - gamma_j) (wrapping at
        // the last panel)
        double* sex = szc + np;
        double* sez = sex + np;
        PanelF32* fpan = reinterpret_cast<PanelF32*>(sez + np);
        float* fg = reinterpret_cast<float*>(fpan + np);
        float* fdg = fg + np;
        if (s_loaded != k) {
            for (int j = threadIdx.x; j < np; j += blockDim.x) {
                sxc[j] = d.xc[j];
                szc[j] = d.zc[j];
                if (f32) {
                    const double dsj = d.ds[j];
                    sex[j] = d.xc[j] + dsj * d.cth[j];
                    sez[j] = d.zc[j] + dsj * d.sth[j];
                    fpan[j] = PanelF32{(float)d.cth[j], (float)d.sth[j], (float)dsj,
                                       (float)(1.0 / dsj), (float)d.c2th[j], (float)d.s2th[j]};
                    const double g0 = d.gamma[j], g1 = d.gamma[j == np - 1 ? 0 : j + 1];
                    fg[j] = (float)g0;
                    fdg[j] = (float)(g1 - g0);
                } else {
                    sds[j] = d.ds[j];
                    sct[j] = d.cth[j];
                    sst[j] = d.sth[j];
                    sc2[j] = d.c2th[j];
                    ss2[j] = d.s2th[j];
                    sg[j] = d.gamma[j];
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) s_loaded = k;
        const uint32_t n = st[e.inst].n;
        const uint32_t i = (item - s_pre[k]) * 256 + threadIdx.x;
        if (i < n) {
            const double xi = d.x[i], zi = d.z[i];
            double us = 0.0, ws = 0.0;
            if (f32) {
#pragma unroll 2
                for (int j = 0; j < np; ++j)
                    sheet_pair_f32((float)(xi - sxc[j]), (float)(zi - szc[j]),
                                   (float)(xi - sex[j]), (float)(zi - sez[j]), fpan[j], fg[j],
                                   fdg[j], us, ws);
            } else {
                for (int j = 0; j < np; ++j)
                    sheet_pair_f64(dsub(xi, sxc[j]), dsub(zi, szc[j]), sds[j], sct[j], sst[j],
                                   sc2[j], ss2[j], sg[j], (j == np - 1) ? sg[0] : sg[j + 1], us,
                                   ws);
            }
            const double uvs = dmul(us, kRpi2), wvs = dmul(ws, kRpi2);
            d.uvs[i] = uvs;
            d.wvs[i] = wvs;
            if (mode >= 1) {
                const double vx = dmul(dadd(dadd(d.u[i], uvs), d.ux), d.dt);
                const double vz = dmul(dadd(dadd(d.w[i], wvs), d.uz), d.dt);
                if (mode == 1) {
                    d.x[i] = dadd(xi, vx);
                    d.z[i] = dadd(zi, vz);
                } else {
                    const int s = mode - 2;
                    const double a = s == 0 ? 0.0 : (s == 1 ? -17. / 32 : -32. / 27);
                    const double bb = s == 0 ? 1. / 4 : (s == 1 ? 8. / 9 : 3. / 4);
                    const double q1o = s == 0 ? 0.0 : d.q1[i];
                    const double q2o = s == 0 ? 0.0 : d.q2[i];
                    const double q1 = dadd(dmul(a, q1o), vx);
                    const double q2 = dadd(dmul(a, q2o), vz);
                    d.q1[i] = q1;
                    d.q2[i] = q2;
                    d.x[i] = dadd(xi, dmul(bb, q1));
                    d.z[i] = dadd(zi, dmul(bb, q2));
                }
            }
        }
        __syncthreads();
    }
}

__global__ void k_convect_update(const InstDesc* __restrict__ table,
                                 const InstState* __restrict__ st,
                                 const ListEntry* __restrict__ list, int nlist, int mode) {
    const ListEntry e = list[blockIdx.y];
    const InstDesc& d = table[e.inst];
    const uint32_t n = st[e.inst].n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double vx = dmul(dadd(dadd(d.u[i], d.uvs[i]), d.ux), d.dt);
        const double vz = dmul(dadd(dadd(d.w[i], d.wvs[i]), d.uz), d.dt);
        if (mode == 1) {
            d.x[i] = dadd(d.x[i], vx);
            d.z[i] = dadd(d.z[i], vz);
        } else {
            const int s = mode - 2;
            const double a = s == 0 ? 0.0 : (s == 1 ? -17. / 32 : -32. / 27);
            const double bb = s == 0 ? 1. / 4 : (s == 1 ? 8. / 9 : 3. / 4);
            const double q1 = dadd(dmul(a, s == 0 ? 0.0 : d.q1[i]), vx);
            const double q2 = dadd(dmul(a, s == 0 ? 0.0 : d.q2[i]), vz);
            d.q1[i] = q1;
            d.q2[i] = q2;
            d.x[i] = dadd(d.x[i], dmul(bb, q1));
            d.z[i] = dadd(d.z[i], dmul(bb, q2));
        }
    }
}

// ---- loads (src/VortexSheet.cpp:489-513), one block per simulation ---------------
__global__ void k_loads(const InstDesc* __restrict__ table, InstState* __restrict__ st,
                        const ListEntry* __restrict__ list) {
    extern __shared__ double s_P[];
    const ListEntry e = list[blockIdx.x];
    const InstDesc& d = table[e.inst];
    const int np = d.np;
    if (threadIdx.x != 0) return;
    const double c = ddiv(-d.rho, d.dt);
    s_P[0] = 0.0;
    for (int i = 0; i < np - 1; ++i) s_P[i + 1] = dadd(s_P[i], dmul(c, dmul(d.gamma[i], d.ds[i])));
    for (int i = 0; i < np - 1; ++i) s_P[i] = dmul(0.5, dadd(s_P[i], s_P[i + 1]));
    s_P[np - 1] = dmul(0.5, dadd(s_P[np - 1], s_P[0]));
    double pmax = s_P[0];
    for (int i = 1; i < np; ++i)
        if (s_P[i] > pmax) pmax = s_P[i];
    const double pref = dmul(dmul(dmul(0.5, d.rho), d.Ur), d.Ur);
    const double shift = dmul(dsub(pref, pmax), 1.0);
    double sx = 0.0, sz = 0.0;
    for (int i = 0; i < np; ++i) {
        const double Pi = dadd(s_P[i], shift);
        sx = dadd(sx, dmul(dmul(Pi, d.enx[i]), d.ds[i]));
        sz = dadd(sz, dmul(dmul(Pi, d.enz[i]), d.ds[i]));
    }
    const double fx = -sx, fz = -sz;
    const double den = dmul(dmul(dmul(dmul(0.5, d.rho), d.area), d.Ur), d.Ur);
    InstState& s = st[e.inst];
    s.fx = fx;
    s.fz = fz;
    s.cd = ddiv(fx, den);
    s.cl = ddiv(fz, den);
}

__global__ void k_step_counter(InstState* __restrict__ st, const ListEntry* __restrict__ list,
                               int nlist) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nlist) st[list[k].inst].step += 1;
}

}  // namespace

void influence_matrix(const double* xp, const double* zp, const double* xc, const double* zc,
                      const double* ds, const double* theta, int np, double* pq_scratch,
                      double* A, cudaStream_t s) {
    double* p = pq_scratch;
    double* q = pq_scratch + (size_t)np * np;
    dim3 g((np + 127) / 128, np);
    k_pq<<<g, 128, 0, s>>>(xp, zp, xc, zc, ds, theta, np, p, q);
    dim3 g2((np + 127) / 128, np + 1);
    k_assemble_A<<<g2, 128, 0, s>>>(p, q, ds, np, A);
}

size_t pseudo_inverse_work_doubles(int np) {
    const size_t m = (size_t)np + 1;
    return m * (np + m) + 2 * m + 2 * (size_t)np + 8;
}

cudaError_t pseudo_inverse(const double* A, int np, double* P, double* work, cudaStream_t s) {
    const int m = np + 1, cols = np + m;
    double* M = work;
    double* vbuf = M + (size_t)m * cols;
    double* v0s = vbuf + 2 * (size_t)m;
    double* taus = v0s + np;
    k_load_aug<<<256, 256, 0, s>>>(A, np, M);
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // Register-resident path: one warp per column of [A | I], all resident.
    auto reg_path = [&](auto kqr, auto kbs) -> int {
        int per = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kqr, 256, 0);
        const int blocks = (cols + 7) / 8;
        if (blocks > per * sms) return 0;  // not co-resident: use the general path
        void* args[] = {&M, &np, &vbuf, &v0s, &taus};
        cudaError_t e = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kqr),
                                                    dim3(blocks), dim3(256), args, 0, s);
        if (e != cudaSuccess) return -1;
        kbs<<<(m + 7) / 8, 256, 0, s>>>(M, np, P);
        return 1;
    };
    int done = 0;
    if (m <= 32 * 9) done = reg_path(k_qr_reg<9>, k_backsub_reg<9>);
    else if (m <= 32 * 17) done = reg_path(k_qr_reg<17>, k_backsub_reg<17>);
    else if (m <= 32 * 33) done = reg_path(k_qr_reg<33>, k_backsub_reg<33>);
    if (done < 0) return cudaGetLastError();
    if (done > 0) return cudaGetLastError();
    // General path: one warp per column of A (columns in memory), then Q^T
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_qr_coop, 256, 0);
    const int blocks = std::max(1, std::min((np + 7) / 8, std::max(1, per_sm) * sms));
    void* args[] = {&M, &np, &vbuf, &v0s, &taus};
    cudaError_t e = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_qr_coop),
                                                dim3(blocks), dim3(256), args, 0, s);
    if (e != cudaSuccess) return e;
    const int g = (m + 3) / 4;  // 4 warps (columns) per block
    if (m <= 32 * 9) k_form_qt<9><<<g, 128, 0, s>>>(M, np, v0s, taus);
    else if (m <= 32 * 17) k_form_qt<17><<<g, 128, 0, s>>>(M, np, v0s, taus);
    else if (m <= 32 * 33) k_form_qt<33><<<g, 128, 0, s>>>(M, np, v0s, taus);
    else k_form_qt<65><<<g, 128, 0, s>>>(M, np, v0s, taus);  // np <= 2048
    // warps per block such that the per-warp right-hand sides fit 48 KB of shared memory
    const int wpb = std::max(1, std::min(4, (int)(48 * 1024 / (sizeof(double) * np))));
    k_backsub<<<(m + wpb - 1) / wpb, wpb * 32, sizeof(double) * np * wpb, s>>>(M, np, P);
    return cudaGetLastError();
}

void sheet_solve(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
                 int max_np, cudaStream_t s) {
    (void)st;
    const int rows_per_block = 8;
    dim3 g((max_np + 1 + rows_per_block - 1) / rows_per_block, nlist);
    k_gemv_P<<<g, rows_per_block * 32, 0, s>>>(table, list, 0);
    // One refinement step with the FP64 residual of the full (np+1)-row system.
    k_residual<<<g, rows_per_block * 32, 0, s>>>(table, list);
    k_gemv_P<<<g, rows_per_block * 32, 0, s>>>(table, list, 1);
}

void sheet_velocity(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
                    int mode, int max_np, const Workspace& ws, int sms, cudaStream_t s) {
    const size_t smem = sizeof(double) * 8 * (size_t)max_np;
    static bool attr = false;  // set once, before any graph capture (first call is eager)
    if (!attr) {
        cudaFuncSetAttribute(k_sheet_velocity, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             200 * 1024);
        attr = true;
    }
    cudaMemsetAsync(ws.work + 1, 0, sizeof(unsigned), s);
    k_sheet_velocity<<<sms * 4, 256, smem, s>>>(table, st, list, nlist, mode, ws.work + 1);
}

void sheet_at(const InstDesc& d, const double* px, const double* pz, uint32_t n, double* uvs,
              double* wvs, cudaStream_t s) {
    if (n == 0) return;
    k_sheet_at<<<(n + 127) / 128, 128, 0, s>>>(d.xc, d.zc, d.ds, d.cth, d.sth, d.c2th, d.s2th,
                                               d.gamma, d.np, px, pz, n, uvs, wvs);
}

void convect_update(const InstDesc* table, InstState* st, const ListEntry* list, int nlist,
                    int mode, const Workspace& ws, int sms, cudaStream_t s) {
    (void)ws;
    dim3 g(std::max(1, sms * 4 / std::max(1, nlist)), nlist);
    k_convect_update<<<g, 256, 0, s>>>(table, st, list, nlist, mode);
}

void loads(const InstDesc* table, InstState* st, const ListEntry* list, int nlist, int max_np,
           cudaStream_t s) {
    k_loads<<<nlist, 32, sizeof(double) * max_np, s>>>(table, st, list);
}

void step_counter(InstState* st, const ListEntry* list, int nlist, cudaStream_t s) {
    k_step_counter<<<(nlist + 127) / 128, 128, 0, s>>>(st, list, nlist);
}

}  // namespace dvmk
