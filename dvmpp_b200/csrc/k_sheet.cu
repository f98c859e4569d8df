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
#include <algorithm>
#include <cfloat>

#include <cooperative_groups.h>
#include <vector>

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

// Bodies factorised together in one register-resident launch: bodies of one
// register class share its grid barriers, so k bodies cost about as much as one
// (a step is barrier-bound: ~1.2 us of a ~2 us step at np = 512).  Block b
// belongs to the last body whose qr_block0 (k_qr_reg) or bs_block0
// (k_backsub_reg) is <= b; a body's arithmetic does not depend on the others.
constexpr int kQrMaxBodies = 8;
struct QrBody {
    double* M;
    double* vbuf;
    double* v0s;
    double* taus;
    double* P;
    int np;
    int qr_block0;
    int bs_block0;
};
struct QrGroup {
    QrBody b[kQrMaxBodies];
    int nb;
    int maxnp;
};

__device__ __forceinline__ int qr_body_of(const QrGroup& G, bool backsub) {
    int k = 0;
    while (k + 1 < G.nb &&
           (int)blockIdx.x >= (backsub ? G.b[k + 1].bs_block0 : G.b[k + 1].qr_block0))
        ++k;
    return k;
}

// Register-resident variant for m <= 32 CH: one warp owns one column of the
// augmented [A | I] for the whole factorisation (CH values per lane), so a step
// reads only the reflector from memory.  Step k: every warp with a column
// c > k applies H_k; the warp owning column k+1 then forms reflector k+1 from
// its registers (double-buffered v).  The identity columns become Q^T in
// place.  At the end each warp stores its column of M.  Every block takes the
// group's maxnp - 1 grid barriers; a body's steps end at its own np.
template <int CH>
__global__ void __launch_bounds__(256, 2) k_qr_reg(const __grid_constant__ QrGroup G) {
    cg::grid_group grid = cg::this_grid();
    const QrBody& B = G.b[qr_body_of(G, false)];
    double* __restrict__ M = B.M;
    double* __restrict__ vbuf = B.vbuf;
    double* __restrict__ v0s = B.v0s;
    double* __restrict__ taus = B.taus;
    const int np = B.np;
    const int m = np + 1, cols = np + m;
    const int lane = threadIdx.x & 31;
    const int c = (int)(((blockIdx.x - B.qr_block0) * blockDim.x + threadIdx.x) >> 5);
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
    for (int k = 0; k < G.maxnp; ++k) {
        if (k < np && own && c > k) {
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
        if (k + 1 < G.maxnp) grid.sync();
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
__global__ void __launch_bounds__(256) k_backsub_reg(const __grid_constant__ QrGroup G) {
    const QrBody& B = G.b[qr_body_of(G, true)];
    const double* __restrict__ M = B.M;
    double* __restrict__ P = B.P;
    const int np = B.np;
    const int m = np + 1;
    const int lane = threadIdx.x & 31;
    const int c = (int)(((blockIdx.x - B.bs_block0) * blockDim.x + threadIdx.x) >> 5);
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
// The panel terms of src/VortexSheet.cpp:235-249 in FP32 for the FP32-precision
// instances, two blobs per thread in packed FP32x2 arithmetic, with the log
// and the angle evaluated by this file's own polynomials (no library
// log1pf / logf / atan2f: those sequences made the term issue-bound at ~150
// instructions).  The blobs' offsets from the panel's origin (its
// collocation point) are formed in FP64 and rounded once.
//
// Far regime -- |x| <= 1/4 with x = ds (ds + 2 c1) / c2, and an angle
// |c7| <= atan(1/4) with the blob in front of both panel ends (X > 0) --
// c6 = log1p(x) by L(x) and c7 = atan(Y / X) by T(s), packed.  A warp whose
// blobs are all far from the panel (a vote), which is nearly every (warp,
// panel) pair, stops there; otherwise each lane replaces its near values:
// c6 = log(|p-e|^2 / |p-s|^2) by log_pos when |x| > 1/4 (a blob next to the
// panel's end, where 1 + x cancels; the end offsets are formed in FP64 too),
// and c7 by the any-angle atan2_any.  A far value gets the same bits on
// either path, so a blob's result never depends on its warp-mates.
//
// The contribution px g0 + qx g1 is evaluated as (px + qx) g0 + qx (g1 - g0):
// px + qx = -c6/2 sin - c7 cos has no cancellation, whereas px and qx
// separately are O(1) terms that cancel to O(ds / r) for distant blobs, so
// this grouping keeps FP32 rounding relative to the result (the FP64
// instances keep the reference's grouping).

// Coefficients from dvmpp_b200/csrc/fit_polys.py (Lawson's algorithm,
// minimax relative error; each FP32 Horner evaluation is within 1.8e-7 of the
// function, relative).
// atan2(y, x) for any quadrant: q = min(|x|, |y|) / max(|x|, |y|) in [0, 1],
// atan(q) = q G(q^2) (degree 9 in q^2), then the octant: pi/2 - a when
// |y| > |x|, pi - a when x < 0, and the sign of y (so atan2(+-0, x < 0) is
// +-pi, as the C library's).
__device__ __forceinline__ float atan2_any(float y, float x) {
    const float ax = fabsf(x), ay = fabsf(y);
    const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
    const float q = mx > 0.0f ? mn * rcp_approx(mx) : 0.0f;
    const float s = q * q;
    float p = -1.753928023e-03f;
    p = fmaf(p, s, 1.072693430e-02f);
    p = fmaf(p, s, -3.080458008e-02f);
    p = fmaf(p, s, 5.755208433e-02f);
    p = fmaf(p, s, -8.377314359e-02f);
    p = fmaf(p, s, 1.094202995e-01f);
    p = fmaf(p, s, -1.426193267e-01f);
    p = fmaf(p, s, 1.999826580e-01f);
    p = fmaf(p, s, -3.333328366e-01f);
    p = fmaf(p, s, 1.0f);
    float a = q * p;
    if (ay > ax) a = 1.57079637f - a;
    if (x < 0.0f) a = 3.14159274f - a;
    return copysignf(a, y);
}
// Natural log of y > 0: y = 2^e m with m in [sqrt(1/2), sqrt(2)) (exponent
// and mantissa from the bits), log(y) = e ln 2 + log1p(m - 1) and
// log1p(f) = 2 atanh(u), u = f / (2 + f) in [-0.172, 0.172], summed by its
// Taylor series 2 u (1 + u^2/3 + ... + u^10/11) (truncation below 1e-10,
// relative).  y = 0 gives -inf and anything not positive NaN, as log does.
__device__ __forceinline__ float log_pos(float y) {
    const int b = __float_as_int(y);
    const int e = (b - 0x3f3504f3) >> 23;
    const float m = __int_as_float(b - (e << 23));
    const float u = (m - 1.0f) * rcp_approx(m + 1.0f);
    const float s = u * u;
    float p = 1.0f / 11.0f;
    p = fmaf(p, s, 1.0f / 9.0f);
    p = fmaf(p, s, 1.0f / 7.0f);
    p = fmaf(p, s, 1.0f / 5.0f);
    p = fmaf(p, s, 1.0f / 3.0f);
    p = fmaf(p, s, 1.0f);
    const float r = fmaf((float)e, 0.693147182f, 2.0f * u * p);
    return y > 0.0f ? (y < INFINITY ? r : y) : (y == 0.0f ? -INFINITY : __int_as_float(0x7fc00000));
}

// log1p(x) = x L(x) for |x| <= 1/4 (degree 7), both halves of a packed pair.
__device__ __forceinline__ uint64_t f2log1p_quarter(uint64_t x) {
    uint64_t p = f2pack(-1.400713623e-01f, -1.400713623e-01f);
    p = f2fma(p, x, f2pack(1.578133851e-01f, 1.578133851e-01f));
    p = f2fma(p, x, f2pack(-1.659528315e-01f, -1.659528315e-01f));
    p = f2fma(p, x, f2pack(1.994014233e-01f, 1.994014233e-01f));
    p = f2fma(p, x, f2pack(-2.500122786e-01f, -2.500122786e-01f));
    p = f2fma(p, x, f2pack(3.333409131e-01f, 3.333409131e-01f));
    p = f2fma(p, x, f2pack(-4.999999404e-01f, -4.999999404e-01f));
    p = f2fma(p, x, f2pack(1.0f, 1.0f));
    return f2mul(x, p);
}
// atan(t) = t T(t^2) for |t| <= 1/4 (degree 3 in t^2), both halves.
__device__ __forceinline__ uint64_t f2atan_quarter(uint64_t t) {
    const uint64_t s = f2mul(t, t);
    uint64_t p = f2pack(-1.299096644e-01f, -1.299096644e-01f);
    p = f2fma(p, s, f2pack(1.995062530e-01f, 1.995062530e-01f));
    p = f2fma(p, s, f2pack(-3.333272338e-01f, -3.333272338e-01f));
    p = f2fma(p, s, f2pack(1.0f, 1.0f));
    return f2mul(t, p);
}

// FP32 panel constants, each duplicated into both halves of a packed pair so
// that one 16-byte shared load brings two of them for both blobs of a thread:
// .x and .y of each field are (v, v) pairs.
struct PanelX2 {
    ulonglong2 cs;  // (cos th, cos th), (sin th, sin th)
    ulonglong2 dd;  // (ds, ds), (1/ds, 1/ds)
    ulonglong2 cc;  // (cos -2th, ...), (sin -2th, ...)
    ulonglong2 gd;  // (gamma_j, ...), (gamma_{j+1} - gamma_j, ...)
};

// The near-regime values of one blob (see above): c6 by log_pos from the
// FP64-formed end offsets when |x| > 1/4, c7 by atan2_any when the angle is
// wide; other values are left as the far evaluations gave them.
__device__ __forceinline__ void near_values(double xi, double zi, double ex, double ez, float x,
                                            float c2, float Y, float X, bool near_log, bool wide,
                                            float& c6, float& c7) {
    if (near_log) {
        const float dxe = (float)(xi - ex), dze = (float)(zi - ez);
        c6 = log_pos(fmaf(dxe, dxe, dze * dze) / c2);
    }
    if (wide) c7 = atan2_any(Y, X);
    (void)x;
}

// Sum of the panel terms at two points (blob a in the low half, blob b in the
// high half of every packed value) over the np panels staged in shared
// memory.  Every lane of the warp must call it: the regime is voted.
__device__ __forceinline__ void sheet_sum_f32x2(double xa, double za, double xb, double zb,
                                                int np, const double* __restrict__ sxc,
                                                const double* __restrict__ szc,
                                                const double* __restrict__ sex,
                                                const double* __restrict__ sez,
                                                const PanelX2* __restrict__ pan, double& ua,
                                                double& wa, double& ub, double& wb) {
    const uint64_t two = f2pack(2.0f, 2.0f), half = f2pack(0.5f, 0.5f);
    // Panel terms are summed in FP32 over blocks of eight panels, each block
    // then added in FP64 (a quarter of the conversions and FP64 adds; the
    // bench's FP32-vs-FP64 check gave the same worst-case error as per-term FP64
    // adds).
    for (int j0 = 0; j0 < np; j0 += 8) {
        uint64_t ACU = f2pack(0.0f, 0.0f), ACW = f2pack(0.0f, 0.0f);
        const int jn = min(np, j0 + 8);
#pragma unroll 2
        for (int j = j0; j < jn; ++j) {
            const PanelX2 P = pan[j];
            const uint64_t CT = P.cs.x, ST = P.cs.y, DS = P.dd.x, IDS = P.dd.y;
            const uint64_t C2T = P.cc.x, S2T = P.cc.y, G0 = P.gd.x, DG = P.gd.y;
            const double xc = sxc[j], zc = szc[j];
            const uint64_t DX = f2pack((float)(xa - xc), (float)(xb - xc));
            const uint64_t DZ = f2pack((float)(za - zc), (float)(zb - zc));
            const uint64_t C1 = f2sub(f2pack(0.0f, 0.0f), f2fma(DX, CT, f2mul(DZ, ST)));
            const uint64_t R2 = f2fma(DX, DX, f2mul(DZ, DZ));
            const uint64_t C5 = f2sub(f2mul(DX, ST), f2mul(DZ, CT));
            const float r2a = f2lo(R2), r2b = f2hi(R2);
            const uint64_t XX =
                f2mul(f2mul(DS, f2fma(two, C1, DS)), f2pack(rcp_approx(r2a), rcp_approx(r2b)));
            const uint64_t Y = f2mul(C5, DS);
            const uint64_t X = f2fma(C1, DS, R2);
            const float Xa = f2lo(X), Xb = f2hi(X);
            const uint64_t T = f2mul(Y, f2pack(rcp_approx(Xa), rcp_approx(Xb)));
            const float xxa = f2lo(XX), xxb = f2hi(XX), ta = f2lo(T), tb = f2hi(T);
            const bool nla = !(fabsf(xxa) <= 0.25f), nlb = !(fabsf(xxb) <= 0.25f);
            const bool wa_ = !(Xa > 0.0f && fabsf(ta) <= 0.25f), wb_ = !(Xb > 0.0f && fabsf(tb) <= 0.25f);
            uint64_t C6 = f2log1p_quarter(XX);
            uint64_t C7 = f2atan_quarter(T);
            if (__any_sync(0xffffffffu, nla || nlb || wa_ || wb_)) {
                float c6a = f2lo(C6), c6b = f2hi(C6), c7a = f2lo(C7), c7b = f2hi(C7);
                const double ex = sex[j], ez = sez[j];
                near_values(xa, za, ex, ez, xxa, r2a, f2lo(Y), Xa, nla, wa_, c6a, c7a);
                near_values(xb, zb, ex, ez, xxb, r2b, f2hi(Y), Xb, nlb, wb_, c6b, c7b);
                C6 = f2pack(c6a, c6b);
                C7 = f2pack(c7a, c7b);
            }
            const uint64_t C8 = f2fma(DX, S2T, f2mul(DZ, C2T));
            const uint64_t C9 = f2sub(f2mul(DX, C2T), f2mul(DZ, S2T));
            const uint64_t HC6 = f2mul(half, C6);
            const uint64_t H6 = f2mul(HC6, IDS), C7I = f2mul(C7, IDS);
            // qx = -st + c8 h6 + (c1 ct + c5 st) c7i;  qy = ct + c9 h6 + (c1 st - c5 ct) c7i
            const uint64_t QX = f2fma(f2fma(C1, CT, f2mul(C5, ST)), C7I, f2fma(C8, H6, f2sub(f2pack(0.0f, 0.0f), ST)));
            const uint64_t QY = f2fma(f2sub(f2mul(C1, ST), f2mul(C5, CT)), C7I, f2fma(C9, H6, CT));
            // px + qx = -c6/2 sin - c7 cos;  py + qy = c6/2 cos - c7 sin
            const uint64_t AX = f2sub(f2pack(0.0f, 0.0f), f2fma(HC6, ST, f2mul(C7, CT)));
            const uint64_t AY = f2sub(f2mul(HC6, CT), f2mul(C7, ST));
            const uint64_t TU = f2fma(AX, G0, f2mul(QX, DG));
            const uint64_t TW = f2fma(AY, G0, f2mul(QY, DG));
            ACU = f2add(ACU, TU);
            ACW = f2add(ACW, TW);
        }
        ua += (double)f2lo(ACU);
        ub += (double)f2hi(ACU);
        wa += (double)f2lo(ACW);
        wb += (double)f2hi(ACW);
    }
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

// Convection update of one blob after its sheet velocity (modes 1: Euler; 2..4:
// the three RK3 stages, src/DVMBase.cpp:167-209).
__device__ __forceinline__ void sheet_store(const InstDesc& d, uint32_t i, double us, double ws,
                                            int mode) {
    const double xi = d.x[i], zi = d.z[i];
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

constexpr uint32_t kSheetItem = 512;  // blobs per work item: two per thread
constexpr size_t kSheetSmemPerPanel = 96;  // FP32: 4 FP64 + one PanelX2; FP64: 8 FP64 arrays

__global__ void __launch_bounds__(256) k_sheet_velocity(const InstDesc* __restrict__ table,
                                                        const InstState* __restrict__ st,
                                                        const ListEntry* __restrict__ list,
                                                        int nlist, int mode,
                                                        unsigned* __restrict__ work) {
    extern __shared__ double s_pan[];  // kSheetSmemPerPanel bytes per panel of max_np
    __shared__ unsigned s_pre[1025];
    __shared__ unsigned s_item;
    __shared__ int s_loaded;
    if (threadIdx.x == 0) {
        unsigned acc = 0;
        for (int k = 0; k < nlist; ++k) {
            s_pre[k] = acc;
            acc += (st[list[k].inst].n + kSheetItem - 1) / kSheetItem;
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
        // FP64 layout after xc, zc: ds, cos, sin, cos -2th, sin -2th, gamma
        double* sds = szc + np;
        double* sct = sds + np;
        double* sst = sct + np;
        double* sc2 = sst + np;
        double* ss2 = sc2 + np;
        double* sg = ss2 + np;
        // FP32 layout after xc, zc: the panel ends (FP64), then np PanelX2
        double* sex = szc + np;
        double* sez = sex + np;
        PanelX2* pan = reinterpret_cast<PanelX2*>(sez + np);
        if (s_loaded != k) {
            for (int j = threadIdx.x; j < np; j += blockDim.x) {
                sxc[j] = d.xc[j];
                szc[j] = d.zc[j];
                if (f32) {
                    const double dsj = d.ds[j];
                    sex[j] = d.xc[j] + dsj * d.cth[j];
                    sez[j] = d.zc[j] + dsj * d.sth[j];
                    const double g0 = d.gamma[j], g1 = d.gamma[j == np - 1 ? 0 : j + 1];
                    auto dup = [](double v) {
                        const float f = (float)v;
                        return f2pack(f, f);
                    };
                    PanelX2 P;
                    P.cs = make_ulonglong2(dup(d.cth[j]), dup(d.sth[j]));
                    P.dd = make_ulonglong2(dup(dsj), dup(1.0 / dsj));
                    P.cc = make_ulonglong2(dup(d.c2th[j]), dup(d.s2th[j]));
                    P.gd = make_ulonglong2(dup(g0), dup(g1 - g0));
                    pan[j] = P;
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
        const uint32_t ia = (item - s_pre[k]) * kSheetItem + threadIdx.x, ib = ia + 256;
        const bool acta = ia < n, actb = ib < n;
        if (f32) {
            // every lane runs the panel loop (its warp votes on the regime); a
            // blob slot past the count evaluates a point far from the body
            const double far_x = sxc[0] + 1.0e3, far_z = szc[0] + 1.0e3;
            double ua = 0.0, wa = 0.0, ub = 0.0, wb = 0.0;
            sheet_sum_f32x2(acta ? d.x[ia] : far_x, acta ? d.z[ia] : far_z,
                            actb ? d.x[ib] : far_x, actb ? d.z[ib] : far_z, np, sxc, szc, sex,
                            sez, pan, ua, wa, ub, wb);
            if (acta) sheet_store(d, ia, ua, wa, mode);
            if (actb) sheet_store(d, ib, ub, wb, mode);
        } else {
            for (int h = 0; h < 2; ++h) {
                const uint32_t i = h ? ib : ia;
                if (i >= n) continue;
                const double xi = d.x[i], zi = d.z[i];
                double us = 0.0, ws = 0.0;
                for (int j = 0; j < np; ++j)
                    sheet_pair_f64(dsub(xi, sxc[j]), dsub(zi, szc[j]), sds[j], sct[j], sst[j],
                                   sc2[j], ss2[j], sg[j], (j == np - 1) ? sg[0] : sg[j + 1], us,
                                   ws);
                sheet_store(d, i, us, ws, mode);
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

namespace {

// A body's factorisation workspace: M = [A | I] (m x (np + m), column-major),
// then the reflector buffer (2 m), v0s (np) and taus (np).
QrBody qr_body(int np, double* P, double* work) {
    const int m = np + 1, cols = np + m;
    QrBody b{};
    b.M = work;
    b.vbuf = b.M + (size_t)m * cols;
    b.v0s = b.vbuf + 2 * (size_t)m;
    b.taus = b.v0s + np;
    b.P = P;
    b.np = np;
    return b;
}

// Register class of m rows: CH = 9, 17, 33 values per lane, or -1 (general path).
int qr_class(int m) { return m <= 32 * 9 ? 0 : m <= 32 * 17 ? 1 : m <= 32 * 33 ? 2 : -1; }

template <int CH>
cudaError_t qr_group_launch(QrGroup& G, int qr_blocks, int bs_blocks, cudaStream_t s) {
    void* args[] = {&G};
    cudaError_t e = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_qr_reg<CH>),
                                                dim3(qr_blocks), dim3(256), args, 0, s);
    if (e != cudaSuccess) return e;
    k_backsub_reg<CH><<<bs_blocks, 256, 0, s>>>(G);
    return cudaGetLastError();
}

cudaError_t qr_group_launch(int cls, QrGroup& G, int qr_blocks, int bs_blocks, cudaStream_t s) {
    if (cls == 0) return qr_group_launch<9>(G, qr_blocks, bs_blocks, s);
    if (cls == 1) return qr_group_launch<17>(G, qr_blocks, bs_blocks, s);
    return qr_group_launch<33>(G, qr_blocks, bs_blocks, s);
}

// General path: one warp per column of A (columns in memory), then Q^T.
cudaError_t qr_general(const QrBody& b, int sms, cudaStream_t s) {
    double* M = b.M;
    double* vbuf = b.vbuf;
    double* v0s = b.v0s;
    double* taus = b.taus;
    int np = b.np;
    const int m = np + 1;
    int per_sm = 0;
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
    k_backsub<<<(m + wpb - 1) / wpb, wpb * 32, sizeof(double) * np * wpb, s>>>(M, np, b.P);
    return cudaGetLastError();
}

}  // namespace

cudaError_t pseudo_inverse_many(int n, const double* const* A, const int* np, double* const* P,
                                double* const* work, cudaStream_t s, int* launches) {
    int nl = 0;  // QR-stage launches (the loads of [A | I] are counted by the caller)
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int per[3] = {0, 0, 0};  // co-resident register-path blocks per SM, by class
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[0], k_qr_reg<9>, 256, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[1], k_qr_reg<17>, 256, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[2], k_qr_reg<33>, 256, 0);
    std::vector<QrBody> bodies(n);
    std::vector<int> cls(n);
    for (int i = 0; i < n; ++i) {
        bodies[i] = qr_body(np[i], P[i], work[i]);
        k_load_aug<<<256, 256, 0, s>>>(A[i], np[i], bodies[i].M);
        const int m = np[i] + 1, c = qr_class(m);
        // register path when one warp per column of [A | I] fits the GPU at once
        cls[i] = (c >= 0 && (np[i] + m + 7) / 8 <= per[c] * sms) ? c : -1;
    }
    // Register path: bodies of a class in order, up to kQrMaxBodies per launch and
    // as many as are co-resident together.
    for (int c = 0; c < 3; ++c) {
        QrGroup G{};
        int qb = 0, bb = 0;
        for (int i = 0; i <= n; ++i) {
            const bool last = i == n;
            if (!last && cls[i] != c) continue;
            const int need = last ? 0 : (2 * np[i] + 1 + 7) / 8;
            if (G.nb > 0 && (last || G.nb == kQrMaxBodies || qb + need > per[c] * sms)) {
                const cudaError_t e = qr_group_launch(c, G, qb, bb, s);
                if (e != cudaSuccess) return e;
                nl += 2;
                G = QrGroup{};
                qb = bb = 0;
            }
            if (last) break;
            QrBody b = bodies[i];
            b.qr_block0 = qb;
            b.bs_block0 = bb;
            G.b[G.nb++] = b;
            G.maxnp = std::max(G.maxnp, np[i]);
            qb += need;
            bb += (np[i] + 1 + 7) / 8;
        }
    }
    for (int i = 0; i < n; ++i) {
        if (cls[i] >= 0) continue;
        const cudaError_t e = qr_general(bodies[i], sms, s);
        if (e != cudaSuccess) return e;
        nl += 3;
    }
    if (launches) *launches = nl;
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
    const size_t smem = kSheetSmemPerPanel * (size_t)max_np;
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
