// Device helpers shared by the kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace dvmk {

// FP64 operations with exactly one rounding each, so that expressions written
// with them round like the reference's C++ compiled without FP contraction.
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// One MUFU reciprocal (relative error below 2^-22), +inf for 0.
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// One MUFU base-2 exponential (relative error below 2^-22 on B200-class parts).
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Packed FP32x2 arithmetic (sm_100): one instruction operates on a pair of
// values (two targets, or two blobs), halving the issue slots of a loop; each
// half is rounded exactly like the scalar instruction (round-to-nearest).
__device__ __forceinline__ uint64_t f2pack(float lo, float hi) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
// (one unpacking move; measured 0.7 % faster in the pair loop than shifts)
#pragma nv_diag_suppress 550  // the unpacked half that is not returned
__device__ __forceinline__ float f2lo(uint64_t v) {
    float lo, hi;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
    return lo;
}
__device__ __forceinline__ float f2hi(uint64_t v) {
    float lo, hi;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
    return hi;
}
#pragma nv_diag_default 550
__device__ __forceinline__ uint64_t f2sub(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t f2mul(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t f2fma(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

__device__ __forceinline__ uint64_t f2add(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11): 10 rounds of the
// 4x32 bijection with multipliers 0xD2511F53 / 0xCD9E8D57 and Weyl key
// increments 0x9E3779B9 / 0xBB67AE85.
struct U4 {
    uint32_t a, b, c, d;
};
__device__ __forceinline__ U4 philox4x32_10(U4 ctr, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, ctr.a);
        const uint32_t lo0 = 0xD2511F53u * ctr.a;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, ctr.c);
        const uint32_t lo1 = 0xCD9E8D57u * ctr.c;
        ctr = U4{hi1 ^ ctr.b ^ k0, lo1, hi0 ^ ctr.d ^ k1, lo0};
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return ctr;
}
// Two 53-bit uniforms in (0, 1] from one Philox block.
__device__ __forceinline__ void philox_uniform2(uint64_t seed, uint32_t i, uint32_t step,
                                                uint32_t uid, uint32_t stream, double& r1,
                                                double& r2) {
    const U4 o = philox4x32_10(U4{i, step, uid, stream}, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double s = 1.0 / 9007199254740992.0;  // 2^-53
    r1 = ((double)(((uint64_t)(o.a >> 5) << 26) | (o.b >> 6)) + 1.0) * s;
    r2 = ((double)(((uint64_t)(o.c >> 5) << 26) | (o.d >> 6)) + 1.0) * s;
}

// Largest k with pre[k] <= item (pre ascending, pre[0] = 0).
__device__ __forceinline__ int locate(const unsigned* pre, int nlist, unsigned item) {
    int lo = 0, hi = nlist - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

}  // namespace dvmk
