// Device helpers shared by the search kernels (sm_100a).
//
//  * TMA 1-D bulk copies (cp.async.bulk, no multicast) completing on an
//    mbarrier, with bounded waits;
//  * 64-bit ordered (distance, id) keys;
//  * L2Sqr / InnerProductDistance evaluated by one thread in exactly the
//    floating-point order of the reference's AVX-512 build
//    (hnswlib/space_l2.h:6-253, hnswlib/space_ip.h:6-398; see the oracle for
//    the derivation of the tail and reduction orders).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace hnswgpu {

constexpr unsigned FULL = 0xffffffffu;
constexpr uint32_t INVALID_ID = 0xffffffffu;
constexpr uint32_t EXP_BIT = 0x80000000u;                 // "expanded" flag in a key's id field
constexpr uint64_t KEY_MASK = ~(uint64_t)EXP_BIT;         // key without the flag
// Bounded mbarrier wait: each try_wait may suspend the thread for up to
// MBAR_SUSPEND_NS (it wakes as soon as the phase completes), at most
// MBAR_SPIN_LIMIT times -- a few seconds in total before giving up.
constexpr uint32_t MBAR_SPIN_LIMIT = 1u << 16;
constexpr uint32_t MBAR_SUSPEND_NS = 50000;

// ------------------------------------------------------------------ keys
// Order-preserving map of a float to uint32 (monotone on all non-NaN values).
__device__ __forceinline__ uint32_t fkey(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float funkey(uint32_t k) {
    uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    return __uint_as_float(u);
}
__device__ __forceinline__ uint64_t mkkey(float d, uint32_t id) { return ((uint64_t)fkey(d) << 32) | id; }
__device__ __forceinline__ uint32_t khi(uint64_t k) { return (uint32_t)(k >> 32); }
__device__ __forceinline__ uint32_t kid(uint64_t k) { return (uint32_t)k & ~EXP_BIT; }

// Slot of node `id` in a direct-mapped visited cache of 2^log2v entries.
__device__ __forceinline__ uint32_t vis_slot(uint32_t id, uint32_t log2v) {
    return (id * 0x9E3779B1u) >> (32 - log2v);
}

__device__ __forceinline__ uint64_t shfl64(uint64_t v, int src) {
    uint32_t lo = __shfl_sync(FULL, (uint32_t)v, src);
    uint32_t hi = __shfl_sync(FULL, (uint32_t)(v >> 32), src);
    return ((uint64_t)hi << 32) | lo;
}
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ------------------------------------------------------ mbarrier + bulk copy
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// Bounded wait for the completion of the phase with parity `parity`: at most
// `limit` tries (each may suspend up to MBAR_SUSPEND_NS); false when it gave up.
__device__ __forceinline__ bool mbar_wait_limit(uint64_t* bar, uint32_t parity, uint32_t limit) {
    uint32_t addr = smem_u32(bar);
    for (uint32_t it = 0; it < limit; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity), "r"(MBAR_SUSPEND_NS)
            : "memory");
        if (done) return true;
    }
    return false;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    return mbar_wait_limit(bar, parity, MBAR_SPIN_LIMIT);
}
// One TMA bulk copy global -> shared (no multicast); `bytes` and both
// addresses are multiples of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// --------------------------------------------------------------- distances
// q, x: 16-byte aligned float arrays of at least round_up(dim, 4) floats.
// All arithmetic is IEEE round-to-nearest: __fadd_rn / __fmul_rn / __fmaf_rn
// so that nvcc cannot contract or reorder anything.

__device__ __forceinline__ float l2_simd16(const float* __restrict__ q, const float* __restrict__ x, int n16) {
    float acc[16];
#pragma unroll
    for (int l = 0; l < 16; l++) acc[l] = 0.f;
    const float4* q4 = reinterpret_cast<const float4*>(q);
    const float4* x4 = reinterpret_cast<const float4*>(x);
    for (int c = 0; c < n16; c++) {
#pragma unroll
        for (int u = 0; u < 4; u++) {
            float4 a = q4[4 * c + u], b = x4[4 * c + u];
            float t0 = __fsub_rn(a.x, b.x), t1 = __fsub_rn(a.y, b.y), t2 = __fsub_rn(a.z, b.z),
                  t3 = __fsub_rn(a.w, b.w);
            acc[4 * u + 0] = __fmaf_rn(t0, t0, acc[4 * u + 0]);
            acc[4 * u + 1] = __fmaf_rn(t1, t1, acc[4 * u + 1]);
            acc[4 * u + 2] = __fmaf_rn(t2, t2, acc[4 * u + 2]);
            acc[4 * u + 3] = __fmaf_rn(t3, t3, acc[4 * u + 3]);
        }
    }
    float r = acc[0];
#pragma unroll
    for (int l = 1; l < 16; l++) r = __fadd_rn(r, acc[l]);
    return r;
}

__device__ __forceinline__ float l2_simd4(const float* __restrict__ q, const float* __restrict__ x, int n4) {
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
    const float4* q4 = reinterpret_cast<const float4*>(q);
    const float4* x4 = reinterpret_cast<const float4*>(x);
    for (int c = 0; c < n4; c++) {
        float4 a = q4[c], b = x4[c];
        float t0 = __fsub_rn(a.x, b.x), t1 = __fsub_rn(a.y, b.y), t2 = __fsub_rn(a.z, b.z), t3 = __fsub_rn(a.w, b.w);
        a0 = __fmaf_rn(t0, t0, a0);
        a1 = __fmaf_rn(t1, t1, a1);
        a2 = __fmaf_rn(t2, t2, a2);
        a3 = __fmaf_rn(t3, t3, a3);
    }
    return __fadd_rn(__fadd_rn(__fadd_rn(a0, a1), a2), a3);
}

// Scalar L2Sqr tail as the reference compiler emits it: 4-wide in-order
// rounded products, then fma for the last qty % 4 terms.
__device__ __forceinline__ float l2_scalar(const float* q, const float* x, int qty) {
    float r = 0.f;
    int n4 = qty & ~3;
    for (int i = 0; i < n4; i++) {
        float t = __fsub_rn(q[i], x[i]);
        r = __fadd_rn(r, __fmul_rn(t, t));
    }
    for (int i = n4; i < qty; i++) {
        float t = __fsub_rn(q[i], x[i]);
        r = __fmaf_rn(t, t, r);
    }
    return r;
}

__device__ __forceinline__ float dist_l2(const float* q, const float* x, int dim) {
    if ((dim & 15) == 0) return l2_simd16(q, x, dim >> 4);
    if ((dim & 3) == 0) return l2_simd4(q, x, dim >> 2);
    if (dim > 16) {
        int d16 = dim & ~15;
        return __fadd_rn(l2_simd16(q, x, dim >> 4), l2_scalar(q + d16, x + d16, dim - d16));
    }
    if (dim > 4) {
        int d4 = dim & ~3;
        return __fadd_rn(l2_simd4(q, x, dim >> 2), l2_scalar(q + d4, x + d4, dim - d4));
    }
    return l2_scalar(q, x, dim);
}

// AVX-512 inner product body + GCC's _mm512_reduce_add_ps tree.
__device__ __forceinline__ float ip_simd16(const float* __restrict__ q, const float* __restrict__ x, int n16) {
    float acc[16];
#pragma unroll
    for (int l = 0; l < 16; l++) acc[l] = 0.f;
    const float4* q4 = reinterpret_cast<const float4*>(q);
    const float4* x4 = reinterpret_cast<const float4*>(x);
    for (int c = 0; c < n16; c++) {
#pragma unroll
        for (int u = 0; u < 4; u++) {
            float4 a = q4[4 * c + u], b = x4[4 * c + u];
            acc[4 * u + 0] = __fmaf_rn(a.x, b.x, acc[4 * u + 0]);
            acc[4 * u + 1] = __fmaf_rn(a.y, b.y, acc[4 * u + 1]);
            acc[4 * u + 2] = __fmaf_rn(a.z, b.z, acc[4 * u + 2]);
            acc[4 * u + 3] = __fmaf_rn(a.w, b.w, acc[4 * u + 3]);
        }
    }
    float t3[8], t6[4];
#pragma unroll
    for (int i = 0; i < 8; i++) t3[i] = __fadd_rn(acc[i + 8], acc[i]);
#pragma unroll
    for (int i = 0; i < 4; i++) t6[i] = __fadd_rn(t3[i + 4], t3[i]);
    return __fadd_rn(__fadd_rn(t6[0], t6[2]), __fadd_rn(t6[1], t6[3]));
}

// AVX 8-lane inner product folded to 4 lanes, then SSE 4-lane chunks.
__device__ __forceinline__ float ip_simd4(const float* __restrict__ q, const float* __restrict__ x, int qty) {
    int n16 = qty >> 4, n4 = qty >> 2;
    float a8[8];
#pragma unroll
    for (int i = 0; i < 8; i++) a8[i] = 0.f;
    const float4* q4 = reinterpret_cast<const float4*>(q);
    const float4* x4 = reinterpret_cast<const float4*>(x);
    for (int c = 0; c < n16; c++) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            float4 a0 = q4[4 * c + 2 * h], b0 = x4[4 * c + 2 * h];
            float4 a1 = q4[4 * c + 2 * h + 1], b1 = x4[4 * c + 2 * h + 1];
            a8[0] = __fmaf_rn(a0.x, b0.x, a8[0]);
            a8[1] = __fmaf_rn(a0.y, b0.y, a8[1]);
            a8[2] = __fmaf_rn(a0.z, b0.z, a8[2]);
            a8[3] = __fmaf_rn(a0.w, b0.w, a8[3]);
            a8[4] = __fmaf_rn(a1.x, b1.x, a8[4]);
            a8[5] = __fmaf_rn(a1.y, b1.y, a8[5]);
            a8[6] = __fmaf_rn(a1.z, b1.z, a8[6]);
            a8[7] = __fmaf_rn(a1.w, b1.w, a8[7]);
        }
    }
    float s0 = __fadd_rn(a8[0], a8[4]), s1 = __fadd_rn(a8[1], a8[5]), s2 = __fadd_rn(a8[2], a8[6]),
          s3 = __fadd_rn(a8[3], a8[7]);
    for (int c = 4 * n16; c < n4; c++) {
        float4 a = q4[c], b = x4[c];
        s0 = __fmaf_rn(a.x, b.x, s0);
        s1 = __fmaf_rn(a.y, b.y, s1);
        s2 = __fmaf_rn(a.z, b.z, s2);
        s3 = __fmaf_rn(a.w, b.w, s3);
    }
    return __fadd_rn(__fadd_rn(__fadd_rn(s0, s1), s2), s3);
}

__device__ __forceinline__ float ip_scalar(const float* q, const float* x, int qty) {
    float r = 0.f;
    for (int i = 0; i < qty; i++) r = __fmaf_rn(q[i], x[i], r);
    return r;
}

__device__ __forceinline__ float dist_ip(const float* q, const float* x, int dim) {
    if ((dim & 15) == 0) return __fsub_rn(1.0f, ip_simd16(q, x, dim >> 4));
    if ((dim & 3) == 0) return __fsub_rn(1.0f, ip_simd4(q, x, dim));
    if (dim > 16) {
        int d16 = dim & ~15;
        return __fsub_rn(1.0f, __fadd_rn(ip_simd16(q, x, dim >> 4), ip_scalar(q + d16, x + d16, dim - d16)));
    }
    if (dim > 4) {
        int d4 = dim & ~3;
        return __fsub_rn(1.0f, __fadd_rn(ip_simd4(q, x, d4), ip_scalar(q + d4, x + d4, dim - d4)));
    }
    return __fsub_rn(1.0f, ip_scalar(q, x, dim));
}

template <int SPACE>
__device__ __forceinline__ float group4_reduce(float c0, float c1, float c2, float c3);

// The dim % 16 == 0 distance split over a group of 4 lanes (a = lane & 3):
// lane a keeps the reference's accumulators 4a .. 4a+3 (one float4 of each
// 16-float chunk), so one LDS.128 per chunk per lane feeds 8 vectors per warp
// instruction.  The cross-lane reduction reproduces the reference order
// exactly: L2 sums the 16 accumulators left to right (space_l2.h:49-51), IP
// applies GCC's _mm512_reduce_add_ps tree then 1 - x.  All 32 lanes must call
// it (it shuffles); the result is valid in lanes with a == 0.
template <int SPACE>
__device__ __forceinline__ float group4_dist16(const float* __restrict__ q, const float* __restrict__ x, int n16,
                                               int a) {
    const float4* q4 = reinterpret_cast<const float4*>(q);
    const float4* x4 = reinterpret_cast<const float4*>(x);
    float c0 = 0.f, c1 = 0.f, c2 = 0.f, c3 = 0.f;
    for (int c = 0; c < n16; c++) {
        float4 qv = q4[4 * c + a], xv = x4[4 * c + a];
        if (SPACE == 0) {
            float t0 = __fsub_rn(qv.x, xv.x), t1 = __fsub_rn(qv.y, xv.y), t2 = __fsub_rn(qv.z, xv.z),
                  t3 = __fsub_rn(qv.w, xv.w);
            c0 = __fmaf_rn(t0, t0, c0);
            c1 = __fmaf_rn(t1, t1, c1);
            c2 = __fmaf_rn(t2, t2, c2);
            c3 = __fmaf_rn(t3, t3, c3);
        } else {
            c0 = __fmaf_rn(qv.x, xv.x, c0);
            c1 = __fmaf_rn(qv.y, xv.y, c1);
            c2 = __fmaf_rn(qv.z, xv.z, c2);
            c3 = __fmaf_rn(qv.w, xv.w, c3);
        }
    }
    return group4_reduce<SPACE>(c0, c1, c2, c3);
}

// Cross-lane reduction of group4_dist16: lane a of a 4-lane group holds the
// reference's accumulators 4a .. 4a+3.
template <int SPACE>
__device__ __forceinline__ float group4_reduce(float c0, float c1, float c2, float c3) {
    if (SPACE == 0) {
        // accumulators 4..15 from the three lanes to the right
        float b0 = __shfl_down_sync(FULL, c0, 1), b1 = __shfl_down_sync(FULL, c1, 1);
        float b2 = __shfl_down_sync(FULL, c2, 1), b3 = __shfl_down_sync(FULL, c3, 1);
        float e0 = __shfl_down_sync(FULL, c0, 2), e1 = __shfl_down_sync(FULL, c1, 2);
        float e2 = __shfl_down_sync(FULL, c2, 2), e3 = __shfl_down_sync(FULL, c3, 2);
        float f0 = __shfl_down_sync(FULL, c0, 3), f1 = __shfl_down_sync(FULL, c1, 3);
        float f2 = __shfl_down_sync(FULL, c2, 3), f3 = __shfl_down_sync(FULL, c3, 3);
        float r = __fadd_rn(__fadd_rn(__fadd_rn(c0, c1), c2), c3);
        r = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(r, b0), b1), b2), b3);
        r = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(r, e0), e1), e2), e3);
        r = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(r, f0), f1), f2), f3);
        return r;
    } else {
        // T3[i] = a[i+8] + a[i]: lanes 0,1 pair with lanes 2,3
        float u0 = __fadd_rn(__shfl_down_sync(FULL, c0, 2), c0);
        float u1 = __fadd_rn(__shfl_down_sync(FULL, c1, 2), c1);
        float u2 = __fadd_rn(__shfl_down_sync(FULL, c2, 2), c2);
        float u3 = __fadd_rn(__shfl_down_sync(FULL, c3, 2), c3);
        // T6[i] = T3[i+4] + T3[i]: lane 0 pairs with lane 1
        float v0 = __fadd_rn(__shfl_down_sync(FULL, u0, 1), u0);
        float v1 = __fadd_rn(__shfl_down_sync(FULL, u1, 1), u1);
        float v2 = __fadd_rn(__shfl_down_sync(FULL, u2, 1), u2);
        float v3 = __fadd_rn(__shfl_down_sync(FULL, u3, 1), u3);
        return __fsub_rn(1.0f, __fadd_rn(__fadd_rn(v0, v2), __fadd_rn(v1, v3)));
    }
}

template <int SPACE>
__device__ __forceinline__ float distance(const float* q, const float* x, int dim) {
    if (SPACE == 0) return dist_l2(q, x, dim);
    return dist_ip(q, x, dim);
}

// normalize_vector (python_bindings/bindings.cpp:241-248), run by one lane:
// returns the scale 1 / (sqrt(sum x^2) + 1e-30) with the sum in the
// reference compiler's order (4-wide in-order rounded products + fma tail).
__device__ __forceinline__ float norm_scale(const float* x, int dim) {
    float s = 0.f;
    int n4 = dim & ~3;
    for (int i = 0; i < n4; i++) s = __fadd_rn(s, __fmul_rn(x[i], x[i]));
    for (int i = n4; i < dim; i++) s = __fmaf_rn(x[i], x[i], s);
    return __fdiv_rn(1.0f, __fadd_rn(__fsqrt_rn(s), 1e-30f));
}

}  // namespace hnswgpu
