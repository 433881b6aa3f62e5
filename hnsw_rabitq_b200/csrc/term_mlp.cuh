// Learned early termination of the level-0 beam: the search-state features
// and the in-warp inference of the termination network (sm_100a).
//
// Every `term_period` expansions the beam computes a feature vector of its
// state; a 6 -> 64 -> 64 -> 1 ReLU network (fp16 weights and activations on
// the tensor cores, fp32 accumulation)
// maps it to the logit of "the current top-k is already the final one", and
// the query stops when the logit exceeds a calibrated threshold.  The same
// two functions serve the checkpoint traces the network is trained on, the
// in-search inference and the stand-alone inference kernel used to test it,
// so the three cannot drift apart.
#pragma once
#include <cuda_fp16.h>

#include <cstdint>

#include "hnsw_search.h"

namespace hnswgpu {

// Features of the beam after `e` level-0 expansions:
//   f0 log2(1 + e)                      f3 log2(1 + d_entry / |d_k|)
//   f1 d_1 / |d_k|                      f4 log2(1 + |q|^2)
//   f2 (d_next - d_k) / |d_k|           f5 expansions since the top-k last changed / T
// d_1 / d_k: best and k-th pool distances; d_next: the distance of the
// candidate expanded next; d_entry: the level-0 entry point's distance.
__device__ __forceinline__ void term_features(float e, float d1, float dk, float dn, float d_entry, float qn,
                                              float since_change, float inv_period, float f[kTermFeatures]) {
    const float a = fabsf(dk) + 1e-30f;
    f[0] = __log2f(1.0f + e);
    f[1] = fminf(fmaxf(d1 / a, -4.f), 4.f);
    f[2] = fminf(fmaxf((dn - dk) / a, -4.f), 4.f);
    f[3] = __log2f(1.0f + fminf(fmaxf(d_entry / a, 0.f), 1e6f));
    f[4] = __log2f(1.0f + qn);
    f[5] = fminf(since_change * inv_period, 16.f);
}

__device__ __forceinline__ void mma_f16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                        uint32_t b0, uint32_t b1) {
    asm("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_half2(float lo, float hi) {
    const __half2 h = __floats2half2_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// The network's logit for one feature vector (identical in every lane),
// computed by the whole warp (converged) on the tensor cores.  Each layer is
// a row vector times a 64-column weight matrix: the vector is replicated in
// every row of the m16n8k16 A operand, so every lane's accumulators hold
// units 8v + 2t and 8v + 2t + 1 of tile v; the layer-1 accumulators, after
// bias and ReLU, are exactly the A fragments of layer 2.  Operands are fp16
// (standardised features, hidden activations, weights), accumulation fp32.
// `m` is the packed inference form (pack_term_model).
__device__ __forceinline__ float term_logit(const float* __restrict__ m, const float f[kTermFeatures], int lane) {
    constexpr unsigned kFull = 0xffffffffu;
    const int t = lane & 3;
    const float* mu = m;
    const float* inv_sigma = m + kTermFeatures;
    const float b3 = __ldg(m + 2 * kTermFeatures);
    const float4* b1f = reinterpret_cast<const float4*>(m + 16) + t * 4;         // [t][8] float2
    const float4* b2f = reinterpret_cast<const float4*>(m + 16 + 64) + t * 4;
    const uint4* w3f = reinterpret_cast<const uint4*>(m + kTermPackedFloats) + t * 2;  // [t][8] half2
    const uint4* W1f = reinterpret_cast<const uint4*>(m + kTermPackedFloats) + 8 + lane * 2;
    const uint4* W2f = reinterpret_cast<const uint4*>(m + kTermPackedFloats) + 8 + 64 + lane * 16;
    // layer 1: A row = (x[2t], x[2t + 1]) for k = 2t, 2t + 1 (features 6, 7 and k >= 8 are zero)
    float x0 = 0.f, x1 = 0.f;
#pragma unroll
    for (int i = 0; i < kTermFeatures; i += 2) {
        if (2 * t == i) {
            x0 = (f[i] - __ldg(mu + i)) * __ldg(inv_sigma + i);
            x1 = (f[i + 1] - __ldg(mu + i + 1)) * __ldg(inv_sigma + i + 1);
        }
    }
    const uint32_t ax = pack_half2(x0, x1);
    uint32_t w1[8];
    {
        const uint4 u0 = __ldg(W1f), u1 = __ldg(W1f + 1);
        w1[0] = u0.x; w1[1] = u0.y; w1[2] = u0.z; w1[3] = u0.w;
        w1[4] = u1.x; w1[5] = u1.y; w1[6] = u1.z; w1[7] = u1.w;
    }
    __syncwarp();
    uint32_t a2[8];  // layer-2 A fragments: tile v of layer 1 as (unit 8v + 2t, 8v + 2t + 1)
#pragma unroll
    for (int v = 0; v < 8; v++) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        mma_f16(c, ax, ax, 0u, 0u, w1[v], 0u);
        const float4 bb = __ldg(b1f + (v >> 1));
        const float bx = (v & 1) ? bb.z : bb.x, by = (v & 1) ? bb.w : bb.y;
        a2[v] = pack_half2(fmaxf(c[0] + bx, 0.f), fmaxf(c[1] + by, 0.f));
    }
    // layer 2: k-step s uses units 16s + 2t (+1) (tile 2s) and 16s + 2t + 8 (+9) (tile 2s + 1)
    float acc[8][4];
#pragma unroll
    for (int v = 0; v < 8; v++) acc[v][0] = acc[v][1] = acc[v][2] = acc[v][3] = 0.f;
#pragma unroll
    for (int st = 0; st < 4; st++) {
        uint32_t wb[16];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const uint4 u = __ldg(W2f + st * 4 + i);
            wb[4 * i] = u.x; wb[4 * i + 1] = u.y; wb[4 * i + 2] = u.z; wb[4 * i + 3] = u.w;
        }
#pragma unroll
        for (int v = 0; v < 8; v++)
            mma_f16(acc[v], a2[2 * st], a2[2 * st], a2[2 * st + 1], a2[2 * st + 1], wb[2 * v], wb[2 * v + 1]);
    }
    float sum = 0.f;
#pragma unroll
    for (int v = 0; v < 8; v += 2) {
        const float4 bb = __ldg(b2f + (v >> 1));
        const uint4 wq = __ldg(w3f + (v >> 2));
        const uint32_t wa = (v & 2) ? wq.z : wq.x, wc = (v & 2) ? wq.w : wq.y;
        const float2 o0 = __half22float2(*reinterpret_cast<const __half2*>(&wa));
        const float2 o1 = __half22float2(*reinterpret_cast<const __half2*>(&wc));
        sum = fmaf(o0.x, fmaxf(acc[v][0] + bb.x, 0.f), sum);
        sum = fmaf(o0.y, fmaxf(acc[v][1] + bb.y, 0.f), sum);
        sum = fmaf(o1.x, fmaxf(acc[v + 1][0] + bb.z, 0.f), sum);
        sum = fmaf(o1.y, fmaxf(acc[v + 1][1] + bb.w, 0.f), sum);
    }
    sum += __shfl_xor_sync(kFull, sum, 1);
    sum += __shfl_xor_sync(kFull, sum, 2);
    return sum + b3;
}

}  // namespace hnswgpu
