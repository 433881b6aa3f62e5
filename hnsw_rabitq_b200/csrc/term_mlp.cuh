// Learned early termination of the level-0 beam: the search-state features
// and the in-warp inference of the termination network (sm_100a).
//
// Every `term_period` expansions the beam computes a feature vector of its
// state; a 16 -> 64 -> 64 -> 1 ReLU network (fp16 weights and activations on
// the tensor cores, fp32 accumulation)
// maps it to the logit of "the current top-k is already the final one", and
// the query stops when the logit exceeds a calibrated threshold.  The same
// functions serve the checkpoint traces the network is trained on, the
// in-search inference and the stand-alone inference kernel used to test it,
// so the three cannot drift apart.
#pragma once
#include <cuda_fp16.h>

#include <cstdint>

#include "device_common.cuh"
#include "hnsw_search.h"

namespace hnswgpu {

// Features of the beam after `e` level-0 expansions (a = |d_k|):
//   f0  log2(1 + e)                    f8  log2(1 + n(0.1))
//   f1  d_1 / a                        f9  log2(1 + n(0.25))
//   f2  (d_next - d_k) / a             f10 log2(1 + n(0.5))
//   f3  log2(1 + d_entry / a)          f11 waiting candidates / ef
//   f4  log2(1 + |q|^2)                f12 beam size / ef
//   f5  expansions since the top-k     f13 log2(1 + expansions that changed
//       last changed / T                   the top-k)
//   f6  (d_wait - d_k) / a             f14 distance evaluations per expansion
//   f7  (d_worst - d_k) / a                since the previous checkpoint
//                                      f15 (d_median - d_k) / a
// d_1 / d_k: best and k-th beam distances; d_next: the candidate expanded
// next; d_entry: the level-0 entry point's distance; waiting candidates: beam
// entries not expanded yet, d_wait the closest of them (after the ones taken
// for expansion), n(x) how many are closer than d_k + x a; d_worst / d_median:
// the beam's last and middle entries.  Ratios are clamped to [-4, 4].
struct TermInputs {
    float e, d1, dk, dn, d_entry, qn;
    float since_change, inv_period;
    float nchange;    // expansions that changed the top-k so far
    float eval_rate;  // distance evaluations per expansion since the previous checkpoint
};

// (d - d_k) / |d_k| clamped to [-4, 4]; inv_a = 1 / |d_k|
__device__ __forceinline__ float term_ratio(float d, float dk, float inv_a) {
    return fminf(fmaxf((d - dk) * inv_a, -4.f), 4.f);
}

// f6 .. f12 and f15 from the sorted beam (distance key << 32 | id, EXP_BIT on
// expanded entries), psize >= 1 entries; whole warp, identical in every lane.
__device__ __forceinline__ void term_pool_features(const uint64_t* pool, int psize, int ef, float dk, int lane,
                                                   float f[kTermFeatures]) {
    const float a = fabsf(dk) + 1e-30f, inv_a = 1.0f / a;
    const uint32_t t1 = fkey(dk + 0.1f * a), t2 = fkey(dk + 0.25f * a), t3 = fkey(dk + 0.5f * a);
    int n1 = 0, n2 = 0, n3 = 0, nw = 0;
    uint32_t first_wait = 0xffffffffu;
    for (int b = 0; b < psize; b += 32) {
        const int i = b + lane;
        const uint64_t e = i < psize ? pool[i] : ~0ull;
        const uint32_t h = khi(e);
        const bool w = i < psize && !((uint32_t)e & EXP_BIT);
        const unsigned mw = __ballot_sync(0xffffffffu, w);
        if (first_wait == 0xffffffffu && mw) first_wait = __shfl_sync(0xffffffffu, h, __ffs(mw) - 1);
        nw += __popc(mw);
        n1 += __popc(__ballot_sync(0xffffffffu, w && h < t1));
        n2 += __popc(__ballot_sync(0xffffffffu, w && h < t2));
        n3 += __popc(__ballot_sync(0xffffffffu, w && h < t3));
    }
    const float inv_ef = 1.0f / (float)ef;
    f[6] = first_wait == 0xffffffffu ? 4.f : term_ratio(funkey(first_wait), dk, inv_a);
    f[7] = term_ratio(funkey(khi(pool[psize - 1])), dk, inv_a);
    f[8] = __log2f(1.0f + (float)n1);
    f[9] = __log2f(1.0f + (float)n2);
    f[10] = __log2f(1.0f + (float)n3);
    f[11] = (float)nw * inv_ef;
    f[12] = (float)psize * inv_ef;
    f[15] = term_ratio(funkey(khi(pool[psize >> 1])), dk, inv_a);
}

// All features: the scalar ones here, the beam's from term_pool_features.
__device__ __forceinline__ void term_features(const TermInputs& in, const uint64_t* pool, int psize, int ef,
                                              int lane, float f[kTermFeatures]) {
    const float inv_a = 1.0f / (fabsf(in.dk) + 1e-30f);
    f[0] = __log2f(1.0f + in.e);
    f[1] = fminf(fmaxf(in.d1 * inv_a, -4.f), 4.f);
    f[2] = term_ratio(in.dn, in.dk, inv_a);
    f[3] = __log2f(1.0f + fminf(fmaxf(in.d_entry * inv_a, 0.f), 1e6f));
    f[4] = __log2f(1.0f + in.qn);
    f[5] = fminf(in.since_change * in.inv_period, 16.f);
    f[13] = __log2f(1.0f + in.nchange);
    f[14] = fminf(in.eval_rate, 64.f);
    term_pool_features(pool, psize, ef, in.dk, lane, f);
}

// Trace mode: float32 distances (in any summation order) of the first w beam
// entries, recomputed from the float32 rows, so that the checkpoints of a
// low-precision beam are labelled by what its re-rank would return.  `q` is
// the (normalised) query padded with zeros to row_floats; 8 rows per pass,
// 4 lanes per row; whole warp.
template <int SPACE>
__device__ __forceinline__ void trace_dists(const SearchParams& p, const float* q, const uint64_t* pool, int w,
                                            int lane, float* out) {
    const int a = lane & 3;
    const int n4 = (int)(p.row_floats >> 2);
    const float4* q4 = reinterpret_cast<const float4*>(q);
    for (int b = 0; b < w; b += 8) {
        const int v = b + (lane >> 2);
        uint32_t id = v < w ? kid(pool[v]) : 0u;
        if (id >= p.count) id = 0;
        const float4* x4 = reinterpret_cast<const float4*>(p.vecs + (size_t)id * p.row_floats);
        float acc = 0.f;
        for (int c = a; c < n4; c += 4) {
            const float4 x = __ldg(x4 + c), y = q4[c];
            if (SPACE == 0) {
                const float d0 = y.x - x.x, d1 = y.y - x.y, d2 = y.z - x.z, d3 = y.w - x.w;
                acc = fmaf(d0, d0, fmaf(d1, d1, fmaf(d2, d2, fmaf(d3, d3, acc))));
            } else {
                acc = fmaf(y.x, x.x, fmaf(y.y, x.y, fmaf(y.z, x.z, fmaf(y.w, x.w, acc))));
            }
        }
        acc += __shfl_xor_sync(0xffffffffu, acc, 1);
        acc += __shfl_xor_sync(0xffffffffu, acc, 2);
        if (a == 0 && v < w) out[v] = SPACE == 0 ? acc : 1.0f - acc;
    }
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
// `m` is the packed inference form (pack_term_model), in global memory or,
// with SMEM, in shared memory.
// Loads of the packed network: read-only cache, or shared memory (SMEM).
template <bool SMEM, class T>
__device__ __forceinline__ T term_ld(const T* p) {
    if (SMEM) return *p;
    return __ldg(p);
}

template <bool SMEM = false>
__device__ __forceinline__ float term_logit(const float* __restrict__ m, const float f[kTermFeatures], int lane) {
    constexpr unsigned kFull = 0xffffffffu;
    const int t = lane & 3;
    const float* mu = m;
    const float* inv_sigma = m + kTermFeatures;
    const float b3 = term_ld<SMEM>(m + 2 * kTermFeatures);
    const float4* b1f = reinterpret_cast<const float4*>(m + kTermPackedHead) + t * 4;  // [t][8] float2
    const float4* b2f = reinterpret_cast<const float4*>(m + kTermPackedHead + 64) + t * 4;
    const uint4* w3f = reinterpret_cast<const uint4*>(m + kTermPackedFloats) + t * 2;  // [t][8] half2
    const uint4* W1f = reinterpret_cast<const uint4*>(m + kTermPackedFloats) + 8 + lane * 4;
    const uint4* W2f = reinterpret_cast<const uint4*>(m + kTermPackedFloats) + 8 + 128 + lane * 16;
    // layer 1: A row = (x[2t], x[2t + 1]) for k = 2t, 2t + 1 and (x[2t + 8],
    // x[2t + 9]) for k = 2t + 8, 2t + 9
    float x0 = 0.f, x1 = 0.f, x2 = 0.f, x3 = 0.f;
#pragma unroll
    for (int i = 0; i < 8; i += 2) {
        if (2 * t == i) {
            x0 = (f[i] - term_ld<SMEM>(mu + i)) * term_ld<SMEM>(inv_sigma + i);
            x1 = (f[i + 1] - term_ld<SMEM>(mu + i + 1)) * term_ld<SMEM>(inv_sigma + i + 1);
            x2 = (f[i + 8] - term_ld<SMEM>(mu + i + 8)) * term_ld<SMEM>(inv_sigma + i + 8);
            x3 = (f[i + 9] - term_ld<SMEM>(mu + i + 9)) * term_ld<SMEM>(inv_sigma + i + 9);
        }
    }
    const uint32_t ax = pack_half2(x0, x1), ay = pack_half2(x2, x3);
    __syncwarp();
    uint32_t a2[8];  // layer-2 A fragments: tile v of layer 1 as (unit 8v + 2t, 8v + 2t + 1)
#pragma unroll
    for (int v = 0; v < 8; v++) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        const uint2 w = term_ld<SMEM>(reinterpret_cast<const uint2*>(W1f) + v);
        mma_f16(c, ax, ax, ay, ay, w.x, w.y);
        const float4 bb = term_ld<SMEM>(b1f + (v >> 1));
        const float bx = (v & 1) ? bb.z : bb.x, by = (v & 1) ? bb.w : bb.y;
        a2[v] = pack_half2(fmaxf(c[0] + bx, 0.f), fmaxf(c[1] + by, 0.f));
    }
    // layer 2, one output tile at a time (few live accumulators): k-step s
    // uses units 16s + 2t (+1) (tile 2s) and 16s + 2t + 8 (+9) (tile 2s + 1);
    // then bias, ReLU and the output weights of the tile's units 8v + 2t, + 1
    float sum = 0.f;
#pragma unroll 2
    for (int v = 0; v < 8; v++) {
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int st = 0; st < 4; st++) {
            const uint2 w = term_ld<SMEM>(reinterpret_cast<const uint2*>(W2f) + st * 8 + v);
            mma_f16(acc, a2[2 * st], a2[2 * st], a2[2 * st + 1], a2[2 * st + 1], w.x, w.y);
        }
        const float2 bb = term_ld<SMEM>(reinterpret_cast<const float2*>(b2f) + v);
        const uint32_t wv = term_ld<SMEM>(reinterpret_cast<const uint32_t*>(w3f) + v);
        const float2 o = __half22float2(*reinterpret_cast<const __half2*>(&wv));
        sum = fmaf(o.x, fmaxf(acc[0] + bb.x, 0.f), sum);
        sum = fmaf(o.y, fmaxf(acc[1] + bb.y, 0.f), sum);
    }
    sum += __shfl_xor_sync(kFull, sum, 1);
    sum += __shfl_xor_sync(kFull, sum, 2);
    return sum + b3;
}

}  // namespace hnswgpu
