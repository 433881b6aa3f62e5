// Learned early termination of the level-0 beam: the search-state features
// and the in-warp inference of the termination network (sm_100a).
//
// Every `term_period` expansions the beam computes a feature vector of its
// state; a 6 -> 64 -> 64 -> 1 ReLU network (fp16 weights, fp32 accumulation)
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

// The network's logit for one feature vector (identical in every lane),
// computed by the whole warp: lane j owns hidden units 2j and 2j + 1 of both
// hidden layers.  `m` is the packed inference form (pack_term_model), read
// with coalesced loads: each step of layer 2 reads 256 contiguous bytes.
__device__ __forceinline__ float term_logit(const float* __restrict__ m, const float f[kTermFeatures], int lane) {
    constexpr unsigned kFull = 0xffffffffu;
    const float* mu = m;
    const float* inv_sigma = m + kTermFeatures;
    const float* b1 = m + 2 * kTermFeatures;
    const float* b2 = b1 + kTermHidden;
    const float b3 = __ldg(b2 + kTermHidden);
    const __half* W1 = reinterpret_cast<const __half*>(m + kTermPackedFloats);
    const uint2* W2 = reinterpret_cast<const uint2*>(W1 + kTermHidden * kTermW1Stride);
    const __half2* w3 = reinterpret_cast<const __half2*>(W1 + kTermHidden * kTermW1Stride + kTermHidden * kTermHidden);
    float x[kTermFeatures];
#pragma unroll
    for (int i = 0; i < kTermFeatures; i++) x[i] = (f[i] - __ldg(mu + i)) * __ldg(inv_sigma + i);
    // layer 1: rows 2j and 2j + 1 of W1 are 32 contiguous bytes
    const float2 bb1 = __ldg(reinterpret_cast<const float2*>(b1) + lane);
    float h1[2] = {bb1.x, bb1.y};
#pragma unroll
    for (int s = 0; s < 2; s++) {
        const uint4 raw = __ldg(reinterpret_cast<const uint4*>(W1) + 2 * lane + s);
        const __half2* w = reinterpret_cast<const __half2*>(&raw);
        float acc = h1[s];
#pragma unroll
        for (int i = 0; i < kTermFeatures / 2; i++) {
            const float2 wf = __half22float2(w[i]);
            acc = fmaf(wf.y, x[2 * i + 1], fmaf(wf.x, x[2 * i], acc));
        }
        h1[s] = fmaxf(acc, 0.f);
    }
    // layer 2: unit pair (2p, 2p + 1) of layer 1 lives in lane p
    const float2 bb2 = __ldg(reinterpret_cast<const float2*>(b2) + lane);
    float acc0 = bb2.x, acc1 = bb2.y;
#pragma unroll 8
    for (int pr = 0; pr < kTermHidden / 2; pr++) {
        const float ha = __shfl_sync(kFull, h1[0], pr), hb = __shfl_sync(kFull, h1[1], pr);
        const uint2 raw = __ldg(W2 + pr * (kTermHidden / 2) + lane);
        const float2 w0 = __half22float2(*reinterpret_cast<const __half2*>(&raw.x));
        const float2 w1 = __half22float2(*reinterpret_cast<const __half2*>(&raw.y));
        acc0 = fmaf(w0.y, hb, fmaf(w0.x, ha, acc0));
        acc1 = fmaf(w1.y, hb, fmaf(w1.x, ha, acc1));
    }
    const float2 o = __half22float2(w3[lane]);
    float sum = fmaf(o.y, fmaxf(acc1, 0.f), o.x * fmaxf(acc0, 0.f));
#pragma unroll
    for (int s = 16; s; s >>= 1) sum += __shfl_xor_sync(kFull, sum, s);
    return sum + b3;
}

}  // namespace hnswgpu
