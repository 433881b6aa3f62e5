// Training of the early-termination network on the GPU (sm_100a): forward,
// backward and Adam kernels, plus the stand-alone inference kernel that runs
// the search's own in-warp network on given feature vectors.
//
// Network: x = (f - mu) * inv_sigma; h1 = relu(W1 x + b1); h2 = relu(W2 h1 + b2);
// logit = w3 . h2 + b3.  Loss: class-weighted binary cross-entropy,
//   pos_weight * y * softplus(-logit) + (1 - y) * softplus(logit),
// averaged over the batch.  Parameters are float32 (kTermParams, layout in
// hnsw_search.h); mu / inv_sigma are fixed by the caller and get no gradient.
//
// term_grad_kernel: one CTA of 128 threads per 128 samples, one thread per
// sample for the forward and the activation gradients (activations kept in
// shared memory, rows padded to 65 floats so the per-sample rows fall in
// distinct banks); then the CTA reduces the weight gradients over its
// samples (dW2 as a 64 x 128 x 64 product, 32 outputs per thread) and writes
// one partial-gradient row.  term_adam_kernel sums the rows in a fixed order
// (deterministic) and applies Adam.  The sizes are tiny (4.7k parameters),
// so CUDA cores, not tensor cores, do this work.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "hnsw_search.h"
#include "term_mlp.cuh"

namespace hnswgpu {

void pack_term_model(const float* params, unsigned char* out) {
    float* f = reinterpret_cast<float*>(out);
    for (int i = 0; i < kTermPackedFloats; i++) f[i] = 0.f;
    for (int i = 0; i < kTermFeatures; i++) {
        f[i] = params[kTermOffMu + i];
        f[kTermFeatures + i] = params[kTermOffInvSigma + i];
    }
    f[2 * kTermFeatures] = params[kTermOffB3];
    float* b1f = f + kTermPackedHead;
    float* b2f = b1f + 4 * 8 * 2;
    for (int t = 0; t < 4; t++)
        for (int v = 0; v < 8; v++)
            for (int e = 0; e < 2; e++) {
                b1f[(t * 8 + v) * 2 + e] = params[kTermOffB1 + 8 * v + 2 * t + e];
                b2f[(t * 8 + v) * 2 + e] = params[kTermOffB2 + 8 * v + 2 * t + e];
            }
    __half* h = reinterpret_cast<__half*>(out + (size_t)kTermPackedFloats * 4);
    // w3f[t][v]
    for (int t = 0; t < 4; t++)
        for (int v = 0; v < 8; v++)
            for (int e = 0; e < 2; e++) h[(t * 8 + v) * 2 + e] = __float2half_rn(params[kTermOffW3 + 8 * v + 2 * t + e]);
    h += 4 * 8 * 2;
    // W1f[lane][v][hh]
    for (int lane = 0; lane < 32; lane++) {
        const int g = lane >> 2, t = lane & 3;
        for (int v = 0; v < 8; v++)
            for (int hh = 0; hh < 2; hh++)
                for (int e = 0; e < 2; e++) {
                    const int feat = 2 * t + 8 * hh + e;
                    h[((lane * 8 + v) * 2 + hh) * 2 + e] =
                        __float2half_rn(params[kTermOffW1 + (8 * v + g) * kTermFeatures + feat]);
                }
    }
    h += 32 * 8 * 2 * 2;
    // W2f[lane][s][v][hh]
    for (int lane = 0; lane < 32; lane++) {
        const int g = lane >> 2, t = lane & 3;
        for (int st = 0; st < 4; st++)
            for (int v = 0; v < 8; v++)
                for (int hh = 0; hh < 2; hh++)
                    for (int e = 0; e < 2; e++) {
                        const int j = 16 * st + 2 * t + 8 * hh + e;
                        h[(((lane * 4 + st) * 8 + v) * 2 + hh) * 2 + e] =
                            __float2half_rn(params[kTermOffW2 + (8 * v + g) * kTermHidden + j]);
                    }
    }
}

namespace {

constexpr int kTile = 128;           // samples per CTA
constexpr int kRow = kTermHidden + 1;  // padded activation row

struct TrainSmem {
    float W1[kTermHidden * kTermFeatures];
    float b1[kTermHidden];
    float W2[kTermHidden * kTermHidden];
    float b2[kTermHidden];
    float w3[kTermHidden];
    float x[kTile * kTermFeatures];
    float dl[kTile];
    float h1[kTile * kRow];
    float h2[kTile * kRow];
    float dz1[kTile * kRow];
    float dz2[kTile * kRow];
    float loss[kTile / 32];
};

// Partial gradient of samples [start + 128 * blockIdx.x, ...) of the order
// `perm` (identity when null), scaled by `scale` (1 / batch size).
__global__ void __launch_bounds__(kTile) term_grad_kernel(const float* __restrict__ params,
                                                          const float* __restrict__ feats,
                                                          const float* __restrict__ labels,
                                                          const uint32_t* __restrict__ perm, uint64_t start,
                                                          uint64_t end, float pos_weight, float scale,
                                                          float* __restrict__ part, float* __restrict__ part_loss) {
    extern __shared__ __align__(16) unsigned char raw[];
    TrainSmem& s = *reinterpret_cast<TrainSmem*>(raw);
    const int t = threadIdx.x;
    for (int i = t; i < kTermHidden * kTermFeatures; i += kTile) s.W1[i] = params[kTermOffW1 + i];
    for (int i = t; i < kTermHidden * kTermHidden; i += kTile) s.W2[i] = params[kTermOffW2 + i];
    if (t < kTermHidden) {
        s.b1[t] = params[kTermOffB1 + t];
        s.b2[t] = params[kTermOffB2 + t];
        s.w3[t] = params[kTermOffW3 + t];
    }
    const float b3 = params[kTermOffB3];
    const uint64_t pos = start + (uint64_t)blockIdx.x * kTile + t;
    const bool valid = pos < end;
    const uint64_t sample = valid ? (perm ? perm[pos] : pos) : 0;
    float* x = s.x + t * kTermFeatures;
#pragma unroll
    for (int i = 0; i < kTermFeatures; i++)
        x[i] = valid ? (feats[sample * kTermFeatures + i] - params[kTermOffMu + i]) * params[kTermOffInvSigma + i]
                     : 0.f;
    __syncthreads();
    // ---- forward
    float* h1 = s.h1 + t * kRow;
    float* h2 = s.h2 + t * kRow;
    for (int u = 0; u < kTermHidden; u++) {
        float a = s.b1[u];
#pragma unroll
        for (int i = 0; i < kTermFeatures; i++) a = fmaf(s.W1[u * kTermFeatures + i], x[i], a);
        h1[u] = fmaxf(a, 0.f);
    }
    float logit = b3;
    for (int u = 0; u < kTermHidden; u++) {
        float a = s.b2[u];
        for (int j = 0; j < kTermHidden; j++) a = fmaf(s.W2[u * kTermHidden + j], h1[j], a);
        h2[u] = fmaxf(a, 0.f);
        logit = fmaf(s.w3[u], h2[u], logit);
    }
    // ---- loss and d loss / d logit
    const float y = valid ? labels[sample] : 0.f;
    const float sp_pos = fmaxf(logit, 0.f) + log1pf(expf(-fabsf(logit)));  // softplus(logit)
    const float sp_neg = sp_pos - logit;                                   // softplus(-logit)
    const float prob = 1.f / (1.f + expf(-logit));
    float loss = valid ? pos_weight * y * sp_neg + (1.f - y) * sp_pos : 0.f;
    const float g = valid ? (pos_weight * y * (prob - 1.f) + (1.f - y) * prob) * scale : 0.f;
    s.dl[t] = g;
    // ---- backward through the hidden layers
    float* dz2 = s.dz2 + t * kRow;
    float* dz1 = s.dz1 + t * kRow;
    for (int u = 0; u < kTermHidden; u++) dz2[u] = h2[u] > 0.f ? g * s.w3[u] : 0.f;
    for (int j = 0; j < kTermHidden; j++) {
        float a = 0.f;
        for (int u = 0; u < kTermHidden; u++) a = fmaf(s.W2[u * kTermHidden + j], dz2[u], a);
        dz1[j] = h1[j] > 0.f ? a : 0.f;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if ((t & 31) == 0) s.loss[t >> 5] = loss;
    __syncthreads();
    // ---- weight gradients, summed over this CTA's samples
    float* out = part + (size_t)blockIdx.x * kTermParams;
    {
        const int u = t >> 1, j0 = (t & 1) * 32;
        float acc[32];
#pragma unroll
        for (int j = 0; j < 32; j++) acc[j] = 0.f;
        for (int r = 0; r < kTile; r++) {
            const float a = s.dz2[r * kRow + u];
            const float* hr = s.h1 + r * kRow + j0;
#pragma unroll
            for (int j = 0; j < 32; j++) acc[j] = fmaf(a, hr[j], acc[j]);
        }
#pragma unroll
        for (int j = 0; j < 32; j++) out[kTermOffW2 + u * kTermHidden + j0 + j] = acc[j];
    }
    for (int e = t; e < kTermHidden * kTermFeatures; e += kTile) {
        const int u = e / kTermFeatures, i = e % kTermFeatures;
        float a = 0.f;
        for (int r = 0; r < kTile; r++) a = fmaf(s.dz1[r * kRow + u], s.x[r * kTermFeatures + i], a);
        out[kTermOffW1 + e] = a;
    }
    if (t < kTermHidden) {
        float a1 = 0.f, a2 = 0.f, a3 = 0.f;
        for (int r = 0; r < kTile; r++) {
            a1 += s.dz1[r * kRow + t];
            a2 += s.dz2[r * kRow + t];
            a3 = fmaf(s.dl[r], s.h2[r * kRow + t], a3);
        }
        out[kTermOffB1 + t] = a1;
        out[kTermOffB2 + t] = a2;
        out[kTermOffW3 + t] = a3;
    } else if (t == kTermHidden) {
        float a = 0.f;
        for (int r = 0; r < kTile; r++) a += s.dl[r];
        out[kTermOffB3] = a;
        float l = 0.f;
        for (int w = 0; w < kTile / 32; w++) l += s.loss[w];
        part_loss[blockIdx.x] = l * scale;
    } else if (t >= kTermHidden + 1 && t < kTermHidden + 1 + 2 * kTermFeatures) {
        out[kTermOffMu + (t - kTermHidden - 1)] = 0.f;  // mu, inv_sigma: fixed
    }
}

// Sum of the partial rows, in block order (no atomics: deterministic).
__global__ void term_reduce_kernel(const float* __restrict__ part, const float* __restrict__ part_loss, int nparts,
                                   float* __restrict__ grad, float* __restrict__ loss) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kTermParams) {
        float a = 0.f;
        for (int b = 0; b < nparts; b++) a += part[(size_t)b * kTermParams + i];
        grad[i] = a;
    }
    if (i == 0) {
        float l = 0.f;
        for (int b = 0; b < nparts; b++) l += part_loss[b];
        *loss = l;
    }
}

// Adam over the trainable parameters (W1 onwards), decoupled weight decay
// on the weight matrices; also accumulates the batch loss into `epoch_loss`.
__global__ void term_adam_kernel(float* __restrict__ params, float* __restrict__ m, float* __restrict__ v,
                                 const float* __restrict__ part, const float* __restrict__ part_loss, int nparts,
                                 float lr, float beta1, float beta2, float eps, float wd, float bc1, float bc2,
                                 float* __restrict__ epoch_loss) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        float l = 0.f;
        for (int b = 0; b < nparts; b++) l += part_loss[b];
        *epoch_loss += l;
    }
    if (i < kTermOffW1 || i >= kTermParams) return;
    float g = 0.f;
    for (int b = 0; b < nparts; b++) g += part[(size_t)b * kTermParams + i];
    const float mi = beta1 * m[i] + (1.f - beta1) * g;
    const float vi = beta2 * v[i] + (1.f - beta2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const bool is_weight = (i >= kTermOffW1 && i < kTermOffB1) || (i >= kTermOffW2 && i < kTermOffB2) ||
                           (i >= kTermOffW3 && i < kTermOffB3);
    float p = params[i];
    if (is_weight) p -= lr * wd * p;
    p -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    params[i] = p;
}

// One warp per feature vector: the search's own inference function.
__global__ void term_logits_kernel(const float* __restrict__ model, const float* __restrict__ feats, uint64_t n,
                                   float* __restrict__ out) {
    const uint64_t row = (uint64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    float f[kTermFeatures];
#pragma unroll
    for (int i = 0; i < kTermFeatures; i++) f[i] = feats[row * kTermFeatures + i];
    const float l = term_logit(model, f, lane);
    if (lane == 0) out[row] = l;
}

template <typename T>
struct DevArray {
    T* p = nullptr;
    cudaError_t alloc(size_t n) { return cudaMalloc((void**)&p, std::max<size_t>(n, 1) * sizeof(T)); }
    ~DevArray() {
        if (p) cudaFree(p);
    }
};

#define TERM_CHECK(x)                          \
    do {                                       \
        cudaError_t e_ = (x);                  \
        if (e_ != cudaSuccess) return e_;      \
    } while (0)

cudaError_t grad_launch(const float* dparams, const float* dfeats, const float* dlabels, const uint32_t* dperm,
                        uint64_t start, uint64_t end, float pos_weight, float scale, float* dpart, float* dpart_loss,
                        cudaStream_t st) {
    const unsigned blocks = (unsigned)((end - start + kTile - 1) / kTile);
    const int smem = (int)sizeof(TrainSmem);
    TERM_CHECK(cudaFuncSetAttribute(term_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    term_grad_kernel<<<blocks, kTile, smem, st>>>(dparams, dfeats, dlabels, dperm, start, end, pos_weight, scale,
                                                   dpart, dpart_loss);
    return cudaGetLastError();
}

}  // namespace

cudaError_t term_loss_grad(const float* params, const float* feats, const float* labels, uint64_t n,
                           float pos_weight, float* out_loss, float* out_grad) {
    DevArray<float> dp, df, dy, dpart, dpl, dg, dl;
    const uint64_t blocks = (n + kTile - 1) / kTile;
    TERM_CHECK(dp.alloc(kTermParams));
    TERM_CHECK(df.alloc(n * kTermFeatures));
    TERM_CHECK(dy.alloc(n));
    TERM_CHECK(dpart.alloc(blocks * kTermParams));
    TERM_CHECK(dpl.alloc(blocks));
    TERM_CHECK(dg.alloc(kTermParams));
    TERM_CHECK(dl.alloc(1));
    TERM_CHECK(cudaMemcpy(dp.p, params, kTermParams * 4, cudaMemcpyHostToDevice));
    TERM_CHECK(cudaMemcpy(df.p, feats, n * kTermFeatures * 4, cudaMemcpyHostToDevice));
    TERM_CHECK(cudaMemcpy(dy.p, labels, n * 4, cudaMemcpyHostToDevice));
    TERM_CHECK(grad_launch(dp.p, df.p, dy.p, nullptr, 0, n, pos_weight, 1.0f / (float)n, dpart.p, dpl.p, 0));
    term_reduce_kernel<<<(kTermParams + 255) / 256, 256>>>(dpart.p, dpl.p, (int)blocks, dg.p, dl.p);
    TERM_CHECK(cudaGetLastError());
    TERM_CHECK(cudaMemcpy(out_grad, dg.p, kTermParams * 4, cudaMemcpyDeviceToHost));
    TERM_CHECK(cudaMemcpy(out_loss, dl.p, 4, cudaMemcpyDeviceToHost));
    return cudaSuccess;
}

cudaError_t term_train(const float* feats, const float* labels, uint64_t n, float* params, uint32_t epochs,
                       uint32_t batch, float lr, float pos_weight, float weight_decay, uint64_t seed,
                       float* out_epoch_loss) {
    if (batch == 0) batch = 1024;
    DevArray<float> dp, df, dy, dm, dv, dpart, dpl, del;
    DevArray<uint32_t> dperm;
    const uint64_t max_blocks = (batch + kTile - 1) / kTile;
    TERM_CHECK(dp.alloc(kTermParams));
    TERM_CHECK(df.alloc(n * kTermFeatures));
    TERM_CHECK(dy.alloc(n));
    TERM_CHECK(dm.alloc(kTermParams));
    TERM_CHECK(dv.alloc(kTermParams));
    TERM_CHECK(dpart.alloc(max_blocks * kTermParams));
    TERM_CHECK(dpl.alloc(max_blocks));
    TERM_CHECK(del.alloc(std::max<uint32_t>(epochs, 1)));
    TERM_CHECK(dperm.alloc(n));
    TERM_CHECK(cudaMemcpy(dp.p, params, kTermParams * 4, cudaMemcpyHostToDevice));
    TERM_CHECK(cudaMemcpy(df.p, feats, n * kTermFeatures * 4, cudaMemcpyHostToDevice));
    TERM_CHECK(cudaMemcpy(dy.p, labels, n * 4, cudaMemcpyHostToDevice));
    TERM_CHECK(cudaMemset(dm.p, 0, kTermParams * 4));
    TERM_CHECK(cudaMemset(dv.p, 0, kTermParams * 4));
    TERM_CHECK(cudaMemset(del.p, 0, std::max<uint32_t>(epochs, 1) * 4));
    std::vector<uint32_t> perm(n);
    std::iota(perm.begin(), perm.end(), 0u);
    std::mt19937_64 rng(seed);
    const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
    uint64_t step = 0;
    for (uint32_t ep = 0; ep < epochs; ep++) {
        std::shuffle(perm.begin(), perm.end(), rng);
        TERM_CHECK(cudaMemcpy(dperm.p, perm.data(), n * 4, cudaMemcpyHostToDevice));
        uint64_t nb = 0;
        for (uint64_t b0 = 0; b0 < n; b0 += batch, nb++) {
            const uint64_t b1 = std::min<uint64_t>(n, b0 + batch);
            const int parts = (int)((b1 - b0 + kTile - 1) / kTile);
            TERM_CHECK(grad_launch(dp.p, df.p, dy.p, dperm.p, b0, b1, pos_weight, 1.0f / (float)(b1 - b0), dpart.p,
                                   dpl.p, 0));
            step++;
            const float bc1 = 1.f - (float)std::pow(0.9, (double)step);
            const float bc2 = 1.f - (float)std::pow(0.999, (double)step);
            term_adam_kernel<<<(kTermParams + 255) / 256, 256>>>(dp.p, dm.p, dv.p, dpart.p, dpl.p, parts, lr, beta1,
                                                                 beta2, eps, weight_decay, bc1, bc2, del.p + ep);
            TERM_CHECK(cudaGetLastError());
        }
        if (out_epoch_loss) {
            float l = 0.f;
            TERM_CHECK(cudaMemcpy(&l, del.p + ep, 4, cudaMemcpyDeviceToHost));
            out_epoch_loss[ep] = nb ? l / (float)nb : 0.f;
        }
    }
    TERM_CHECK(cudaMemcpy(params, dp.p, kTermParams * 4, cudaMemcpyDeviceToHost));
    return cudaSuccess;
}

cudaError_t term_logits(const float* params, const float* feats, uint64_t n, float* out) {
    std::vector<unsigned char> packed(kTermPackedBytes);
    pack_term_model(params, packed.data());
    DevArray<unsigned char> dmodel;
    DevArray<float> df, dout;
    TERM_CHECK(dmodel.alloc(kTermPackedBytes));
    TERM_CHECK(df.alloc(n * kTermFeatures));
    TERM_CHECK(dout.alloc(n));
    TERM_CHECK(cudaMemcpy(dmodel.p, packed.data(), kTermPackedBytes, cudaMemcpyHostToDevice));
    TERM_CHECK(cudaMemcpy(df.p, feats, n * kTermFeatures * 4, cudaMemcpyHostToDevice));
    if (n) {
        term_logits_kernel<<<(unsigned)((n + 7) / 8), 256>>>(reinterpret_cast<const float*>(dmodel.p), df.p, n, dout.p);
        TERM_CHECK(cudaGetLastError());
    }
    TERM_CHECK(cudaMemcpy(out, dout.p, n * 4, cudaMemcpyDeviceToHost));
    return cudaSuccess;
}

}  // namespace hnswgpu
