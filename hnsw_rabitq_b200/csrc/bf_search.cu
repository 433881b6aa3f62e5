// Exact brute-force k-NN on B200 (sm_100a), FP32 in the reference's order.
//
// Replaces BruteforceSearch::searchKnn (hnswlib/bruteforce.h:106-125).  Its
// result is, for every query, the k smallest (distance, label) pairs over the
// allowed rows: the reference's max-heap of std::pair<float, labeltype>
// accepts `dist <= lastdist || size < k` and pops the largest pair, so ties at
// the k-th distance are resolved by label.  This kernel computes the same set
// with the same FP32 distances (device_common.cuh), hence bit-identical
// outputs.
//
// Work decomposition: a CTA owns a tile of 4 * warps queries (4 per warp) and
// streams the whole database through shared memory in tiles of `tile_rows`
// rows, double buffered with TMA bulk copies (cp.async.bulk, no multicast).
// Each lane evaluates one database row against its warp's 4 queries, so a
// row loaded from shared memory is reused 4 times and the query reads are
// broadcasts.  Accepted (distance, row) pairs go to a small per-query buffer;
// when it fills, the warp merges it with the running top-k by a bitonic sort
// in shared memory, which also tightens the acceptance threshold.
#include <cuda_runtime.h>

#include <cstdint>

#include "bf_search.h"
#include "device_common.cuh"

namespace hnswgpu {

namespace {

constexpr int kQPW = 4;       // queries per warp
constexpr int kBuf = 64;      // per-query candidate buffer

struct BfLayout {
    uint32_t warps, tile_rows, qstride, xstride, sort_size, k;
    uint32_t off_bar, off_q, off_x, off_topdk, off_toplab, off_bufdk, off_bufrow, off_meta, off_sortk, off_sortl,
        total;
};

__device__ __forceinline__ void bitonic_sort_warp(uint32_t* sk, uint64_t* sl, int n, int lane) {
    for (int size = 2; size <= n; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = lane; i < n; i += 32) {
                int j = i ^ stride;
                if (j > i) {
                    bool up = (i & size) == 0;
                    uint32_t ki = sk[i], kj = sk[j];
                    uint64_t li = sl[i], lj = sl[j];
                    bool gt = ki > kj || (ki == kj && li > lj);
                    if (gt == up) {
                        sk[i] = kj;
                        sk[j] = ki;
                        sl[i] = lj;
                        sl[j] = li;
                    }
                }
            }
            __syncwarp();
        }
    }
}

template <int SPACE>
__device__ __forceinline__ void dist4_simd16(const float* __restrict__ x, const float* __restrict__ q, int qstride,
                                             int n16, float out[kQPW]) {
    float a[kQPW][16];
#pragma unroll
    for (int qq = 0; qq < kQPW; qq++)
#pragma unroll
        for (int l = 0; l < 16; l++) a[qq][l] = 0.f;
    const float4* x4 = reinterpret_cast<const float4*>(x);
    for (int c = 0; c < n16; c++) {
        float4 xv[4];
#pragma unroll
        for (int u = 0; u < 4; u++) xv[u] = x4[4 * c + u];
#pragma unroll
        for (int qq = 0; qq < kQPW; qq++) {
            const float4* q4 = reinterpret_cast<const float4*>(q + qq * qstride);
#pragma unroll
            for (int u = 0; u < 4; u++) {
                float4 qv = q4[4 * c + u];
                if (SPACE == 0) {
                    float t0 = __fsub_rn(qv.x, xv[u].x), t1 = __fsub_rn(qv.y, xv[u].y), t2 = __fsub_rn(qv.z, xv[u].z),
                          t3 = __fsub_rn(qv.w, xv[u].w);
                    a[qq][4 * u + 0] = __fmaf_rn(t0, t0, a[qq][4 * u + 0]);
                    a[qq][4 * u + 1] = __fmaf_rn(t1, t1, a[qq][4 * u + 1]);
                    a[qq][4 * u + 2] = __fmaf_rn(t2, t2, a[qq][4 * u + 2]);
                    a[qq][4 * u + 3] = __fmaf_rn(t3, t3, a[qq][4 * u + 3]);
                } else {
                    a[qq][4 * u + 0] = __fmaf_rn(qv.x, xv[u].x, a[qq][4 * u + 0]);
                    a[qq][4 * u + 1] = __fmaf_rn(qv.y, xv[u].y, a[qq][4 * u + 1]);
                    a[qq][4 * u + 2] = __fmaf_rn(qv.z, xv[u].z, a[qq][4 * u + 2]);
                    a[qq][4 * u + 3] = __fmaf_rn(qv.w, xv[u].w, a[qq][4 * u + 3]);
                }
            }
        }
    }
#pragma unroll
    for (int qq = 0; qq < kQPW; qq++) {
        if (SPACE == 0) {
            float r = a[qq][0];
#pragma unroll
            for (int l = 1; l < 16; l++) r = __fadd_rn(r, a[qq][l]);
            out[qq] = r;
        } else {
            float t3[8], t6[4];
#pragma unroll
            for (int i = 0; i < 8; i++) t3[i] = __fadd_rn(a[qq][i + 8], a[qq][i]);
#pragma unroll
            for (int i = 0; i < 4; i++) t6[i] = __fadd_rn(t3[i + 4], t3[i]);
            out[qq] = __fsub_rn(1.0f, __fadd_rn(__fadd_rn(t6[0], t6[2]), __fadd_rn(t6[1], t6[3])));
        }
    }
}

template <int SPACE>
__global__ void bf_exact_kernel(BfParams p, BfLayout L) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L.off_bar);
    float* qs = reinterpret_cast<float*>(smem + L.off_q);
    float* xs = reinterpret_cast<float*>(smem + L.off_x);
    const int dim = (int)p.dim, k = (int)p.k, TQ = (int)L.warps * kQPW;
    const uint32_t q0 = blockIdx.x * TQ;
    // ---- queries (zero rows past the batch), cosine normalisation
    for (int i = tid; i < TQ * (int)L.qstride; i += blockDim.x) {
        int r = i / (int)L.qstride, c = i % (int)L.qstride;
        uint32_t qi = q0 + r;
        qs[i] = (qi < p.nq && c < dim) ? p.queries[(size_t)qi * dim + c] : 0.f;
    }
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
    }
    fence_mbar_init();
    __syncthreads();
    if (p.normalize) {
        for (int r = warp; r < TQ; r += L.warps) {
            float sc = 0.f;
            if (lane == 0) sc = norm_scale(qs + r * L.qstride, dim);
            sc = __shfl_sync(FULL, sc, 0);
            for (int c = lane; c < dim; c += 32) qs[r * L.qstride + c] = __fmul_rn(qs[r * L.qstride + c], sc);
        }
    }
    // ---- per-query state, owned by the warp
    uint32_t* topdk = reinterpret_cast<uint32_t*>(smem + L.off_topdk);
    uint64_t* toplab = reinterpret_cast<uint64_t*>(smem + L.off_toplab);
    uint32_t* bufdk = reinterpret_cast<uint32_t*>(smem + L.off_bufdk);
    uint32_t* bufrow = reinterpret_cast<uint32_t*>(smem + L.off_bufrow);
    uint32_t* sk = reinterpret_cast<uint32_t*>(smem + L.off_sortk) + warp * L.sort_size;
    uint64_t* sl = reinterpret_cast<uint64_t*>(smem + L.off_sortl) + warp * L.sort_size;
    int cnt[kQPW], bcnt[kQPW];
    uint32_t thr[kQPW];
#pragma unroll
    for (int qq = 0; qq < kQPW; qq++) {
        cnt[qq] = 0;
        bcnt[qq] = 0;
        thr[qq] = 0xffffffffu;
    }
    const float* myq = qs + (size_t)warp * kQPW * L.qstride;

    auto merge = [&](int qq) {
        const int ql = warp * kQPW + qq;
        const int n = cnt[qq] + bcnt[qq];
        const uint32_t* td = topdk + (size_t)ql * k;
        const uint64_t* tl = toplab + (size_t)ql * k;
        const uint32_t* bd = bufdk + (size_t)ql * kBuf;
        const uint32_t* br = bufrow + (size_t)ql * kBuf;
        for (int i = lane; i < (int)L.sort_size; i += 32) {
            if (i < cnt[qq]) {
                sk[i] = td[i];
                sl[i] = tl[i];
            } else if (i < n) {
                sk[i] = bd[i - cnt[qq]];
                sl[i] = p.labels[br[i - cnt[qq]]];
            } else {
                sk[i] = 0xffffffffu;
                sl[i] = ~0ull;
            }
        }
        __syncwarp();
        bitonic_sort_warp(sk, sl, (int)L.sort_size, lane);
        int nc = min(k, n);
        uint32_t* tdw = topdk + (size_t)ql * k;
        uint64_t* tlw = toplab + (size_t)ql * k;
        for (int i = lane; i < nc; i += 32) {
            tdw[i] = sk[i];
            tlw[i] = sl[i];
        }
        __syncwarp();
        cnt[qq] = nc;
        bcnt[qq] = 0;
        thr[qq] = nc == k ? tdw[k - 1] : 0xffffffffu;
        __syncwarp();
    };

    // ---- stream the database
    const uint32_t row_bytes = p.row_floats * 4;
    const uint32_t ntiles = (p.count + L.tile_rows - 1) / L.tile_rows;
    auto issue = [&](uint32_t t) {
        // called by warp 0 only
        uint32_t r0 = t * L.tile_rows;
        uint32_t nr = min(L.tile_rows, p.count - r0);
        float* dst = xs + (size_t)(t & 1) * L.tile_rows * L.xstride;
        if (lane == 0) mbar_arrive_expect_tx(&bars[t & 1], nr * row_bytes);
        __syncwarp();
        for (uint32_t r = lane; r < nr; r += 32)
            bulk_g2s(dst + (size_t)r * L.xstride, p.vecs + (size_t)(r0 + r) * p.row_floats, row_bytes, &bars[t & 1]);
    };
    if (warp == 0) {
        fence_proxy_async_smem();
        if (ntiles > 0) issue(0);
        if (ntiles > 1) issue(1);
    }
    bool ok = true;
    for (uint32_t t = 0; t < ntiles; t++) {
        if (!mbar_wait(&bars[t & 1], (t >> 1) & 1u)) ok = false;
        if (!__syncthreads_and(ok)) {
            // a bounded wait gave up: flag it, wait (bounded) for copies still
            // in flight into this CTA's shared memory, and leave
            if (tid == 0) {
                atomicOr(p.status, 0x1u);
                mbar_wait(&bars[0], 0);
                mbar_wait(&bars[1], 0);
            }
            return;
        }
        const uint32_t r0 = t * L.tile_rows;
        const uint32_t nr = min(L.tile_rows, p.count - r0);
        const float* xt = xs + (size_t)(t & 1) * L.tile_rows * L.xstride;
        for (uint32_t rb = 0; rb < nr; rb += 32) {
            const uint32_t r = rb + lane;
            const bool valid = r < nr;
            const uint32_t row = r0 + r;
            float d[kQPW];
            const float* xr = xt + (size_t)(valid ? r : 0) * L.xstride;
            if ((dim & 15) == 0) {
                dist4_simd16<SPACE>(xr, myq, (int)L.qstride, dim >> 4, d);
            } else {
#pragma unroll
                for (int qq = 0; qq < kQPW; qq++) d[qq] = distance<SPACE>(myq + qq * L.qstride, xr, dim);
            }
            const bool allowed = valid && (!p.allow || p.allow[row]);
#pragma unroll
            for (int qq = 0; qq < kQPW; qq++) {
                uint32_t dk = fkey(d[qq]);
                bool acc = allowed && (cnt[qq] < k || dk <= thr[qq]);
                unsigned m = __ballot_sync(FULL, acc);
                if (m) {
                    const int ql = warp * kQPW + qq;
                    int pos = bcnt[qq] + __popc(m & lanemask_lt());
                    if (acc) {
                        bufdk[(size_t)ql * kBuf + pos] = dk;
                        bufrow[(size_t)ql * kBuf + pos] = row;
                    }
                    bcnt[qq] += __popc(m);
                    __syncwarp();
                    if (bcnt[qq] > kBuf - 32) merge(qq);
                }
            }
        }
        __syncthreads();
        if (warp == 0 && t + 2 < ntiles) {
            fence_proxy_async_smem();
            issue(t + 2);
        }
    }
    // ---- final merge and output
#pragma unroll
    for (int qq = 0; qq < kQPW; qq++) {
        if (bcnt[qq]) merge(qq);
        const uint32_t qi = q0 + warp * kQPW + qq;
        if (qi >= p.nq) continue;
        const int ql = warp * kQPW + qq;
        for (int i = lane; i < k; i += 32) {
            bool have = i < cnt[qq];
            p.out_labels[(size_t)qi * k + i] = have ? toplab[(size_t)ql * k + i] : ~0ull;
            p.out_dists[(size_t)qi * k + i] = have ? funkey(topdk[(size_t)ql * k + i]) : __int_as_float(0x7f800000);
        }
        if (lane == 0) p.out_counts[qi] = cnt[qq];
    }
}

bool make_layout(BfLayout& L, uint32_t warps, uint32_t tile_rows, const BfParams& p, size_t max_smem) {
    L.warps = warps;
    L.tile_rows = tile_rows;
    L.qstride = p.row_floats;
    L.xstride = p.row_floats + 4;
    L.k = p.k;
    uint32_t s = 1;
    while (s < p.k + kBuf) s <<= 1;
    L.sort_size = s;
    const uint32_t TQ = warps * kQPW;
    size_t off = 0;
    auto take = [&](size_t bytes, size_t align) {
        off = (off + align - 1) / align * align;
        size_t o = off;
        off += bytes;
        return (uint32_t)o;
    };
    L.off_bar = take(16, 16);
    L.off_q = take((size_t)TQ * L.qstride * 4, 16);
    L.off_x = take((size_t)2 * tile_rows * L.xstride * 4, 128);
    L.off_topdk = take((size_t)TQ * p.k * 4, 8);
    L.off_toplab = take((size_t)TQ * p.k * 8, 8);
    L.off_bufdk = take((size_t)TQ * kBuf * 4, 8);
    L.off_bufrow = take((size_t)TQ * kBuf * 4, 8);
    L.off_meta = take(16, 16);
    L.off_sortk = take((size_t)warps * s * 4, 8);
    L.off_sortl = take((size_t)warps * s * 8, 8);
    L.total = (uint32_t)((off + 127) / 128 * 128);
    return L.total <= max_smem;
}

}  // namespace

cudaError_t launch_bf_search(const BfParams& p, int space, int num_sms, cudaStream_t stream) {
    (void)num_sms;
    if (p.nq == 0) return cudaSuccess;
    int dev = 0, max_optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    BfLayout L{};
    bool found = false;
    const uint32_t warps_opts[] = {8, 4, 2, 1};
    const uint32_t tile_opts[] = {64, 32, 16, 8};
    for (uint32_t w : warps_opts) {
        for (uint32_t t : tile_opts)
            if (make_layout(L, w, t, p, (size_t)max_optin)) {
                found = true;
                break;
            }
        if (found) break;
    }
    if (!found) return cudaErrorInvalidConfiguration;
    const void* fn = space == 0 ? (const void*)bf_exact_kernel<0> : (const void*)bf_exact_kernel<1>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
    if (e != cudaSuccess) return e;
    const uint32_t TQ = L.warps * kQPW;
    const uint32_t blocks = (p.nq + TQ - 1) / TQ;
    if (space == 0)
        bf_exact_kernel<0><<<blocks, L.warps * 32, L.total, stream>>>(p, L);
    else
        bf_exact_kernel<1><<<blocks, L.warps * 32, L.total, stream>>>(p, L);
    return cudaGetLastError();
}

}  // namespace hnswgpu
