// Low-precision traversal copies of the index vectors (sm_100a).
//
// One warp per row reads the resident float32 row and writes
//   bf16: round-to-nearest bf16 per element (exact for integers up to 256,
//         i.e. for 8-bit image / SIFT-style data);
//   fp8 : e4m3 per element of x / s with s = max|x| / 448 (the largest finite
//         e4m3), saturating; the row's 16-byte tail holds s and the squared
//         norm of the dequantized row (s * e4m3 value per element), for the
//         |q|^2 - 2 q.x + |x|^2 form of the tensor-core distances.
// The search kernel accumulates distances from these copies in fp32 and then
// re-ranks its best candidates with the exact float32 rows.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "hnsw_search.h"

namespace hnswgpu {

uint32_t traversal_row_bytes(uint32_t prec, uint32_t dim) {
    if (prec == 1) return (dim * 2 + 15) / 16 * 16;
    if (prec == 2) return (dim + 15) / 16 * 16 + 16;
    return (dim * 4 + 15) / 16 * 16;
}

namespace {

__global__ void quantize_rows_kernel(const float* __restrict__ src, uint32_t count, uint32_t dim, uint32_t src_stride,
                                     uint32_t prec, uint32_t row_bytes, unsigned char* __restrict__ dst) {
    const uint64_t row = (uint64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (row >= count) return;
    const float* x = src + row * src_stride;
    unsigned char* out = dst + row * row_bytes;
    if (prec == 1) {
        __nv_bfloat16* o = reinterpret_cast<__nv_bfloat16*>(out);
        for (uint32_t i = lane; i < row_bytes / 2; i += 32) o[i] = __float2bfloat16_rn(i < dim ? x[i] : 0.f);
        return;
    }
    float amax = 0.f;
    for (uint32_t i = lane; i < dim; i += 32) amax = fmaxf(amax, fabsf(x[i]));
#pragma unroll
    for (int o = 16; o; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    const float scale = amax > 0.f ? amax / 448.0f : 1.0f;
    const float inv = 1.0f / scale;
    const uint32_t data_bytes = row_bytes - 16;
    float sq = 0.f;  // squared norm of the dequantized row (scale * e4m3 value)
    for (uint32_t i = 2 * lane; i < data_bytes; i += 64) {
        float2 v = make_float2(i < dim ? x[i] * inv : 0.f, i + 1 < dim ? x[i + 1] * inv : 0.f);
        __nv_fp8x2_storage_t q = __nv_cvt_float2_to_fp8x2(v, __NV_SATFINITE, __NV_E4M3);
        *reinterpret_cast<__nv_fp8x2_storage_t*>(out + i) = q;
        const float2 back = __half22float2(__half2(__nv_cvt_fp8x2_to_halfraw2(q, __NV_E4M3)));
        const float a = scale * back.x, b = scale * back.y;
        sq = fmaf(a, a, fmaf(b, b, sq));
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
    if (lane < 4) reinterpret_cast<float*>(out + data_bytes)[lane] = lane == 0 ? scale : (lane == 1 ? sq : 0.f);
}

}  // namespace

cudaError_t launch_quantize_rows(const float* src, uint32_t count, uint32_t dim, uint32_t src_stride, uint32_t prec,
                                 unsigned char* dst, cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    const uint32_t rows_per_block = 8;
    const unsigned blocks = (count + rows_per_block - 1) / rows_per_block;
    quantize_rows_kernel<<<blocks, rows_per_block * 32, 0, stream>>>(src, count, dim, src_stride, prec,
                                                                     traversal_row_bytes(prec, dim), dst);
    return cudaGetLastError();
}

}  // namespace hnswgpu
