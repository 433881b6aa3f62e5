// Launch parameters of the brute-force search kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace hnswgpu {

struct BfParams {
    const float* vecs;       // count x row_floats, zero padded
    const uint64_t* labels;  // count
    const uint8_t* allow;    // optional mask over row ids
    uint32_t count, dim, row_floats;
    const float* queries;    // nq x dim
    uint32_t nq, k, normalize;
    uint64_t* out_labels;
    float* out_dists;
    int32_t* out_counts;
    uint32_t* status;        // bit 0x1 set when a bounded wait gives up
};

cudaError_t launch_bf_search(const BfParams& p, int space, int num_sms, cudaStream_t stream);

}  // namespace hnswgpu
