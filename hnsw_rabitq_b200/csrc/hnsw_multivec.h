// Launch parameters of the multi-vector search kernel (hnsw_multivec.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "hnsw_search.h"

namespace hnswgpu {

struct MvParams {
    const float* vecs;            // count x row_floats
    const uint32_t* links0;       // count x maxM0, unused slots 0xffffffff
    const uint32_t* upper_off;
    const uint32_t* upper_links;
    const uint32_t* docs;         // document id per element
    uint32_t count, dim, row_floats, maxM, maxM0, ep;
    int32_t maxlevel;
    const float* queries;         // nq x dim
    uint32_t nq;
    uint32_t num_docs, ef_coll;   // MultiVectorSearchStopCondition(space, num_docs, ef_collection)
    uint32_t cap;                 // result slots per query
    uint32_t top_cap;             // top_candidates / condition heap entries (candidate_set: 2x)
    uint32_t doc_log2, vis_log2;  // document table / visited set sizes (powers of two)
    uint32_t max_expansions;
    uint64_t* out_ids;            // nq x cap internal ids
    float* out_dists;
    int32_t* out_counts;          // result size, or -1 (more than cap, or an overflow)
    uint32_t* status;
};

size_t multivec_smem(const MvParams& p);
cudaError_t launch_hnsw_multivec(const MvParams& p, int num_sms, cudaStream_t stream);

}  // namespace hnswgpu
