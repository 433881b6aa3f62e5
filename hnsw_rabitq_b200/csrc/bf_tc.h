// Tensor-core brute force (bf_tc.cu): launch parameters and host entry points.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace hnswgpu {

// Scores pass (MODE 0: filter-append) / threshold pass (MODE 1).
struct TcArgs {
    uint32_t nq;               // queries (rows of the query map)
    uint32_t n_rows;           // rows of the row map (the sample in MODE 1)
    uint64_t row_step;         // global row id = map row x row_step
    uint32_t k_blocks;         // 128-byte K blocks per row
    uint32_t chunk_tiles;      // MODE 0: 256-row tiles per work item
    const float2* rowinfo;     // per map row: (|x|^2, scale), padded to whole 256-row tiles
    const float* qscale;       // per query: scale of its low-precision row
    const uint8_t* allow;      // optional per-row mask
    float* tau;                // per query: threshold (MODE 0 reads, MODE 1 writes)
    uint32_t* cnt;             // MODE 0: candidates per query
    uint64_t* buf;             // MODE 0: nq x cap (distance key << 32 | row)
    uint32_t cap;
    uint32_t* status;
};

struct TcSelectArgs {
    uint32_t nq, k, R, cap, sort_cap, dim, row_floats, sampled;
    const uint32_t* cnt;
    const uint64_t* buf;
    const float* qf;           // float32 queries (normalised for cosine)
    const float* vecs;         // float32 rows
    const uint64_t* labels;
    uint64_t* out_labels;
    float* out_dists;
    int32_t* out_counts;
    uint8_t* flags;            // 1: answer this query with the exact kernel
    uint32_t* trace;           // optional: 4 per query, [0] = candidates found
};

size_t tc_smem_bytes();
cudaError_t launch_fp64_distances(const float* q, uint64_t nq, uint32_t m, uint32_t dim, const float* vecs,
                                  uint32_t row_floats, const uint32_t* rows, int space, int normalize, double* out,
                                  cudaStream_t st);
size_t tc_select_smem(uint32_t sort_cap, uint32_t dim, uint32_t R);
cudaError_t tc_encode_map(void* base, uint32_t prec, uint64_t rows, uint32_t dim, uint64_t row_pitch_bytes,
                          uint32_t box_rows, CUtensorMap* out);
cudaError_t launch_tc_scores(const CUtensorMap& qm, const CUtensorMap& xm, const TcArgs& a, uint32_t prec, int space,
                             int mode, int num_sms, cudaStream_t st);
cudaError_t launch_tc_rowinfo(const float* vecs, uint32_t count, uint32_t dim, uint32_t row_floats,
                              const unsigned char* tcopy, uint32_t trow_bytes, uint32_t prec, float2* out,
                              cudaStream_t st);
cudaError_t launch_tc_query_prep(const float* q, uint32_t nq, uint32_t dim, uint32_t normalize, uint32_t prec,
                                 uint32_t trow_bytes, float* qf, unsigned char* qt, float* qscale, cudaStream_t st);
cudaError_t launch_tc_fill(float* p, uint64_t n, float v, cudaStream_t st);
cudaError_t launch_scan_mask(const uint32_t* deleted_bits, const uint8_t* allow, uint64_t n, uint8_t* out,
                             cudaStream_t st);
cudaError_t launch_tc_gather_info(const float2* info, uint64_t n_sample, uint64_t step, float2* out,
                                  cudaStream_t st);
cudaError_t launch_tc_select(const TcSelectArgs& a, int space, cudaStream_t st);
cudaError_t launch_tc_gather(const float* src, const uint32_t* idx, uint32_t n, uint32_t dim, float* dst,
                             cudaStream_t st);
cudaError_t launch_tc_scatter(const uint32_t* idx, uint32_t n, uint32_t k, const uint64_t* l, const float* d,
                              const int32_t* c, uint64_t* ol, float* od, int32_t* oc, cudaStream_t st);

}  // namespace hnswgpu
