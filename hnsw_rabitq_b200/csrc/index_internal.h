// Internal host-side declarations shared by the C-ABI translation units
// (index_api.cu: loading and search entry points; server.cu: the serving
// loop).  Not part of the public interface.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "hnswgpu.h"
#include "hnsw_search.h"

namespace hnswgpu_host {

extern thread_local std::string g_last_error;

struct ApiError : std::runtime_error {
    int code;
    ApiError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        throw ApiError(e == cudaErrorMemoryAllocation ? HNSWGPU_ERR_NOMEM : HNSWGPU_ERR_CUDA,
                       std::string(what) + ": " + cudaGetErrorString(e));
    }
}

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        release();
        if (count == 0) return;
        cuda_check(cudaMalloc((void**)&p, count * sizeof(T)), "cudaMalloc");
        n = count;
    }
    void ensure(size_t count) {
        if (count > n) alloc(count);
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    size_t bytes() const { return n * sizeof(T); }
    ~DevBuf() { release(); }
};

}  // namespace hnswgpu_host

struct hnswgpu_index {
    template <class T>
    using DevBuf = hnswgpu_host::DevBuf<T>;
    int is_bf = 0;
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    int space = 0;
    uint64_t dim = 0;
    uint32_t row_floats = 0;
    uint64_t count = 0, max_elements = 0;
    uint64_t M = 0, maxM = 0, maxM0 = 0, efc = 0, ef = 10;
    int32_t maxlevel = 0;
    uint32_t ep = 0;
    std::vector<uint64_t> labels;
    std::unordered_map<uint64_t, uint32_t> lookup;
    std::vector<uint32_t> deleted;  // host copy of the bitmap
    bool links_unique = true;       // no level-0 list repeats an id
    uint64_t num_deleted = 0;
    DevBuf<float> vecs;
    DevBuf<uint32_t> links0, upper_off, upper_links, deleted_bits;
    DevBuf<uint64_t> dlabels;
    DevBuf<uint32_t> docs;  // multi-vector index: document id per element (else empty)
    // per-call workspace
    DevBuf<uint32_t> counters;  // ring of work counters
    uint32_t next_counter = 0;
    DevBuf<uint32_t> status;
    DevBuf<unsigned char> io;  // host-pointer calls: queries + outputs
    DevBuf<uint8_t> allow;
    DevBuf<float> bf_norms;    // brute force: per-row helper values
    DevBuf<unsigned char> tcopy[3];  // low-precision traversal copies (index 1 bf16, 2 fp8)
    DevBuf<unsigned char> term_model;  // learned termination: packed network
    DevBuf<uint64_t> cand_spill;       // tie-exact mode: candidate-heap tails
    DevBuf<uint32_t> tie_list;         // tie-exact mode: [0] count, then the queries to replay
    // share of listed queries per ef, read back without blocking: the word
    // tie_list[0] is copied to pinned memory after a listing pass
    uint32_t* tie_host = nullptr;
    cudaEvent_t tie_ev = nullptr;
    uint64_t tie_pending_ef = 0, tie_pending_nq = 0;
    struct TieShare {
        float share = 0.f;
        uint32_t calls = 0;  // one-pass calls since the share was measured
    };
    std::unordered_map<uint64_t, TieShare> tie_share;
    DevBuf<float2> tc_rowinfo[3];      // tensor-core brute force: (|x|^2, scale) per row and precision
    // tensor-core brute force: per-call workspace
    DevBuf<float> tc_qf, tc_qscale, tc_tau;
    DevBuf<float2> tc_sinfo;           // helpers of the sampled rows
    DevBuf<unsigned char> tc_qt;
    DevBuf<uint32_t> tc_cnt, tc_idx;
    DevBuf<uint64_t> tc_buf;
    DevBuf<uint8_t> tc_flags;
    DevBuf<uint8_t> scan_mask;         // exact scan over an index with deletions
    uint32_t term_period = 0;
    float term_logit = 0.f;
    // registered filters (hnswgpu_filter_create): id - 1 -> device mask
    std::vector<std::unique_ptr<DevBuf<uint8_t>>> filters;
    std::string source_path;  // HNSW index file this index was loaded from (saveIndex)
    // guards the index state; mutable so that the const allocation-free
    // search can hold it while it reads that state
    mutable std::mutex mu;
    ~hnswgpu_index() {
        if (tie_host) cudaFreeHost(tie_host);
        if (tie_ev) cudaEventDestroy(tie_ev);
    }
    uint64_t device_bytes() const {
        return vecs.bytes() + links0.bytes() + upper_off.bytes() + upper_links.bytes() + deleted_bits.bytes() +
               dlabels.bytes() + bf_norms.bytes() + tcopy[1].bytes() + tcopy[2].bytes();
    }
};


namespace hnswgpu_host {

// Kernel distance family of an index: 0 = squared L2 (float32 rows, or the
// uint8 rows of L2SpaceI widened exactly to float32), 1 = inner product.
inline int kspace(const hnswgpu_index* h) {
    return h->space == HNSWGPU_SPACE_IP || h->space == HNSWGPU_SPACE_COSINE ? 1 : 0;
}

// Learned-termination settings of one launch (mode 1: record checkpoints,
// 2: stop early with the index's network).
struct TermCfg {
    uint32_t mode = 0, period = 0, max_ckpt = 0, width = 0;
    float* feat = nullptr;
    uint32_t* ids = nullptr;
    float* dists = nullptr;
    uint32_t* count = nullptr;
};

int fail(int code, const std::string& msg);

template <class F>
int guarded(F fn) {
    try {
        g_last_error.clear();
        return fn();
    } catch (const ApiError& e) {
        return fail(e.code, e.what());
    } catch (const std::bad_alloc&) {
        return fail(HNSWGPU_ERR_NOMEM, "Not enough memory");
    } catch (const std::exception& e) {
        return fail(HNSWGPU_ERR_ARG, e.what());
    }
}

void set_device(hnswgpu_index* h);
void ensure_traversal_copy(hnswgpu_index* h, uint32_t prec);
// Launch parameters of one HNSW search on device buffers (no allocation).
hnswgpu::SearchParams hnsw_params(const hnswgpu_index* h, const float* dq, uint64_t nq, uint64_t k, uint64_t ef,
                                  const uint8_t* dallow, uint64_t* dl, float* dd, int32_t* dc, uint32_t* dtrace,
                                  bool exact, uint32_t prec = 0, uint32_t rerank = 0, bool spill = false);
// One search launch (HNSW beam, or brute force / exact scan) on device
// buffers on stream `st`; the caller holds h->mu.
void run_search(hnswgpu_index* h, const float* dq, uint64_t nq, uint64_t k, uint64_t ef, const uint8_t* dallow,
                uint64_t* dl, float* dd, int32_t* dc, uint32_t* dtrace, cudaStream_t st, bool exact,
                uint32_t prec = 0, uint32_t rerank = 0, const TermCfg* term = nullptr, bool scan = false,
                bool replay_all = false);

}  // namespace hnswgpu_host
