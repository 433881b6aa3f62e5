// Host side of libhnswgpu: index-file loading, device layout, C-ABI entry
// points (declared in include/hnswgpu.h).
//
// Device layout of a HierarchicalNSW index (repacked from the reference's
// array-of-structs level-0 block, hnswlib/hnswalg.h:120-124, whose vector
// offset 4 + 4*maxM0 is not 16-byte aligned):
//   vecs        count x row_floats float32, row_floats = round_up(dim, 4),
//               zero padded -> every row is a 16-byte aligned TMA source;
//   links0      count x maxM0 uint32 neighbour ids, list order preserved,
//               unused slots 0xffffffff (the count is implied);
//   upper_off   per node: row index of its level-1 list in upper_links, or
//               0xffffffff when the node has no upper levels;
//   upper_links rows of (1 + maxM) uint32 = [count][ids] per (node, level),
//               copied verbatim from the reference's linkLists_ blocks;
//   labels      count x uint64 external labels;
//   deleted     bitmap over internal ids (byte 2 bit 0 of the level-0 header,
//               hnswalg.h:872-885).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "hnswgpu.h"
#include "bf_search.h"
#include "bf_tc.h"
#include "device_common.cuh"
#include "hnsw_search.h"
#include "hnsw_multivec.h"

// smallest visited cache of a beam, log2 entries (the cache grows with ef
// up to 2^12 entries)
#ifndef HNSWGPU_VIS_LOG2_MIN
#define HNSWGPU_VIS_LOG2_MIN 10
#endif

static_assert(HNSWGPU_TERM_PARAMS == hnswgpu::kTermParams, "termination parameter count");
static_assert(HNSWGPU_TERM_FEATURES == hnswgpu::kTermFeatures, "termination feature count");

#include "index_internal.h"

// staging slots of the float32 beam (dim % 16 == 0): rows gathered per TMA
// batch.  On 1M x 128 at ef 52, 12 or 10 slots with 18-20 resident CTAs per SM
// measured no faster than 16 slots with 16 CTAs (6.03-6.24 vs 6.26 M QPS).
#ifndef HNSWGPU_FP32_SLOTS
#define HNSWGPU_FP32_SLOTS 16
#endif

#ifdef HNSWGPU_TC_TIMING
namespace hnswgpu {
cudaError_t tc_timing_read(unsigned long long* out);
}
#endif

namespace hnswgpu_host {
thread_local std::string g_last_error;
}  // namespace hnswgpu_host
using namespace hnswgpu_host;

namespace {
template <class T>
void rd(std::istream& in, T& v) {
    in.read((char*)&v, sizeof(T));
}

// Read-only, seekable stream buffer over a caller's memory (an index image,
// e.g. the bytes of a pickled state): the file loader reads it in place.
class MemBuf : public std::streambuf {
public:
    MemBuf(const char* p, size_t n) {
        char* b = const_cast<char*>(p);
        setg(b, b, b + n);
    }

protected:
    pos_type seekoff(off_type off, std::ios_base::seekdir dir, std::ios_base::openmode) override {
        const std::ptrdiff_t size = egptr() - eback();
        const std::ptrdiff_t base = dir == std::ios_base::beg ? 0 : dir == std::ios_base::cur ? gptr() - eback() : size;
        if (off < -base || off > size - base) return pos_type(off_type(-1));
        setg(eback(), eback() + base + off, egptr());
        return pos_type(base + off);
    }
    pos_type seekpos(pos_type pos, std::ios_base::openmode m) override {
        return seekoff(off_type(pos), std::ios_base::beg, m);
    }
};
}  // namespace

namespace hnswgpu_host {

void set_device(hnswgpu_index* h) { cuda_check(cudaSetDevice(h->device), "cudaSetDevice"); }

void init_common(hnswgpu_index* h, int device) {
    h->device = device;
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    cuda_check(cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");
    cuda_check(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    h->counters.alloc(512);  // 256 (work, done) pairs, used round robin
    cuda_check(cudaMemset(h->counters.p, 0, h->counters.bytes()), "cudaMemset");
    h->status.alloc(1);
    cuda_check(cudaMemset(h->status.p, 0, 4), "cudaMemset");
}

// HierarchicalNSW::loadIndex (hnswlib/hnswalg.h:715-821) plus the structural
// checks a GPU kernel needs before it may follow the links (ids in range,
// upper-level lists present where the descent reads them).
void load_hnsw_stream(hnswgpu_index* h, std::istream& in, int space, uint64_t dim, uint64_t max_elements_i,
                      bool multivector) {
    in.seekg(0, in.end);
    const std::streamoff total = in.tellg();
    in.seekg(0, in.beg);
    uint64_t offsetLevel0, max_elements, cur, size_data, label_offset, offsetData, maxM, maxM0, M, efc;
    int32_t maxlevel;
    uint32_t ep;
    double mult;
    rd(in, offsetLevel0);
    rd(in, max_elements);
    rd(in, cur);
    rd(in, size_data);
    rd(in, label_offset);
    rd(in, offsetData);
    rd(in, maxlevel);
    rd(in, ep);
    rd(in, maxM);
    rd(in, maxM0);
    rd(in, M);
    rd(in, mult);
    rd(in, efc);
    const char* corrupt = "Index seems to be corrupted or unsupported";
    if (!in) throw ApiError(HNSWGPU_ERR_FORMAT, corrupt);
    const std::streamoff header_end = in.tellg();
    // file-length walk (hnswalg.h:753-769)
    if (size_data != 0 && cur > (uint64_t)(total - header_end) / size_data) throw ApiError(HNSWGPU_ERR_FORMAT, corrupt);
    std::streamoff pos = header_end + (std::streamoff)(cur * size_data);
    in.seekg(pos, in.beg);
    std::vector<uint32_t> ll_sizes(cur);
    for (uint64_t i = 0; i < cur; i++) {
        if (pos < 0 || pos >= total) throw ApiError(HNSWGPU_ERR_FORMAT, corrupt);
        uint32_t sz;
        rd(in, sz);
        pos += 4;
        ll_sizes[i] = sz;
        if (sz) {
            pos += sz;
            in.seekg(sz, in.cur);
        }
    }
    if (pos != total) throw ApiError(HNSWGPU_ERR_FORMAT, corrupt);
    in.clear();
    // layout consistency the kernels rely on
    const uint64_t size_links0 = maxM0 * 4 + 4, size_links = maxM * 4 + 4;
    // bytes per stored element: float32, or uint8 for L2SpaceI
    const uint64_t elem = space == HNSWGPU_SPACE_L2_UINT8 ? 1 : 4;
    if (space == HNSWGPU_SPACE_L2_UINT8 && dim * 65025ull >= (1ull << 24))
        throw ApiError(HNSWGPU_ERR_UNSUPPORTED,
                       "uint8 L2 needs dim <= 258 (integer distances exact in float32)");
    // a multi-vector index (MultiVectorL2Space, hnswlib/stop_condition.h:7-76)
    // stores a 32-bit document id right after each vector
    const uint64_t doc_bytes = multivector ? 4 : 0;
    if (offsetLevel0 != 0 || offsetData != size_links0 || label_offset != offsetData + dim * elem + doc_bytes ||
        size_data != label_offset + 8)
        throw ApiError(HNSWGPU_ERR_FORMAT,
                       "index layout does not match dim=" + std::to_string(dim) + " (" + corrupt + ")");
    if (maxM0 == 0 || maxM0 > 4096 || maxM > 4096) throw ApiError(HNSWGPU_ERR_UNSUPPORTED, "unsupported M");
    if (cur > 0x7fffffffull) throw ApiError(HNSWGPU_ERR_UNSUPPORTED, "more than 2^31-1 elements");
    if (cur > 0 && (ep >= cur || maxlevel < 0)) throw ApiError(HNSWGPU_ERR_FORMAT, corrupt);

    h->space = space;
    h->dim = dim;
    h->count = cur;
    h->max_elements = max_elements_i < cur ? max_elements : max_elements_i;
    h->M = M;
    h->maxM = maxM;
    h->maxM0 = maxM0;
    h->efc = efc;
    h->ef = 10;
    h->maxlevel = maxlevel;
    h->ep = ep;
    h->row_floats = (uint32_t)((dim + 3) / 4 * 4);

    // level-0 block -> vectors, links, labels, delete marks
    in.seekg(header_end, in.beg);
    const size_t chunk_rows = std::max<size_t>(1, (64u << 20) / std::max<uint64_t>(size_data, 1));
    std::vector<char> buf(chunk_rows * size_data);
    std::vector<float> hv(cur * h->row_floats, 0.f);
    std::vector<uint32_t> hl(cur * maxM0, 0xffffffffu);
    h->labels.resize(cur);
    std::vector<uint32_t> hdocs(multivector ? cur : 0);
    h->deleted.assign((cur + 31) / 32 + 1, 0u);
    h->num_deleted = 0;
    for (uint64_t r0 = 0; r0 < cur; r0 += chunk_rows) {
        size_t nr = (size_t)std::min<uint64_t>(chunk_rows, cur - r0);
        in.read(buf.data(), nr * size_data);
        if (!in) throw ApiError(HNSWGPU_ERR_FORMAT, corrupt);
        for (size_t r = 0; r < nr; r++) {
            const char* rec = buf.data() + r * size_data;
            uint64_t i = r0 + r;
            uint16_t cnt;
            memcpy(&cnt, rec, 2);
            if (cnt > maxM0) throw ApiError(HNSWGPU_ERR_FORMAT, corrupt);
            const uint32_t* ids = (const uint32_t*)(rec + 4);
            for (uint32_t j = 0; j < cnt; j++) {
                uint32_t v;
                memcpy(&v, ids + j, 4);
                if (v >= cur) throw ApiError(HNSWGPU_ERR_FORMAT, "cand error");
                hl[i * maxM0 + j] = v;
            }
            if (rec[2] & 1) {
                h->deleted[i >> 5] |= 1u << (i & 31);
                h->num_deleted++;
            }
            if (elem == 1) {
                const unsigned char* u = reinterpret_cast<const unsigned char*>(rec + offsetData);
                for (uint64_t c = 0; c < dim; c++) hv[i * h->row_floats + c] = (float)u[c];
            } else {
                memcpy(&hv[i * h->row_floats], rec + offsetData, dim * 4);
            }
            if (multivector) memcpy(&hdocs[i], rec + offsetData + dim * 4, 4);
            uint64_t lab;
            memcpy(&lab, rec + label_offset, 8);
            h->labels[i] = lab;
            h->lookup[lab] = (uint32_t)i;
        }
    }
    // level-0 lists that repeat an id (hnswlib never writes one) need the
    // kernel's per-list duplicate check
    {
        std::vector<uint32_t> stamp(cur, 0xffffffffu);
        h->links_unique = true;
        for (uint64_t i = 0; i < cur && h->links_unique; i++)
            for (uint64_t j = 0; j < maxM0; j++) {
                uint32_t v = hl[i * maxM0 + j];
                if (v == 0xffffffffu) break;
                if (stamp[v] == (uint32_t)i) {
                    h->links_unique = false;
                    break;
                }
                stamp[v] = (uint32_t)i;
            }
    }
    // upper levels (hnswalg.h:795-809)
    std::vector<uint32_t> hoff(cur, 0xffffffffu);
    std::vector<int> level(cur, 0);
    uint64_t upper_rows = 0;
    for (uint64_t i = 0; i < cur; i++) {
        uint32_t sz = ll_sizes[i];
        if (sz % size_links) throw ApiError(HNSWGPU_ERR_FORMAT, corrupt);
        level[i] = (int)(sz / size_links);
        if (sz) {
            hoff[i] = (uint32_t)upper_rows;
            upper_rows += sz / size_links;
        }
    }
    if (cur > 0 && level[ep] < maxlevel) throw ApiError(HNSWGPU_ERR_FORMAT, corrupt);
    std::vector<uint32_t> hup(std::max<uint64_t>(upper_rows, 1) * (maxM + 1), 0u);
    in.seekg(header_end + (std::streamoff)(cur * size_data), in.beg);
    for (uint64_t i = 0; i < cur; i++) {
        uint32_t sz;
        rd(in, sz);
        if (!sz) continue;
        char* dst = (char*)(hup.data() + (size_t)hoff[i] * (maxM + 1));
        in.read(dst, sz);
        for (int L = 1; L <= level[i]; L++) {
            const uint32_t* row = hup.data() + ((size_t)hoff[i] + L - 1) * (maxM + 1);
            uint32_t c = row[0] & 0xffffu;
            if (c > maxM) throw ApiError(HNSWGPU_ERR_FORMAT, corrupt);
            for (uint32_t j = 0; j < c; j++)
                if (row[1 + j] >= cur || level[row[1 + j]] < L) throw ApiError(HNSWGPU_ERR_FORMAT, "cand error");
        }
    }
    if (!in) throw ApiError(HNSWGPU_ERR_FORMAT, corrupt);

    h->vecs.alloc(std::max<size_t>(hv.size(), 4));
    h->links0.alloc(std::max<size_t>(hl.size(), 1));
    h->upper_off.alloc(std::max<size_t>(hoff.size(), 1));
    h->upper_links.alloc(hup.size());
    h->dlabels.alloc(std::max<size_t>(cur, 1));
    h->deleted_bits.alloc(h->deleted.size());
    auto up = [&](void* d, const void* s, size_t b) {
        if (b) cuda_check(cudaMemcpy(d, s, b, cudaMemcpyHostToDevice), "cudaMemcpy");
    };
    up(h->vecs.p, hv.data(), hv.size() * 4);
    up(h->links0.p, hl.data(), hl.size() * 4);
    up(h->upper_off.p, hoff.data(), hoff.size() * 4);
    up(h->upper_links.p, hup.data(), hup.size() * 4);
    up(h->dlabels.p, h->labels.data(), cur * 8);
    up(h->deleted_bits.p, h->deleted.data(), h->deleted.size() * 4);
    if (multivector) {
        h->docs.alloc(std::max<size_t>(cur, 1));
        up(h->docs.p, hdocs.data(), cur * 4);
    }
}

void load_hnsw_file(hnswgpu_index* h, const char* path, int space, uint64_t dim, uint64_t max_elements_i,
                    bool multivector) {
    std::ifstream in(path, std::ios::binary);
    if (!in.is_open()) throw ApiError(HNSWGPU_ERR_IO, "Cannot open file");
    load_hnsw_stream(h, in, space, dim, max_elements_i, multivector);
}

// BruteforceSearch::loadIndex (hnswlib/bruteforce.h:142-161).
void load_bf_file(hnswgpu_index* h, const char* path, int space, uint64_t dim) {
    std::ifstream in(path, std::ios::binary);
    if (!in.is_open()) throw ApiError(HNSWGPU_ERR_IO, "Cannot open file");
    in.seekg(0, in.end);
    const std::streamoff total = in.tellg();
    in.seekg(0, in.beg);
    uint64_t maxel, size_per, cur;
    rd(in, maxel);
    rd(in, size_per);
    rd(in, cur);
    const char* corrupt = "Index seems to be corrupted or unsupported";
    if (!in) throw ApiError(HNSWGPU_ERR_FORMAT, corrupt);
    size_per = dim * 4 + 8;  // recomputed from the space, as bruteforce.h:153
    if (cur > maxel || (uint64_t)(total - 24) < cur * size_per) throw ApiError(HNSWGPU_ERR_FORMAT, corrupt);
    if (cur > 0xfffffffeull) throw ApiError(HNSWGPU_ERR_UNSUPPORTED, "more than 2^32-2 elements");
    h->is_bf = 1;
    h->space = space;
    h->dim = dim;
    h->count = cur;
    h->max_elements = maxel;
    h->row_floats = (uint32_t)((dim + 3) / 4 * 4);
    std::vector<float> hv(cur * h->row_floats, 0.f);
    h->labels.resize(cur);
    std::vector<char> row(size_per);
    for (uint64_t i = 0; i < cur; i++) {
        in.read(row.data(), size_per);
        memcpy(&hv[i * h->row_floats], row.data(), dim * 4);
        uint64_t lab;
        memcpy(&lab, row.data() + dim * 4, 8);
        h->labels[i] = lab;
        h->lookup[lab] = (uint32_t)i;
    }
    if (!in) throw ApiError(HNSWGPU_ERR_FORMAT, corrupt);
    h->vecs.alloc(std::max<size_t>(hv.size(), 4));
    h->dlabels.alloc(std::max<size_t>(cur, 1));
    if (!hv.empty()) cuda_check(cudaMemcpy(h->vecs.p, hv.data(), hv.size() * 4, cudaMemcpyHostToDevice), "cudaMemcpy");
    if (cur) cuda_check(cudaMemcpy(h->dlabels.p, h->labels.data(), cur * 8, cudaMemcpyHostToDevice), "cudaMemcpy");
}

__global__ void normalize_rows_kernel(float* v, uint64_t n, uint32_t dim, uint32_t stride) {
    uint64_t r = (uint64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x / 32);
    int lane = threadIdx.x & 31;
    if (r >= n) return;
    float* x = v + r * stride;
    float sc = 0.f;
    if (lane == 0) sc = hnswgpu::norm_scale(x, (int)dim);
    sc = __shfl_sync(0xffffffffu, sc, 0);
    for (uint32_t i = lane; i < dim; i += 32) x[i] = __fmul_rn(x[i], sc);
}

void create_bf_from_rows(hnswgpu_index* h, int space, uint64_t dim, const float* data, const uint64_t* labels,
                         uint64_t n, uint64_t max_elements) {
    if (n > 0xfffffffeull) throw ApiError(HNSWGPU_ERR_UNSUPPORTED, "more than 2^32-2 elements");
    h->is_bf = 1;
    h->space = space;
    h->dim = dim;
    h->count = n;
    h->max_elements = std::max(max_elements, n);
    h->row_floats = (uint32_t)((dim + 3) / 4 * 4);
    h->labels.assign(labels, labels + n);
    for (uint64_t i = 0; i < n; i++) h->lookup[labels[i]] = (uint32_t)i;
    std::vector<float> hv(n * h->row_floats, 0.f);
    for (uint64_t i = 0; i < n; i++) memcpy(&hv[i * h->row_floats], data + i * dim, dim * 4);
    h->vecs.alloc(std::max<size_t>(hv.size(), 4));
    h->dlabels.alloc(std::max<size_t>(n, 1));
    if (n) {
        cuda_check(cudaMemcpy(h->vecs.p, hv.data(), hv.size() * 4, cudaMemcpyHostToDevice), "cudaMemcpy");
        cuda_check(cudaMemcpy(h->dlabels.p, labels, n * 8, cudaMemcpyHostToDevice), "cudaMemcpy");
        if (space == HNSWGPU_SPACE_COSINE) {
            unsigned blocks = (unsigned)((n + 7) / 8);
            normalize_rows_kernel<<<blocks, 256, 0, h->stream>>>(h->vecs.p, n, (uint32_t)dim, h->row_floats);
            cuda_check(cudaGetLastError(), "normalize launch");
            cuda_check(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
        }
    }
}

uint32_t next_pow2_log2(uint64_t v) {
    uint32_t l = 0;
    while ((1ull << l) < v) l++;
    return l;
}

#ifdef HNSWGPU_PHASE_TIMING
unsigned long long* g_phase_buf = nullptr;
#endif

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}


void ensure_traversal_copy(hnswgpu_index* h, uint32_t prec) {
    if (prec != 1 && prec != 2) throw ApiError(HNSWGPU_ERR_ARG, "precision must be HNSWGPU_PREC_BF16 or _FP8");
    if (h->tcopy[prec].p || h->count == 0) return;
    const uint32_t rb = hnswgpu::traversal_row_bytes(prec, (uint32_t)h->dim);
    h->tcopy[prec].alloc(h->count * rb);
    cuda_check(hnswgpu::launch_quantize_rows(h->vecs.p, (uint32_t)h->count, (uint32_t)h->dim, h->row_floats, prec,
                                             h->tcopy[prec].p, h->stream),
               "quantize launch");
    cuda_check(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
}

// Launch parameters of one HNSW search on device buffers (no allocation;
// work_counter / done_counter / status are left for the caller to set).
hnswgpu::SearchParams hnsw_params(const hnswgpu_index* h, const float* dq, uint64_t nq, uint64_t k, uint64_t ef,
                                  const uint8_t* dallow, uint64_t* dl, float* dd, int32_t* dc, uint32_t* dtrace,
                                  bool exact, uint32_t prec, uint32_t rerank, bool spill) {
    hnswgpu::SearchParams p{};
    p.vecs = h->vecs.p;
    p.links0 = h->links0.p;
    p.upper_off = h->upper_off.p;
    p.upper_links = h->upper_links.p;
    p.labels = h->dlabels.p;
    p.deleted_bits = h->num_deleted ? h->deleted_bits.p : nullptr;
    p.allow = dallow;
    p.count = (uint32_t)h->count;
    p.dim = (uint32_t)h->dim;
    p.row_floats = h->row_floats;
    p.row_bytes = h->row_floats * 4;
    p.maxM = (uint32_t)h->maxM;
    p.maxM0 = (uint32_t)h->maxM0;
    p.ep = h->ep;
    p.maxlevel = h->maxlevel;
    p.queries = dq;
    p.nq = (uint32_t)nq;
    p.q_stride = (uint32_t)h->dim;
    p.k = (uint32_t)k;
    p.ef = (uint32_t)std::max(ef, k);
    p.bare = (h->num_deleted == 0 && dallow == nullptr) ? 1u : 0u;
    p.normalize = h->space == HNSWGPU_SPACE_COSINE ? 1u : 0u;
    p.max_expansions = (uint32_t)std::min<uint64_t>(0xffffff00ull, 2 * h->count + 1024);
    p.out_labels = dl;
    p.out_dists = dd;
    p.out_counts = dc;
    p.trace = dtrace;
    // Staging rows: the 4-lanes-per-row path reads 8 rows per LDS.128 pass, a
    // row pad of 16 floats puts consecutive rows half a bank cycle apart
    // (conflict-free quarter warps); the one-lane-per-row path wants 4.
    p.fast16 = (h->dim % 16 == 0) ? 1u : 0u;
    p.links_unique = h->links_unique ? 1u : 0u;
    p.stage_stride = h->row_floats + (p.fast16 ? 16u : 4u);
    uint32_t slots = (uint32_t)((9u * 1024u + 512u) / (p.stage_stride * 4));
    p.stage_slots = std::max(1u, std::min(p.fast16 ? (uint32_t)HNSWGPU_FP32_SLOTS : 32u, slots));
    p.extra_cap = p.bare ? 0u : std::max<uint32_t>(128u, 4u * p.ef);
    p.exact = exact ? 1u : 0u;
    p.pool_cap = exact ? p.ef + 32u : p.ef;
    // The reference's candidate heap is never pruned.  Its peak per query
    // (oracle traces, 1M x 128, M=16): median ~2.5-3 x ef, 99th percentile
    // ~7-8 x ef, maximum ~10 x ef at small ef.  With a spill area the
    // shared-memory head holds 4 x ef and the global tail 24 x ef more;
    // without one (the allocation-free entry point) shared memory holds it all.
    if (exact && spill) {
        p.cand_cap = std::max<uint32_t>(128u, 4u * p.ef);
        p.cand_spill_cap = std::max<uint32_t>(1024u, 24u * p.ef);
    } else {
        p.cand_cap = exact ? std::max<uint32_t>(512u, 12u * p.ef) : 0u;
    }
    p.log2_vis = std::min<uint32_t>(12, std::max<uint32_t>(HNSWGPU_VIS_LOG2_MIN, next_pow2_log2(16ull * p.ef)));
    if (prec) {
        const char* need =
            "low-precision traversal needs dim % 16 == 0, maxM0 <= 32 (fp8 without deletions or a filter: "
            "maxM0 <= 64) and the id tie order";
        if (!p.fast16 || exact) throw ApiError(HNSWGPU_ERR_UNSUPPORTED, need);
        if (!h->tcopy[prec].p) throw ApiError(HNSWGPU_ERR_ARG, "traversal copy not built");
        p.prec = prec;
        p.tvecs = h->tcopy[prec].p;
        p.trow_bytes = hnswgpu::traversal_row_bytes(prec, (uint32_t)h->dim);
        if (p.maxM0 > 32 && !hnswgpu::lean_eligible(p)) throw ApiError(HNSWGPU_ERR_UNSUPPORTED, need);
        // staging stride: a multiple of 64 bytes with an odd count of 64-byte
        // units, so the two rows a quarter warp reads hit disjoint bank halves
        uint32_t st = (p.trow_bytes + 63) / 64;
        if ((st & 1) == 0) st++;
        p.tstage_bytes = st * 64;
        p.tslots = prec == 2 ? 32u : 16u;
        p.stage_slots = 8;  // float32 rows: upper-layer descent and re-rank batches
        p.rerank = (uint32_t)std::max<uint64_t>(k, rerank ? std::min<uint64_t>(rerank, p.ef) : p.ef);
#ifdef HNSWGPU_BOUNDS_CHECK
        if (getenv("HNSWGPU_DEBUG_NO_RERANK")) p.rerank = 0;
#endif
    }
    // the lean fp8 beam (no row staging, tensor-core distances, two link rows
    // per iteration where maxM0 <= 32) serves unfiltered id-order fp8 searches
    p.lean = hnswgpu::lean_eligible(p) ? 1u : 0u;
    p.lean_w = p.maxM0 <= 32 ? 2u : 1u;
    // (the lean beam's learned-stop kernels, four warps per CTA beside one
    // copy of the network, are budgeted in apply_term)
    const size_t wpb = p.lean ? hnswgpu::kLeanWarpsPerBlock : hnswgpu::kWarpsPerBlock;
    size_t ws = hnswgpu::warp_smem_layout(p);
    int max_optin = 0;
    cuda_check(cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device), "attr");
    while (!p.lean && ws * wpb > (size_t)max_optin && p.log2_vis > 8) {
        p.log2_vis--;
        ws = hnswgpu::warp_smem_layout(p);
    }
    while (exact && ws * wpb > (size_t)max_optin && p.cand_cap > 4u * p.ef) {
        p.cand_cap -= p.ef;
        ws = hnswgpu::warp_smem_layout(p);
    }
    if (ws * wpb > (size_t)max_optin)
        throw ApiError(HNSWGPU_ERR_UNSUPPORTED, "ef too large for the per-query shared-memory budget");
    return p;
}


void apply_term(const hnswgpu_index* h, hnswgpu::SearchParams& p, const TermCfg* t) {
    if (!t || !t->mode) return;
    if (p.exact) throw ApiError(HNSWGPU_ERR_UNSUPPORTED, "learned termination needs the id tie order");
    p.term_mode = t->mode;
    if (t->mode == 1) {
        if (t->period == 0) throw ApiError(HNSWGPU_ERR_ARG, "checkpoint period must be > 0");
        if (p.prec && !p.bare)
            throw ApiError(HNSWGPU_ERR_UNSUPPORTED,
                           "checkpoint recording over a low-precision copy needs an index without deletes and no "
                           "filter");
        p.term_period = t->period;
        p.term_max_ckpt = t->max_ckpt;
        p.ckpt_feat = t->feat;
        p.ckpt_ids = t->ids;
        p.ckpt_dists = t->dists;
        p.ckpt_width = t->width ? t->width : p.k;
        p.ckpt_count = t->count;
    } else {
        if (!h->term_model.p) throw ApiError(HNSWGPU_ERR_STATE, "no termination model set");
        if (std::isinf(h->term_logit) && h->term_logit > 0) {  // never stops: the plain beam
            p.term_mode = 0;
            return;
        }
        p.term_period = h->term_period;
        p.term_model = reinterpret_cast<const float*>(h->term_model.p);
        p.term_logit = h->term_logit;
    }
    // A learned stop usually ends a query long before a large cap: size the
    // visited cache for that (at most 2^11 entries; a miss only repeats a
    // distance, results do not depend on it) so that a large cap does not
    // cost occupancy.
    if (p.log2_vis > 11) {
        p.log2_vis = 11;
        hnswgpu::warp_smem_layout(p);
    }
    if (p.term_mode == 2 && p.lean) {
        int max_optin = 0;
        cuda_check(cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device), "attr");
        if (hnswgpu::kLeanModelSmem + (size_t)p.warp_smem * hnswgpu::kLeanWarpsPerBlockLearned > (size_t)max_optin)
            throw ApiError(HNSWGPU_ERR_UNSUPPORTED, "ef too large for the learned stop's per-query shared-memory budget");
    }
}

// Global tails of the tie-exact candidate heaps, one per resident warp (at
// most 32 CTAs per SM), owned by the index.
static void attach_spill(hnswgpu_index* h, hnswgpu::SearchParams& p, cudaStream_t st) {
    const uint64_t warps = (uint64_t)h->num_sms * 32u * hnswgpu::kWarpsPerBlock;
    const uint64_t need = warps * p.cand_spill_cap;
    if (h->cand_spill.n < need) {
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        h->cand_spill.alloc(need);
    }
    p.cand_spill = h->cand_spill.p;
    p.cand_spill_warps = (uint32_t)warps;
}

static void take_counter_slot(hnswgpu_index* h, hnswgpu::SearchParams& p) {
    const uint32_t slot = h->next_counter++ % (uint32_t)(h->counters.n / 2);
    p.work_counter = h->counters.p + 2 * slot;
    p.done_counter = h->counters.p + 2 * slot + 1;
}

// Two-pass tie-exact mode: the replay pass runs one query per warp and takes
// about one replayed query's latency, whatever the share listed.  Above this
// share of listed queries (e.g. integer-valued data at large ef) the single
// pass that replays every query is the faster one.
constexpr float kTwoPassMaxShare = 0.3f;

// Fold in the listed share of the last listing pass once its copy landed.
static void poll_tie_share(hnswgpu_index* h) {
    if (!h->tie_pending_nq) return;
    const cudaError_t e = cudaEventQuery(h->tie_ev);
    if (e == cudaErrorNotReady) {
        if (cudaPeekAtLastError() == cudaErrorNotReady) (void)cudaGetLastError();
        return;
    }
    cuda_check(e, "cudaEventQuery");
    h->tie_share[h->tie_pending_ef] = {(float)*h->tie_host / (float)h->tie_pending_nq, 0u};
    h->tie_pending_nq = 0;
}

// One HNSW search on device buffers, scratch from the index.  The tie-exact
// mode of an unfiltered float32 beam runs in two launches: the id-order beam
// answers every query and lists those whose run met a tie that can steer the
// reference's heaps (for the others the two orders make the same decisions, so
// the results are the reference's); the heap replay then reruns only the
// listed queries, reading the list's length on the device.
void run_hnsw(hnswgpu_index* h, const float* dq, uint64_t nq, uint64_t k, uint64_t ef, const uint8_t* dallow,
              uint64_t* dl, float* dd, int32_t* dc, uint32_t* dtrace, cudaStream_t st, bool exact, uint32_t prec,
              uint32_t rerank, const TermCfg* term, bool replay_all) {
    if (prec) ensure_traversal_copy(h, prec);
    hnswgpu::SearchParams p = hnsw_params(h, dq, nq, k, ef, dallow, dl, dd, dc, dtrace, exact, prec, rerank, true);
    apply_term(h, p, term);
    p.status = h->status.p;
    const int space = kspace(h);
    hnswgpu::SearchParams p1{};
    bool two_pass = exact && !replay_all && p.fast16 && p.bare && p.maxM0 <= 32;
    if (two_pass) {
        // a share measured above the bound picks the single pass; every 64th
        // call at that ef measures it again
        poll_tie_share(h);
        auto it = h->tie_share.find(p.ef);
        if (it != h->tie_share.end() && it->second.share > kTwoPassMaxShare && ++it->second.calls % 64 != 0)
            two_pass = false;
    }
    if (two_pass) {
        // the listing pass merges into ef + 1 slots to see the first entry dropped
        p1 = hnsw_params(h, dq, nq, k, ef, dallow, dl, dd, dc, dtrace, false);
        p1.pool_cap = p1.ef + 1;
        int max_optin = 0;
        cuda_check(cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device), "attr");
        two_pass = hnswgpu::warp_smem_layout(p1) * hnswgpu::kWarpsPerBlock <= (size_t)max_optin;
    }
    if (two_pass) {
        p1.status = h->status.p;
        if (h->tie_list.n < nq + 1) {
            cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
            h->tie_list.alloc(nq + 1);
        }
        cuda_check(cudaMemsetAsync(h->tie_list.p, 0, 4, st), "cudaMemsetAsync");
        p1.tie_count = h->tie_list.p;
        p1.tie_list = h->tie_list.p + 1;
        take_counter_slot(h, p1);
        cuda_check(hnswgpu::launch_hnsw_search(p1, space, h->num_sms, st, nullptr), "hnsw_search launch");
        p.qcount = h->tie_list.p;
        p.qlist = h->tie_list.p + 1;
        if (!h->tie_pending_nq) {
            if (!h->tie_host) cuda_check(cudaHostAlloc((void**)&h->tie_host, 4, cudaHostAllocDefault), "cudaHostAlloc");
            if (!h->tie_ev) cuda_check(cudaEventCreateWithFlags(&h->tie_ev, cudaEventDisableTiming), "cudaEventCreate");
            cuda_check(cudaMemcpyAsync(h->tie_host, h->tie_list.p, 4, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
            cuda_check(cudaEventRecord(h->tie_ev, st), "cudaEventRecord");
            h->tie_pending_ef = p.ef;
            h->tie_pending_nq = nq;
        }
    }
    if (exact) attach_spill(h, p, st);
#ifdef HNSWGPU_PHASE_TIMING
    static unsigned long long* phase_buf = nullptr;
    if (!phase_buf) {
        cuda_check(cudaMalloc((void**)&phase_buf, 10 * sizeof(unsigned long long)), "cudaMalloc");
        cuda_check(cudaMemset(phase_buf, 0, 10 * sizeof(unsigned long long)), "cudaMemset");
    }
    p.phase_cycles = phase_buf;
    g_phase_buf = phase_buf;
#endif
    take_counter_slot(h, p);
    cuda_check(hnswgpu::launch_hnsw_search(p, space, h->num_sms, st, nullptr), "hnsw_search launch");
}

// Epsilon search of a batch on device buffers: searchStopConditionClosest
// with EpsilonSearchStopCondition(eps, min_c, max_c), the tie-exact general
// loop with ef = k = max_c (hnswalg.h:1326-1377, stop_condition.h:219-275).
void run_epsilon(hnswgpu_index* h, const float* dq, uint64_t nq, float eps, uint64_t min_c, uint64_t max_c,
                 const uint8_t* dallow, uint64_t* dl, float* dd, int32_t* dc, cudaStream_t st) {
    hnswgpu::SearchParams p = hnsw_params(h, dq, nq, max_c, max_c, dallow, dl, dd, dc, nullptr, true, 0, 0, true);
    if (!p.bare) {
        // Until min_num_candidates allowed results are held the loop accepts
        // every neighbour, so a selective filter queues many disallowed
        // candidates: give their list room for up to 2048 (or the index)
        // where shared memory allows.
        const uint32_t want = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(2048, 4ull * p.ef), h->count + 1);
        if (want > p.extra_cap) {
            hnswgpu::SearchParams wider = p;
            wider.extra_cap = want;
            int max_optin = 0;
            cuda_check(cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device), "attr");
            if (hnswgpu::warp_smem_layout(wider) * hnswgpu::kWarpsPerBlock <= (size_t)max_optin) p = wider;
        }
    }
    p.eps_mode = 1;
    p.eps = eps;
    p.eps_min = (uint32_t)min_c;
    p.status = h->status.p;
    attach_spill(h, p, st);
    take_counter_slot(h, p);
    cuda_check(hnswgpu::launch_hnsw_search(p, kspace(h), h->num_sms, st, nullptr),
               "hnsw_search launch");
}

// Exact brute force of a batch on device buffers (bf_search.cu).
static void run_bf_exact(hnswgpu_index* h, const float* dq, uint64_t nq, uint64_t k, const uint8_t* dallow,
                         uint64_t* dl, float* dd, int32_t* dc, cudaStream_t st) {
    hnswgpu::BfParams b{};
    b.vecs = h->vecs.p;
    b.labels = h->dlabels.p;
    b.allow = dallow;
    b.count = (uint32_t)h->count;
    b.dim = (uint32_t)h->dim;
    b.row_floats = h->row_floats;
    b.queries = dq;
    b.nq = (uint32_t)nq;
    b.k = (uint32_t)k;
    b.normalize = h->space == HNSWGPU_SPACE_COSINE ? 1u : 0u;
    b.out_labels = dl;
    b.out_dists = dd;
    b.out_counts = dc;
    b.status = h->status.p;
    cuda_check(hnswgpu::launch_bf_search(b, kspace(h), h->num_sms, st), "bf_search launch");
}

static uint32_t pow2_at_least(uint64_t v) {
    uint32_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

// Tensor-core brute force (bf_tc.cu) of a BruteforceSearch index over its
// bf16 / fp8 copy: sampled threshold, tcgen05 scores with fused candidate
// filtering, selection of the R best and exact float32 re-rank; queries the
// filter could not bound are answered by the exact kernel.  Synchronises.
void run_bf_tc(hnswgpu_index* h, const float* dq, uint64_t nq, uint64_t k, uint32_t rerank, const uint8_t* dallow,
               uint64_t* dl, float* dd, int32_t* dc, uint32_t* dtrace, cudaStream_t st, uint32_t prec) {
    const uint64_t n = h->count;
    const uint32_t dim = (uint32_t)h->dim;
    const uint64_t R = std::max<uint64_t>(k, rerank ? rerank : 4 * k);
    if (R > 1024) throw ApiError(HNSWGPU_ERR_UNSUPPORTED, "tensor-core brute force: over-fetch (rerank, or 4 k) must be <= 1024");
    if (nq > 0x7fffffffull) throw ApiError(HNSWGPU_ERR_ARG, "batch too large");
    const bool first = !h->tc_rowinfo[prec].p;
    ensure_traversal_copy(h, prec);
    const uint32_t trow = hnswgpu::traversal_row_bytes(prec, dim);
    if (first) {
        h->tc_rowinfo[prec].alloc((n + 255) / 256 * 256);  // whole tiles: read by 2 KB bulk copies
        cuda_check(hnswgpu::launch_tc_rowinfo(h->vecs.p, (uint32_t)n, dim, h->row_floats, h->tcopy[prec].p, trow, prec,
                                              h->tc_rowinfo[prec].p, h->stream),
                   "rowinfo launch");
        cuda_check(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    }
    // sampling: about 5 R rows of the whole set below the 16th-best sampled distance
    const bool sampled = n > 16384;
    uint64_t step = 1, n_sample = n, cap = n;
    if (sampled) {
        const uint64_t S = std::min<uint64_t>(8192, std::max<uint64_t>(64, 16 * n / (5 * R)));
        step = std::max<uint64_t>(1, n / S);
        n_sample = (n + step - 1) / step;
        const uint64_t expected = 16 * n / n_sample;
        cap = std::min<uint64_t>(16384, pow2_at_least(std::max<uint64_t>(3 * expected, 2 * R)));
    }
    const uint32_t sort_cap = pow2_at_least(std::max<uint64_t>(cap, 1));
    const size_t sel_smem = hnswgpu::tc_select_smem(sort_cap, dim, (uint32_t)R);
    int max_optin = 0;
    cuda_check(cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device), "attr");
    if (sel_smem + 1024 > (size_t)max_optin)
        throw ApiError(HNSWGPU_ERR_UNSUPPORTED, "tensor-core brute force: candidate list too large for shared memory");
    h->tc_qf.ensure(nq * dim);
    h->tc_qt.ensure(nq * trow + 16);
    h->tc_qscale.ensure(nq);
    h->tc_tau.ensure(nq);
    h->tc_cnt.ensure(nq);
    h->tc_flags.ensure(nq);
    h->tc_buf.ensure(nq * cap);
    cuda_check(hnswgpu::launch_tc_query_prep(dq, (uint32_t)nq, dim, h->space == HNSWGPU_SPACE_COSINE, prec, trow,
                                             h->tc_qf.p, h->tc_qt.p, h->tc_qscale.p, st),
               "query prep launch");
    CUtensorMap qmap, xmap, smap;
    cuda_check(hnswgpu::tc_encode_map(h->tc_qt.p, prec, nq, dim, trow, 128, &qmap), "tensor map (queries)");
    cuda_check(hnswgpu::tc_encode_map(h->tcopy[prec].p, prec, n, dim, trow, 256, &xmap), "tensor map (rows)");
    const int space = kspace(h);
    hnswgpu::TcArgs a{};
    a.nq = (uint32_t)nq;
    a.k_blocks = (dim * (prec == 1 ? 2u : 1u) + 127) / 128;
    a.rowinfo = h->tc_rowinfo[prec].p;
    a.qscale = h->tc_qscale.p;
    a.allow = dallow;
    a.tau = h->tc_tau.p;
    a.cnt = h->tc_cnt.p;
    a.buf = h->tc_buf.p;
    a.cap = (uint32_t)cap;
    a.status = h->status.p;
    if (sampled) {
        cuda_check(hnswgpu::tc_encode_map(h->tcopy[prec].p, prec, n_sample, dim, (uint64_t)trow * step, 256, &smap),
                   "tensor map (sample)");
        h->tc_sinfo.ensure((n_sample + 255) / 256 * 256);
        cuda_check(hnswgpu::launch_tc_gather_info(h->tc_rowinfo[prec].p, n_sample, step, h->tc_sinfo.p, st),
                   "gather launch");
        hnswgpu::TcArgs t = a;
        t.n_rows = (uint32_t)n_sample;
        t.row_step = step;
        t.rowinfo = h->tc_sinfo.p;
        t.chunk_tiles = 1;
        cuda_check(hnswgpu::launch_tc_scores(qmap, smap, t, prec, space, 1, h->num_sms, st), "threshold launch");
    } else {
        cuda_check(hnswgpu::launch_tc_fill(h->tc_tau.p, nq, __builtin_inff(), st), "fill launch");
    }
    cuda_check(cudaMemsetAsync(h->tc_cnt.p, 0, nq * 4, st), "cudaMemsetAsync");
    a.n_rows = (uint32_t)n;
    a.row_step = 1;
    {
        // Work items are (query tile, 16 row tiles), ordered row-chunk major:
        // the CTAs running at one time share one or two chunks (a few MB of
        // rows), so each row tile comes from HBM once and from L2 for every
        // other query tile.  Chunks of ~100 MB (a few items per CTA) missed
        // L2 and re-read the rows ~11 times.
        const uint64_t n_tiles = (n + 255) / 256;
        a.chunk_tiles = (uint32_t)std::min<uint64_t>(16, n_tiles);
    }
    cuda_check(hnswgpu::launch_tc_scores(qmap, xmap, a, prec, space, 0, h->num_sms, st), "scores launch");
    if (dtrace) cuda_check(cudaMemsetAsync(dtrace, 0, nq * 16, st), "cudaMemsetAsync");
    hnswgpu::TcSelectArgs sa{};
    sa.nq = (uint32_t)nq;
    sa.k = (uint32_t)k;
    sa.R = (uint32_t)R;
    sa.cap = (uint32_t)cap;
    sa.sort_cap = sort_cap;
    sa.dim = dim;
    sa.row_floats = h->row_floats;
    sa.sampled = sampled ? 1u : 0u;
    sa.cnt = h->tc_cnt.p;
    sa.buf = h->tc_buf.p;
    sa.qf = h->tc_qf.p;
    sa.vecs = h->vecs.p;
    sa.labels = h->dlabels.p;
    sa.out_labels = dl;
    sa.out_dists = dd;
    sa.out_counts = dc;
    sa.flags = h->tc_flags.p;
    sa.trace = dtrace;
    cuda_check(hnswgpu::launch_tc_select(sa, space, st), "select launch");
    // queries the filter could not bound: exact kernel
    std::vector<uint8_t> flags(nq);
    cuda_check(cudaMemcpyAsync(flags.data(), h->tc_flags.p, nq, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    uint32_t status = 0;
    cuda_check(cudaMemcpyAsync(&status, h->status.p, 4, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    if (status & HNSWGPU_STATUS_TIMEOUT) throw ApiError(HNSWGPU_ERR_KERNEL, "tensor-core kernel timed out waiting");
    std::vector<uint32_t> redo;
    for (uint64_t i = 0; i < nq; i++)
        if (flags[i]) redo.push_back((uint32_t)i);
    if (!redo.empty()) {
        const uint64_t m = redo.size();
        h->tc_idx.ensure(m);
        DevBuf<float> rq, rd;
        DevBuf<uint64_t> rl;
        DevBuf<int32_t> rc;
        rq.alloc(m * dim);
        rd.alloc(m * k);
        rl.alloc(m * k);
        rc.alloc(m);
        cuda_check(cudaMemcpyAsync(h->tc_idx.p, redo.data(), m * 4, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
        cuda_check(hnswgpu::launch_tc_gather(dq, h->tc_idx.p, (uint32_t)m, dim, rq.p, st), "gather launch");
        run_bf_exact(h, rq.p, m, k, dallow, rl.p, rd.p, rc.p, st);
        cuda_check(hnswgpu::launch_tc_scatter(h->tc_idx.p, (uint32_t)m, (uint32_t)k, rl.p, rd.p, rc.p, dl, dd, dc, st),
                   "scatter launch");
        if (dtrace) {
            // mark fallback queries in trace[2]
            std::vector<uint32_t> tr(nq * 4);
            cuda_check(cudaMemcpyAsync(tr.data(), dtrace, nq * 16, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
            cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
            for (uint32_t i : redo) tr[(size_t)i * 4 + 2] = 1;
            cuda_check(cudaMemcpyAsync(dtrace, tr.data(), nq * 16, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
        }
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    }
}

void run_search(hnswgpu_index* h, const float* dq, uint64_t nq, uint64_t k, uint64_t ef, const uint8_t* dallow,
                uint64_t* dl, float* dd, int32_t* dc, uint32_t* dtrace, cudaStream_t st, bool exact,
                uint32_t prec, uint32_t rerank, const TermCfg* term, bool scan, bool replay_all) {
    if (scan && !h->is_bf && h->num_deleted) {
        // deleted elements are never returned: fold them into the row mask
        h->scan_mask.ensure(h->count);
        cuda_check(hnswgpu::launch_scan_mask(h->deleted_bits.p, dallow, h->count, h->scan_mask.p, st), "mask launch");
        dallow = h->scan_mask.p;
    }
    if (h->is_bf && prec) {
        run_bf_tc(h, dq, nq, k, rerank, dallow, dl, dd, dc, dtrace, st, prec);
    } else if (h->is_bf || scan) {
        hnswgpu::BfParams b{};
        b.vecs = h->vecs.p;
        b.labels = h->dlabels.p;
        b.allow = dallow;
        b.count = (uint32_t)h->count;
        b.dim = (uint32_t)h->dim;
        b.row_floats = h->row_floats;
        b.queries = dq;
        b.nq = (uint32_t)nq;
        b.k = (uint32_t)k;
        b.normalize = h->space == HNSWGPU_SPACE_COSINE ? 1u : 0u;
        b.out_labels = dl;
        b.out_dists = dd;
        b.out_counts = dc;
        b.status = h->status.p;
        cuda_check(hnswgpu::launch_bf_search(b, kspace(h), h->num_sms, st),
                   "bf_search launch");
    } else {
        run_hnsw(h, dq, nq, k, ef, dallow, dl, dd, dc, dtrace, st, exact, prec, rerank, term, replay_all);
    }
}

}  // namespace hnswgpu_host

#ifdef HNSWGPU_BOUNDS_CHECK
namespace hnswgpu {
cudaError_t read_debug_record(unsigned long long* out);
cudaError_t read_lean_debug_record(unsigned long long* out);
}
#endif

extern "C" {

const char* hnswgpu_last_error(void) { return g_last_error.c_str(); }

const char* hnswgpu_version(void) { return "hnswgpu 0.1 (sm_100a)"; }

int hnswgpu_load_hnsw(const char* path, int space, uint64_t dim, uint64_t max_elements, int device,
                      hnswgpu_index** out) {
    return guarded([&] {
        if (!path || !out || dim == 0) return fail(HNSWGPU_ERR_ARG, "invalid argument");
        if (space < 0 || space > 3) return fail(HNSWGPU_ERR_ARG, "Space name must be one of l2, ip, or cosine.");
        *out = nullptr;
        std::unique_ptr<hnswgpu_index> h(new hnswgpu_index());
        init_common(h.get(), device);
        load_hnsw_file(h.get(), path, space, dim, max_elements, false);
        h->source_path = path;
        *out = h.release();
        return HNSWGPU_OK;
    });
}

int hnswgpu_load_hnsw_buffer(const void* data, uint64_t size, int space, uint64_t dim, uint64_t max_elements,
                             int device, hnswgpu_index** out) {
    return guarded([&] {
        if (!data || !out || dim == 0) return fail(HNSWGPU_ERR_ARG, "invalid argument");
        if (space < 0 || space > 3) return fail(HNSWGPU_ERR_ARG, "Space name must be one of l2, ip, or cosine.");
        *out = nullptr;
        std::unique_ptr<hnswgpu_index> h(new hnswgpu_index());
        init_common(h.get(), device);
        MemBuf mb(static_cast<const char*>(data), (size_t)size);
        std::istream in(&mb);
        load_hnsw_stream(h.get(), in, space, dim, max_elements, false);
        *out = h.release();
        return HNSWGPU_OK;
    });
}

int hnswgpu_load_hnsw_multivector(const char* path, uint64_t dim, uint64_t max_elements, int device,
                                  hnswgpu_index** out) {
    return guarded([&] {
        if (!path || !out || dim == 0) return fail(HNSWGPU_ERR_ARG, "invalid argument");
        *out = nullptr;
        std::unique_ptr<hnswgpu_index> h(new hnswgpu_index());
        init_common(h.get(), device);
        load_hnsw_file(h.get(), path, HNSWGPU_SPACE_L2, dim, max_elements, true);
        h->source_path = path;
        *out = h.release();
        return HNSWGPU_OK;
    });
}

int hnswgpu_search_multivector(hnswgpu_index* h, const float* queries, uint64_t nq, uint64_t num_docs,
                               uint64_t ef_collection, uint64_t cap, uint64_t* out_ids, float* out_dists,
                               int32_t* out_counts) {
    return guarded([&] {
        if (!h || h->is_bf || (nq && (!queries || !out_ids || !out_dists || !out_counts)) || cap == 0)
            return fail(HNSWGPU_ERR_ARG, "invalid argument");
        if (!h->docs.p) return fail(HNSWGPU_ERR_STATE, "not a multi-vector index (hnswgpu_load_hnsw_multivector)");
        if (num_docs == 0) return fail(HNSWGPU_ERR_ARG, "num_docs must be > 0");
        if (nq > 0x7fffffffull || cap > 0xffffffffull || num_docs > 0xffffffffull || ef_collection > 0xffffffffull)
            return fail(HNSWGPU_ERR_ARG, "batch too large");
        if (h->num_deleted)
            return fail(HNSWGPU_ERR_UNSUPPORTED, "multi-vector search over an index with deleted elements");
        if (h->maxM0 > 64) return fail(HNSWGPU_ERR_UNSUPPORTED, "multi-vector search needs maxM0 <= 64");
        std::lock_guard<std::mutex> g(h->mu);
        set_device(h);
        if (nq == 0) return HNSWGPU_OK;
        if (h->count == 0) {
            memset(out_counts, 0, nq * 4);
            for (uint64_t i = 0; i < nq * cap; i++) {
                out_ids[i] = ~0ull;
                out_dists[i] = __builtin_inff();
            }
            return HNSWGPU_OK;
        }
        hnswgpu::MvParams p{};
        p.vecs = h->vecs.p;
        p.links0 = h->links0.p;
        p.upper_off = h->upper_off.p;
        p.upper_links = h->upper_links.p;
        p.docs = h->docs.p;
        p.count = (uint32_t)h->count;
        p.dim = (uint32_t)h->dim;
        p.row_floats = h->row_floats;
        p.maxM = (uint32_t)h->maxM;
        p.maxM0 = (uint32_t)h->maxM0;
        p.ep = h->ep;
        p.maxlevel = h->maxlevel;
        p.nq = (uint32_t)nq;
        p.num_docs = (uint32_t)num_docs;
        p.ef_coll = (uint32_t)ef_collection;
        p.cap = (uint32_t)cap;
        p.max_expansions = (uint32_t)std::min<uint64_t>(0xffffff00ull, 2 * h->count + 1024);
        // the largest layout that fits: top_candidates up to 2048 entries,
        // the document table and the visited set sized from the index
        int max_optin = 0;
        cuda_check(cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device), "attr");
        p.top_cap = 2048;
        p.doc_log2 = 12;
        p.vis_log2 = (uint32_t)std::min<uint64_t>(14, std::max<uint64_t>(10, next_pow2_log2(2 * h->count)));
        while (hnswgpu::multivec_smem(p) > (size_t)max_optin && p.top_cap > 256) p.top_cap /= 2;
        while (hnswgpu::multivec_smem(p) > (size_t)max_optin && p.vis_log2 > 10) p.vis_log2--;
        if (hnswgpu::multivec_smem(p) > (size_t)max_optin)
            return fail(HNSWGPU_ERR_UNSUPPORTED, "multi-vector search: dim too large for the shared-memory layout");
        DevBuf<float> dq;
        DevBuf<uint64_t> di;
        DevBuf<float> dd;
        DevBuf<int32_t> dc;
        dq.alloc(nq * h->dim);
        di.alloc(nq * cap);
        dd.alloc(nq * cap);
        dc.alloc(nq);
        cuda_check(cudaMemcpyAsync(dq.p, queries, nq * h->dim * 4, cudaMemcpyHostToDevice, h->stream), "cudaMemcpyAsync");
        p.queries = dq.p;
        p.out_ids = di.p;
        p.out_dists = dd.p;
        p.out_counts = dc.p;
        p.status = h->status.p;
        cuda_check(hnswgpu::launch_hnsw_multivec(p, h->num_sms, h->stream), "multivector launch");
        cuda_check(cudaMemcpyAsync(out_ids, di.p, nq * cap * 8, cudaMemcpyDeviceToHost, h->stream), "cudaMemcpyAsync");
        cuda_check(cudaMemcpyAsync(out_dists, dd.p, nq * cap * 4, cudaMemcpyDeviceToHost, h->stream), "cudaMemcpyAsync");
        cuda_check(cudaMemcpyAsync(out_counts, dc.p, nq * 4, cudaMemcpyDeviceToHost, h->stream), "cudaMemcpyAsync");
        cuda_check(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
        return HNSWGPU_OK;
    });
}

int hnswgpu_load_bf(const char* path, int space, uint64_t dim, int device, hnswgpu_index** out) {
    return guarded([&] {
        if (!path || !out || dim == 0) return fail(HNSWGPU_ERR_ARG, "invalid argument");
        if (space == HNSWGPU_SPACE_L2_UINT8)
            return fail(HNSWGPU_ERR_UNSUPPORTED, "uint8 L2 (L2SpaceI) is supported for HNSW indexes only");
        if (space < 0 || space > 2) return fail(HNSWGPU_ERR_ARG, "Space name must be one of l2, ip, or cosine.");
        *out = nullptr;
        std::unique_ptr<hnswgpu_index> h(new hnswgpu_index());
        init_common(h.get(), device);
        load_bf_file(h.get(), path, space, dim);
        *out = h.release();
        return HNSWGPU_OK;
    });
}

int hnswgpu_create_bf(int space, uint64_t dim, const float* data, const uint64_t* labels, uint64_t n,
                      uint64_t max_elements, int device, hnswgpu_index** out) {
    return guarded([&] {
        if (!out || dim == 0 || (n && (!data || !labels))) return fail(HNSWGPU_ERR_ARG, "invalid argument");
        if (space == HNSWGPU_SPACE_L2_UINT8)
            return fail(HNSWGPU_ERR_UNSUPPORTED, "uint8 L2 (L2SpaceI) is supported for HNSW indexes only");
        if (space < 0 || space > 2) return fail(HNSWGPU_ERR_ARG, "Space name must be one of l2, ip, or cosine.");
        *out = nullptr;
        std::unique_ptr<hnswgpu_index> h(new hnswgpu_index());
        init_common(h.get(), device);
        create_bf_from_rows(h.get(), space, dim, data, labels, n, max_elements);
        *out = h.release();
        return HNSWGPU_OK;
    });
}

int hnswgpu_build_traversal_copy(hnswgpu_index* h, uint32_t precision) {
    return guarded([&] {
        if (!h || h->is_bf) return fail(HNSWGPU_ERR_ARG, "invalid argument");
        std::lock_guard<std::mutex> g(h->mu);
        set_device(h);
        ensure_traversal_copy(h, precision);
        return HNSWGPU_OK;
    });
}

int hnswgpu_free(hnswgpu_index* h) {
    if (!h) return HNSWGPU_OK;
    cudaSetDevice(h->device);
    if (h->stream) {
        cudaStreamSynchronize(h->stream);
        cudaStreamDestroy(h->stream);
    }
    delete h;
    return HNSWGPU_OK;
}

int hnswgpu_get_info(const hnswgpu_index* h, hnswgpu_info* o) {
    if (!h || !o) return fail(HNSWGPU_ERR_ARG, "invalid argument");
    memset(o, 0, sizeof(*o));
    o->count = h->count;
    o->max_elements = h->max_elements;
    o->dim = h->dim;
    o->M = h->M;
    o->maxM = h->maxM;
    o->maxM0 = h->maxM0;
    o->ef_construction = h->efc;
    o->ef = h->ef;
    o->num_deleted = h->num_deleted;
    o->maxlevel = h->maxlevel;
    o->enterpoint = h->ep;
    o->space = h->space;
    o->is_bruteforce = h->is_bf;
    o->device_bytes = h->device_bytes();
    return HNSWGPU_OK;
}

int hnswgpu_set_ef(hnswgpu_index* h, uint64_t ef) {
    if (!h) return fail(HNSWGPU_ERR_ARG, "invalid argument");
    std::lock_guard<std::mutex> g(h->mu);
    h->ef = ef;
    return HNSWGPU_OK;
}

int hnswgpu_get_labels(const hnswgpu_index* h, uint64_t* out) {
    if (!h || (!out && h->count)) return fail(HNSWGPU_ERR_ARG, "invalid argument");
    if (h->count) memcpy(out, h->labels.data(), h->count * 8);
    return HNSWGPU_OK;
}

static int set_mark(hnswgpu_index* h, uint64_t label, bool mark) {
    return guarded([&] {
        if (!h) return fail(HNSWGPU_ERR_ARG, "invalid argument");
        if (h->is_bf) return fail(HNSWGPU_ERR_UNSUPPORTED, "brute-force indexes have no delete marks");
        std::lock_guard<std::mutex> g(h->mu);
        auto it = h->lookup.find(label);
        if (it == h->lookup.end()) return fail(HNSWGPU_ERR_LABEL, "Label not found");
        uint32_t id = it->second;
        uint32_t& w = h->deleted[id >> 5];
        bool cur = (w >> (id & 31)) & 1u;
        if (mark && cur) return fail(HNSWGPU_ERR_STATE, "The requested to delete element is already deleted");
        if (!mark && !cur) return fail(HNSWGPU_ERR_STATE, "The requested to undelete element is not deleted");
        w ^= 1u << (id & 31);
        h->num_deleted += mark ? 1 : (uint64_t)-1;
        set_device(h);
        cuda_check(cudaMemcpyAsync(h->deleted_bits.p + (id >> 5), &w, 4, cudaMemcpyHostToDevice, h->stream),
                   "cudaMemcpyAsync");
        cuda_check(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
        return HNSWGPU_OK;
    });
}

int hnswgpu_mark_deleted(hnswgpu_index* h, uint64_t label) { return set_mark(h, label, true); }
int hnswgpu_unmark_deleted(hnswgpu_index* h, uint64_t label) { return set_mark(h, label, false); }

int hnswgpu_search(hnswgpu_index* h, const float* queries, uint64_t nq, uint64_t k, const hnswgpu_search_opts* opts,
                   uint64_t* out_labels, float* out_dists, int32_t* out_counts) {
    return guarded([&] {
        if (!h || k == 0 || (nq && (!queries || !out_labels || !out_dists || !out_counts)))
            return fail(HNSWGPU_ERR_ARG, "invalid argument");
        if (nq > 0xffffffffull || k > 0xffffffffull) return fail(HNSWGPU_ERR_ARG, "batch too large");
        hnswgpu_search_opts o{};
        if (opts) o = *opts;
        const bool dev = (o.flags & HNSWGPU_DEVICE_PTRS) != 0;
        const bool want_trace = (o.flags & HNSWGPU_TRACE) && o.trace;
        const bool exact = (o.flags & HNSWGPU_EXACT_TIES) != 0;
        const bool scan = (o.flags & HNSWGPU_EXACT_SCAN) != 0;
        const bool replay_all = (o.flags & HNSWGPU_REPLAY_ALL) != 0;
        TermCfg term;
        if (o.flags & HNSWGPU_LEARNED_STOP) term.mode = 2;
        if (scan && term.mode) return fail(HNSWGPU_ERR_ARG, "HNSWGPU_EXACT_SCAN excludes HNSWGPU_LEARNED_STOP");
        const uint64_t ef = o.ef ? o.ef : h->ef;
        cudaStream_t st = o.stream ? (cudaStream_t)o.stream : h->stream;
        std::lock_guard<std::mutex> g(h->mu);
        set_device(h);
        const uint8_t* dfilter = nullptr;  // a registered filter's device mask
        if (o.filter) {
            if (o.allow) return fail(HNSWGPU_ERR_ARG, "give either an allow mask or a registered filter, not both");
            if (o.filter > h->filters.size() || !h->filters[o.filter - 1])
                return fail(HNSWGPU_ERR_ARG, "unknown filter id");
            dfilter = h->filters[o.filter - 1]->p;
        }
        if (nq == 0) return HNSWGPU_OK;
        if (h->count == 0) {
            // empty index: searchKnn returns nothing (hnswalg.h:1272)
            if (dev) {
                cuda_check(cudaMemsetAsync(out_counts, 0, nq * 4, st), "cudaMemsetAsync");
                cuda_check(cudaMemsetAsync(out_labels, 0xff, nq * k * 8, st), "cudaMemsetAsync");
                cuda_check(cudaMemsetAsync(out_dists, 0x7f, nq * k * 4, st), "cudaMemsetAsync");
            } else {
                memset(out_counts, 0, nq * 4);
                for (uint64_t i = 0; i < nq * k; i++) {
                    out_labels[i] = ~0ull;
                    out_dists[i] = __builtin_inff();
                }
            }
            return HNSWGPU_OK;
        }
        if (dev) {
            run_search(h, queries, nq, k, ef, dfilter ? dfilter : o.allow, out_labels, out_dists, out_counts,
                       want_trace ? o.trace : nullptr, st, exact, o.precision, o.rerank, &term, scan, replay_all);
            return HNSWGPU_OK;
        }
        // host pointers: stage through the index's device I/O buffer
        const size_t qb = nq * h->dim * 4, lb = nq * k * 8, db = nq * k * 4, cb = nq * 4,
                     tb = want_trace ? nq * 16 : 0;
        auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
        h->io.ensure(al(qb) + al(lb) + al(db) + al(cb) + al(tb));
        unsigned char* base = h->io.p;
        float* dq = (float*)base;
        uint64_t* dl = (uint64_t*)(base + al(qb));
        float* dd = (float*)(base + al(qb) + al(lb));
        int32_t* dc = (int32_t*)(base + al(qb) + al(lb) + al(db));
        uint32_t* dt = want_trace ? (uint32_t*)(base + al(qb) + al(lb) + al(db) + al(cb)) : nullptr;
        const uint8_t* dallow = dfilter;
        if (o.allow) {
            h->allow.ensure(h->count);
            cuda_check(cudaMemcpyAsync(h->allow.p, o.allow, h->count, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
            dallow = h->allow.p;
        }
        cuda_check(cudaMemcpyAsync(dq, queries, qb, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
        run_search(h, dq, nq, k, ef, dallow, dl, dd, dc, dt, st, exact, o.precision, o.rerank, &term, scan,
                   replay_all);
        cuda_check(cudaMemcpyAsync(out_labels, dl, lb, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        cuda_check(cudaMemcpyAsync(out_dists, dd, db, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        cuda_check(cudaMemcpyAsync(out_counts, dc, cb, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        if (dt) cuda_check(cudaMemcpyAsync(o.trace, dt, tb, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        uint32_t status = 0;
        cuda_check(cudaMemcpyAsync(&status, h->status.p, 4, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        if (status & HNSWGPU_STATUS_TIMEOUT) {
            cudaMemsetAsync(h->status.p, 0, 4, st);
            cudaStreamSynchronize(st);
            return fail(HNSWGPU_ERR_KERNEL, "search kernel timed out waiting for a copy");
        }
        return HNSWGPU_OK;
    });
}

int hnswgpu_filter_create(hnswgpu_index* h, const uint8_t* allow, uint32_t* out_id) {
    return guarded([&] {
        if (!h || !out_id || (h->count && !allow)) return fail(HNSWGPU_ERR_ARG, "invalid argument");
        std::lock_guard<std::mutex> g(h->mu);
        set_device(h);
        std::unique_ptr<DevBuf<uint8_t>> buf(new DevBuf<uint8_t>());
        buf->alloc(std::max<uint64_t>(h->count, 1));
        if (h->count) {
            cuda_check(cudaMemcpyAsync(buf->p, allow, h->count, cudaMemcpyHostToDevice, h->stream), "cudaMemcpyAsync");
            cuda_check(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
        }
        size_t slot = 0;
        while (slot < h->filters.size() && h->filters[slot]) slot++;
        if (slot == h->filters.size()) h->filters.emplace_back();
        h->filters[slot] = std::move(buf);
        *out_id = (uint32_t)slot + 1;
        return HNSWGPU_OK;
    });
}

int hnswgpu_filter_destroy(hnswgpu_index* h, uint32_t id) {
    return guarded([&] {
        if (!h) return fail(HNSWGPU_ERR_ARG, "invalid argument");
        std::lock_guard<std::mutex> g(h->mu);
        if (id == 0 || id > h->filters.size() || !h->filters[id - 1]) return fail(HNSWGPU_ERR_ARG, "unknown filter id");
        set_device(h);
        // searches queued on the index's stream may still read it
        cuda_check(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
        h->filters[id - 1].reset();
        return HNSWGPU_OK;
    });
}

int hnswgpu_save_hnsw(hnswgpu_index* h, const char* path) {
    return guarded([&] {
        if (!h || !path || h->is_bf) return fail(HNSWGPU_ERR_ARG, "hnswgpu_save_hnsw needs an HNSW index");
        std::lock_guard<std::mutex> g(h->mu);
        if (h->source_path.empty()) return fail(HNSWGPU_ERR_STATE, "the index was not loaded from a file");
        std::ifstream in(h->source_path, std::ios::binary);
        if (!in.is_open()) throw ApiError(HNSWGPU_ERR_IO, "Cannot open file");
        std::vector<char> bytes((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
        // header (hnswalg.h:685-712), then the level-0 block: rewrite the
        // delete mark of every element (bit 0 of byte 2 of its record,
        // hnswalg.h:872-885) from the current marks
        const size_t header = 8 * 6 + 4 + 4 + 8 * 3 + 8 + 8;
        uint64_t size_data = 0;
        if (bytes.size() < header) throw ApiError(HNSWGPU_ERR_FORMAT, "Index seems to be corrupted or unsupported");
        memcpy(&size_data, bytes.data() + 24, 8);
        if (bytes.size() < header + h->count * size_data)
            throw ApiError(HNSWGPU_ERR_FORMAT, "Index seems to be corrupted or unsupported");
        for (uint64_t i = 0; i < h->count; i++) {
            char& flags = bytes[header + i * size_data + 2];
            const bool del = (h->deleted[i >> 5] >> (i & 31)) & 1u;
            flags = del ? (char)(flags | 1) : (char)(flags & ~1);
        }
        std::ofstream out(path, std::ios::binary);
        if (!out.is_open()) throw ApiError(HNSWGPU_ERR_IO, "Cannot open file");
        out.write(bytes.data(), (std::streamsize)bytes.size());
        if (!out) throw ApiError(HNSWGPU_ERR_IO, "write failed");
        return HNSWGPU_OK;
    });
}

int hnswgpu_search_epsilon(hnswgpu_index* h, const float* queries, uint64_t nq, float epsilon,
                           uint64_t min_candidates, uint64_t max_candidates, const hnswgpu_search_opts* opts,
                           uint64_t* out_ids, float* out_dists, int32_t* out_counts) {
    return guarded([&] {
        if (!h || h->is_bf || (nq && (!queries || !out_ids || !out_dists || !out_counts)))
            return fail(HNSWGPU_ERR_ARG, "invalid argument");
        if (max_candidates == 0 || min_candidates > max_candidates)
            return fail(HNSWGPU_ERR_ARG, "need 0 < max_num_candidates and min_num_candidates <= max_num_candidates");
        if (std::isnan(epsilon)) return fail(HNSWGPU_ERR_ARG, "epsilon is NaN");
        if (nq > 0xffffffffull || max_candidates > 0xffffffffull) return fail(HNSWGPU_ERR_ARG, "batch too large");
        hnswgpu_search_opts o{};
        if (opts) o = *opts;
        if ((o.flags & ~(uint32_t)HNSWGPU_DEVICE_PTRS) || o.precision || o.filter)
            return fail(HNSWGPU_ERR_UNSUPPORTED,
                        "epsilon search: only HNSWGPU_DEVICE_PTRS may be set, float32 only, an allow mask rather "
                        "than a registered filter (it always replays the reference's heaps)");
        const bool dev = (o.flags & HNSWGPU_DEVICE_PTRS) != 0;
        const uint64_t m = max_candidates;
        cudaStream_t st = o.stream ? (cudaStream_t)o.stream : h->stream;
        std::lock_guard<std::mutex> g(h->mu);
        set_device(h);
        if (nq == 0) return HNSWGPU_OK;
        if (h->count == 0) {
            if (dev) {
                cuda_check(cudaMemsetAsync(out_counts, 0, nq * 4, st), "cudaMemsetAsync");
                cuda_check(cudaMemsetAsync(out_ids, 0xff, nq * m * 8, st), "cudaMemsetAsync");
                cuda_check(cudaMemsetAsync(out_dists, 0x7f, nq * m * 4, st), "cudaMemsetAsync");
            } else {
                memset(out_counts, 0, nq * 4);
                for (uint64_t i = 0; i < nq * m; i++) {
                    out_ids[i] = ~0ull;
                    out_dists[i] = __builtin_inff();
                }
            }
            return HNSWGPU_OK;
        }
        if (dev) {
            run_epsilon(h, queries, nq, epsilon, min_candidates, m, o.allow, out_ids, out_dists, out_counts, st);
            return HNSWGPU_OK;
        }
        const size_t qb = nq * h->dim * 4, lb = nq * m * 8, db = nq * m * 4, cb = nq * 4;
        auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
        h->io.ensure(al(qb) + al(lb) + al(db) + al(cb));
        unsigned char* base = h->io.p;
        float* dq = (float*)base;
        uint64_t* dl = (uint64_t*)(base + al(qb));
        float* dd = (float*)(base + al(qb) + al(lb));
        int32_t* dc = (int32_t*)(base + al(qb) + al(lb) + al(db));
        const uint8_t* dallow = nullptr;
        if (o.allow) {
            h->allow.ensure(h->count);
            cuda_check(cudaMemcpyAsync(h->allow.p, o.allow, h->count, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
            dallow = h->allow.p;
        }
        cuda_check(cudaMemcpyAsync(dq, queries, qb, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
        run_epsilon(h, dq, nq, epsilon, min_candidates, m, dallow, dl, dd, dc, st);
        cuda_check(cudaMemcpyAsync(out_ids, dl, lb, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        cuda_check(cudaMemcpyAsync(out_dists, dd, db, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        cuda_check(cudaMemcpyAsync(out_counts, dc, cb, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        uint32_t status = 0;
        cuda_check(cudaMemcpyAsync(&status, h->status.p, 4, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        if (status & HNSWGPU_STATUS_TIMEOUT) {
            cudaMemsetAsync(h->status.p, 0, 4, st);
            cudaStreamSynchronize(st);
            return fail(HNSWGPU_ERR_KERNEL, "search kernel timed out waiting for a copy");
        }
        return HNSWGPU_OK;
    });
}

int hnswgpu_search_noalloc(const hnswgpu_index* h, const float* d_queries, uint64_t nq, uint64_t k, uint64_t ef,
                           uint32_t flags, const uint8_t* d_allow, uint64_t* d_labels, float* d_dists,
                           int32_t* d_counts, void* stream) {
    return guarded([&] {
        if (!h || h->is_bf) return fail(HNSWGPU_ERR_ARG, "hnswgpu_search_noalloc needs an HNSW index");
        if (k == 0 || (nq && (!d_queries || !d_labels || !d_dists || !d_counts)))
            return fail(HNSWGPU_ERR_ARG, "invalid argument");
        // The fixed scratch holds one 32-bit work counter: it hands out query
        // indices, so a call may carry at most 2^31 - 1 queries.
        if (nq > 0x7fffffffull)
            return fail(HNSWGPU_ERR_ARG, "hnswgpu_search_noalloc: nq must be < 2^31 (fixed 256-byte scratch)");
        if (k > 0xffffffffull) return fail(HNSWGPU_ERR_ARG, "hnswgpu_search_noalloc: k must be < 2^32");
        if (flags & ~(uint32_t)HNSWGPU_EXACT_TIES)
            return fail(HNSWGPU_ERR_ARG, "hnswgpu_search_noalloc: only HNSWGPU_EXACT_TIES may be set");
        // the index must not change (set_ef, mark_deleted, ...) while the
        // launch parameters are read from it
        std::lock_guard<std::mutex> g(h->mu);
        cuda_check(cudaSetDevice(h->device), "cudaSetDevice");
        if (nq == 0) return HNSWGPU_OK;
        cudaStream_t st = (cudaStream_t)stream;
        if (h->count == 0) {
            cuda_check(cudaMemsetAsync(d_counts, 0, nq * 4, st), "cudaMemsetAsync");
            cuda_check(cudaMemsetAsync(d_labels, 0xff, nq * k * 8, st), "cudaMemsetAsync");
            cuda_check(cudaMemsetAsync(d_dists, 0x7f, nq * k * 4, st), "cudaMemsetAsync");
            return HNSWGPU_OK;
        }
        uint32_t* scratch = nullptr;
        cuda_check(hnswgpu::noalloc_scratch_address(h->device, &scratch), "cudaGetSymbolAddress");
        hnswgpu::SearchParams p = hnsw_params(h, d_queries, nq, k, ef ? ef : h->ef, d_allow, d_labels, d_dists,
                                              d_counts, nullptr, (flags & HNSWGPU_EXACT_TIES) != 0);
        p.work_counter = scratch + 0;
        p.done_counter = scratch + 1;
        p.status = scratch + 2;
        // the two counters must start at zero: clear what a previous call (or
        // an interrupted one) may have left; the status word is left alone, so
        // that its bits accumulate until hnswgpu_noalloc_get_status reads them
        cuda_check(cudaMemsetAsync(scratch, 0, 2 * sizeof(uint32_t), st), "cudaMemsetAsync");
        cuda_check(hnswgpu::launch_hnsw_search(p, kspace(h), h->num_sms, st, nullptr),
                   "hnsw_search launch");
        return HNSWGPU_OK;
    });
}

int hnswgpu_noalloc_get_status(int device, void* stream, uint32_t* out_bits) {
    return guarded([&] {
        if (!out_bits) return fail(HNSWGPU_ERR_ARG, "invalid argument");
        cuda_check(cudaSetDevice(device), "cudaSetDevice");
        uint32_t* scratch = nullptr;
        cuda_check(hnswgpu::noalloc_scratch_address(device, &scratch), "cudaGetSymbolAddress");
        cudaStream_t st = (cudaStream_t)stream;
        uint32_t v = 0;
        // ordered after the searches queued on `stream`; the copy into
        // pageable host memory allocates nothing
        cuda_check(cudaMemcpyAsync(&v, scratch + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, st),
                   "cudaMemcpyAsync");
        cuda_check(cudaMemsetAsync(scratch + 2, 0, sizeof(uint32_t), st), "cudaMemsetAsync");
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        *out_bits = v;
        return HNSWGPU_OK;
    });
}

int hnswgpu_selftest_wait_timeout(int device, uint32_t* out_bits) {
    return guarded([&] {
        if (!out_bits) return fail(HNSWGPU_ERR_ARG, "invalid argument");
        cuda_check(cudaSetDevice(device), "cudaSetDevice");
        DevBuf<uint32_t> st;
        st.alloc(1);
        cuda_check(cudaMemset(st.p, 0, 4), "cudaMemset");
        // 64 tries of at most 50 us each: the wait gives up within ~3 ms
        cuda_check(hnswgpu::launch_wait_timeout_selftest(64, st.p, nullptr), "selftest launch");
        cuda_check(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
        uint32_t v = 0;
        cuda_check(cudaMemcpy(&v, st.p, 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
        *out_bits = v;
        return HNSWGPU_OK;
    });
}

int hnswgpu_fp64_distances(hnswgpu_index* h, const float* queries, uint64_t nq, const uint64_t* labels, uint64_t m,
                           double* out) {
    return guarded([&] {
        if (!h || (nq && m && (!queries || !labels || !out))) return fail(HNSWGPU_ERR_ARG, "invalid argument");
        if (m > 0xffffffffull) return fail(HNSWGPU_ERR_ARG, "too many rows per query");
        std::lock_guard<std::mutex> g(h->mu);
        set_device(h);
        if (!nq || !m) return HNSWGPU_OK;
        std::vector<uint32_t> rows(nq * m);
        for (uint64_t i = 0; i < nq * m; i++) {
            auto it = h->lookup.find(labels[i]);
            rows[i] = it == h->lookup.end() ? 0xffffffffu : it->second;
        }
        DevBuf<float> dq;
        DevBuf<uint32_t> dr;
        DevBuf<double> dout;
        dq.alloc(nq * h->dim);
        dr.alloc(nq * m);
        dout.alloc(nq * m);
        cuda_check(cudaMemcpyAsync(dq.p, queries, nq * h->dim * 4, cudaMemcpyHostToDevice, h->stream), "cudaMemcpyAsync");
        cuda_check(cudaMemcpyAsync(dr.p, rows.data(), nq * m * 4, cudaMemcpyHostToDevice, h->stream), "cudaMemcpyAsync");
        cuda_check(hnswgpu::launch_fp64_distances(dq.p, nq, (uint32_t)m, (uint32_t)h->dim, h->vecs.p, h->row_floats, dr.p,
                                                  kspace(h),
                                                  h->space == HNSWGPU_SPACE_COSINE ? 1 : 0, dout.p, h->stream),
                   "fp64 distance launch");
        cuda_check(cudaMemcpyAsync(out, dout.p, nq * m * 8, cudaMemcpyDeviceToHost, h->stream), "cudaMemcpyAsync");
        cuda_check(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
        return HNSWGPU_OK;
    });
}

int hnswgpu_set_termination_model(hnswgpu_index* h, const float* params, uint32_t period, float logit_threshold) {
    return guarded([&] {
        if (!h || h->is_bf) return fail(HNSWGPU_ERR_ARG, "a termination model needs an HNSW index");
        std::lock_guard<std::mutex> g(h->mu);
        set_device(h);
        if (!params) {
            cuda_check(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
            h->term_model.release();
            return HNSWGPU_OK;
        }
        if (period == 0) return fail(HNSWGPU_ERR_ARG, "period must be > 0");
        for (int i = 0; i < hnswgpu::kTermParams; i++)
            if (!std::isfinite(params[i])) return fail(HNSWGPU_ERR_ARG, "termination model has non-finite values");
        std::vector<unsigned char> packed(hnswgpu::kTermPackedBytes);
        hnswgpu::pack_term_model(params, packed.data());
        h->term_model.ensure(packed.size());
        // ordered after every search already queued on the index's stream
        cuda_check(cudaMemcpyAsync(h->term_model.p, packed.data(), packed.size(), cudaMemcpyHostToDevice, h->stream),
                   "cudaMemcpyAsync");
        cuda_check(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
        h->term_period = period;
        h->term_logit = logit_threshold;
        return HNSWGPU_OK;
    });
}

int hnswgpu_search_checkpoints(hnswgpu_index* h, const float* queries, uint64_t nq, uint64_t k,
                               const hnswgpu_search_opts* opts, uint32_t period, uint32_t max_ckpt,
                               uint32_t ids_width, float* out_feat, uint32_t* out_ids, float* out_ckpt_dists,
                               uint32_t* out_nckpt, uint64_t* out_labels, float* out_dists, int32_t* out_counts) {
    return guarded([&] {
        if (!h || h->is_bf || k == 0 || period == 0)
            return fail(HNSWGPU_ERR_ARG, "invalid argument");
        if (nq && (!queries || !out_labels || !out_dists || !out_counts || !out_nckpt ||
                   (max_ckpt && (!out_feat || !out_ids))))
            return fail(HNSWGPU_ERR_ARG, "invalid argument");
        if (nq > 0xffffffffull || k > 0xffffffffull) return fail(HNSWGPU_ERR_ARG, "batch too large");
        const uint64_t w = ids_width ? ids_width : k;
        if (w < k || w > 4096) return fail(HNSWGPU_ERR_ARG, "ids_width must be 0 or in [k, 4096]");
        hnswgpu_search_opts o{};
        if (opts) o = *opts;
        if (o.flags & ~(uint32_t)HNSWGPU_TRACE)
            return fail(HNSWGPU_ERR_ARG, "hnswgpu_search_checkpoints: host pointers and the id tie order only");
        std::lock_guard<std::mutex> g(h->mu);
        set_device(h);
        if (nq == 0 || h->count == 0) return fail(HNSWGPU_ERR_ARG, "empty batch or index");
        const uint64_t ef = o.ef ? o.ef : h->ef;
        cudaStream_t st = o.stream ? (cudaStream_t)o.stream : h->stream;
        const size_t rows = (size_t)nq * max_ckpt;
        DevBuf<float> dq, dd, df, dx;
        DevBuf<uint64_t> dl;
        DevBuf<int32_t> dc;
        DevBuf<uint32_t> di, dn;
        dq.alloc(nq * h->dim);
        dl.alloc(nq * k);
        dd.alloc(nq * k);
        dc.alloc(nq);
        dn.alloc(nq);
        df.alloc(rows * hnswgpu::kTermFeatures);
        di.alloc(rows * w);
        if (out_ckpt_dists) dx.alloc(rows * w);
        cuda_check(cudaMemcpyAsync(dq.p, queries, nq * h->dim * 4, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
        TermCfg term;
        term.mode = 1;
        term.period = period;
        term.max_ckpt = max_ckpt;
        term.feat = df.p;
        term.ids = di.p;
        term.width = (uint32_t)w;
        term.dists = out_ckpt_dists ? dx.p : nullptr;
        term.count = dn.p;
        run_hnsw(h, dq.p, nq, k, ef, nullptr, dl.p, dd.p, dc.p, nullptr, st, false, o.precision, o.rerank, &term,
                 false);
        cuda_check(cudaMemcpyAsync(out_labels, dl.p, nq * k * 8, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        cuda_check(cudaMemcpyAsync(out_dists, dd.p, nq * k * 4, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        cuda_check(cudaMemcpyAsync(out_counts, dc.p, nq * 4, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        cuda_check(cudaMemcpyAsync(out_nckpt, dn.p, nq * 4, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        if (rows) {
            cuda_check(cudaMemcpyAsync(out_feat, df.p, rows * hnswgpu::kTermFeatures * 4, cudaMemcpyDeviceToHost, st),
                       "cudaMemcpyAsync");
            cuda_check(cudaMemcpyAsync(out_ids, di.p, rows * w * 4, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
            if (out_ckpt_dists)
                cuda_check(cudaMemcpyAsync(out_ckpt_dists, dx.p, rows * w * 4, cudaMemcpyDeviceToHost, st),
                           "cudaMemcpyAsync");
        }
        uint32_t status = 0;
        cuda_check(cudaMemcpyAsync(&status, h->status.p, 4, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        if (status & HNSWGPU_STATUS_TIMEOUT) {
            cudaMemsetAsync(h->status.p, 0, 4, st);
            cudaStreamSynchronize(st);
            return fail(HNSWGPU_ERR_KERNEL, "search kernel timed out waiting for a copy");
        }
        return HNSWGPU_OK;
    });
}

int hnswgpu_term_train(int device, const float* feats, const float* labels, uint64_t n,
                       const hnswgpu_term_train_opts* opts, float* params, float* out_epoch_loss) {
    return guarded([&] {
        if (!feats || !labels || !params || !opts || n == 0) return fail(HNSWGPU_ERR_ARG, "invalid argument");
        if (n > 0xffffffffull) return fail(HNSWGPU_ERR_ARG, "too many samples");
        cuda_check(cudaSetDevice(device), "cudaSetDevice");
        cuda_check(hnswgpu::term_train(feats, labels, n, params, opts->epochs, opts->batch, opts->lr,
                                       opts->pos_weight, opts->weight_decay, opts->seed, out_epoch_loss),
                   "termination training");
        return HNSWGPU_OK;
    });
}

int hnswgpu_term_loss_grad(int device, const float* params, const float* feats, const float* labels, uint64_t n,
                           float pos_weight, float* out_loss, float* out_grad) {
    return guarded([&] {
        if (!feats || !labels || !params || !out_loss || !out_grad || n == 0)
            return fail(HNSWGPU_ERR_ARG, "invalid argument");
        cuda_check(cudaSetDevice(device), "cudaSetDevice");
        cuda_check(hnswgpu::term_loss_grad(params, feats, labels, n, pos_weight, out_loss, out_grad),
                   "termination gradient");
        return HNSWGPU_OK;
    });
}

int hnswgpu_term_logits(int device, const float* params, const float* feats, uint64_t n, float* out_logits) {
    return guarded([&] {
        if (!params || (n && (!feats || !out_logits))) return fail(HNSWGPU_ERR_ARG, "invalid argument");
        cuda_check(cudaSetDevice(device), "cudaSetDevice");
        cuda_check(hnswgpu::term_logits(params, feats, n, out_logits), "termination inference");
        return HNSWGPU_OK;
    });
}

int hnswgpu_get_status(hnswgpu_index* h, uint32_t* out_bits) {
    return guarded([&] {
        if (!h || !out_bits) return fail(HNSWGPU_ERR_ARG, "invalid argument");
        std::lock_guard<std::mutex> g(h->mu);
        set_device(h);
        uint32_t v = 0;
        cuda_check(cudaMemcpyAsync(&v, h->status.p, 4, cudaMemcpyDeviceToHost, h->stream), "cudaMemcpyAsync");
        cuda_check(cudaMemsetAsync(h->status.p, 0, 4, h->stream), "cudaMemsetAsync");
        cuda_check(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
        *out_bits = v;
        return HNSWGPU_OK;
    });
}

#ifdef HNSWGPU_BOUNDS_CHECK
// Self-checking builds only: first recorded violation (code, a, b, block).
HNSWGPU_API int hnswgpu_debug_record(unsigned long long* out) {
    cudaDeviceSynchronize();
    if (hnswgpu::read_lean_debug_record(out) != cudaSuccess) return HNSWGPU_ERR_CUDA;
    if (out[0]) return HNSWGPU_OK;
    return hnswgpu::read_debug_record(out) == cudaSuccess ? HNSWGPU_OK : HNSWGPU_ERR_CUDA;
}
#endif

#ifdef HNSWGPU_TC_TIMING
HNSWGPU_API int hnswgpu_tc_timing(unsigned long long* out) {
    return hnswgpu::tc_timing_read(out) == cudaSuccess ? 0 : -4;
}
#endif
#ifdef HNSWGPU_PHASE_TIMING
// Profiling builds only: per-phase cycle totals of all searches since the
// last call (10 counters), cleared on read.
HNSWGPU_API int hnswgpu_phase_cycles(unsigned long long* out) {
    if (!g_phase_buf) return fail(HNSWGPU_ERR_ARG, "no search ran");
    cudaDeviceSynchronize();
    cudaMemcpy(out, g_phase_buf, 10 * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaMemset(g_phase_buf, 0, 10 * sizeof(unsigned long long));
    return HNSWGPU_OK;
}
#endif

}  // extern "C"
