// Multi-vector search on B200 (sm_100a): searchStopConditionClosest with a
// MultiVectorSearchStopCondition (hnswlib/hnswalg.h:1326-1377,
// hnswlib/stop_condition.h:146-216) over an index of a MultiVectorL2Space,
// whose elements carry a 32-bit document id right after the vector.
//
// One warp per query.  The warp computes the distances in parallel (one lane
// per neighbour, the reference's float32 summation order) and keeps the
// visited set exact (an open-addressing hash set in shared memory, so no node
// is ever evaluated twice, as the reference's visited list guarantees); lane 0
// replays, operation by operation, the reference's three heaps --
// top_candidates and candidate_set (CompareByFirst, hnswalg.h:165-170) and the
// condition's own max-heap of (distance, document) pairs -- and its per-
// document counter (a hash table in shared memory).  The loop's size tests
// count distinct documents (curr_num_docs against ef_collection =
// max(ef_collection, num_docs)); each eviction from top_candidates pops the
// condition's heap; at the end filter_results pops it again and trims the
// result until num_docs documents remain.  The result holds internal ids, as
// the reference's does.
//
// Capacities (top_candidates and the condition's heap: top_cap entries;
// candidate_set: 2 top_cap; documents: 2^doc_log2; visited nodes:
// 2^vis_log2) are fixed per launch; a query that outgrows one stops and
// raises HNSWGPU_STATUS_OVERFLOW_BIT.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "device_common.cuh"
#include "hnsw_multivec.h"
#include "ref_heap.h"

namespace hnswgpu {

namespace {

constexpr uint32_t kEmpty = 0xffffffffu;

// std::pair<float, unsigned int>'s order on (distance key << 32 | document).
struct PairLess {
    __device__ __forceinline__ bool operator()(uint64_t a, uint64_t b) const { return a < b; }
};

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// Slot of document `doc` in the counter table (keys kEmpty when free), or
// -1 when the table is full.
__device__ __forceinline__ int doc_slot(uint32_t* keys, uint32_t mask, uint32_t doc) {
    uint32_t h = mix32(doc) & mask;
    for (uint32_t probe = 0; probe <= mask; probe++) {
        if (keys[h] == doc) return (int)h;
        if (keys[h] == kEmpty) {
            keys[h] = doc;
            return (int)h;
        }
        h = (h + 1) & mask;
    }
    return -1;
}

struct MvSmem {
    float* q;
    float* d;         // distances of one expansion's neighbours (link order)
    uint32_t* nid;    // their ids; INVALID_ID when already visited
    uint64_t* top;
    uint64_t* cand;
    uint64_t* res;    // the condition's (distance, document) heap
    uint32_t* dkeys;  // document counter: keys
    uint32_t* dcnt;   //                    counts
    uint32_t* vis;    // visited node ids (hash set)
};

// Exact visited test-and-set of distinct ids by the lanes that hold one:
// true when the id was not visited yet.  `full` is set when the set is full.
__device__ __forceinline__ bool vis_claim(uint32_t* vis, uint32_t mask, uint32_t id, bool& full) {
    uint32_t h = mix32(id) & mask;
    for (uint32_t probe = 0; probe <= mask; probe++) {
        const uint32_t old = atomicCAS(vis + h, kEmpty, id);
        if (old == kEmpty) return true;
        if (old == id) return false;
        h = (h + 1) & mask;
    }
    full = true;
    return false;
}

__device__ void mv_search(const MvParams& p, const MvSmem& s, uint32_t qi, int lane) {
    const int dim = (int)p.dim;
    const float* qg = p.queries + (size_t)qi * p.dim;
    for (int i = lane; i < (int)p.row_floats; i += 32) s.q[i] = i < dim ? qg[i] : 0.f;
    const uint32_t vmask = (1u << p.vis_log2) - 1, dmask = (1u << p.doc_log2) - 1;
    for (uint32_t i = lane; i <= vmask; i += 32) s.vis[i] = kEmpty;
    for (uint32_t i = lane; i <= dmask; i += 32) {
        s.dkeys[i] = kEmpty;
        s.dcnt[i] = 0;
    }
    __syncwarp();
    auto row = [&](uint32_t id) { return p.vecs + (size_t)id * p.row_floats; };

    // ---- upper-layer greedy descent (hnswalg.h:1274-1302), exact distances
    uint32_t cur = p.ep;
    float curd = dist_l2(s.q, row(cur), dim);
    for (int level = p.maxlevel; level > 0; level--) {
        while (true) {
            const uint32_t* lr = p.upper_links + (size_t)(p.upper_off[cur] + (uint32_t)(level - 1)) * (p.maxM + 1);
            const int cnt = (int)(lr[0] & 0xffffu);
            float best = curd;
            uint32_t best_id = INVALID_ID;
            for (int c0 = 0; c0 < cnt; c0 += 32) {
                const int n = min(32, cnt - c0);
                const uint32_t id = lane < n ? lr[1 + c0 + lane] : INVALID_ID;
                float d = lane < n ? dist_l2(s.q, row(id), dim) : __int_as_float(0x7f800000);
                float m = d;
#pragma unroll
                for (int o = 16; o; o >>= 1) m = fminf(m, __shfl_xor_sync(FULL, m, o));
                if (m < best) {
                    const unsigned hit = __ballot_sync(FULL, lane < n && d == m);
                    best = m;
                    best_id = __shfl_sync(FULL, id, __ffs(hit) - 1);
                }
            }
            if (best_id == INVALID_ID) break;
            cur = best_id;
            curd = best;
        }
    }

    // ---- level-0 loop of searchStopConditionClosest (lane 0 replays the heaps)
    const uint32_t ef_coll = max(p.ef_coll, p.num_docs);
    const int tcap = (int)p.top_cap, ccap = 2 * (int)p.top_cap;
    int tn = 0, cn = 0, rn = 0;          // heap sizes (lane 0)
    uint32_t cur_docs = 0;
    float lb = curd;
    bool overflow = false;
    // add_point / remove_point of the condition (stop_condition.h:160-182)
    auto add_point = [&](uint32_t id, float d) {
        const uint32_t doc = p.docs[id];
        const int sl = doc_slot(s.dkeys, dmask, doc);
        if (sl < 0 || rn >= tcap) {
            overflow = true;
            return;
        }
        if (s.dcnt[sl]++ == 0) cur_docs++;
        ref_heap_push(s.res, rn, ((uint64_t)fkey(d) << 32) | doc, PairLess());
    };
    auto remove_point = [&](uint32_t id) {
        const int sl = doc_slot(s.dkeys, dmask, p.docs[id]);
        if (sl >= 0 && --s.dcnt[sl] == 0) cur_docs--;
        ref_heap_pop(s.res, rn, PairLess());
    };
    bool full = false;
    if (lane == 0) {
        vis_claim(s.vis, vmask, cur, full);
        ref_heap_push(s.top, tn, mkkey(curd, cur), TopLess());
        add_point(cur, curd);
        ref_heap_push(s.cand, cn, mkkey(curd, cur), CandLess());
    }
    __syncwarp();
    uint32_t expansions = 0;
    while (true) {
        uint32_t c = INVALID_ID;
        int go = 0;
        if (lane == 0 && cn > 0 && !overflow) {
            const uint64_t cp = s.cand[0];
            const float cd = funkey((uint32_t)(cp >> 32));
            if (!(cd > lb && cur_docs == ef_coll)) {
                ref_heap_pop(s.cand, cn, CandLess());
                c = kid(cp);
                go = 1;
            }
        }
        if (!__shfl_sync(FULL, go, 0)) break;
        c = __shfl_sync(FULL, c, 0);
        if (++expansions > p.max_expansions) {
            overflow = true;
            break;
        }
        // neighbours in link order, two slots per lane
        const uint32_t* ll = p.links0 + (size_t)c * p.maxM0;
        bool vfull = false;
        for (int h = 0; h < 2; h++) {
            const int j = lane + 32 * h;
            const uint32_t id = j < (int)p.maxM0 ? ll[j] : INVALID_ID;
            bool fresh = id != INVALID_ID;
            const unsigned peers = __match_any_sync(FULL, id);
            fresh = fresh && __ffs(peers) - 1 == lane;  // a repeated id: its first slot
            // a repeat across the two slot sets: the second one yields
            if (h == 1 && fresh) {
                for (int t = 0; t < 32 && fresh; t++)
                    if (s.nid[t] == id && t < (int)p.maxM0) fresh = false;
            }
            if (fresh) fresh = vis_claim(s.vis, vmask, id, vfull);
            s.nid[j] = fresh ? id : INVALID_ID;
            s.d[j] = fresh ? dist_l2(s.q, row(id), dim) : 0.f;
            __syncwarp();
        }
        if (__any_sync(FULL, vfull)) overflow = true;
        if (lane == 0 && !overflow) {
            for (int j = 0; j < (int)p.maxM0 && j < 64; j++) {
                const uint32_t id = s.nid[j];
                if (id == INVALID_ID) continue;
                const float d = s.d[j];
                if (cur_docs < ef_coll || lb > d) {
                    if (cn >= ccap || tn >= tcap) {
                        overflow = true;
                        break;
                    }
                    ref_heap_push(s.cand, cn, mkkey(d, id), CandLess());
                    ref_heap_push(s.top, tn, mkkey(d, id), TopLess());
                    add_point(id, d);
                    while (cur_docs > ef_coll && tn > 0) {
                        const uint32_t gone = kid(ref_heap_pop(s.top, tn, TopLess()));
                        remove_point(gone);
                    }
                    if (tn > 0) lb = funkey((uint32_t)(s.top[0] >> 32));
                }
            }
        }
        overflow = __shfl_sync(FULL, (int)overflow, 0) != 0;
        __syncwarp();
    }
    // ---- result: top_candidates popped closest first, then filter_results
    if (lane == 0) {
        int n = tn;
        uint64_t* out = s.cand;  // idle now; at least tn entries
        for (int i = tn - 1; i >= 0; i--) out[i] = ref_heap_pop(s.top, n, TopLess());
        int rsz = tn;
        while (cur_docs > p.num_docs && rsz > 0 && rn > 0) {
            const uint32_t doc = (uint32_t)s.res[0];
            const int sl = doc_slot(s.dkeys, dmask, doc);
            if (sl >= 0 && --s.dcnt[sl] == 0) cur_docs--;
            ref_heap_pop(s.res, rn, PairLess());
            rsz--;
        }
        const int kept = rsz <= (int)p.cap ? rsz : -1;
        uint64_t* oid = p.out_ids + (size_t)qi * p.cap;
        float* od = p.out_dists + (size_t)qi * p.cap;
        for (int i = 0; i < (int)p.cap; i++) {
            const bool have = i < rsz;
            oid[i] = have ? (uint64_t)kid(out[i]) : ~0ull;
            od[i] = have ? funkey((uint32_t)(out[i] >> 32)) : __int_as_float(0x7f800000);
        }
        p.out_counts[qi] = overflow ? -1 : kept;
        if (overflow) atomicOr(p.status, HNSWGPU_STATUS_OVERFLOW_BIT);
    }
    __syncwarp();
}

__global__ void __launch_bounds__(32) hnsw_multivec_kernel(MvParams p) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    MvSmem s;
    unsigned char* b = smem;
    s.top = reinterpret_cast<uint64_t*>(b);
    b += (size_t)p.top_cap * 8;
    s.cand = reinterpret_cast<uint64_t*>(b);
    b += (size_t)p.top_cap * 16;
    s.res = reinterpret_cast<uint64_t*>(b);
    b += (size_t)p.top_cap * 8;
    s.d = reinterpret_cast<float*>(b);
    b += 64 * 4;
    s.nid = reinterpret_cast<uint32_t*>(b);
    b += 64 * 4;
    s.dkeys = reinterpret_cast<uint32_t*>(b);
    b += ((size_t)4 << p.doc_log2);
    s.dcnt = reinterpret_cast<uint32_t*>(b);
    b += ((size_t)4 << p.doc_log2);
    s.vis = reinterpret_cast<uint32_t*>(b);
    b += ((size_t)4 << p.vis_log2);
    s.q = reinterpret_cast<float*>(b);
    for (uint32_t qi = blockIdx.x; qi < p.nq; qi += gridDim.x) mv_search(p, s, qi, lane);
}

}  // namespace

size_t multivec_smem(const MvParams& p) {
    return (size_t)p.top_cap * 32 + 64 * 8 + ((size_t)8 << p.doc_log2) + ((size_t)4 << p.vis_log2) +
           (size_t)p.row_floats * 4;
}

cudaError_t launch_hnsw_multivec(const MvParams& p, int num_sms, cudaStream_t stream) {
    const size_t smem = multivec_smem(p);
    cudaError_t e = cudaFuncSetAttribute(hnsw_multivec_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const unsigned blocks = (unsigned)std::min<uint64_t>(p.nq, (uint64_t)num_sms * 2);
    if (blocks == 0) return cudaSuccess;
    hnsw_multivec_kernel<<<blocks, 32, smem, stream>>>(p);
    return cudaGetLastError();
}

}  // namespace hnswgpu
