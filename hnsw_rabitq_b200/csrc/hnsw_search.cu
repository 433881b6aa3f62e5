// Batched HNSW k-NN search on B200 (sm_100a): one warp per query.
//
// Replaces HierarchicalNSW::searchKnn (hnswlib/hnswalg.h:1269-1323) and its
// level-0 beam searchBaseLayerST (hnswlib/hnswalg.h:308-440) for a whole
// batch of queries in one launch.
//
// Per warp (= per query in flight) the shared memory holds
//   * the query row,
//   * a staging area that TMA bulk copies fill with the neighbour vectors of
//     the node being expanded (one 16-byte aligned row per neighbour),
//   * the candidate pool: up to ef (distance, id) keys sorted ascending, each
//     with an "expanded" flag -- it plays the role of both of the reference's
//     heaps (top_candidates and candidate_set, hnswalg.h:321-322),
//   * for filtered / delete-aware searches, a second sorted list of accepted
//     nodes that may not be returned (deleted or rejected by the filter) but
//     must still be expanded (hnswalg.h:398-412),
//   * a direct-mapped visited cache of node ids that replaces the
//     VisitedListPool (hnswlib/visited_list_pool.h).
//
// Exactness.  The warp evaluates all neighbours of one expansion in parallel
// and then applies the reference's sequential acceptance test
// (`top.size() < ef || lowerBound > dist`, hnswalg.h:395, neighbours in link
// order) in closed form: neighbour j is accepted iff
//     #{pool entries with d <= d_j} + #{earlier allowed neighbours with d <= d_j} < ef,
// which equals the sequential test because lowerBound after the earlier
// insertions is the ef-th smallest distance among the pool and the earlier
// neighbours.  A node that misses in the visited cache but was seen before is
// either still in the pool / second list (found by exact key lookup and
// skipped) or has d >= lowerBound and is rejected again, so cache misses cost
// only a repeated distance, never a different result.  Ties in distance are
// broken by internal id; on the same index the kernel therefore returns the
// reference's labels except where distances tie exactly (the oracle's
// "canonical" mode computes exactly this kernel's result).
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>

#include "device_common.cuh"
#include "hnsw_search.h"
#include "launch_cache.h"
#include "ref_heap.h"
#include "term_mlp.cuh"

namespace hnswgpu {

namespace {

struct WarpSmem {
    uint64_t* bar;
    uint32_t* cbuf;      // 32 ids: compaction of one expansion's fresh neighbours
    float* q;
    float* stage;
    uint64_t* pool;
    uint64_t* extra;
    uint32_t* vis;
    uint64_t* topheap;   // tie-exact mode: replay of top_candidates
    SplitHeap candheap;  // tie-exact mode: replay of candidate_set
    int cand_total;      // tie-exact mode: its capacity (shared + spill)
    uint64_t* accbuf;    // tie-exact mode: accepted keys of one chunk, link order
    uint64_t* evbuf;     // tie-exact mode: keys evicted from top_candidates
};

// Optional self-checks (compile with -DHNSWGPU_BOUNDS_CHECK; the shipped
// library is built without them): every staging copy and staged-row read is
// checked against the warp's shared-memory layout and the source buffer; the
// first violation is recorded in g_dbg and the access is skipped (a skipped
// copy completes its bytes on the mbarrier so the wait stays consistent).
#ifdef HNSWGPU_BOUNDS_CHECK
__device__ unsigned long long g_dbg[8];
__device__ __forceinline__ bool dbg_ok(bool cond, unsigned code, unsigned long long a, unsigned long long b) {
    if (cond) return true;
    if (atomicCAS(&g_dbg[0], 0ull, (unsigned long long)code) == 0ull) {
        g_dbg[1] = a;
        g_dbg[2] = b;
        g_dbg[3] = blockIdx.x;
    }
    return false;
}
__device__ __forceinline__ void mbar_complete_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.complete_tx.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
#define DBG_OK(cond, code, a, b) dbg_ok((cond), (code), (unsigned long long)(a), (unsigned long long)(b))
#else
#define DBG_OK(cond, code, a, b) true
#endif

// Staging copy with the optional checks: dst must lie in this warp's staging
// region [stage, pool), src inside [base, base + nrows * row_bytes).
__device__ __forceinline__ void stage_copy(const SearchParams& p, const WarpSmem& s, void* dst, const void* base,
                                           uint64_t row, uint64_t nrows, uint32_t row_bytes, unsigned code) {
#ifdef HNSWGPU_BOUNDS_CHECK
    const unsigned char* dp = static_cast<const unsigned char*>(dst);
    const unsigned char* lo = reinterpret_cast<const unsigned char*>(s.stage);
    const unsigned char* hi = reinterpret_cast<const unsigned char*>(s.pool);
    const bool ok = DBG_OK(dp >= lo && dp + row_bytes <= hi && ((uintptr_t)dp & 15) == 0 && (row_bytes & 15) == 0,
                           code, dp - lo, row_bytes) &&
                    DBG_OK(row < nrows, code + 1, row, nrows);
#else
    const bool ok = true;
#endif
    if (ok) {
        bulk_g2s(dst, static_cast<const unsigned char*>(base) + row * row_bytes, row_bytes, s.bar);
    } else {
#ifdef HNSWGPU_BOUNDS_CHECK
        mbar_complete_tx(s.bar, row_bytes);
#endif
    }
}

__device__ __forceinline__ bool is_allowed(const SearchParams& p, uint32_t id) {
    if (p.deleted_bits && ((p.deleted_bits[id >> 5] >> (id & 31)) & 1u)) return false;
    if (p.allow && !p.allow[id]) return false;
    return true;
}

// Count of entries of the sorted array with (key & KEY_MASK) < key.
__device__ __forceinline__ int lower_bound_key(const uint64_t* a, int n, uint64_t key) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if ((a[mid] & KEY_MASK) < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}
// Count of entries whose distance key is <= dk.
__device__ __forceinline__ int upper_bound_hi(const uint64_t* a, int n, uint32_t dk) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (khi(a[mid]) <= dk) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Insertion position of `key` (distance key dk, node id) in the sorted array
// given cnt = upper_bound_hi(a, n, dk), walking back over the (rare) entries
// that tie in distance.  Sets dup when the key is already present.
__device__ __forceinline__ int insert_pos(const uint64_t* a, int cnt, uint32_t dk, uint32_t id, bool& dup) {
    int pos = cnt;
    while (pos > 0) {
        uint64_t e = a[pos - 1];
        if (khi(e) != dk) break;
        uint32_t eid = kid(e);
        if (eid == id) {
            dup = true;
            break;
        }
        if (eid < id) break;
        pos--;
    }
    return pos;
}

// Remove the nev (<= 32) distinct keys ev[0..nev) (all present) from the
// sorted array a[0, size), keeping the order of the rest.
__device__ __forceinline__ void remove_keys(uint64_t* a, int& size, const uint64_t* ev, int nev, int lane) {
    int myidx = lane < nev ? lower_bound_key(a, size, ev[lane] & KEY_MASK) : 0x7fffffff;
    int minidx = myidx;
#pragma unroll
    for (int o = 16; o; o >>= 1) minidx = min(minidx, __shfl_xor_sync(FULL, minidx, o));
    for (int base = minidx; base < size; base += 32) {
        int i = base + lane;
        bool have = i < size;
        uint64_t e = have ? a[i] : 0;
        int before = 0;
        bool gone = false;
        for (int t = 0; t < nev; t++) {
            int it = __shfl_sync(FULL, myidx, t);
            before += (it < i);
            gone |= (it == i);
        }
        __syncwarp();
        if (have && !gone) a[i - before] = e;
        __syncwarp();
    }
    size -= nev;
}

// First unexpanded entry at index >= hint, or -1.  Updates hint.
__device__ __forceinline__ int find_unexpanded(const uint64_t* a, int n, int& hint, int lane) {
    for (int b = hint; b < n; b += 32) {
        int i = b + lane;
        bool u = i < n && !((uint32_t)a[i] & EXP_BIT);
        unsigned m = __ballot_sync(FULL, u);
        if (m) {
            hint = b + __ffs(m) - 1;
            return hint;
        }
    }
    hint = n;
    return -1;
}

// Unexpanded entries of the sorted array a[from, n) whose distance key is dk,
// where a[from] is the first unexpanded entry (so all such entries follow it).
__device__ __forceinline__ int unexpanded_with_dist(const uint64_t* a, int n, int from, uint32_t dk, int lane) {
    int c = 0;
    for (int b = from; b < n; b += 32) {
        const int i = b + lane;
        const uint64_t e = i < n ? a[i] : ~0ull;
        const bool same = i < n && khi(e) == dk;
        c += __popc(__ballot_sync(FULL, same && !((uint32_t)e & EXP_BIT)));
        if (!__shfl_sync(FULL, same, 31)) break;
    }
    return c;
}

// Insert the keys held by the lanes of `amask` (distinct, not present in the
// array; `pos` = lower_bound_key of the lane's key) into the sorted array a[0,
// size), keeping at most cap entries.  Returns the smallest insertion index.
__device__ __forceinline__ int merge_sorted(uint64_t* a, int& size, int cap, unsigned amask, uint64_t key, int pos,
                                            int lane) {
    // `key` may carry EXP_BIT (inserted already expanded); order ignores it
    const uint64_t kc = key & KEY_MASK;
    int na = __popc(amask);
    bool mine = (amask >> lane) & 1u;
    int rank = 0;
    for (unsigned m = amask; m; m &= m - 1) {
        int src = __ffs(m) - 1;
        uint64_t k2 = shfl64(kc, src);
        rank += (k2 < kc);
    }
    const int mpos = (int)__reduce_min_sync(FULL, mine ? (unsigned)pos : 0x7fffffffu);
    if (size > mpos) {
        // Move the entries [mpos, size) right, last chunk first.
        int nmove = size - mpos;
        for (int base = mpos + ((nmove - 1) & ~31); base >= mpos; base -= 32) {
            int i = base + lane;
            bool have = i < size;
            uint64_t e = have ? a[i] : 0;
            uint64_t em = e & KEY_MASK;
            int sh = 0;
            for (unsigned m = amask; m; m &= m - 1) {
                int src = __ffs(m) - 1;
                uint64_t k2 = shfl64(kc, src);
                sh += (k2 < em);
            }
            __syncwarp();
            if (have && i + sh < cap) a[i + sh] = e;
            __syncwarp();
        }
    }
    int np = pos + rank;
    if (mine && np < cap) a[np] = key;
    __syncwarp();
    size = min(size + na, cap);
    return mpos;
}

// Stage the rows of up to `cnt` nodes into stage slots [0, cnt): lane `slot`
// ... the calling lane copies row `id` into slot `slot` when `mine`.
__device__ __forceinline__ bool stage_rows(const SearchParams& p, WarpSmem& s, uint32_t& phase, bool mine,
                                           uint32_t id, int slot, int cnt, int lane) {
    if (cnt == 0) return true;
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0) mbar_arrive_expect_tx(s.bar, (uint32_t)cnt * p.row_bytes);
    __syncwarp();
    if (mine) stage_copy(p, s, s.stage + (size_t)slot * p.stage_stride, p.vecs, id, p.count, p.row_bytes, 10);
    bool ok = mbar_wait(s.bar, phase);
    phase ^= 1u;
    return __all_sync(FULL, ok);
}

template <int SPACE>
__device__ __forceinline__ float stage_dist(const SearchParams& p, const WarpSmem& s, int slot) {
    return distance<SPACE>(s.q, s.stage + (size_t)slot * p.stage_stride, (int)p.dim);
}

struct Counters {
    uint32_t upper_hops, upper_dists, l0_exp, l0_dists;
};



// Optional per-phase cycle accounting (compile with -DHNSWGPU_PHASE_TIMING;
// the shipped library is built without it).  Phases: 0 query setup,
// 1 upper-layer descent, 2 candidate selection, 3 link row + visited cache,
// 4 staging wait, 5 distance arithmetic, 6 acceptance, 7 heap replay,
// 8 pool / list maintenance, 9 result output.
#ifdef HNSWGPU_PHASE_TIMING
struct PhaseClock {
    long long last = 0;
    long long acc[10] = {0};
    __device__ void start() { last = clock64(); }
    __device__ void mark(int i) {
        long long t = clock64();
        acc[i] += t - last;
        last = t;
    }
};
#define PT_MARK(i) pc.mark(i)
#else
struct PhaseClock {
    __device__ void start() {}
    __device__ void mark(int) {}
};
#define PT_MARK(i)
#endif

// Distances of `cnt` (<= 32) nodes held by lanes [0, cnt) (id per lane);
// result returned in the owning lane.  False on a wait timeout.
// Rows are staged `stage_slots` at a time.  For dim % 16 == 0 each group of
// 4 lanes evaluates one staged row (8 rows per pass, group4_dist16); other
// dimensions use one lane per row with the scalar-order routine.
template <int SPACE, bool FAST16>
__device__ __forceinline__ bool lane_distances(const SearchParams& p, WarpSmem& s, uint32_t& phase, uint32_t id,
                                               int cnt, int lane, float& d, PhaseClock& pc) {
    d = __int_as_float(0x7f800000);
    for (int s0 = 0; s0 < cnt; s0 += (int)p.stage_slots) {
        const int n = min((int)p.stage_slots, cnt - s0);
        const bool mine = lane >= s0 && lane < s0 + n;
        if (!stage_rows(p, s, phase, mine, id, lane - s0, n, lane)) return false;
        PT_MARK(4);
        if (FAST16) {
            const int a = lane & 3;
            for (int g = 0; g < n; g += 8) {
                const int v = min(g + (lane >> 2), n - 1);
                float r = group4_dist16<SPACE>(s.q, s.stage + (size_t)v * p.stage_stride, (int)(p.dim >> 4), a);
                const int rel = lane - s0 - g;  // this lane's row within the pass
                float got = __shfl_sync(FULL, r, (rel & 7) << 2);
                if (rel >= 0 && rel < 8 && mine) d = got;
            }
        } else {
            float dt = lane < n ? stage_dist<SPACE>(p, s, lane) : 0.f;
            float got = __shfl_sync(FULL, dt, (lane - s0) & 31);
            if (mine) d = got;
        }
        PT_MARK(5);
    }
    return true;
}

// ------------------------------------------------------------------------
// Pipelined level-0 beam for dim % 16 == 0 and maxM0 <= 32 (with deletes or a
// filter in the id tie order only).  Same decisions as the general loop; the
// difference is scheduling: as soon as the acceptance of the current
// expansion is known, the next candidate is fixed (id tie order: the first
// unexpanded of pool + accepted; tie-exact order: the candidate heap's top,
// predicted whenever its distance is unique), and its link row, visited-cache
// update and first TMA batch are issued before the pool merge / heap replay
// of the current expansion, which then run under that memory latency.
// Where the rows of one staging batch come from: the float32 rows, or the
// low-precision traversal copy.
struct RowSrc {
    const unsigned char* base;
    uint32_t row_bytes;    // bytes per row in global memory (= bytes copied)
    uint32_t stage_bytes;  // staging stride
    uint32_t slots;        // rows per batch
};

template <int PREC>
__device__ __forceinline__ RowSrc trav_src(const SearchParams& p) {
    if (PREC == 0) return RowSrc{reinterpret_cast<const unsigned char*>(p.vecs), p.row_bytes, p.stage_stride * 4,
                                 p.stage_slots};
    return RowSrc{p.tvecs, p.trow_bytes, p.tstage_bytes, p.tslots};
}

__device__ __forceinline__ bool stage_src(const SearchParams& p, WarpSmem& s, uint32_t& phase, const RowSrc& r,
                                          bool mine, uint32_t id, int slot, int cnt, int lane) {
    if (cnt == 0) return true;
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0) mbar_arrive_expect_tx(s.bar, (uint32_t)cnt * r.row_bytes);
    __syncwarp();
    if (mine)
        stage_copy(p, s, reinterpret_cast<unsigned char*>(s.stage) + (size_t)slot * r.stage_bytes, r.base, id,
                   p.count, r.row_bytes, 20);
    bool ok = mbar_wait(s.bar, phase);
    phase ^= 1u;
    return __all_sync(FULL, ok);
}

struct Fetch {
    uint32_t id;     // this lane's neighbour id (link order), or INVALID_ID
    bool fresh;      // evaluated now (missed in the visited cache)
    unsigned nmask;  // fresh lanes
    int nnew;        // number of fresh lanes
    uint32_t cid2;   // id of the lane-th fresh neighbour (lanes < nnew)
    int n0;          // rows of the first staging batch in flight
    bool allowed;    // FILTER: this lane's neighbour may be returned (not deleted, passes the filter)
};

// FILTER: also read each fresh neighbour's delete bit and filter byte (used
// only after the row gather, so their latency overlaps it) and never admit
// `skip` (a disallowed entry point, never stored with its distance).
template <int PREC, bool FILTER = false>
__device__ __forceinline__ void fetch_links(const SearchParams& p, WarpSmem& s, uint32_t c, int lane, Fetch& f,
                                            uint32_t skip = INVALID_ID) {
    const RowSrc rs = trav_src<PREC>(p);
    const uint32_t* lrow = p.links0 + (size_t)c * p.maxM0;
    const uint32_t id = lane < (int)p.maxM0 ? __ldg(lrow + lane) : INVALID_ID;
    bool fresh = id != INVALID_ID && (!FILTER || id != skip);
    if (!p.links_unique) {
        unsigned peers = __match_any_sync(FULL, id);
        fresh = fresh && (__ffs(peers) - 1 == lane);
    }
    const uint32_t slot = fresh ? vis_slot(id, p.log2_vis) : 0;
    if (fresh && s.vis[slot] == id) fresh = false;
    __syncwarp();
    if (fresh) s.vis[slot] = id;
    f.id = id;
    f.fresh = fresh;
    f.allowed = !FILTER || !fresh || is_allowed(p, id);
    f.nmask = __ballot_sync(FULL, fresh);
    f.nnew = __popc(f.nmask);
    // compact the fresh ids (link order kept) through shared memory: lane i
    // then holds the i-th fresh id (lanes >= nnew hold stale values)
    if (fresh) s.cbuf[__popc(f.nmask & lanemask_lt())] = id;
    __syncwarp();
    f.cid2 = s.cbuf[lane];
    f.n0 = min((int)rs.slots, f.nnew);
    if (f.n0 > 0) {
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive_expect_tx(s.bar, (uint32_t)f.n0 * rs.row_bytes);
        __syncwarp();
        if (lane < f.n0)
            stage_copy(p, s, reinterpret_cast<unsigned char*>(s.stage) + (size_t)lane * rs.stage_bytes, rs.base,
                       f.cid2, p.count, rs.row_bytes, 30);
    }
}

// Approximate distances from staged low-precision rows [0, n) into the
// compacted lanes [s0, s0 + n): 4 lanes per row over 16-byte chunks, fp32
// accumulation in any order (these distances only steer the beam; returned
// distances come from the float32 re-rank).
template <int SPACE, int PREC>
__device__ __forceinline__ void batch_dist_lowp(const SearchParams& p, const WarpSmem& s, int n, int s0, int lane,
                                                float& dc) {
    const int a = lane & 3;
    const int nch = (int)(p.trow_bytes - (PREC == 2 ? 16u : 0u)) / 16;  // 16-byte chunks of data
    const float4* q4 = reinterpret_cast<const float4*>(s.q);
    const unsigned char* stage = reinterpret_cast<const unsigned char*>(s.stage);
    for (int g = 0; g < n; g += 8) {
        const int v = min(g + (lane >> 2), n - 1);
        const unsigned char* row = stage + (size_t)v * p.tstage_bytes;
        if (!DBG_OK(row + p.trow_bytes <= reinterpret_cast<const unsigned char*>(s.pool) && v >= 0, 40,
                    (size_t)v * p.tstage_bytes, n))
            row = stage;
        const uint4* r16 = reinterpret_cast<const uint4*>(row);
        float acc = 0.f;
        float sc = 1.f;
        if (PREC == 2) sc = *reinterpret_cast<const float*>(row + p.trow_bytes - 16);
        for (int c = a; c < nch; c += 4) {
            const uint4 raw = r16[c];
            const uint32_t w[4] = {raw.x, raw.y, raw.z, raw.w};
            if (PREC == 1) {
                // 8 bf16 = elements 8c .. 8c+7
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const float4 qv = q4[2 * c + h];
                    const float x0 = __uint_as_float(w[2 * h] << 16), x1 = __uint_as_float(w[2 * h] & 0xffff0000u);
                    const float x2 = __uint_as_float(w[2 * h + 1] << 16),
                                x3 = __uint_as_float(w[2 * h + 1] & 0xffff0000u);
                    if (SPACE == 0) {
                        float t0 = qv.x - x0, t1 = qv.y - x1, t2 = qv.z - x2, t3 = qv.w - x3;
                        acc = fmaf(t0, t0, acc);
                        acc = fmaf(t1, t1, acc);
                        acc = fmaf(t2, t2, acc);
                        acc = fmaf(t3, t3, acc);
                    } else {
                        acc = fmaf(qv.x, x0, acc);
                        acc = fmaf(qv.y, x1, acc);
                        acc = fmaf(qv.z, x2, acc);
                        acc = fmaf(qv.w, x3, acc);
                    }
                }
            } else {
                // 16 e4m3 = elements 16c .. 16c+15
#pragma unroll
                for (int h = 0; h < 4; h++) {
                    const float4 qv = q4[4 * c + h];
                    const __half2 lo = __half2(__nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)(w[h] & 0xffffu), __NV_E4M3));
                    const __half2 hi = __half2(__nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)(w[h] >> 16), __NV_E4M3));
                    const float2 xa = __half22float2(lo), xb = __half22float2(hi);
                    if (SPACE == 0) {
                        float t0 = fmaf(sc, xa.x, -qv.x), t1 = fmaf(sc, xa.y, -qv.y), t2 = fmaf(sc, xb.x, -qv.z),
                              t3 = fmaf(sc, xb.y, -qv.w);
                        acc = fmaf(t0, t0, acc);
                        acc = fmaf(t1, t1, acc);
                        acc = fmaf(t2, t2, acc);
                        acc = fmaf(t3, t3, acc);
                    } else {
                        acc = fmaf(qv.x, xa.x, acc);
                        acc = fmaf(qv.y, xa.y, acc);
                        acc = fmaf(qv.z, xb.x, acc);
                        acc = fmaf(qv.w, xb.y, acc);
                    }
                }
            }
        }
        acc += __shfl_xor_sync(FULL, acc, 1);
        acc += __shfl_xor_sync(FULL, acc, 2);
        float r = acc;
        if (SPACE != 0) r = __fsub_rn(1.0f, PREC == 2 ? __fmul_rn(sc, acc) : acc);
        const int t = lane - s0 - g;
        const float got = __shfl_sync(FULL, r, (t & 7) << 2);
        if (t >= 0 && t < 8 && t + g < n) dc = got;
    }
}

// Distances of the staged rows [0, n) into the compacted lanes [s0, s0 + n).
template <int SPACE>
__device__ __forceinline__ void batch_dist(const SearchParams& p, const WarpSmem& s, const float4* qr, int n, int s0,
                                           int lane, float& dc) {
    const int a = lane & 3;
    const int n16 = (int)(p.dim >> 4);
    for (int g = 0; g < n; g += 8) {
        const int v = min(g + (lane >> 2), n - 1);
        const float4* x4 = reinterpret_cast<const float4*>(s.stage + (size_t)v * p.stage_stride);
        if (!DBG_OK(reinterpret_cast<const unsigned char*>(x4) + p.row_bytes <=
                        reinterpret_cast<const unsigned char*>(s.pool),
                    50, (size_t)v * p.stage_stride * 4, n))
            x4 = reinterpret_cast<const float4*>(s.stage);
        float r;
        if (n16 <= 8) {
            // query chunks held in registers (qr[c] = this lane's float4 of chunk c)
            float c0 = 0.f, c1 = 0.f, c2 = 0.f, c3 = 0.f;
#pragma unroll
            for (int c = 0; c < 8; c++) {
                if (c < n16) {
                    const float4 qv = qr[c], xv = x4[4 * c + a];
                    if (SPACE == 0) {
                        float t0 = __fsub_rn(qv.x, xv.x), t1 = __fsub_rn(qv.y, xv.y), t2 = __fsub_rn(qv.z, xv.z),
                              t3 = __fsub_rn(qv.w, xv.w);
                        c0 = __fmaf_rn(t0, t0, c0);
                        c1 = __fmaf_rn(t1, t1, c1);
                        c2 = __fmaf_rn(t2, t2, c2);
                        c3 = __fmaf_rn(t3, t3, c3);
                    } else {
                        c0 = __fmaf_rn(qv.x, xv.x, c0);
                        c1 = __fmaf_rn(qv.y, xv.y, c1);
                        c2 = __fmaf_rn(qv.z, xv.z, c2);
                        c3 = __fmaf_rn(qv.w, xv.w, c3);
                    }
                }
            }
            r = group4_reduce<SPACE>(c0, c1, c2, c3);
        } else {
            r = group4_dist16<SPACE>(s.q, reinterpret_cast<const float*>(x4), n16, a);
        }
        const int t = lane - s0 - g;  // compacted index of this lane within the pass
        const float got = __shfl_sync(FULL, r, (t & 7) << 2);
        if (t >= 0 && t < 8 && t + g < n) dc = got;
    }
}

// Distances of all fresh neighbours of a fetched list; result in the owning
// (link-order) lane.
template <int SPACE, int PREC>
__device__ __forceinline__ bool fetch_distances(const SearchParams& p, WarpSmem& s, uint32_t& phase, const Fetch& f,
                                                const float4* qr, int lane, float& d, PhaseClock& pc) {
    float dc = __int_as_float(0x7f800000);
    const RowSrc rs = trav_src<PREC>(p);
    if (f.n0 > 0) {
        const bool ok = mbar_wait(s.bar, phase);
        phase ^= 1u;
        if (!__all_sync(FULL, ok)) return false;
        PT_MARK(4);
        if (PREC == 0) batch_dist<SPACE>(p, s, qr, f.n0, 0, lane, dc);
        else batch_dist_lowp<SPACE, PREC>(p, s, f.n0, 0, lane, dc);
        PT_MARK(5);
    }
    for (int s0 = f.n0; s0 < f.nnew; s0 += (int)rs.slots) {
        const int n = min((int)rs.slots, f.nnew - s0);
        const bool mine = lane >= s0 && lane < s0 + n;
        if (!stage_src(p, s, phase, rs, mine, f.cid2, lane - s0, n, lane)) return false;
        PT_MARK(4);
        if (PREC == 0) batch_dist<SPACE>(p, s, qr, n, s0, lane, dc);
        else batch_dist_lowp<SPACE, PREC>(p, s, n, s0, lane, dc);
        PT_MARK(5);
    }
    const int ci = __popc(f.nmask & lanemask_lt());
    d = __shfl_sync(FULL, dc, ci & 31);
    return true;
}

// ---- learned early termination (see term_mlp.cuh)
struct TermState {
    uint32_t last_change = 0;  // expansion count when the top-k last changed
    uint32_t nchange = 0;      // expansions that changed the top-k
    uint32_t nckpt = 0;        // checkpoints taken
    uint32_t next = 0;         // expansion count at which the next checkpoint falls due
    uint32_t prev_e = 0, prev_d = 0;  // expansions and distance evaluations at the previous checkpoint
};

// A checkpoint falls due every term_period expansions; it is taken (trace
// mode records it, learned mode consults the network) at the first
// expansion from then on where the top-k has not changed for a period and no
// unexpanded candidate is closer than the current k-th result -- the only
// states in which stopping can keep the top-k.  Advances the due count once
// taken.
__device__ __forceinline__ bool term_due(const SearchParams& p, const WarpSmem& s, uint32_t e, int psize,
                                         uint32_t next_dk, TermState& ts) {
    if (ts.next == 0) ts.next = p.term_period;
    if (e < ts.next || e - ts.last_change < p.term_period || psize < (int)p.k || !(next_dk > khi(s.pool[p.k - 1])))
        return false;
    while (ts.next <= e) ts.next += p.term_period;
    return true;
}

__device__ __forceinline__ TermInputs term_inputs(const SearchParams& p, float e, float d1, float dk, float dn,
                                                  float d_entry, float qn, uint32_t dists, const TermState& ts) {
    TermInputs in;
    in.e = e;
    in.d1 = d1;
    in.dk = dk;
    in.dn = dn;
    in.d_entry = d_entry;
    in.qn = qn;
    in.since_change = e - (float)ts.last_change;
    in.inv_period = 1.0f / (float)p.term_period;
    in.nchange = (float)ts.nchange;
    in.eval_rate = (float)(dists - ts.prev_d) / fmaxf(e - (float)ts.prev_e, 1.0f);
    return in;
}

// Trace mode: the ids of the first ckpt_width beam entries of a checkpoint
// row, and (when asked for) their float32 distances.
template <int SPACE>
__device__ __forceinline__ void term_record_ids(const SearchParams& p, const WarpSmem& s, int lane, size_t row,
                                                int psize) {
    const int w = (int)p.ckpt_width;
    for (int i = lane; i < w; i += 32) p.ckpt_ids[row * w + i] = i < psize ? kid(s.pool[i]) : INVALID_ID;
    if (p.ckpt_dists) {
        float* out = p.ckpt_dists + row * w;
        for (int i = psize + lane; i < w; i += 32) out[i] = __int_as_float(0x7f800000);
        trace_dists<SPACE>(p, s.q, s.pool, min(w, psize), lane, out);
    }
}

// Checkpoint after `e` level-0 expansions (`dists` distance evaluations),
// with a next candidate of distance key `next_dk` waiting: trace mode records
// the features and the first beam ids; learned mode returns true when the
// network says stop.
template <int SPACE, int TERM>
__device__ __forceinline__ bool term_checkpoint(const SearchParams& p, const WarpSmem& s, int lane, uint32_t qi,
                                                uint32_t e, uint32_t dists, int psize, uint32_t next_dk,
                                                float d_entry, float qn, TermState& ts) {
    if (psize == 0) return false;  // nothing admissible found yet
    const int kq = (int)p.k;
    const int kk = min(kq, psize);
    float fe[kTermFeatures];
    term_features(term_inputs(p, (float)e, funkey(khi(s.pool[0])), funkey(khi(s.pool[kk - 1])), funkey(next_dk),
                              d_entry, qn, dists, ts),
                  s.pool, psize, (int)p.ef, lane, fe);
    ts.prev_e = e;
    ts.prev_d = dists;
    if (TERM == 1) {
        if (ts.nckpt + 1 < p.term_max_ckpt) {  // the last row is kept for the final state
            const size_t row = (size_t)qi * p.term_max_ckpt + ts.nckpt;
            if (lane < kTermFeatures) p.ckpt_feat[row * kTermFeatures + lane] = fe[lane];
            term_record_ids<SPACE>(p, s, lane, row, psize);
        }
        ts.nckpt++;
        return false;
    }
    return term_logit(p.term_model, fe, lane) > p.term_logit;
}

// Trace mode, end of the beam: the final row holds its first beam ids
// (before any re-rank) and the features of that state; labels of earlier
// rows refer to it.
template <int SPACE>
__device__ __forceinline__ void term_final_row(const SearchParams& p, const WarpSmem& s, int lane, uint32_t qi,
                                               uint32_t e, uint32_t dists, int psize, float d_entry, float qn,
                                               const TermState& ts) {
    if (p.term_max_ckpt == 0) {
        if (lane == 0) p.ckpt_count[qi] = 0;
        return;
    }
    const int kq = (int)p.k;
    const uint32_t r = min(ts.nckpt, p.term_max_ckpt - 1);
    const size_t row = (size_t)qi * p.term_max_ckpt + r;
    const int kk = min(kq, psize);
    const float d1 = kk > 0 ? funkey(khi(s.pool[0])) : 0.f;
    const float dk = kk > 0 ? funkey(khi(s.pool[kk - 1])) : 0.f;
    float fe[kTermFeatures];
    if (psize > 0) {
        term_features(term_inputs(p, (float)e, d1, dk, dk, d_entry, qn, dists, ts), s.pool, psize, (int)p.ef, lane,
                      fe);
    } else {
        for (int i = 0; i < kTermFeatures; i++) fe[i] = 0.f;
    }
    if (lane < kTermFeatures) p.ckpt_feat[row * kTermFeatures + lane] = fe[lane];
    term_record_ids<SPACE>(p, s, lane, row, psize);
    if (lane == 0) p.ckpt_count[qi] = r + 1;
}

// TIES (id order only): flag the query (status kTieBit) when its run meets a
// distance tie that can make the reference's heaps decide differently from the
// (distance, id) order.  With acceptance by counting (independent of heap
// layout), the two runs agree step by step unless (a) the candidate popped next
// shares its distance with another unexpanded candidate, or (b) the entries
// dropped from the full pool tie with its new worst entry (an evicted entry that
// stays in candidate_set at lowerBound would still be expanded); (c), the
// top-k boundary tie, is checked by the caller.
//
// FILTER (id order only): deletions and / or an allow mask, as in the
// reference's non-bare-bone loop (hnswalg.h:330-440).  Accepted neighbours that
// may not be returned go to the sorted list s.extra instead of the pool: they
// are candidates (expanded in distance order) but never results.  A candidate
// taken from that list ends the search when the pool is full and its distance
// is above lowerBound; list entries beyond lowerBound are dropped, since they
// can only end the search.  A disallowed entry point (ep_ok false) is expanded
// first and never stored.
template <int SPACE, bool EXACT, int PREC, int TERM, bool TIES = false, bool FILTER = false>
__device__ bool base_pipelined(const SearchParams& p, WarpSmem& s, uint32_t& phase, int lane, Counters& ct,
                               PhaseClock& pc, const float4* qr, uint32_t ep, float d0, int& psize, int& tsz,
                               uint32_t& status, uint32_t qi, float qn, bool ep_ok = true) {
    const int ef = (int)p.ef;
    const int kq = (int)p.k;
    TermState ts;
    const int pcap = (int)p.pool_cap;
    int hint_p = 0, csz = 0;
    int xsize = 0, hint_x = 0;  // FILTER: the list of disallowed candidates
    const int xcap = (int)p.extra_cap;
    const uint32_t skip_id = FILTER && !ep_ok ? ep : INVALID_ID;
    // the entry point is pushed and popped at once (hnswalg.h:325-359)
    if (lane == 0 && (!FILTER || ep_ok)) {
        s.pool[0] = mkkey(d0, ep) | (EXACT ? 0u : EXP_BIT);
        if (EXACT) s.topheap[0] = mkkey(d0, ep);
    }
    psize = !FILTER || ep_ok ? 1 : 0;
    tsz = EXACT ? 1 : 0;
    __syncwarp();
    Fetch f;
    fetch_links<PREC, FILTER>(p, s, ep, lane, f, skip_id);
    ct.l0_exp += 1;
    PT_MARK(3);
    while (true) {
        ct.l0_dists += f.nnew;
        float d;
        if (!fetch_distances<SPACE, PREC>(p, s, phase, f, qr, lane, d, pc)) return false;
        // ---- acceptance (closed form of hnswalg.h:395 over the link order)
        const uint32_t dk = fkey(d);
        const bool full = psize == ef;
        const uint32_t lbk = full ? khi(s.pool[psize - 1]) : 0xffffffffu;
        bool live = f.fresh && !(full && dk >= lbk);
        uint64_t key = ((uint64_t)dk << 32) | f.id;
        int posP = 0, cntP = 0, posX = 0;
        if (live) {
            bool dup = false;
            cntP = upper_bound_hi(s.pool, psize, dk);
            posP = insert_pos(s.pool, cntP, dk, f.id, dup);
            if (FILTER && !dup) posX = insert_pos(s.extra, upper_bound_hi(s.extra, xsize, dk), dk, f.id, dup);
            if (dup) live = false;
        }
        const bool allowed = !FILTER || f.allowed;
        const unsigned amask = __ballot_sync(FULL, live && allowed);
        int cntN = 0;
        for (unsigned m = amask; m; m &= m - 1) {
            const int src2 = __ffs(m) - 1;
            const uint32_t dk2 = __shfl_sync(FULL, dk, src2);
            cntN += (src2 < lane && dk2 <= dk);
        }
        const bool accept = live && cntP + cntN < ef;
        const unsigned pmask = __ballot_sync(FULL, accept && allowed);
        const unsigned xmask = FILTER ? __ballot_sync(FULL, accept && !allowed) : 0u;
        if (TERM && __any_sync(FULL, accept && allowed && cntP + cntN < kq)) {
            ts.last_change = ct.l0_exp;
            ts.nchange++;
        }
        PT_MARK(6);
        // ---- the next candidate
        // smallest accepted key: the smallest distance key, then the smallest
        // id among the lanes holding it (two warp reductions)
        const uint32_t kmin_hi = __reduce_min_sync(FULL, accept ? dk : 0xffffffffu);
        const uint32_t kmin_lo = __reduce_min_sync(FULL, accept && dk == kmin_hi ? f.id : 0xffffffffu);
        const uint64_t kmin = ((uint64_t)kmin_hi << 32) | kmin_lo;
        bool have_next = false, spec = false, next_extra = false;
        uint32_t next = INVALID_ID, next_dk = 0xffffffffu;
        if (!EXACT) {
            int ip = find_unexpanded(s.pool, psize, hint_p, lane);
            const uint64_t kp = ip >= 0 ? (s.pool[ip] & KEY_MASK) : ~0ull;
            int ix = -1;
            uint64_t kx = ~0ull;
            if (FILTER) {
                ix = find_unexpanded(s.extra, xsize, hint_x, lane);
                kx = ix >= 0 ? (s.extra[ix] & KEY_MASK) : ~0ull;
            }
            if (kx < kp && kx < kmin) {
                // a disallowed candidate from the list (FILTER only)
                have_next = true;
                next_extra = true;
                next_dk = khi(kx);
                next = kid(kx);
                __syncwarp();
                if (lane == 0) s.extra[ix] |= EXP_BIT;
                __syncwarp();
            } else if (kp != ~0ull || kmin != ~0ull) {
                have_next = true;
                next_dk = khi(kmin < kp ? kmin : kp);
                if (TIES) {  // (a): candidate_set's top must be unique by distance
                    int same = __popc(__ballot_sync(FULL, accept && dk == next_dk));
                    if (ip >= 0) same += unexpanded_with_dist(s.pool, psize, ip, next_dk, lane);
                    if (same > 1) status |= kTieBit;
                }
                if (kmin < kp) {
                    next = (uint32_t)kmin;
                    if (FILTER) next_extra = __any_sync(FULL, accept && !allowed && key == kmin);
                    if (accept && key == kmin) key |= EXP_BIT;  // inserted already expanded
                } else {
                    next = kid(kp);
                    __syncwarp();
                    if (lane == 0) s.pool[ip] |= EXP_BIT;
                    __syncwarp();
                }
            }
        } else {
            // candidate_set after this expansion's pushes: its top is the
            // smallest of the current heap top and the accepted keys; when
            // that distance is unique the heap layout cannot matter
            const uint64_t r0 = csz > 0 ? s.candheap[0] : ~0ull;
            const uint32_t r0d = khi(r0);
            const bool r0tie = (csz > 1 && khi(s.candheap[1]) == r0d) || (csz > 2 && khi(s.candheap[2]) == r0d);
            const uint32_t ad = khi(kmin);
            const uint32_t nd = min(r0d, ad);
            const int acount = __popc(__ballot_sync(FULL, accept && dk == nd));
            const int mult = (csz > 0 && r0d == nd ? 1 + (r0tie ? 1 : 0) : 0) + acount;
            if ((csz > 0 || kmin != ~0ull) && mult == 1) {
                spec = true;
                next = r0d == nd && csz > 0 ? kid(r0) : (uint32_t)kmin;
            }
        }
        Fetch fn;
        if (have_next || spec) fetch_links<PREC, FILTER>(p, s, next, lane, fn, skip_id);
        PT_MARK(2);
        // ---- bookkeeping of this expansion, under the latency of the next fetch
        int nev = 0;
        if (EXACT && pmask) {
            if (accept) s.accbuf[__popc(pmask & lanemask_lt())] = key;
            __syncwarp();
            const int na = __popc(pmask);
            uint32_t ovf = 0;
            if (lane == 0) {
                int cn = csz, tn = tsz;
                for (int t = 0; t < na; t++) {
                    const uint64_t e = s.accbuf[t];
                    if (cn < s.cand_total) ref_heap_push(s.candheap, cn, e, CandLess());
                    else ovf = 1;
                    ref_heap_push(s.topheap, tn, e, TopLess());
                    if (tn > ef) s.evbuf[nev++] = ref_heap_pop(s.topheap, tn, TopLess());
                }
                csz = cn;
                tsz = tn;
            }
            csz = __shfl_sync(FULL, csz, 0);
            tsz = __shfl_sync(FULL, tsz, 0);
            nev = __shfl_sync(FULL, nev, 0);
            if (__shfl_sync(FULL, ovf, 0)) status |= HNSWGPU_STATUS_OVERFLOW_BIT;
            __syncwarp();
            PT_MARK(7);
        }
        if (pmask) {
            const int m = merge_sorted(s.pool, psize, pcap, pmask, key, posP, lane);
            hint_p = min(hint_p, m);
            if (TIES && psize > ef) {
                // (b): the merge kept one entry more than ef (pool_cap is
                // ef + 1): the first one dropped, next to the new worst
                if (khi(s.pool[ef]) == khi(s.pool[ef - 1])) status |= kTieBit;
                psize = ef;
            }
        }
        if (FILTER) {
            if (xmask) {
                if (xsize + __popc(xmask) > xcap) status |= HNSWGPU_STATUS_OVERFLOW_BIT;
                const int m = merge_sorted(s.extra, xsize, xcap, xmask, key, posX, lane);
                hint_x = min(hint_x, m);
            }
            if (psize == ef && xsize > 0) {
                // list entries beyond lowerBound can never be expanded
                xsize = upper_bound_hi(s.extra, xsize, khi(s.pool[psize - 1]));
                hint_x = min(hint_x, xsize);
            }
            if (next_extra && psize == ef && next_dk > khi(s.pool[ef - 1])) {
                // the reference pops it and stops (hnswalg.h:345-347): drain
                // the speculative fetch
                if (fn.n0 > 0) {
                    mbar_wait(s.bar, phase);
                    phase ^= 1u;
                }
                break;
            }
            if (have_next && ct.l0_exp >= p.max_expansions) {
                // Entries dropped from a full list can be re-admitted after a
                // visited-cache miss, and a search that never fills its pool
                // (a filter that rejects almost everything) keeps dropping
                // them: bound the expansions and flag the query.
                status |= HNSWGPU_STATUS_OVERFLOW_BIT;
                if (fn.n0 > 0) {
                    mbar_wait(s.bar, phase);
                    phase ^= 1u;
                }
                break;
            }
        }
        if (EXACT && nev) remove_keys(s.pool, psize, s.evbuf, nev, lane);
        if (!EXACT) {
            // the expansion after `next` is most often the first unexpanded
            // entry now: pull its link row into L2 while `next` runs
            int h2 = hint_p;
            const int nx = find_unexpanded(s.pool, psize, h2, lane);
            if (nx >= 0 && lane == 0) prefetch_l2(p.links0 + (size_t)kid(s.pool[nx]) * p.maxM0);
        }
        PT_MARK(8);
        if (TIES && (status & kTieBit)) {
            // listed for the heap replay, which recomputes the whole query:
            // drain the prefetched expansion and stop here
            if (have_next && fn.n0 > 0) {
                mbar_wait(s.bar, phase);
                phase ^= 1u;
            }
            break;
        }
        if (TERM && have_next && term_due(p, s, ct.l0_exp, psize, next_dk, ts) &&
            term_checkpoint<SPACE, TERM>(p, s, lane, qi, ct.l0_exp, ct.l0_dists, psize, next_dk, d0, qn, ts)) {
            // confident that the top-k is final: drain the prefetched
            // expansion and stop
            if (fn.n0 > 0) {
                mbar_wait(s.bar, phase);
                phase ^= 1u;
            }
            break;
        }
        if (EXACT) {
            // the reference's loop head: top of candidate_set vs lowerBound
            bool go = false;
            uint32_t top_id = INVALID_ID;
            if (csz > 0) {
                const uint64_t c = s.candheap[0];
                const uint32_t lb = khi(s.pool[psize - 1]);
                go = !(khi(c) > lb);
                top_id = kid(c);
            }
            if (!go) {
                if (spec && fn.n0 > 0) {  // drain the unused copies
                    mbar_wait(s.bar, phase);
                    phase ^= 1u;
                }
                break;
            }
            __syncwarp();
            if (lane == 0) {
                int n = csz;
                ref_heap_pop(s.candheap, n, CandLess());
                if (n > 0) prefetch_l2(p.links0 + (size_t)kid(s.candheap[0]) * p.maxM0);
            }
            csz--;
            __syncwarp();
            if (spec && top_id != next) {
                // only after a full candidate heap dropped a push (flagged as
                // an overflow): fetch the actual top instead
                if (fn.n0 > 0) {
                    mbar_wait(s.bar, phase);
                    phase ^= 1u;
                }
                spec = false;
            }
            if (!spec) fetch_links<PREC>(p, s, top_id, lane, fn);
        } else if (!have_next) {
            break;
        }
        f = fn;
        ct.l0_exp += 1;
        PT_MARK(2);
    }
    if (TERM == 1) term_final_row<SPACE>(p, s, lane, qi, ct.l0_exp, ct.l0_dists, psize, d0, qn, ts);
    return true;
}

// Exact re-rank after a low-precision beam: the best `rerank` pool entries
// (ordered by approximate distance) get their float32 rows staged (staging
// area + the now idle visited cache) and their distances recomputed in the
// reference's summation order; the pool is then re-sorted by the exact
// (distance, id) keys, so the k returned distances are bit-exact.
template <int SPACE>
__device__ bool rerank_fp32(const SearchParams& p, WarpSmem& s, uint32_t& phase, int lane, const float4* qr,
                            int& psize) {
    const int R = min(psize, (int)p.rerank);
    const RowSrc rs{reinterpret_cast<const unsigned char*>(p.vecs), p.row_bytes, p.stage_stride * 4, p.rr_slots};
#ifdef HNSWGPU_BOUNDS_CHECK
    for (int r = lane; r < psize; r += 32)
        for (int t = 0; t < psize; t++)
            if (t != r) DBG_OK(kid(s.pool[t]) != kid(s.pool[r]), 120, kid(s.pool[r]), (t << 16) | r);
    __syncwarp();
#endif
    for (int b = 0; b < R; b += (int)rs.slots) {
        const int nb = min((int)rs.slots, R - b);
        uint32_t id = lane < nb ? kid(s.pool[b + lane]) : 0u;
        if (!DBG_OK(id < p.count && b + lane < (int)p.pool_cap, 70, id, b + lane)) id = 0;
        if (!stage_src(p, s, phase, rs, lane < nb, id, lane, nb, lane)) return false;
        float dc = 0.f;
        batch_dist<SPACE>(p, s, qr, nb, 0, lane, dc);
        __syncwarp();
        if (lane < nb) s.pool[b + lane] = mkkey(dc, id);
        __syncwarp();
    }
#ifdef HNSWGPU_BOUNDS_CHECK
    for (int r = lane; r < R; r += 32)
        for (int t = 0; t < R; t++)
            if (t != r) DBG_OK(s.pool[t] != s.pool[r], 130, s.pool[r], (t << 16) | r);
    __syncwarp();
#endif
    // rank by counting; the staging area is free again and holds the result
    uint64_t* tmp = reinterpret_cast<uint64_t*>(s.stage);
    for (int r = lane; r < R; r += 32) {
        const uint64_t kr = s.pool[r];
        int rank = 0;
        for (int t = 0; t < R; t++) rank += s.pool[t] < kr || (s.pool[t] == kr && t < r);
        if (DBG_OK(rank < R && reinterpret_cast<unsigned char*>(tmp + rank + 1) <= reinterpret_cast<unsigned char*>(s.pool),
                   60, rank, R))
            tmp[rank] = kr;
    }
    __syncwarp();
    for (int r = lane; r < R; r += 32) s.pool[r] = tmp[r];
    __syncwarp();
    psize = R;
    return true;
}

template <int SPACE, bool FAST16, bool EXACT, int PREC, int TERM, bool TIES = false, bool FILTER = false>
__device__ bool search_one(const SearchParams& p, WarpSmem& s, uint32_t& phase, uint32_t qi, int lane,
                           Counters& ct, PhaseClock& pc) {
    pc.start();
    const int dim = (int)p.dim;
    const uint32_t ef = p.ef;
    // ---- query row (normalised for the cosine space)
    const float* qg = p.queries + (size_t)qi * p.q_stride;
    for (int i = lane; i < (int)p.row_floats; i += 32) s.q[i] = i < dim ? qg[i] : 0.f;
    __syncwarp();
    if (p.normalize) {
        float sc = 0.f;
        if (lane == 0) sc = norm_scale(s.q, dim);
        sc = __shfl_sync(FULL, sc, 0);
        __syncwarp();
        for (int i = lane; i < dim; i += 32) s.q[i] = __fmul_rn(s.q[i], sc);
        __syncwarp();
    }
    const uint32_t nvis = 1u << p.log2_vis;
    for (uint32_t i = lane; i < nvis; i += 32) s.vis[i] = INVALID_ID;

    PT_MARK(0);
    // ---- upper-layer greedy descent (hnswalg.h:1274-1302)
    uint32_t cur = p.ep;
    float curd;
    if (!lane_distances<SPACE, FAST16>(p, s, phase, cur, 1, lane, curd, pc)) return false;
    curd = __shfl_sync(FULL, curd, 0);
    ct.upper_dists += 1;
    const uint32_t up_stride = p.maxM + 1;
    for (int level = p.maxlevel; level > 0; level--) {
        while (true) {
            const uint32_t* row = p.upper_links + (size_t)(p.upper_off[cur] + (uint32_t)(level - 1)) * up_stride;
            int cnt = (int)(row[0] & 0xffffu);
            ct.upper_hops += 1;
            ct.upper_dists += cnt;
            float best = curd;
            uint32_t best_id = INVALID_ID;
            for (int c0 = 0; c0 < cnt; c0 += 32) {
                int n = min(32, cnt - c0);
                uint32_t id = lane < n ? row[1 + c0 + lane] : INVALID_ID;
                float d;
                if (!lane_distances<SPACE, FAST16>(p, s, phase, id, n, lane, d, pc)) return false;
                float m = lane < n ? d : __int_as_float(0x7f800000);
#pragma unroll
                for (int o = 16; o; o >>= 1) m = fminf(m, __shfl_xor_sync(FULL, m, o));
                if (m < best) {
                    unsigned hit = __ballot_sync(FULL, lane < n && d == m);
                    best = m;
                    best_id = __shfl_sync(FULL, id, __ffs(hit) - 1);
                }
            }
            if (best_id == INVALID_ID) break;
            cur = best_id;
            curd = best;
        }
    }

    PT_MARK(1);
    // ---- level-0 beam (hnswalg.h:308-440)
    const bool bare = p.bare != 0;
    int psize = 0, xsize = 0, hint_p = 0, hint_x = 0;
    const int xcap = (int)p.extra_cap;
    uint32_t status = 0;
    // A disallowed entry point is queued with the sentinel distance FLT_MAX
    // (hnswalg.h:336-337) and never evaluated, so the exact-key lookup cannot
    // recognise it when the visited cache misses on it later: skip it by id.
    uint32_t skip_id = INVALID_ID;
    // ef, or ef + 32 in tie-exact mode (ef + 1 in a tie-listing pass, for
    // the pipelined beam only)
    const int pcap = TIES ? (int)ef : (int)p.pool_cap;
    int tsz = 0, csz = 0;               // tie-exact mode: heap sizes (warp-uniform)
    const uint64_t sentinel = mkkey(__int_as_float(0x7f7fffff), cur);
    // FILTER kernels run the id order only (the host never pairs it with EXACT)
    const bool pipe = FAST16 && (bare || FILTER) && p.maxM0 <= 32 && !p.eps_mode;
    float qn = 0.f;
    if (TERM) {  // |q|^2, a feature of the termination network
        for (uint32_t i = lane; i < p.dim; i += 32) qn = fmaf(s.q[i], s.q[i], qn);
#pragma unroll
        for (int o = 16; o; o >>= 1) qn += __shfl_xor_sync(FULL, qn, o);
    }
    TermState ts;
    if (pipe) {
        float d0;
        if (PREC == 0) {
            if (!lane_distances<SPACE, FAST16>(p, s, phase, cur, 1, lane, d0, pc)) return false;
        } else {
            // every pool key of a low-precision beam must come from the same
            // (approximate) arithmetic: a node re-reached after a visited-cache
            // miss is recognised by its exact (distance, id) key
            const RowSrc rs = trav_src<PREC>(p);
            if (!stage_src(p, s, phase, rs, lane == 0, cur, 0, 1, lane)) return false;
            d0 = 0.f;
            batch_dist_lowp<SPACE, PREC>(p, s, 1, 0, lane, d0);
        }
        d0 = __shfl_sync(FULL, d0, 0);
        ct.l0_dists += 1;
        if (lane == 0) s.vis[vis_slot(cur, p.log2_vis)] = cur;
        float4 qr[8];
        const int n16 = (int)(p.dim >> 4);
        const float4* q4 = reinterpret_cast<const float4*>(s.q);
#pragma unroll
        for (int c = 0; c < 8; c++) qr[c] = c < n16 ? q4[4 * c + (lane & 3)] : make_float4(0.f, 0.f, 0.f, 0.f);
        __syncwarp();
        if (!base_pipelined<SPACE, EXACT, PREC, TERM, TIES, FILTER>(p, s, phase, lane, ct, pc, qr, cur, d0, psize,
                                                                    tsz, status, qi, qn, bare || is_allowed(p, cur)))
            return false;
        // (c): the reference pops top_candidates down to k by distance
        if (TIES && psize > (int)p.k && khi(s.pool[p.k - 1]) == khi(s.pool[p.k])) status |= kTieBit;
        if (PREC != 0 && !rerank_fp32<SPACE>(p, s, phase, lane, qr, psize)) return false;
    } else {
    if (TIES) status |= kTieBit;  // only the pipelined beam checks its ties
    if (bare || is_allowed(p, cur)) {
        float d0;
        if (!lane_distances<SPACE, FAST16>(p, s, phase, cur, 1, lane, d0, pc)) return false;
        d0 = __shfl_sync(FULL, d0, 0);
        ct.l0_dists += 1;
        if (lane == 0) s.pool[0] = mkkey(d0, cur);
        psize = 1;
        if (EXACT) {
            if (lane == 0) {
                s.topheap[0] = mkkey(d0, cur);
                s.candheap[0] = mkkey(d0, cur);
            }
            tsz = csz = 1;
        }
    } else {
        if (EXACT) {
            if (lane == 0) s.candheap[0] = sentinel;
            csz = 1;
        } else {
            if (lane == 0) s.extra[0] = sentinel;
            xsize = 1;
        }
        skip_id = cur;
    }
    if (lane == 0) s.vis[vis_slot(cur, p.log2_vis)] = cur;
    __syncwarp();

    while (true) {
      uint32_t cid;
      if (EXACT) {
        // ---- next candidate: the reference's candidate_set.top() (hnswalg.h:343-359)
        if (csz == 0) break;
        const uint64_t c = s.candheap[0];
        const uint32_t lbk = psize > 0 ? khi(s.pool[psize - 1]) : fkey(__int_as_float(0x7f7fffff));
        bool stop = bare ? (khi(c) > lbk) : (khi(c) > lbk && psize == (int)ef);
        // EpsilonSearchStopCondition::should_stop_search (stop_condition.h:242-253):
        // its item count is top_candidates' size, which the pool mirrors here
        if (p.eps_mode && khi(c) > fkey(p.eps) && psize >= (int)p.eps_min) stop = true;
        if (stop) break;
        __syncwarp();
        if (lane == 0) {
            int n = csz;
            ref_heap_pop(s.candheap, n, CandLess());
            if (n > 0) prefetch_l2(p.links0 + (size_t)kid(s.candheap[0]) * p.maxM0);
        }
        csz--;
        __syncwarp();
        cid = kid(c);
        ct.l0_exp += 1;
      } else {
        int ip = find_unexpanded(s.pool, psize, hint_p, lane);
        int ix = bare ? -1 : find_unexpanded(s.extra, xsize, hint_x, lane);
        uint64_t kp = ip >= 0 ? (s.pool[ip] & KEY_MASK) : ~0ull;
        uint64_t kx = ix >= 0 ? (s.extra[ix] & KEY_MASK) : ~0ull;
        if (ip < 0 && ix < 0) break;
        bool from_extra = kx < kp;
        if (from_extra && psize == (int)ef && khi(kx) > khi(s.pool[psize - 1])) break;
        uint64_t ck = from_extra ? kx : kp;
        if (TERM && ct.l0_exp > 0 && term_due(p, s, ct.l0_exp, psize, khi(ck), ts) &&
            term_checkpoint<SPACE, TERM>(p, s, lane, qi, ct.l0_exp, ct.l0_dists, psize, khi(ck), curd, qn, ts))
            break;
        __syncwarp();
        if (lane == 0) {
            if (from_extra) s.extra[ix] = ck | EXP_BIT;
            else s.pool[ip] = ck | EXP_BIT;
        }
        __syncwarp();
        cid = kid(ck);
        ct.l0_exp += 1;
        {
            // the next expansion is most often the next unexpanded pool entry:
            // start pulling its link row into L2 now
            int h2 = hint_p;
            int nx = find_unexpanded(s.pool, psize, h2, lane);
            if (nx >= 0 && lane == 0) prefetch_l2(p.links0 + (size_t)kid(s.pool[nx]) * p.maxM0);
        }
      }
        PT_MARK(2);
        if (ct.l0_exp > p.max_expansions) {
            // only reachable after a candidate-list overflow (nodes dropped
            // from the list can be re-admitted); stop and flag the query
            status |= HNSWGPU_STATUS_OVERFLOW_BIT;
            break;
        }
        const uint32_t* lrow = p.links0 + (size_t)cid * p.maxM0;
        for (uint32_t c0 = 0; c0 < p.maxM0; c0 += 32) {
            uint32_t j = c0 + lane;
            uint32_t id = j < p.maxM0 ? __ldg(lrow + j) : INVALID_ID;
            bool valid = id != INVALID_ID;
            if (__ballot_sync(FULL, valid) == 0) break;
            // duplicate ids within one list: keep the first occurrence
            unsigned peers = __match_any_sync(FULL, id);
            bool fresh = valid && (__ffs(peers) - 1 == lane) && id != skip_id;
            uint32_t slot = fresh ? vis_slot(id, p.log2_vis) : 0;
            if (fresh && s.vis[slot] == id) fresh = false;
            __syncwarp();
            if (fresh) s.vis[slot] = id;
            unsigned nmask = __ballot_sync(FULL, fresh);
            int nnew = __popc(nmask);
            PT_MARK(3);
            if (nnew == 0) continue;
            ct.l0_dists += nnew;
            // compact the fresh ids to lanes [0, nnew), evaluate, route back
            int ci = __popc(nmask & lanemask_lt());
            if (fresh) s.cbuf[ci] = id;  // lane i then holds the i-th fresh id
            __syncwarp();
            uint32_t cid2 = s.cbuf[lane];
            __syncwarp();
            float dc;
            if (!lane_distances<SPACE, FAST16>(p, s, phase, cid2, nnew, lane, dc, pc)) return false;
            float d = __shfl_sync(FULL, dc, ci & 31);
            // ---- acceptance (closed form of the sequential test)
            uint32_t dk = fkey(d);
            bool full = psize == (int)ef;
            uint32_t lbk = full ? khi(s.pool[psize - 1]) : 0xffffffffu;
            bool live = fresh && !(full && dk >= lbk);
            uint64_t key = ((uint64_t)dk << 32) | id;
            int posP = 0, posX = 0, cntP = 0;
            if (live) {
                bool dup = false;
                cntP = upper_bound_hi(s.pool, psize, dk);
                posP = insert_pos(s.pool, cntP, dk, id, dup);
                if (!bare && !dup) posX = insert_pos(s.extra, upper_bound_hi(s.extra, xsize, dk), dk, id, dup);
                if (dup) live = false;
            }
            bool allowed = bare || (live && is_allowed(p, id));
            unsigned amask = __ballot_sync(FULL, live && allowed);
            int cntN = 0;
            for (unsigned m = amask; m; m &= m - 1) {
                int src2 = __ffs(m) - 1;
                uint32_t dk2 = __shfl_sync(FULL, dk, src2);
                cntN += (src2 < lane && dk2 <= dk);
            }
            bool accept = live && (uint32_t)(cntP + cntN) < ef;
            unsigned pmask = __ballot_sync(FULL, accept && allowed);
            if (TERM && __any_sync(FULL, accept && allowed && cntP + cntN < (int)p.k)) {
                ts.last_change = ct.l0_exp;
                ts.nchange++;
            }
            unsigned xmask = bare ? 0u : __ballot_sync(FULL, accept && !allowed);
            PT_MARK(6);
            int nev = 0;
            if (EXACT && (pmask | xmask)) {
                // replay the reference's heap operations for the accepted
                // neighbours in link order (hnswalg.h:398-429): every one
                // enters candidate_set; allowed ones enter top_candidates,
                // which then drops its top while it holds more than ef.
                const unsigned amask2 = pmask | xmask;
                if (accept) s.accbuf[__popc(amask2 & lanemask_lt())] = key | (allowed ? EXP_BIT : 0u);
                __syncwarp();
                const int na = __popc(amask2);
                uint32_t ovf = 0;
                if (lane == 0) {
                    int cn = csz, tn = tsz;
                    for (int t = 0; t < na; t++) {
                        uint64_t e = s.accbuf[t];
                        const bool al = ((uint32_t)e & EXP_BIT) != 0;
                        e &= KEY_MASK;
                        if (cn < s.cand_total) ref_heap_push(s.candheap, cn, e, CandLess());
                        else ovf = 1;
                        if (al) {
                            ref_heap_push(s.topheap, tn, e, TopLess());
                            if (tn > (int)ef) s.evbuf[nev++] = ref_heap_pop(s.topheap, tn, TopLess());
                        }
                    }
                    csz = cn;
                    tsz = tn;
                }
                csz = __shfl_sync(FULL, csz, 0);
                tsz = __shfl_sync(FULL, tsz, 0);
                nev = __shfl_sync(FULL, nev, 0);
                if (__shfl_sync(FULL, ovf, 0)) status |= HNSWGPU_STATUS_OVERFLOW_BIT;
                __syncwarp();
                PT_MARK(7);
            }
            if (pmask) {
                int m = merge_sorted(s.pool, psize, pcap, pmask, key, posP, lane);
                hint_p = min(hint_p, m);
            }
            if (EXACT && nev) remove_keys(s.pool, psize, s.evbuf, nev, lane);
            if (xmask) {
                if (xsize + __popc(xmask) > xcap) status |= HNSWGPU_STATUS_OVERFLOW_BIT;
                int m = merge_sorted(s.extra, xsize, xcap, xmask, key, posX, lane);
                hint_x = min(hint_x, m);
            }
            if (!bare && psize == (int)ef && xsize > 0) {
                // entries beyond lowerBound can never be expanded again
                xsize = upper_bound_hi(s.extra, xsize, khi(s.pool[psize - 1]));
                hint_x = min(hint_x, xsize);
            }
            PT_MARK(8);
        }
    }
    PT_MARK(2);
    if (TERM == 1) term_final_row<SPACE>(p, s, lane, qi, ct.l0_exp, ct.l0_dists, psize, curd, qn, ts);
    }  // general loop

    const uint32_t k = p.k;
    if (EXACT && p.eps_mode) {
        // searchStopConditionClosest (hnswalg.h:1365-1374): top_candidates
        // popped into the result from its back (closest first, equal
        // distances in the heap's pop order), then filter_results drops the
        // trailing entries beyond epsilon.  The result carries internal ids,
        // as the reference's does.
        int tn = tsz;
        if (lane == 0)
            for (int i = tn - 1; i >= 0; i--) s.pool[i] = ref_heap_pop(s.topheap, tn, TopLess());
        __syncwarp();
        const uint32_t ek = fkey(p.eps);
        int cnt = 0;
        for (int base = 0; base < tsz; base += 32) {
            const int i = base + lane;
            cnt += __popc(__ballot_sync(FULL, i < tsz && khi(s.pool[i]) <= ek));
        }
        cnt = min(cnt, (int)k);
        uint64_t* oid = p.out_labels + (size_t)qi * k;
        float* odist = p.out_dists + (size_t)qi * k;
        for (int r = lane; r < (int)k; r += 32) {
            oid[r] = r < cnt ? (uint64_t)kid(s.pool[r]) : ~0ull;
            odist[r] = r < cnt ? funkey(khi(s.pool[r])) : __int_as_float(0x7f800000);
        }
        if (lane == 0) {
            p.out_counts[qi] = cnt;
            if (status) atomicOr(p.status, status);
        }
        return true;
    }
    if (EXACT) {
        // the reference pops top_candidates down to k (hnswalg.h:1314-1316);
        // keep in the pool exactly the entries left in the heap
        int tn = tsz;
        if (lane == 0)
            while (tn > (int)k) ref_heap_pop(s.topheap, tn, TopLess());
        tn = __shfl_sync(FULL, tn, 0);
        __syncwarp();
        for (int t = lane; t < tn; t += 32) {
            int pos = lower_bound_key(s.pool, psize, s.topheap[t] & KEY_MASK);
            s.pool[pos] |= EXP_BIT;
        }
        __syncwarp();
        int out = 0;
        for (int base = 0; base < psize; base += 32) {
            int i = base + lane;
            bool keep = i < psize && ((uint32_t)s.pool[i] & EXP_BIT);
            unsigned m = __ballot_sync(FULL, keep);
            uint64_t e = keep ? (s.pool[i] & KEY_MASK) : 0;
            __syncwarp();
            if (keep) s.pool[out + __popc(m & lanemask_lt())] = e;
            out += __popc(m);
            __syncwarp();
        }
        psize = out;
    }
    // ---- results: the k smallest pool entries, ordered by (distance, label)
    const int kk = min((int)k, psize);
    uint64_t* olab = p.out_labels + (size_t)qi * k;
    float* odist = p.out_dists + (size_t)qi * k;
    for (int r = lane; r < kk; r += 32) {
        uint64_t e = s.pool[r];
        if (!DBG_OK(kid(e) < p.count, 80 + (PREC << 2), kid(e), r)) e = 0;
        uint32_t dk = khi(e);
        uint64_t lab = p.labels[kid(e)];
        int st = r;
        while (st > 0 && khi(s.pool[st - 1]) == dk) st--;
        int below = 0;
        for (int t = st; t < kk && khi(s.pool[t]) == dk; t++) {
            const uint32_t tid = kid(s.pool[t]);
            uint64_t lt = DBG_OK(tid < p.count, 90, tid, t) ? p.labels[tid] : 0;
            if (t != r && (lt < lab || (lt == lab && t < r))) below++;
        }
        if (DBG_OK(st + below < kk, 100, st + below, kk)) {
            olab[st + below] = lab;
            odist[st + below] = funkey(dk);
        }
    }
    for (int r = kk + lane; r < (int)k; r += 32) {
        olab[r] = ~0ull;
        odist[r] = __int_as_float(0x7f800000);
    }
    if (TIES && (status & kTieBit) && lane == 0) p.tie_list[atomicAdd(p.tie_count, 1u)] = qi;
    status &= ~kTieBit;
    if (lane == 0) {
        p.out_counts[qi] = kk;
        if (status) atomicOr(p.status, status);
    }
    PT_MARK(9);
    return true;
}

template <int SPACE, bool FAST16, bool EXACT, int PREC, int TERM, bool TIES, bool FILTER>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, PREC ? HNSWGPU_MINB_LOWP : kMinBlocks)
    hnsw_search_kernel(SearchParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* base = smem + (size_t)warp * p.warp_smem;
    WarpSmem s;
    s.bar = reinterpret_cast<uint64_t*>(base);
    s.cbuf = reinterpret_cast<uint32_t*>(base + 16);
    s.q = reinterpret_cast<float*>(base + p.off_query);
    s.stage = reinterpret_cast<float*>(base + p.off_stage);
    s.pool = reinterpret_cast<uint64_t*>(base + p.off_pool);
    s.extra = reinterpret_cast<uint64_t*>(base + p.off_extra);
    s.vis = reinterpret_cast<uint32_t*>(base + p.off_vis);
    s.topheap = reinterpret_cast<uint64_t*>(base + p.off_top);
    {
        const uint32_t gw = blockIdx.x * kWarpsPerBlock + warp;
        const bool spill = p.cand_spill != nullptr && gw < p.cand_spill_warps;
        s.candheap = SplitHeap{reinterpret_cast<uint64_t*>(base + p.off_cand),
                               spill ? p.cand_spill + (size_t)gw * p.cand_spill_cap : nullptr, (int)p.cand_cap};
        s.cand_total = (int)p.cand_cap + (spill ? (int)p.cand_spill_cap : 0);
    }
    s.accbuf = reinterpret_cast<uint64_t*>(base + p.off_acc);
    s.evbuf = reinterpret_cast<uint64_t*>(base + p.off_ev);
    if (lane == 0) mbar_init(s.bar, 1);
    fence_mbar_init();
    __syncwarp();
    uint32_t phase = 0;
    PhaseClock pc;
    // a list pass runs the queries a previous launch on this stream listed
    const uint32_t nrun = p.qcount ? min(*p.qcount, p.nq) : p.nq;
    while (true) {
        uint32_t qi = 0;
        if (lane == 0) {
            qi = atomicAdd(p.work_counter, 1u);
            if (p.qlist && qi < nrun) qi = p.qlist[qi];
            else if (qi >= nrun) qi = 0xffffffffu;
        }
        qi = __shfl_sync(FULL, qi, 0);
        if (qi >= p.nq) break;
        Counters ct = {0, 0, 0, 0};
        if (!search_one<SPACE, FAST16, EXACT, PREC, TERM, TIES, FILTER>(p, s, phase, qi, lane, ct, pc)) {
            if (lane == 0) atomicOr(p.status, HNSWGPU_STATUS_TIMEOUT_BIT);
            // wait (bounded) for this warp's copies still in flight, then leave
            mbar_wait(s.bar, phase);
            break;
        }
        if (p.trace && lane == 0) {
            uint32_t* t = p.trace + (size_t)qi * 4;
            t[0] = ct.upper_hops;
            t[1] = ct.upper_dists;
            t[2] = ct.l0_exp;
            t[3] = ct.l0_dists;
        }
    }
#ifdef HNSWGPU_PHASE_TIMING
    if (lane == 0 && p.phase_cycles)
        for (int i = 0; i < 10; i++) atomicAdd(p.phase_cycles + i, (unsigned long long)pc.acc[i]);
#endif
    // The last block to finish re-arms this launch's work counter, so the
    // next launch that draws the same counter slot starts from zero.
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(p.done_counter, 1u) == gridDim.x - 1) {
            *p.work_counter = 0;
            *p.done_counter = 0;
            __threadfence();
        }
    }
}

}  // namespace

size_t warp_smem_layout(SearchParams& p) {
    if (p.lean) return lean_smem_layout(p);
    size_t off = 16 + 128;  // mbarrier (8 bytes) + pad, then the 32-entry id compaction buffer
    p.off_query = (uint32_t)off;
    off += (size_t)p.row_floats * 4;
    off = (off + 15) & ~(size_t)15;
    // staging area followed by the visited cache: after the beam the two
    // together stage the float32 rows of the re-rank
    p.off_stage = (uint32_t)off;
    size_t stage = (size_t)p.stage_slots * p.stage_stride * 4;
    if (p.prec) stage = std::max(stage, (size_t)p.tslots * p.tstage_bytes);
    off += (stage + 15) & ~(size_t)15;
    p.off_vis = (uint32_t)off;
    off += ((size_t)1 << p.log2_vis) * 4;
    p.rr_slots = p.prec ? (uint32_t)std::min<size_t>(32, (off - p.off_stage) / ((size_t)p.stage_stride * 4)) : 0;
    off = (off + 7) & ~(size_t)7;
    p.off_pool = (uint32_t)off;
    off += (size_t)p.pool_cap * 8;
    p.off_top = (uint32_t)off;
    off += p.exact ? ((size_t)p.ef + 1) * 8 : 0;
    p.off_cand = (uint32_t)off;
    off += p.exact ? (size_t)p.cand_cap * 8 : 0;
    p.off_acc = (uint32_t)off;
    off += p.exact ? 32 * 8 : 0;
    p.off_ev = (uint32_t)off;
    off += p.exact ? 32 * 8 : 0;
    p.off_extra = (uint32_t)off;
    off += (size_t)p.extra_cap * 8;
    off = (off + 127) & ~(size_t)127;
    p.warp_smem = (uint32_t)off;
    return off;
}

namespace {
template <int SPACE, bool FAST16, bool EXACT, int PREC, int TERM = 0, bool TIES = false, bool FILTER = false>
cudaError_t launch_t(const SearchParams& p, int num_sms, cudaStream_t stream, int* blocks_out) {
    // per-instantiation, per-device cache of the opt-in shared-memory size and occupancy
    static LaunchCache cache;
    const void* fn = (const void*)hnsw_search_kernel<SPACE, FAST16, EXACT, PREC, TERM, TIES, FILTER>;
    const size_t smem = (size_t)p.warp_smem * kWarpsPerBlock;
    int occ_per_sm = 0;
    cudaError_t e = cache.blocks_per_sm(fn, kWarpsPerBlock * 32, smem, &occ_per_sm);
    if (e != cudaSuccess) return e;
    if (occ_per_sm < 1) return cudaErrorInvalidConfiguration;
    uint64_t need = (p.nq + kWarpsPerBlock - 1) / kWarpsPerBlock;
    uint64_t blocks = (uint64_t)occ_per_sm * (uint64_t)num_sms;
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    if (blocks_out) *blocks_out = (int)blocks;
    hnsw_search_kernel<SPACE, FAST16, EXACT, PREC, TERM, TIES, FILTER>
        <<<(unsigned)blocks, kWarpsPerBlock * 32, smem, stream>>>(p);
    return cudaGetLastError();
}

template <int SPACE, bool EXACT>
cudaError_t launch_s(const SearchParams& p, int num_sms, cudaStream_t stream, int* blocks_out) {
    return p.fast16 ? launch_t<SPACE, true, EXACT, 0>(p, num_sms, stream, blocks_out)
                    : launch_t<SPACE, false, EXACT, 0>(p, num_sms, stream, blocks_out);
}

template <int SPACE>
cudaError_t launch_lowp(const SearchParams& p, int num_sms, cudaStream_t stream, int* blocks_out) {
    // low-precision traversal: dim % 16 == 0, id tie order (checked by the host)
    return p.prec == 1 ? launch_t<SPACE, true, false, 1>(p, num_sms, stream, blocks_out)
                       : launch_t<SPACE, true, false, 2>(p, num_sms, stream, blocks_out);
}
// learned termination (id tie order; checked by the host)
template <int SPACE, int TERM>
cudaError_t launch_term_p(const SearchParams& p, int num_sms, cudaStream_t stream, int* blocks_out) {
    if (p.prec == 0)
        return p.fast16 ? launch_t<SPACE, true, false, 0, TERM>(p, num_sms, stream, blocks_out)
                        : launch_t<SPACE, false, false, 0, TERM>(p, num_sms, stream, blocks_out);
    return p.prec == 1 ? launch_t<SPACE, true, false, 1, TERM>(p, num_sms, stream, blocks_out)
                       : launch_t<SPACE, true, false, 2, TERM>(p, num_sms, stream, blocks_out);
}

template <int SPACE>
cudaError_t launch_term(const SearchParams& p, int num_sms, cudaStream_t stream, int* blocks_out) {
    return p.term_mode == 1 ? launch_term_p<SPACE, 1>(p, num_sms, stream, blocks_out)
                            : launch_term_p<SPACE, 2>(p, num_sms, stream, blocks_out);
}
}  // namespace

#ifdef HNSWGPU_BOUNDS_CHECK
cudaError_t read_debug_record(unsigned long long* out) {
    cudaError_t e = cudaMemcpyFromSymbol(out, g_dbg, sizeof(unsigned long long) * 8);
    if (e != cudaSuccess) return e;
    unsigned long long z[8] = {0};
    return cudaMemcpyToSymbol(g_dbg, z, sizeof(z));
}
#endif

// ---------------------------------------------------------------------------
// Fixed scratch for hnswgpu_search_noalloc: the search kernel's work counter,
// finished-CTA counter and status word, in a file-scope device array instead
// of memory allocated per index.  Every GPU that loads the library holds these
// 256 bytes until the process exits; all calls on a device share them.
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoallocScratchWords];

cudaError_t noalloc_scratch_address(int device, uint32_t** out) {
    // Resolved once per device, with that device current: in host code the
    // symbol's name is only a host-side stand-in, not a device address.  Two
    // threads making their first call at once both resolve it and store the
    // same value; the slots are atomics, so that is well defined.  The cached
    // address belongs to the device's current context: after a
    // cudaDeviceReset on that device the library must be unloaded and loaded
    // again before this entry point is used.
    static std::atomic<uint32_t*> addr[kMaxDevices];
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    uint32_t* a = addr[device].load(std::memory_order_acquire);
    if (!a) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        a = static_cast<uint32_t*>(ptr);
        addr[device].store(a, std::memory_order_release);
    }
    *out = a;
    return cudaSuccess;
}

// Self-test of the bounded wait and of the status path that reports it: the
// thread arms an mbarrier phase for 16 bytes that no copy will ever deliver
// (no copy is issued, so nothing is in flight when it gives up), waits at most
// `limit` tries, and records HNSWGPU_STATUS_TIMEOUT_BIT as a search would.
__global__ void wait_timeout_selftest_kernel(uint32_t limit, uint32_t* status) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    fence_mbar_init();
    __syncwarp();
    if (threadIdx.x == 0) mbar_arrive_expect_tx(&bar, 16);
    __syncwarp();
    const bool ok = mbar_wait_limit(&bar, 0, limit);
    if (threadIdx.x == 0 && !ok) atomicOr(status, HNSWGPU_STATUS_TIMEOUT_BIT);
}

cudaError_t launch_wait_timeout_selftest(uint32_t limit, uint32_t* status, cudaStream_t stream) {
    wait_timeout_selftest_kernel<<<1, 32, 0, stream>>>(limit, status);
    return cudaGetLastError();
}

// Pipelined beam over an index with deletions and / or a filter (id order,
// dim % 16 == 0, maxM0 <= 32; learned stop or none).
template <int SPACE, int TERM>
cudaError_t launch_filter_t(const SearchParams& p, int num_sms, cudaStream_t stream, int* blocks_out) {
    if (p.prec == 0) return launch_t<SPACE, true, false, 0, TERM, false, true>(p, num_sms, stream, blocks_out);
    return p.prec == 1 ? launch_t<SPACE, true, false, 1, TERM, false, true>(p, num_sms, stream, blocks_out)
                       : launch_t<SPACE, true, false, 2, TERM, false, true>(p, num_sms, stream, blocks_out);
}
template <int SPACE>
cudaError_t launch_filter(const SearchParams& p, int num_sms, cudaStream_t stream, int* blocks_out) {
    return p.term_mode == 2 ? launch_filter_t<SPACE, 2>(p, num_sms, stream, blocks_out)
                            : launch_filter_t<SPACE, 0>(p, num_sms, stream, blocks_out);
}

cudaError_t launch_hnsw_search(const SearchParams& p, int space, int num_sms, cudaStream_t stream, int* blocks_out) {
    if (p.lean) return lean_eligible(p) ? launch_hnsw_lean(p, space, num_sms, stream, blocks_out) : cudaErrorInvalidValue;
    if (!p.bare && !p.exact && p.fast16 && p.maxM0 <= 32 && p.term_mode != 1 && !p.tie_list)
        return space == 0 ? launch_filter<0>(p, num_sms, stream, blocks_out)
                          : launch_filter<1>(p, num_sms, stream, blocks_out);
    if (p.tie_list) {
        // id-order beam that lists its tie-steered queries (float32, 4-lane
        // distances, no filter or deletes: checked by the host)
        if (p.exact || p.prec || p.term_mode || !p.fast16 || !p.bare || p.maxM0 > 32 || p.pool_cap != p.ef + 1 ||
            !p.tie_count)
            return cudaErrorInvalidValue;
        return space == 0 ? launch_t<0, true, false, 0, 0, true>(p, num_sms, stream, blocks_out)
                          : launch_t<1, true, false, 0, 0, true>(p, num_sms, stream, blocks_out);
    }
    if (p.term_mode) return space == 0 ? launch_term<0>(p, num_sms, stream, blocks_out)
                                       : launch_term<1>(p, num_sms, stream, blocks_out);
    if (p.prec) return space == 0 ? launch_lowp<0>(p, num_sms, stream, blocks_out)
                                  : launch_lowp<1>(p, num_sms, stream, blocks_out);
    if (space == 0)
        return p.exact ? launch_s<0, true>(p, num_sms, stream, blocks_out)
                       : launch_s<0, false>(p, num_sms, stream, blocks_out);
    return p.exact ? launch_s<1, true>(p, num_sms, stream, blocks_out)
                   : launch_s<1, false>(p, num_sms, stream, blocks_out);
}

}  // namespace hnswgpu
